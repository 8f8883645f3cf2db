"""Volume sharding across GPUs: DivVolume (cuFDK/mpiFDK.h:52-177) restated.

Each rank of `size` reconstructs one mirror-symmetric slab pair of the volume: top slab
z in [rank*d, rank*d + d) and bottom slab z in [nz - rank*d - d, nz - rank*d), d = nz/(2*size).
Every rank filters all views itself, so the reconstruction needs no collective; only the
final gather of slabs (optional) moves data.  Volumes of 8192^2 or more in x/y use plain
slabs instead (no mirror pairing), as the reference does (mpiFDK.h:61-63, 150-175).
"""
from __future__ import annotations

from dataclasses import dataclass

from .backprojection import BoxT


@dataclass
class SlabPair:
    top: object      # Box
    bottom: object   # Box (depth 0 when not mirror-paired)
    symmetric: bool

    @property
    def depth(self) -> int:
        return int(self.top.depth + self.bottom.depth)

    def z_indices(self):
        """Volume z index of each storage slice, in storage order (top, then bottom ascending)."""
        zs = list(range(int(self.top.z), int(self.top.z + self.top.depth)))
        zs += list(range(int(self.bottom.z), int(self.bottom.z + self.bottom.depth)))
        return zs


def div_volume(nx: int, ny: int, nz: int, rank: int, size: int) -> SlabPair:
    if size <= 0 or (size & (size - 1)) != 0:
        raise ValueError("size must be a power of two (mpiFDK.h:55)")
    if not 0 <= rank < size:
        raise ValueError("rank out of range")
    symmetric = not (nx >= 8192 and ny >= 8192)
    if symmetric:
        sub_nz = nz // size
        if sub_nz % 2 or sub_nz * size != nz:
            raise ValueError("nz must split into even slabs")
        d = sub_nz // 2
        top = BoxT(0, 0, rank * d, nx, ny, d)
        bottom = BoxT(0, 0, nz - 1 - rank * d - d + 1, nx, ny, d)
        assert top.z + bottom.z + bottom.depth - 1 == nz - 1
        return SlabPair(top, bottom, True)
    if nz % size:
        raise ValueError("nz must be divisible by size")
    d = nz // size
    return SlabPair(BoxT(0, 0, d * rank, nx, ny, d), BoxT(0, 0, d * rank, nx, ny, 0), False)
