"""Multi-GPU sharding host logic (DivVolume, cuFDK/mpiFDK.h:52-177) on CPU ranks over gloo:
slab pairs are disjoint, cover the volume, keep the mirror rule, and need no data-path
collective (only the final gather, exercised here with all_gather_object); each rank's slab
pair, reconstructed by the oracle, assembles into the whole-volume reconstruction."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from fdk_b200.shard import div_volume


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, size, port, nz, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=size)
    try:
        sp = div_volume(64, 64, nz, rank, size)
        gathered = [None] * size
        dist.all_gather_object(gathered, sp.z_indices())
        if rank == 0:
            q.put(gathered)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("size", [2, 4])
def test_slab_pairs_cover_volume(size):
    nz = 64
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, size, port, nz, q)) for r in range(size)]
    for p in procs:
        p.start()
    gathered = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    allz = sorted(z for zs in gathered for z in zs)
    assert allz == list(range(nz))
    for r, zs in enumerate(gathered):
        half = len(zs) // 2
        top, bot = zs[:half], zs[half:]
        assert [nz - 1 - z for z in reversed(top)] == bot  # mirror pairs


def _oracle_slab_worker(rank, size, port, q):
    """One CPU rank: the oracle's FP64 backprojection of its slab pair only (no collective on the
    data path), then the slabs are gathered to rank 0."""
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=size)
    try:
        from oracle import oracle as O
        from tests.helpers import oracle_filtered, phantom_views, small_param

        n = 32
        p = small_param(n, 40, 40, 8)
        _, proj = phantom_views(p, seed=9, n_ell=6)
        filt = oracle_filtered(p, proj)
        sp = div_volume(n, n, n, rank, size)
        d = int(sp.top.depth)
        top = [0, 0, int(sp.top.z), n, n, d]
        vol = np.zeros(n * n * 2 * d, np.float64)
        O.bp_f64(vol, top, d, n, filt, p.proj_matrices(np.float64))
        gathered = [None] * size
        dist.all_gather_object(gathered, (sp.z_indices(), O.transform_volume(vol.astype(np.float32), n, n, 2 * d)))
        if rank == 0:
            whole = np.zeros(n * n * n, np.float64)
            O.bp_f64(whole, [0, 0, 0, n, n, n // 2], n // 2, n, filt, p.proj_matrices(np.float64))
            want = O.transform_volume(whole.astype(np.float32), n, n, n)
            full = np.full((n, n, n), np.nan, np.float32)
            for zs, slab in gathered:
                full[zs] = slab
            q.put(bool(np.array_equal(full, want)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("size", [2, 4])
def test_oracle_slab_pairs_assemble_the_whole_volume(size):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_oracle_slab_worker, args=(r, size, port, q)) for r in range(size)]
    for p in procs:
        p.start()
    ok = q.get(timeout=180)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert ok


def test_div_volume_rules():
    sp = div_volume(2048, 2048, 2048, 0, 1)
    assert sp.symmetric and sp.top.depth == 1024 and sp.bottom.z == 1024
    with pytest.raises(ValueError):
        div_volume(64, 64, 64, 0, 3)
    big = div_volume(8192, 8192, 64, 1, 2)
    assert not big.symmetric and big.top.z == 32 and big.bottom.depth == 0
