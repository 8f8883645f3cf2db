"""The quarter-turn backprojection (bp_sym.cuh): views v, v + N/4, v + N/2, v + 3N/4 of a
circular scan about a square, centred grid see columns related by a quarter turn at one detector
position, so the reconstructor backprojects such quadruples four at a time when they share a
batch.  Checked against the same reconstructor without the pairing (FDK_BP_SYM=0) and against the
oracle (FP64 pipeline; the reference kernel's arithmetic for FP32), with quadruples and unpaired
views in one batch, both orbit directions, grids whose quadrant is not a whole number of tiles,
detector-edge slices, and a geometry without the symmetry (the pairing must switch itself off)."""
import os

import numpy as np
import pytest

import fdk_b200 as F
from fdk_b200.phantom import phantom_for, project
from tests.helpers import knife_edge_mask, oracle_bp_f64, oracle_filtered, phantom_views, rel_l2, small_param

pytestmark = pytest.mark.gpu


def quarter_order(n_proj, chunk):
    """(first, count) pushes: `chunk` consecutive views from each quarter in turn."""
    q = n_proj // 4
    return [(b + k * q, min(chunk, q - b)) for b in range(0, q, chunk) for k in range(4)]


def run(p, precision, proj, order, batch, pair=True, slab=None):
    os.environ["FDK_BP_SYM"] = "1" if pair else "0"  # MIXED pairs only on request
    try:
        r = F.Reconstructor(p, precision, batch=batch, slab=slab)
    finally:
        os.environ.pop("FDK_BP_SYM", None)
    kind = r.bp_kernel
    for first, n in order:
        r.push(np.ascontiguousarray(proj[first:first + n]), first)
    vol = r.volume().copy()
    r.close()
    return vol, kind


@pytest.mark.parametrize("precision", ["fp32", "mixed"])
@pytest.mark.parametrize("n,views,direction", [(64, 16, -1), (40, 24, -1), (48, 20, 1)])
def test_quarter_turn_pairing_matches_unpaired_and_oracle(precision, n, views, direction):
    p = small_param(n, n, n, views)
    p.direction = direction
    _, proj = phantom_views(p, seed=n)
    order = quarter_order(views, 2)
    got, kind = run(p, precision, proj, order, batch=views)
    ref, kind0 = run(p, precision, proj, order, batch=views, pair=False)
    assert kind == "quarter-turn" and kind0 == "staged"
    m = knife_edge_mask(p, [0, 0, 0, n, n, n // 2], n // 2)
    e_pair = rel_l2(got[m], ref[m])
    filt = oracle_filtered(p, proj)
    f64, _ = oracle_bp_f64([0, 0, 0, n, n, n // 2], n // 2, n, filt, p.proj_matrices(np.float64))
    e64 = rel_l2(got[m], f64[m])
    print(precision, n, views, direction, "paired vs unpaired", e_pair, "vs fp64", e64)
    if precision == "fp32":
        assert e_pair <= 3e-6 and e64 <= 1e-5  # two FP32 summation orders
    else:
        assert e_pair <= 5e-4 and e64 <= 1e-3


@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_quadruples_and_unpaired_views_in_one_batch(precision):
    """16 views of a 32-view scan in one batch: 3 whole orbits (12 views) and 4 views whose
    partners never come -- the pairs go to the quarter-turn kernel, the rest to the staged one."""
    n = 48
    p = small_param(n, n, n, 32)
    _, proj = phantom_views(p, seed=4)
    order = [(0, 3), (8, 3), (16, 3), (24, 3), (5, 2), (13, 1), (30, 1)]
    got, kind = run(p, precision, proj, order, batch=16)
    ref, _ = run(p, precision, proj, order, batch=16, pair=False)
    assert kind == "quarter-turn"
    m = knife_edge_mask(p, [0, 0, 0, n, n, n // 2], n // 2)
    assert rel_l2(got[m], ref[m]) <= (3e-6 if precision == "fp32" else 5e-4)


def test_default_pairing_is_fp32_only():
    """Without FDK_BP_SYM the FP32 reconstructor pairs views and the MIXED one runs the staged
    kernel (measured faster for FP16 views)."""
    os.environ.pop("FDK_BP_SYM", None)
    p = small_param(32, 32, 32, 16)
    kinds = {}
    for prec in ("fp32", "mixed", "fp32_exact"):
        r = F.Reconstructor(p, prec, batch=16)
        kinds[prec] = r.bp_kernel
        r.close()
    assert kinds == {"fp32": "quarter-turn", "mixed": "staged", "fp32_exact": "exact"}


def test_pairing_switches_off_without_the_symmetry():
    """A grid that is not square, a view count that is not a multiple of 4, and a sub-slab reach
    the staged kernel alone; results still match the oracle."""
    p = small_param(32, 40, 32, 18)
    r = F.Reconstructor(p, "fp32", batch=18)
    assert r.bp_kernel == "staged"
    r.close()
    q = small_param(32, 40, 32, 16)
    q.ny = 24
    r = F.Reconstructor(q, "fp32", batch=16)
    assert r.bp_kernel == "staged"
    r.close()


def test_full_size_c2_paired_matches_unpaired():
    """512^3 from 512 views of 512^2 in quarter order (every batch pairs all its views)."""
    import torch

    p = F.config("c2")
    dev = torch.empty((p.nProj, p.nv, p.nu), dtype=torch.float32, device="cuda")
    project(p, phantom_for(p, 2, 20), 0, p.nProj, dev.data_ptr())
    torch.cuda.synchronize()
    vols = {}
    for pair in (True, False):
        os.environ["FDK_BP_SYM"] = "1" if pair else "0"
        r = F.Reconstructor(p, "mixed", batch=256)
        os.environ.pop("FDK_BP_SYM", None)
        for first, n in quarter_order(p.nProj, 8):
            r.push_device(dev[first:].data_ptr(), first, n)
        vols[pair] = (r.volume().astype(np.float64), r.bp_kernel)
        r.close()
    assert vols[True][1] == "quarter-turn" and vols[False][1] == "staged"
    e = rel_l2(vols[True][0], vols[False][0])
    print("c2 mixed paired vs unpaired", e)
    assert e <= 3e-4
