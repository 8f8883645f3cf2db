"""The MIXED interpolation layout's arithmetic, emulated on the CPU in numpy.

to_lerp_kernel (fdk_b200/csrc/bp.cu) stores, per FP16 mirror value E(v) of a batch whose largest
magnitude is M, e = E(v) 2^-k and d = (E(v+1) - E(v)) 2^(14-k) in FP16, with 2^k just above M
(k = ilogb(M) + 1).  The staged kernels sample v = vi + fv as one FP16 fused multiply-add,
e + (fv 2^-14) d, where fv 2^-14 is the FP16 subnormal whose mantissa is the 10-bit fixed-point
fraction, and the launch's accumulator scale multiplies 2^k back.  An FP16 FMA rounds once, so
computing g * d + e in float64 (exact here: an 11-bit by 11-bit product) and rounding to float16
reproduces it.  These checks need no GPU: the scale keeps d inside FP16's range at any batch
maximum, the sample carries the roundings of E and d only, and on uncorrelated data it is more
accurate than the layout's first form (a = E - d with 1 + fv, whose a was rounded)."""
import math

import numpy as np

F16_MAX = 65504.0


def _k(m: float) -> int:
    return math.frexp(m)[1] if m > 0 else 0  # frexp's exponent is ilogb(m) + 1


def _layout(E: np.ndarray):
    """e and d of one row of FP16 values E (as to_lerp_kernel), and 2^k."""
    k = _k(float(np.abs(E.astype(np.float64)).max()))
    e0 = E.astype(np.float32)
    e1 = np.append(e0[1:], e0[-1])  # d = 0 at the last row
    e = (e0 * np.float32(2.0 ** -k)).astype(np.float16)
    d = ((e1 - e0) * np.float32(2.0 ** (14 - k))).astype(np.float16)
    return e, d, 2.0 ** k


def _sample(e, d, scale, vi, f):
    """e + (f / 1024 * 2^-14) d rounded once to FP16, times 2^k."""
    g = np.float16(f * 2.0 ** -24)  # the subnormal with mantissa f: exactly f 2^-24
    assert float(g) == f * 2.0 ** -24
    r = np.float16(float(e[vi]) + float(g) * float(d[vi]))
    return float(r) * scale


def _sample_first_form(E, vi, f):
    """The first form: a = E(v) - d, d = E(v+1) - E(v) in FP16, sample a + (1 + fv) d."""
    e0, e1 = np.float32(E[vi]), np.float32(E[vi + 1])
    d = np.float16(e1 - e0)
    a = np.float16(e0 - np.float32(d))
    return float(np.float16(float(a) + (1.0 + f / 1024.0) * float(d)))


def test_d_stays_inside_fp16_at_any_batch_maximum():
    rng = np.random.default_rng(0)
    for m in (6.0e-8, 1.0e-5, 3.0e-3, 1.0, 700.0, 30000.0, F16_MAX):
        E = (rng.uniform(-1, 1, 4096) * m).astype(np.float16)
        E[0], E[1] = np.float16(m), np.float16(-m)  # the largest possible difference, 2M
        e, d, _ = _layout(E)
        assert np.isfinite(e).all() and np.isfinite(d).all(), m
        assert np.abs(d.astype(np.float64)).max() < 2.0 ** 15, m
        assert np.abs(e.astype(np.float64)).max() <= 1.0, m


def test_sample_carries_the_roundings_of_e_and_d_only():
    rng = np.random.default_rng(1)
    E = (rng.standard_normal(2048) * 50).astype(np.float16)
    e, d, s = _layout(E)
    M = float(np.abs(E.astype(np.float64)).max())
    for vi in rng.integers(0, 2046, 400):
        f = int(rng.integers(0, 1024))
        fv = f / 1024.0
        exact = float(E[vi]) + fv * (float(E[vi + 1]) - float(E[vi]))
        got = _sample(e, d, s, vi, f)
        # one FP16 rounding of d (relative 2^-11, times fv) and of the sum (half an ulp of a value
        # below 2M), absolute at most 2^-25 M below FP16's normal range
        dd = abs(float(E[vi + 1]) - float(E[vi]))
        bound = fv * dd * 2.0 ** -11 + max(abs(exact), 2.0 ** -13 * M) * 2.0 ** -11 + 2.0 ** -24 * M
        assert abs(got - exact) <= bound, (vi, f, got, exact, bound)


def test_more_accurate_than_the_first_form_on_uncorrelated_values():
    rng = np.random.default_rng(2)
    E = (rng.standard_normal(8192) * 10).astype(np.float16)
    e, d, s = _layout(E)
    err_new, err_old, ref = 0.0, 0.0, 0.0
    for vi in range(0, 8190, 3):
        f = int(rng.integers(0, 1024))
        exact = float(E[vi]) + f / 1024.0 * (float(E[vi + 1]) - float(E[vi]))
        err_new += (_sample(e, d, s, vi, f) - exact) ** 2
        err_old += (_sample_first_form(E, vi, f) - exact) ** 2
        ref += exact ** 2
    assert err_new < 0.5 * err_old, (math.sqrt(err_new / ref), math.sqrt(err_old / ref))
