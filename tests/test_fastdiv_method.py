"""The constant-divisor division the pfwi step kernel uses in place of
__fdiv_rn (pywave_b200/csrc/pfwi.cu: DivC, div_bmr, div_small), restated in
numpy and checked against IEEE float32 division on sampled numerators.

The CUDA library checks every divisor exhaustively on the GPU at set-up and
falls back to __fdiv_rn if any quotient differs; this CPU test pins the
method itself (Brisebarre, Muller and Raina, IEEE Trans. Computers 53(8),
2004, plus the scaled path with the remainder tie fix for tiny numerators)
for the spacings the tests and benchmarks use."""
import numpy as np
import pytest

f32 = np.float32
LD = np.longdouble
K = 89  # DIV_SMALL_K


def _consts(d):
    """zh, zl, xmin, xmax as prepare_div computes them."""
    z0 = f32(1.0 / float(d))
    zh, err = z0, abs(1.0 - float(z0) * float(d))
    for c in (np.nextafter(z0, f32(0)), np.nextafter(z0, f32(np.inf))):
        e = abs(1.0 - float(c) * float(d))
        if e < err or (e == err and (int(c.view(np.uint32)) & 1) == 0):
            zh, err = c, e
    zl = f32((1.0 - float(zh) * float(d)) / float(d))
    fmin, fmax = float(np.finfo(f32).tiny), float(np.finfo(f32).max)
    lo = max(fmin / float(zh), fmin * float(d))
    if zl != 0:
        lo = max(lo, fmin / abs(float(zl)))
    lo *= 4
    hi = min(fmax / 4 / float(zh), fmax / 4 * float(d), fmax)
    return zh, zl, f32(lo), f32(hi)


def _fma(a, b, c):
    """RN(a*b + c) for float32 arrays: a*b is exact in double, the sum exact in
    the 64-bit-significand long double, then one rounding to float32."""
    return (a.astype(np.float64) * b.astype(np.float64)).astype(LD).__add__(c.astype(LD)).astype(f32)


def _bmr(x, zh, zl):
    t = (x.astype(np.float64) * np.float64(zl)).astype(f32)  # RN(x*zl)
    q = _fma(x, np.full_like(x, zh), t)
    return np.copysign(q, x)


def _small(x, d, zh, zl):
    xs = (x * f32(2.0 ** K)).astype(f32)
    qs = _bmr(xs, zh, zl)
    q = np.copysign((qs * f32(2.0 ** -K)).astype(f32), x)
    t = np.abs((qs * f32(2.0 ** (149 - K))).astype(f32))
    n = np.trunc(t)
    tie = (t - n) == f32(0.5)
    r = _fma(-qs, np.full_like(qs, d), xs)  # exact remainder
    nn = np.where(tie, n, 0).astype(np.uint32)
    k = nn + (((r > 0) == (x > 0)) & (r != 0)).astype(np.uint32)
    tie_res = (k | (x.view(np.uint32) & np.uint32(0x80000000))).view(f32)
    return np.where(tie & (r != 0), tie_res, q)


@pytest.mark.skipif(np.finfo(np.longdouble).nmant < 63,
                    reason="the exact FMA emulation needs an 80-bit long double")
@pytest.mark.parametrize("h", [0.01, 10.0, 0.012, 0.008, 0.03, 0.005, 0.025])
def test_constant_divisor_division_is_correctly_rounded(h):
    d = f32(f32(h) * f32(h))
    zh, zl, xmin, xmax = _consts(d)
    assert xmin <= f32(2.0 ** (K - 149)) and float(xmin) * 2.0 ** K <= float(xmax)
    rng = np.random.default_rng(int(h * 1e4))
    # numerators in [xmin, xmax]: random bit patterns plus a full binade sample
    umin, umax = int(xmin.view(np.uint32)), int(xmax.view(np.uint32))
    u = rng.integers(umin, umax + 1, 1 << 20, dtype=np.int64).astype(np.uint32)
    x = np.concatenate([u.view(f32), (f32(1.0) + np.arange(1 << 18, dtype=f32) * f32(2.0 ** -18))])
    x = np.concatenate([x, -x])
    assert np.array_equal(_bmr(x, zh, zl).view(np.uint32), (x / d).view(np.uint32))
    # below xmin: every one of the smallest 2^16 subnormals, then random patterns
    u = np.concatenate([np.arange(1, 1 << 16, dtype=np.uint32),
                        rng.integers(1, umin, 1 << 20, dtype=np.int64).astype(np.uint32)])
    x = u.view(f32)
    x = np.concatenate([x, -x])
    assert np.array_equal(_small(x, d, zh, zl).view(np.uint32), (x / d).view(np.uint32))
    # zeros keep their sign
    z = np.array([0.0, -0.0], f32)
    assert np.array_equal(_bmr(z, zh, zl).view(np.uint32), (z / d).view(np.uint32))
