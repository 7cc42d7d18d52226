"""The FP64 sweeps divide by the diagonal through its stored reciprocal y = RN(1/d) and Markstein's
correction (baas_b200/csrc/device_common.cuh, div_rcp), which must give the IEEE correctly rounded
quotient the reference's `(b - sum) / diag` gives (merge/SpTRSV.cpp, the per-row division of the
forward and backward sweeps). baas_test_divide runs it on device arrays; every quotient is compared
bit for bit with numpy's division (correctly rounded) and with the GPU's __ddiv_rn, on random
operands over the whole exponent range, on quotients made to lie next to a rounding midpoint, and
on the special values (zeros, subnormals, infinities, NaNs, the fall-back range boundaries)."""
import numpy as np
import pytest

from baas_b200 import _native

pytestmark = pytest.mark.gpu


def _divide(a, b, mode):
    import torch

    da = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()
    db = torch.from_numpy(np.ascontiguousarray(b, dtype=np.float64)).cuda()
    dq = torch.empty_like(da)
    _native.check(_native.lib().baas_test_divide(da.data_ptr(), db.data_ptr(), dq.data_ptr(), da.numel(), mode, None), "baas_test_divide")
    return dq.cpu().numpy()


def _same_bits(x, y):
    nan = np.isnan(x) & np.isnan(y)
    return nan | (x.view(np.int64) == y.view(np.int64))


def _check(a, b):
    with np.errstate(all="ignore"):
        want = a / b
    got = _divide(a, b, 0)
    ieee = _divide(a, b, 1)
    ok = _same_bits(got, want)
    bad = np.flatnonzero(~ok)
    assert bad.size == 0, [(a[i], b[i], got[i], want[i]) for i in bad[:5]]
    assert np.all(_same_bits(ieee, want))


def _mantissa(rng, n):
    return 1.0 + rng.random(n)


def test_random_operands_all_exponents():
    rng = np.random.default_rng(11)
    n = 1 << 22
    a = np.ldexp(_mantissa(rng, n), rng.integers(-1020, 1020, n)) * rng.choice([-1.0, 1.0], n)
    b = np.ldexp(_mantissa(rng, n), rng.integers(-1020, 1020, n)) * rng.choice([-1.0, 1.0], n)
    _check(a, b)


def test_sweep_like_operands():
    """Diagonals of an IC0 factor and residuals of moderate size: all on the fast path."""
    rng = np.random.default_rng(12)
    n = 1 << 22
    b = rng.uniform(0.05, 20.0, n)
    a = rng.standard_normal(n) * np.ldexp(1.0, rng.integers(-60, 60, n))
    _check(a, b)


def test_quotients_next_to_midpoints():
    """q in [1, 2) and m = q + 2^-53, the midpoint between q and the next double; a ~ b * m (and
    its two neighbours) puts a / b within about an ulp of the midpoint, the hardest case for the
    final rounding."""
    rng = np.random.default_rng(13)
    n = 1 << 21
    b = _mantissa(rng, n) * np.ldexp(1.0, rng.integers(-40, 40, n))
    q = _mantissa(rng, n)
    a = b * q + b * np.ldexp(1.0, -53)
    a2 = np.nextafter(a, np.inf)
    a3 = np.nextafter(a, -np.inf)
    _check(np.concatenate([a, a2, a3]), np.concatenate([b, b, b]))


def test_exact_quotients_and_powers_of_two():
    rng = np.random.default_rng(14)
    n = 1 << 20
    b = _mantissa(rng, n) * np.ldexp(1.0, rng.integers(-500, 500, n))
    k = rng.integers(1, 1 << 20, n).astype(np.float64)
    _check(b * k, b)
    _check(k, np.ldexp(1.0, rng.integers(-900, 900, n)))


def test_special_and_boundary_values():
    tiny = np.finfo(np.float64).tiny
    specials = np.array([
        0.0, -0.0, 1.0, -1.0, 3.0, np.inf, -np.inf, np.nan, tiny, tiny / 8, 5e-324, -5e-324,
        np.finfo(np.float64).max, -np.finfo(np.float64).max, 2.0 ** -960, 2.0 ** 960,
        np.nextafter(2.0 ** -960, 0), np.nextafter(2.0 ** -960, 1), np.nextafter(2.0 ** 960, 0),
        np.nextafter(2.0 ** 960, np.inf), 2.0 ** -1000, 2.0 ** 1000, 1e-300, 1e300, 0.1, 7.0,
    ])
    a, b = np.meshgrid(specials, specials)
    _check(a.ravel(), b.ravel())
    # quotients whose size crosses the fall-back boundary while both operands are inside it
    rng = np.random.default_rng(15)
    n = 1 << 18
    ea = rng.integers(-960, 960, n)
    eb = np.clip(ea + rng.integers(-970, 970, n), -960, 959)
    _check(np.ldexp(_mantissa(rng, n), ea), np.ldexp(_mantissa(rng, n), eb))
