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


def test_fast_path_declines_exactly_outside_its_range():
    """mode 2 reports the quotients div_fast declines: a = -0, |a| < 2^-460, |a| >= 2^461,
    non-finite a, and divisors outside [2^-500, 2^500); a = +0 and ordinary values stay fast."""
    a = np.array([1.0, -3.5, 0.0, -0.0, 2.0 ** -460, 2.0 ** -461, 2.0 ** 460, 2.0 ** 461, 5e-324, np.inf, np.nan,
                  1.0, 1.0, 1.0, 1.0])
    b = np.array([3.0, 7.0, 2.0, 2.0, 1.5, 1.5, 1.5, 1.5, 1.5, 1.5, 1.5, 2.0 ** 499, 2.0 ** 500, 2.0 ** -500,
                  2.0 ** -501])
    want = np.array([0, 0, 0, 1, 0, 1, 0, 1, 1, 1, 1, 0, 1, 0, 1], dtype=np.float64)
    assert np.array_equal(_divide(a, b, 2), want)
    _check(a, b)


def _bits(x):
    return np.ascontiguousarray(x, dtype=np.float64).view(np.int64)


def test_sweep_repeats_with_ieee_division():
    """A right-hand side of -0.0 on rows without dependencies: div_fast would return +0, so the
    sweep must notice and repeat with IEEE divisions; the result matches the oracle bit for bit,
    signs of zeros included."""
    import torch

    from baas_b200 import KERNEL_SPTRSV, DeviceCSR, Schedule, gen
    from oracle.oracle import Port

    L, _, b = gen.sptrsv_case(48, 0)
    b = b.copy()
    b[:5] = -0.0
    s = Schedule(L, kind=KERNEL_SPTRSV, nthread=8)
    x = torch.zeros(L.n, dtype=torch.float64, device="cuda")
    s.forward(DeviceCSR.from_host(L), torch.from_numpy(b).cuda(), x)
    want = Port.lower_solve(L, b)
    assert np.signbit(want[0])
    assert np.array_equal(_bits(x.cpu().numpy()), _bits(want))


def test_iccg_and_batched_repeat_with_ieee_division():
    """ICCG with b[0] = -0.0 starts its first lower sweep with -0 / L00 and must repeat the launch
    with IEEE divisions; the iterate equals the one for b[0] = +0.0 (both are IEEE-exact runs of
    the same iteration) and so does the iteration count. Same for a batched solve."""
    import torch

    from baas_b200 import KERNEL_ICCG, BatchSchedule, DeviceCSR, Schedule, gen

    A = gen.laplace3d(12, 1e-3)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8)
    dA = DeviceCSR.from_host(A)
    out = []
    for z in (0.0, -0.0):
        b = gen.uniform_rhs(A.n, 1)
        b[0] = z
        x = torch.zeros(A.n, dtype=torch.float64, device="cuda")
        it, rel = s.iccg(dA, torch.from_numpy(b).cuda(), x, tol=1e-10)
        out.append((it, x.cpu().numpy()))
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1])

    systems = [gen.laplace2d(9), gen.vardiff2d(11, seed=2)]
    bs = BatchSchedule(systems, parts=3)
    C = bs.combined
    dC = DeviceCSR.from_host(C)
    res = []
    for z in (0.0, -0.0):
        B = gen.uniform_rhs(C.n, 7, nrhs=2).reshape(2, C.n)
        B[0, bs.sys_off[1]] = z
        X = torch.zeros((2, C.n), dtype=torch.float64, device="cuda")
        it, rel = bs.iccg_batched(dC, torch.from_numpy(B).cuda(), X, tol=1e-10)
        res.append((it.copy(), X.cpu().numpy()))
    assert np.array_equal(res[0][0], res[1][0])
    assert np.array_equal(res[0][1], res[1][1])
