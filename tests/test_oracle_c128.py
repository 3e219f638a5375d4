"""The oracle's complex J (LHLWorkspace{ComplexF64}) against the reference's own relations,
on CPU: the reduction reconstructs J with |l| <= 1 (test/core_tests.jl:5-21 with a complex
J), solves match a dense solve (:241-249), the complex reduction of a real J matches the
complex-shift-on-real path (:251-280: x == xf, refinement backward error), and a complex
reduction of a real J takes the real reduction's pivots.  The reference's matrices come from
Julia's MersenneTwister, which is not reproduced here: these are the same families from
numpy's seeded generator."""
import math

import numpy as np
import pytest

from oracle import oracle as O

SHIFTS = ((0.4 + 0.7j, -1.0), (1.0, -0.05 + 0.3j), (0.0, 1j), (-3.0 + 2j, 2.0 - 1j), (1.0, -0.05))


def crandn(g, *shape):
    return g.standard_normal(shape) + 1j * g.standard_normal(shape)


def bwd(W, x, b):
    """test/core_tests.jl:3: ||b - W x||_inf / (||W||_inf ||x||_inf + ||b||_inf)."""
    r = b - W @ x
    return np.abs(r).max() / (np.abs(W).sum(axis=1).max() * np.abs(x).max() + np.abs(b).max())


def test_modulus_is_hypot():
    """abs(z) of the complex path is hypot(re, im): the restated algorithm agrees with the C
    library's hypot bit for bit on a wide sample, and handles zeros, huge and tiny parts."""
    g = np.random.default_rng(1)
    z = g.standard_normal((5000, 2)) * np.exp(g.uniform(-300, 300, (5000, 1)))
    for a, b in z:
        assert O.cabs(complex(a, b)) == math.hypot(a, b)
    assert O.cabs(0j) == 0.0
    assert O.cabs(3 + 4j) == 5.0
    assert O.cabs(complex(-2.0, 0.0)) == 2.0
    assert O.cabs(complex(1e308, 1e308)) == math.hypot(1e308, 1e308)
    assert O.cabs(complex(5e-324, 5e-324)) == math.hypot(5e-324, 5e-324)
    assert math.isinf(O.cabs(complex(math.inf, math.nan)))


@pytest.mark.parametrize("n", [1, 2, 3, 4, 17, 80, 128, 200])
@pytest.mark.parametrize("balance", [True, False])
def test_complex_reduction_reconstructs_J(n, balance):
    g = np.random.default_rng(n)
    J = crandn(g, n, n)
    R = O.reduce_c128(J, balance)
    Z, Zi = R.Z(), R.Zinv()
    H = np.triu(R.factors, -1)
    assert np.allclose(Z @ Zi, np.eye(n), rtol=0, atol=1e-10)
    assert np.linalg.norm(Z @ H @ Zi - J) <= 1e-10 * np.linalg.norm(J)
    assert np.all(np.abs(np.tril(R.factors, -2)) <= 1.0)
    # balancing factors are powers of two and scale * iscale == 1 exactly
    assert np.all(np.frexp(R.scale)[0] == 0.5)
    assert np.all(R.scale * R.iscale == 1.0)
    # Ht holds H transposed, zero below its subdiagonal band
    assert np.array_equal(R.Ht, H.T)


def test_complex_solve_matches_dense():
    """test/core_tests.jl:241-249: n = 30, gamma = 0.2 + 0.3i, lhl_shift!(ws, 1, -gamma)."""
    g = np.random.default_rng(13)
    n = 30
    J = crandn(g, n, n)
    b = crandn(g, n)
    gam = 0.2 + 0.3j
    R = O.reduce_c128(J)
    S = O.shift_c128(R, 1, -gam)
    x = O.ldiv_c128(R, S, b)
    xr = np.linalg.solve(np.eye(n) - gam * J, b)
    assert np.linalg.norm(x - xr) <= 1e-9 * np.linalg.norm(xr)


@pytest.mark.parametrize("n", [1, 2, 3, 5, 40, 129])
def test_complex_reduction_of_real_J_matches_complex_shifts(n):
    """test/core_tests.jl:251-280: a real J with complex shifts (ws) against the complex
    reduction of complex.(J) (wf): the two solves agree to 1e-9, both match the dense solve,
    and one refinement step with the complex W brings the backward error under 50 eps."""
    g = np.random.default_rng(n)
    J = g.standard_normal((n, n))
    b = crandn(np.random.default_rng(n + 7), n)
    Rr = O.reduce(J)
    Rc = O.reduce_c128(J.astype(np.complex128))
    assert np.array_equal(Rr.ipiv, Rc.ipiv)
    eps = np.finfo(float).eps
    for s, t in SHIFTS:
        W = s * np.eye(n) + t * J
        x = O.ldiv_complex(Rr, O.shift_complex(Rr, s, t), b)
        Sf = O.shift_c128(Rc, s, t)
        xf = O.ldiv_c128(Rc, Sf, b)
        xd = np.linalg.solve(W, b)
        assert np.linalg.norm(x - xd) <= 1e-9 * np.linalg.norm(xd)
        assert np.linalg.norm(x - xf) <= 1e-9 * np.linalg.norm(x)
        y = O.refine_c128(Rc, Sf, J, b, xf, 1)
        assert bwd(W, y, b) <= 2 * bwd(W, xf, b) + eps
        assert bwd(W, y, b) < 50 * eps


def xref_extended(J, s, t, b, iters=6):
    """The solution of (s I + t J) x = b to far below FP64 rounding: FP64 solves corrected by
    residuals computed in 80-bit extended precision (the reference's test uses BigFloat at 128
    bits, test/core_tests.jl:264-268; extended precision resolves errors down to ~1e-18 here)."""
    n = J.shape[0]
    L = np.clongdouble
    W64 = s * np.eye(n) + t * J
    WL = L(s) * np.eye(n, dtype=L) + L(t) * J.astype(L)
    bL = b.astype(L)
    x = np.linalg.solve(W64, b).astype(L)
    for _ in range(iters):
        r = bL - WL @ x
        x = x + np.linalg.solve(W64, r.astype(np.complex128)).astype(L)
    return x


def ferr(v, xref):
    return float(np.linalg.norm(v.astype(np.clongdouble) - xref) / np.linalg.norm(xref))


@pytest.mark.parametrize("n", [1, 2, 3, 5, 40, 129])
def test_complex_shifts_forward_error_within_10x_of_complex_reduction(n):
    """test/core_tests.jl:264-268: the forward error of complex shifts on a real reduction is
    at most 10 x the complex reduction's (+ 100 eps), against a high-precision solution."""
    g = np.random.default_rng(n)
    J = g.standard_normal((n, n))
    b = crandn(np.random.default_rng(n + 7), n)
    Rr = O.reduce(J)
    Rc = O.reduce_c128(J.astype(np.complex128))
    eps = np.finfo(float).eps
    for s, t in SHIFTS:
        xr = xref_extended(J, s, t, b)
        x = O.ldiv_complex(Rr, O.shift_complex(Rr, s, t), b)
        xf = O.ldiv_c128(Rc, O.shift_c128(Rc, s, t), b)
        assert ferr(x, xr) <= 10 * ferr(xf, xr) + 100 * eps, (s, t, ferr(x, xr), ferr(xf, xr))


def test_complex_singular_shift_reports_info():
    """A zero pivot is reported in info, not raised (test/core_tests.jl:235-239)."""
    R = O.reduce_c128(np.array([[1.0, 0.0], [0.0, 2.0]], dtype=np.complex128))
    S = O.shift_c128(R, 1, -1.0)
    assert S.info != 0
    S = O.shift_c128(R, 1j, 1.0)
    assert S.info == 0


def test_complex_tie_matrix_pivots_first_max():
    """Gaussian-integer matrices have many equal moduli: the pivot is the first maximum (the
    strict > scan of F:470-477), so the complex reduction of an integer J equals the real one's
    pivots, and a rotated copy (J * i) has the same pivots (|i z| = |z| exactly)."""
    g = np.random.default_rng(5)
    for n in (9, 33, 64):
        J = g.integers(-2, 3, (n, n)).astype(float)
        Rr = O.reduce(J)
        Rc = O.reduce_c128(J.astype(np.complex128))
        Ri = O.reduce_c128(1j * J.astype(np.complex128))
        assert np.array_equal(Rr.ipiv, Rc.ipiv)
        assert np.array_equal(Rc.ipiv, Ri.ipiv)


# The reference's blocked generic reduction, which it runs for a complex J at n >= 768
# (src/LHLFactorization.jl:398, :705): the blocked order restated in the oracle (path 1).
@pytest.mark.parametrize("nb", [1, 3, 16])
@pytest.mark.parametrize("n", [3, 4, 17, 80, 200])
def test_complex_blocked_reconstructs_J(n, nb):
    g = np.random.default_rng(n + 7 * nb)
    J = crandn(g, n, n)
    R = O.reduce_c128(J, True, path=1, nb=nb)
    Z, Zi = R.Z(), R.Zinv()
    H = np.triu(R.factors, -1)
    assert np.linalg.norm(Z @ H @ Zi - J) <= 1e-10 * np.linalg.norm(J)
    assert np.all(np.abs(np.tril(R.factors, -2)) <= 1.0)
    assert np.array_equal(R.Ht, H.T)


@pytest.mark.parametrize("kind", ["randn", "tie"])
@pytest.mark.parametrize("n", [5, 40, 100, 300])
def test_complex_blocked_pivots_match_unblocked(n, kind):
    """test/threading.jl:58-79 and test/core_tests.jl:61-92 with a complex J: the blocked and
    unblocked orders take the same pivots, and their factors differ by at most 100 n eps ||F||."""
    g = np.random.default_rng(n)
    if kind == "tie":
        J = (g.integers(-2, 3, (n, n)) + 1j * g.integers(-2, 3, (n, n))).astype(np.complex128)
    else:
        J = crandn(g, n, n)
    U = O.reduce_c128(J, True, path=0)
    for nb in (2, 16):
        B = O.reduce_c128(J, True, path=1, nb=nb)
        assert np.array_equal(U.ipiv, B.ipiv), nb
        assert np.array_equal(U.scale, B.scale)
        assert np.linalg.norm(B.factors - U.factors) <= 100 * n * np.finfo(float).eps * np.linalg.norm(U.factors)


def _same_bits(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint8), np.ascontiguousarray(b).view(np.uint8))


def test_reference_order_above_768_against_the_device_order():
    """The reference's choice (path 2) is the unblocked order below n = 768 and the blocked one
    (nb = 16) from 768 on.  The device runs the unblocked order at every n, bit for bit with
    path 0; at n = 800 its pivots equal the reference order's and H and L lie within
    100 n eps of it (measured: about 1e-11 relative)."""
    g = np.random.default_rng(800)
    J = crandn(g, 767, 767) / math.sqrt(767)
    a, b = O.reduce_c128(J, path=2), O.reduce_c128(J, path=0)
    assert _same_bits(a.factors, b.factors)
    n = 800
    J = crandn(g, n, n) / math.sqrt(n)
    ref = O.reduce_c128(J, path=2)
    blk = O.reduce_c128(J, path=1, nb=16)
    assert _same_bits(ref.factors, blk.factors)
    dev_order = O.reduce_c128(J, path=0)
    assert np.array_equal(ref.ipiv, dev_order.ipiv)
    tol = 100 * n * np.finfo(float).eps
    for part in (lambda F: np.triu(F, -1), lambda F: np.tril(F, -2)):
        Fr, Fd = part(ref.factors), part(dev_order.factors)
        assert np.linalg.norm(Fd - Fr) <= tol * np.linalg.norm(Fr)


@pytest.mark.parametrize("n", [6, 33, 70])
def test_complex_blocked_zero_columns(n):
    """Zero pivots skip their step (F:812-813) in the blocked order too, panels wider than n
    included: the same pivots as the unblocked order, and J reconstructed."""
    g = np.random.default_rng(5 + n)
    J = crandn(g, n, n)
    J[:, 2] = 0
    J[5:, 1] = 0
    J[:, n // 2] = 0
    U = O.reduce_c128(J, path=0)
    for nb in (2, 16, 64):
        B = O.reduce_c128(J, path=1, nb=nb)
        assert np.array_equal(U.ipiv, B.ipiv), nb
        H = np.triu(B.factors, -1)
        assert np.linalg.norm(B.Z() @ H @ B.Zinv() - J) <= 1e-12 * np.linalg.norm(J)
