"""The CPU oracle against the reference's own relation tests (test/core_tests.jl).

The reference ships no golden vectors; its tests pin the algorithm by relations.  Each test
below restates one of them on the oracle (numpy PCG64 inputs stand in for Julia's
MersenneTwister streams, which cannot be reproduced here)."""
import numpy as np
import pytest

from oracle import oracle as O


def rng(seed):
    return np.random.default_rng(seed)


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


# test/core_tests.jl:5-21 -- reduction reconstructs J, multipliers bounded by 1
@pytest.mark.parametrize("n", [1, 2, 3, 4, 17, 80, 128, 200, 301, 600])
@pytest.mark.parametrize("balance", [True, False])
def test_reconstruction(n, balance):
    J = rng(n).standard_normal((n, n))
    R = O.reduce(J, balance=balance)
    Z, Zi = R.Z(), R.Zinv()
    assert np.allclose(Z @ Zi, np.eye(n), atol=1e-10)
    assert rel(Z @ R.H @ Zi, J) < 1e-10
    if n > 2:
        assert np.abs(np.tril(R.factors, -2)).max() <= 1.0


# test/core_tests.jl:23-36 -- shifted solves against a dense LU
@pytest.mark.parametrize("n", [1, 2, 3, 5, 40, 129, 260])
def test_shifted_solves(n):
    J = rng(n).standard_normal((n, n))
    b = rng(n + 7).standard_normal(n)
    R = O.reduce(J)
    for s, t in ((1.0, 0.0), (1.0, -1e-8), (1.0, -0.05), (1.0, 1.7), (0.0, 1.0), (-3.0, 2.0)):
        W = s * np.eye(n) + t * J
        if np.linalg.matrix_rank(W) < n:
            continue
        S = O.shift(R, s, t)
        x = O.ldiv(R, S, b)
        assert rel(x, np.linalg.solve(W, b)) < 1e-9
        if n <= 260:
            assert O.bwd(W, x, b) < 50 * np.finfo(float).eps


# test/core_tests.jl:61-92 and test/threading.jl:58-79 -- blocked agrees with unblocked
@pytest.mark.parametrize("n", [160, 163, 200, 257])
@pytest.mark.parametrize("balance", [True, False])
def test_blocked_vs_unblocked(n, balance):
    J = rng(n).standard_normal((n, n))
    A = O.balance_raw(J)[0] if balance else J
    Fb, ipb = O.reduce_blocked_ptr_raw(A)
    Fg, ipg = O.reduce_blocked_raw(A)
    Fu, ipu = O.reduce_unblocked_raw(A)
    assert (ipb == ipu).all() and (ipg == ipu).all()
    eps = np.finfo(float).eps
    assert np.linalg.norm(Fb - Fu) <= 100 * n * eps * np.linalg.norm(Fu)
    assert np.linalg.norm(Fg - Fu) <= 100 * n * eps * np.linalg.norm(Fu)
    assert np.abs(np.tril(Fb, -2)).max() <= 1.0


def test_blocked_vs_unblocked_ties():
    J = rng(9).integers(-1, 2, (150, 150)).astype(float)
    A = O.balance_raw(J)[0]
    Fb, ipb = O.reduce_blocked_ptr_raw(A)
    Fu, ipu = O.reduce_unblocked_raw(A)
    assert (ipb == ipu).all()
    assert rel(Fb, Fu) < 1e-10


@pytest.mark.parametrize("n", list(range(3, 40)))
def test_blocked_small_panels(n):
    """Every panel shape, including pulled columns, against the unblocked path (nb = 4)."""
    for seed in range(3):
        J = rng(1000 * n + seed).standard_normal((n, n))
        Fb, ipb = O.reduce_blocked_ptr_raw(J, nb=4)
        Fu, ipu = O.reduce_unblocked_raw(J)
        assert (ipb == ipu).all()
        assert rel(Fb, Fu) < 1e-12


# test/core_tests.jl:115-212 -- the shift LU against the test file's own reference
def shift_ref(Ht, sigma, tau):
    """Pure-Python restatement of `_lhl_shift_ref!` (test/core_tests.jl:119-171).  With a
    float32 Ht and np.float32 sigma, tau every operation rounds to float32 (T = Float32)."""
    n = Ht.shape[0]
    Gt = np.zeros((n, n), dtype=Ht.dtype)
    swap = np.zeros(n, dtype=bool)
    rdiag = np.zeros(n, dtype=Ht.dtype)
    r = np.array([tau * Ht[j, 0] for j in range(n)])
    r[0] += sigma
    info = 0
    for k in range(n - 1):
        a = r[k]
        b = tau * Ht[k, k + 1]
        if abs(b) > abs(a):
            swap[k] = True
            Gt[k, k] = b
            l = a / b
            Gt[k, k + 1] = l
            for j in range(k + 1, n):
                g = tau * Ht[j, k + 1]
                Gt[j, k] = g
                r[j] -= l * g
            Gt[k + 1, k] += sigma
            r[k + 1] -= l * sigma
        else:
            swap[k] = False
            Gt[k, k] = a
            if a == 0:
                if info == 0:
                    info = k + 1
                l = 0.0
            else:
                l = b / a
            Gt[k, k + 1] = l
            for j in range(k + 1, n):
                rj = r[j]
                Gt[j, k] = rj
                r[j] = tau * Ht[j, k + 1] - l * rj
            r[k + 1] += sigma
    Gt[n - 1, n - 1] = r[n - 1]
    swap[n - 1] = False
    if Gt[n - 1, n - 1] == 0 and info == 0:
        info = n
    for j in range(n):
        rdiag[j] = 1.0 / Gt[j, j] if Gt[j, j] != 0 else np.inf
    U = np.array([Gt[j, k] for k in range(n) for j in range(k, n)])
    l = np.array([Gt[k, k + 1] for k in range(n - 1)])
    return U, l, swap, rdiag, info


def same_state(a, b):
    for u, v in zip(a[:4], b[:4]):
        u = np.asarray(u)
        v = np.asarray(v)
        if u.shape != v.shape:
            return False
        if u.dtype == np.float64:
            if not np.array_equal(u.view(np.int64), v.view(np.int64)):
                return False
        elif not np.array_equal(u.astype(np.int64), v.astype(np.int64)):
            return False
    return a[4] == b[4]


@pytest.mark.parametrize("n", list(range(1, 40)) + [63, 64, 65, 120])
@pytest.mark.parametrize("tie", [False, True])
def test_shift_matches_test_reference(n, tie):
    g = rng(31 + n + 1000 * tie)
    J = g.integers(-2, 3, (n, n)).astype(float) if tie else g.standard_normal((n, n))
    R = O.reduce(J)
    for s, t in ((1, -0.1), (0, 1), (1, -3), (2, 0), (0, 0)):
        with np.errstate(divide="ignore", invalid="ignore"):
            S = O.shift(R, s, t)
            ref = shift_ref(R.Ht, float(s), float(t))
        st = S.state()
        st = (st[0], st[1], st[2].astype(bool), st[3], st[4])
        assert same_state(st, ref), (n, tie, s, t)


# test/core_tests.jl:235-239
def test_singular_shift_reported():
    R = O.reduce(np.array([[1.0, 0.0], [0.0, 2.0]]))
    S = O.shift(R, 1.0, -1.0)
    assert S.info != 0


# test/core_tests.jl:337-380 -- pivoting families and near-nilpotent, one refinement step
def wilkinson(n):
    return np.array([[1.0 if i == j else (1.0 if j == n - 1 else (-1.0 if i > j else 0.0))
                      for j in range(n)] for i in range(n)])


def test_pivoting_families_refined():
    n = 100
    mats = {
        "randn": rng(1).standard_normal((n, n)),
        "wilkinson": wilkinson(n),
        "graded": np.diag(10.0 ** np.linspace(-8, 8, n)) @ rng(3).standard_normal((n, n))
        @ np.diag(10.0 ** np.linspace(8, -8, n)),
    }
    b = rng(42).standard_normal(n)
    for name, J in mats.items():
        R = O.reduce(J)
        assert np.abs(np.tril(R.factors, -2)).max() <= 1 + np.finfo(float).eps
        for g in (1e-3, 1.0, 1e3):
            S = O.shift(R, 1.0, -g)
            if S.info != 0:
                continue
            x = O.ldiv(R, S, b)
            W = np.eye(n) - g * J
            x = O.refine(R, S, J, b, x, 1)
            assert O.bwd(W, x, b) < 1e-13, (name, g)


def test_near_nilpotent_refined():
    n = 60
    J = np.triu(rng(17).standard_normal((n, n)), 1)
    J[n - 1, 0] = 1e-8
    b = rng(18).standard_normal(n)
    g = 0.5
    W = np.eye(n) - g * J
    R = O.reduce(J)
    S = O.shift(R, 1.0, -g)
    raw = O.ldiv(R, S, b)
    ref = O.refine(R, S, J, b, raw, 1)
    assert O.bwd(W, ref, b) <= O.bwd(W, raw, b)
    assert O.bwd(W, ref, b) < 1e-13


def test_batch_driver_matches_single():
    n = 90
    J = rng(7).standard_normal((n, n))
    R = O.reduce(J)
    sig = np.ones(5)
    tau = -np.array([0.01, 0.02, 0.05, 0.1, 0.3])
    B = np.asfortranarray(rng(8).standard_normal((n, 5)))
    X, info = O.shift_solve_batch(R, J, sig, tau, B, steps=1)
    for s in range(5):
        S = O.shift(R, sig[s], tau[s])
        x = O.ldiv(R, S, B[:, s])
        x = O.refine(R, S, J, B[:, s], x, 1)
        assert np.array_equal(x, X[:, s])
        assert info[s] == S.info


# ---- complex shifts on a real reduction (test/core_tests.jl:214-233, :251-280) ----------

def _cdiv(a, b):
    """Baudin & Smith's robust complex division on (re, im) pairs, written independently of
    the oracle's C code (the oracle's stand-in for Julia's ComplexF64 `/`)."""
    (ar, ai), (c, d) = a, b

    def two(a_, b_, c_, d_, r, t):
        if r != 0.0:
            br = b_ * r
            return (a_ + br) * t if br != 0.0 else a_ * t + (b_ * t) * r
        return (a_ + d_ * (b_ / c_)) * t

    if abs(d) <= abs(c):
        r = d / c
        t = 1.0 / (c + d * r)
        return two(ar, ai, c, d, r, t), two(ai, -ar, c, d, r, t)
    r = c / d
    t = 1.0 / (d + c * r)
    return two(ai, ar, d, c, r, t), -two(ar, -ai, d, c, r, t)


def shift_ref_complex(Ht, sigma, tau):
    """Pure-Python restatement of the complex shift LU (F:2529-2594 with TG = ComplexF64;
    `_lhl_shift_ref!` of test/core_tests.jl:119-171 on complex values): complex products
    (ac - bd, ad + bc), tau times a real Ht entry scaling both parts (a shift on a real
    reduction) or a complex product (a complex reduction's Ht), pivot magnitude |re| + |im|.
    Returns (U, l, swap, rdiag, info) as complex arrays."""
    n = Ht.shape[0]
    sr, si = sigma.real, sigma.imag
    tr, ti = tau.real, tau.imag
    mul = lambda a, b: (a[0] * b[0] - a[1] * b[1], a[0] * b[1] + a[1] * b[0])  # noqa: E731
    sub = lambda a, b: (a[0] - b[0], a[1] - b[1])  # noqa: E731
    add = lambda a, b: (a[0] + b[0], a[1] + b[1])  # noqa: E731
    if np.iscomplexobj(Ht):
        sc = lambda h: mul((tr, ti), (h.real, h.imag))  # noqa: E731
    else:
        sc = lambda h: (tr * h, ti * h)  # noqa: E731
    mag = lambda a: abs(a[0]) + abs(a[1])  # noqa: E731
    r = [sc(Ht[j, 0]) for j in range(n)]
    r[0] = add(r[0], (sr, si))
    G = {}
    swap = [0] * n
    lv = []
    info = 0
    for k in range(n - 1):
        a = r[k]
        b = sc(Ht[k, k + 1])
        if mag(b) > mag(a):
            swap[k] = 1
            G[(k, k)] = b
            l = _cdiv(a, b)
            for j in range(k + 1, n):
                g = sc(Ht[j, k + 1])
                G[(j, k)] = g
                r[j] = sub(r[j], mul(l, g))
            G[(k + 1, k)] = add(G[(k + 1, k)], (sr, si))
            r[k + 1] = sub(r[k + 1], mul(l, (sr, si)))
        else:
            G[(k, k)] = a
            if a == (0.0, 0.0):
                info = info or (k + 1)
                l = (0.0, 0.0)
            else:
                l = _cdiv(b, a)
            for j in range(k + 1, n):
                rj = r[j]
                G[(j, k)] = rj
                r[j] = sub(sc(Ht[j, k + 1]), mul(l, rj))
            r[k + 1] = add(r[k + 1], (sr, si))
        lv.append(l)
    G[(n - 1, n - 1)] = r[n - 1]
    if r[n - 1] == (0.0, 0.0) and info == 0:
        info = n
    U = O.cpack([G[(j, k)][0] for k in range(n) for j in range(k, n)], [G[(j, k)][1] for k in range(n) for j in range(k, n)])
    q = [_cdiv((1.0, 0.0), G[(j, j)]) for j in range(n)]
    rd = O.cpack([v[0] for v in q], [v[1] for v in q])
    return U, O.cpack([v[0] for v in lv], [v[1] for v in lv]), np.array(swap, dtype=np.uint8), rd, info


def cstate(S):
    n, po, G = S.n, S.po, S.Gt
    U = O.cpack([G[j, k] for k in range(n) for j in range(k, n)], [G[po + j, k] for k in range(n) for j in range(k, n)])
    l = O.cpack([G[k, k + 1] for k in range(n - 1)], [G[po + k, k + 1] for k in range(n - 1)])
    return U, l, S.swap[:n].copy(), S.rdiag[:n].copy(), S.info


def cbits_equal(a, b):
    a = np.ascontiguousarray(a, dtype=np.complex128)
    b = np.ascontiguousarray(b, dtype=np.complex128)
    return a.shape == b.shape and np.array_equal(a.view(np.int64), b.view(np.int64))


@pytest.mark.filterwarnings("ignore::RuntimeWarning")  # the (0, 0) shift divides by zero, as in the reference
@pytest.mark.parametrize("n", list(range(1, 41)) + [64, 65, 130])
@pytest.mark.parametrize("tie", [False, True])
def test_c128_shift_matches_restatement(n, tie):
    """test/core_tests.jl:192-201 for T = ComplexF64: the shift LU of a complex reduction (complex
    Ht), bit for bit against the independent restatement, over the reference test's shifts;
    tie matrices are rand(-2:2) promoted to complex, as the test's tie_matrix does."""
    g = rng(31 + n)
    if tie:
        J = g.integers(-2, 3, (n, n)).astype(np.complex128)
    else:
        J = g.standard_normal((n, n)) + 1j * g.standard_normal((n, n))
    R = O.reduce_c128(J)
    for s, t in ((1, -0.1), (0, 1), (1, -3), (2, 0), (0, 0)):
        S = O.shift_c128(R, s, t)
        U, l, sw, rd, info = shift_ref_complex(R.Ht, complex(s), complex(t))
        Uo, lo, swo, rdo, infoo = cstate(S)
        assert cbits_equal(U, Uo) and cbits_equal(l, lo) and np.array_equal(sw, swo)
        assert info == infoo
        if info == 0:
            assert cbits_equal(rd, rdo)


@pytest.mark.filterwarnings("ignore::RuntimeWarning")  # the (0, 0) shift divides by zero, as in the reference
@pytest.mark.parametrize("n", list(range(1, 25)) + [64, 65, 130])
@pytest.mark.parametrize("tie", [False, True])
def test_complex_shift_matches_restatement(n, tie):
    """test/core_tests.jl:214-233: the complex-on-real shift LU, bit for bit against an
    independent restatement, for the reference test's five shifts."""
    g = rng(32 + n)
    J = g.integers(-2, 3, (n, n)).astype(float) if tie else g.standard_normal((n, n))
    R = O.reduce(J)
    for s, t in ((0.4 + 0.7j, -1), (1, -0.1 + 0.2j), (0, 1j), (2j, 0), (0, 0)):
        S = O.shift_complex(R, s, t)
        U, l, sw, rd, info = shift_ref_complex(R.Ht, complex(s), complex(t))
        Uo, lo, swo, rdo, infoo = cstate(S)
        assert cbits_equal(U, Uo) and cbits_equal(l, lo) and np.array_equal(sw, swo)
        assert info == infoo
        if info == 0:
            assert cbits_equal(rd, rdo)


@pytest.mark.parametrize("n", [1, 2, 3, 5, 40, 129, 260, 600])
def test_complex_shifts_on_a_real_reduction(n):
    """test/core_tests.jl:251-280: solves against a dense complex LU (rtol 1e-9), and one
    refinement step with the complex system matrix: bwd <= 2 bwd(x) + eps and < 50 eps."""
    J = rng(n).standard_normal((n, n))
    g = rng(n + 7)
    b = g.standard_normal(n) + 1j * g.standard_normal(n)
    R = O.reduce(J)
    eps = np.finfo(float).eps
    for s, t in ((0.4 + 0.7j, -1.0), (1.0, -0.05 + 0.3j), (0.0, 1j), (-3.0 + 2j, 2.0 - 1j), (1.0, -0.05)):
        W = s * np.eye(n) + t * J
        S = O.shift_complex(R, s, t)
        x = O.ldiv_complex(R, S, b)
        xr = np.linalg.solve(W, b)
        assert np.linalg.norm(x - xr) <= 1e-9 * np.linalg.norm(xr)
        y = O.refine_complex(R, S, J, b, x, 1)
        assert O.bwd(W, y, b) <= 2 * O.bwd(W, x, b) + eps
        assert O.bwd(W, y, b) < 50 * eps


SHIFTS_REF = ((1.0, -0.1), (0.0, 1.0), (1.0, -3.0), (2.0, 0.0), (0.0, 0.0))


@pytest.mark.parametrize("n", list(range(1, 34)) + [64, 130, 257])
@pytest.mark.parametrize("tie", [False, True])
def test_shift_f32_matches_restatement(n, tie):
    """LHLWorkspace{Float32}'s shift LU (test/core_tests.jl:192-203 with T = Float32): the
    oracle's float restatement against the pure-Python one run in numpy float32, bit for bit,
    on upper Hessenberg matrices (random, and with ties and zeros)."""
    g = rng(900 + n)
    H = g.integers(-2, 3, (n, n)) if tie else g.standard_normal((n, n))
    H = np.triu(H.astype(np.float32), -1)
    Ht = np.asfortranarray(H.T)
    for s, t in SHIFTS_REF:
        U, l, sw, rd, info = shift_ref(Ht, np.float32(s), np.float32(t))
        S = O.shift_f32(Ht, s, t)
        Uo, lo, swo, rdo, infoo = S.state()
        assert info == infoo, (s, t)
        assert np.array_equal(np.asarray(swo, dtype=bool), sw)
        for a, b in ((U, Uo), (l, lo), (rd, rdo)):
            a32 = np.asarray(a, dtype=np.float32)
            b32 = np.asarray(b).astype(np.float32)
            assert np.array_equal(b32.astype(np.float64), np.asarray(b)), "not float values"
            assert np.array_equal(a32.view(np.int32), b32.view(np.int32)), (s, t)


def test_balancing_ends_on_an_infinite_norm():
    """An infinite entry: the reference's balancing loops never end (c = r = Inf keeps c >= 2r true,
    F:313-320); the oracle carries the device's bounds on them, which finite norms never reach, and
    decides "no scaling" for such an index.  Pivots stay valid row indices and the NaNs propagate."""
    n = 40
    J = rng(7).standard_normal((n, n))
    J[n - 3, 3] = np.inf
    J[5, 7] = np.nan
    R = O.reduce(J)
    assert all(k + 2 <= R.ipiv[k] <= n for k in range(n - 2))
    assert np.isnan(R.factors).any()
    assert np.all(R.scale * R.iscale == 1.0)
    C = O.reduce_c128(J.astype(np.complex128))
    assert all(k + 2 <= C.ipiv[k] <= n for k in range(n - 2))
