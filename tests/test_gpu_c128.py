"""A complex J (LHLWorkspace{ComplexF64}) on the device through the C ABI: the reduction
(ipiv, factors, Ht, scale, perm) and the shift LU (planar Gt, swap, rdiag, info) bit for bit
against the oracle, applyZ! / applyZinv! bit for bit, solves against the oracle and a dense
solve (test/core_tests.jl:241-249), the complex reduction of a real J against complex shifts
on the real reduction (:251-280), refinement with the complex W, save / load, and the
reference's errors."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

SHIFTS = ((0.4 + 0.7j, -1.0), (1.0, -0.05 + 0.3j), (0.0, 1j), (-3.0 + 2j, 2.0 - 1j), (1.0, -0.05))


def _mods():
    import torch
    import lhl_gpu as G
    return torch, G


def dev(a):
    torch, _ = _mods()
    return torch.as_tensor(np.asfortranarray(a)).cuda()


def host(t):
    return t.detach().cpu().numpy()


def crandn(g, *shape):
    return g.standard_normal(shape) + 1j * g.standard_normal(shape)


def bits_equal(a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    return a.shape == b.shape and a.dtype == b.dtype and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def bwd(W, x, b):
    r = b - W @ x
    return np.abs(r).max() / (np.abs(W).sum(axis=1).max() * np.abs(x).max() + np.abs(b).max())


def matrix(n, kind, seed):
    g = np.random.default_rng(seed)
    if kind == "tie":  # Gaussian integers: many equal moduli
        return (g.integers(-2, 3, (n, n)) + 1j * g.integers(-2, 3, (n, n))).astype(np.complex128)
    if kind == "graded":  # rows and columns over ten orders of magnitude: balancing scales
        d = 10.0 ** np.linspace(-5, 5, n)
        return (crandn(g, n, n) * d[:, None]) / d[None, :]
    return crandn(g, n, n)


@pytest.mark.parametrize("n", list(range(1, 18)) + [31, 64, 65, 129, 256, 300, 600, 767, 768, 769, 800, 1030])
@pytest.mark.parametrize("kind", ["randn", "tie", "graded"])
@pytest.mark.parametrize("balance", [True, False])
def test_complex_reduction_bitexact(n, kind, balance):
    """The reference's own order at every n: unblocked below _lhl_block_min(ComplexF64) = 768,
    the generic blocked form (nb = 16) from there (F:398-399, F:703-706)."""
    torch, G = _mods()
    J = matrix(n, kind, 100 + n)
    R = O.reduce_c128(J, balance, path=2)
    ws = G.lhl(dev(J), balance=balance)
    assert ws.dtype == torch.complex128 and ws.shift.is_complex
    torch.cuda.synchronize()
    ws.check()
    assert np.array_equal(host(ws.ipiv), R.ipiv)
    assert bits_equal(host(ws.scale), R.scale)
    assert bits_equal(host(ws.factors), R.factors)
    assert bits_equal(host(ws.Ht), R.Ht)
    assert np.array_equal(host(ws.perm), R.perm) and np.array_equal(host(ws.iperm), R.iperm)


@pytest.mark.parametrize("n", list(range(1, 121)) + [511, 512, 520])
@pytest.mark.parametrize("tie", [False, True])
def test_c128_shift_bitexact_reference_orders(n, tie):
    """test/core_tests.jl:192-201 for T = ComplexF64 at its orders (1:120, 511, 512, 520): the
    device shift LU on a complex Ht, bit for bit against the oracle (itself pinned to the
    independent restatement in tests/test_oracle.py), the reference test's five shifts;
    tie matrices are rand(-2:2) promoted to complex."""
    torch, G = _mods()
    g = np.random.default_rng(31 + n + 1000 * tie)
    J = g.integers(-2, 3, (n, n)).astype(np.complex128) if tie else crandn(g, n, n)
    R = O.reduce_c128(J)
    ws = G.LHLWorkspace(n, dtype=torch.complex128)
    ws.Ht.copy_(dev(R.Ht))
    for s, t in ((1, -0.1), (0, 1), (1, -3), (2, 0), (0, 0)):
        with np.errstate(divide="ignore", invalid="ignore"):
            So = O.shift_c128(R, s, t)
        G.lhl_shift_(ws, s, t)
        sh = ws.shift
        Gt = host(sh.Gt())
        po = sh.po
        assert sh.info == So.info
        assert bits_equal(host(sh.swap())[:n], So.swap[:n])
        for off in (0, po):
            assert bits_equal(Gt[off:off + n, :n].T[np.triu_indices(n)], So.Gt[off:off + n, :n].T[np.triu_indices(n)])
            assert bits_equal(Gt[off + np.arange(n - 1), np.arange(1, n)], So.Gt[off + np.arange(n - 1), np.arange(1, n)])
        if So.info == 0:
            assert bits_equal(host(sh.rdiag())[:n], So.rdiag[:n])


@pytest.mark.parametrize("n", [1, 2, 3, 5, 16, 33, 128, 129, 257, 600])
def test_complex_shift_and_z_bitexact(n):
    """The shift LU on the complex Ht and the two Z applications are the oracle's operations in
    the oracle's order; the solve differs from it only in the back substitution's summation
    order (tolerance 1e-12)."""
    torch, G = _mods()
    g = np.random.default_rng(7 * n)
    J = crandn(g, n, n)
    R = O.reduce_c128(J)
    ws = G.lhl(dev(J))
    b = crandn(g, n)
    for s, t in SHIFTS + ((0.0, 0.0),):
        G.lhl_shift_(ws, s, t)
        So = O.shift_c128(R, s, t)
        sh = ws.shift
        Gt = host(sh.Gt())
        assert sh.info == So.info
        assert bits_equal(host(sh.swap())[:n], So.swap[:n])
        assert bits_equal(host(sh.rdiag())[:n], So.rdiag[:n])
        for k in range(n):
            for off in (0, sh.po):
                assert bits_equal(Gt[off + k:off + n, k], So.Gt[off + k:off + n, k]), (s, t, k)
        if So.info:
            continue
        x = host(G.lhl_ldiv_(dev(b), ws))
        xo = O.ldiv_c128(R, So, b)
        assert np.linalg.norm(x - xo) <= 1e-12 * np.linalg.norm(xo)
    for fn_dev, fn_o in ((G.applyZ_, O.apply_z_c128), (G.applyZinv_, O.apply_zinv_c128)):
        X = crandn(g, n, 3)
        Xd = dev(X)
        fn_dev(Xd, ws)
        for c in range(3):
            assert bits_equal(host(Xd)[:, c], fn_o(R, X[:, c]))


def test_complex_solve_matches_dense():
    """test/core_tests.jl:241-249: n = 30, gamma = 0.2 + 0.3i."""
    torch, G = _mods()
    g = np.random.default_rng(13)
    n = 30
    J = crandn(g, n, n)
    b = crandn(g, n)
    gam = 0.2 + 0.3j
    ws = G.lhl(dev(J))
    G.lhl_shift_(ws, 1, -gam)
    x = host(G.lhl_ldiv_(dev(b), ws))
    xr = np.linalg.solve(np.eye(n) - gam * J, b)
    assert np.linalg.norm(x - xr) <= 1e-9 * np.linalg.norm(xr)


@pytest.mark.parametrize("n", [1, 2, 3, 5, 40, 129, 260, 600])
def test_complex_reduction_vs_complex_shifts_on_real(n):
    """test/core_tests.jl:251-280 on the device: ws = lhl(J; shift = ComplexF64), wf =
    lhl(complex.(J)); x == xf to 1e-9, both against the dense solve, one refinement step with
    the complex W (through the complex J) under 50 eps."""
    torch, G = _mods()
    g = np.random.default_rng(n)
    J = g.standard_normal((n, n))
    b = crandn(np.random.default_rng(n + 7), n)
    ws = G.lhl(dev(J), shift_complex=True)
    wf = G.lhl(dev(J.astype(np.complex128)))
    assert np.array_equal(host(ws.ipiv), host(wf.ipiv))
    Jc = dev(J.astype(np.complex128))
    eps = np.finfo(float).eps
    for s, t in SHIFTS:
        W = s * np.eye(n) + t * J
        G.lhl_shift_(ws, s, t)
        G.lhl_shift_(wf, s, t)
        x = host(G.lhl_ldiv_(dev(b), ws))
        xf_d = G.lhl_ldiv_(dev(b), wf)
        xf = host(xf_d)
        xd = np.linalg.solve(W, b)
        assert np.linalg.norm(x - xd) <= 1e-9 * np.linalg.norm(xd)
        assert np.linalg.norm(x - xf) <= 1e-9 * np.linalg.norm(x)
        G.lhl_refine_(xf_d, Jc, dev(b), wf, 1)
        y = host(xf_d)
        assert bwd(W, y, b) <= 2 * bwd(W, xf, b) + eps
        assert bwd(W, y, b) < 50 * eps


@pytest.mark.parametrize("n", [1, 2, 3, 5, 40, 129])
def test_complex_shifts_forward_error_within_10x_of_complex_reduction(n):
    """test/core_tests.jl:264-268 on the device: err(x) <= 10 err(xf) + 100 eps against a
    high-precision solution (FP64 solves corrected by extended-precision residuals)."""
    torch, G = _mods()
    g = np.random.default_rng(n)
    J = g.standard_normal((n, n))
    b = crandn(np.random.default_rng(n + 7), n)
    ws = G.lhl(dev(J), shift_complex=True)
    wf = G.lhl(dev(J.astype(np.complex128)))
    L = np.clongdouble
    eps = np.finfo(float).eps
    for s, t in SHIFTS:
        W64 = s * np.eye(n) + t * J
        WL = L(s) * np.eye(n, dtype=L) + L(t) * J.astype(L)
        xr = np.linalg.solve(W64, b).astype(L)
        for _ in range(6):
            xr = xr + np.linalg.solve(W64, (b.astype(L) - WL @ xr).astype(np.complex128)).astype(L)
        G.lhl_shift_(ws, s, t)
        G.lhl_shift_(wf, s, t)
        x = host(G.lhl_ldiv_(dev(b), ws)).astype(L)
        xf = host(G.lhl_ldiv_(dev(b), wf)).astype(L)
        ex = float(np.linalg.norm(x - xr) / np.linalg.norm(xr))
        ef = float(np.linalg.norm(xf - xr) / np.linalg.norm(xr))
        assert ex <= 10 * ef + 100 * eps, (s, t, ex, ef)


def test_complex_refinement_to_tolerance_and_gmres():
    """Several shifts and right-hand sides per shift on one complex reduction: fixed-point
    refinement to a tolerance and GMRES-IR both reach 1e-12, the residuals checked on the host."""
    torch, G = _mods()
    g = np.random.default_rng(3)
    n, S, rps = 200, 4, 3
    J = crandn(g, n, n) / np.sqrt(n)
    ws = G.LHLWorkspace(n, dtype=torch.complex128)
    G.lhl_reduce_(ws, dev(J), True)
    sh = G.LHLShift(n, S, complex=True)
    sig = torch.tensor(1.0 + 0.3j * np.arange(S), dtype=torch.complex128).cuda()
    tau = torch.tensor(-0.5 + 0.1j * np.arange(S), dtype=torch.complex128).cuda()
    G.lhl_shift_batched_(sh, ws, sig, tau)
    B = crandn(g, n, S * rps)
    Jd, Bd = dev(J), dev(B)
    for how in ("tol", "gmres"):
        X = torch.zeros((S * rps, n), dtype=torch.complex128, device="cuda").t()
        X.copy_(Bd)
        G.lhl_ldiv_(X, sh, ws, rhs_per_shift=rps)
        if how == "tol":
            res = G.lhl_refine_tol_(X, Jd, Bd, sh, ws, tol=1e-12, max_steps=6, rhs_per_shift=rps)
        else:
            res = G.lhl_refine_gmres_(X, Jd, Bd, sh, ws, tol=1e-12, max_cycles=4, restart=4, rhs_per_shift=rps)
        Xh = host(X)
        sg, tu = host(sig), host(tau)
        for c in range(S * rps):
            s = c // rps
            W = sg[s] * np.eye(n) + tu[s] * J
            rel = np.linalg.norm(B[:, c] - W @ Xh[:, c]) / np.linalg.norm(B[:, c])
            assert rel <= 1e-12, (how, c, rel)
        assert float(host(res).max()) <= 1e-12


def test_complex_above_block_threshold():
    """n = 1000 (>= 768: the reference's blocked form): the factors reconstruct J and are the
    oracle's blocked factors bit for bit, the pivots are the unblocked order's
    (test/threading.jl:58-79), and a shifted solve agrees with a dense solve to 1e-9."""
    torch, G = _mods()
    g = np.random.default_rng(1000)
    n = 1000
    J = crandn(g, n, n)
    ws = G.lhl(dev(J))
    H = np.triu(host(ws.factors), -1)
    Zi = dev(np.eye(n, dtype=np.complex128))
    G.applyZinv_(Zi, ws)
    Z = dev(np.eye(n, dtype=np.complex128))
    G.applyZ_(Z, ws)
    Zh, Zih = host(Z), host(Zi)
    assert np.linalg.norm(Zh @ H @ Zih - J) <= 1e-9 * np.linalg.norm(J)
    assert np.abs(np.tril(host(ws.factors), -2)).max() <= 1.0
    Ru = O.reduce_c128(J, True, path=0)
    assert np.array_equal(host(ws.ipiv), Ru.ipiv)
    assert bits_equal(host(ws.factors), O.reduce_c128(J, True, path=2).factors)
    b = crandn(g, n)
    G.lhl_shift_(ws, 1, -0.01 + 0.02j)
    x = host(G.lhl_ldiv_(dev(b), ws))
    xr = np.linalg.solve(np.eye(n) - (0.01 - 0.02j) * J, b)
    assert np.linalg.norm(x - xr) <= 1e-9 * np.linalg.norm(xr)


def test_complex_save_load(tmp_path):
    torch, G = _mods()
    g = np.random.default_rng(4)
    n = 77
    J = crandn(g, n, n)
    ws = G.lhl(dev(J))
    b = crandn(g, n)
    G.lhl_shift_(ws, 1, -0.1j)
    x = host(G.lhl_ldiv_(dev(b), ws))
    p = str(tmp_path / "ws.npz")
    ws.save(p)
    w2 = G.LHLWorkspace.load(p)
    assert w2.dtype == torch.complex128
    G.lhl_shift_(w2, 1, -0.1j)
    assert bits_equal(host(G.lhl_ldiv_(dev(b), w2)), x)


def test_complex_workspace_errors():
    torch, G = _mods()
    n = 6
    J = crandn(np.random.default_rng(0), n, n)
    ws = G.lhl(dev(J))
    with pytest.raises(G.ArgumentError):  # a real J on a complex workspace
        G.lhl_reduce_(ws, dev(J.real.copy()), True)
    with pytest.raises(G.ArgumentError):  # an LHLShift{Float64} cannot serve it (F:2463-2465)
        G.lhl_shift_(G.LHLShift(n, 1), ws, 1.0, -0.5)
    with pytest.raises(G.ArgumentError):  # a real x cannot hold the solution
        G.lhl_ldiv_(dev(np.ones(n)), ws)
    with pytest.raises(G.ArgumentError):  # the mixed form is real only
        G.LHLWorkspace(n, G.LHL_PREC_MIXED, dtype=torch.complex128)
    with pytest.raises(G.ArgumentError):  # a complex J on a real workspace
        G.lhl_reduce_(G.LHLWorkspace(n), dev(J), True)
    with pytest.raises(G.DimensionMismatch):
        G.lhl_ldiv_(dev(np.ones(n + 1, dtype=np.complex128)), ws)
    # real shifts are converted on a complex shift object
    G.lhl_shift_(ws, 2.0, -0.5)
    assert ws.shift.info == 0


@pytest.mark.parametrize("complex_j", [False, True])
def test_complex_solves_at_2048(complex_j):
    """n = 2048: the planar Hessenberg solve's dynamic shared memory is exactly 32 KB there, which
    with its static tiles passes the 48 KB default; complex shifts on a real J and a complex J
    both solve against a dense solve to 1e-9."""
    torch, G = _mods()
    n = 2048
    g = np.random.default_rng(2048)
    J = g.standard_normal((n, n)) / np.sqrt(n)
    if complex_j:
        J = J + 1j * g.standard_normal((n, n)) / np.sqrt(n)
    b = crandn(g, n)
    ws = G.lhl(dev(J)) if complex_j else G.lhl(dev(J), shift_complex=True)
    s, t = 1.0, -0.3 + 0.2j
    G.lhl_shift_(ws, s, t)
    x = host(G.lhl_ldiv_(dev(b), ws))
    xr = np.linalg.solve(s * np.eye(n) + t * J, b)
    assert np.linalg.norm(x - xr) <= 1e-9 * np.linalg.norm(xr)


@pytest.mark.parametrize("n", [30, 200, 800])
def test_complexf32_workspace(n):
    """LHLWorkspace{ComplexF32} (a complex64 J): test/core_tests.jl:241-249's solve with
    T = ComplexF32 and the Float32 tolerance (rtol 1e-3), ComplexF32 right-hand sides in and out;
    the factors and Ht hold ComplexF32 values and are the ComplexF64 reduction of the rounded J,
    rounded (bit for bit against the oracle's reduction, the reference's order from n = 768);
    a complex128 J on the same workspace is rounded on the way in; save / load."""
    torch, G = _mods()
    g = np.random.default_rng(13 + n)
    J = crandn(g, n, n).astype(np.complex64)
    b = crandn(g, n).astype(np.complex64)
    gam = np.complex64(0.2 + 0.3j)
    ws = G.lhl(dev(J))
    assert ws.dtype == torch.complex64 and ws.shift.is_complex
    ws.check()
    R = O.reduce_c128(J.astype(np.complex128), True, path=2)
    F = host(ws.factors)
    assert np.array_equal(F, R.factors.astype(np.complex64).astype(np.complex128))
    assert np.array_equal(host(ws.Ht), R.Ht.astype(np.complex64).astype(np.complex128))
    assert np.array_equal(host(ws.ipiv), R.ipiv)
    G.lhl_shift_(ws, 1, complex(-gam))
    x = G.lhl_ldiv_(dev(b), ws)
    assert x.dtype == torch.complex64
    W = np.eye(n) - gam.astype(np.complex128) * J.astype(np.complex128)
    xr = np.linalg.solve(W, b.astype(np.complex128))
    assert np.linalg.norm(host(x) - xr) <= 1e-3 * np.linalg.norm(xr)
    # a complex128 J is rounded to ComplexF32 on the way in: the same reduction
    w2 = G.LHLWorkspace(n, dtype=torch.complex64)
    G.lhl_reduce_(w2, dev(J.astype(np.complex128)), True)
    assert np.array_equal(host(w2.factors), F)
    if n == 30:
        import tempfile, os
        with tempfile.TemporaryDirectory() as d:
            pth = os.path.join(d, "ws.npz")
            ws.save(pth)
            w3 = G.LHLWorkspace.load(pth)
            assert w3.dtype == torch.complex64 and np.array_equal(host(w3.factors), F)
