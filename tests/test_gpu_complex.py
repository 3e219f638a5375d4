"""Complex shifts on a real reduction (LHLShift{ComplexF64} on LHLWorkspace{Float64}) on the
device, through the C ABI: the shift LU bit for bit against the oracle (planar Gt, swap,
rdiag, info), solves against a dense complex LU and the oracle (test/core_tests.jl:251-280),
refinement to 1e-10 on a resolvent sweep shaped like config 5, and the reference's errors."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

SHIFTS = ((0.4 + 0.7j, -1.0), (1.0, -0.1 + 0.2j), (0.0, 1j), (2j, 0.0), (-3.0 + 2j, 2.0 - 1j))


def _mods():
    import torch
    import lhl_gpu as G
    return torch, G


def dev(a):
    torch, _ = _mods()
    return torch.as_tensor(np.asfortranarray(a)).cuda()


def host(t):
    return t.detach().cpu().numpy()


def rng(seed):
    return np.random.default_rng(seed)


def bits_equal(a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    return a.shape == b.shape and a.dtype == b.dtype and np.array_equal(a.view(np.uint8), b.view(np.uint8))


@pytest.mark.parametrize("n", list(range(1, 101)) + [255, 256, 257, 511, 512, 513, 520, 700, 1024, 2048])
@pytest.mark.parametrize("tie", [False, True])
def test_complex_shift_bitexact(n, tie):
    """The device shift LU (planar Gt, swap, rdiag, info) is bit-identical to the oracle's."""
    torch, G = _mods()
    g = rng(32 + n)
    J = g.integers(-2, 3, (n, n)).astype(float) if tie else g.standard_normal((n, n))
    R = O.reduce(J)
    ws = G.lhl(dev(J), shift_complex=True)
    for s, t in SHIFTS + ((0.0, 0.0),):
        G.lhl_shift_(ws, s, t)
        So = O.shift_complex(R, s, t)
        sh = ws.shift
        assert sh.po == So.po
        Gt = host(sh.Gt())
        torch.cuda.synchronize()
        # every entry the elimination writes: rows k..n of column k and row k of column k+1, both planes
        for k in range(n):
            for off in (0, sh.po):
                assert bits_equal(Gt[off + k:off + n, k], So.Gt[off + k:off + n, k]), (s, t, k)
                if k + 1 < n:
                    assert bits_equal(Gt[off + k, k + 1:k + 2], So.Gt[off + k, k + 1:k + 2])
        assert np.array_equal(host(sh.swap())[:n], So.swap[:n])
        assert sh.info == So.info
        if So.info == 0:
            assert bits_equal(host(sh.rdiag()), So.rdiag[:n])


@pytest.mark.parametrize("n", [1, 2, 3, 5, 40, 129, 260, 600])
def test_complex_solves(n):
    """test/core_tests.jl:251-280 on the device: solves against a dense complex LU (rtol 1e-9) and
    the oracle's, and one refinement step: bwd <= 2 bwd(x) + eps and < 50 eps."""
    torch, G = _mods()
    J = rng(n).standard_normal((n, n))
    g = rng(n + 7)
    b = g.standard_normal(n) + 1j * g.standard_normal(n)
    R = O.reduce(J)
    Jd = dev(J)
    ws = G.lhl(Jd, shift_complex=True)
    eps = np.finfo(float).eps
    for s, t in ((0.4 + 0.7j, -1.0), (1.0, -0.05 + 0.3j), (0.0, 1j), (-3.0 + 2j, 2.0 - 1j), (1.0, -0.05)):
        W = s * np.eye(n) + t * J
        G.lhl_shift_(ws, s, t)
        x = G.lhl_ldiv_(dev(b), ws)
        xh = host(x)
        xr = np.linalg.solve(W, b)
        assert np.linalg.norm(xh - xr) <= 1e-9 * np.linalg.norm(xr)
        xo = O.ldiv_complex(R, O.shift_complex(R, s, t), b)
        assert np.linalg.norm(xh - xo) <= 1e-9 * np.linalg.norm(xo)
        y = host(G.lhl_refine_(x.clone(), Jd, dev(b), ws, 1))
        assert O.bwd(W, y, b) <= 2 * O.bwd(W, xh, b) + eps
        assert O.bwd(W, y, b) < 50 * eps


@pytest.mark.parametrize("n", [60, 700])
def test_complex_batched_matches_single(n):
    torch, G = _mods()
    J = rng(3 + n).standard_normal((n, n))
    ws = G.lhl(dev(J), shift_complex=True)
    sig = np.array([0.5 + 1j, -1.0 + 3j, 0.2j, 2.0])
    tau = np.array([-1.0, -1.0 + 0.1j, 1.0, -0.5j])
    sh = G.LHLShift(n, 4, complex=True)
    G.lhl_shift_batched_(sh, ws, dev(sig), dev(tau))
    B = rng(4).standard_normal((n, 8)) + 1j * rng(5).standard_normal((n, 8))
    X = dev(B)
    G.lhl_ldiv_(X, sh, ws, rhs_per_shift=2)
    Xh = host(X)
    for s in range(4):
        G.lhl_shift_(ws, sig[s], tau[s])
        assert bits_equal(host(ws.shift.Gt()), host(sh.Gt(s)))
        for r in range(2):
            x1 = host(G.lhl_ldiv_(dev(B[:, 2 * s + r]), ws))
            assert bits_equal(x1, Xh[:, 2 * s + r])


@pytest.mark.parametrize("n,rps,ncols", [(1, 4, 8), (2, 4, 5), (33, 11, 30), (100, 32, 96), (1000, 8, 24),
                                          (2049, 5, 14)])
def test_complex_multi_rhs_solve_matches_one_vector_solves(n, rps, ncols):
    """Several right-hand sides per shift take the multi-vector Hessenberg solve (groups of up
    to eight vectors of one shift per CTA; partial groups, a partial last shift and odd orders
    included); each column agrees with the one-vector solve of the same shift slot to 1e-10
    (the two sum in different orders; W's condition is up to ~1e3 here) and its backward error
    is as small as that solve's."""
    torch, G = _mods()
    J = rng(50 + n).standard_normal((n, n)) / np.sqrt(max(n, 1))
    ws = G.lhl(dev(J), shift_complex=True)
    S = (ncols + rps - 1) // rps
    g = rng(51)
    sig = g.uniform(-2.0, 0.0, S) + 1j * g.uniform(0.0, 10.0, S)
    tau = -np.ones(S, dtype=complex)
    sh = G.LHLShift(n, S, complex=True)
    G.lhl_shift_batched_(sh, ws, dev(sig), dev(tau))
    B = rng(52).standard_normal((n, ncols)) + 1j * rng(53).standard_normal((n, ncols))
    X = dev(B)
    G.lhl_ldiv_(X, sh, ws, rhs_per_shift=rps)
    Xh = host(X)
    eps = np.finfo(float).eps
    for c in range(ncols):
        G.lhl_shift_(ws, sig[c // rps], tau[c // rps])
        x1 = host(G.lhl_ldiv_(dev(np.ascontiguousarray(B[:, c])), ws))
        assert np.linalg.norm(Xh[:, c] - x1) <= 1e-10 * np.linalg.norm(x1), (n, rps, c)
        W = sig[c // rps] * np.eye(n) + tau[c // rps] * J
        assert O.bwd(W, Xh[:, c], B[:, c]) <= 4 * O.bwd(W, x1, B[:, c]) + 50 * eps, (n, rps, c)


@pytest.mark.parametrize("n,S,rps,precision", [(3, 20, 32, "fp64"), (65, 17, 32, "fp64"), (200, 9, 64, "mixed"),
                                                (1030, 17, 32, "fp64"), (1030, 17, 32, "mixed")])
def test_complex_wide_sweeps_match_one_vector_solves(n, S, rps, precision):
    """From 1024 real columns (512 complex right-hand sides) on, the L sweeps of the solve run as
    64-column tensor-pipe tiles (FP64 MMAs; the mixed form's diagonal blocks by their inverses).
    Sampled columns agree with one-vector solves of the same shift to 1e-10, edges of the
    64-row and 64-column tiles included."""
    torch, G = _mods()
    J = rng(70 + n).standard_normal((n, n)) / np.sqrt(n)
    prec = G.LHL_PREC_MIXED if precision == "mixed" else G.LHL_PREC_FP64
    ws = G.lhl(dev(J), precision=prec, shift_complex=True)
    ws.check()
    g = rng(71)
    sig = g.uniform(-2.0, 0.0, S) + 1j * g.uniform(0.0, 10.0, S)
    tau = -np.ones(S, dtype=complex)
    sh = G.LHLShift(n, S, complex=True)
    G.lhl_shift_batched_(sh, ws, dev(sig), dev(tau))
    ncols = S * rps - 3  # a partial last shift and column tile
    assert 2 * ncols >= 1024
    B = rng(72).standard_normal((n, ncols)) + 1j * rng(73).standard_normal((n, ncols))
    X = dev(B)
    G.lhl_ldiv_(X, sh, ws, rhs_per_shift=rps)
    Xh = host(X)
    for c in sorted({0, 1, 31, 32, 63, ncols // 2, ncols - 1}):
        G.lhl_shift_(ws, sig[c // rps], tau[c // rps])
        x1 = host(G.lhl_ldiv_(dev(np.ascontiguousarray(B[:, c])), ws))
        assert np.linalg.norm(Xh[:, c] - x1) <= 1e-10 * np.linalg.norm(x1), (n, c)


def test_complex_many_rhs_chain_is_deterministic():
    """The many-right-hand-side kernels (64-column tensor-pipe L sweeps, the multi-vector
    Hessenberg solve, the tensor-pipe residual) give the same bits on a second run: every sum
    has a fixed order, none depends on which CTA or warp finishes first."""
    torch, G = _mods()
    n, S, rps = 300, 20, 32
    J = rng(80).standard_normal((n, n)) / np.sqrt(n)
    ws = G.lhl(dev(J), shift_complex=True)
    g = rng(81)
    sig = g.uniform(-2.0, 0.0, S) + 1j * g.uniform(0.0, 10.0, S)
    sh = G.LHLShift(n, S, complex=True)
    G.lhl_shift_batched_(sh, ws, dev(sig), dev(-np.ones(S, dtype=complex)))
    B = rng(82).standard_normal((n, S * rps)) + 1j * rng(83).standard_normal((n, S * rps))
    Jd, Bd = dev(J), dev(B)
    out = []
    for _ in range(2):
        X = Bd.clone()
        G.lhl_ldiv_(X, sh, ws, rhs_per_shift=rps)
        res = G.lhl_refine_tol_(X, Jd, Bd, sh, ws, tol=0.0, max_steps=2, rhs_per_shift=rps)
        out.append((host(X), host(res)))
    assert np.array_equal(np.ascontiguousarray(out[0][0]).view(np.uint64), np.ascontiguousarray(out[1][0]).view(np.uint64))
    assert np.array_equal(out[0][1], out[1][1])
    assert (out[0][1] <= 1e-12).all()


@pytest.mark.parametrize("n,nrhs,rps", [(1, 16, 4), (37, 16, 1), (200, 45, 5), (1030, 64, 32)])
def test_complex_residual_many_rhs(n, nrhs, rps):
    """From 16 complex right-hand sides on, the residual r = b - (sigma x + tau J x) runs as a
    tensor-pipe GEMM (FP64 MMAs); its norms agree with numpy's to 1e-12 relative, with edges of
    the 128-row and 32-column tiles and a partial last shift."""
    torch, G = _mods()
    J = rng(60 + n).standard_normal((n, n))
    ws = G.lhl(dev(J), shift_complex=True)
    S = (nrhs + rps - 1) // rps
    g = rng(61)
    sig = g.uniform(-2.0, 0.0, S) + 1j * g.uniform(0.0, 10.0, S)
    tau = g.uniform(-1.0, 1.0, S) + 1j * g.uniform(-1.0, 1.0, S)
    sh = G.LHLShift(n, S, complex=True)
    G.lhl_shift_batched_(sh, ws, dev(sig), dev(tau))
    B = rng(62).standard_normal((n, nrhs)) + 1j * rng(63).standard_normal((n, nrhs))
    X = rng(64).standard_normal((n, nrhs)) + 1j * rng(65).standard_normal((n, nrhs))
    got = host(G.residual_norms(sh, dev(J), dev(B), dev(X), rhs_per_shift=rps))
    for c in range(nrhs):
        s = c // rps
        r = B[:, c] - (sig[s] * X[:, c] + tau[s] * (J @ X[:, c]))
        want = np.linalg.norm(r) / np.linalg.norm(B[:, c])
        assert abs(got[c] - want) <= 1e-12 * want, (n, c, got[c], want)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_resolvent_sweep_reaches_1e10(precision):
    """Config 5's shape at n = 1024: J ~ N(0,1)/sqrt(n), complex shifts s = a + ib with a in
    [-2, 0], b in [0, 10], (sigma, tau) = (s, -1), four complex N(0,1) right-hand sides per
    shift, refined to relative residual <= 1e-10 in both forms."""
    torch, G = _mods()
    n, S, Rr = 1024, 8, 4
    J = rng(10).standard_normal((n, n)) / np.sqrt(n)
    g = rng(11)
    s = g.uniform(-2.0, 0.0, S) + 1j * g.uniform(0.0, 10.0, S)
    g2 = rng(12)
    B = g2.standard_normal((n, S * Rr)) + 1j * g2.standard_normal((n, S * Rr))
    Jd = dev(J)
    prec = G.LHL_PREC_MIXED if precision == "mixed" else G.LHL_PREC_FP64
    ws = G.lhl(Jd, precision=prec, shift_complex=True)
    ws.check()
    sh = G.LHLShift(n, S, complex=True)
    G.lhl_shift_batched_(sh, ws, dev(s), dev(-np.ones(S, dtype=complex)))
    Bd = dev(B)
    X = Bd.clone()
    G.lhl_ldiv_(X, sh, ws, rhs_per_shift=Rr)
    res = host(G.lhl_refine_tol_(X, Jd, Bd, sh, ws, tol=1e-10, max_steps=16, rhs_per_shift=Rr))
    assert (res <= 1e-10).all(), res
    Xh = host(X)
    for c in (0, S * Rr - 1):
        W = s[c // Rr] * np.eye(n) - J
        assert np.linalg.norm(B[:, c] - W @ Xh[:, c]) <= 1.0001e-10 * np.linalg.norm(B[:, c])


def test_complex_errors_mirror_the_reference():
    torch, G = _mods()
    n = 6
    J = rng(1).standard_normal((n, n))
    ws = G.lhl(dev(J))
    with pytest.raises(G.ArgumentError):  # complex shift on a real LHLShift (F:2466-2472)
        G.lhl_shift_(ws, 1.0, -0.3j)
    G.lhl_shift_(ws, 1.0, -0.3)
    # complex x with a real shift: the reference's generic path (F:3052-3074), the two parts
    # solved as real vectors
    z = dev(np.arange(1.0, n + 1) + 1j * np.ones(n))
    assert G.lhl_ldiv_(z, ws) is z
    xr = host(G.lhl_ldiv_(dev(np.arange(1.0, n + 1)), ws))
    xi = host(G.lhl_ldiv_(dev(np.ones(n)), ws))
    assert np.allclose(host(z), xr + 1j * xi, rtol=1e-13, atol=0)
    wc = G.lhl(dev(J), shift_complex=True)
    G.lhl_shift_(wc, 1.0 + 1j, -0.3)
    with pytest.raises(G.ArgumentError):  # a real x cannot hold a complex shift's solution (F:3084-3085)
        G.lhl_ldiv_(dev(np.ones(n)), wc)
    x = dev(np.ones(n) + 0j)
    assert G.lhl_ldiv_(x, wc) is x
    # a real shift on a complex LHLShift is converted (F:2474-2475)
    G.lhl_shift_(wc, 2.0, -0.5)
    Wr = 2.0 * np.eye(n) - 0.5 * J
    b = rng(2).standard_normal(n) + 0j
    assert np.allclose(host(G.lhl_ldiv_(dev(b), wc)), np.linalg.solve(Wr, b), rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("n", [4099, 8192])
@pytest.mark.parametrize("complex_ht", [False, True])
def test_complex_shift_bitexact_large(n, complex_ht):
    """The 1024-thread complex shift LU (4096 < n <= 8192, config 5's size) on a random upper
    Hessenberg H placed straight into a workspace's Ht: bit for bit against the oracle."""
    torch, G = _mods()
    g = rng(n)
    H = np.triu(g.standard_normal((n, n)), -1)
    if complex_ht:
        H = H + 1j * np.triu(g.standard_normal((n, n)), -1)
    Ht = np.asfortranarray(H.T)
    if complex_ht:
        ws = G.LHLWorkspace(n, dtype=torch.complex128)
    else:
        ws = G.LHLWorkspace(n, shift_complex=True)
    ws.Ht.copy_(dev(Ht))
    R = O.ReductionC(n) if complex_ht else O.Reduction(n)
    R.Ht = Ht
    s, t = 0.4 + 0.7j, -1.0 + 0.1j
    G.lhl_shift_(ws, s, t)
    So = O.shift_c128(R, s, t) if complex_ht else O.shift_complex(R, s, t)
    sh = ws.shift
    Gt = host(sh.Gt())
    assert sh.info == So.info
    iu = np.triu_indices(n)
    for off in (0, sh.po):
        assert bits_equal(Gt[off:off + n, :n].T[iu], So.Gt[off:off + n, :n].T[iu])
        assert bits_equal(Gt[off + np.arange(n - 1), np.arange(1, n)], So.Gt[off + np.arange(n - 1), np.arange(1, n)])
    assert np.array_equal(host(sh.swap())[:n], So.swap[:n])
    assert bits_equal(host(sh.rdiag()), So.rdiag[:n])


@pytest.mark.parametrize("n,rps,groups", [(33, 11, [(1, 0), (1, 1), (4, 0)]), (1000, 8, [(2, 0)]),
                                          (2049, 11, [(0, 1), (3, 0), (5, 0), (5, 1)]),
                                          (1000, 32, [(s, g) for s in range(4) for g in range(4)]),
                                          (1000, 32, [(s, g) for s in range(6) for g in range(4)])])
def test_few_groups_refine_through_the_grid_wide_solve(n, rps, groups):
    """Refinement steps where only a few groups of right-hand sides (<= 16) are above the
    tolerance take the grid-wide planar Hessenberg solve (hess_cplx_tail_kernel: the CTAs shared
    out among the groups) instead of one CTA per group; with 24 groups left the multi-vector
    kernel keeps them.  Columns zeroed and refined by one step equal W~^-1 b again, to 1e-10 of
    the multi-vector kernel's solution, and the columns already at the tolerance are left bit for
    bit."""
    torch, G = _mods()
    S = 6
    ncols = S * rps
    J = rng(60 + n).standard_normal((n, n)) / np.sqrt(n)
    Jd = dev(J)
    ws = G.lhl(Jd, shift_complex=True)
    g = rng(61)
    sig = g.uniform(-2.0, 0.0, S) + 1j * g.uniform(0.0, 10.0, S)
    tau = -np.ones(S, dtype=complex)
    sh = G.LHLShift(n, S, complex=True)
    G.lhl_shift_batched_(sh, ws, dev(sig), dev(tau))
    B = rng(62).standard_normal((n, ncols)) + 1j * rng(63).standard_normal((n, ncols))
    Bd = dev(B)
    X = Bd.clone()
    G.lhl_ldiv_(X, sh, ws, rhs_per_shift=rps)
    Xh = host(X)
    active = sorted({s * rps + gg * 8 + v for s, gg in groups for v in range(8)
                     if gg * 8 + v < rps})
    X2 = X.clone()
    X2[:, active] = 0
    G.lhl_refine_tol_(X2, Jd, Bd, sh, ws, tol=1e-8, max_steps=1, rhs_per_shift=rps)
    X2h = host(X2)
    for c in range(ncols):
        if c in active:
            assert np.linalg.norm(X2h[:, c] - Xh[:, c]) <= 1e-10 * np.linalg.norm(Xh[:, c]), (n, c)
        else:
            assert bits_equal(X2h[:, c], Xh[:, c]), (n, c)


@pytest.mark.parametrize("T", ["float64", "float32"])
@pytest.mark.parametrize("n", [3, 7, 33, 130, 331, 500])
def test_complex_vectors_on_a_real_shift_like_the_reference(n, T):
    """test/core_tests.jl:38-58's third solve: z = lhl_ldiv!(complex.(b), ws) on a real shift
    (another element type: the generic path) agrees with W \\ b at the element type's tolerance;
    the imaginary part stays zero; and lhl_refine! with complex vectors refines both parts as the
    real refinement does."""
    torch, G = _mods()
    dt = np.float64 if T == "float64" else np.float32
    J = rng(n).standard_normal((n, n)).astype(dt)
    b = rng(n + 7).standard_normal(n).astype(dt)
    ws = G.lhl(dev(J))
    G.lhl_shift_(ws, 1, -0.05)
    W = np.eye(n) - dt(0.05) * J.astype(np.float64)
    z = dev(b.astype(np.complex128 if T == "float64" else np.complex64))
    G.lhl_ldiv_(z, ws)
    zh = host(z).astype(np.complex128)
    xr = np.linalg.solve(W, b.astype(np.float64))
    assert np.linalg.norm(zh.real - xr) <= (1e-9 if T == "float64" else 1e-3) * np.linalg.norm(xr)
    assert np.all(zh.imag == 0)
    if T == "float64":
        Jd = dev(J)
        B = b + 1j * rng(n + 8).standard_normal(n)
        x = G.lhl_ldiv_(dev(B), ws)
        G.lhl_refine_(x, Jd, dev(B), ws, 1)
        xre = G.lhl_ldiv_(dev(B.real.copy()), ws)
        G.lhl_refine_(xre, Jd, dev(B.real.copy()), ws, 1)
        xim = G.lhl_ldiv_(dev(B.imag.copy()), ws)
        G.lhl_refine_(xim, Jd, dev(B.imag.copy()), ws, 1)
        assert np.allclose(host(x), host(xre) + 1j * host(xim), rtol=1e-12, atol=0)
        assert O.bwd(W, host(x), B) < 50 * np.finfo(float).eps
