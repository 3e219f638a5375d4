"""Parity of the CUDA path with the CPU oracle, through the library's C ABI (via the
lhl_gpu host mirror).  Plain FP64 form: reduction (pivots, factors, Ht, D) and shift LU
(Gt, swap, rdiag, info) bit for bit; solves within the reference tests' tolerances and
the 1e-12 relative residual after one refinement step."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _mods():
    import torch
    import lhl_gpu as G
    return torch, G


def dev(a):
    torch, _ = _mods()
    t = torch.as_tensor(np.asfortranarray(a)).cuda()
    return t


def host(t):
    return t.detach().cpu().numpy()


def bits_equal(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return a.shape == b.shape and np.array_equal(a.view(np.int64), b.view(np.int64))


def rng(seed):
    return np.random.default_rng(seed)


REDUCE_SIZES = [1, 2, 3, 4, 5, 7, 8, 9, 17, 31, 64, 80, 128, 200, 301, 400, 499, 500, 501, 520, 600, 777, 1030]


@pytest.mark.parametrize("n", REDUCE_SIZES)
@pytest.mark.parametrize("balance", [True, False])
def test_reduce_bitexact(n, balance):
    torch, G = _mods()
    J = rng(n).standard_normal((n, n))
    R = O.reduce(J, balance=balance)
    ws = G.lhl(dev(J), balance=balance)
    ws.check()
    assert np.array_equal(host(ws.ipiv), R.ipiv)
    assert bits_equal(host(ws.scale), R.scale)
    assert bits_equal(host(ws.factors), R.factors)
    assert bits_equal(host(ws.Ht), R.Ht)
    assert np.array_equal(host(ws.perm), R.perm) and np.array_equal(host(ws.iperm), R.iperm)


@pytest.mark.parametrize("n", [150, 520])
def test_reduce_ties_and_zeros_bitexact(n):
    """rand(-1:1) matrices: exact zeros, ties in the pivot search, pulled columns."""
    torch, G = _mods()
    J = rng(9).integers(-1, 2, (n, n)).astype(float)
    R = O.reduce(J)
    ws = G.lhl(dev(J))
    ws.check()
    assert np.array_equal(host(ws.ipiv), R.ipiv)
    assert bits_equal(host(ws.factors), R.factors)


def test_reduce_graded_balancing_bitexact():
    """A graded matrix that balancing rescales: D, then the blocked reduction."""
    torch, G = _mods()
    n = 600
    J = np.diag(10.0 ** np.linspace(-6, 6, n)) @ rng(3).standard_normal((n, n)) @ np.diag(10.0 ** np.linspace(6, -6, n))
    R = O.reduce(J)
    assert (R.scale != 1.0).any()
    ws = G.lhl(dev(J))
    ws.check()
    assert bits_equal(host(ws.scale), R.scale)
    assert np.array_equal(host(ws.ipiv), R.ipiv)
    assert bits_equal(host(ws.factors), R.factors)


SHIFTS = [(1.0, -0.1), (0.0, 1.0), (1.0, -3.0), (2.0, 0.0), (0.0, 0.0)]


@pytest.mark.parametrize("n", list(range(1, 301)) + [511, 512, 513, 520, 640, 768, 1000, 1024, 2048])
@pytest.mark.parametrize("tie", [False, True])
def test_shift_bitexact(n, tie):
    """test/core_tests.jl:192-212 on the device: the shift LU state against the oracle's
    restatement of `_lhl_shift_ref!`, bit for bit, including zero pivots, at the reference
    test's orders (1:300 and 511 ... 1024) plus config 2's 2048."""
    torch, G = _mods()
    g = rng(31 + n + 1000 * tie)
    J = g.integers(-2, 3, (n, n)).astype(float) if tie else g.standard_normal((n, n))
    R = O.reduce(J)
    ws = G.LHLWorkspace(n)
    ws.Ht.copy_(dev(R.Ht))
    for s, t in SHIFTS:
        with np.errstate(divide="ignore", invalid="ignore"):
            S = O.shift(R, s, t)
        G.lhl_shift_(ws, s, t)
        torch.cuda.synchronize()
        Gt = host(ws.shift.Gt())
        U = Gt[:n, :n].T[np.triu_indices(n)]  # Gt[j, k] for k = 0.., j = k.. (column order)
        l = Gt[np.arange(n - 1), np.arange(1, n)]
        U0, l0, sw0, rd0, info0 = S.state()
        assert bits_equal(U, U0), (n, s, t)
        assert bits_equal(l, l0)
        assert np.array_equal(host(ws.shift.swap()), sw0)
        assert bits_equal(host(ws.shift.rdiag()), rd0)
        assert ws.shift.info == info0


@pytest.mark.parametrize("n", [1, 2, 3, 5, 40, 129, 260, 400, 600])
def test_shifted_solves(n):
    """test/core_tests.jl:23-36 on the device: solves against a dense LU, rtol 1e-9, and the
    backward error bound of :38-59; agreement with the oracle's solve."""
    torch, G = _mods()
    J = rng(n).standard_normal((n, n))
    b = rng(n + 7).standard_normal(n)
    R = O.reduce(J)
    ws = G.lhl(dev(J))
    for s, t in ((1.0, 0.0), (1.0, -1e-8), (1.0, -0.05), (1.0, 1.7), (0.0, 1.0), (-3.0, 2.0)):
        W = s * np.eye(n) + t * J
        if np.linalg.matrix_rank(W) < n:
            continue
        G.lhl_shift_(ws, s, t)
        x = host(G.lhl_ldiv_(dev(b), ws))
        xr = np.linalg.solve(W, b)
        assert np.linalg.norm(x - xr) <= 1e-9 * np.linalg.norm(xr)
        xo = O.ldiv(R, O.shift(R, s, t), b)
        assert np.linalg.norm(x - xo) <= 1e-9 * np.linalg.norm(xo)
        eps = np.finfo(float).eps
        # the reference bounds the raw solve's backward error for (1, -0.05) at n <= 500
        # (test/core_tests.jl:38-59); for every shift, the device solve's backward error
        # stays within a small factor of the oracle's (their summation orders differ)
        if (s, t) == (1.0, -0.05) and n <= 500:
            assert O.bwd(W, x, b) < 50 * eps
        assert O.bwd(W, x, b) <= max(4 * O.bwd(W, xo, b), 50 * eps)


def test_config1_refined_residual():
    """Config 1: J 400x400, three shifts (1, -g), one ldiv + one refinement step each;
    relative residual <= 1e-12, and the solution agrees with the oracle's."""
    torch, G = _mods()
    from lhl_gpu import configs
    c = configs.config1()
    n = c["n"]
    R = O.reduce(c["J"])
    Jd = dev(c["J"])
    ws = G.lhl(Jd)
    ws.check()
    assert np.array_equal(host(ws.ipiv), R.ipiv)
    assert bits_equal(host(ws.factors), R.factors)
    sh = G.LHLShift(n, 3)
    G.lhl_shift_batched_(sh, ws, dev(c["sigma"]), dev(c["tau"]))
    B = dev(c["B"])
    X = B.clone()
    G.lhl_ldiv_(X, sh, ws)
    G.lhl_refine_(X, Jd, B, sh, ws, 1)
    res = host(G.residual_norms(sh, Jd, B, X))
    assert (res <= 1e-12).all(), res
    for s in range(3):
        So = O.shift(R, c["sigma"][s], c["tau"][s])
        xo = O.refine(R, So, c["J"], c["B"][:, s], O.ldiv(R, So, c["B"][:, s]), 1)
        x = host(X[:, s])
        assert np.linalg.norm(x - xo) <= 1e-11 * np.linalg.norm(xo)


@pytest.mark.parametrize("n", [50, 700])
def test_batched_shifts_match_single(n):
    torch, G = _mods()
    J = rng(7 + n).standard_normal((n, n))
    ws = G.lhl(dev(J))
    sig = np.ones(6)
    tau = -np.array([1e-4, 1e-3, 0.01, 0.05, 0.1, 0.3])
    sh = G.LHLShift(n, 6)
    G.lhl_shift_batched_(sh, ws, dev(sig), dev(tau))
    B = rng(8).standard_normal((n, 12))
    X = dev(B)
    G.lhl_ldiv_(X, sh, ws, rhs_per_shift=2)
    Xh = host(X)
    for s in range(6):
        G.lhl_shift_(ws, sig[s], tau[s])
        assert bits_equal(host(ws.shift.Gt()), host(sh.Gt(s)))
        for r in range(2):
            x1 = host(G.lhl_ldiv_(dev(B[:, 2 * s + r]), ws))
            assert bits_equal(x1, Xh[:, 2 * s + r])


@pytest.mark.parametrize("n", [3, 37, 600])
def test_applyZ_roundtrip(n):
    """test/core_tests.jl:5-21 and test/Interface/public_interface.jl:15-19."""
    torch, G = _mods()
    J = rng(n).standard_normal((n, n))
    ws = G.lhl(dev(J))
    x0 = rng(1).standard_normal(n)
    x = dev(x0)
    assert G.applyZ_(x, ws) is x
    assert G.applyZinv_(x, ws) is x
    assert np.allclose(host(x), x0, rtol=1e-10, atol=1e-12)
    R = O.reduce(J)
    assert np.allclose(host(G.applyZ_(dev(x0), ws)), O.apply_z(R, x0), rtol=1e-12, atol=1e-13)


def test_singular_shift_reported():
    torch, G = _mods()
    ws = G.lhl(dev(np.array([[1.0, 0.0], [0.0, 2.0]])))
    G.lhl_shift_(ws, 1.0, -1.0)
    assert ws.shift.info != 0


def test_errors_mirror_the_reference():
    torch, G = _mods()
    ws = G.lhl(dev(rng(1).standard_normal((6, 6))))
    with pytest.raises(G.DimensionMismatch):
        G.lhl_ldiv_(dev(np.zeros(7)), ws)
    with pytest.raises(G.DimensionMismatch):
        G.applyZ_(dev(np.zeros(5)), ws)
    with pytest.raises(G.ArgumentError):
        G.lhl_shift_(ws, 1.0, -0.3j)
    sh = G.LHLShift(5)
    with pytest.raises(G.DimensionMismatch):
        G.lhl_ldiv_(dev(np.zeros(6)), sh, ws)
    with pytest.raises(G.DimensionMismatch):
        G.lhl(dev(np.zeros((3, 4))))
    # mutating calls return their first argument (test/Interface/public_interface.jl:7-18)
    assert G.lhl_shift_(ws, 1.0, -0.1) is ws
    x = dev(np.ones(6))
    assert G.lhl_ldiv_(x, ws) is x


def test_workspace_and_shift_resize_like_the_reference():
    """test/core_tests.jl:107-112: lhl! onto a workspace of another order resizes it; :306-310:
    lhl_shift! resizes a shift object to the workspace.  Both then solve like fresh objects."""
    torch, G = _mods()
    n = 40
    ws = G.lhl(dev(rng(4).standard_normal((n, n))))
    J3 = rng(6).standard_normal((2 * n, 2 * n))
    assert G.lhl_(ws, dev(J3)) is ws and ws.n == 2 * n and ws.shift.n == 2 * n
    R = O.reduce(J3)
    assert np.array_equal(host(ws.ipiv), R.ipiv) and bits_equal(host(ws.factors), R.factors)
    b3 = rng(7).standard_normal(2 * n)
    G.lhl_shift_(ws, 1.0, -0.3)
    x = host(G.lhl_ldiv_(dev(b3), ws))
    xr = np.linalg.solve(np.eye(2 * n) - 0.3 * J3, b3)
    assert np.linalg.norm(x - xr) <= 1e-9 * np.linalg.norm(xr)  # isapprox, rtol = 1e-9
    sh = G.LHLShift(n, 1, complex=True)
    assert G.lhl_shift_(sh, ws, 1.0, -0.3j) is sh and sh.n == 2 * n
    b2 = rng(8).standard_normal(2 * n) + 1j * rng(9).standard_normal(2 * n)
    xc = host(G.lhl_ldiv_(dev(b2), sh, ws))
    xr = np.linalg.solve(np.eye(2 * n) - 0.3j * J3, b2)
    assert np.linalg.norm(xc - xr) <= 1e-9 * np.linalg.norm(xr)


def _wilkinson(n):
    J = -np.tril(np.ones((n, n)), -1) + np.eye(n)
    J[:, n - 1] = 1.0
    return J


@pytest.mark.parametrize("family", ["randn", "wilkinson", "graded"])
def test_pivoting_is_what_makes_it_work(family):
    """test/core_tests.jl:337-363 on the device: |l| <= 1 + eps on the families that break an
    unpivoted reduction, and one refinement step with the caller's W takes the reference's
    backward error below 1e-13 (the oracle reaches about 1e-16 on these)."""
    torch, G = _mods()
    n = 100
    if family == "randn":
        J = rng(1).standard_normal((n, n))
    elif family == "wilkinson":
        J = _wilkinson(n)
    else:
        J = np.diag(10.0 ** np.linspace(-8, 8, n)) @ rng(3).standard_normal((n, n)) @ \
            np.diag(10.0 ** np.linspace(8, -8, n))
    b = rng(42).standard_normal(n)
    ws = G.lhl(dev(J))
    assert np.abs(np.tril(host(ws.factors), -2)).max() <= 1 + np.finfo(float).eps
    for g in (1e-3, 1.0, 1e3):
        G.lhl_shift_(ws, 1.0, -g)
        if ws.info != 0:
            continue
        W = np.eye(n) - g * J
        x = G.lhl_ldiv_(dev(b), ws)
        G.lhl_refine_system_(x, dev(W), dev(b), ws, 1)
        assert O.bwd(W, host(x), b) < 1e-13, (family, g)


def test_refinement_recovers_backward_error_where_kappa_Z_is_enormous():
    """test/core_tests.jl:365-380 on the device: strictly upper triangular J with a 1e-8 corner,
    every pivot near zero; one refinement step does not lose and ends below 1e-13 (the oracle:
    6.5e-12 raw, 2.8e-17 refined)."""
    torch, G = _mods()
    n = 60
    J = np.triu(rng(17).standard_normal((n, n)), 1)
    J[n - 1, 0] = 1e-8
    b = rng(18).standard_normal(n)
    W = np.eye(n) - 0.5 * J
    ws = G.lhl(dev(J))
    G.lhl_shift_(ws, 1.0, -0.5)
    raw = G.lhl_ldiv_(dev(b), ws)
    refined = raw.clone()
    G.lhl_refine_system_(refined, dev(W), dev(b), ws, 1)
    assert O.bwd(W, host(refined), b) <= O.bwd(W, host(raw), b)
    assert O.bwd(W, host(refined), b) < 1e-13


def test_barrier_timeout_reports_and_recovers():
    """A grid-barrier wait limit of 1 ns expires: the reduction returns LHL_ERR_TIMEOUT
    instead of hanging, and the same workspace then reduces correctly."""
    torch, G = _mods()
    n = 600
    J = rng(5).standard_normal((n, n))
    ws = G.LHLWorkspace(n)
    ws.set_barrier_limit_ns(1)
    G.lhl_reduce_(ws, dev(J), True)
    with pytest.raises(G.LHLDeviceError):
        ws.check()
    ws.set_barrier_limit_ns(2_000_000_000)
    G.lhl_reduce_(ws, dev(J), True)
    ws.check()
    R = O.reduce(J)
    assert np.array_equal(host(ws.ipiv), R.ipiv)
    assert bits_equal(host(ws.factors), R.factors)


@pytest.mark.parametrize("n", [300, 600])
def test_nan_and_inf_inputs_end_with_valid_pivots(n):
    """A J holding a NaN and an Inf: the reduction (unblocked at n = 300, blocked with TMA GEMV
    tiles at n = 600) ends without a timeout and leaves only valid interchanges, and the shift
    and solve that follow run (their values are not finite).  The wait limit is short, so a stall
    would end as LHL_ERR_TIMEOUT rather than hold the GPU.  Balancing ends on the infinite norm
    where the reference's _lhl_balance! (F:313-320) would not."""
    torch, G = _mods()
    rng = np.random.default_rng(n)
    J = rng.standard_normal((n, n))
    J[5, 7] = np.nan
    J[n - 3, 2] = np.inf
    ws = G.LHLWorkspace(n, G.LHL_PREC_FP64)
    ws.set_barrier_limit_ns(500_000_000)
    G.lhl_reduce_(ws, dev(J), True)
    ws.check()
    ip = host(ws.ipiv)[: n - 2]
    assert ((ip >= np.arange(2, n)) & (ip <= n)).all()
    G.lhl_shift_(ws, 1.0, -0.05)
    x = G.lhl_ldiv_(torch.ones(n, dtype=torch.float64, device="cuda"), ws)
    torch.cuda.synchronize()
    assert x.shape == (n,)
