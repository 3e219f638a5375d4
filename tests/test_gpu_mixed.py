"""The mixed form (LHL_PREC_MIXED) on the device: FP32 reduction with FP64-accumulated column
updates, then FP64 shifts, solves and refinement to a tolerance.

Its contract is not bitwise: the factors must be a valid ELMHES similarity of J to FP32
accuracy (Z H Z^-1 = J within 2 eps32 n^1.5, |l| <= 1, valid interchanges), and every shifted
solve must reach relative residual <= 1e-10 after FP64 refinement.  Forward errors are
checked against the FP64 oracle's refined solutions."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

EPS32 = float(np.finfo(np.float32).eps)


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


def as_oracle(ws):
    """The device factorization as an oracle Reduction (for Z, Z^-1 and oracle solves)."""
    n = ws.n
    R = O.Reduction(n)
    R.factors = np.asfortranarray(host(ws.factors))
    R.ipiv = host(ws.ipiv)[: max(n - 2, 0)].copy()
    R.scale = host(ws.scale).copy()
    R.iscale = host(ws.iscale).copy()
    R.perm = host(ws.perm).copy()
    R.iperm = host(ws.iperm).copy()
    R.Ht = np.asfortranarray(host(ws.Ht))
    return R


def mixed(J, balance=True):
    torch, G = _mods()
    ws = G.lhl(dev(J), balance=balance, precision=G.LHL_PREC_MIXED)
    ws.check()
    return ws


def check_similarity(ws, J):
    n = ws.n
    R = as_oracle(ws)
    ip = R.ipiv
    assert all(k + 2 <= ip[k] <= n for k in range(n - 2)), ip
    # perm / iperm (written by the reduction kernel from its row labels) are ipiv's (F:376-387)
    perm = np.arange(1, n + 1)
    for k in range(n - 2):
        p = int(ip[k])
        perm[k + 1], perm[p - 1] = perm[p - 1], perm[k + 1]
    assert np.array_equal(R.perm, perm)
    iperm = np.empty(n, dtype=np.int64)
    iperm[perm - 1] = np.arange(1, n + 1)
    assert np.array_equal(R.iperm, iperm)
    F = R.factors
    if n > 2:
        assert np.abs(np.tril(F, -2)).max() <= 1.0 + 4 * EPS32
    assert np.isfinite(F).all()
    H = np.triu(F, -1)
    err = np.linalg.norm(R.Z() @ H @ R.Zinv() - J) / np.linalg.norm(J)
    assert err <= 2.0 * EPS32 * max(n, 4) ** 1.5, err
    return R


@pytest.mark.parametrize("n", [3, 4, 5, 17, 64, 130, 400, 777, 1030])
@pytest.mark.parametrize("balance", [True, False])
def test_mixed_reduction_is_a_similarity(n, balance):
    J = rng(n).standard_normal((n, n))
    ws = mixed(J, balance)
    check_similarity(ws, J)
    # balancing is the plain form's, in FP64: D bit-identical to the oracle's
    R64 = O.reduce(J, balance=balance)
    assert np.array_equal(host(ws.scale), R64.scale)


def test_mixed_ties_zeros_and_zero_columns():
    """rand(-1:1) entries (ties, exact zeros) and whole zero columns (zero pivots, F:470)."""
    n = 150
    J = rng(9).integers(-1, 2, (n, n)).astype(float)
    check_similarity(mixed(J), J)
    J2 = rng(10).standard_normal((n, n))
    J2[:, :3] = 0.0
    J2[:, 70] = 0.0
    check_similarity(mixed(J2, balance=False), J2)


def test_mixed_graded_matrix():
    n = 300
    J = np.diag(10.0 ** np.linspace(-4, 4, n)) @ rng(3).standard_normal((n, n)) @ np.diag(10.0 ** np.linspace(4, -4, n))
    ws = mixed(J)
    R64 = O.reduce(J)
    assert np.array_equal(host(ws.scale), R64.scale)
    check_similarity(ws, J)


def _solve_to_tol(ws, Jd, sig, tau, B, tol=1e-10, max_steps=12):
    torch, G = _mods()
    n = ws.n
    S = len(sig)
    sh = G.LHLShift(n, S)
    G.lhl_shift_batched_(sh, ws, dev(sig), dev(tau))
    Bd = dev(B)
    X = Bd.clone()
    G.lhl_ldiv_(X, sh, ws, rhs_per_shift=B.shape[1] // S)
    res = G.lhl_refine_tol_(X, Jd, Bd, sh, ws, tol=tol, max_steps=max_steps, rhs_per_shift=B.shape[1] // S)
    return host(X), host(res), sh


def test_mixed_config1_reaches_1e10():
    """Config 1 through the mixed form: residual <= 1e-10 (checked on the host too), forward
    error against the FP64 oracle's refined solution."""
    torch, G = _mods()
    from lhl_gpu import configs
    c = configs.config1()
    J = c["J"]
    ws = mixed(J)
    X, res, _ = _solve_to_tol(ws, dev(J), c["sigma"], c["tau"], c["B"])
    assert (res <= 1e-10).all(), res
    R64 = O.reduce(J)
    for s in range(3):
        W = c["sigma"][s] * np.eye(c["n"]) + c["tau"][s] * J
        b = c["B"][:, s]
        assert np.linalg.norm(b - W @ X[:, s]) <= 1.0001e-10 * np.linalg.norm(b)
        So = O.shift(R64, c["sigma"][s], c["tau"][s])
        xo = O.refine(R64, So, J, b, O.ldiv(R64, So, b), 1)
        assert np.linalg.norm(X[:, s] - xo) <= 1e-8 * np.linalg.norm(xo)


def test_mixed_config2_all_shifts_reach_1e10():
    """Config 2 (n = 2048, 64 shifts (1, -g), g log-uniform in [1e-4, 1e-1]) through the mixed
    form: every shift reaches relative residual <= 1e-10.  Most need 1-4 refinement steps; the
    slowest (g = 0.0354, I - g J close to singular) converges at about 0.2 per step."""
    torch, G = _mods()
    from lhl_gpu import configs
    c = configs.config2()
    J = c["J"]
    Jd = dev(J)
    ws = G.lhl(Jd, precision=G.LHL_PREC_MIXED)
    ws.check()
    X, res, _ = _solve_to_tol(ws, Jd, c["sigma"], c["tau"], c["B"], max_steps=24)
    assert (res <= 1e-10).all(), res
    for s in (0, int(np.argmax(-c["tau"])), 48):
        W = c["sigma"][s] * np.eye(c["n"]) + c["tau"][s] * J
        b = c["B"][:, s]
        assert np.linalg.norm(b - W @ X[:, s]) <= 1.0001e-10 * np.linalg.norm(b)


@pytest.mark.parametrize("n", [3, 4, 5, 17, 18, 40, 100, 131, 300, 600])
@pytest.mark.parametrize("balance", [True, False])
def test_panel_delayed_kernel_is_a_similarity(n, balance):
    """The panel-delayed FP32 kernel (the one the mixed form uses when its rows no longer fit in
    shared memory), forced at small orders through the test hook: a valid ELMHES similarity of J
    to FP32 accuracy, with panels of 16 steps that end inside and at the end of the reduction;
    and the eager FP32 kernel's pivots over the early steps (late steps pick among near-ties
    that the two kernels' roundings may order differently)."""
    torch, G = _mods()
    J = rng(300 + n).standard_normal((n, n))
    ws = G.LHLWorkspace(n, G.LHL_PREC_MIXED)
    ws.set_mixed_kernel(2)
    G.lhl_reduce_(ws, dev(J), balance)
    ws.check()
    check_similarity(ws, J)
    we = G.LHLWorkspace(n, G.LHL_PREC_MIXED)
    we.set_mixed_kernel(1)
    G.lhl_reduce_(we, dev(J), balance)
    we.check()
    m = min(n - 2, 120)
    assert np.array_equal(host(ws.ipiv)[:m], host(we.ipiv)[:m])


def test_mixed_rows_in_global_memory():
    """n = 2600: the FP32 rows no longer fit in shared memory (global-memory rows)."""
    torch, G = _mods()
    n = 2600
    J = rng(26).standard_normal((n, n))
    Jd = dev(J)
    ws = G.lhl(Jd, precision=G.LHL_PREC_MIXED)
    ws.check()
    ip = host(ws.ipiv)
    assert all(k + 2 <= ip[k] <= n for k in range(n - 2))
    sig = np.ones(6)
    tau = -np.array([1e-4, 1e-3, 3e-3, 1e-2, 3e-2, 1e-1])
    B = rng(27).standard_normal((n, 6))
    X, res, _ = _solve_to_tol(ws, Jd, sig, tau, B, max_steps=24)
    assert (res <= 1e-10).all(), res


def test_mixed_refine_tol_matches_fixed_steps_when_tol_zero():
    """lhl_refine_tol with tol = 0 performs the same updates as lhl_refine with that many steps."""
    torch, G = _mods()
    n = 200
    J = rng(4).standard_normal((n, n))
    Jd = dev(J)
    ws = mixed(J)
    sh = G.LHLShift(n, 2)
    G.lhl_shift_batched_(sh, ws, dev(np.ones(2)), dev(np.array([-0.01, -0.05])))
    B = dev(rng(5).standard_normal((n, 2)))
    X1 = B.clone()
    G.lhl_ldiv_(X1, sh, ws)
    X2 = X1.clone()
    G.lhl_refine_(X1, Jd, B, sh, ws, 3)
    G.lhl_refine_tol_(X2, Jd, B, sh, ws, tol=0.0, max_steps=3)
    assert np.array_equal(host(X1), host(X2))


def test_mixed_exchange_timeout_reports_and_recovers():
    """A wait limit of 1 ns on the per-step exchange: LHL_ERR_TIMEOUT, then a correct rerun."""
    torch, G = _mods()
    n = 600
    J = rng(5).standard_normal((n, n))
    ws = G.LHLWorkspace(n, G.LHL_PREC_MIXED)
    ws.set_barrier_limit_ns(1)
    G.lhl_reduce_(ws, dev(J), True)
    with pytest.raises(G.LHLDeviceError):
        ws.check()
    ws.set_barrier_limit_ns(2_000_000_000)
    G.lhl_reduce_(ws, dev(J), True)
    ws.check()
    check_similarity(ws, J)
