"""lhl_refine_gmres (GMRES-IR) on the device through the C ABI.

Against the oracle's restatement (oracle.gmres_ir) on the device's own factors (the mixed
form's FP32 reduction: a weak preconditioner, so that cycles take several Arnoldi steps);
on a config-2-shaped problem every column reaches 1e-10; converged columns are left bit-for-bit alone; host_check only changes when the
host stops launching; complex shifts (GMRES on the realified system) against the oracle and
on a config-5-shaped sweep; the error cases."""
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
    return torch.as_tensor(np.asfortranarray(a)).cuda()


def host(t):
    return t.detach().cpu().numpy()


def rng(seed):
    return np.random.default_rng(seed)


def as_oracle(ws):
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


def problem(n, S, rps, seed, precision):
    torch, G = _mods()
    J = rng(seed).standard_normal((n, n))
    g = 10.0 ** rng(seed + 1).uniform(-3.0, -1.0, S)
    Jd = dev(J)
    ws = G.lhl(Jd, precision=precision)
    ws.check()
    sh = G.LHLShift(n, S)
    G.lhl_shift_batched_(sh, ws, dev(np.ones(S)), dev(-g))
    B = rng(seed + 2).standard_normal((n, S * rps))
    return J, g, Jd, ws, sh, B


@pytest.mark.parametrize("n", [1, 2, 3, 37, 300, 513, 1030])
def test_gmres_matches_the_oracle(n):
    """One cycle of 3 Arnoldi steps (tol = 0: no early stop) from x = 0, on the mixed form's
    factors, against oracle.gmres_ir with the same factors and shift LUs."""
    torch, G = _mods()
    S, rps = 3, 2
    J, g, Jd, ws, sh, B = problem(n, S, rps, 10 + n, G.LHL_PREC_MIXED)
    X = dev(np.zeros((n, S * rps)))
    res = host(G.lhl_refine_gmres_(X, Jd, dev(B), sh, ws, tol=0.0, max_cycles=1, restart=3,
                                   rhs_per_shift=rps))
    Xh = host(X)
    R = as_oracle(ws)
    for c in range(S * rps):
        s = c // rps
        W = np.eye(n) - g[s] * J
        So = O.shift(R, 1.0, -g[s])
        xo, relo, _ = O.gmres_ir(lambda v: W @ v, lambda v: O.ldiv(R, So, v), B[:, c], np.zeros(n), 0.0,
                                 max_cycles=1, restart=3)
        assert np.linalg.norm(Xh[:, c] - xo) <= 1e-8 * np.linalg.norm(xo), c
        # the reported residual is the device x's own; the oracle's is a small difference of
        # x-sized terms, which x agreeing to 1e-8 can move by a few per cent
        rh = np.linalg.norm(B[:, c] - W @ Xh[:, c]) / np.linalg.norm(B[:, c])
        assert abs(res[c] - rh) <= 1e-3 * rh + 1e-12, (c, res[c], rh)  # 1e-12: the FP64 floor
        assert abs(res[c] - relo) <= 0.1 * relo + 1e-12, (c, res[c], relo)


def test_gmres_config2_shaped_mixed():
    """Config 2's shapes (n = 2048, 64 shifts (1, -g), g log-uniform in [1e-4, 1e-1], one
    right-hand side each) on the mixed form: every column at <= 1e-10 after at most 3 cycles
    of GMRES(6)."""
    torch, G = _mods()
    from lhl_gpu import configs
    c = configs.config2()
    n, S = c["n"], 64
    Jd = dev(c["J"])
    ws = G.lhl(Jd, precision=G.LHL_PREC_MIXED)
    ws.check()
    sh = G.LHLShift(n, S)
    G.lhl_shift_batched_(sh, ws, dev(c["sigma"]), dev(c["tau"]))
    Bd = dev(c["B"])
    X0 = Bd.clone()
    G.lhl_ldiv_(X0, sh, ws)
    X = X0.clone()
    res = host(G.lhl_refine_gmres_(X, Jd, Bd, sh, ws, tol=1e-10, max_cycles=3, restart=6))
    assert (res <= 1e-10).all(), res.max()
    Xh = host(X)
    for col in (0, 17, 48, 63):
        W = c["sigma"][col] * np.eye(n) + c["tau"][col] * c["J"]
        b = c["B"][:, col]
        assert np.linalg.norm(b - W @ Xh[:, col]) <= 1.0001e-10 * np.linalg.norm(b)
    ws.check()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gmres_leaves_converged_columns_alone(precision):
    torch, G = _mods()
    n, S, rps = 400, 4, 2
    prec = G.LHL_PREC_MIXED if precision == "mixed" else G.LHL_PREC_FP64
    J, g, Jd, ws, sh, B = problem(n, S, rps, 3, prec)
    Bd = dev(B)
    X = Bd.clone()
    G.lhl_ldiv_(X, sh, ws, rhs_per_shift=rps)
    G.lhl_refine_tol_(X, Jd, Bd, sh, ws, tol=1e-13, max_steps=8, rhs_per_shift=rps)
    Xh = host(X).copy()
    Xh[:, 1::2] = 0.0  # every other column starts from zero
    X = dev(Xh)
    res = host(G.lhl_refine_gmres_(X, Jd, Bd, sh, ws, tol=1e-10, max_cycles=4, restart=6, rhs_per_shift=rps))
    assert (res <= 1e-10).all()
    out = host(X)
    assert np.array_equal(out[:, 0::2].view(np.int64), Xh[:, 0::2].view(np.int64))
    assert not np.array_equal(out[:, 1::2], Xh[:, 1::2])


def test_gmres_host_check_changes_nothing_but_the_launches():
    torch, G = _mods()
    n, S = 700, 5
    J, g, Jd, ws, sh, B = problem(n, S, 1, 7, G.LHL_PREC_MIXED)
    Bd = dev(B)
    X0 = Bd.clone()
    G.lhl_ldiv_(X0, sh, ws)
    Xa, Xb = X0.clone(), X0.clone()
    ra = host(G.lhl_refine_gmres_(Xa, Jd, Bd, sh, ws, tol=1e-10, max_cycles=5, restart=4, host_check=True))
    rb = host(G.lhl_refine_gmres_(Xb, Jd, Bd, sh, ws, tol=1e-10, max_cycles=5, restart=4, host_check=False))
    assert (ra <= 1e-10).all()
    assert np.array_equal(host(Xa).view(np.int64), host(Xb).view(np.int64))
    assert np.array_equal(ra.view(np.int64), rb.view(np.int64))


def test_gmres_zero_cycles_only_measures():
    torch, G = _mods()
    n, S = 90, 3
    J, g, Jd, ws, sh, B = problem(n, S, 1, 8, G.LHL_PREC_FP64)
    Bd = dev(B)
    X = dev(rng(9).standard_normal((n, S)))
    X0 = host(X).copy()
    res = host(G.lhl_refine_gmres_(X, Jd, Bd, sh, ws, tol=1e-10, max_cycles=0))
    assert np.array_equal(host(X), X0)
    ref = host(G.residual_norms(sh, Jd, Bd, X))
    assert np.allclose(res, ref, rtol=1e-14, atol=0)


def test_gmres_errors():
    torch, G = _mods()
    n = 8
    J, g, Jd, ws, sh, B = problem(n, 2, 1, 11, G.LHL_PREC_FP64)
    Bd = dev(B)
    X = Bd.clone()
    for restart in (0, 33):
        with pytest.raises(G.ArgumentError):
            G.lhl_refine_gmres_(X, Jd, Bd, sh, ws, restart=restart)
    with pytest.raises(G.ArgumentError):
        G.lhl_refine_gmres_(X, Jd, Bd, sh, ws, max_cycles=-1)
    with pytest.raises(G.DimensionMismatch):
        G.lhl_refine_gmres_(X, Jd, dev(B[:, :1]), sh, ws)
    with pytest.raises(G.DimensionMismatch):  # 3 columns, one per shift, 2 shifts
        G.lhl_refine_gmres_(dev(np.ones((n, 3))), Jd, dev(np.ones((n, 3))), sh, ws)
    with pytest.raises(G.ArgumentError):  # complex vectors with a real shift batch
        G.lhl_refine_gmres_(dev(np.ones(n) + 0j), Jd, dev(np.ones(n) + 0j), sh, ws)
    wc = G.lhl(Jd, shift_complex=True)
    shc = G.LHLShift(n, 1, complex=True)
    G.lhl_shift_batched_(shc, wc, dev(np.array([1.0 + 1j])), dev(np.array([-0.1 + 0j])))
    with pytest.raises(G.ArgumentError):  # a real x cannot hold a complex shift's solution
        G.lhl_refine_gmres_(dev(np.ones(n)), Jd, dev(np.ones(n)), shc, wc)


def cplx_problem(n, S, rps, seed, precision):
    """Config 5's form: J ~ N(0,1)/sqrt(n), shifts (s, -1) with s = a + ib, a in [-2, 0],
    b in [0, 10], complex N(0,1) right-hand sides."""
    torch, G = _mods()
    J = rng(seed).standard_normal((n, n)) / np.sqrt(n)
    g = rng(seed + 1)
    s = g.uniform(-2.0, 0.0, S) + 1j * g.uniform(0.0, 10.0, S)
    Jd = dev(J)
    ws = G.lhl(Jd, precision=precision, shift_complex=True)
    ws.check()
    sh = G.LHLShift(n, S, complex=True)
    G.lhl_shift_batched_(sh, ws, dev(s), dev(-np.ones(S, dtype=complex)))
    g2 = rng(seed + 2)
    B = g2.standard_normal((n, S * rps)) + 1j * g2.standard_normal((n, S * rps))
    return J, s, Jd, ws, sh, B


@pytest.mark.parametrize("n", [3, 129, 600])
def test_gmres_complex_matches_the_oracle(n):
    """Complex shifts: one cycle of 3 Arnoldi steps of the realified GMRES from x = 0, on the
    mixed form's factors, against oracle.gmres_ir with the same factors and shift LUs."""
    torch, G = _mods()
    S, rps = 2, 2
    J, s, Jd, ws, sh, B = cplx_problem(n, S, rps, 40 + n, G.LHL_PREC_MIXED)
    X = dev(np.zeros((n, S * rps), dtype=complex))
    res = host(G.lhl_refine_gmres_(X, Jd, dev(B), sh, ws, tol=0.0, max_cycles=1, restart=3,
                                   rhs_per_shift=rps))
    Xh = host(X)
    R = as_oracle(ws)
    for c in range(S * rps):
        W = s[c // rps] * np.eye(n) - J
        So = O.shift_complex(R, s[c // rps], -1.0)
        xo, relo, _ = O.gmres_ir(lambda v: W @ v, lambda v: O.ldiv_complex(R, So, v), B[:, c],
                                 np.zeros(n, dtype=complex), 0.0, max_cycles=1, restart=3)
        assert np.linalg.norm(Xh[:, c] - xo) <= 1e-8 * np.linalg.norm(xo), c
        rh = np.linalg.norm(B[:, c] - W @ Xh[:, c]) / np.linalg.norm(B[:, c])
        assert abs(res[c] - rh) <= 1e-3 * rh + 1e-12, (c, res[c], rh)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gmres_complex_resolvent_sweep(precision):
    """Config 5's shape at n = 1024 (8 complex shifts x 4 right-hand sides): every column at
    <= 1e-10 by GMRES-IR, checked again on the host."""
    torch, G = _mods()
    n, S, rps = 1024, 8, 4
    prec = G.LHL_PREC_MIXED if precision == "mixed" else G.LHL_PREC_FP64
    J, s, Jd, ws, sh, B = cplx_problem(n, S, rps, 10, prec)
    Bd = dev(B)
    X = Bd.clone()
    G.lhl_ldiv_(X, sh, ws, rhs_per_shift=rps)
    res = host(G.lhl_refine_gmres_(X, Jd, Bd, sh, ws, tol=1e-10, max_cycles=4, restart=6, rhs_per_shift=rps))
    assert (res <= 1e-10).all(), res.max()
    Xh = host(X)
    for c in (0, S * rps - 1):
        W = s[c // rps] * np.eye(n) - J
        assert np.linalg.norm(B[:, c] - W @ Xh[:, c]) <= 1.0001e-10 * np.linalg.norm(B[:, c])


def test_gmres_stagnated_columns_stop():
    """tol below FP64's reach: every column stops refining once a cycle fails to halve its
    residual, so 12 and 40 allowed cycles give bit-identical results, with or without the host
    check, at a residual near the FP64 floor."""
    torch, G = _mods()
    n, S = 600, 4
    J, g, Jd, ws, sh, B = problem(n, S, 1, 21, G.LHL_PREC_MIXED)
    Bd = dev(B)
    X0 = Bd.clone()
    G.lhl_ldiv_(X0, sh, ws)
    outs = []
    for cyc, hc in ((12, True), (40, True), (40, False)):
        X = X0.clone()
        r = host(G.lhl_refine_gmres_(X, Jd, Bd, sh, ws, tol=1e-30, max_cycles=cyc, restart=4, host_check=hc))
        outs.append((host(X), r))
    for X, r in outs[1:]:
        assert np.array_equal(X.view(np.int64), outs[0][0].view(np.int64))
        assert np.array_equal(r.view(np.int64), outs[0][1].view(np.int64))
    assert (outs[0][1] < 1e-12).all()
