"""Run-to-run determinism on the device: the same inputs give the same bits twice, for every form's
reduction (the plain blocked and unblocked kernels, the mixed form's exchange between CTAs, the complex
J, the batched kernels), the shift LUs, the solves (whose cooperative L^-1 sweep takes its blocks in
whatever order they become ready) and the refinements.  No sum anywhere depends on timing."""
import numpy as np
import pytest

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


def same_bits(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def run_once(J, B, taus, precision, complex_j=False):
    torch, G = _mods()
    n, S = J.shape[0], len(taus)
    if complex_j:
        ws = G.LHLWorkspace(n, dtype=torch.complex128)
    else:
        ws = G.LHLWorkspace(n, precision)
    G.lhl_reduce_(ws, dev(J), True)
    sh = G.LHLShift(n, S, complex=complex_j)
    sig = torch.ones(S, dtype=torch.float64, device="cuda")
    tau = dev(taus)
    if complex_j:
        sig, tau = sig.to(torch.complex128), tau.to(torch.complex128)
    G.lhl_shift_batched_(sh, ws, sig, tau)
    X = dev(B).clone()
    G.lhl_ldiv_(X, sh, ws)
    x0 = host(X).copy()
    if precision == G.LHL_PREC_MIXED:
        res = G.lhl_refine_gmres_(X, dev(J), dev(B), sh, ws, tol=1e-12, max_cycles=3, restart=3)
    else:
        res = G.lhl_refine_tol_(X, dev(J), dev(B), sh, ws, tol=1e-13, max_steps=3)
    torch.cuda.synchronize()
    ws.check()
    out = [host(ws.factors), host(ws.Ht), host(ws.ipiv), host(ws.scale), host(ws.perm)]
    out += [host(sh.Gt(s)) for s in range(S)] + [host(sh.rdiag(s)) for s in range(S)]
    return out + [x0, host(X), host(res)]


@pytest.mark.parametrize("case", ["plain-300", "plain-700", "mixed-2048", "mixed-400", "complex-300"])
def test_twice_the_same_bits(case):
    torch, G = _mods()
    form, n = case.split("-")
    n = int(n)
    g = np.random.default_rng(n)
    J = g.standard_normal((n, n)) / np.sqrt(n)
    S = 6
    B = g.standard_normal((n, S))
    if form == "complex":
        J = J + 1j * g.standard_normal((n, n)) / np.sqrt(n)
        B = B + 1j * g.standard_normal((n, S))
    taus = -(10.0 ** g.uniform(-3, -0.5, S))
    prec = G.LHL_PREC_MIXED if form == "mixed" else G.LHL_PREC_FP64
    a = run_once(J, B, taus, prec, complex_j=form == "complex")
    b = run_once(J, B, taus, prec, complex_j=form == "complex")
    for k, (u, v) in enumerate(zip(a, b)):
        assert same_bits(u, v), (case, k)


def test_batched_twice_the_same_bits():
    torch, G = _mods()
    ns = [17, 64, 100, 256, 33]
    S, R = 3, 2
    g = np.random.default_rng(5)
    mats = [g.standard_normal((n, n)) - 5 * np.eye(n) for n in ns]
    rhs = [g.standard_normal((n, S * R)) for n in ns]
    outs = []
    for _ in range(2):
        bt = G.LHLBatch(ns, S)
        Jd = torch.as_tensor(bt.pack_matrices(mats)).cuda()
        Bd = torch.as_tensor(bt.pack_rhs(rhs)).cuda()
        Xd = torch.empty_like(Bd)
        sig = torch.ones(len(ns) * S, dtype=torch.float64, device="cuda")
        tau = torch.full((len(ns) * S,), -0.05, dtype=torch.float64, device="cuda")
        G.lhl_reduce_batched_(bt, Jd)
        G.lhl_shift_batched_all_(bt, sig, tau)
        res = G.lhl_solve_batched_(bt, Jd, Bd, Xd, R)
        torch.cuda.synchronize()
        outs.append([host(bt.factors(m)) for m in range(len(ns))] + [host(Xd), host(res)])
    for u, v in zip(*outs):
        assert same_bits(u, v)
