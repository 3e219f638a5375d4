"""The tuner's device side: every shift-LU launch shape gives the bits of the default shape
(real and complex shifts), and a tuning pass on a small workload picks choices that reach the
tolerance and keeps them in the cache."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mods():
    import torch
    import lhl_gpu as G
    from lhl_gpu import tune as T
    return torch, G, T


def _state(torch, sh, count, n):
    out = []
    for s in range(count):
        G_ = sh.Gt(s)
        out.append(G_.contiguous().cpu().numpy().view(np.int64).copy())
        r = sh.rdiag(s)
        r = torch.view_as_real(r) if r.is_complex() else r
        out.append(r.contiguous().cpu().numpy().view(np.int64).copy())
        out.append(sh.swap(s).cpu().numpy().copy())
    out.append(sh.info_all[:count].cpu().numpy().copy())
    return out


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("n", [37, 300, 1100])
def test_every_launch_shape_gives_the_same_bits(n, cplx):
    torch, G, T = _mods()
    rng = np.random.default_rng(n)
    J = torch.as_tensor(np.asfortranarray(rng.standard_normal((n, n)))).cuda()
    ws = G.lhl(J)
    S = 3
    sh = G.LHLShift(n, S, complex=cplx)
    if cplx:
        sig = torch.as_tensor(np.array([1 + 2j, -0.5 + 0.1j, 3j])).cuda()
        tau = torch.as_tensor(np.array([-1 + 0j, 0.7 - 0.2j, 1 + 0j])).cuda()
    else:
        sig = torch.as_tensor(np.array([1.0, 0.0, 2.0])).cuda()
        tau = torch.as_tensor(np.array([-0.1, 1.0, -3.0])).cuda()
    G.lhl_shift_batched_(sh, ws, sig, tau)
    torch.cuda.synchronize()
    ref = _state(torch, sh, S, n)
    variants = G.shift_variants(cplx, n)
    assert variants
    for v in variants:
        ws.set_shift_variant(0 if cplx else v, v if cplx else 0)
        G.lhl_shift_batched_(sh, ws, sig, tau)
        torch.cuda.synchronize()
        got = _state(torch, sh, S, n)
        assert all(np.array_equal(a, b) for a, b in zip(ref, got)), (n, cplx, v)
    shapes = {v: G.shift_variant_shape(cplx, v) for v in range(1, 16)}
    bad = [v for v, sh_ in shapes.items() if sh_ is not None and sh_[0] * sh_[1] < n]
    for v in bad:  # a shape that does not cover the order is refused on the host
        with pytest.raises(G.ArgumentError):
            ws.set_shift_variant(0 if cplx else v, v if cplx else 0)


def test_tuning_pass_on_a_small_workload(tmp_path):
    torch, G, T = _mods()
    n, S = 300, 8
    rng = np.random.default_rng(7)
    Jh = rng.standard_normal((n, n))
    J = torch.as_tensor(np.asfortranarray(Jh)).cuda()
    sig = torch.ones(S, dtype=torch.float64, device="cuda")
    tau = torch.as_tensor(-np.logspace(-3, -1, S)).cuda()
    B = torch.as_tensor(np.asfortranarray(rng.standard_normal((n, S)))).cuda()
    ws = G.LHLWorkspace(n, G.LHL_PREC_MIXED)
    best_k, ktr = T.tune_mixed_kernel(torch, ws, lambda: G.lhl_reduce_(ws, J, True))
    assert best_k in (1, 2) and len(ktr) == 2
    G.lhl_reduce_(ws, J, True)
    sh = G.LHLShift(n, S)
    v, vtr = T.tune_shift_variant(G, torch, ws, sh, sig, tau)
    assert v in G.shift_variants(False, n) and all(t["same_bits"] for t in vtr)
    ws.set_shift_variant(v, 0)
    X = B.clone()
    res = torch.empty(S, dtype=torch.float64, device="cuda")

    def chain(ch):
        G.lhl_shift_batched_(sh, ws, sig, tau)
        X.copy_(B)
        G.lhl_ldiv_(X, sh, ws)
        if ch[0] == "gmres":
            G.lhl_refine_gmres_(X, J, B, sh, ws, tol=1e-10, max_cycles=ch[1], restart=ch[2], res=res)
        else:
            G.lhl_refine_tol_(X, J, B, sh, ws, tol=1e-10, max_steps=ch[1], res=res)

    best, rtr = T.tune_refine(torch, "mixed", chain, lambda: bool((res <= 1e-10).all().item()))
    assert best is not None and any(t["ok"] for t in rtr)
    p = str(tmp_path / "tuning.json")
    key = T.workload_key(torch.cuda.get_device_name(), False, n, "mixed", 1)
    T.save_cache(T.record({}, key, {"refine": list(best), "shift_variant": [v, 0], "mixed_kernel": best_k}), p)
    got = T.lookup(torch.cuda.get_device_name(), False, n, "mixed", 1, path=p)
    assert got["refine"] == list(best) and got["shift_variant"] == [v, 0]
