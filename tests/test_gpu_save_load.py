"""Workspace save / load (lhl_ws_import): a reloaded workspace shifts and solves bit for bit
like the one that was saved, in both forms."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("n", [1, 2, 5, 300, 777])
def test_save_load_round_trip(tmp_path, precision, n):
    import torch
    import lhl_gpu as G
    g = np.random.default_rng(n)
    J = g.standard_normal((n, n))
    Jd = torch.as_tensor(np.asfortranarray(J)).cuda()
    prec = G.LHL_PREC_MIXED if precision == "mixed" else G.LHL_PREC_FP64
    ws = G.lhl(Jd, precision=prec)
    path = str(tmp_path / "ws.npz")
    ws.save(path)
    w2 = G.LHLWorkspace.load(path)
    assert w2.n == n and w2.precision == prec
    for name in ("factors", "Ht", "ipiv", "perm", "iperm", "scale", "iscale"):
        a, b = getattr(ws, name).cpu().numpy(), getattr(w2, name).cpu().numpy()
        assert np.array_equal(np.ascontiguousarray(a).view(np.uint8), np.ascontiguousarray(b).view(np.uint8)), name
    B = torch.as_tensor(np.asfortranarray(g.standard_normal((n, 3)))).cuda()
    sig = torch.ones(3, dtype=torch.float64, device="cuda")
    tau = torch.tensor([-0.01, -0.05, -0.2], dtype=torch.float64, device="cuda")
    out = []
    for w in (ws, w2):
        sh = G.LHLShift(n, 3)
        G.lhl_shift_batched_(sh, w, sig, tau)
        X = B.clone()
        G.lhl_ldiv_(X, sh, w)
        out.append(X.cpu().numpy())
    assert np.array_equal(out[0].view(np.int64), out[1].view(np.int64))


def test_load_rejects_an_empty_workspace(tmp_path):
    import torch
    import lhl_gpu as G
    ws = G.LHLWorkspace(4)
    with pytest.raises(G.ArgumentError):
        ws.save(str(tmp_path / "x.npz"))
