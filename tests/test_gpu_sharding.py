"""lhl_gpu.sharding on one GPU: a one-rank NCCL group runs the sharded per-shift chain, whose
solutions are bit-identical to the unsharded chain's (the same kernels on the same slice)."""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_sharded_chain_one_rank(precision):
    import torch
    import torch.distributed as dist
    import lhl_gpu as G
    from lhl_gpu import sharding as SH
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()))
    dist.init_process_group("nccl", rank=0, world_size=1, device_id=torch.device("cuda", 0))
    try:
        g = np.random.default_rng(3)
        n, S, R = 300, 5, 2
        J = g.standard_normal((n, n))
        Jd = torch.as_tensor(np.asfortranarray(J)).cuda()
        prec = G.LHL_PREC_MIXED if precision == "mixed" else G.LHL_PREC_FP64
        ws = G.lhl(Jd, precision=prec)
        sig = torch.ones(S, dtype=torch.float64, device="cuda")
        tau = torch.as_tensor(-(10.0 ** g.uniform(-3, -1, S))).cuda()
        B = torch.as_tensor(np.asfortranarray(g.standard_normal((n, S * R)))).cuda()
        X, res = SH.sharded_chain(G, ws, Jd, B, sig, tau, rhs_per_shift=R, tol=1e-10)
        assert (res.cpu().numpy() <= 1e-10).all()
        sh = G.LHLShift(n, S)
        G.lhl_shift_batched_(sh, ws, sig, tau)
        X2 = B.clone()
        G.lhl_ldiv_(X2, sh, ws, rhs_per_shift=R)
        G.lhl_refine_gmres_(X2, Jd, B, sh, ws, tol=1e-10, rhs_per_shift=R)
        assert np.array_equal(X.cpu().numpy().view(np.int64), X2.cpu().numpy().view(np.int64))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("form", ["fp64", "mixed", "complex"])
@pytest.mark.parametrize("n", [5, 300, 777])
def test_packed_reduction_imports_bit_for_bit(form, n):
    """The buffer broadcast_reduction sends (pack_reduction), unpacked and imported into a fresh
    workspace, shifts and solves bit for bit like the workspace it came from."""
    import torch
    import lhl_gpu as G
    from lhl_gpu import sharding as SH
    g = np.random.default_rng(n)
    cj = form == "complex"
    J = g.standard_normal((n, n)) + (1j * g.standard_normal((n, n)) if cj else 0)
    Jd = torch.as_tensor(np.asfortranarray(J)).cuda()
    prec = G.LHL_PREC_MIXED if form == "mixed" else G.LHL_PREC_FP64
    ws = G.lhl(Jd, precision=prec)
    buf = SH.pack_reduction({k: getattr(ws, k) for k in G.REDUCTION_ARRAYS}, n, cj)
    w2 = G.LHLWorkspace(n, prec, dtype=ws.dtype)
    w2.import_arrays(SH.unpack_reduction(buf, n, cj))
    for name in G.REDUCTION_ARRAYS:
        a, b = getattr(ws, name).cpu(), getattr(w2, name).cpu()
        if a.is_complex():
            a, b = torch.view_as_real(a.contiguous()), torch.view_as_real(b.contiguous())
        assert np.array_equal(a.contiguous().numpy().view(np.uint8), b.contiguous().numpy().view(np.uint8)), name
    B = g.standard_normal((n, 3)) + (1j * g.standard_normal((n, 3)) if cj else 0)
    Bd = torch.as_tensor(np.asfortranarray(B)).cuda()
    dt = torch.complex128 if cj else torch.float64
    sig = torch.ones(3, dtype=dt, device="cuda")
    tau = torch.tensor([-0.01, -0.05, -0.2], dtype=dt, device="cuda")
    out = []
    for w in (ws, w2):
        sh = G.LHLShift(n, 3, complex=cj)
        G.lhl_shift_batched_(sh, w, sig, tau)
        X = Bd.clone()
        G.lhl_ldiv_(X, sh, w)
        out.append(torch.view_as_real(X).cpu().numpy() if cj else X.cpu().numpy())
    assert np.array_equal(out[0].view(np.int64), out[1].view(np.int64))


def test_broadcast_reduction_one_rank():
    """broadcast_reduction's collectives over NCCL in a one-rank group: the source keeps its
    reduction, and a source without one makes the call raise."""
    import torch
    import torch.distributed as dist
    import lhl_gpu as G
    from lhl_gpu import sharding as SH
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()))
    dist.init_process_group("nccl", rank=0, world_size=1, device_id=torch.device("cuda", 0))
    try:
        n = 64
        J = np.random.default_rng(1).standard_normal((n, n))
        ws = G.lhl(torch.as_tensor(np.asfortranarray(J)).cuda())
        before = ws.factors.cpu().numpy().copy()
        assert SH.broadcast_reduction(ws, src=0) is ws
        assert np.array_equal(before.view(np.int64), ws.factors.cpu().numpy().view(np.int64))
        with pytest.raises(ValueError):
            SH.broadcast_reduction(G.LHLWorkspace(n), src=0)
    finally:
        dist.destroy_process_group()
