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
