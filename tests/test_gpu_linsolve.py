"""The solver-interface route (README.md:56-70) on the device: lhl_gpu.linsolve's
LHLFactorization solves W = J - (m / gamma) I to 1e-10 for a sequence of gamma values from one
reduction, in both forms; a non-scalar mass matrix and gamma = 0 are refused."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_update_gamma_reuses_the_reduction(precision):
    import torch
    import lhl_gpu as G
    from lhl_gpu.linsolve import LHLFactorization
    n = 400
    g = np.random.default_rng(0)
    J = g.standard_normal((n, n))
    b = g.standard_normal(n)
    Jd = torch.as_tensor(np.asfortranarray(J)).cuda()
    bd = torch.as_tensor(b).cuda()
    prec = G.LHL_PREC_MIXED if precision == "mixed" else G.LHL_PREC_FP64
    cache = LHLFactorization(Jd, 0.01, mass_matrix=2.0, precision=prec)
    factors = cache.ws.factors.clone()
    for gamma in (0.01, 0.013, 0.021):
        cache.update_gamma(gamma)
        x = cache.solve(bd).cpu().numpy()
        W = J - (2.0 / gamma) * np.eye(n)
        assert np.linalg.norm(b - W @ x) <= 1.0001e-10 * np.linalg.norm(b)
    assert torch.equal(cache.ws.factors, factors)  # one reduction for every gamma


def test_refusals():
    import torch
    import lhl_gpu as G
    from lhl_gpu.linsolve import LHLFactorization
    J = torch.eye(4, dtype=torch.float64, device="cuda") * 3.0
    with pytest.raises(G.ArgumentError):
        LHLFactorization(J, 0.1, mass_matrix=torch.eye(4, dtype=torch.float64, device="cuda"))
    c = LHLFactorization(J, 0.1)
    with pytest.raises(G.ArgumentError):
        c.update_gamma(0.0)
