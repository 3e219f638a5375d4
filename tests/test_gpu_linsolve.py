"""The solver-interface route (README.md:56-70) on the device: lhl_gpu.linsolve's
LHLFactorization solves W = J - (m / gamma) I to 1e-10 for a sequence of gamma values from one
reduction, in both forms; a diagonal or dense mass matrix through refinement with W itself; a
wrong-sized mass matrix and gamma = 0 are refused."""
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


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("form", ["diagonal", "dense"])
def test_mass_matrix_through_the_system_matrix(precision, form):
    """W = J - M / gamma with M not a multiple of I: the shift factorises J - (mean diag M / gamma) I,
    and GMRES-IR with W itself reaches 1e-10 for every gamma, still from one reduction."""
    import torch
    import lhl_gpu as G
    from lhl_gpu.linsolve import LHLFactorization
    n = 300
    g = np.random.default_rng(1)
    J = g.standard_normal((n, n)) / np.sqrt(n)
    d = 1.0 + 0.3 * g.uniform(-1, 1, n)
    M = np.diag(d) if form == "diagonal" else np.diag(d) + 0.02 * g.standard_normal((n, n)) / np.sqrt(n)
    b = g.standard_normal(n)
    Jd = torch.as_tensor(np.asfortranarray(J)).cuda()
    Md = torch.as_tensor(d).cuda() if form == "diagonal" else torch.as_tensor(np.asfortranarray(M)).cuda()
    bd = torch.as_tensor(b).cuda()
    prec = G.LHL_PREC_MIXED if precision == "mixed" else G.LHL_PREC_FP64
    cache = LHLFactorization(Jd, 0.01, mass_matrix=Md, precision=prec, max_steps=12)
    assert abs(cache.m - np.diag(M).mean()) <= 1e-12
    factors = cache.ws.factors.clone()
    for gamma in (0.01, 0.02, 0.05):
        cache.update_gamma(gamma)
        x = cache.solve(bd).cpu().numpy()
        W = J - M / gamma
        assert np.linalg.norm(b - W @ x) <= 1.0001e-10 * np.linalg.norm(b), gamma
    assert torch.equal(cache.ws.factors, factors)


def test_refusals():
    import torch
    import lhl_gpu as G
    from lhl_gpu.linsolve import LHLFactorization
    J = torch.eye(4, dtype=torch.float64, device="cuda") * 3.0
    with pytest.raises(G.DimensionMismatch):
        LHLFactorization(J, 0.1, mass_matrix=torch.ones(5, dtype=torch.float64, device="cuda"))
    with pytest.raises(G.ArgumentError):
        LHLFactorization(J, 0.1, mass_matrix=torch.tensor([1.0, -1.0, 1.0, -1.0], device="cuda"))
    c = LHLFactorization(J, 0.1)
    with pytest.raises(G.ArgumentError):
        c.update_gamma(0.0)
