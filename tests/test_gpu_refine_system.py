"""lhl_refine!(x, A, b, sh, ws, steps) with the caller's system matrix (lhl_refine_system, F:3144-3157
as the reference takes A): with A = sigma I + tau J it performs the updates of lhl_refine (J-based)
to rounding; it takes a single slot of a batch; a system matrix the factorisation only approximates
still converges (fixed-point and GMRES-IR); complex shifts take a complex A; bad arguments are
refused before any launch."""
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


def bwd(W, x, b):
    r = b - W @ x
    return np.abs(r).max() / (np.abs(W).sum(axis=1).max() * np.abs(x).max() + np.abs(b).max())


@pytest.mark.parametrize("n", [1, 5, 40, 129, 600])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_system_matrix_matches_J_form(n, precision):
    torch, G = _mods()
    g = np.random.default_rng(n)
    J = g.standard_normal((n, n))
    b = g.standard_normal(n)
    prec = G.LHL_PREC_MIXED if precision == "mixed" else G.LHL_PREC_FP64
    ws = G.lhl(dev(J), precision=prec)
    s, t = 1.0, -0.05
    G.lhl_shift_(ws, s, t)
    W = s * np.eye(n) + t * J
    x0 = G.lhl_ldiv_(dev(b), ws)
    xa, xj = x0.clone(), x0.clone()
    G.lhl_refine_system_(xa, dev(W), dev(b), ws, 2)
    G.lhl_refine_(xj, dev(J), dev(b), ws, 2)
    xa, xj = host(xa), host(xj)
    assert np.linalg.norm(xa - xj) <= 1e-12 * np.linalg.norm(xj)
    if precision == "fp64":
        assert bwd(W, xa, b) < 50 * np.finfo(float).eps


def test_system_matrix_uses_one_slot_of_a_batch():
    torch, G = _mods()
    n, S = 200, 5
    g = np.random.default_rng(3)
    J = g.standard_normal((n, n))
    ws = G.lhl(dev(J))
    sh = G.LHLShift(n, S)
    taus = -np.array([0.01, 0.02, 0.05, 0.1, 0.2])
    G.lhl_shift_batched_(sh, ws, torch.ones(S, dtype=torch.float64, device="cuda"), dev(taus))
    slot = 3
    W = np.eye(n) + taus[slot] * J
    B = g.standard_normal((n, 4))
    X = dev(B).clone()  # start from x = b: every column refines with slot 3's factorisation
    res = torch.empty(4, dtype=torch.float64, device="cuda")
    G.lhl_refine_system_(X, dev(W), dev(B), sh, ws, 8, slot=slot, tol=1e-13, res=res)
    Xh = host(X)
    for c in range(4):
        assert np.linalg.norm(B[:, c] - W @ Xh[:, c]) <= 1e-13 * np.linalg.norm(B[:, c])
    assert float(host(res).max()) <= 1e-13


@pytest.mark.parametrize("gmres", [False, True])
def test_approximate_factorisation_converges(gmres):
    """A = I - 0.05 (J + E) with a perturbation E the factorisation does not know: fixed-point and
    GMRES-IR with A itself both reach 1e-12."""
    torch, G = _mods()
    n = 256
    g = np.random.default_rng(8)
    J = g.standard_normal((n, n)) / np.sqrt(n)
    E = 0.05 * g.standard_normal((n, n)) / np.sqrt(n)
    ws = G.lhl(dev(J))
    G.lhl_shift_(ws, 1.0, -0.5)
    A = np.eye(n) - 0.5 * (J + E)
    B = g.standard_normal((n, 3))
    X = G.lhl_ldiv_(dev(B).clone(), ws, rhs_per_shift=3)
    res = torch.empty(3, dtype=torch.float64, device="cuda")
    G.lhl_refine_system_(X, dev(A), dev(B), ws, 30 if not gmres else 6, tol=1e-12, gmres=gmres, res=res)
    Xh = host(X)
    for c in range(3):
        assert np.linalg.norm(B[:, c] - A @ Xh[:, c]) <= 1e-12 * np.linalg.norm(B[:, c])


@pytest.mark.parametrize("complex_j", [False, True])
def test_complex_system_matrix(complex_j):
    """A complex shift on a real reduction, and a complex reduction: the system matrix is the complex
    W = sigma I + tau J; one step matches the J-form refinement and brings bwd under 50 eps."""
    torch, G = _mods()
    n = 129
    g = np.random.default_rng(11)
    J = g.standard_normal((n, n)) + (1j * g.standard_normal((n, n)) if complex_j else 0)
    b = g.standard_normal(n) + 1j * g.standard_normal(n)
    ws = G.lhl(dev(J)) if complex_j else G.lhl(dev(J), shift_complex=True)
    s, t = 0.4 + 0.7j, -1.0 + 0.2j
    G.lhl_shift_(ws, s, t)
    W = s * np.eye(n) + t * J
    x0 = G.lhl_ldiv_(dev(b), ws)
    xa, xj = x0.clone(), x0.clone()
    G.lhl_refine_system_(xa, dev(W.astype(np.complex128)), dev(b), ws, 1)
    G.lhl_refine_(xj, dev(J.astype(np.complex128) if complex_j else J), dev(b), ws, 1)
    xa, xj = host(xa), host(xj)
    assert np.linalg.norm(xa - xj) <= 1e-12 * np.linalg.norm(xj)
    assert bwd(W, xa, b) < 50 * np.finfo(float).eps


def test_system_refusals():
    torch, G = _mods()
    n = 8
    J = np.eye(n) * 2.0
    ws = G.lhl(dev(J))
    G.lhl_shift_(ws, 1.0, -0.1)
    x = dev(np.ones(n))
    with pytest.raises(G.DimensionMismatch):
        G.lhl_refine_system_(x, dev(np.eye(n + 1)), dev(np.ones(n)), ws, 1)
    with pytest.raises(G.DimensionMismatch):  # no slot 1 in a one-slot shift object
        G.lhl_refine_system_(x, dev(np.eye(n)), dev(np.ones(n)), ws, 1, slot=1)
    with pytest.raises(G.ArgumentError):  # a real shift object takes a real A
        G.lhl_refine_system_(x, dev(np.eye(n, dtype=np.complex128)), dev(np.ones(n)), ws, 1)


def test_complex_vectors_with_a_real_A_on_a_real_shift():
    """lhl_refine!(x, A, b, ws, steps) with complex x and b, a real A and a real shift (the
    reference's generic path): the same as refining the real and imaginary parts on their own,
    and the returned residuals are at the FP64 floor, as the complex columns' ||b - A x|| / ||b||."""
    torch, G = _mods()
    n = 60
    g = np.random.default_rng(61)
    J = g.standard_normal((n, n))
    A = np.eye(n) - 0.1 * J
    b = g.standard_normal((n, 2)) + 1j * g.standard_normal((n, 2))
    ws = G.lhl(dev(J))
    G.lhl_shift_(ws, 1, -0.1)
    x = G.lhl_ldiv_(dev(b), ws, rhs_per_shift=2)
    res = torch.empty(2, dtype=torch.float64, device="cuda")
    G.lhl_refine_system_(x, dev(A), dev(b), ws, 2, res=res)
    xr = G.lhl_ldiv_(dev(np.ascontiguousarray(b.real)), ws, rhs_per_shift=2)
    G.lhl_refine_system_(xr, dev(A), dev(np.ascontiguousarray(b.real)), ws, 2)
    xi = G.lhl_ldiv_(dev(np.ascontiguousarray(b.imag)), ws, rhs_per_shift=2)
    G.lhl_refine_system_(xi, dev(A), dev(np.ascontiguousarray(b.imag)), ws, 2)
    assert np.allclose(host(x), host(xr) + 1j * host(xi), rtol=1e-12, atol=0)
    xh = host(x)
    want = np.linalg.norm(b - A @ xh, axis=0) / np.linalg.norm(b, axis=0)
    assert np.all(want <= 1e-13) and np.all(host(res) <= 1e-13)  # both at the FP64 floor
