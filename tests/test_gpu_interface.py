"""test/Interface/public_interface.jl on the device, testset by testset, through the host mirror
(a trailing `_` stands for `!`; torch CUDA tensors stand for the Julia arrays).  The one line
not carried over is `LHLWorkspace{Float64}(9; shift = ComplexF32)`: the mirror has no ComplexF32
shift type to refuse."""
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


def approx(x, y, rtol=np.sqrt(np.finfo(float).eps)):
    """Julia's isapprox: ||x - y|| <= rtol max(||x||, ||y||), default rtol sqrt(eps)."""
    return np.linalg.norm(x - y) <= rtol * max(np.linalg.norm(x), np.linalg.norm(y))


def test_generic_workspace_lifecycle():
    torch, G = _mods()
    g = np.random.default_rng(1)
    J = g.standard_normal((5, 5))
    ws = G.LHLWorkspace(5)
    Jd = dev(J)
    assert G.lhl_reduce_(ws, Jd[:, :], False) is ws
    assert G.lhl_shift_(ws, 1.0, -0.1) is ws
    b = g.standard_normal(5)
    x = dev(b)
    assert G.lhl_ldiv_(x, ws) is x
    assert approx(host(x), np.linalg.solve(np.eye(5) - 0.1 * J, b))
    x0 = g.standard_normal(5)
    t = dev(x0)
    assert G.applyZ_(t, ws) is t
    assert G.applyZinv_(t, ws) is t
    assert approx(host(t), x0)


def test_generic_allocating_and_reusing_entry_points():
    torch, G = _mods()
    g = np.random.default_rng(2)
    ws = G.lhl(dev(g.standard_normal((4, 4)))[:, :], balance=False)
    assert isinstance(ws, G.LHLWorkspace)
    J2 = g.standard_normal((6, 6))
    assert G.lhl_(ws, dev(J2), balance=True) is ws  # a 4x4 workspace takes a 6x6 J
    G.lhl_shift_(ws, 1.0, 0.2)
    b = g.standard_normal(6)
    assert approx(host(G.lhl_ldiv_(dev(b), ws)), np.linalg.solve(np.eye(6) + 0.2 * J2, b))


def test_generic_iterative_refinement():
    torch, G = _mods()
    g = np.random.default_rng(3)
    J = g.standard_normal((7, 7))
    b = g.standard_normal(7)
    ws = G.lhl(dev(J))
    A = np.eye(7) - 0.05 * J
    G.lhl_shift_(ws, 1.0, -0.05)
    x = G.lhl_ldiv_(dev(b), ws)
    assert G.lhl_refine_system_(x, dev(A), dev(b), ws, 1) is x
    assert approx(A @ host(x), b, rtol=1e-10)


def test_generic_complex_shifts_against_a_real_reduction():
    torch, G = _mods()
    g = np.random.default_rng(4)
    J = g.standard_normal((9, 9))
    b = g.standard_normal(9)
    tau = -0.05 + 0.02j
    W = np.eye(9) + tau * J
    ws = G.lhl(dev(J)[:, :], shift_complex=True)
    assert ws.shift.is_complex and ws.dtype == torch.float64
    G.lhl_shift_(ws, 1.0, tau)
    assert approx(host(G.lhl_ldiv_(dev(b.astype(complex)), ws)), np.linalg.solve(W, b))
    # a second, complex shift held alongside the workspace's own real one
    wr = G.lhl(dev(J))
    sh = G.LHLShift(wr, complex=True)
    assert sh.is_complex and sh.n == 9
    assert G.lhl_shift_(wr, 1.0, -0.05) is wr
    assert G.lhl_shift_(sh, wr, 1.0, tau) is sh
    assert approx(host(G.lhl_ldiv_(dev(b), wr)), np.linalg.solve(np.eye(9) - 0.05 * J, b))
    zc = G.lhl_ldiv_(dev(b.astype(complex)), sh, wr)
    assert approx(host(zc), np.linalg.solve(W, b))
    assert G.lhl_refine_system_(zc, dev(W), dev(b.astype(complex)), sh, wr, 1) is zc
    assert approx(W @ host(zc), b, rtol=1e-10)
    assert G.LHLShift(9, complex=True).is_complex


@pytest.mark.parametrize("thread", [True, False])
def test_generic_thread_keyword_and_shift_field_forwarding(thread):
    torch, G = _mods()
    J = np.random.default_rng(5).standard_normal((11, 11))
    Jd = dev(J)
    ws = G.LHLWorkspace(11)
    assert G.lhl_reduce_(ws, Jd, True, thread) is ws
    assert G.lhl_(ws, Jd, thread=thread) is ws
    assert isinstance(G.lhl(Jd, thread=thread), G.LHLWorkspace)
    ws = G.lhl(Jd)
    G.lhl_shift_(ws, 1.0, -0.25)
    # the shift-dependent fields are reachable through the workspace as well
    assert ws.Gt.data_ptr() == ws.shift.Gt().data_ptr()
    assert ws.rdiag.data_ptr() == ws.shift.rdiag().data_ptr()
    assert ws.swap.data_ptr() == ws.shift.swap().data_ptr()
    assert ws.σ == ws.shift.σ == 1.0 and ws.τ == ws.shift.τ == -0.25
    assert ws.info == ws.shift.info == 0
