"""LHLWorkspace{Float32} on the device (the reference's element type T = Float32, F:703-705).

The shift LU bit for bit against the oracle's float restatement on the device's Ht
(test/core_tests.jl:192-212 with T = Float32); solves against a dense LU with the reference's
Float32 bounds (test/core_tests.jl:38-58: rtol 1e-3 and a backward error below 50 eps32 up to
n = 500); the reduction is a valid similarity with float factors and the FP64 pivots; float
right-hand sides in and out; a Float64 workspace takes float J exactly; complex shifts on a
Float32 workspace are refused."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

SHIFTS = ((1.0, -0.1), (0.0, 1.0), (1.0, -3.0), (2.0, 0.0), (0.0, 0.0))
EPS32 = float(np.finfo(np.float32).eps)


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


def bits_equal(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return a.shape == b.shape and np.array_equal(a.view(np.int64), b.view(np.int64))


def is_float_valued(a):
    a = np.asarray(a, dtype=np.float64)
    return np.array_equal(a.astype(np.float32).astype(np.float64), a, equal_nan=True)


@pytest.mark.parametrize("n", list(range(1, 34)) + [64, 255, 256, 257, 511, 512, 520, 1000, 1024])
@pytest.mark.parametrize("tie", [False, True])
def test_f32_shift_bitexact(n, tie):
    torch, G = _mods()
    g = rng(500 + n + 1000 * tie)
    J = (g.integers(-2, 3, (n, n)) if tie else g.standard_normal((n, n))).astype(np.float32)
    ws = G.lhl(dev(J))
    assert ws.dtype == torch.float32
    Ht = host(ws.Ht)
    assert is_float_valued(Ht)
    for s, t in SHIFTS:
        with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
            S = O.shift_f32(Ht, s, t)
        G.lhl_shift_(ws, s, t)
        torch.cuda.synchronize()
        Gt = host(ws.shift.Gt())
        U = np.array([Gt[j, k] for k in range(n) for j in range(k, n)])
        l = np.array([Gt[k, k + 1] for k in range(n - 1)])
        U0, l0, sw0, rd0, info0 = S.state()
        assert bits_equal(U, U0), (n, s, t)
        assert bits_equal(l, l0)
        assert np.array_equal(host(ws.shift.swap()), sw0)
        assert bits_equal(host(ws.shift.rdiag()), rd0)
        assert ws.shift.info == info0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("n", [3, 7, 33, 130, 331, 500])
def test_f32_solves(n, precision):
    torch, G = _mods()
    J = rng(n).standard_normal((n, n)).astype(np.float32)
    b = rng(n + 7).standard_normal(n).astype(np.float32)
    prec = G.LHL_PREC_MIXED if precision == "mixed" else G.LHL_PREC_FP64
    ws = G.lhl(dev(J), precision=prec)
    G.lhl_shift_(ws, 1, -0.05)
    W = np.eye(n, dtype=np.float32) - np.float32(0.05) * J
    x = host(G.lhl_ldiv_(dev(b), ws))
    assert x.dtype == np.float32
    xr = np.linalg.solve(W.astype(np.float64), b.astype(np.float64))
    assert np.linalg.norm(x - xr) <= 1e-3 * np.linalg.norm(xr)
    bwd = np.linalg.norm(b - W @ x, np.inf) / (np.linalg.norm(W, np.inf) * np.linalg.norm(x, np.inf)
                                               + np.linalg.norm(b, np.inf))
    assert bwd < 50 * EPS32, bwd
    # a block of float right-hand sides, and FP64 vectors on the same workspace
    B = rng(n + 8).standard_normal((n, 3)).astype(np.float32)
    X = host(G.lhl_ldiv_(dev(B), ws, rhs_per_shift=3))
    for c in range(3):
        xc = np.linalg.solve(W.astype(np.float64), B[:, c].astype(np.float64))
        assert np.linalg.norm(X[:, c] - xc) <= 1e-3 * np.linalg.norm(xc)
    x64 = host(G.lhl_ldiv_(dev(b.astype(np.float64)), ws))
    assert np.linalg.norm(x64 - xr) <= 1e-3 * np.linalg.norm(xr)


@pytest.mark.parametrize("n", [5, 80, 300, 600])
def test_f32_reduction_is_a_float_similarity(n):
    """Plain form: the FP64 reduction of the widened J, rounded: FP64 pivots, float factors,
    Z H Z^-1 = J to float accuracy, |l| <= 1."""
    torch, G = _mods()
    J = rng(70 + n).standard_normal((n, n)).astype(np.float32)
    ws = G.lhl(dev(J))
    R64 = O.reduce(J.astype(np.float64))
    assert np.array_equal(host(ws.ipiv)[: max(n - 2, 0)], R64.ipiv)
    F = host(ws.factors)
    assert is_float_valued(F) and is_float_valued(host(ws.Ht))
    assert np.array_equal(host(ws.scale), R64.scale)
    R = O.Reduction(n)
    R.factors = np.asfortranarray(F)
    R.ipiv = host(ws.ipiv)[: max(n - 2, 0)].copy()
    R.scale = host(ws.scale).copy()
    R.iscale = host(ws.iscale).copy()
    R.perm = host(ws.perm).copy()
    R.iperm = host(ws.iperm).copy()
    R.Ht = np.asfortranarray(host(ws.Ht))
    Jd = J.astype(np.float64)
    rel = np.linalg.norm(R.Z() @ R.H @ R.Zinv() - Jd) / np.linalg.norm(Jd)
    assert rel <= 2 * EPS32 * n ** 1.5, rel  # the mixed form's bound: rounding the factors to float
    if n > 2:
        assert np.abs(np.tril(F, -2)).max() <= 1.0


def test_f64_workspace_takes_float_J_exactly():
    torch, G = _mods()
    n = 200
    J = rng(9).standard_normal((n, n)).astype(np.float32)
    ws = G.LHLWorkspace(n)
    G.lhl_reduce_(ws, dev(J), True)
    w2 = G.lhl(dev(J.astype(np.float64)))
    assert bits_equal(host(ws.factors), host(w2.factors))


def test_f32_refuses_complex_shifts():
    torch, G = _mods()
    J = rng(3).standard_normal((6, 6)).astype(np.float32)
    with pytest.raises(G.ArgumentError):
        G.lhl(dev(J), shift_complex=True)
    ws = G.lhl(dev(J))
    sh = G.LHLShift(6, 1, complex=True)
    with pytest.raises(G.ArgumentError):
        G.lhl_shift_batched_(sh, ws, dev(np.array([1.0 + 1j])), dev(np.array([-0.5 + 0j])))
