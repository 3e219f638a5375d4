"""LHLWorkspace{Float32} on the device (the reference's element type T = Float32, F:703-705).

The shift LU bit for bit against the oracle's float restatement on the device's Ht
(test/core_tests.jl:192-212 with T = Float32); solves against a dense LU with the reference's
Float32 bounds (test/core_tests.jl:38-58: rtol 1e-3 and a backward error below 50 eps32 up to
n = 500); the reduction bit for bit against the oracle's float restatement below n = 1024 and,
from there, a valid similarity with float factors and the FP64 pivots; float
right-hand sides in and out; a Float64 workspace takes float J exactly; ComplexF32 shifts and
vectors on a Float32 workspace (test/core_tests.jl:324-329)."""
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


F32_SIZES = list(range(1, 34)) + [64, 130, 255, 256, 257, 499, 500, 511, 512, 520, 777, 1000, 1023, 1024, 1025, 1100,
                                    1500, 2048]


def _f32_matrix(n, kind):
    g = rng(4000 + n)
    if kind == "tie":
        return g.integers(-2, 3, (n, n)).astype(np.float32)
    J = g.standard_normal((n, n))
    if kind == "graded":
        D = 2.0 ** g.integers(-10, 11, n)
        J = (J * D[None, :]) / D[:, None]
    return J.astype(np.float32)


@pytest.mark.parametrize("n", F32_SIZES)
@pytest.mark.parametrize("kind", ["gauss", "tie", "graded"])
def test_f32_reduction_bitexact(n, kind):
    """The Float32 workspace reduces in float, as the reference does: balancing (F:299-340,
    Tr = Float32), then below _lhl_block_min(Float32) = 1024 the unblocked ELMHES (F:466-678)
    and from there the blocked pointer path (F:765-1006).  ipiv, factors, Ht, scale, iscale,
    perm and iperm bit for bit against the oracle's float restatement, with and without
    balancing, through both entry points (J as float and as float64 rounded on the way in)."""
    torch, G = _mods()
    J = _f32_matrix(n, kind)
    for balance in (True, False):
        R = O.reduce_f32(J.astype(np.float64), balance=balance)
        for Jd in (dev(J), dev(J.astype(np.float64))):
            ws = G.LHLWorkspace(n, dtype=torch.float32)
            G.lhl_reduce_(ws, Jd, balance)
            ws.check()
            assert bits_equal(host(ws.factors), R.factors), (n, kind, balance)
            assert np.array_equal(host(ws.ipiv)[: max(n - 2, 0)], R.ipiv)
            assert bits_equal(host(ws.Ht), R.Ht)
            assert bits_equal(host(ws.scale), R.scale) and bits_equal(host(ws.iscale), R.iscale)
            assert np.array_equal(host(ws.perm), R.perm) and np.array_equal(host(ws.iperm), R.iperm)


def test_f32_reduction_timeout_reports_and_recovers():
    """The float reduction's grid barriers are bounded like the FP64 ones: a 1 ns limit ends it
    with LHL_ERR_TIMEOUT, and the same workspace then reduces bit-exactly.  A graded matrix, so
    that the other CTAs wait at a barrier while CTA 0 takes the balancing decisions."""
    torch, G = _mods()
    n = 1000
    J = _f32_matrix(n, "graded")
    ws = G.LHLWorkspace(n, dtype=torch.float32)
    ws.set_barrier_limit_ns(1)
    G.lhl_reduce_(ws, dev(J), True)
    with pytest.raises(G.LHLDeviceError):
        ws.check()
    ws.set_barrier_limit_ns(2_000_000_000)
    G.lhl_reduce_(ws, dev(J), True)
    ws.check()
    R = O.reduce_f32(J.astype(np.float64))
    assert bits_equal(host(ws.factors), R.factors)


@pytest.mark.parametrize("n", [1024, 1100])
def test_f32_blocked_orders_are_a_float_similarity(n):
    """From n = 1024 (the blocked float form): float factors, Z H Z^-1 = J to float accuracy,
    |l| <= 1.  (The pivots are the oracle's float ones, bit for bit above; near the end of an
    order this large they can differ from the Float64 reduction's on near-ties.)"""
    torch, G = _mods()
    J = rng(70 + n).standard_normal((n, n)).astype(np.float32)
    ws = G.lhl(dev(J))
    F = host(ws.factors)
    assert is_float_valued(F) and is_float_valued(host(ws.Ht))
    assert np.array_equal(host(ws.scale), O.reduce_f32(J.astype(np.float64)).scale)
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
    assert np.abs(np.tril(F, -2)).max() <= 1.0


def test_f64_workspace_takes_float_J_exactly():
    torch, G = _mods()
    n = 200
    J = rng(9).standard_normal((n, n)).astype(np.float32)
    ws = G.LHLWorkspace(n)
    G.lhl_reduce_(ws, dev(J), True)
    w2 = G.lhl(dev(J.astype(np.float64)))
    assert bits_equal(host(ws.factors), host(w2.factors))


def test_f32_complex_shifts_like_the_reference():
    """test/core_tests.jl:324-329: lhl(J32; shift = ComplexF32), lhl_shift!(w32, 0.4 + 0.7im, -1),
    lhl_ldiv! of a ComplexF32 vector against the dense solve, rtol 1e-3.  The shift is stored
    rounded to ComplexF32; a block of ComplexF32 right-hand sides and a batch of shifts too."""
    torch, G = _mods()
    n = 70
    J = rng(95).standard_normal((n, n)).astype(np.float32)
    b = (rng(96).standard_normal(n) + 1j * rng(97).standard_normal(n)).astype(np.complex64)
    ws = G.lhl(dev(J), shift_complex=True)
    assert ws.dtype == torch.float32 and ws.shift.is_complex
    s = np.complex64(0.4 + 0.7j)
    G.lhl_shift_(ws, complex(s), -1.0)
    x = G.lhl_ldiv_(dev(b), ws)
    assert x.dtype == torch.complex64
    W = s * np.eye(n) - J.astype(np.complex128)
    xr = np.linalg.solve(W, b.astype(np.complex128))
    assert np.linalg.norm(host(x) - xr) <= 1e-3 * np.linalg.norm(xr)
    assert ws.shift.σ == complex(s)  # stored rounded to ComplexF32 (0.4 and 0.7 are not floats)
    # a batch of complex shifts, several ComplexF32 right-hand sides each
    S, R = 3, 2
    sh = G.LHLShift(ws, S, complex=True)  # LHLShift{ComplexF32}(ws)
    sigs = np.array([0.4 + 0.7j, 1.5 - 0.2j, 3j], dtype=np.complex128)
    taus = np.array([-1.0 + 0j, -0.5 + 0.1j, 1.0 + 0j], dtype=np.complex128)
    G.lhl_shift_batched_(sh, ws, dev(sigs), dev(taus))
    B = (rng(98).standard_normal((n, S * R)) + 1j * rng(99).standard_normal((n, S * R))).astype(np.complex64)
    X = host(G.lhl_ldiv_(dev(B), sh, ws, rhs_per_shift=R))
    for c in range(S * R):
        sg, tg = sigs[c // R].astype(np.complex64), taus[c // R].astype(np.complex64)
        Wc = sg * np.eye(n) + tg * J.astype(np.complex128)
        xc = np.linalg.solve(Wc, B[:, c].astype(np.complex128))
        assert np.linalg.norm(X[:, c] - xc) <= 1e-3 * np.linalg.norm(xc), c


def test_f32_mixed_form_above_the_blocked_threshold():
    """A mixed Float32 workspace from n = 1024 takes the mixed reduction rounded to float (no
    blocked float scratch): float factors, a float-accurate similarity, solves within the Float32
    tolerance."""
    torch, G = _mods()
    n = 1100
    J = rng(1100).standard_normal((n, n)).astype(np.float32)
    ws = G.lhl(dev(J), precision=G.LHL_PREC_MIXED)
    ws.check()
    F = host(ws.factors)
    assert is_float_valued(F) and is_float_valued(host(ws.Ht))
    assert np.abs(np.tril(F, -2)).max() <= 1.0
    b = rng(1101).standard_normal(n).astype(np.float32)
    G.lhl_shift_(ws, 1, -0.05)
    x = host(G.lhl_ldiv_(dev(b), ws))
    W = np.eye(n) - 0.05 * J.astype(np.float64)
    xr = np.linalg.solve(W, b.astype(np.float64))
    assert np.linalg.norm(x - xr) <= 1e-3 * np.linalg.norm(xr)


def test_element_type_entry_points_refuse_the_wrong_workspace():
    """lhl_reduce_c64 / lhl_reduce_c128 need a complex-J workspace, lhl_reduce and lhl_reduce_f32
    a real one (LHL_ERR_ARG, the reference's ArgumentError)."""
    import ctypes
    torch, G = _mods()
    L = G._lib
    real = G.LHLWorkspace(8, dtype=torch.float32)
    cplx = G.LHLWorkspace(8, dtype=torch.complex64)
    Jc = torch.zeros((8, 8), dtype=torch.complex64, device="cuda")
    Jr = torch.zeros((8, 8), dtype=torch.float32, device="cuda")
    assert L.lhl_reduce_c64(real._h, ctypes.c_void_p(Jc.data_ptr()), 8, 1, None) == G.LHL_ERR_ARG
    assert L.lhl_reduce_f32(cplx._h, ctypes.c_void_p(Jr.data_ptr()), 8, 1, None) == G.LHL_ERR_ARG
    assert L.lhl_reduce_c64(cplx._h, ctypes.c_void_p(Jc.data_ptr()), 4, 1, None) == G.LHL_ERR_DIM


def test_shift_types_follow_the_reference_rule():
    """An LHLShift{TG} serves an LHLWorkspace{T} only for TG = T or Complex{real(T)}
    (F:2461-2465; test/core_tests.jl:315: LHLShift{ComplexF64} on a Float32 workspace is an
    ArgumentError), and the other way round."""
    torch, G = _mods()
    J32 = rng(3).standard_normal((3, 3)).astype(np.float32)
    w32 = G.lhl(dev(J32))
    with pytest.raises(G.ArgumentError):
        G.lhl_shift_(G.LHLShift(3, complex=True), w32, 1, 1)      # LHLShift{ComplexF64}
    with pytest.raises(G.ArgumentError):
        G.lhl_shift_(G.LHLShift(3), w32, 1, 1)                    # LHLShift{Float64}
    G.lhl_shift_(G.LHLShift(3, complex=True, single=True), w32, 1, 1)   # LHLShift{ComplexF32}
    G.lhl_shift_(G.LHLShift(w32), w32, 1, 1)                      # LHLShift{Float32}(ws)
    w64 = G.lhl(dev(J32.astype(np.float64)))
    with pytest.raises(G.ArgumentError):
        G.lhl_shift_(G.LHLShift(3, single=True), w64, 1, 1)       # LHLShift{Float32} on Float64
    with pytest.raises(G.ArgumentError):
        G.lhl_shift_(G.LHLShift(3, complex=True, single=True), w64, 1, 1)
    G.lhl_shift_(G.LHLShift(3, complex=True), w64, 1, 1)
