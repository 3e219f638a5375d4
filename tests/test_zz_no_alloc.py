"""lhl_reduce_noalloc, the reduction entry point that allocates nothing.

It serves callers that cannot call cudaMalloc (a host that owns a fixed device-memory
budget, a Julia session whose CUDA.jl pool must remain the only allocator): every input and
output is passed in, and the scratch lives in a fixed static device array of the library.
Checked here through the C ABI against the allocating entry point (lhl_reduce through a
workspace) on the same inputs, two calls in a row, for both the unblocked (n < 500) and
the blocked path.  The file sorts last so that a run stopping at its first failure has
already run every other test."""
import ctypes as C
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(REPO, "lhl.jl_b200", "liblhl_gpu.so")


def _noalloc_fn():
    L = C.CDLL(LIB)
    f = L.lhl_reduce_noalloc
    vp, i64 = C.c_void_p, C.c_int64
    f.argtypes = [i64, vp, i64, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp]
    f.restype = C.c_int
    return f


def _check_fn():
    L = C.CDLL(LIB)
    L.lhl_reduce_noalloc_check.argtypes = [C.c_void_p]
    L.lhl_reduce_noalloc_check.restype = C.c_int
    L.lhl_reduce_noalloc_set_barrier_limit_ns.argtypes = [C.c_uint64]
    L.lhl_reduce_noalloc_set_barrier_limit_ns.restype = C.c_int
    return L.lhl_reduce_noalloc_check, L.lhl_reduce_noalloc_set_barrier_limit_ns


def _outputs(n):
    import torch
    F = torch.empty((n, n), dtype=torch.float64, device="cuda").t()   # column-major
    H = torch.empty((n, n), dtype=torch.float64, device="cuda").t()
    ip = torch.zeros(max(n - 2, 1), dtype=torch.int64, device="cuda")
    pm = torch.zeros(n, dtype=torch.int64, device="cuda")
    ipm = torch.zeros(n, dtype=torch.int64, device="cuda")
    sc = torch.zeros(n, dtype=torch.float64, device="cuda")
    isc = torch.zeros(n, dtype=torch.float64, device="cuda")
    return F, H, ip, pm, ipm, sc, isc


def _bits(t):
    return t.detach().cpu().numpy().view(np.int64)


# 1 and 2: no elimination step (dipiv may be NULL); 3: the smallest unblocked case; odd orders take
# the blocked path's plain loads, even ones its TMA boxes; 1024 fills the scratch to its bounds
@pytest.mark.parametrize("n", [1, 2, 3, 400, 499, 501, 600, 1023, 1024])
def test_noalloc_matches_workspace_reduction_twice(n):
    import torch
    import lhl_gpu as G
    f = _noalloc_fn()
    check, _ = _check_fn()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):
        rng = np.random.default_rng(100 * n + call)
        J = torch.as_tensor(np.asfortranarray(rng.standard_normal((n, n)))).cuda()
        ws = G.lhl(J)  # the existing, allocating entry point
        ws.check()
        F, H, ip, pm, ipm, sc, isc = _outputs(n)
        dip = ip.data_ptr() if n > 2 else None
        rc = f(n, J.data_ptr(), n, 1, F.data_ptr(), H.data_ptr(), dip, pm.data_ptr(), ipm.data_ptr(),
               sc.data_ptr(), isc.data_ptr(), stream)
        assert rc == 0
        assert check(stream) == 0
        torch.cuda.synchronize()
        if n > 2:
            assert np.array_equal(ip[: n - 2].cpu().numpy(), ws.ipiv.cpu().numpy())
        assert np.array_equal(_bits(F), _bits(ws.factors))
        assert np.array_equal(_bits(H), _bits(ws.Ht))
        assert np.array_equal(pm.cpu().numpy(), ws.perm.cpu().numpy())
        assert np.array_equal(ipm.cpu().numpy(), ws.iperm.cpu().numpy())
        assert np.array_equal(_bits(sc), _bits(ws.scale))
        assert np.array_equal(_bits(isc), _bits(ws.iscale))


def test_noalloc_reports_an_expired_wait_then_recovers():
    """A 1 ns wait limit makes the blocked reduction give up at its first grid barrier; the check
    entry point returns LHL_ERR_TIMEOUT once (then the word is clear), and with the default
    limit back the next call is bit-identical to the workspace's reduction."""
    import torch
    import lhl_gpu as G
    f = _noalloc_fn()
    check, set_limit = _check_fn()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    n = 600
    rng = np.random.default_rng(7)
    J = torch.as_tensor(np.asfortranarray(rng.standard_normal((n, n)))).cuda()
    F, H, ip, pm, ipm, sc, isc = _outputs(n)
    args = (n, J.data_ptr(), n, 1, F.data_ptr(), H.data_ptr(), ip.data_ptr(), pm.data_ptr(), ipm.data_ptr(),
            sc.data_ptr(), isc.data_ptr(), stream)
    try:
        assert set_limit(1) == 0
        assert f(*args) == 0
        assert check(stream) == 4           # LHL_ERR_TIMEOUT
        assert check(stream) == 0           # read once, then cleared
    finally:
        set_limit(0)
    assert f(*args) == 0
    assert check(stream) == 0
    ws = G.lhl(J)
    ws.check()
    assert np.array_equal(ip[: n - 2].cpu().numpy(), ws.ipiv.cpu().numpy())
    assert np.array_equal(_bits(F), _bits(ws.factors))


def test_noalloc_rejects_sizes_beyond_its_maximum():
    import torch
    f = _noalloc_fn()
    x = torch.zeros(4, dtype=torch.float64, device="cuda")
    p = x.data_ptr()
    assert f(1025, p, 1025, 1, p, p, p, p, p, p, p, None) == 2   # LHL_ERR_DIM
    assert f(-1, p, 1, 1, p, p, p, p, p, p, p, None) == 2
