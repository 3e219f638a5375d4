"""Python host mirror of LHLFactorization.jl's API over liblhl_gpu.so (sm_100a).

The Julia names map one to one (a trailing underscore marks the mutating `!` forms):

    lhl(J; balance)                 -> lhl(J, balance=True)            (src/LHLFactorization.jl:3179)
    lhl!(ws, J; balance)            -> lhl_(ws, J, balance=True)       (:3192)
    lhl_reduce!(ws, J, balance)     -> lhl_reduce_(ws, J, balance)     (:355)
    lhl_shift!(ws, sigma, tau)      -> lhl_shift_(ws, sigma, tau)      (:2456)
    lhl_shift!(sh, ws, sigma, tau)  -> lhl_shift_(sh, ws, sigma, tau)  (:2461)
    lhl_ldiv!(x, ws) / (x, sh, ws)  -> lhl_ldiv_(x, ws) / (x, sh, ws)  (:3052-3054)
    lhl_refine!(x, A, b, ws, steps) -> lhl_refine_(x, J, b, ws, steps) (:3144; A = sigma I + tau J)
    applyZ!(x, ws) / applyZinv!     -> applyZ_(x, ws) / applyZinv_      (:2069, :2104)

Arrays are torch CUDA float64 tensors.  Matrices may have any strides; vectors and the
columns of an (n, k) right-hand-side block are solved in place.  Mutating calls return
their first mutated argument, as in the reference.  Errors mirror the reference:
ArgumentError and DimensionMismatch (both ValueError subclasses).

There is no CPU fallback: importing this module without liblhl_gpu.so, or calling it
without a CUDA device, raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(os.path.dirname(_HERE), "liblhl_gpu.so")

LHL_OK, LHL_ERR_ARG, LHL_ERR_DIM, LHL_ERR_CUDA, LHL_ERR_TIMEOUT, LHL_ERR_ALLOC = range(6)
LHL_PREC_FP64, LHL_PREC_MIXED = 0, 1
# the arrays a reduction leaves in a workspace, in lhl_ws_import's argument order
REDUCTION_ARRAYS = ("factors", "Ht", "ipiv", "perm", "iperm", "scale", "iscale")


class ArgumentError(ValueError):
    pass


class DimensionMismatch(ValueError):
    pass


class LHLDeviceError(RuntimeError):
    pass


class _WsView(C.Structure):
    _fields_ = [("n", C.c_int64), ("factors", C.c_void_p), ("Ht", C.c_void_p), ("ipiv", C.c_void_p),
                ("perm", C.c_void_p), ("iperm", C.c_void_p), ("scale", C.c_void_p), ("iscale", C.c_void_p)]


class _ShView(C.Structure):
    _fields_ = [("n", C.c_int64), ("nshifts", C.c_int64), ("ldg", C.c_int64), ("Gt", C.c_void_p),
                ("swap", C.c_void_p), ("rdiag", C.c_void_p), ("info", C.c_void_p), ("sigma", C.c_void_p),
                ("tau", C.c_void_p), ("po", C.c_int64), ("is_complex", C.c_int32)]


def _load():
    if not os.path.exists(_LIB_PATH):
        raise ImportError(f"liblhl_gpu.so not built ({_LIB_PATH}); run lhl.jl_b200/build.py")
    L = C.CDLL(_LIB_PATH)
    vp, i64, i32, d = C.c_void_p, C.c_int64, C.c_int, C.c_double
    sig = {
        "lhl_ws_create": [i64, i32, C.POINTER(vp)],
        "lhl_ws_destroy": [vp],
        "lhl_ws_get_view": [vp, C.POINTER(_WsView)],
        "lhl_ws_check": [vp, vp],
        "lhl_ws_set_barrier_limit_ns": [vp, C.c_uint64],
        "lhl_ws_set_mixed_kernel": [vp, i32],
        "lhl_ws_set_shift_variant": [vp, i32, i32],
        "lhl_shift_variant_shape": [i32, i32, C.POINTER(C.c_int), C.POINTER(C.c_int)],
        "lhl_reduce": [vp, vp, i64, i32, vp],
        "lhl_ws_phase_ns": [vp, C.POINTER(C.c_uint64), vp],
        "lhl_ws_probe_ns": [vp, C.POINTER(C.c_uint64), vp],
        "lhl_ws_set_probes": [vp, i32],
        "lhl_ws_import": [vp, vp, vp, vp, vp, vp, vp, vp, vp],
        "lhl_ws_create_f32": [i64, i32, C.POINTER(vp)],
        "lhl_reduce_f32": [vp, vp, i64, i32, vp],
        "lhl_ldiv_f32": [vp, vp, vp, i64, i64, i64, vp],
        "lhl_ws_create_c128": [i64, C.POINTER(vp)],
        "lhl_ws_create_c64": [i64, C.POINTER(vp)],
        "lhl_refine_system": [vp, vp, i64, vp, i64, vp, i64, vp, i64, vp, vp, i64, d, i32, vp],
        "lhl_refine_system_gmres": [vp, vp, i64, vp, i64, vp, i64, vp, i64, vp, vp, i64, d, i32, i32, i32, vp],
        "lhl_reduce_c128": [vp, vp, i64, i32, vp],
        "lhl_reduce_c64": [vp, vp, i64, i32, vp],
        "lhl_shift_create_f32": [i64, i64, C.POINTER(vp)],
        "lhl_shift_create_complex64": [i64, i64, C.POINTER(vp)],
        "lhl_ldiv_complex_rhs": [vp, vp, vp, i64, i64, i64, vp],
        "lhl_shift_create": [i64, i64, C.POINTER(vp)],
        "lhl_shift_destroy": [vp],
        "lhl_shift_get_view": [vp, C.POINTER(_ShView)],
        "lhl_shift_batched": [vp, vp, i64, i64, vp, vp, vp],
        "lhl_shift": [vp, vp, i64, d, d, vp],
        "lhl_shift_create_complex": [i64, i64, C.POINTER(vp)],
        "lhl_batch_create": [i64, vp, i64, C.POINTER(vp)],
        "lhl_batch_destroy": [vp],
        "lhl_batch_get_view": [vp, vp],
        "lhl_reduce_batched": [vp, vp, i32, vp],
        "lhl_shift_batched_all": [vp, vp, vp, vp],
        "lhl_solve_batched": [vp, vp, vp, vp, i64, d, i32, vp, vp],
        "lhl_shift_complex": [vp, vp, i64, d, d, d, d, vp],
        "lhl_shift_batched_complex": [vp, vp, i64, i64, vp, vp, vp],
        "lhl_ldiv": [vp, vp, vp, i64, i64, i64, vp],
        "lhl_refine": [vp, vp, vp, i64, vp, i64, vp, i64, vp, i64, i64, i32, vp],
        "lhl_refine_tol": [vp, vp, vp, i64, vp, i64, vp, i64, vp, vp, i64, i64, d, i32, vp],
        "lhl_refine_gmres": [vp, vp, vp, i64, vp, i64, vp, i64, vp, vp, i64, i64, d, i32, i32, i32, vp],
        "lhl_residual_norms": [vp, vp, i64, vp, i64, vp, i64, vp, vp, i64, i64, vp],
        "lhl_applyZ": [vp, vp, i64, i64, vp],
        "lhl_applyZinv": [vp, vp, i64, i64, vp],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int
    L.lhl_version.restype = C.c_char_p
    return L


_lib = _load()


def lib():
    return _lib


def _check(rc, what=""):
    if rc == LHL_OK:
        return
    if rc == LHL_ERR_ARG:
        raise ArgumentError(what)
    if rc == LHL_ERR_DIM:
        raise DimensionMismatch(what)
    if rc == LHL_ERR_TIMEOUT:
        raise LHLDeviceError(f"{what}: a bounded grid-barrier wait expired")
    if rc == LHL_ERR_ALLOC:
        raise MemoryError(what)
    raise LHLDeviceError(f"{what}: CUDA error (status {rc})")


def _stream(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


class _BatchView(C.Structure):
    _fields_ = [("count", C.c_int64), ("shifts", C.c_int64), ("total_n", C.c_int64), ("total_nn", C.c_int64),
                ("total_g", C.c_int64), ("factors", C.c_void_p), ("Ht", C.c_void_p), ("ipiv", C.c_void_p),
                ("perm", C.c_void_p), ("iperm", C.c_void_p), ("scale", C.c_void_p), ("iscale", C.c_void_p),
                ("Gt", C.c_void_p), ("swap", C.c_void_p), ("rdiag", C.c_void_p), ("info", C.c_void_p),
                ("sigma", C.c_void_p), ("tau", C.c_void_p)]


class _DevArray:
    """A zero-copy torch view of device memory owned by the library."""

    def __init__(self, ptr, shape, dtype, strides=None):
        self.__cuda_array_interface__ = {
            "shape": tuple(shape), "typestr": dtype, "data": (int(ptr or 0), False), "version": 3,
            "strides": strides,
        }


def _view(ptr, shape, typestr="<f8", strides=None):
    if any(s == 0 for s in shape):
        return torch.empty(shape, dtype={"<f8": torch.float64, "<i8": torch.int64, "|u1": torch.uint8,
                                         "<i4": torch.int32, "<c16": torch.complex128}[typestr], device="cuda")
    return torch.as_tensor(_DevArray(ptr, shape, typestr, strides), device="cuda")


def _colmajor(M: torch.Tensor) -> torch.Tensor:
    """A tensor whose memory is M in column-major order with leading dimension rows."""
    if M.dim() != 2:
        raise DimensionMismatch("matrix expected")
    if M.stride(0) == 1 and M.stride(1) >= max(M.shape[0], 1):
        return M
    return M.t().contiguous().t()


def _require_cuda_f64(x: torch.Tensor, name: str, cplx: bool = False):
    if not isinstance(x, torch.Tensor) or not x.is_cuda:
        raise ArgumentError(f"{name} must be a CUDA tensor")
    want = torch.complex128 if cplx else torch.float64
    if x.dtype != want:
        if cplx:
            raise ArgumentError(f"{name} must be complex128: a real vector cannot hold the solution of a "
                                "complex shift (F:3084-3085)")
        raise ArgumentError(f"{name} must be float64 (complex shifts need an LHLShift built for them)")


def _require_cuda_real(x: torch.Tensor, name: str):
    if not isinstance(x, torch.Tensor) or not x.is_cuda:
        raise ArgumentError(f"{name} must be a CUDA tensor")
    if x.dtype not in (torch.float64, torch.float32):
        raise ArgumentError(f"{name} must be float64 or float32")


def _shift_creator(complex_: bool, single: bool):
    if single:
        return _lib.lhl_shift_create_complex64 if complex_ else _lib.lhl_shift_create_f32
    return _lib.lhl_shift_create_complex if complex_ else _lib.lhl_shift_create


class LHLShift:
    """``LHLShift{Float64}(n)`` or, with ``complex=True``, ``LHLShift{ComplexF64}(n)`` on a real
    reduction: a batch of ``nshifts`` shift slots (src/LHLFactorization.jl:84-116).  A complex
    shift object's Gt is planar: (2 po) x n per slot, real parts in rows 0..n-1, imaginary
    parts in rows po..po+n-1.  ``single=True`` makes ``LHLShift{Float32}`` /
    ``LHLShift{ComplexF32}``, the shift objects of single-precision workspaces; given a workspace
    instead of an order (``LHLShift{TG}(ws)``), the precision is the workspace's.  An
    ``LHLShift{TG}`` serves an ``LHLWorkspace{T}`` only for TG = T or Complex{real(T)}."""

    def __init__(self, n, nshifts: int = 1, complex: bool = False, single: bool = None):
        if isinstance(n, LHLWorkspace):
            if single is None:
                single = n.single
            n = n.n
        self.single = bool(single)
        self._h = C.c_void_p()
        _check(_shift_creator(complex, self.single)(int(n), int(nshifts), C.byref(self._h)), "LHLShift")
        self.n = int(n)
        self.nshifts = int(nshifts)
        v = _ShView()
        _check(_lib.lhl_shift_get_view(self._h, C.byref(v)))
        self._v = v
        self.is_complex = bool(v.is_complex)
        self.po = int(v.po)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.lhl_shift_destroy(h)
            self._h = None

    def _resize(self, n: int) -> "LHLShift":
        """``_lhl_resize!(sh, n)`` (F:277-292): the same slots and shift type at order n; the
        slots' factorisations are dropped.  The device object is replaced."""
        n = int(n)
        if n == self.n:
            return self
        h = C.c_void_p()
        _check(_shift_creator(self.is_complex, self.single)(n, self.nshifts, C.byref(h)), "LHLShift")
        old, self._h = self._h, h
        if old is not None and old.value:
            _lib.lhl_shift_destroy(old)
        v = _ShView()
        _check(_lib.lhl_shift_get_view(self._h, C.byref(v)))
        self._v = v
        self.n = n
        self.po = int(v.po)
        return self

    @property
    def ldg(self):
        return int(self._v.ldg)

    def Gt(self, slot: int = 0) -> torch.Tensor:
        n, ldg = self.n, self.ldg
        base = self._v.Gt + 8 * slot * ldg * n
        return _view(base, (ldg, n), strides=(8, 8 * ldg))

    def swap(self, slot: int = 0) -> torch.Tensor:
        return _view(self._v.swap + slot * self.n, (self.n,), "|u1")

    def rdiag(self, slot: int = 0) -> torch.Tensor:
        if self.is_complex:
            return torch.view_as_complex(_view(self._v.rdiag + 16 * slot * self.n, (self.n, 2)))
        return _view(self._v.rdiag + 8 * slot * self.n, (self.n,))

    @property
    def info_all(self) -> torch.Tensor:
        return _view(self._v.info, (self.nshifts,), "<i4")

    @property
    def sigma_all(self) -> torch.Tensor:
        if self.is_complex:
            return torch.view_as_complex(_view(self._v.sigma, (self.nshifts, 2)))
        return _view(self._v.sigma, (self.nshifts,))

    @property
    def tau_all(self) -> torch.Tensor:
        if self.is_complex:
            return torch.view_as_complex(_view(self._v.tau, (self.nshifts, 2)))
        return _view(self._v.tau, (self.nshifts,))

    @property
    def info(self) -> int:
        torch.cuda.current_stream().synchronize()
        return int(self.info_all[0].item())

    @property
    def σ(self):
        v = self.sigma_all[0].item()
        return v if self.is_complex else float(v)

    @property
    def τ(self):
        v = self.tau_all[0].item()
        return v if self.is_complex else float(v)


class LHLWorkspace:
    """``LHLWorkspace{T}(n)`` on the device (src/LHLFactorization.jl:144-178), T = Float64
    (``dtype=torch.float64``), Float32 or ComplexF64 (``dtype=torch.complex128``: a complex J,
    whose shifts are complex; its factors and Ht are complex128 views).

    Holds the reduction and, in ``.shift``, one shift slot (the reference's ``ws.shift``);
    the shift fields are forwarded as in the reference (F:182-191)."""

    _SHIFT_FIELDS = ("Gt", "rdiag", "swap", "info", "σ", "τ")

    def __init__(self, n: int, precision: int = LHL_PREC_FP64, shift_complex: bool = False,
                 dtype: torch.dtype = torch.float64):
        self._h = C.c_void_p()
        if dtype == torch.float32:  # LHLWorkspace{Float32}; shift_complex: LHLShift{ComplexF32}
            _check(_lib.lhl_ws_create_f32(int(n), int(precision), C.byref(self._h)), "LHLWorkspace")
        elif dtype == torch.float64:
            _check(_lib.lhl_ws_create(int(n), int(precision), C.byref(self._h)), "LHLWorkspace")
        elif dtype in (torch.complex128, torch.complex64):  # LHLWorkspace{ComplexF64 / ComplexF32} (F:164-169)
            if precision != LHL_PREC_FP64:
                raise ArgumentError("a complex workspace has the FP64 form only")
            create = _lib.lhl_ws_create_c128 if dtype == torch.complex128 else _lib.lhl_ws_create_c64
            _check(create(int(n), C.byref(self._h)), "LHLWorkspace")
            shift_complex = True
        else:
            raise ArgumentError(f"element type {dtype} is not supported (float64, float32, complex128 or complex64)")
        self.dtype = dtype
        self.cj = dtype in (torch.complex128, torch.complex64)  # a complex J (its factors are complex128 views)
        self.single = dtype in (torch.float32, torch.complex64)  # Float32 / ComplexF32 element type
        self.device = torch.device("cuda", torch.cuda.current_device())  # where its arrays live
        self.n = int(n)
        self.precision = precision
        self.shift_complex = bool(shift_complex)
        v = _WsView()
        _check(_lib.lhl_ws_get_view(self._h, C.byref(v)))
        self._v = v
        # ws.shift: LHLShift{Float64}, or LHLShift{ComplexF64} for shift = Complex{T} (F:164-178)
        self.shift = LHLShift(self.n, 1, complex=self.shift_complex, single=self.single)
        self.reduced = False

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.lhl_ws_destroy(h)
            self._h = None

    def _resize(self, n: int) -> "LHLWorkspace":
        """``_lhl_resize!(ws, n)`` (F:256-275): a workspace of order n in place of this one, with
        the same form, element type and shift type; the reduction is dropped and ``ws.shift``
        takes the new order.  The device workspace is replaced; probe and wait-limit settings
        carry over."""
        n = int(n)
        if n == self.n:
            return self
        new = LHLWorkspace(n, self.precision, self.shift_complex, dtype=self.dtype)
        old, self._h = self._h, new._h
        new._h = None  # the handle now belongs to self
        if old is not None and old.value:
            _lib.lhl_ws_destroy(old)
        self._v = new._v
        self.n = n
        self.shift = new.shift
        self.reduced = False
        self.__dict__.pop("_J_keepalive", None)
        if self.__dict__.get("_probes"):
            _check(_lib.lhl_ws_set_probes(self._h, 1), "set_probes")
        if self.__dict__.get("_limit_ns") is not None:
            _check(_lib.lhl_ws_set_barrier_limit_ns(self._h, int(self._limit_ns)))
        if self.__dict__.get("_mixed_kernel"):
            _check(_lib.lhl_ws_set_mixed_kernel(self._h, int(self._mixed_kernel)), "set_mixed_kernel")
        sv = self.__dict__.get("_shift_variant")
        if sv:  # launch shapes chosen for the old order serve the new one only if they still cover it
            rv = sv[0] if sv[0] in shift_variants(False, n) else 0
            cv = sv[1] if sv[1] in shift_variants(True, n) else 0
            self.set_shift_variant(rv, cv)
        return self

    def __getattr__(self, name):
        if name in LHLWorkspace._SHIFT_FIELDS:
            sh = self.__dict__["shift"]
            a = getattr(sh, name)
            return a() if callable(a) else a
        raise AttributeError(name)

    # device views (column-major n x n tensors are returned as (n, n) with strides (1, n))
    @property
    def factors(self) -> torch.Tensor:
        n = self.n
        if self.cj:
            return _view(self._v.factors, (n, n), "<c16", strides=(16, 16 * n))
        return _view(self._v.factors, (n, n), strides=(8, 8 * n))

    @property
    def Ht(self) -> torch.Tensor:
        n = self.n
        if self.cj:
            return _view(self._v.Ht, (n, n), "<c16", strides=(16, 16 * n))
        return _view(self._v.Ht, (n, n), strides=(8, 8 * n))

    @property
    def ipiv(self) -> torch.Tensor:
        return _view(self._v.ipiv, (max(self.n - 2, 0),), "<i8")

    @property
    def perm(self) -> torch.Tensor:
        return _view(self._v.perm, (self.n,), "<i8")

    @property
    def iperm(self) -> torch.Tensor:
        return _view(self._v.iperm, (self.n,), "<i8")

    @property
    def scale(self) -> torch.Tensor:
        return _view(self._v.scale, (self.n,))

    @property
    def iscale(self) -> torch.Tensor:
        return _view(self._v.iscale, (self.n,))

    def check(self, stream=None):
        """Wait for the stream and raise a device-side error recorded by the last reduction."""
        _check(_lib.lhl_ws_check(self._h, _stream(stream)), "lhl_reduce")

    def phase_ns(self, stream=None):
        """Device wall time of the last reduction by phase (see lhl_ws_phase_ns)."""
        buf = (C.c_uint64 * 8)()
        _check(_lib.lhl_ws_phase_ns(self._h, buf, _stream(stream)), "phase_ns")
        names = ["balance", "pivot_gemv", "rows", "panel_swaps_trsm", "panel_gemm", "barrier_wait_cta0",
                 "step_table_cta0", "total"]
        return {nm: buf[i] for i, nm in enumerate(names) if nm}

    def probe_ns(self, stream=None):
        buf = (C.c_uint64 * 16)()
        _check(_lib.lhl_ws_probe_ns(self._h, buf, _stream(stream)), "probe_ns")
        return list(buf)

    def save(self, path: str, stream=None):
        """Write the reduction (factors, Ht, ipiv, perm, iperm, scale, iscale) and the
        workspace's order and precision to an .npz file; `load` restores it."""
        if not self.reduced:
            raise ArgumentError("the workspace holds no reduction")
        torch.cuda.current_stream().synchronize() if stream is None else stream.synchronize()
        np.savez(path, n=self.n, precision=self.precision, shift_complex=self.shift_complex,
                 f32=self.dtype == torch.float32, c128=self.dtype == torch.complex128,
                 c64=self.dtype == torch.complex64,
                 factors=self.factors.cpu().numpy(), Ht=self.Ht.cpu().numpy(), ipiv=self.ipiv.cpu().numpy(),
                 perm=self.perm.cpu().numpy(), iperm=self.iperm.cpu().numpy(), scale=self.scale.cpu().numpy(),
                 iscale=self.iscale.cpu().numpy())

    @classmethod
    def load(cls, path: str, stream=None) -> "LHLWorkspace":
        """A workspace holding the reduction saved by `save` (lhl_ws_import of the C ABI)."""
        d = np.load(path)
        dt = torch.float64
        if "f32" in d and bool(d["f32"]):
            dt = torch.float32
        elif "c128" in d and bool(d["c128"]):
            dt = torch.complex128
        elif "c64" in d and bool(d["c64"]):
            dt = torch.complex64
        ws = cls(int(d["n"]), int(d["precision"]), bool(d["shift_complex"]), dtype=dt)
        ws.import_arrays({k: torch.as_tensor(np.asarray(d[k])).cuda() for k in REDUCTION_ARRAYS}, stream)
        (stream or torch.cuda.current_stream()).synchronize()
        return ws

    def import_arrays(self, arrays, stream=None) -> "LHLWorkspace":
        """Take a reduction made elsewhere (lhl_ws_import of the C ABI): `arrays` maps the names
        of REDUCTION_ARRAYS to CUDA tensors, factors and Ht (n, n) of the workspace's element
        storage (complex128 for a complex J, float64 otherwise), ipiv (n-2), perm and iperm (n)
        int64, scale and iscale (n) float64.  Copies are taken on the stream; the arrays may be
        released once it has passed them."""
        n = self.n
        mat = torch.complex128 if self.cj else torch.float64
        want = {"factors": (mat, (n, n)), "Ht": (mat, (n, n)), "ipiv": (torch.int64, (max(n - 2, 0),)),
                "perm": (torch.int64, (n,)), "iperm": (torch.int64, (n,)), "scale": (torch.float64, (n,)),
                "iscale": (torch.float64, (n,))}
        dev = {}
        for k in REDUCTION_ARRAYS:
            t = arrays[k]
            dt, shape = want[k]
            if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != dt:
                raise ArgumentError(f"{k} must be a CUDA {dt} tensor")
            if tuple(t.shape) != shape:
                raise DimensionMismatch(f"{k} has shape {tuple(t.shape)}, expected {shape}")
            if t.dim() == 2:  # column-major with leading dimension n
                dev[k] = t if (t.stride(0) == 1 and t.stride(1) == n) else t.t().contiguous().t()
            else:
                dev[k] = t.contiguous()
        if n:
            _check(_lib.lhl_ws_import(self._h, *[C.c_void_p(dev[k].data_ptr()) for k in REDUCTION_ARRAYS],
                                      _stream(stream)), "lhl_ws_import")
        self.reduced = True
        return self

    def set_probes(self, on: bool = True):
        """Record the reduction's device timers (phase_ns, probe_ns); off by default."""
        _check(_lib.lhl_ws_set_probes(self._h, int(bool(on))), "set_probes")
        self._probes = bool(on)

    def set_mixed_kernel(self, which: int):
        """Test hook (mixed form): 0 by the order, 1 the eager FP32 kernel, 2 the panel-delayed one."""
        _check(_lib.lhl_ws_set_mixed_kernel(self._h, int(which)), "set_mixed_kernel")
        self._mixed_kernel = int(which)

    def set_barrier_limit_ns(self, ns: int):
        _check(_lib.lhl_ws_set_barrier_limit_ns(self._h, int(ns)))
        self._limit_ns = int(ns)

    def set_shift_variant(self, real_variant: int = 0, complex_variant: int = 0):
        """Launch shape of the shift LU for shifts on this workspace (0: by the order; see
        shift_variants).  Every shape gives the same bits."""
        _check(_lib.lhl_ws_set_shift_variant(self._h, int(real_variant), int(complex_variant)), "set_shift_variant")
        self._shift_variant = (int(real_variant), int(complex_variant))


def shift_variant_shape(is_complex: bool, variant: int):
    """(threads, elements per thread) of shift-LU launch shape `variant`, or None past the last."""
    T, E = C.c_int(), C.c_int()
    if _lib.lhl_shift_variant_shape(int(bool(is_complex)), int(variant), C.byref(T), C.byref(E)) != LHL_OK:
        return None
    return T.value, E.value


def shift_variants(is_complex: bool, n: int):
    """The shift-LU launch shapes (1-based) that serve order n (threads x elements >= n)."""
    out, v = [], 1
    while True:
        sh = shift_variant_shape(is_complex, v)
        if sh is None:
            return out
        if sh[0] * sh[1] >= n:
            out.append(v)
        v += 1


# ---------------------------------------------------------------------------------------
def lhl_reduce_(ws: LHLWorkspace, J: torch.Tensor, balance: bool, thread=True, stream=None) -> LHLWorkspace:
    """``lhl_reduce!(ws, J, balance)`` (F:355).  J is not modified.  A workspace of another
    order is resized to J's first, as the reference does (F:357)."""
    if ws.cj and isinstance(J, torch.Tensor) and J.dtype == torch.complex64:
        if not J.is_cuda:
            raise ArgumentError("J must be a CUDA tensor")
    elif ws.cj:
        _require_cuda_f64(J, "J", True)
    elif isinstance(J, torch.Tensor) and J.dtype == torch.float32:
        _require_cuda_real(J, "J")
    else:
        _require_cuda_f64(J, "J")
    if J.dim() != 2 or J.shape[0] != J.shape[1]:
        raise DimensionMismatch(f"matrix is not square: dimensions are {tuple(J.shape)}")
    ws._resize(J.shape[0])
    Jc = _colmajor(J)
    ld = max(Jc.stride(1), 1)
    fn = _lib.lhl_reduce_f32 if Jc.dtype == torch.float32 else _lib.lhl_reduce
    if Jc.dtype == torch.complex128:
        fn = _lib.lhl_reduce_c128
    elif Jc.dtype == torch.complex64:
        fn = _lib.lhl_reduce_c64
    _check(fn(ws._h, C.c_void_p(Jc.data_ptr()), ld, int(bool(balance)), _stream(stream)), "lhl_reduce")
    ws.reduced = True
    ws._J_keepalive = Jc
    return ws


def lhl(J: torch.Tensor, balance: bool = True, thread=True, precision: int = LHL_PREC_FP64,
        shift_complex: bool = False, stream=None) -> LHLWorkspace:
    """``lhl(J; balance=true, shift=...)`` (F:3179): allocate a workspace and reduce J into it;
    ``shift_complex=True`` is ``shift = ComplexF64`` (complex shifts on the real reduction); a
    complex128 J makes an ``LHLWorkspace{ComplexF64}``, a complex64 one an ``LHLWorkspace{ComplexF32}``."""
    if isinstance(J, torch.Tensor) and J.dtype == torch.complex128:
        _require_cuda_f64(J, "J", True)
    elif isinstance(J, torch.Tensor) and J.dtype == torch.complex64:
        if not J.is_cuda:
            raise ArgumentError("J must be a CUDA tensor")
    else:
        _require_cuda_real(J, "J")
    if J.dim() != 2 or J.shape[0] != J.shape[1]:
        raise DimensionMismatch(f"matrix is not square: dimensions are {tuple(J.shape)}")
    ws = LHLWorkspace(J.shape[0], precision, shift_complex, dtype=J.dtype)
    return lhl_reduce_(ws, J, balance, thread, stream)


def lhl_(ws: LHLWorkspace, J: torch.Tensor, balance: bool = True, thread=True, stream=None) -> LHLWorkspace:
    """``lhl!(ws, J; balance)`` (F:3192).  A workspace of another order is resized in place."""
    return lhl_reduce_(ws, J, balance, thread, stream)


def _shift_args(a):
    if len(a) == 3:
        ws, sigma, tau = a
        return ws.shift, ws, sigma, tau, ws
    if len(a) == 4:
        sh, ws, sigma, tau = a
        return sh, ws, sigma, tau, sh
    raise TypeError("lhl_shift_(ws, sigma, tau) or lhl_shift_(sh, ws, sigma, tau)")


def lhl_shift_(*args, slot: int = 0, stream=None):
    """``lhl_shift!(ws, sigma, tau)`` / ``lhl_shift!(sh, ws, sigma, tau)`` (F:2456-2489)."""
    sh, ws, sigma, tau, ret = _shift_args(args)
    if ws.cj and not sh.is_complex:
        raise ArgumentError("an LHLShift{Float64} cannot serve a workspace of element type ComplexF64")
    if not sh.is_complex:
        for v in (sigma, tau):
            if isinstance(v, complex) and v.imag != 0:
                raise ArgumentError(f"complex shift ({sigma}, {tau}) on a real LHLShift")
    sh._resize(ws.n)  # _lhl_resize!(sh, n), F:2476
    if sh.is_complex:
        sigma, tau = complex(sigma), complex(tau)
        _check(_lib.lhl_shift_complex(sh._h, ws._h, int(slot), sigma.real, sigma.imag, tau.real, tau.imag,
                                      _stream(stream)), "lhl_shift")
        return ret
    sigma = float(sigma.real if isinstance(sigma, complex) else sigma)
    tau = float(tau.real if isinstance(tau, complex) else tau)
    _check(_lib.lhl_shift(sh._h, ws._h, int(slot), sigma, tau, _stream(stream)), "lhl_shift")
    return ret


def lhl_shift_batched_(sh: LHLShift, ws: LHLWorkspace, sigmas: torch.Tensor, taus: torch.Tensor, s0: int = 0,
                       stream=None) -> LHLShift:
    """Load len(sigmas) shifts into slots s0.. of ``sh`` in one launch (device arrays; complex128
    arrays for complex shifts, which need a complex ``sh``)."""
    if sigmas.is_complex() or taus.is_complex():
        if not sh.is_complex:
            raise ArgumentError("complex shifts on a real LHLShift")
        sigmas = sigmas.to(torch.complex128).contiguous()
        taus = taus.to(torch.complex128).contiguous()
        if sigmas.numel() != taus.numel():
            raise DimensionMismatch("sigmas and taus differ in length")
        _check(_lib.lhl_shift_batched_complex(sh._h, ws._h, int(s0), sigmas.numel(), C.c_void_p(sigmas.data_ptr()),
                                              C.c_void_p(taus.data_ptr()), _stream(stream)), "lhl_shift_batched")
        return sh
    _require_cuda_f64(sigmas, "sigmas")
    _require_cuda_f64(taus, "taus")
    sigmas = sigmas.contiguous()
    taus = taus.contiguous()
    if sigmas.numel() != taus.numel():
        raise DimensionMismatch("sigmas and taus differ in length")
    _check(_lib.lhl_shift_batched(sh._h, ws._h, int(s0), sigmas.numel(), C.c_void_p(sigmas.data_ptr()),
                                  C.c_void_p(taus.data_ptr()), _stream(stream)), "lhl_shift_batched")
    return sh


def _as_cols(x: torch.Tensor, n: int):
    if x.dim() == 1:
        if x.shape[0] != n:
            raise DimensionMismatch(f"x has length {x.shape[0]}, the workspace is {n}x{n}")
        if x.stride(0) != 1 and n > 1:  # one element: any stride
            raise ArgumentError("x must be contiguous")
        return x, 1, n
    if x.dim() == 2:
        if x.shape[0] != n:
            raise DimensionMismatch(f"x has {x.shape[0]} rows, the workspace is {n}x{n}")
        if x.stride(0) != 1 and x.shape[1] > 1 and n > 1:  # one row: only the column stride counts
            raise ArgumentError("x must be column-major (stride (1, ld))")
        return x, x.shape[1], max(x.stride(1), n) if x.shape[1] > 1 else n
    raise DimensionMismatch("x must be a vector or an (n, k) block")


def _split_complex(v: torch.Tensor, n: int) -> torch.Tensor:
    """A complex (n,) or (n, k) tensor as real column pairs: (n, 2k) float64, column-major,
    column 2c holding the real parts of column c and 2c + 1 its imaginary parts."""
    k = 1 if v.dim() == 1 else v.shape[1]
    r = torch.empty((2 * k, n), dtype=torch.float64, device=v.device).t()
    r.unflatten(1, (k, 2)).copy_(torch.view_as_real(v.reshape(n, k)))
    return r


def _join_complex(r: torch.Tensor, v: torch.Tensor) -> None:
    """The inverse of _split_complex, into v."""
    n = r.shape[0]
    k = 1 if v.dim() == 1 else v.shape[1]
    torch.view_as_real(v.view(n, k) if v.dim() == 1 else v).copy_(r.unflatten(1, (k, 2)))


def lhl_ldiv_(x: torch.Tensor, *args, rhs_per_shift: int = 1, stream=None) -> torch.Tensor:
    """``lhl_ldiv!(x, ws)`` / ``lhl_ldiv!(x, sh, ws)`` (F:3052-3068).  Column j of an (n, k)
    block uses shift slot j // rhs_per_shift."""
    if len(args) == 1:
        ws = args[0]
        sh = ws.shift
    else:
        sh, ws = args
    if x.is_complex() and not sh.is_complex:
        # the generic path (F:3052-3074): a real shift solves the real and imaginary parts
        if sh.n != ws.n:
            raise DimensionMismatch(f"the LHLShift is {sh.n}x{sh.n}, the workspace {ws.n}x{ws.n}")
        if not x.is_cuda:
            raise ArgumentError("x must be a CUDA tensor")
        xd = x if x.dtype == torch.complex128 else x.to(torch.complex128)
        xx, k, ld = _as_cols(xd, ws.n)
        _check(_lib.lhl_ldiv_complex_rhs(sh._h, ws._h, C.c_void_p(xx.data_ptr()), ld, k, int(rhs_per_shift),
                                         _stream(stream)), "lhl_ldiv")
        if xd is not x:
            x.copy_(xd)
        return x
    if x.dtype == torch.float32 and not sh.is_complex:  # float vectors: widened, solved, rounded back
        _require_cuda_real(x, "x")
        fn = _lib.lhl_ldiv_f32
    elif x.dtype == torch.complex64 and sh.is_complex:  # ComplexF32 vectors, the same way
        if not x.is_cuda:
            raise ArgumentError("x must be a CUDA tensor")
        fn = _lib.lhl_ldiv_f32
    else:
        _require_cuda_f64(x, "x", sh.is_complex)
        fn = _lib.lhl_ldiv
    if sh.n != ws.n:
        raise DimensionMismatch(f"the LHLShift is {sh.n}x{sh.n}, the workspace {ws.n}x{ws.n}")
    xx, k, ld = _as_cols(x, ws.n)
    _check(fn(sh._h, ws._h, C.c_void_p(xx.data_ptr()), ld, k, int(rhs_per_shift), _stream(stream)), "lhl_ldiv")
    return x


def lhl_refine_(x: torch.Tensor, J: torch.Tensor, b: torch.Tensor, *args, steps: int = 1, rhs_per_shift: int = 1,
                stream=None) -> torch.Tensor:
    """``lhl_refine!(x, A, b, ws, steps)`` with A = sigma I + tau J given by J and the shift
    slot's (sigma, tau) (F:3144-3157).  Forms: (x, J, b, ws, steps) or (x, J, b, sh, ws, steps)."""
    if len(args) == 2:
        ws, steps = args
        sh = ws.shift
    elif len(args) == 3:
        sh, ws, steps = args
    elif len(args) == 1:
        ws = args[0]
        sh = ws.shift
    else:
        raise TypeError("lhl_refine_(x, J, b, ws, steps) or (x, J, b, sh, ws, steps)")
    if steps <= 0:
        return x
    _require_cuda_f64(J, "J", ws.cj)
    if not sh.is_complex and isinstance(x, torch.Tensor) and x.dtype == torch.complex128:
        # complex vectors on a real shift (the reference's generic path, F:3144-3157 with F:3052-3074):
        # A = sigma I + tau J is real, so the real and imaginary parts refine as two real columns
        _require_cuda_f64(b, "b", True)
        xr, br = _split_complex(x, ws.n), _split_complex(b, ws.n)
        lhl_refine_(xr, J, br, sh, ws, steps, rhs_per_shift=2 * rhs_per_shift, stream=stream)
        _join_complex(xr, x)
        return x
    for t, nm in ((x, "x"), (b, "b")):
        _require_cuda_f64(t, nm, sh.is_complex)
    n = ws.n
    xx, k, ldx = _as_cols(x, n)
    bb, kb, ldb = _as_cols(b, n)
    if kb != k:
        raise DimensionMismatch("x and b differ in column count")
    Jc = _colmajor(J)
    dt = torch.complex128 if sh.is_complex else torch.float64
    R = torch.empty((k, n), dtype=dt, device=x.device).t() if k > 1 else torch.empty(n, dtype=dt, device=x.device)
    ldr = n
    if ldx != ldr:
        raise ArgumentError("x must have leading dimension n")
    _check(_lib.lhl_refine(sh._h, ws._h, C.c_void_p(Jc.data_ptr()), max(Jc.stride(1), n), C.c_void_p(bb.data_ptr()),
                           ldb, C.c_void_p(xx.data_ptr()), ldx, C.c_void_p(R.data_ptr()), k, int(rhs_per_shift),
                           int(steps), _stream(stream)), "lhl_refine")
    return x


def lhl_refine_tol_(x: torch.Tensor, J: torch.Tensor, b: torch.Tensor, sh: LHLShift, ws: LHLWorkspace,
                    tol: float = 1e-10, max_steps: int = 8, rhs_per_shift: int = 1, R: torch.Tensor = None,
                    res: torch.Tensor = None, stream=None) -> torch.Tensor:
    """Refinement to a tolerance (lhl_refine_tol of the C ABI): up to `max_steps` steps of
    ``lhl_refine!`` (F:3144-3157); columns already at relative residual <= tol are skipped on
    the device.  Returns the per-column final relative residuals (device tensor); x is updated
    in place.  `R` (n x k scratch) and `res` (k) may be passed to avoid allocation."""
    _require_cuda_f64(J, "J", ws.cj)
    for t, nm in ((x, "x"), (b, "b")):
        _require_cuda_f64(t, nm, sh.is_complex)
    n = ws.n
    xx, k, ldx = _as_cols(x, n)
    bb, kb, ldb = _as_cols(b, n)
    if kb != k:
        raise DimensionMismatch("x and b differ in column count")
    if ldx != n:
        raise ArgumentError("x must have leading dimension n")
    Jc = _colmajor(J)
    if R is None:
        R = torch.empty((k, n), dtype=torch.complex128 if sh.is_complex else torch.float64, device=x.device)
    if res is None:
        res = torch.empty(k, dtype=torch.float64, device=x.device)
    if R.numel() < n * k or res.numel() < k:
        raise DimensionMismatch("scratch too small")
    _check(_lib.lhl_refine_tol(sh._h, ws._h, C.c_void_p(Jc.data_ptr()), max(Jc.stride(1), n),
                               C.c_void_p(bb.data_ptr()), ldb, C.c_void_p(xx.data_ptr()), ldx,
                               C.c_void_p(R.data_ptr()), C.c_void_p(res.data_ptr()), k, int(rhs_per_shift),
                               float(tol), int(max_steps), _stream(stream)), "lhl_refine_tol")
    return res


def lhl_refine_gmres_(x: torch.Tensor, J: torch.Tensor, b: torch.Tensor, sh: LHLShift, ws: LHLWorkspace,
                      tol: float = 1e-10, max_cycles: int = 4, restart: int = 8, rhs_per_shift: int = 1,
                      host_check: bool = True, R: torch.Tensor = None, res: torch.Tensor = None,
                      stream=None) -> torch.Tensor:
    """Refinement by GMRES-IR (lhl_refine_gmres of the C ABI): up to `max_cycles` cycles of
    GMRES(`restart`) on the correction equation, left-preconditioned by the shift's
    factorisation, for every column above relative residual `tol`.  Returns the per-column
    final relative residuals (device tensor); x is updated in place.  For complex shifts x and b
    are complex128 and GMRES runs on the realified system."""
    _require_cuda_f64(J, "J", ws.cj)
    for t, nm in ((x, "x"), (b, "b")):
        _require_cuda_f64(t, nm, sh.is_complex)
    n = ws.n
    xx, k, ldx = _as_cols(x, n)
    bb, kb, ldb = _as_cols(b, n)
    if kb != k:
        raise DimensionMismatch("x and b differ in column count")
    if ldx != n:
        raise ArgumentError("x must have leading dimension n")
    Jc = _colmajor(J)
    if R is None:
        R = torch.empty((k, n), dtype=torch.complex128 if sh.is_complex else torch.float64, device=x.device)
    if res is None:
        res = torch.empty(k, dtype=torch.float64, device=x.device)
    if R.numel() < n * k or res.numel() < k:
        raise DimensionMismatch("scratch too small")
    _check(_lib.lhl_refine_gmres(sh._h, ws._h, C.c_void_p(Jc.data_ptr()), max(Jc.stride(1), n),
                                 C.c_void_p(bb.data_ptr()), ldb, C.c_void_p(xx.data_ptr()), ldx,
                                 C.c_void_p(R.data_ptr()), C.c_void_p(res.data_ptr()), k, int(rhs_per_shift),
                                 float(tol), int(max_cycles), int(restart), int(bool(host_check)),
                                 _stream(stream)), "lhl_refine_gmres")
    return res


def lhl_refine_system_(x: torch.Tensor, A: torch.Tensor, b: torch.Tensor, *args, slot: int = 0, tol: float = 0.0,
                       gmres: bool = False, restart: int = 8, host_check: bool = True, R: torch.Tensor = None,
                       res: torch.Tensor = None, stream=None) -> torch.Tensor:
    """``lhl_refine!(x, A, b, ws, steps)`` / ``lhl_refine!(x, A, b, sh, ws, steps)`` (F:3144-3157)
    with the caller's system matrix A, as the reference takes it: r = b - A x, lhl_ldiv! by shift
    slot ``slot``, x += r, ``steps`` times (tol = 0); with tol > 0 a column stops once its relative
    residual is <= tol (at most ``steps`` steps), and with ``gmres=True`` the steps are GMRES-IR
    cycles of GMRES(restart).  A may differ from sigma I + tau J (a mass matrix in W = J - M/gamma):
    the refinement converges to A^-1 b where the slot's factorisation is close enough to A.  Every
    column of x uses the same slot.  Returns x; ``res`` (if given) receives the final relative
    residuals."""
    if len(args) == 2:
        ws, steps = args
        sh = ws.shift
    elif len(args) == 3:
        sh, ws, steps = args
    else:
        raise TypeError("lhl_refine_system_(x, A, b, ws, steps) or (x, A, b, sh, ws, steps)")
    cplx = sh.is_complex
    if (not cplx and isinstance(x, torch.Tensor) and x.dtype == torch.complex128 and isinstance(A, torch.Tensor)
            and not A.is_complex()):
        # complex vectors, a real A and a real shift (the reference's generic path): the real and
        # imaginary parts refine as real columns of the same slot
        _require_cuda_f64(b, "b", True)
        xr, br = _split_complex(x, ws.n), _split_complex(b, ws.n)
        r2 = None if res is None else torch.empty(xr.shape[1], dtype=torch.float64, device=xr.device)
        lhl_refine_system_(xr, A, br, sh, ws, steps, slot=slot, tol=tol, gmres=gmres, restart=restart,
                           host_check=host_check, res=r2, stream=stream)
        _join_complex(xr, x)
        if res is not None:  # a complex column's residual from its two parts' (2-norms combine)
            part = torch.nan_to_num(r2 * br.norm(dim=0)).view(-1, 2)  # ||r_re||, ||r_im|| per column
            res.copy_(part.norm(dim=1) / torch.linalg.vector_norm(b.reshape(ws.n, -1), dim=0))
        return x
    _require_cuda_f64(A, "A", cplx)
    for t, nm in ((x, "x"), (b, "b")):
        _require_cuda_f64(t, nm, cplx)
    n = ws.n
    if A.dim() != 2 or tuple(A.shape) != (n, n):
        raise DimensionMismatch(f"A is {tuple(A.shape)}, the workspace is {n}x{n}")
    xx, k, ldx = _as_cols(x, n)
    bb, kb, ldb = _as_cols(b, n)
    if kb != k:
        raise DimensionMismatch("x and b differ in column count")
    if ldx != n:
        raise ArgumentError("x must have leading dimension n")
    Ac = _colmajor(A)
    dt = torch.complex128 if cplx else torch.float64
    if R is None:
        R = torch.empty((k, n), dtype=dt, device=x.device)
    if res is None:
        res = torch.empty(k, dtype=torch.float64, device=x.device)
    if R.numel() < n * k or res.numel() < k:
        raise DimensionMismatch("scratch too small")
    ptrs = (C.c_void_p(Ac.data_ptr()), max(Ac.stride(1), n), C.c_void_p(bb.data_ptr()), ldb,
            C.c_void_p(xx.data_ptr()), ldx, C.c_void_p(R.data_ptr()), C.c_void_p(res.data_ptr()), k, float(tol))
    if gmres:
        _check(_lib.lhl_refine_system_gmres(sh._h, ws._h, int(slot), *ptrs, int(steps), int(restart),
                                            int(bool(host_check)), _stream(stream)), "lhl_refine_system_gmres")
    else:
        _check(_lib.lhl_refine_system(sh._h, ws._h, int(slot), *ptrs, int(steps), _stream(stream)),
               "lhl_refine_system")
    return x


def residual_norms(sh: LHLShift, J: torch.Tensor, b: torch.Tensor, x: torch.Tensor, rhs_per_shift: int = 1,
                   stream=None) -> torch.Tensor:
    """||b - (sigma I + tau J) x||_2 / ||b||_2 per column, on the device (J complex128 when the
    slots were loaded from a complex reduction)."""
    n = sh.n
    xx, k, ldx = _as_cols(x, n)
    bb, _, ldb = _as_cols(b, n)
    Jc = _colmajor(J)
    R = torch.empty((k, n), dtype=torch.complex128 if sh.is_complex else torch.float64, device=x.device)
    out = torch.empty(k, dtype=torch.float64, device=x.device)
    _check(_lib.lhl_residual_norms(sh._h, C.c_void_p(Jc.data_ptr()), max(Jc.stride(1), n), C.c_void_p(bb.data_ptr()),
                                   ldb, C.c_void_p(xx.data_ptr()), ldx, C.c_void_p(R.data_ptr()),
                                   C.c_void_p(out.data_ptr()), k, int(rhs_per_shift), _stream(stream)),
           "residual_norms")
    return out


def applyZ_(x: torch.Tensor, ws: LHLWorkspace, stream=None) -> torch.Tensor:
    """``applyZ!(x, ws)``: x <- Z x (F:2069)."""
    _require_cuda_f64(x, "x", ws.cj)
    xx, k, ld = _as_cols(x, ws.n)
    _check(_lib.lhl_applyZ(ws._h, C.c_void_p(xx.data_ptr()), ld, k, _stream(stream)), "applyZ")
    return x


def applyZinv_(x: torch.Tensor, ws: LHLWorkspace, stream=None) -> torch.Tensor:
    """``applyZinv!(x, ws)``: x <- Z^-1 x (F:2104)."""
    _require_cuda_f64(x, "x", ws.cj)
    xx, k, ld = _as_cols(x, ws.n)
    _check(_lib.lhl_applyZinv(ws._h, C.c_void_p(xx.data_ptr()), ld, k, _stream(stream)), "applyZinv")
    return x


class LHLBatch:
    """Many independent real matrices of uneven order (n <= 512) with ``shifts`` shifts each:
    the batched form of ``lhl``, ``lhl_shift!``, ``lhl_ldiv!`` and ``lhl_refine!`` (one launch
    per phase; see lhl_batch_create in include/lhl_gpu.h for the packed layout)."""

    def __init__(self, ns, shifts: int):
        self.ns = np.asarray(ns, dtype=np.int64)
        self.count = int(self.ns.size)
        self.S = int(shifts)
        self._h = C.c_void_p()
        nsc = np.ascontiguousarray(self.ns)
        _check(_lib.lhl_batch_create(self.count, C.c_void_p(nsc.ctypes.data), self.S, C.byref(self._h)), "LHLBatch")
        v = _BatchView()
        _check(_lib.lhl_batch_get_view(self._h, C.byref(v)))
        self._v = v
        self.off2 = np.concatenate([[0], np.cumsum(self.ns * self.ns)])
        self.off1 = np.concatenate([[0], np.cumsum(self.ns)])
        self.offg = np.concatenate([[0], np.cumsum(self.S * (self.ns + 4) * self.ns)])

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.lhl_batch_destroy(h)
            self._h = None

    # packing of host data
    def pack_matrices(self, mats) -> np.ndarray:
        return np.concatenate([np.asarray(A, dtype=np.float64).ravel(order="F") for A in mats])

    def pack_rhs(self, blocks) -> np.ndarray:
        """blocks[m]: n_m x (S R), column s R + r is right-hand side r of shift s."""
        return np.concatenate([np.asarray(X, dtype=np.float64).ravel(order="F") for X in blocks])

    def unpack_rhs(self, packed, R: int):
        out = []
        o = 0
        for n in self.ns:
            k = int(n) * self.S * R
            out.append(np.asarray(packed[o:o + k]).reshape((self.S * R, int(n))).T)
            o += k
        return out

    # device views of matrix m (and shift s)
    def factors(self, m: int) -> torch.Tensor:
        n = int(self.ns[m])
        return _view(self._v.factors + 8 * int(self.off2[m]), (n, n), strides=(8, 8 * n))

    def Ht(self, m: int) -> torch.Tensor:
        n = int(self.ns[m])
        return _view(self._v.Ht + 8 * int(self.off2[m]), (n, n), strides=(8, 8 * n))

    def ipiv(self, m: int) -> torch.Tensor:
        n = int(self.ns[m])
        return _view(self._v.ipiv + 8 * int(self.off1[m]), (max(n - 2, 0),), "<i8")

    def scale(self, m: int) -> torch.Tensor:
        return _view(self._v.scale + 8 * int(self.off1[m]), (int(self.ns[m]),))

    def perm(self, m: int) -> torch.Tensor:
        return _view(self._v.perm + 8 * int(self.off1[m]), (int(self.ns[m]),), "<i8")

    def Gt(self, m: int, s: int) -> torch.Tensor:
        n = int(self.ns[m])
        base = self._v.Gt + 8 * (int(self.offg[m]) + s * (n + 4) * n)
        return _view(base, (n + 4, n), strides=(8, 8 * (n + 4)))

    def rdiag(self, m: int, s: int) -> torch.Tensor:
        n = int(self.ns[m])
        return _view(self._v.rdiag + 8 * (self.S * int(self.off1[m]) + s * n), (n,))

    def swap(self, m: int, s: int) -> torch.Tensor:
        n = int(self.ns[m])
        return _view(self._v.swap + (self.S * int(self.off1[m]) + s * n), (n,), "|u1")

    @property
    def info(self) -> torch.Tensor:
        return _view(self._v.info, (self.count * self.S,), "<i4")


def lhl_reduce_batched_(b: LHLBatch, J: torch.Tensor, balance: bool = True, stream=None) -> LHLBatch:
    """lhl_reduce! of every matrix of the batch (J: packed, see LHLBatch.pack_matrices)."""
    _require_cuda_f64(J, "J")
    if J.numel() != int(b.off2[-1]):
        raise DimensionMismatch("packed J has the wrong length")
    _check(_lib.lhl_reduce_batched(b._h, C.c_void_p(J.data_ptr()), int(bool(balance)), _stream(stream)),
           "lhl_reduce_batched")
    return b


def lhl_shift_batched_all_(b: LHLBatch, sigmas: torch.Tensor, taus: torch.Tensor, stream=None) -> LHLBatch:
    """lhl_shift! of every (matrix, shift): sigmas, taus have count x S entries, matrix-major."""
    for t, nm in ((sigmas, "sigmas"), (taus, "taus")):
        _require_cuda_f64(t, nm)
        if t.numel() != b.count * b.S:
            raise DimensionMismatch(f"{nm} must have count x shifts entries")
    sigmas, taus = sigmas.contiguous(), taus.contiguous()
    _check(_lib.lhl_shift_batched_all(b._h, C.c_void_p(sigmas.data_ptr()), C.c_void_p(taus.data_ptr()),
                                      _stream(stream)), "lhl_shift_batched_all")
    return b


def lhl_solve_batched_(b: LHLBatch, J: torch.Tensor, B: torch.Tensor, X: torch.Tensor, rhs_per_shift: int,
                       tol: float = 1e-10, max_steps: int = 8, res: torch.Tensor = None, stream=None) -> torch.Tensor:
    """Every right-hand side solved and refined to `tol` on chip (lhl_solve_batched); returns
    the final relative residuals (count x S x R)."""
    for t, nm in ((J, "J"), (B, "B"), (X, "X")):
        _require_cuda_f64(t, nm)
    k = b.count * b.S * int(rhs_per_shift)
    if B.numel() != int(b.off1[-1]) * b.S * int(rhs_per_shift) or X.numel() != B.numel():
        raise DimensionMismatch("packed B / X have the wrong length")
    if res is None:
        res = torch.empty(k, dtype=torch.float64, device=B.device)
    _check(_lib.lhl_solve_batched(b._h, C.c_void_p(J.data_ptr()), C.c_void_p(B.data_ptr()),
                                  C.c_void_p(X.data_ptr()), int(rhs_per_shift), float(tol), int(max_steps),
                                  C.c_void_p(res.data_ptr()), _stream(stream)), "lhl_solve_batched")
    return res


def version() -> str:
    return _lib.lhl_version().decode()


__all__ = ["LHLWorkspace", "LHLShift", "lhl", "lhl_", "lhl_reduce_", "lhl_shift_", "lhl_shift_batched_",
           "lhl_refine_tol_", "lhl_refine_gmres_", "LHLBatch", "lhl_reduce_batched_", "lhl_shift_batched_all_", "lhl_solve_batched_",
           "lhl_ldiv_", "lhl_refine_", "applyZ_", "applyZinv_", "residual_norms", "ArgumentError",
           "DimensionMismatch", "LHLDeviceError", "LHL_PREC_FP64", "LHL_PREC_MIXED", "version", "lib"]
