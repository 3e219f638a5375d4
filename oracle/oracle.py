"""CPU oracle for the LHL hot path: ctypes bindings to ``liblhl_oracle.so``.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py``, always as the checker or the
timed CPU baseline, never by the product path.

The C source (``lhl_oracle.c``) restates src/LHLFactorization.jl function by function; see
its header for what pins it.  Arrays are numpy, column-major (``order='F'``) float64;
``ipiv``/``perm``/``iperm`` are int64 with 1-based values, like the reference's.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liblhl_oracle.so")
_lib = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="F_CONTIGUOUS")
_dv = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_iv = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_u8 = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_i32 = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build() -> str:
    """Compile the oracle with its Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        i, d = C.c_int, C.c_double
        L.lhlo_balance.argtypes = [i, _dp, i, _dv, _dv]
        L.lhlo_reduce_unblocked.argtypes = [i, _dp, i, _iv]
        L.lhlo_reduce_blocked.argtypes = [i, _dp, i, _iv, i]
        L.lhlo_reduce_blocked_ptr.argtypes = [i, _dp, i, _iv, i]
        L.lhlo_reduce.argtypes = [i, _dp, i, i, i, i, _dp, i, _iv, _dv, _dv, _iv, _iv, _dp]
        L.lhlo_reduce.restype = i
        L.lhlo_reduce_f32.argtypes = [i, _dp, i, i, _dp, i, _iv, _dv, _dv, _iv, _iv, _dp]
        L.lhlo_reduce_f32.restype = i
        L.lhlo_reduce_blocked_ptr_f32_raw.argtypes = [i, _dp, i, _iv]
        L.lhlo_reduce_blocked_ptr_f32_raw.restype = i
        L.lhlo_shift.argtypes = [i, _dp, i, d, d, _dp, i, _u8, _dv, _dv]
        L.lhlo_shift.restype = i
        L.lhlo_shift_f32.argtypes = [i, _dp, i, d, d, _dp, i, _u8, _dv, _dv]
        L.lhlo_shift_f32.restype = i
        L.lhlo_ldiv.argtypes = [i, _dp, i, _iv, _iv, _dv, _dv, _dp, i, _u8, _dv, _dv, _dv]
        L.lhlo_applyZ.argtypes = [i, _dp, i, _iv, _dv, _dv, _dv]
        L.lhlo_applyZinv.argtypes = [i, _dp, i, _iv, _dv, _dv, _dv]
        L.lhlo_refine.argtypes = [i, _dp, i, d, d, _dv, _dp, i, _iv, _iv, _dv, _dv, _dp, i, _u8, _dv,
                                  _dv, i, _dv, _dv]
        L.lhlo_shift_solve_batch.argtypes = [i, _dp, i, _dp, _dp, i, _iv, _iv, _dv, _dv, i, _dv, _dv,
                                             _dp, _dp, i, _i32]
        L.lhlo_shift_solve_batch.restype = i
        L.lhlo_shift_complex.argtypes = [i, _dp, i, d, d, d, d, _dp, i, i, _u8, _dv, _dv]
        L.lhlo_shift_complex.restype = i
        L.lhlo_ldiv_complex.argtypes = [i, _dp, i, _iv, _iv, _dv, _dv, _dp, i, i, _u8, _dv, _dv, _dv]
        L.lhlo_cabs.argtypes = [d, d]
        L.lhlo_cabs.restype = d
        L.lhlo_reduce_c128.argtypes = [i, _dv, i, i, _dv, i, _iv, _dv, _dv, _iv, _iv, _dv]
        L.lhlo_reduce_c128.restype = i
        L.lhlo_reduce_c128_path.argtypes = [i, _dv, i, i, _dv, i, _iv, _dv, _dv, _iv, _iv, _dv, i, i]
        L.lhlo_reduce_c128_path.restype = i
        L.lhlo_shift_c128.argtypes = [i, _dv, i, d, d, d, d, _dp, i, i, _u8, _dv, _dv]
        L.lhlo_shift_c128.restype = i
        L.lhlo_applyZinv_c128.argtypes = [i, _dv, i, _iv, _dv, _dv]
        L.lhlo_applyZ_c128.argtypes = [i, _dv, i, _iv, _dv, _dv]
        L.lhlo_ldiv_c128.argtypes = [i, _dv, i, _iv, _iv, _dv, _dv, _dp, i, i, _u8, _dv, _dv, _dv]
        L.lhlo_num_threads.restype = i
        _lib = L
    return _lib


def num_threads() -> int:
    return int(lib().lhlo_num_threads())


class Reduction:
    """The outputs of ``lhl_reduce!`` (F:355-390) for a real Float64 J."""

    def __init__(self, n):
        self.n = n
        self.factors = np.zeros((n, n), order="F")
        self.ipiv = np.zeros(max(n - 2, 0), dtype=np.int64)
        self.scale = np.ones(n)
        self.iscale = np.ones(n)
        self.perm = np.arange(1, n + 1, dtype=np.int64)
        self.iperm = np.arange(1, n + 1, dtype=np.int64)
        self.Ht = np.zeros((n, n), order="F")

    @property
    def H(self):
        return np.triu(self.factors, -1)

    @property
    def L(self):
        """Unit lower triangular L with L[i, k+1] = factors[i, k] for i >= k+2 (0-based: i >= k+2)."""
        n = self.n
        Lm = np.eye(n)
        for k in range(n - 2):
            Lm[k + 2:, k + 1] = self.factors[k + 2:, k]
        return Lm

    def Z(self):
        """Z = D P L as a dense matrix (columns: applyZ of unit vectors)."""
        n = self.n
        Zm = np.eye(n, order="F")
        for j in range(n):
            Zm[:, j] = apply_z(self, Zm[:, j].copy())
        return Zm

    def Zinv(self):
        n = self.n
        Zm = np.eye(n, order="F")
        for j in range(n):
            Zm[:, j] = apply_zinv(self, Zm[:, j].copy())
        return Zm


def _ipiv_buf(n):
    return np.zeros(max(n - 2, 1), dtype=np.int64)


def reduce(J, balance=True, path=0, nb=16) -> Reduction:
    """``lhl(J; balance)``: path 0 = the reference's choice (pointer blocked at n >= 500), 1 = unblocked, 2 = generic blocked, 3 = pointer blocked."""
    J = np.asfortranarray(J, dtype=np.float64)
    n = J.shape[0]
    R = Reduction(n)
    ip = _ipiv_buf(n)
    F = np.zeros((max(n, 1), max(n, 1)), order="F")
    Ht = np.zeros((max(n, 1), max(n, 1)), order="F")
    sc = np.ones(max(n, 1))
    isc = np.ones(max(n, 1))
    pm = np.zeros(max(n, 1), dtype=np.int64)
    ipm = np.zeros(max(n, 1), dtype=np.int64)
    Jp = J if n > 0 else np.zeros((1, 1), order="F")
    rc = lib().lhlo_reduce(n, Jp, max(n, 1), int(balance), path, nb, F, max(n, 1), ip, sc, isc, pm, ipm, Ht)
    assert rc == 0
    R.factors = F[:n, :n].copy(order="F")
    R.ipiv = ip[: max(n - 2, 0)].copy()
    R.scale, R.iscale = sc[:n].copy(), isc[:n].copy()
    R.perm, R.iperm = pm[:n].copy(), ipm[:n].copy()
    R.Ht = Ht[:n, :n].copy(order="F")
    return R


def reduce_f32(J, balance=True) -> Reduction:
    """``lhl(J)`` on ``LHLWorkspace{Float32}``: J rounded to float, balancing and the reduction in
    float arithmetic (lhlo_reduce_f32): unblocked below n = 1024, the blocked pointer path from
    there, as the reference chooses.  The arrays hold float values in float64."""
    J = np.asfortranarray(J, dtype=np.float64)
    n = J.shape[0]
    R = Reduction(n)
    ip = _ipiv_buf(n)
    F = np.zeros((max(n, 1), max(n, 1)), order="F")
    Ht = np.zeros((max(n, 1), max(n, 1)), order="F")
    sc = np.ones(max(n, 1))
    isc = np.ones(max(n, 1))
    pm = np.zeros(max(n, 1), dtype=np.int64)
    ipm = np.zeros(max(n, 1), dtype=np.int64)
    Jp = J if n > 0 else np.zeros((1, 1), order="F")
    rc = lib().lhlo_reduce_f32(n, Jp, max(n, 1), int(balance), F, max(n, 1), ip, sc, isc, pm, ipm, Ht)
    assert rc == 0
    R.factors = F[:n, :n].copy(order="F")
    R.ipiv = ip[: max(n - 2, 0)].copy()
    R.scale, R.iscale = sc[:n].copy(), isc[:n].copy()
    R.perm, R.iperm = pm[:n].copy(), ipm[:n].copy()
    R.Ht = Ht[:n, :n].copy(order="F")
    return R


def reduce_blocked_f32_raw(A):
    """The reference's blocked Float32 form alone (nb = 16, no balancing) at any n, on A rounded
    to float: (factors in float64 storage, ipiv)."""
    A = np.asfortranarray(np.asarray(A, dtype=np.float32).astype(np.float64))
    n = A.shape[0]
    ip = _ipiv_buf(n)
    assert lib().lhlo_reduce_blocked_ptr_f32_raw(n, A if n > 0 else np.zeros((1, 1), order="F"), max(n, 1), ip) == 0
    return A, ip[: max(n - 2, 0)].copy()


def reduce_unblocked_raw(A):
    """``_lhl_reduce_unblocked!`` on a copy of A (no balancing): returns (factors, ipiv)."""
    A = np.array(A, dtype=np.float64, order="F", copy=True)
    n = A.shape[0]
    ip = _ipiv_buf(n)
    lib().lhlo_reduce_unblocked(n, A, max(n, 1), ip)
    return A, ip[: max(n - 2, 0)].copy()


def reduce_blocked_raw(A, nb=16):
    A = np.array(A, dtype=np.float64, order="F", copy=True)
    n = A.shape[0]
    ip = _ipiv_buf(n)
    lib().lhlo_reduce_blocked(n, A, max(n, 1), ip, nb)
    return A, ip[: max(n - 2, 0)].copy()


def balance_raw(A):
    A = np.array(A, dtype=np.float64, order="F", copy=True)
    n = A.shape[0]
    d = np.ones(n)
    isc = np.ones(n)
    lib().lhlo_balance(n, A, n, d, isc)
    return A, d, isc


class Shift:
    """The outputs of ``lhl_shift!`` for a real shift (F:2456-2594)."""

    def __init__(self, n):
        self.n = n
        self.ldg = n + 4
        self.Gt = np.zeros((self.ldg, max(n, 1)), order="F")
        self.swap = np.zeros(max(n, 1), dtype=np.uint8)
        self.rdiag = np.zeros(max(n, 1))
        self.info = 0
        self.sigma = 0.0
        self.tau = 0.0

    def state(self):
        """(U, l, swap, rdiag, info) exactly as test/core_tests.jl:173-190 extracts it."""
        n = self.n
        G = self.Gt
        U = G[:n, :n].T[np.triu_indices(n)]  # G[j, k] for k = 0.., j = k.. (column order)
        l = G[np.arange(n - 1), np.arange(1, n)]
        return U, l, self.swap[:n].copy(), self.rdiag[:n].copy(), self.info


def shift(R: Reduction, sigma, tau) -> Shift:
    n = R.n
    S = Shift(n)
    w = np.zeros(max(n, 1))
    Ht = R.Ht if n > 0 else np.zeros((1, 1), order="F")
    S.info = int(lib().lhlo_shift(n, Ht, max(n, 1), float(sigma), float(tau), S.Gt, S.ldg, S.swap, S.rdiag, w))
    S.sigma, S.tau = float(sigma), float(tau)
    return S


def shift_f32(Ht, sigma, tau) -> Shift:
    """lhl_shift! of an LHLWorkspace{Float32} on the n x n Ht (float values; any float dtype),
    in float arithmetic (lhlo_shift_f32)."""
    Ht = np.asfortranarray(np.asarray(Ht, dtype=np.float32), dtype=np.float64)
    n = Ht.shape[0]
    S = Shift(n)
    w = np.zeros(max(n, 1))
    H = Ht if n > 0 else np.zeros((1, 1), order="F")
    S.info = int(lib().lhlo_shift_f32(n, H, max(n, 1), float(sigma), float(tau), S.Gt, S.ldg, S.swap, S.rdiag, w))
    S.sigma, S.tau = float(np.float32(sigma)), float(np.float32(tau))
    return S


def ldiv(R: Reduction, S: Shift, b):
    x = np.array(b, dtype=np.float64, copy=True)
    y = np.zeros(max(R.n, 1))
    lib().lhlo_ldiv(R.n, R.factors, max(R.n, 1), R.perm, R.iperm, R.scale, R.iscale, S.Gt, S.ldg, S.swap,
                    S.rdiag, x, y)
    return x


def apply_z(R: Reduction, x):
    x = np.array(x, dtype=np.float64, copy=True)
    y = np.zeros(max(R.n, 1))
    lib().lhlo_applyZ(R.n, R.factors, max(R.n, 1), R.iperm, R.scale, x, y)
    return x


def apply_zinv(R: Reduction, x):
    x = np.array(x, dtype=np.float64, copy=True)
    y = np.zeros(max(R.n, 1))
    lib().lhlo_applyZinv(R.n, R.factors, max(R.n, 1), R.perm, R.iscale, x, y)
    return x


def refine(R: Reduction, S: Shift, J, b, x, steps=1):
    J = np.asfortranarray(J, dtype=np.float64)
    x = np.array(x, dtype=np.float64, copy=True)
    b = np.ascontiguousarray(b, dtype=np.float64)
    r = np.zeros(max(R.n, 1))
    y = np.zeros(max(R.n, 1))
    lib().lhlo_refine(R.n, J, max(R.n, 1), S.sigma, S.tau, b, R.factors, max(R.n, 1), R.perm, R.iperm, R.scale,
                      R.iscale, S.Gt, S.ldg, S.swap, S.rdiag, x, steps, r, y)
    return x


def shift_solve_batch(R: Reduction, J, sigmas, taus, B, steps=1):
    """S shifts, one RHS each (columns of B, n x S): shift LU + ldiv + `steps` refinements."""
    n = R.n
    sig = np.ascontiguousarray(sigmas, dtype=np.float64)
    tau = np.ascontiguousarray(taus, dtype=np.float64)
    S = sig.shape[0]
    B = np.asfortranarray(B, dtype=np.float64)
    X = np.zeros((n, S), order="F")
    info = np.zeros(S, dtype=np.int32)
    rc = lib().lhlo_shift_solve_batch(n, np.asfortranarray(J, dtype=np.float64), n, R.Ht, R.factors, n, R.perm,
                                      R.iperm, R.scale, R.iscale, S, sig, tau, B, X, steps, info)
    assert rc == 0
    return X, info


def bwd(W, x, b):
    """The reference tests' backward error (test/core_tests.jl:3)."""
    return np.linalg.norm(b - W @ x, np.inf) / (np.linalg.norm(W, np.inf) * np.linalg.norm(x, np.inf)
                                                 + np.linalg.norm(b, np.inf))


def reduce_blocked_ptr_raw(A, nb=16):
    """The pointer blocked path (what the reference runs for Float64, n >= 500), no balancing."""
    A = np.array(A, dtype=np.float64, order="F", copy=True)
    n = A.shape[0]
    ip = _ipiv_buf(n)
    lib().lhlo_reduce_blocked_ptr(n, A, max(n, 1), ip, nb)
    return A, ip[: max(n - 2, 0)].copy()


def cpack(re, im):
    """Complex array from its parts, keeping the signs of zeros (re + 1j*im does not)."""
    z = np.empty(np.shape(re), dtype=np.complex128)
    z.real = re
    z.imag = im
    return z


def plane_offset(n: int) -> int:
    """Rows per plane of a complex shift's planar Gt: n plus a zero pad of at least 4, even
    (so that the imaginary plane starts on a 16-byte boundary)."""
    po = n + 4
    return po + (po & 1)


class ShiftC:
    """The outputs of ``lhl_shift!`` for a complex shift on a real reduction (LHLShift{ComplexF64}
    on LHLWorkspace{Float64}): planar Gt (real parts rows 0..n-1, imaginary rows po..po+n-1)."""

    def __init__(self, n):
        self.n = n
        self.po = plane_offset(n)
        self.ldg = 2 * self.po
        self.Gt = np.zeros((self.ldg, max(n, 1)), order="F")
        self.swap = np.zeros(max(n, 1), dtype=np.uint8)
        self.rdiag = np.zeros(max(n, 1), dtype=np.complex128)
        self.info = 0
        self.sigma = 0j
        self.tau = 0j

    def U(self):
        n, po = self.n, self.po
        G = self.Gt
        Um = np.zeros((n, n), dtype=np.complex128)
        for k in range(n):
            Um[k, k:] = cpack(G[k:n, k], G[po + k:po + n, k])
        return Um


def shift_complex(R: Reduction, sigma, tau) -> ShiftC:
    n = R.n
    S = ShiftC(n)
    w = np.zeros(2 * max(n, 1))
    Ht = R.Ht if n > 0 else np.zeros((1, 1), order="F")
    rd = np.zeros(2 * max(n, 1))
    sigma, tau = complex(sigma), complex(tau)
    S.info = int(lib().lhlo_shift_complex(n, Ht, max(n, 1), sigma.real, sigma.imag, tau.real, tau.imag, S.Gt,
                                          S.ldg, S.po, S.swap, rd, w))
    S.rdiag = cpack(rd[0::2][:max(n, 1)], rd[1::2][:max(n, 1)])
    S.sigma, S.tau = sigma, tau
    return S


def ldiv_complex(R: Reduction, S: ShiftC, b):
    x = np.array(b, dtype=np.complex128, copy=True)
    xv = x.view(np.float64)
    y = np.zeros(2 * S.po)
    rd = np.empty(2 * max(R.n, 1))
    rd[0::2] = S.rdiag.real
    rd[1::2] = S.rdiag.imag
    lib().lhlo_ldiv_complex(R.n, R.factors, max(R.n, 1), R.perm, R.iperm, R.scale, R.iscale, S.Gt, S.ldg, S.po,
                            S.swap, rd, xv, y)
    return x


def refine_complex(R: Reduction, S: ShiftC, J, b, x, steps=1):
    """lhl_refine!(x, sI + tJ, b, sh, ws, steps) (F:3144-3157) with the residual in numpy."""
    W = S.sigma * np.eye(R.n) + S.tau * np.asarray(J)
    x = np.array(x, dtype=np.complex128, copy=True)
    for _ in range(steps):
        r = b - W @ x
        x = x + ldiv_complex(R, S, r)
    return x


def gmres_ir(matvec, precond, b, x, tol, max_cycles=4, restart=8):
    """GMRES-IR for one column, the algorithm lhl_refine_gmres runs on the device: restarted
    GMRES (Saad and Schultz, 1986: Arnoldi with Givens rotations) on the correction equation
    W d = r, left-preconditioned by the factorisation (Carson and Higham, 2017), here with
    classical Gram-Schmidt applied twice.  A cycle starts while ||r|| / ||b|| > tol; its Arnoldi
    steps stop once |g_{j+1}| / beta <= min(0.5, 0.1 tol / (||r|| / ||b||)), at a breakdown, or
    after `restart` steps.  No new cycle starts once a cycle failed to halve the residual (the
    attainable accuracy).  Returns (x, relative residual, preconditioner applications).
    Complex b / x: the same real algorithm on the realified system (an interleaved complex
    vector of n entries is a real vector of 2n; the real inner product is Re<v, w>)."""
    if np.iscomplexobj(b) or np.iscomplexobj(x):
        def to_r(v):
            return np.ascontiguousarray(v, dtype=np.complex128).view(np.float64)

        def to_c(v):
            return np.ascontiguousarray(v, dtype=np.float64).view(np.complex128)

        xr, rel, k = gmres_ir(lambda v: to_r(matvec(to_c(v))), lambda v: to_r(precond(to_c(v))), to_r(b),
                              to_r(x), tol, max_cycles, restart)
        return to_c(xr), rel, k
    b = np.asarray(b, dtype=np.float64)
    x = np.array(x, dtype=np.float64, copy=True)
    nb = np.linalg.norm(b)
    m = restart
    napply = 0
    rel = np.inf
    prev = None
    for cyc in range(max_cycles + 1):
        r = b - matvec(x)
        rel = np.linalg.norm(r) / nb if nb > 0 else np.linalg.norm(r)
        if cyc == max_cycles or not rel > tol:
            break
        if prev is not None and not rel <= 0.5 * prev:
            break  # stagnated: the residual did not halve over the last cycle
        prev = rel
        z = precond(r)
        napply += 1
        beta = np.linalg.norm(z)
        if not (beta > 0 and np.isfinite(beta)):
            break
        eta = min(0.5, 0.1 * tol / rel)
        V = [z / beta]
        Hr = np.zeros((m, m))
        cs = np.zeros(m)
        sn = np.zeros(m)
        g = np.zeros(m + 1)
        g[0] = beta
        jd = 0
        for j in range(m):
            w = precond(matvec(V[j]))
            napply += 1
            h1 = np.array([v @ w for v in V])
            w = w - sum(h * v for h, v in zip(h1, V))
            h2 = np.array([v @ w for v in V])
            w = w - sum(h * v for h, v in zip(h2, V))
            hn = np.linalg.norm(w)
            V.append(w / hn if hn > 0 and np.isfinite(hn) else np.zeros_like(w))
            hc = np.concatenate([h1 + h2, [hn]])
            for i in range(j):
                a_, b_ = hc[i], hc[i + 1]
                hc[i] = cs[i] * a_ + sn[i] * b_
                hc[i + 1] = -sn[i] * a_ + cs[i] * b_
            rr = np.hypot(hc[j], hc[j + 1])
            cs[j], sn[j] = (hc[j] / rr, hc[j + 1] / rr) if rr > 0 else (1.0, 0.0)
            Hr[:j, j] = hc[:j]
            Hr[j, j] = rr
            g[j + 1] = -sn[j] * g[j]
            g[j] = cs[j] * g[j]
            jd = j + 1
            est = abs(g[j + 1]) / beta
            if not est > eta or not hn > 0 or not np.isfinite(est):
                break
        y = np.zeros(jd)
        for i in range(jd - 1, -1, -1):
            v = g[i] - Hr[i, i + 1:jd] @ y[i + 1:jd]
            y[i] = v / Hr[i, i] if Hr[i, i] != 0 else 0.0
        x = x + sum(y[i] * V[i] for i in range(jd))
    return x, rel, napply


# ---------------------------------------------------------------------------------------------
# A complex J (LHLWorkspace{ComplexF64}): lhlo_reduce_c128 and friends in lhl_oracle.c.
# Complex matrices cross as complex128 arrays (interleaved pairs), column-major.
# ---------------------------------------------------------------------------------------------
def _cflat(a):
    """The interleaved float64 view of a Fortran-ordered complex128 array."""
    return np.asfortranarray(a, dtype=np.complex128).ravel(order="F").view(np.float64)


class ReductionC(Reduction):
    """The outputs of ``lhl_reduce!`` for a complex J: complex factors and Ht, real scale."""

    @property
    def L(self):
        n = self.n
        Lm = np.eye(n, dtype=np.complex128)
        for k in range(n - 2):
            Lm[k + 2:, k + 1] = self.factors[k + 2:, k]
        return Lm

    def Z(self):
        n = self.n
        Zm = np.eye(n, dtype=np.complex128, order="F")
        for j in range(n):
            Zm[:, j] = apply_z_c128(self, Zm[:, j].copy())
        return Zm

    def Zinv(self):
        n = self.n
        Zm = np.eye(n, dtype=np.complex128, order="F")
        for j in range(n):
            Zm[:, j] = apply_zinv_c128(self, Zm[:, j].copy())
        return Zm


def cabs(z) -> float:
    """abs(z) of the complex reduction (the hypot algorithm the oracle and the device share)."""
    z = complex(z)
    return float(lib().lhlo_cabs(z.real, z.imag))


def reduce_c128(J, balance=True, path=0, nb=16) -> ReductionC:
    """``lhl(J; balance)`` for a complex J.  path 0: the unblocked ELMHES at every n (the
    device's order); 1: the generic blocked order with panels of nb; 2: the reference's
    choice, blocked (nb = 16) iff n >= 768 (F:398, F:705)."""
    J = np.asfortranarray(J, dtype=np.complex128)
    n = J.shape[0]
    R = ReductionC(n)
    m = max(n, 1)
    Jf = _cflat(J) if n > 0 else np.zeros(2)
    F = np.zeros(2 * m * m)
    Ht = np.zeros(2 * m * m)
    ip = _ipiv_buf(n)
    sc, isc = np.ones(m), np.ones(m)
    pm, ipm = np.zeros(m, dtype=np.int64), np.zeros(m, dtype=np.int64)
    rc = lib().lhlo_reduce_c128_path(n, Jf, m, int(balance), F, m, ip, sc, isc, pm, ipm, Ht, int(path), int(nb))
    assert rc == 0
    R.factors = F.view(np.complex128).reshape((m, m), order="F")[:n, :n].copy(order="F")
    R.Ht = Ht.view(np.complex128).reshape((m, m), order="F")[:n, :n].copy(order="F")
    R.ipiv = ip[: max(n - 2, 0)].copy()
    R.scale, R.iscale = sc[:n].copy(), isc[:n].copy()
    R.perm, R.iperm = pm[:n].copy(), ipm[:n].copy()
    return R


def shift_c128(R: ReductionC, sigma, tau) -> ShiftC:
    """``lhl_shift!(ws, sigma, tau)`` on a complex reduction (planar Gt, as ShiftC)."""
    n = R.n
    S = ShiftC(n)
    w = np.zeros(2 * max(n, 1))
    Ht = _cflat(R.Ht) if n > 0 else np.zeros(2)
    rd = np.zeros(2 * max(n, 1))
    sigma, tau = complex(sigma), complex(tau)
    S.info = int(lib().lhlo_shift_c128(n, Ht, max(n, 1), sigma.real, sigma.imag, tau.real, tau.imag, S.Gt, S.ldg,
                                       S.po, S.swap, rd, w))
    S.rdiag = cpack(rd[0::2][:max(n, 1)], rd[1::2][:max(n, 1)])
    S.sigma, S.tau = sigma, tau
    return S


def apply_zinv_c128(R: ReductionC, x):
    x = np.array(x, dtype=np.complex128, copy=True)
    lib().lhlo_applyZinv_c128(R.n, _cflat(R.factors) if R.n else np.zeros(2), max(R.n, 1), R.perm, R.iscale,
                              x.view(np.float64))
    return x


def apply_z_c128(R: ReductionC, x):
    x = np.array(x, dtype=np.complex128, copy=True)
    lib().lhlo_applyZ_c128(R.n, _cflat(R.factors) if R.n else np.zeros(2), max(R.n, 1), R.iperm, R.scale,
                           x.view(np.float64))
    return x


def ldiv_c128(R: ReductionC, S: ShiftC, b):
    x = np.array(b, dtype=np.complex128, copy=True)
    y = np.zeros(2 * S.po)
    rd = np.empty(2 * max(R.n, 1))
    rd[0::2] = S.rdiag.real
    rd[1::2] = S.rdiag.imag
    lib().lhlo_ldiv_c128(R.n, _cflat(R.factors) if R.n else np.zeros(2), max(R.n, 1), R.perm, R.iperm, R.scale,
                         R.iscale, S.Gt, S.ldg, S.po, S.swap, rd, x.view(np.float64), y)
    return x


def refine_c128(R: ReductionC, S: ShiftC, J, b, x, steps=1):
    """lhl_refine!(x, sI + tJ, b, sh, ws, steps) on a complex reduction, residual in numpy."""
    W = S.sigma * np.eye(R.n) + S.tau * np.asarray(J, dtype=np.complex128)
    x = np.array(x, dtype=np.complex128, copy=True)
    for _ in range(steps):
        x = x + ldiv_c128(R, S, b - W @ x)
    return x
