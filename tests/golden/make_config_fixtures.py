"""Writes the oracle's results on the seeded benchmark configurations 2 and 5 as small
fixtures (tests/golden/config_<c>.npz), for the device parity tests at full size (config 3's
are computed where its test runs; see the note at the end).

    python tests/golden/make_config_fixtures.py [c2 c5]

The oracle (oracle/lhl_oracle.c, the CPU restatement of src/LHLFactorization.jl) reduces
each configuration's J with the reference's Float64 path (balancing F:299-340, the pointer
blocked reduction F:765-2001, Ht F:2005-2061, perm F:376-387).  Full matrices at n = 8192
are 512 MB each, so the fixture keeps:

  * the SHA-256 of J's bytes (column-major), to show that the device test generated the same
    input from the same seed;
  * ipiv in full, and the SHA-256 of factors, Ht, scale, iscale, perm and iperm (bit parity);
  * for a sample of the configuration's shifts, the SHA-256 of the shift LU state exactly as
    test/core_tests.jl:173-190 extracts it (U by columns, l, swap, rdiag, info), real shifts
    for c2 / c3 and complex shifts on the real reduction for c5 (planar Gt, F:2529-2594);
  * for a sample of right-hand sides, the oracle's FP64 solution refined by two lhl_refine!
    steps (F:3144-3157), the forward-error reference, with its relative residual.

Run once on the CPU (about a minute for c5 on 8 threads); the GPU tests read only the .npz.
"""
from __future__ import annotations

import hashlib
import importlib.util
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle import oracle as O  # noqa: E402


def _configs():
    spec = importlib.util.spec_from_file_location(
        "lhl_configs", os.path.join(REPO, "lhl.jl_b200", "lhl_gpu", "configs.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def sha_colmajor(M) -> str:
    """SHA-256 of a matrix's bytes in column-major order."""
    return sha(np.asarray(M).T)


def shift_state_sha(S) -> str:
    """test/core_tests.jl:173-190's state of a real shift LU, hashed: U by columns (Gt[k:n, k]),
    l (Gt[k, k+1]), swap, rdiag, info."""
    n = S.n
    h = hashlib.sha256()
    for k in range(n):
        h.update(np.ascontiguousarray(S.Gt[k:n, k]).tobytes())
    h.update(np.ascontiguousarray(S.Gt[np.arange(n - 1), np.arange(1, n)]).tobytes())
    h.update(np.ascontiguousarray(S.swap[:n]).tobytes())
    h.update(np.ascontiguousarray(S.rdiag[:n]).tobytes())
    h.update(np.int64(S.info).tobytes())
    return h.hexdigest()


def shift_state_sha_complex(S) -> str:
    """The same for a complex shift's planar Gt: per column k the real plane Gt[k:n, k], then
    the imaginary plane Gt[po+k:po+n, k]; l from both planes; swap; rdiag as (re, im) pairs; info."""
    n, po = S.n, S.po
    h = hashlib.sha256()
    for k in range(n):
        h.update(np.ascontiguousarray(S.Gt[k:n, k]).tobytes())
        h.update(np.ascontiguousarray(S.Gt[po + k:po + n, k]).tobytes())
    r = np.arange(n - 1)
    h.update(np.ascontiguousarray(S.Gt[r, r + 1]).tobytes())
    h.update(np.ascontiguousarray(S.Gt[po + r, r + 1]).tobytes())
    h.update(np.ascontiguousarray(S.swap[:n]).tobytes())
    rd = np.empty(2 * n)
    rd[0::2] = S.rdiag[:n].real
    rd[1::2] = S.rdiag[:n].imag
    h.update(rd.tobytes())
    h.update(np.int64(S.info).tobytes())
    return h.hexdigest()


def c5_rhs(c, columns):
    """Config 5's right-hand sides (seed 12): column j of the n x (S R) complex block, drawn as
    the benchmark draws the whole block (real parts, then imaginary parts)."""
    g = c["rng"]
    n, S, R = c["n"], len(c["sigma"]), c["nrhs"]
    re = g.standard_normal((n, S * R))
    im = g.standard_normal((n, S * R))
    return np.stack([O.cpack(re[:, j], im[:, j]) for j in columns], axis=1)


def config(name: str):
    cf = _configs()
    return {"c2": cf.config2, "c3": cf.config3, "c5": cf.config5}[name]()


def reference_results(name: str, c) -> dict:
    """The oracle's results on configuration `name` (inputs `c` from lhl_gpu.configs), as the
    fixture holds them."""
    J = c["J"]
    n = J.shape[0]
    R = O.reduce(J)
    out = {"n": np.int64(n), "J_sha": sha_colmajor(J), "ipiv": R.ipiv,
           "factors_sha": sha_colmajor(R.factors), "Ht_sha": sha_colmajor(R.Ht), "scale_sha": sha(R.scale),
           "iscale_sha": sha(R.iscale), "perm_sha": sha(R.perm), "iperm_sha": sha(R.iperm)}
    sig, tau = np.asarray(c["sigma"]), np.asarray(c["tau"])
    S = len(sig)
    if name == "c5":
        shifts = [0, S - 1]
        R_rhs = c["nrhs"]
        cols = [0, (S - 1) * R_rhs + R_rhs - 1]   # the first RHS of shift 0, the last RHS of the last shift
        B = c5_rhs(c, cols)
        hashes, X, res = [], [], []
        for s in shifts:
            Sh = O.shift_complex(R, sig[s], tau[s])
            hashes.append(shift_state_sha_complex(Sh))
        for i, col in enumerate(cols):
            s = col // R_rhs
            Sh = O.shift_complex(R, sig[s], tau[s])
            b = B[:, i]
            x = O.ldiv_complex(R, Sh, b)
            x = O.refine_complex(R, Sh, J, b, x, steps=2)
            W_x = sig[s] * x + tau[s] * (J @ x.real + 1j * (J @ x.imag))
            res.append(np.linalg.norm(b - W_x) / np.linalg.norm(b))
            X.append(x)
        out.update(shift_index=np.array(shifts), shift_sha=np.array(hashes), rhs_columns=np.array(cols),
                   x_ref=np.stack(X, axis=1), x_ref_relres=np.array(res))
    else:
        order = np.argsort(np.abs(sig) + np.abs(tau))
        shifts = sorted({0, S - 1, int(order[0]), int(order[-1])})
        B = c["B"]
        hashes, X, res = [], [], []
        for s in shifts:
            Sh = O.shift(R, sig[s], tau[s])
            hashes.append(shift_state_sha(Sh))
            b = B[:, s]
            x = O.ldiv(R, Sh, b)
            x = O.refine(R, Sh, J, b, x, steps=2)
            res.append(np.linalg.norm(b - (sig[s] * x + tau[s] * (J @ x))) / np.linalg.norm(b))
            X.append(x)
        out.update(shift_index=np.array(shifts), shift_sha=np.array(hashes), rhs_columns=np.array(shifts),
                   x_ref=np.stack(X, axis=1), x_ref_relres=np.array(res))
    return out


def make(name: str):
    c = config(name)
    t0 = time.time()
    out = reference_results(name, c)
    path = os.path.join(HERE, f"config_{name}.npz")
    np.savez_compressed(path, **out)
    print(f"{name}: n = {int(out['n'])}, oracle results in {time.time() - t0:.1f} s on {O.num_threads()} threads; "
          f"shifts {out['shift_index'].tolist()}; x_ref residuals {np.asarray(out['x_ref_relres']).tolist()}; "
          f"{os.path.getsize(path)} bytes -> {path}", flush=True)


# Config 3's J = Q diag(-lam) Q^-1 + 0.01 G goes through LAPACK's inverse and a BLAS product,
# whose rounding depends on the host's BLAS kernels and thread count, so its bits are not the
# same on every machine: its parity test calls reference_results on the machine it runs on
# (about 10 s of oracle time) instead of reading a fixture.  Configs 2 and 5 are plain draws
# from the seeded generator and identical everywhere.
if __name__ == "__main__":
    O.build()
    for name in (sys.argv[1:] or ["c2", "c5"]):
        make(name)
