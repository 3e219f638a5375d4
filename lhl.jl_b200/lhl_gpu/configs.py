"""Seeded synthetic inputs of the five benchmark configurations (numpy PCG64).

No public dataset is involved: each configuration is defined by its generator.  Matrices
are returned column-major (numpy order='F'), right-hand sides as (n, k) Fortran arrays.
"""
from __future__ import annotations

import numpy as np


def rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def config1():
    """Plain method, small: J 400x400 N(0,1) (seed 0), b N(0,1) (seed 1); shifts (1, -g),
    g in {0.01, 0.013, 0.021}; one ldiv per shift plus one refinement step."""
    n = 400
    J = np.asfortranarray(rng(0).standard_normal((n, n)))
    b = rng(1).standard_normal(n)
    g = np.array([0.01, 0.013, 0.021])
    B = np.asfortranarray(np.repeat(b[:, None], 3, axis=1))
    return dict(name="c1", n=n, J=J, sigma=np.ones(3), tau=-g, B=B, steps=1)


def config2(nshifts: int = 64):
    """Plain FP64 blocked path: J 2048x2048 N(0,1) (seed 2); 64 shifts (1, -g), g log-uniform
    in [1e-4, 1e-1] (seed 3); one N(0,1) right-hand side per shift (seed 4)."""
    n = 2048
    J = np.asfortranarray(rng(2).standard_normal((n, n)))
    g = 10.0 ** rng(3).uniform(-4.0, -1.0, nshifts)
    B = np.asfortranarray(rng(4).standard_normal((n, nshifts)))
    return dict(name="c2", n=n, J=J, sigma=np.ones(nshifts), tau=-g, B=B, steps=1)


def config3(n: int = 4096, nshifts: int = 256):
    """Precision: stiff J = Q diag(-lam) Q^-1 + 0.01 N(0,1), Q = I + N(0,1)/sqrt(n),
    lam log-uniform in [1, 1e4] (seed 5; Q^-1 by an FP64 LU); shifts (-1/(dt g), 1) with
    dt g log-uniform in [1e-5, 1e-2] (seed 6); one N(0,1) right-hand side per shift (seed 7)."""
    g5 = rng(5)
    Q = np.eye(n) + g5.standard_normal((n, n)) / np.sqrt(n)
    lam = 10.0 ** g5.uniform(0.0, 4.0, n)
    E = g5.standard_normal((n, n))
    J = (Q * (-lam)) @ np.linalg.inv(Q) + 0.01 * E
    dtg = 10.0 ** rng(6).uniform(-5.0, -2.0, nshifts)
    B = np.asfortranarray(rng(7).standard_normal((n, nshifts)))
    return dict(name="c3", n=n, J=np.asfortranarray(J), sigma=-1.0 / dtg, tau=np.ones(nshifts), B=B, steps=1)


def config4(count: int = 4096, seed: int = 8):
    """Batching: `count` independent J, n uniform-integer in [16, 256], N(0,1) - 5 I (seed 8);
    8 shifts (1, -g) per matrix, g log-uniform in [1e-3, 1e-1]; 4 N(0,1) RHS per shift (seed 9)."""
    g8 = rng(seed)
    ns = g8.integers(16, 257, count)
    mats = [np.asfortranarray(g8.standard_normal((int(m), int(m))) - 5.0 * np.eye(int(m))) for m in ns]
    g9 = rng(9)
    gam = 10.0 ** g9.uniform(-3.0, -1.0, (count, 8))
    rhs = [np.asfortranarray(g9.standard_normal((int(m), 32))) for m in ns]
    return dict(name="c4", ns=ns, mats=mats, sigma=np.ones((count, 8)), tau=-gam, rhs=rhs)


def config5(n: int = 8192, nshifts: int = 128, nrhs: int = 32):
    """Complex shifts on a real matrix: J N(0,1)/sqrt(n) (seed 10); s = a + ib, a ~ U[-2, 0],
    b ~ U[0, 10] (seed 11), (sigma, tau) = (s, -1); 32 complex N(0,1) RHS per shift (seed 12)."""
    J = np.asfortranarray(rng(10).standard_normal((n, n)) / np.sqrt(n))
    g11 = rng(11)
    s = g11.uniform(-2.0, 0.0, nshifts) + 1j * g11.uniform(0.0, 10.0, nshifts)
    g12 = rng(12)
    return dict(name="c5", n=n, J=J, sigma=s, tau=-np.ones(nshifts), nrhs=nrhs, rng=g12)
