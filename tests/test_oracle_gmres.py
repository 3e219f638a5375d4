"""The oracle's GMRES-IR (the algorithm of lhl_refine_gmres) on the CPU: it reaches the
tolerance where fixed-point refinement (lhl_refine!, F:3144-3157) contracts slowly, with fewer
preconditioner applications; it stops after one Arnoldi step when the preconditioner is exact;
it leaves a converged column alone."""
import numpy as np
import pytest

from oracle import oracle as O


def rng(seed):
    return np.random.default_rng(seed)


def weak_case(n, seed, delta, closeness):
    """W = I - g J with 1/g close to a real eigenvalue of J; the preconditioner is the
    factorisation of J + delta E (a stand-in for factors computed in lower precision)."""
    g0 = rng(seed)
    J = g0.standard_normal((n, n))
    E = g0.standard_normal((n, n))
    ev = np.linalg.eigvals(J)
    lam = max(ev[np.abs(ev.imag) < 1e-12].real, key=abs)
    g = closeness / lam
    Rp = O.reduce(J + delta * E)
    Sp = O.shift(Rp, 1.0, -g)
    W = np.eye(n) - g * J
    b = g0.standard_normal(n)
    return W, b, (lambda v: W @ v), (lambda v: O.ldiv(Rp, Sp, v))


def richardson(matvec, precond, b, x, tol, max_steps):
    nb = np.linalg.norm(b)
    for s in range(max_steps + 1):
        r = b - matvec(x)
        rel = np.linalg.norm(r) / nb
        if rel <= tol or s == max_steps:
            return x, rel, s
        x = x + precond(r)


@pytest.mark.parametrize("n,seed", [(120, 1), (200, 2), (257, 3)])
def test_gmres_ir_beats_fixed_point_on_a_weak_preconditioner(n, seed):
    W, b, mv, pc = weak_case(n, seed, 3e-3, 0.995)
    x0 = pc(b)
    xr, relr, steps = richardson(mv, pc, b, x0, 1e-10, 60)
    xg, relg, napply = O.gmres_ir(mv, pc, b, x0, 1e-10, max_cycles=6, restart=10)
    assert relg <= 1e-10
    assert np.linalg.norm(b - W @ xg) <= 1.0001e-10 * np.linalg.norm(b)
    assert napply < steps, (napply, steps, relr)


@pytest.mark.parametrize("n", [1, 2, 3, 9, 64])
def test_gmres_ir_exact_preconditioner_one_step(n):
    J = rng(n).standard_normal((n, n))
    R = O.reduce(J)
    S = O.shift(R, 1.0, -0.01)
    W = np.eye(n) - 0.01 * J
    b = rng(n + 1).standard_normal(n)
    x0 = np.zeros(n)
    x, rel, napply = O.gmres_ir(lambda v: W @ v, lambda v: O.ldiv(R, S, v), b, x0, 1e-12, max_cycles=3, restart=5)
    assert rel <= 1e-12
    assert napply <= 4  # z, then one Arnoldi step per cycle


def test_gmres_ir_leaves_a_converged_column_alone():
    n = 50
    J = rng(5).standard_normal((n, n))
    W = np.eye(n) - 0.02 * J
    b = rng(6).standard_normal(n)
    x = np.linalg.solve(W, b)
    R = O.reduce(J)
    S = O.shift(R, 1.0, -0.02)
    y, rel, napply = O.gmres_ir(lambda v: W @ v, lambda v: O.ldiv(R, S, v), b, x, 1e-10)
    assert napply == 0 and np.array_equal(x, y)


@pytest.mark.parametrize("restart", [1, 2, 4])
def test_gmres_ir_short_restarts_still_converge(restart):
    W, b, mv, pc = weak_case(150, 4, 1e-4, 0.9)
    x, rel, _ = O.gmres_ir(mv, pc, b, pc(b), 1e-10, max_cycles=30, restart=restart)
    assert rel <= 1e-10


def test_gmres_ir_complex_realified():
    """Complex shifts on a real reduction: the realified GMRES-IR reaches the tolerance from a
    perturbed preconditioner (the factors of J + 1e-3 E) on a complex shift near an eigenvalue."""
    n = 160
    g0 = rng(7)
    J = g0.standard_normal((n, n)) / np.sqrt(n)
    E = g0.standard_normal((n, n)) / np.sqrt(n)
    ev = np.linalg.eigvals(J)
    s = ev[np.argmax(np.abs(ev.imag))] + 0.02  # close to an eigenvalue: W nearly singular
    W = s * np.eye(n) - J
    Rp = O.reduce(J + 1e-3 * E)
    Sp = O.shift_complex(Rp, s, -1.0)
    b = g0.standard_normal(n) + 1j * g0.standard_normal(n)
    mv = lambda v: W @ v  # noqa: E731
    pc = lambda v: O.ldiv_complex(Rp, Sp, v)  # noqa: E731
    x0 = pc(b)
    x, rel, napply = O.gmres_ir(mv, pc, b, x0, 1e-10, max_cycles=8, restart=8)
    assert rel <= 1e-10
    assert np.linalg.norm(b - W @ x) <= 1.0001e-10 * np.linalg.norm(b)
    assert napply <= 8


def test_gmres_ir_stops_at_its_attainable_accuracy():
    """With a tolerance below FP64's reach the cycles stop once one fails to halve the
    residual, far before max_cycles."""
    W, b, mv, pc = weak_case(150, 4, 1e-4, 0.9)
    x, rel, napply = O.gmres_ir(mv, pc, b, pc(b), 1e-30, max_cycles=40, restart=4)
    assert rel < 1e-12
    assert napply <= 6 * (1 + 4), napply
