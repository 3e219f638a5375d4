"""The oracle's Float32 reduction (LHLWorkspace{Float32} below n = 1024: balancing and the
unblocked ELMHES in float arithmetic) against the reference's own relation tests.

* test/core_tests.jl:422-462 ("explicit-vector trailing update agrees with the generic one",
  T = Float32): the row-block order and the generic paired sweep (F:508-538, restated here in
  numpy float32, where every operation is one IEEE float operation) pick the Float64
  reduction's pivots, and the row-block factors are as close to the Float64 ones as the
  generic ones are (within 4x plus 100 n eps32); on the structured matrices of that test the
  pivots agree and the factors are approximately equal.
* Balancing (F:299-340 with Tr = Float32) restated scalar by scalar in numpy float32 and
  compared bit for bit.
* test/core_tests.jl:5-21 in float: Z H Z^-1 reconstructs J to float accuracy, |l| <= 1.
"""
import numpy as np
import pytest

from oracle import oracle as O

f32 = np.float32


def relerr(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def generic_f32(J):
    """F:466-501 with the generic paired sweep F:508-538, in float32 (no fused operations)."""
    A = np.array(J, dtype=f32, order="F")
    n = A.shape[0]
    ipiv = np.zeros(max(n - 2, 0), dtype=np.int64)
    for k in range(1, n - 1):  # 1-based k = 1 .. n-2
        c = k - 1
        col = np.abs(A[k:, c])
        p = k + int(np.argmax(col))  # first maximum (strict > in the scan)
        ipiv[k - 1] = p + 1
        if p != k:
            A[[k, p], :] = A[[p, k], :]
            A[:, [k, p]] = A[:, [p, k]]
        piv = A[k, c]
        if piv == 0:
            continue
        A[k + 1:, c] = A[k + 1:, c] / piv
        pk = A[k, k]
        if pk != 0:
            A[k + 1:, k] = A[k + 1:, k] - A[k + 1:, c] * pk
        j = k + 1  # 0-based column index of 1-based k+2
        while j + 1 <= n - 1:
            pj, pj1 = A[k, j], A[k, j + 1]
            lv = A[k + 1:, c].copy()
            A[k + 1:, j] = A[k + 1:, j] - lv * pj
            A[k + 1:, j + 1] = A[k + 1:, j + 1] - lv * pj1
            vj, vj1 = A[j, c], A[j + 1, c]
            A[:, k] = A[:, k] + (vj * A[:, j] + vj1 * A[:, j + 1])
            j += 2
        if j <= n - 1:
            pj = A[k, j]
            A[k + 1:, j] = A[k + 1:, j] - A[k + 1:, c] * pj
            vj = A[j, c]
            A[:, k] = A[:, k] + vj * A[:, j]
    return A, ipiv


def balance_f32(J):
    """F:299-340 with Tr = Float32, one scalar float32 operation at a time."""
    A = np.array(J, dtype=f32, order="F")
    n = A.shape[0]
    d = np.ones(n, dtype=f32)
    isc = np.ones(n, dtype=f32)
    two = f32(2)
    for _ in range(20):
        converged = True
        for i in range(n):
            c = f32(0)
            r = f32(0)
            for j in range(n):
                if j == i:
                    continue
                c = f32(c + abs(A[j, i]))
                r = f32(r + abs(A[i, j]))
            if c == 0 or r == 0:
                continue
            f = f32(1)
            s = f32(c + r)
            while c < f32(r / two):
                c, r, f = f32(c * two), f32(r / two), f32(f * two)
            while c >= f32(two * r):
                c, r, f = f32(c / two), f32(r * two), f32(f / two)
            if f32(c + r) < f32(f32(0.95) * s):
                converged = False
                d[i] = f32(d[i] * f)
                isc[i] = f32(isc[i] / f)
                A[i, :] = A[i, :] / f
                A[:, i] = A[:, i] * f
        if converged:
            break
    return A, d, isc


def bits(a):
    return np.asarray(a, dtype=f32).view(np.int32)


@pytest.mark.parametrize("n", list(range(1, 41)) + [64, 100, 127, 128, 129, 200, 257, 300])
def test_rowblock_matches_the_generic_sweep_like_the_reference(n):
    J = np.random.default_rng(n).standard_normal((n, n)).astype(f32)
    R64 = O.reduce(J.astype(np.float64), balance=False, path=1)
    Ae = O.reduce_f32(J, balance=False)
    Ag, ipg = generic_f32(J)
    assert np.array_equal(Ae.factors.astype(f32).astype(np.float64), Ae.factors), "not float values"
    assert np.array_equal(ipg, Ae.ipiv) and np.array_equal(Ae.ipiv, R64.ipiv)
    floor = 100 * n * np.finfo(f32).eps
    assert relerr(Ae.factors, R64.factors) <= 4 * relerr(Ag.astype(np.float64), R64.factors) + floor
    if n > 2:
        assert np.abs(np.tril(Ae.factors, -2)).max() <= 1.0


def _wilkinson(n):
    W = -np.tril(np.ones((n, n)), -1) + np.eye(n)
    W[:, -1] = 1.0
    return W


@pytest.mark.parametrize("which", range(5))
def test_structured_matrices_like_the_reference(which):
    g = np.random.default_rng(9)
    J = [_wilkinson(40), np.eye(30), np.arange(1.0, 10.0).reshape(3, 3),
         np.triu(g.standard_normal((50, 50)), 1), g.integers(-1, 2, (150, 150)).astype(np.float64)][which]
    Ae = O.reduce_f32(J, balance=False)
    Ag, ipg = generic_f32(J)
    assert np.array_equal(ipg, Ae.ipiv)
    assert np.allclose(Ae.factors, Ag, rtol=np.sqrt(np.finfo(f32).eps), atol=0) or \
        relerr(Ae.factors, Ag.astype(np.float64)) <= np.sqrt(np.finfo(f32).eps)


@pytest.mark.parametrize("n", [1, 2, 3, 9, 24, 41])
@pytest.mark.parametrize("graded", [False, True])
def test_balancing_bit_for_bit(n, graded):
    g = np.random.default_rng(300 + n)
    J = g.standard_normal((n, n))
    if graded:
        D = 2.0 ** g.integers(-12, 12, n)
        J = (J * D[None, :]) / D[:, None]
    Ab, d, isc = balance_f32(J)
    R = O.reduce_f32(J, balance=True)
    assert np.array_equal(bits(R.scale), bits(d)) and np.array_equal(bits(R.iscale), bits(isc))
    # the reduction after balancing is the unbalanced reduction of the balanced matrix
    Rb = O.reduce_f32(Ab, balance=False)
    assert np.array_equal(bits(R.factors), bits(Rb.factors)) and np.array_equal(R.ipiv, Rb.ipiv)


@pytest.mark.parametrize("n", [3, 17, 80, 200, 513, 1000])
@pytest.mark.parametrize("balance", [True, False])
def test_float_reconstruction(n, balance):
    J = np.random.default_rng(n).standard_normal((n, n)).astype(f32).astype(np.float64)
    R = O.reduce_f32(J, balance=balance)
    Z, Zi = R.Z(), R.Zinv()
    eps = np.finfo(f32).eps
    assert relerr(Z @ R.H @ Zi, J) < 50 * n * eps
    assert np.abs(np.tril(R.factors, -2)).max() <= 1.0
    for a in (R.factors, R.Ht, R.scale):
        assert np.array_equal(np.asarray(a, dtype=f32).astype(np.float64), a)


@pytest.mark.parametrize("n", [20, 33, 160, 300])
def test_blocked_float_form_like_the_reference(n):
    """test/threading.jl:58-79 with T = Float32: the blocked form takes the unblocked Float64
    reduction's pivots, and its factors are within 100 n eps(Float32) of them."""
    J = np.random.default_rng(n).standard_normal((n, n)).astype(np.float32)
    Ab, ipb = O.reduce_blocked_f32_raw(J)
    Ru = O.reduce(J.astype(np.float64), balance=False, path=1)
    assert np.array_equal(ipb, Ru.ipiv)
    assert np.linalg.norm(Ab - Ru.factors) <= 100 * n * np.finfo(np.float32).eps * np.linalg.norm(Ru.factors)
    assert np.array_equal(Ab.astype(np.float32).astype(np.float64), Ab)


def test_blocked_float_form_on_ties():
    """Gaussian-integer ties (many equal moduli, zero pivots): the blocked and unblocked float
    forms take the same pivots (test/threading.jl:62, the rand(-1:1) matrix)."""
    J = np.random.default_rng(9).integers(-1, 2, (200, 200)).astype(np.float32)
    Ab, ipb = O.reduce_blocked_f32_raw(J)
    Au = O.reduce_f32(J, balance=False)
    assert np.array_equal(ipb, Au.ipiv)


@pytest.mark.parametrize("n", [1024, 1100])
def test_reference_choice_from_1024(n):
    """From n = 1024 reduce_f32 runs the blocked form (the reference's choice, F:398, F:704):
    bit-identical to the raw blocked form after the same balancing, Z H Z^-1 = J to float
    accuracy, |l| <= 1."""
    J = np.random.default_rng(n).standard_normal((n, n)).astype(np.float32).astype(np.float64)
    R = O.reduce_f32(J, balance=False)
    Ab, ipb = O.reduce_blocked_f32_raw(J)
    assert np.array_equal(R.ipiv, ipb) and np.array_equal(R.factors, Ab)
    Rb = O.reduce_f32(J, balance=True)
    Z, Zi = Rb.Z(), Rb.Zinv()
    assert relerr(Z @ Rb.H @ Zi, J) < 50 * n * np.finfo(f32).eps
    assert np.abs(np.tril(Rb.factors, -2)).max() <= 1.0
