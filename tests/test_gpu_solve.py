"""The fit kernel's Gauss-Jordan solve (mrqmin_1_end_opt, Start.cu:2880-3006)
against the oracle's serial full-pivot solve (oracle/ps_oracle.c
pso_gauss_solve), through the ps_probe_solve test hook.

Matrices whose elimination is exact in binary floating point (every pivot
reciprocal, product and difference representable, proven with rational
arithmetic below) make the comparison bit-exact whatever the FMA contraction:
the pivot order, the tie-break (the last maximum in row-major order), the row
swaps and the zero-pivot partial solution must then agree exactly.  Tie-heavy
+-1 matrices (Sylvester Hadamard blocks, rows scaled by powers of two, rows
and columns permuted) exercise the tie-break at every step."""
from fractions import Fraction

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _exact_gj(A, b):
    """The serial solve in rationals; (err, x) if every intermediate value is
    a double, else None."""
    n = len(b)
    a = [[Fraction(float(x)) for x in row] for row in A]
    b = [Fraction(float(x)) for x in b]
    ipiv = [0] * n

    def rep(x):
        return Fraction(float(x)) == x

    for _ in range(n):
        big, irow, icol = Fraction(0), 0, 0
        for j in range(n):
            if ipiv[j] == 1:
                continue
            for k in range(n):
                if ipiv[k] == 0:
                    if abs(a[j][k]) >= big:
                        big, irow, icol = abs(a[j][k]), j, k
                elif ipiv[k] > 1:
                    return 1, b
        ipiv[icol] += 1
        if irow != icol:
            a[irow], a[icol] = a[icol], a[irow]
            b[irow], b[icol] = b[icol], b[irow]
        piv = a[icol][icol]
        if piv == 0:
            return 2, b
        pivinv = 1 / piv
        if not rep(pivinv):
            return None
        a[icol][icol] = Fraction(1)
        a[icol] = [x * pivinv for x in a[icol]]
        b[icol] *= pivinv
        if not all(rep(x) for x in a[icol]) or not rep(b[icol]):
            return None
        for ll in range(n):
            if ll == icol or a[ll][icol] == 0:
                if ll != icol:
                    a[ll][icol] = Fraction(0)
                continue
            dum = a[ll][icol]
            for l in range(n):
                base = 0 if l == icol else a[ll][l]
                p = a[icol][l] * dum
                if not rep(p) or not rep(base - p):
                    return None
                a[ll][l] = base - p
            p = b[icol] * dum
            if not rep(p) or not rep(b[ll] - p):
                return None
            b[ll] -= p
    return 0, b


def _sylvester(n):
    H = np.array([[1.0]])
    while H.shape[0] < n:
        H = np.block([[H, H], [H, -H]])
    return H


def _tie_heavy(rng, sizes):
    """Block-diagonal Hadamard blocks, rows scaled by powers of two, rows and
    columns permuted."""
    n = sum(sizes)
    A = np.zeros((n, n))
    o = 0
    for m in sizes:
        A[o:o + m, o:o + m] = _sylvester(m)
        o += m
    A *= 2.0 ** rng.integers(-2, 3, size=(n, 1))
    return A[rng.permutation(n)][:, rng.permutation(n)]


def _exact_cases(rng):
    cases = []
    specs = [[1], [2], [4], [8], [16], [16, 8, 4], [32], [32, 16, 8], [16, 16, 16, 8],
             [32, 32, 2], [8] * 8 + [4, 2, 1], [8] * 11, [8] * 10 + [4, 4, 1]]
    for sizes in specs:
        for _ in range(4):
            A = _tie_heavy(rng, sizes)
            b = rng.integers(-8, 9, size=A.shape[0]).astype(float)
            ref = _exact_gj(A, b)
            if ref is not None:
                cases.append((A, b, ref))
    return cases


def test_solve_exact_ties_bitwise():
    import oracle
    from ps_claude_opt_b200 import native

    rng = np.random.default_rng(2024)
    cases = _exact_cases(rng)
    assert len(cases) >= 20
    big = 0
    for A, b, (rerr, rx) in cases:
        oerr, ox = oracle.gauss_solve(A, b)
        assert oerr == rerr
        np.testing.assert_array_equal(ox, np.array([float(v) for v in rx]))
        err, x = native.probe_solve(A, b)
        assert err == oerr, A.shape
        np.testing.assert_array_equal(x, ox)
        big = max(big, A.shape[0])
    assert big > 64  # two row slots per thread


def test_solve_zero_pivot_partial_solution():
    """Rank-deficient exact systems end in the zero-pivot path (error 2) with
    the rows swapped and the partial solution the fit then applies."""
    import oracle
    from ps_claude_opt_b200 import native

    rng = np.random.default_rng(7)
    seen = 0
    for sizes in ([4], [8], [16], [16, 8], [8] * 9):
        for dup in range(3):
            A = _tie_heavy(rng, sizes)
            n = A.shape[0]
            i, j = rng.choice(n, 2, replace=False)
            if dup == 0:
                A[i] = A[j]
            elif dup == 1:
                A[:, i] = 0.0
            else:
                A[i] = 0.0
            b = rng.integers(-8, 9, size=n).astype(float)
            ref = _exact_gj(A, b)
            if ref is None:
                continue
            oerr, ox = oracle.gauss_solve(A, b)
            err, x = native.probe_solve(A, b)
            assert oerr == ref[0] == 2
            assert err == 2
            np.testing.assert_array_equal(x, ox)
            seen += 1
    assert seen >= 8
    # the all-zero matrix: the last zero in row-major order is the pivot
    err, x = native.probe_solve(np.zeros((5, 5)), np.arange(5.0))
    assert err == 2 and np.array_equal(x, np.arange(5.0))


@pytest.mark.parametrize("n", [1, 2, 3, 5, 24, 48, 56, 63, 64, 65, 80, 88, 89])
def test_solve_normal_matrices(n):
    """Damped J^T W J-like systems of every size class the fits use: the same
    pivots, so the solutions agree to rounding (the oracle does not contract
    a - b * c into an FMA)."""
    import oracle
    from ps_claude_opt_b200 import native

    rng = np.random.default_rng(100 + n)
    J = rng.standard_normal((3 * n + 5, n)) * np.exp(rng.uniform(-3, 3, size=n))
    A = J.T @ J
    A[np.diag_indices(n)] *= 1.001
    b = rng.standard_normal(n)
    oerr, ox = oracle.gauss_solve(A, b)
    err, x = native.probe_solve(A, b)
    assert err == oerr == 0
    scale = np.abs(ox).max()
    assert np.max(np.abs(x - ox)) <= 1e-9 * scale
    assert np.allclose(A @ x, b, rtol=0, atol=1e-8 * np.abs(A).max() * scale)


def test_solve_nan_paths():
    """NaN is never a pivot; with nothing but NaN left the serial scan takes
    (0, 0), and a second pass over column 0 is the bookkeeping error 1."""
    import oracle
    from ps_claude_opt_b200 import native

    for n in (1, 2, 3, 6):
        A = np.full((n, n), np.nan)
        b = np.ones(n)
        oerr, ox = oracle.gauss_solve(A, b)
        err, x = native.probe_solve(A, b)
        assert err == oerr
        assert np.array_equal(np.isnan(x), np.isnan(ox))
    rng = np.random.default_rng(5)
    for n, (i, j) in [(8, (0, 0)), (8, (3, 5)), (70, (66, 2)), (70, (1, 69))]:
        J = rng.standard_normal((2 * n, n))
        A = J.T @ J
        A[i, j] = np.nan
        b = rng.standard_normal(n)
        oerr, ox = oracle.gauss_solve(A, b)
        err, x = native.probe_solve(A, b)
        assert err == oerr
        assert np.array_equal(np.isnan(x), np.isnan(ox))
