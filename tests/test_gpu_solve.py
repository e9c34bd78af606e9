"""The fit kernel's Gauss-Jordan solve (mrqmin_1_end_opt, Start.cu:2880-3006)
against the oracle's serial full-pivot solve (oracle/ps_oracle.c
pso_gauss_solve), through the ps_probe_solve test hook.

On the exact known-answer systems of solve_cases the comparison is bit-exact
whatever the FMA contraction: pivot order, tie-break, row swaps and the
zero-pivot partial solution must agree exactly."""
import numpy as np
import pytest

import solve_cases

pytestmark = pytest.mark.gpu


def test_solve_exact_ties_bitwise():
    import oracle
    from ps_claude_opt_b200 import native

    cases = solve_cases.exact_cases(np.random.default_rng(2024))
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

    cases = solve_cases.rank_deficient_cases(np.random.default_rng(7))
    assert len(cases) >= 8
    for A, b, ref in cases:
        oerr, ox = oracle.gauss_solve(A, b)
        err, x = native.probe_solve(A, b)
        assert oerr == ref[0] == 2
        assert err == 2
        np.testing.assert_array_equal(x, ox)
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
