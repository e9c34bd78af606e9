"""Known-answer systems for the full-pivot Gauss-Jordan solve (the solve of
mrqmin_1_end_opt, Start.cu:2880-3006): tie-heavy +-1 matrices (Sylvester
Hadamard blocks, rows scaled by powers of two, rows and columns permuted)
whose elimination is exact in binary floating point, proven with rational
arithmetic.  On such a system every correct implementation of the serial
algorithm, with or without FMA contraction, returns the same bits: the pivot
order, the tie-break (the last maximum in row-major order), the row swaps and
the zero-pivot partial solution are all fixed."""
from fractions import Fraction

import numpy as np


def exact_gj(A, b):
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


def sylvester(n):
    H = np.array([[1.0]])
    while H.shape[0] < n:
        H = np.block([[H, H], [H, -H]])
    return H


def tie_heavy(rng, sizes):
    """Block-diagonal Hadamard blocks, rows scaled by powers of two, rows and
    columns permuted."""
    n = sum(sizes)
    A = np.zeros((n, n))
    o = 0
    for m in sizes:
        A[o:o + m, o:o + m] = sylvester(m)
        o += m
    A *= 2.0 ** rng.integers(-2, 3, size=(n, 1))
    return A[rng.permutation(n)][:, rng.permutation(n)]


def exact_cases(rng):
    cases = []
    specs = [[1], [2], [4], [8], [16], [16, 8, 4], [32], [32, 16, 8], [16, 16, 16, 8],
             [32, 32, 2], [8] * 8 + [4, 2, 1], [8] * 11, [8] * 10 + [4, 4, 1]]
    for sizes in specs:
        for _ in range(4):
            A = tie_heavy(rng, sizes)
            b = rng.integers(-8, 9, size=A.shape[0]).astype(float)
            ref = exact_gj(A, b)
            if ref is not None:
                cases.append((A, b, ref))
    return cases


def rank_deficient_cases(rng):
    """Exact systems with a repeated row, a zero column or a zero row: the
    serial solve ends in its zero-pivot path (error 2)."""
    cases = []
    for sizes in ([4], [8], [16], [16, 8], [8] * 9):
        for dup in range(3):
            A = tie_heavy(rng, sizes)
            n = A.shape[0]
            i, j = rng.choice(n, 2, replace=False)
            if dup == 0:
                A[i] = A[j]
            elif dup == 1:
                A[:, i] = 0.0
            else:
                A[i] = 0.0
            b = rng.integers(-8, 9, size=n).astype(float)
            ref = exact_gj(A, b)
            if ref is not None:
                cases.append((A, b, ref))
    return cases
