"""The wide-band factorisation's algorithm against Strut's BandGeneral, on the CPU.

Strut factors the band without interchanges and, at the first column whose pivot test fails (a
sub-diagonal entry strictly larger than the pivot), restarts from the original matrix with a
dense partial-pivot LU (linear_solver_backend.mojo:175-240, 631-680).  The global-memory band path
(`large_factor_kernel`) instead runs one blocked partial-pivot band LU in 3 bw + 1 slots per row,
with the right-hand side carried as one more column: panels of 32 columns factored with whole-row
interchanges, then every trailing column takes the panel's interchanges first and its
eliminations after, in column order.  Both are restated here in plain Python (no fused
multiply-add) and must agree bit for bit: the same interchanges, the same subtractions on every
entry in the same order.  The CUDA kernel itself is checked against the oracle by the GPU tests.
"""
import numpy as np
import pytest

PANEL, TILE = 32, 16


def strut_band_general(A, b, bw):
    """Strut's BandGeneral: band LU without interchanges, dense partial-pivot LU from the
    original matrix when a column's pivot test fails; forward and back substitution."""
    n = A.shape[0]
    M = A.copy()
    dense = False
    for k in range(n):
        i1 = min(n - 1, k + bw)
        prow, pabs = k, 0.0
        for r in range(k, i1 + 1):
            if abs(M[r, k]) > pabs:
                pabs, prow = abs(M[r, k]), r
        assert pabs > 1e-14
        if prow != k:
            dense = True
            break
        for i in range(k + 1, i1 + 1):
            f = M[i, k] / M[k, k]
            M[i, k] = f
            if f == 0.0:
                continue
            for j in range(k + 1, min(n - 1, k + bw) + 1):
                M[i, j] = M[i, j] - f * M[k, j]
    piv = list(range(n))
    if dense:
        M = A.copy()
        for col in range(n):
            prow, pabs = col, abs(M[col, col])
            for row in range(col + 1, n):
                if abs(M[row, col]) > pabs:
                    pabs, prow = abs(M[row, col]), row
            if prow != col:
                M[[col, prow], :] = M[[prow, col], :]
                piv[col], piv[prow] = piv[prow], piv[col]
            for row in range(col + 1, n):
                f = M[row, col] / M[col, col]
                M[row, col] = f
                if f == 0.0:
                    continue
                for j in range(col + 1, n):
                    M[row, j] = M[row, j] - f * M[col, j]
    y = np.zeros(n)
    for i in range(n):
        s = b[piv[i]]
        for j in range(i):
            s = s - M[i, j] * y[j]
        y[i] = s
    return np.triu(M), y, dense


def blocked_partial_pivot(A, b, bw):
    """The global-memory path's schedule: returns U (dense) and L^-1 P b."""
    n = A.shape[0]
    lo, wid = bw, 3 * bw + 1  # row i holds columns i - bw .. i + 2 bw

    def slot(i, j):
        return i * wid + (j - i + lo)

    B = np.zeros(n * wid)
    for i in range(n):
        for j in range(max(0, i - bw), min(n, i + bw + 1)):
            B[slot(i, j)] = A[i, j]
    w = b.copy()
    P = min(PANEL, max(bw, 1))
    for k0 in range(0, n, P):
        kb = min(P, n - k0)
        r1 = min(n - 1, k0 + kb - 1 + bw)
        pr = r1 - k0 + 1
        c1 = min(n - 1, k0 + kb - 1 + 2 * bw)
        # panel: whole rows (multipliers included) interchanged
        pan = np.zeros((pr, kb))
        for r in range(pr):
            for c in range(kb):
                if -bw <= c - r <= 2 * bw:
                    pan[r, c] = B[slot(k0 + r, k0 + c)]
        perm = list(range(pr))
        for c in range(kb):
            last = min(pr - 1, c + bw)
            p, best = c, abs(pan[c, c])
            for r in range(c + 1, last + 1):
                if abs(pan[r, c]) > best:
                    best, p = abs(pan[r, c]), r
            assert best > 1e-14
            if p != c:
                pan[[c, p], :] = pan[[p, c], :]
                perm[c], perm[p] = perm[p], perm[c]
            for r in range(c + 1, last + 1):
                f = pan[r, c] / pan[c, c]
                pan[r, c] = f
                for q in range(c + 1, kb):
                    pan[r, q] = pan[r, q] - f * pan[c, q]
        for r in range(kb):
            for c in range(r, kb):
                B[slot(k0 + r, k0 + c)] = pan[r, c]
        # trailing tiles and the right-hand side: interchanges first, then column order
        ncols = c1 - (k0 + kb) + 1
        ntiles = (-(-ncols // TILE) if ncols > 0 else 0) + 1
        for tile in range(ntiles):
            rhs = tile == ntiles - 1
            j0 = k0 + kb + tile * TILE
            ct = 1 if rhs else min(TILE, c1 - j0 + 1)
            S = np.zeros((pr, ct))
            for r in range(pr):
                src = k0 + perm[r]
                for q in range(ct):
                    if rhs:
                        S[r, q] = w[src]
                    elif -bw <= j0 + q - src <= 2 * bw:
                        S[r, q] = B[slot(src, j0 + q)]
            for sc in range(kb):
                for r in range(sc + 1, pr):
                    for q in range(ct):
                        S[r, q] = S[r, q] - pan[r, sc] * S[sc, q]
            for r in range(pr):
                i = k0 + r
                for q in range(ct):
                    if rhs:
                        w[i] = S[r, q]
                    elif -bw <= j0 + q - i <= 2 * bw:
                        B[slot(i, j0 + q)] = S[r, q]
                    else:
                        assert S[r, q] == 0.0  # no fill beyond 2 bw
    U = np.zeros((n, n))
    for i in range(n):
        for j in range(i, min(n, i + 2 * bw + 1)):
            U[i, j] = B[slot(i, j)]
    return U, w


def _system(n, bw, seed, weak_diagonal):
    rng = np.random.default_rng(seed)
    A = np.zeros((n, n))
    for i in range(n):
        for j in range(max(0, i - bw), min(n, i + bw + 1)):
            A[i, j] = rng.normal()
        if not weak_diagonal or i % 3 == 0:
            A[i, i] = 4.0 * (bw + 1) * np.sign(A[i, i] or 1.0)
    return A, rng.normal(size=n)


@pytest.mark.parametrize("n,bw,weak", [(70, 3, True), (90, 12, True), (75, 33, True), (64, 9, False),
                                       (40, 1, True)])
def test_same_arithmetic_as_band_then_dense(n, bw, weak):
    A, b = _system(n, bw, 100 + n + bw, weak)
    U_ref, y_ref, dense = strut_band_general(A, b, bw)
    U, y = blocked_partial_pivot(A, b, bw)
    assert dense == weak  # the weak-diagonal systems need interchanges, the others none
    assert np.array_equal(U, U_ref)
    assert np.array_equal(y, y_ref)
    x = np.linalg.solve(A, b)
    xs = np.zeros(n)
    for i in range(n - 1, -1, -1):
        s = y[i]
        for j in range(i + 1, n):
            s = s - U[i, j] * xs[j]
        xs[i] = s / U[i, i]
    assert np.max(np.abs(xs - x)) <= 1e-10 * np.max(np.abs(x))
