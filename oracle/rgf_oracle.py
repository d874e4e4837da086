"""numpy restatement of the reference serial RGF (test infrastructure only).

Follows ``src/sinv/algorithms/rgf/rgf.py:17-64`` operation by operation, on
the block-array layout of ``src/sinv/utils/matrices_utils.py:115-151``
(``diag[n,b,b]``, ``upper[n-1,b,b]`` = A_{i,i+1}, ``lower[n-1,b,b]`` = A_{i+1,i}).
The products keep the reference's left-to-right association so that the
rounding matches the reference bit for bit on the same BLAS.
"""

import numpy as np


def rgf(diag, upper, lower, sym_mat=False, save_off_diag=True):
    """Selected inverse of a block-tridiagonal matrix, reference operation order.

    Returns ``(G_diag, G_upper, G_lower)``.  When ``save_off_diag`` is False
    the off-diagonal outputs are all NaN, as in ``rgf.py:41`` where G starts
    as ``A.copy() * np.nan`` and ``rgf.py:55`` skips the off-diagonal writes.
    """
    diag = np.asarray(diag)
    upper = np.asarray(upper)
    lower = np.asarray(lower)
    n = diag.shape[0]
    # rgf.py:41 -- output storage starts as NaN everywhere
    G_diag = np.full_like(diag, np.nan)
    G_upper = np.full_like(upper, np.nan)
    G_lower = np.full_like(lower, np.nan)
    # rgf.py:44 -- g_0 = A_00^{-1}
    G_diag[0] = np.linalg.inv(diag[0])
    # rgf.py:47-48 -- forward sweep of left-connected inverses
    for i in range(1, n):
        G_diag[i] = np.linalg.inv(diag[i] - lower[i - 1] @ G_diag[i - 1] @ upper[i - 1])
    # rgf.py:51-62 -- backward sweep
    for i in range(n - 2, -1, -1):
        g_ii = G_diag[i].copy()
        lf = G_diag[i + 1] @ lower[i] @ g_ii                       # rgf.py:53
        if save_off_diag:
            G_lower[i] = -lf                                        # rgf.py:56
            if sym_mat:
                G_upper[i] = G_lower[i].T                           # rgf.py:58 (plain transpose)
            else:
                G_upper[i] = -g_ii @ upper[i] @ G_diag[i + 1]      # rgf.py:60
        G_diag[i] = g_ii + g_ii @ upper[i] @ lf                     # rgf.py:62
    return G_diag, G_upper, G_lower


def gauss_jordan_inverse(a):
    """Pivot-free in-place Gauss-Jordan inverse (the CUDA kernels' algorithm).

    Not a reference function: the reference calls ``np.linalg.inv`` (LAPACK,
    partially pivoted).  This is the elimination order the device inverse
    uses, kept here so tests can separate "pivot-free elimination error"
    from "kernel error".  Returns ``(inverse, min |pivot|)``.
    """
    a = np.array(a, dtype=np.result_type(a, np.float64), copy=True)
    n = a.shape[0]
    minp = np.inf
    for k in range(n):
        piv = a[k, k]
        minp = min(minp, abs(piv))
        p = 1.0 / piv
        col = a[:, k].copy()
        row = a[k, :] * p
        a -= np.outer(col, row)
        a[k, :] = row
        a[:, k] = -col * p
        a[k, k] = p
    return a, minp


def rgf_flops(n, b):
    """Canonical real-flop count of one RGF selected inversion.

    8 (n-1) complex b^3 GEMMs at 8 real flops per complex multiply-add, plus n
    complex inversions counted as 8 b^3 each: F = 8 b^3 (8 (n-1) + n).  The
    count follows the reference schedule ``rgf.py:47-62`` and does not change
    with the schedule a faster implementation uses.
    """
    return 8.0 * float(b) ** 3 * (8 * (n - 1) + n)
