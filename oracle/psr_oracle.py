"""numpy restatement of the reference parallel Schur reduction (test infrastructure only).

Follows ``src/sinv/algorithms/psr/psr_seqsolve.py:20-943`` with the partition
helper of ``src/sinv/algorithms/psr/psr_utils.py:61-100``.  The reference runs
one partition per MPI process on dense N x N arrays and gathers the reduced
system on rank 0; this restatement runs the partitions one after another on
a dictionary of b x b blocks, with the same block operations in the same order
per partition, and inverts the reduced system densely as the reference does
(``psr_seqsolve.py:470-493``).  Returns the block-tridiagonal part of the
inverse (G_ii, G_{i,i+1}, G_{i+1,i}).
"""

import numpy as np


def divide(n, P):
    """Start block and block count of each partition (``psr_utils.py:61-100``):
    n // P blocks each, the remainder in the first partition."""
    base = n // P
    sizes = [n - base * (P - 1)] + [base] * (P - 1)
    starts = [0]
    for s in sizes[:-1]:
        starts.append(starts[-1] + s)
    return starts, sizes


def check(n, P):
    """``psr_utils.py:14-58``: at least three partitions (``psr_seqsolve.py:43-44``)
    and three block rows per partition."""
    if P < 3:
        raise ValueError("PSR needs at least 3 partitions")
    if n < 3 * P:
        raise ValueError("The number of blocks is to low. There should be at least 3 blockrows per process")


def _blocks(diag, upper, lower):
    n = diag.shape[0]
    A = {(i, i): diag[i].copy() for i in range(n)}
    for i in range(n - 1):
        A[(i, i + 1)] = upper[i].copy()
        A[(i + 1, i)] = lower[i].copy()
    return A


def reduce_topleft(A, L, U, Dinv, s, m):
    """Downward corner elimination, ``psr_seqsolve.py:160-177``."""
    for i in range(s + 1, s + m):
        Di = np.linalg.inv(A[(i - 1, i - 1)])
        Dinv[i - 1] = Di
        L[(i, i - 1)] = A[(i, i - 1)] @ Di
        U[(i - 1, i)] = Di @ A[(i - 1, i)]
        A[(i, i)] = A[(i, i)] - L[(i, i - 1)] @ A[(i - 1, i)]


def reduce_bottomright(A, L, U, Dinv, s, m):
    """Upward corner elimination, ``psr_seqsolve.py:215-232``."""
    for i in range(s + m - 2, s - 1, -1):
        Di = np.linalg.inv(A[(i + 1, i + 1)])
        Dinv[i + 1] = Di
        L[(i, i + 1)] = A[(i, i + 1)] @ Di
        U[(i + 1, i)] = Di @ A[(i + 1, i)]
        A[(i, i)] = A[(i, i)] - L[(i, i + 1)] @ A[(i + 1, i)]


def reduce_central(A, L, U, Dinv, s, m):
    """Central elimination keeping the top row, ``psr_seqsolve.py:270-310``;
    the couplings A[t, i] / A[i, t] (i >= t + 2) start as zero fill-in."""
    t = s
    zero = np.zeros_like(A[(t, t)])
    for i in range(s + 2, s + m):
        Di = np.linalg.inv(A[(i - 1, i - 1)])
        Dinv[i - 1] = Di
        L[(i, i - 1)] = A[(i, i - 1)] @ Di
        L[(t, i - 1)] = A[(t, i - 1)] @ Di
        U[(i - 1, i)] = Di @ A[(i - 1, i)]
        U[(i - 1, t)] = Di @ A[(i - 1, t)]
        A[(i, i)] = A[(i, i)] - L[(i, i - 1)] @ A[(i - 1, i)]
        A[(t, t)] = A[(t, t)] - L[(t, i - 1)] @ A[(i - 1, t)]
        A[(i, t)] = A.get((i, t), zero) - L[(i, i - 1)] @ A[(i - 1, t)]
        A[(t, i)] = A.get((t, i), zero) - L[(t, i - 1)] @ A[(i - 1, i)]


def reduced_rows(starts, sizes):
    """Block rows of the reduced system in its order (``psr_seqsolve.py:336-384``):
    the last row of partition 0, top and bottom rows of every central
    partition, the first row of the last partition."""
    P = len(starts)
    rows = [starts[0] + sizes[0] - 1]
    for p in range(1, P - 1):
        rows += [starts[p], starts[p] + sizes[p] - 1]
    rows.append(starts[P - 1])
    return rows


def produce_topleft(A, L, U, Dinv, G, s, m):
    """``psr_seqsolve.py:694-737`` (the i = s step touches no block)."""
    for i in range(s + m - 1, s, -1):
        G[(i, i - 1)] = -G[(i, i)] @ L[(i, i - 1)]
        G[(i - 1, i)] = -U[(i - 1, i)] @ G[(i, i)]
        G[(i - 1, i - 1)] = Dinv[i - 1] - U[(i - 1, i)] @ G[(i, i - 1)]


def produce_bottomright(A, L, U, Dinv, G, s, m):
    """``psr_seqsolve.py:740-783``."""
    for i in range(s, s + m - 1):
        G[(i, i + 1)] = -G[(i, i)] @ L[(i, i + 1)]
        G[(i + 1, i)] = -U[(i + 1, i)] @ G[(i, i)]
        G[(i + 1, i + 1)] = Dinv[i + 1] - U[(i + 1, i)] @ G[(i, i + 1)]


def produce_central(A, L, U, Dinv, G, s, m):
    """``psr_seqsolve.py:786-900``."""
    t, B = s, s + m - 1
    G[(B, B - 1)] = -G[(B, t)] @ L[(t, B - 1)] - G[(B, B)] @ L[(B, B - 1)]
    G[(B - 1, B)] = -U[(B - 1, B)] @ G[(B, B)] - U[(B - 1, t)] @ G[(t, B)]
    for i in range(B - 1, t, -1):
        G[(t, i)] = -G[(t, t)] @ L[(t, i)] - G[(t, i + 1)] @ L[(i + 1, i)]
        G[(i, t)] = -U[(i, i + 1)] @ G[(i + 1, t)] - U[(i, t)] @ G[(t, t)]
    for i in range(B - 1, t + 1, -1):
        G[(i, i)] = Dinv[i] - U[(i, t)] @ G[(t, i)] - U[(i, i + 1)] @ G[(i + 1, i)]
        G[(i - 1, i)] = -U[(i - 1, t)] @ G[(t, i)] - U[(i - 1, i)] @ G[(i, i)]
        G[(i, i - 1)] = -G[(i, t)] @ L[(t, i - 1)] - G[(i, i)] @ L[(i, i - 1)]
    G[(t + 1, t + 1)] = Dinv[t + 1] - U[(t + 1, t)] @ G[(t, t + 1)] - U[(t + 1, t + 2)] @ G[(t + 2, t + 1)]


def psr(diag, upper, lower, P):
    """Selected inversion by parallel Schur reduction over P partitions.

    Returns ``(G_diag, G_upper, G_lower)``."""
    n, b = diag.shape[0], diag.shape[1]
    check(n, P)
    starts, sizes = divide(n, P)
    A = _blocks(diag, upper, lower)
    L, U, Dinv, G = {}, {}, {}, {}
    for p in range(P):
        f = reduce_topleft if p == 0 else reduce_bottomright if p == P - 1 else reduce_central
        f(A, L, U, Dinv, starts[p], sizes[p])
    # reduced system (block tridiagonal in this order), inverted densely
    rows = reduced_rows(starts, sizes)
    R = len(rows)
    S = np.zeros((R * b, R * b), dtype=np.result_type(diag, upper, lower))
    for x, i in enumerate(rows):
        for y, j in enumerate(rows):
            if (i, j) in A and abs(x - y) <= 1:
                S[x * b:(x + 1) * b, y * b:(y + 1) * b] = A[(i, j)]
    GS = np.linalg.inv(S)
    for x, i in enumerate(rows):
        for y, j in enumerate(rows):
            if abs(x - y) <= 1:
                G[(i, j)] = GS[x * b:(x + 1) * b, y * b:(y + 1) * b]
    for p in range(P):
        f = produce_topleft if p == 0 else produce_bottomright if p == P - 1 else produce_central
        f(A, L, U, Dinv, G, starts[p], sizes[p])
    Gd = np.stack([G[(i, i)] for i in range(n)])
    Gu = np.stack([G[(i, i + 1)] for i in range(n - 1)]) if n > 1 else np.zeros((0, b, b), Gd.dtype)
    Gl = np.stack([G[(i + 1, i)] for i in range(n - 1)]) if n > 1 else np.zeros((0, b, b), Gd.dtype)
    return Gd, Gu, Gl
