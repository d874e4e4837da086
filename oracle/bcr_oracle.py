"""numpy restatement of the reference serial block cyclic reduction (test infrastructure only).

Follows ``src/sinv/algorithms/bcr/bcr_serial.py:19-467`` and the padding /
schedule helpers of ``src/sinv/algorithms/bcr/bcr_utils.py:17-129``.  The
reference works on dense N x N arrays; this restatement keeps the same block
operations in the same order on a dictionary of b x b blocks, which makes it
cheap enough to run at the sizes the tests use.  Identity padding is kept
(``bcr_utils.py:44-71``) so the arithmetic, including the work on padding
rows, is the reference's.
"""

import math

import numpy as np


def distance_to_power_of_two(nblocks):
    """Blocks to add so the count becomes 2^p - 1 (``bcr_utils.py:17-40``)."""
    p = math.ceil(math.log2(nblocks + 1))
    return 2 ** p - 1 - nblocks


def production_rows(level, nblocks):
    """``(i_from, i_prod)`` of one production level (``bcr_utils.py:75-129``,
    inline copy at ``bcr_serial.py:417-434``)."""
    stride = 2 ** level
    i_from = list(range(2 ** (level + 1) - 1, nblocks, 2 ** (level + 1)))
    i_prod = []
    for x, f in enumerate(i_from):
        if x == 0:
            i_prod.append(f - stride)
            i_prod.append(f + stride)
        else:
            if i_prod[x] != f - stride:
                i_prod.append(f - stride)
            i_prod.append(f + stride)
    return i_from, i_prod


class _Blocks(dict):
    """Sparse b x b block store; absent blocks read as zero (the dense
    reference arrays start as ``np.zeros``, ``bcr_serial.py:47-49``)."""

    def __init__(self, b, dtype):
        super().__init__()
        self.b = b
        self.dtype = dtype

    def __missing__(self, key):
        return np.zeros((self.b, self.b), dtype=self.dtype)


def _reduce(A, L, U, row, level, i_elim, nblocks):
    """One reduction towards kept row ``i_elim[row]`` (``bcr_serial.py:66-169``)."""
    off = 2 ** level
    j = i_elim[row]
    i = j - off
    k = j + off
    if i >= 0:                                                   # :119
        A_ii_inv = np.linalg.inv(A[i, i])                       # :121
        U[i, j] = A_ii_inv @ A[i, j]                            # :124-125
        L[j, i] = A[j, i] @ A_ii_inv                            # :127-128
        A[j, j] = A[j, j] - L[j, i] @ A[i, j]                   # :130-133
        # :137 compares against i_elim[0]; the fill-in target h = i - off is
        # an empty slice in the reference when negative, i.e. no write.
        if i != i_elim[0] and i - off >= 0:
            A[j, i - off] = -L[j, i] @ A[i, i - off]            # :138-142
    if k <= nblocks - 1:                                         # :146
        A_kk_inv = np.linalg.inv(A[k, k])                       # :148
        U[k, j] = A_kk_inv @ A[k, j]                            # :150-151
        L[j, k] = A[j, k] @ A_kk_inv                            # :153-154
        A[j, j] = A[j, j] - L[j, k] @ A[k, j]                   # :156-159
        # :163; l = k + off past the last block is an empty slice there.
        if k != i_elim[-1] and k + off <= nblocks - 1:
            A[j, k + off] = -L[j, k] @ A[k, k + off]            # :164-168


def _corner_produce(A, L, U, G, k_from, k_to):
    """``bcr_serial.py:253-304``."""
    G[k_from, k_to] = -1 * G[k_from, k_from] @ L[k_from, k_to]
    G[k_to, k_from] = -U[k_to, k_from] @ G[k_from, k_from]
    G[k_to, k_to] = np.linalg.inv(A[k_to, k_to]) - G[k_to, k_from] @ L[k_from, k_to]


def _center_produce(A, L, U, G, k_above, k_to, k_below):
    """``bcr_serial.py:308-383``."""
    G[k_above, k_to] = (-G[k_above, k_above] @ L[k_above, k_to]
                        - G[k_above, k_below] @ L[k_below, k_to])
    G[k_below, k_to] = (-G[k_below, k_above] @ L[k_above, k_to]
                        - G[k_below, k_below] @ L[k_below, k_to])
    G[k_to, k_above] = (-U[k_to, k_above] @ G[k_above, k_above]
                        - U[k_to, k_below] @ G[k_below, k_above])
    G[k_to, k_below] = (-U[k_to, k_above] @ G[k_above, k_below]
                        - U[k_to, k_below] @ G[k_below, k_below])
    G[k_to, k_to] = (np.linalg.inv(A[k_to, k_to])
                     - G[k_to, k_above] @ L[k_above, k_to]
                     - G[k_to, k_below] @ L[k_below, k_to])


def bcr_blocks(diag, upper, lower):
    """BCR selected inversion on block arrays, reference operation order.

    Returns ``(G_diag, G_upper, G_lower, G_blocks)`` where ``G_blocks`` is the
    full dictionary of produced blocks (the reference's dense G also holds the
    stride-2^l blocks of the production tree).
    """
    diag = np.asarray(diag)
    upper = np.asarray(upper)
    lower = np.asarray(lower)
    n, b = diag.shape[0], diag.shape[1]
    dtype = diag.dtype
    npad = n + distance_to_power_of_two(n)                       # bcr_serial.py:42-45
    A = _Blocks(b, dtype)
    L = _Blocks(b, dtype)
    U = _Blocks(b, dtype)
    G = _Blocks(b, dtype)
    for i in range(n):
        A[i, i] = diag[i].copy()
        if i < n - 1:
            A[i, i + 1] = upper[i].copy()
            A[i + 1, i] = lower[i].copy()
    for i in range(n, npad):                                     # bcr_utils.py:66-69
        A[i, i] = np.eye(b, dtype=dtype)
    # reduce_bcr, bcr_serial.py:173-216
    height = int(math.log2(npad))
    root = 0
    for level in range(height):
        stride = 2 ** (level + 1)
        i_elim = list(range(stride - 1, npad, stride))
        for row in range(len(i_elim)):
            _reduce(A, L, U, row, level, i_elim, npad)
        root = i_elim[-1]
    # invert_block, bcr_serial.py:220-249
    G[root, root] = np.linalg.inv(A[root, root])
    # produce_bcr, bcr_serial.py:387-466
    for level in range(height - 1, -1, -1):
        stride = 2 ** level
        _, i_prod = production_rows(level, npad)
        for x, k_to in enumerate(i_prod):
            if x == 0:
                _corner_produce(A, L, U, G, k_to + stride, k_to)
            if x != 0 and x == len(i_prod) - 1:
                if i_prod[-1] <= npad - stride - 1:
                    _center_produce(A, L, U, G, k_to - stride, k_to, k_to + stride)
                else:
                    _corner_produce(A, L, U, G, k_to - stride, k_to)
            if x != 0 and x != len(i_prod) - 1:
                _center_produce(A, L, U, G, k_to - stride, k_to, k_to + stride)
    G_diag = np.stack([G[i, i] for i in range(n)])
    G_upper = np.stack([G[i, i + 1] for i in range(n - 1)]) if n > 1 else np.zeros((0, b, b), dtype)
    G_lower = np.stack([G[i + 1, i] for i in range(n - 1)]) if n > 1 else np.zeros((0, b, b), dtype)
    return G_diag, G_upper, G_lower, G


def bcr_serial(A, blocksize):
    """Dense-in, dense-out form of ``bcr_serial.py:19-62``.

    The returned dense G holds every block the production tree writes, cropped
    to the unpadded size (``bcr_serial.py:60``).
    """
    A = np.asarray(A)
    n = A.shape[0] // blocksize
    b = blocksize
    diag = np.stack([A[i * b:(i + 1) * b, i * b:(i + 1) * b] for i in range(n)])
    upper = np.stack([A[i * b:(i + 1) * b, (i + 1) * b:(i + 2) * b] for i in range(n - 1)]) \
        if n > 1 else np.zeros((0, b, b), A.dtype)
    lower = np.stack([A[(i + 1) * b:(i + 2) * b, i * b:(i + 1) * b] for i in range(n - 1)]) \
        if n > 1 else np.zeros((0, b, b), A.dtype)
    _, _, _, blocks = bcr_blocks(diag, upper, lower)
    Gd = np.zeros((n * b, n * b), dtype=A.dtype)
    for (r, c), blk in blocks.items():
        if r < n and c < n:
            Gd[r * b:(r + 1) * b, c * b:(c + 1) * b] = blk
    return Gd
