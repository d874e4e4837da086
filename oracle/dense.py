"""Dense FP64 oracle (test infrastructure only).

The reference tests' own oracle: the whole matrix is assembled
(``src/sinv/utils/matrices_utils.py:155-189``), inverted with
``numpy.linalg.inv`` and cut back into block-tridiagonal pieces
(``matrices_utils.py:115-151``); see ``tests/rgf_tests/rgf_test.py:81`` and
``tests/bcr_tests/bcr_serial_test.py:68``.
"""

import numpy as np


def to_dense(diag, upper, lower):
    """Block arrays -> dense matrix (``matrices_utils.py:155-189``)."""
    n, b = diag.shape[0], diag.shape[1]
    A = np.zeros((n * b, n * b), dtype=np.result_type(diag, upper, lower))
    for i in range(n):
        A[i * b:(i + 1) * b, i * b:(i + 1) * b] = diag[i]
        if i < n - 1:
            A[i * b:(i + 1) * b, (i + 1) * b:(i + 2) * b] = upper[i]
            A[(i + 1) * b:(i + 2) * b, i * b:(i + 1) * b] = lower[i]
    return A


def to_blocks(A, b):
    """Dense matrix -> (diag, upper, lower) blocks (``matrices_utils.py:115-151``)."""
    n = int(np.ceil(A.shape[0] / b))
    d = np.zeros((n, b, b), dtype=A.dtype)
    u = np.zeros((max(n - 1, 0), b, b), dtype=A.dtype)
    l = np.zeros((max(n - 1, 0), b, b), dtype=A.dtype)
    for i in range(n):
        d[i] = A[i * b:(i + 1) * b, i * b:(i + 1) * b]
        if i < n - 1:
            u[i] = A[i * b:(i + 1) * b, (i + 1) * b:(i + 2) * b]
            l[i] = A[(i + 1) * b:(i + 2) * b, i * b:(i + 1) * b]
    return d, u, l


def inv_selected(diag, upper, lower):
    """Selected blocks of the dense FP64 inverse (complex128 / float64)."""
    diag = np.asarray(diag)
    wide = np.complex128 if np.iscomplexobj(diag) else np.float64
    A = to_dense(np.asarray(diag, wide), np.asarray(upper, wide), np.asarray(lower, wide))
    return to_blocks(np.linalg.inv(A), diag.shape[1])


def rel_fro(x, ref):
    """Relative Frobenius error ||x - ref|| / ||ref||."""
    x = np.asarray(x)
    ref = np.asarray(ref)
    den = np.linalg.norm(ref)
    if den == 0:
        return float(np.linalg.norm(x))
    return float(np.linalg.norm(x - ref) / den)
