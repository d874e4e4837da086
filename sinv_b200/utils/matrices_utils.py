"""Test-matrix generators and block-tridiagonal converters.

Same names, arguments and outputs as the reference's public helpers in
``src/sinv/utils/matrices_utils.py`` (reached there as ``sinv.utils.matu``),
so code written against the reference keeps working after an import change.
The random generators use numpy's legacy global seed exactly as the reference
does (``matrices_utils.py:37-45``), so a given seed yields the same matrix.
"""

import numpy as np


def generateRandomNumpyMat(matrice_size, is_complex=False, is_symmetric=False, seed=None):
    """Dense random matrix, uniform [0, 1) entries (``matrices_utils.py:12-51``).

    With ``is_complex`` the real part is drawn first, then the imaginary part.
    With ``is_symmetric`` the result is ``A + A.T`` (plain transpose).
    """
    if seed is not None:
        np.random.seed(seed)
    if is_complex:
        re = np.random.rand(matrice_size, matrice_size)
        im = np.random.rand(matrice_size, matrice_size)
        A = re + 1j * im
    else:
        A = np.random.rand(matrice_size, matrice_size)
    if is_symmetric:
        A = A + A.T
    return A


def generateBandedDiagonalMatrix(matrice_size, matrice_bandwidth, is_complex=False,
                                 is_symmetric=False, seed=None):
    """Random matrix with entries outside ``|i - j| <= bandwidth`` zeroed
    (``matrices_utils.py:55-91``)."""
    A = generateRandomNumpyMat(matrice_size, is_complex, is_symmetric, seed)
    idx = np.arange(matrice_size)
    outside = np.abs(idx[:, None] - idx[None, :]) > matrice_bandwidth
    A[outside] = 0
    return A


def transformToSymmetric(A):
    """``A + A.T`` (``matrices_utils.py:95-111``)."""
    return A + A.T


def convertDenseToBlkTridiag(A, blocksize):
    """Dense -> ``(diag[n,b,b], upper[n-1,b,b], lower[n-1,b,b])``
    (``matrices_utils.py:115-151``); ``upper[i]`` = A_{i,i+1},
    ``lower[i]`` = A_{i+1,i}."""
    b = blocksize
    n = int(np.ceil(A.shape[0] / b))
    diag = np.zeros((n, b, b), dtype=A.dtype)
    upper = np.zeros((n - 1, b, b), dtype=A.dtype)
    lower = np.zeros((n - 1, b, b), dtype=A.dtype)
    for i in range(n):
        diag[i] = A[i * b:(i + 1) * b, i * b:(i + 1) * b]
        if i < n - 1:
            upper[i] = A[i * b:(i + 1) * b, (i + 1) * b:(i + 2) * b]
            lower[i] = A[(i + 1) * b:(i + 2) * b, i * b:(i + 1) * b]
    return diag, upper, lower


def convertBlkTridiagToDense(A_diagblk, A_upperblk, A_lowerblk):
    """Block arrays -> dense matrix (``matrices_utils.py:155-189``)."""
    b = A_diagblk.shape[1]
    n = A_diagblk.shape[0]
    A = np.zeros((n * b, n * b), dtype=A_diagblk.dtype)
    for i in range(n):
        A[i * b:(i + 1) * b, i * b:(i + 1) * b] = A_diagblk[i]
        if i < n - 1:
            A[i * b:(i + 1) * b, (i + 1) * b:(i + 2) * b] = A_upperblk[i]
            A[(i + 1) * b:(i + 2) * b, i * b:(i + 1) * b] = A_lowerblk[i]
    return A
