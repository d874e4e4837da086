"""numpy restatement of the reference PDIV / pairwise selected inversion (test infrastructure only).

Follows ``src/sinv/algorithms/pdiv/pdiv_localmap.py:27-1436`` with the
partitioning of ``src/sinv/algorithms/pdiv/pdiv_utils.py:16-171``.  The
reference runs one partition per MPI process (a power of two of them): each
inverts its partition densely (``:94-116``), then log2(P) reduction steps
merge neighbouring groups of processes through the bridge blocks between
them, each process keeping twelve b x b "matrix maps" (how its final blocks
follow from its local inverse) and eight "cross maps" (for the bridge blocks
of the inverse), exchanged point to point (``:188-252``, ``:279-900``);
finally each process produces its tridiagonal blocks and the bridge to the
next partition (``:903-1436``).

Here the processes are emulated one after another.  Every message of a
reduction step carries values from before that step's updates (``get_U`` and
``get_nextprocess_matrixmap`` run before ``update_crossmap`` and
``update_matrixmap``), so each step first snapshots every process's maps and
then updates each process from the snapshot.  The maps a process receives
from its neighbour persist across steps, as ``l_M_ip1`` does in the reference.
Returns the block-tridiagonal part of the inverse (G_ii, G_{i,i+1}, G_{i+1,i}).
"""

import math

import numpy as np

from .psr_oracle import divide


def check(n, P):
    """``pdiv_utils.py:16-81``: a power-of-two process count, no more than the blocks."""
    if P < 1 or not math.log2(P).is_integer():
        raise ValueError("The number of processes must be a power of 2.")
    if n < P:
        raise ValueError("The number of blocks must be greater than the number of processes.")


def middle(start, end):
    """``pdiv_localmap.py:254-276``."""
    return start - 1 + math.ceil((end - start) / 2)


class Part:
    """One process: its inverted partition K (dense) and its maps."""

    def __init__(self, K, b, dtype):
        self.K, self.b = K, b
        self.last = K.shape[0] // b - 1
        eye = np.identity(b, dtype=dtype)
        # initialize_matrixmaps / initialize_crossmaps, :119-185
        self.M = [eye.copy() if i in (0, 3, 4, 7) else np.zeros((b, b), dtype) for i in range(12)]
        self.C = [np.zeros((b, b), dtype) for _ in range(12)]
        self.Mip1 = [np.zeros((b, b), dtype) for _ in range(12)]

    def blk(self, i, j):
        b = self.b
        return self.K[i * b:(i + 1) * b, j * b:(j + 1) * b]

    # produce_* elements, :1003-1180, written over this process's maps M
    def toprow(self, M, col):
        return M[0] @ self.blk(0, col) + M[1] @ self.blk(self.last, col)

    def rightcol(self, M, row):
        return self.blk(row, 0) @ M[2] + self.blk(row, self.last) @ M[3]

    def leftcol(self, M, row):
        return self.blk(row, 0) @ M[4] + self.blk(row, self.last) @ M[5]

    def botrow(self, M, col):
        return M[6] @ self.blk(0, col) + M[7] @ self.blk(self.last, col)

    def element(self, M, r, c):
        f, l = 0, self.last
        return (self.blk(r, c) + self.blk(r, f) @ M[8] @ self.blk(f, c) + self.blk(r, f) @ M[9] @ self.blk(l, c)
                + self.blk(r, l) @ M[10] @ self.blk(f, c) + self.blk(r, l) @ M[11] @ self.blk(l, c))


def crossmap_upper(M, Mn, C, Bu, J, b):
    """``:600-644``."""
    J12 = J[:b, b:]
    C[0] -= M[2] @ Bu @ J12 @ Mn[6]
    C[1] -= M[2] @ Bu @ J12 @ Mn[7]
    C[2] -= M[3] @ Bu @ J12 @ Mn[6]
    C[3] -= M[3] @ Bu @ J12 @ Mn[7]
    C[4] -= Mn[2] @ Bu @ J12 @ M[6]
    C[5] -= Mn[2] @ Bu @ J12 @ M[7]
    C[6] -= Mn[3] @ Bu @ J12 @ M[6]
    C[7] -= Mn[3] @ Bu @ J12 @ M[7]


def crossmap_middle(M, Mn, C, Bu, Bl, J, b):
    """``:647-697``."""
    J11, J22 = J[:b, :b], J[b:, b:]
    C[0] -= M[2] @ Bu @ J11 @ Mn[0]
    C[1] -= M[2] @ Bu @ J11 @ Mn[1]
    C[2] -= M[3] @ Bu @ J11 @ Mn[0]
    C[3] -= M[3] @ Bu @ J11 @ Mn[1]
    C[4] -= Mn[4] @ Bl @ J22 @ M[6]
    C[5] -= Mn[4] @ Bl @ J22 @ M[7]
    C[6] -= Mn[5] @ Bl @ J22 @ M[6]
    C[7] -= Mn[5] @ Bl @ J22 @ M[7]


def crossmap_lower(M, Mn, C, Bl, J, b):
    """``:700-744``."""
    J21 = J[b:, :b]
    C[0] -= M[4] @ Bl @ J21 @ Mn[0]
    C[1] -= M[4] @ Bl @ J21 @ Mn[1]
    C[2] -= M[5] @ Bl @ J21 @ Mn[0]
    C[3] -= M[5] @ Bl @ J21 @ Mn[1]
    C[4] -= Mn[4] @ Bl @ J21 @ M[0]
    C[5] -= Mn[4] @ Bl @ J21 @ M[1]
    C[6] -= Mn[5] @ Bl @ J21 @ M[0]
    C[7] -= Mn[5] @ Bl @ J21 @ M[1]


def matrixmap_upper(M, U, Bu, Bl, J, b):
    """``:780-830``; statement order kept (later lines read earlier updates)."""
    UUR, ULL, DUR, DLL = U[0], U[1], U[4], U[5]
    J11, J12, J22 = J[:b, :b], J[:b, b:], J[b:, b:]
    M[8] = M[8] + M[2] @ Bu @ J12 @ M[6]
    M[9] = M[9] + M[2] @ Bu @ J12 @ M[7]
    M[10] = M[10] + M[3] @ Bu @ J12 @ M[6]
    M[11] = M[11] + M[3] @ Bu @ J12 @ M[7]
    M[0] = M[0] + UUR @ Bu @ J12 @ M[6]
    M[1] = M[1] + UUR @ Bu @ J12 @ M[7]
    M[4] = M[4] + M[2] @ Bu @ J12 @ ULL
    M[5] = M[5] + M[3] @ Bu @ J12 @ ULL
    M[2] = M[2] @ Bu @ J11 @ DUR
    M[3] = M[3] @ Bu @ J11 @ DUR
    M[6] = DLL @ Bl @ J22 @ M[6]
    M[7] = DLL @ Bl @ J22 @ M[7]


def matrixmap_lower(M, U, Bu, Bl, J, b):
    """``:833-900``; statement order kept."""
    UUR, ULL, DUR, DLL = U[0], U[1], U[4], U[5]
    J11, J21, J22 = J[:b, :b], J[b:, :b], J[b:, b:]
    M[8] = M[8] + M[4] @ Bl @ J21 @ M[0]
    M[9] = M[9] + M[4] @ Bl @ J21 @ M[1]
    M[10] = M[10] + M[5] @ Bl @ J21 @ M[0]
    M[11] = M[11] + M[5] @ Bl @ J21 @ M[1]
    M[2] = M[2] + M[4] @ Bl @ J21 @ DUR
    M[3] = M[3] + M[5] @ Bl @ J21 @ DUR
    M[4] = M[4] @ Bl @ J22 @ ULL
    M[5] = M[5] @ Bl @ J22 @ ULL
    M[6] = M[6] + DLL @ Bl @ J21 @ M[0]
    M[7] = M[7] + DLL @ Bl @ J21 @ M[1]
    M[0] = UUR @ Bu @ J11 @ M[0]
    M[1] = UUR @ Bu @ J11 @ M[1]


def pdiv(diag, upper, lower, P):
    """Selected inversion by PDIV over P (a power of two) partitions.

    Returns ``(G_diag, G_upper, G_lower)``."""
    n, b = diag.shape[0], diag.shape[1]
    check(n, P)
    dtype = np.result_type(diag, upper, lower)
    starts, sizes = divide(n, P)   # pdiv_utils.py:84-123 splits as psr_utils.py does
    parts, Bu, Bl = [], [], []
    for s, m in zip(starts, sizes):   # partition_subdomain, pdiv_utils.py:126-171
        A = np.zeros((m * b, m * b), dtype)
        for i in range(m):
            A[i * b:(i + 1) * b, i * b:(i + 1) * b] = diag[s + i]
            if i < m - 1:
                A[i * b:(i + 1) * b, (i + 1) * b:(i + 2) * b] = upper[s + i]
                A[(i + 1) * b:(i + 2) * b, i * b:(i + 1) * b] = lower[s + i]
        parts.append(Part(np.linalg.inv(A), b, dtype))   # invert_partition, :94-116
        if s + m < n:
            Bu.append(upper[s + m - 1])
            Bl.append(lower[s + m - 1])
    eye = np.identity(b, dtype=dtype)
    for step in range(1, int(math.log2(P)) + 1):   # :77-87, update_maps :188-252
        stride = 2 ** step
        snap = [[x.copy() for x in pt.M] for pt in parts]
        for start in range(0, P, stride):
            end = start + stride - 1
            mid = middle(start, end)
            pm, pn = parts[mid], parts[mid + 1]
            U = [pm.toprow(snap[mid], pm.last), pm.leftcol(snap[mid], pm.last),
                 pm.element(snap[mid], pm.last, pm.last),
                 pn.element(snap[mid + 1], 0, 0), pn.rightcol(snap[mid + 1], 0), pn.botrow(snap[mid + 1], 0)]
            J = np.zeros((2 * b, 2 * b), dtype)   # get_J, :373-410
            J[:b, :b] = eye
            J[:b, b:] = -U[3] @ Bl[mid]
            J[b:, :b] = -U[2] @ Bu[mid]
            J[b:, b:] = eye
            J = np.linalg.inv(J)
            for r in range(start, end + 1):
                pt = parts[r]
                if r < end:   # get_nextprocess_matrixmap, :413-470
                    keys = (2, 3, 6, 7) if r < mid else (0, 1, 4, 5)
                    for k in keys:
                        pt.Mip1[k] = snap[r + 1][k].copy()
                if r < mid:   # update_crossmap, :573-597
                    crossmap_upper(pt.M, pt.Mip1, pt.C, Bu[mid], J, b)
                elif r == mid:
                    crossmap_middle(pt.M, pt.Mip1, pt.C, Bu[mid], Bl[mid], J, b)
                elif r < end:
                    crossmap_lower(pt.M, pt.Mip1, pt.C, Bl[mid], J, b)
                if r <= mid:  # update_matrixmap, :747-777
                    matrixmap_upper(pt.M, U, Bu[mid], Bl[mid], J, b)
                else:
                    matrixmap_lower(pt.M, U, Bu[mid], Bl[mid], J, b)
    Gd = np.zeros((n, b, b), dtype)
    Gu = np.zeros((max(n - 1, 0), b, b), dtype)
    Gl = np.zeros((max(n - 1, 0), b, b), dtype)
    for p, (s, m) in enumerate(zip(starts, sizes)):   # produce_partition, :903-1000
        pt = parts[p]
        for i in range(m):
            Gd[s + i] = pt.element(pt.M, i, i)
            if i < m - 1:
                Gu[s + i] = pt.element(pt.M, i, i + 1)
                Gl[s + i] = pt.element(pt.M, i + 1, i)
        if p < P - 1:   # produce_bridges / produce_upper_bridge / produce_lower_bridge, :1297-1436
            q = parts[p + 1]
            N, C = pt.last, pt.C
            p1_N1, p1_NN, p1_1N = pt.blk(N, 0), pt.blk(N, N), pt.blk(0, N)
            p2_11, p2_N1, p2_1N = q.blk(0, 0), q.blk(q.last, 0), q.blk(0, q.last)
            Gu[s + m - 1] = p1_N1 @ C[0] @ p2_11 + p1_N1 @ C[1] @ p2_N1 + p1_NN @ C[2] @ p2_11 + p1_NN @ C[3] @ p2_N1
            Gl[s + m - 1] = p2_11 @ C[4] @ p1_1N + p2_11 @ C[5] @ p1_NN + p2_1N @ C[6] @ p1_1N + p2_1N @ C[7] @ p1_NN
    return Gd, Gu, Gl
