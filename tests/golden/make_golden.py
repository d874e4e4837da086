"""Generate golden fixtures from the reference implementation itself.

Run from the repository root, with the reference sources available::

    python tests/golden/make_golden.py /path/to/reference         # rgf, bcr
    python tests/golden/make_golden.py /path/to/reference --psr   # psr_outputs.npz
    python tests/golden/make_golden.py /path/to/reference --pdiv  # pdiv_outputs.npz

The reference root may also come from the ``SINV_REFERENCE`` environment
variable; there is no default.

``psr_seqsolve`` (``src/sinv/algorithms/psr/psr_seqsolve.py:20-73``) needs at
least three MPI processes; it runs here on P threads that exchange its
``send`` / ``recv`` messages through queues (``ThreadComm``), each thread on
its own copy of the matrix as each MPI process has.  ``pdiv_localmap``
(``src/sinv/algorithms/pdiv/pdiv_localmap.py:27-91``, power-of-two process
counts) runs the same way, each thread given its partition and the bridges.

The reference ``rgf`` (``src/sinv/algorithms/rgf/rgf.py:17-64``) and
``bcr_serial`` (``src/sinv/algorithms/bcr/bcr_serial.py:19-62``) are imported
from the reference's ``src/`` with two import shims:

* ``mpi4py`` is absent; ``bcr_utils.py:13`` imports it at module level but
  the serial path never calls it, so an empty module stands in.
* ``quasi.bsparse`` (the un-vendored container ``rgf.py:13`` imports) is
  replaced by a block-tridiagonal container with the members ``rgf`` uses:
  ``.copy()``, scalar ``*``, ``.blocks[i, j]`` get/set and ``.blockorder``.

Inputs are regenerated by the tests from seeds (the reference tests'
``SEED = 63`` banded generator, ``tests/bcr_tests/bcr_serial_test.py:15,63``,
and the seeded dominant generator); the fixtures hold the reference outputs
and a checksum of each input so generator drift is caught.
"""

import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from sinv_b200.utils import matu  # noqa: E402
from sinv_b200 import workloads  # noqa: E402

# Size lists of the reference tests (tests/rgf_tests/rgf_test.py:46-58,
# tests/bcr_tests/bcr_serial_test.py:42-52): (matrix size, block size).
RGF_SIZES = [(1, 1), (2, 2), (3, 3), (2, 1), (4, 2), (6, 3), (3, 1), (6, 2), (9, 3),
             (128, 8), (128, 16), (128, 32)]
BCR_SIZES = [(9, 1), (18, 2), (27, 3), (12, 1), (24, 2), (36, 3), (256, 8), (240, 10),
             (144, 12)]
SEED = 63
# (is_complex, is_symmetric) combinations stored per algorithm
RGF_VARIANTS = [(True, False), (False, True)]
BCR_VARIANTS = [(True, True), (False, False)]


class BlockTridiag:
    """Duck-typed stand-in for ``quasi.bsparse`` with the members rgf uses."""

    def __init__(self, d, u, l):
        self.d, self.u, self.l = d, u, l
        self.blockorder = d.shape[0]
        self.blocks = self

    def copy(self):
        return BlockTridiag(self.d.copy(), self.u.copy(), self.l.copy())

    def __mul__(self, x):
        return BlockTridiag(self.d * x, self.u * x, self.l * x)

    def _where(self, i, j):
        if i == j:
            return self.d, i
        if j == i + 1:
            return self.u, i
        if i == j + 1:
            return self.l, j
        raise KeyError((i, j))

    def __getitem__(self, ij):
        a, k = self._where(*ij)
        return a[k]

    def __setitem__(self, ij, v):
        a, k = self._where(*ij)
        a[k] = v


def import_reference(ref_root):
    sys.path.insert(0, os.path.join(ref_root, "src"))
    sys.modules["mpi4py"] = types.ModuleType("mpi4py")
    sys.modules["mpi4py"].MPI = types.SimpleNamespace()
    for name in ["quasi", "quasi.bsparse", "quasi.bsparse._base"]:
        sys.modules[name] = types.ModuleType(name)
    sys.modules["quasi.bsparse._base"].bsparse = BlockTridiag
    from sinv.algorithms.rgf import rgf as rgf_mod
    from sinv.algorithms.bcr import bcr_serial as bcr_mod
    return rgf_mod, bcr_mod


def checksum(*arrs):
    return np.array([complex(np.sum(a)) for a in arrs], dtype=np.complex128)


def banded_case(N, b, cplx, sym):
    A = matu.generateBandedDiagonalMatrix(N, np.ceil(b / 2), cplx, sym, SEED)
    return A, matu.convertDenseToBlkTridiag(A, b)


def main(ref_root):
    rgf_mod, bcr_mod = import_reference(ref_root)
    out = {}
    for cplx, sym in RGF_VARIANTS:
        for N, b in RGF_SIZES:
            A, (d, u, l) = banded_case(N, b, cplx, sym)
            G = rgf_mod.rgf(BlockTridiag(d.copy(), u.copy(), l.copy()), sym)
            key = f"rgf_c{int(cplx)}_s{int(sym)}_N{N}_b{b}"
            out[key + "_in"] = checksum(d, u, l)
            out[key + "_d"], out[key + "_u"], out[key + "_l"] = G.d, G.u, G.l
    for cplx, sym in BCR_VARIANTS:
        for N, b in BCR_SIZES:
            A, _ = banded_case(N, b, cplx, sym)
            Gd = bcr_mod.bcr_serial(A.copy(), b)
            gd, gu, gl = matu.convertDenseToBlkTridiag(Gd, b)
            key = f"bcr_c{int(cplx)}_s{int(sym)}_N{N}_b{b}"
            out[key + "_in"] = checksum(A)
            out[key + "_d"], out[key + "_u"], out[key + "_l"] = gd, gu, gl
    # dominant n=10, b=32 complex128, seed 0: rgf in both flag settings, bcr diag
    d, u, l = workloads.dominant(10, 32, seed=0)
    out["dom_in"] = checksum(d, u, l)
    G = rgf_mod.rgf(BlockTridiag(d.copy(), u.copy(), l.copy()))
    out["dom_rgf_d"], out["dom_rgf_u"], out["dom_rgf_l"] = G.d, G.u, G.l
    G = rgf_mod.rgf(BlockTridiag(d.copy(), u.copy(), l.copy()), False, False)
    out["dom_rgf_nooff_d"] = G.d
    out["dom_rgf_nooff_u_isnan"] = np.array(bool(np.all(np.isnan(G.u))))
    Ad = matu.convertBlkTridiagToDense(d, u, l)
    Gd = bcr_mod.bcr_serial(Ad.copy(), 32)
    out["dom_bcr_d"] = matu.convertDenseToBlkTridiag(Gd, 32)[0]
    # a few stride-2^l blocks of the production tree, outside the tridiagonal
    out["dom_bcr_g_0_3"] = Gd[0:32, 96:128]
    out["dom_bcr_g_7_3"] = Gd[224:256, 96:128]
    path = os.path.join(HERE, "reference_outputs.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes,", len(out), "arrays")


# PSR fixtures: the reference test's sizes (tests/psr_tests/psr_test.py:42-52)
# on 3 and 4 partitions where every partition gets 3 block rows.
PSR_SIZES = BCR_SIZES
PSR_VARIANTS = [(True, False), (False, True)]


class ThreadComm:
    """Point-to-point stand-in for ``MPI.COMM_WORLD`` over P threads: ``send`` /
    ``recv`` through one FIFO queue per (source, dest, tag), which is MPI's
    matching rule for blocking point-to-point messages; the rank comes from a
    thread-local."""

    def __init__(self, size):
        import threading
        self.size = size
        self.local = threading.local()
        self.lock = threading.Lock()
        self.q = {}

    def _queue(self, key):
        import queue
        with self.lock:
            return self.q.setdefault(key, queue.Queue())

    def Get_rank(self):
        return self.local.rank

    def Get_size(self):
        return self.size

    def send(self, obj, dest, tag=0):
        self._queue((self.local.rank, dest, tag)).put(np.array(obj, copy=True))

    def recv(self, source, tag=0):
        return self._queue((source, self.local.rank, tag)).get(timeout=600)


def run_psr_reference(psr_mod, A, b, P):
    """The reference ``psr_seqsolve`` (``psr_seqsolve.py:20-73``) on P threads;
    returns rank 0's G (the aggregated result)."""
    import threading
    comm = ThreadComm(P)
    psr_mod.MPI.COMM_WORLD = comm
    out, errs = {}, []

    def rank(r):
        comm.local.rank = r
        try:
            out[r] = psr_mod.psr_seqsolve(A.copy(), b)
        except Exception as e:  # surfaced below
            errs.append(e)

    ts = [threading.Thread(target=rank, args=(r,)) for r in range(P)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    if errs:
        raise errs[0]
    return out[0]


def main_psr(ref_root):
    import_reference(ref_root)  # the same mpi4py / quasi shims as main()
    from sinv.algorithms.psr import psr_seqsolve as psr_mod
    out = {}
    for cplx, sym in PSR_VARIANTS:
        for N, b in PSR_SIZES:
            for P in (3, 4):
                if N // b < 3 * P:
                    continue
                A, _ = banded_case(N, b, cplx, sym)
                G = run_psr_reference(psr_mod, A, b, P)
                gd, gu, gl = matu.convertDenseToBlkTridiag(G, b)
                key = f"psr_c{int(cplx)}_s{int(sym)}_N{N}_b{b}_P{P}"
                out[key + "_in"] = checksum(A)
                out[key + "_d"], out[key + "_u"], out[key + "_l"] = gd, gu, gl
    d, u, l = workloads.dominant(24, 16, seed=0)
    Ad = matu.convertBlkTridiagToDense(d, u, l)
    out["dom_psr_in"] = checksum(d, u, l)
    for P in (3, 4, 8):
        G = run_psr_reference(psr_mod, Ad, 16, P)
        out[f"dom_psr_P{P}_d"], out[f"dom_psr_P{P}_u"], out[f"dom_psr_P{P}_l"] = \
            matu.convertDenseToBlkTridiag(G, 16)
    path = os.path.join(HERE, "psr_outputs.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes,", len(out), "arrays")


# PDIV fixtures: the reference test's sizes (tests/pdiv_tests/pdiv_test.py:45-56)
# on 2, 4 and 8 processes (powers of two, at most one per block).
PDIV_SIZES = [(2, 1), (4, 2), (6, 3), (3, 1), (6, 2), (9, 3), (128, 8), (128, 16), (128, 32)]
PDIV_VARIANTS = [(True, False), (False, True)]


def run_pdiv_reference(pdiv_mod, pdiv_u, A, b, P):
    """The reference ``pdiv_localmap`` (``pdiv_localmap.py:27-91``) on P threads,
    each given its partition and the bridges as ``tests/pdiv_tests/pdiv_test.py:84-88``
    does; returns the assembled (G_diag, G_upper, G_lower)."""
    import threading
    comm = ThreadComm(P)
    pdiv_mod.MPI.COMM_WORLD = comm
    starts, sizes = pdiv_u.divide_matrix(A, P, b)
    K_i, Bu_i, Bl_i = pdiv_u.partition_subdomain(A, starts, sizes, b)
    out, errs = {}, []

    def rank(r):
        comm.local.rank = r
        try:
            out[r] = pdiv_mod.pdiv_localmap(K_i[r].copy(), Bu_i, Bl_i, b)
        except Exception as e:  # surfaced below
            errs.append(e)

    ts = [threading.Thread(target=rank, args=(r,)) for r in range(P)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    if errs:
        raise errs[0]
    n = A.shape[0] // b
    Gd = np.zeros((n, b, b), A.dtype)
    Gu = np.zeros((n - 1, b, b), A.dtype)
    Gl = np.zeros((n - 1, b, b), A.dtype)
    for r in range(P):
        X_d, X_u, X_l = out[r]
        for i in range(sizes[r]):
            Gd[starts[r] + i] = X_d[i]
            if starts[r] + i < n - 1:
                Gu[starts[r] + i] = X_u[i]
                Gl[starts[r] + i] = X_l[i]
    return Gd, Gu, Gl


def main_pdiv(ref_root):
    import_reference(ref_root)  # the same mpi4py / quasi shims as main()
    from sinv.algorithms.pdiv import pdiv_localmap as pdiv_mod
    from sinv.algorithms.pdiv import pdiv_utils as pdiv_u
    pdiv_u.MPI.COMM_WORLD = None
    out = {}
    for cplx, sym in PDIV_VARIANTS:
        for N, b in PDIV_SIZES:
            for P in (2, 4, 8):
                if N // b < P:
                    continue
                A, _ = banded_case(N, b, cplx, sym)
                G = run_pdiv_reference(pdiv_mod, pdiv_u, A, b, P)
                key = f"pdiv_c{int(cplx)}_s{int(sym)}_N{N}_b{b}_P{P}"
                out[key + "_in"] = checksum(A)
                out[key + "_d"], out[key + "_u"], out[key + "_l"] = G
    d, u, l = workloads.dominant(16, 12, seed=0)
    Ad = matu.convertBlkTridiagToDense(d, u, l)
    out["dom_pdiv_in"] = checksum(d, u, l)
    for P in (2, 4, 8, 16):
        out[f"dom_pdiv_P{P}_d"], out[f"dom_pdiv_P{P}_u"], out[f"dom_pdiv_P{P}_l"] = \
            run_pdiv_reference(pdiv_mod, pdiv_u, Ad, 12, P)
    path = os.path.join(HERE, "pdiv_outputs.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes,", len(out), "arrays")


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    root = args[0] if args else os.environ.get("SINV_REFERENCE")
    if not root:
        sys.exit("usage: make_golden.py REFERENCE_ROOT [--psr|--pdiv] (or set SINV_REFERENCE)")
    if "--psr" in sys.argv:
        main_psr(root)
    elif "--pdiv" in sys.argv:
        main_pdiv(root)
    else:
        main(root)
