"""Generate golden fixtures from the reference implementation itself.

Run from the repository root, with the reference sources available::

    python tests/golden/make_golden.py /path/to/reference

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


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
