"""GPU parity of the BCR selected inversion against the reference outputs.

Fixtures: the reference ``bcr_serial`` (``src/sinv/algorithms/bcr/bcr_serial.py:19-62``)
on the reference test's matrices (``tests/bcr_tests/bcr_serial_test.py``,
SEED=63 banded generator) and on the seeded dominant matrix.  Tolerances as
for RGF: <= 1e-12 relative Frobenius on dominant matrices; on the random
banded test matrices the reference test's own ``np.allclose`` bar plus 1e-9
relative to the reference output.
"""

import numpy as np
import pytest

from oracle import bcr_oracle, dense, rgf_oracle
from sinv_b200 import workloads
from sinv_b200.algorithms import bcr_s
from sinv_b200.utils import matu
from tests.golden.make_golden import BCR_SIZES, BCR_VARIANTS, banded_case

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return dense.rel_fro(a, b)


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("sym", [False, True])
@pytest.mark.parametrize("N,b", BCR_SIZES)
def test_reference_test_matrices(golden, cplx, sym, N, b):
    A, _ = banded_case(N, b, cplx, sym)
    G = bcr_s.bcr_serial(A, b)                       # bcr_serial_test.py:65
    gd, gu, gl = matu.convertDenseToBlkTridiag(G, b)
    rd, ru, rl = matu.convertDenseToBlkTridiag(np.linalg.inv(A), b)
    assert np.allclose(gd, rd) and np.allclose(gu, ru) and np.allclose(gl, rl)   # :70-73
    key = f"bcr_c{int(cplx)}_s{int(sym)}_N{N}_b{b}"
    ref = (golden[key + "_d"], golden[key + "_u"], golden[key + "_l"]) if key + "_d" in golden else \
        matu.convertDenseToBlkTridiag(bcr_oracle.bcr_serial(A, b), b)
    for g, r in zip((gd, gu, gl), ref):
        assert _rel(g, r) <= 1e-9


def test_dominant_n10_b32_matches_reference(golden):
    d, u, l = workloads.dominant(10, 32, seed=0)
    Gd, Gu, Gl = bcr_s.bcr_blocks(d, u, l)
    assert _rel(Gd, golden["dom_bcr_d"]) <= 1e-12
    R = dense.inv_selected(d, u, l)
    for g, r in zip((Gd, Gu, Gl), R):
        assert _rel(g, r) <= 1e-12


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 7, 8, 9, 16, 17])
@pytest.mark.parametrize("b", [1, 3, 32, 65])
@pytest.mark.parametrize("dtype", [np.complex128, np.float64])
def test_block_counts_and_sizes(n, b, dtype):
    d, u, l = workloads.dominant(n, b, seed=n * 31 + b, dtype=dtype)
    G = bcr_s.bcr_blocks(d, u, l)
    R = bcr_oracle.bcr_blocks(d, u, l)[:3]
    for g, r in zip(G, R):
        if r.size:
            assert _rel(g, r) <= 1e-12


@pytest.mark.parametrize("n,b", [(6, 130), (12, 128), (33, 64)])
def test_bcr_on_tight_binding(n, b):
    """BCR inverts the undamped diagonal blocks (condition ~1e3 here); the
    reference's own bcr_serial lands ~1e-11 from the dense inverse on these."""
    d, u, l = workloads.tight_binding(n, b, 0.3, seed=n)
    G = bcr_s.bcr_blocks(d, u, l)
    D = dense.inv_selected(d, u, l)
    R = rgf_oracle.rgf(d, u, l)
    for g, x, r in zip(G, D, R):
        assert _rel(g, x) <= 1e-10
        assert _rel(g, r) <= 1e-10


def test_dense_torch_input_and_single_precision():
    import torch
    d, u, l = workloads.dominant(5, 8, seed=3)
    A = matu.convertBlkTridiagToDense(d, u, l)
    G = bcr_s.bcr_serial(torch.from_numpy(A).cuda(), 8)
    assert G.is_cuda
    ref = np.zeros_like(A)
    rd, ru, rl = dense.inv_selected(d, u, l)
    Gd, Gu, Gl = matu.convertDenseToBlkTridiag(G.cpu().numpy(), 8)
    assert _rel(Gd, rd) <= 1e-12 and _rel(Gu, ru) <= 1e-12 and _rel(Gl, rl) <= 1e-12
    G32 = bcr_s.bcr_serial(A.astype(np.complex64), 8)
    assert G32.dtype == np.complex64
    assert _rel(matu.convertDenseToBlkTridiag(G32, 8)[0], rd) <= 1e-5
    del ref
