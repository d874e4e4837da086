"""GPU parity of the PDIV (pairwise) selected inversion, all partitions in one
schedule (``sinvb_pdiv_z`` / ``_d``).

Reference: ``src/sinv/algorithms/pdiv/pdiv_localmap.py:27-1436``.  Checked
against the reference's own outputs (``tests/golden/pdiv_outputs.npz``, the
reference ``pdiv_localmap`` run on 2, 4 and 8 processes), the oracle
restatement (``oracle/pdiv_oracle.py``) and the dense inverse.  Tolerances:

  * the reference test's ``np.allclose`` against the dense inverse
    (``tests/pdiv_tests/pdiv_test.py:134-136``), and within 10x the
    reference's own distance to the dense inverse plus 1e-10 (the partition
    blocks come from pivot-free RGF sweeps, about 1e-13 from exact on these
    matrices, where the reference inverts each partition with LAPACK);
  * <= 1e-12 on diagonally dominant matrices;
  * in-band tight-binding matrices: the map stage amplifies the partition
    blocks' rounding about a thousandfold, so the bound is the larger of 10x
    the oracle's distance to the dense inverse and 1e-9.
"""

import os

import numpy as np
import pytest

from oracle import dense, pdiv_oracle, rgf_oracle
from sinv_b200 import workloads
from sinv_b200.algorithms import pdiv_lm, pdiv_u
from sinv_b200.utils import matu
from tests.golden.make_golden import PDIV_SIZES, PDIV_VARIANTS, banded_case

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _worst(G, R):
    return max([dense.rel_fro(np.asarray(g), r) for g, r in zip(G, R) if np.asarray(r).size] or [0.0])


@pytest.fixture(scope="module")
def pdiv_golden():
    return np.load(os.path.join(HERE, "golden", "pdiv_outputs.npz"))


CASES = [(c, s, N, b, P) for c, s in PDIV_VARIANTS for N, b in PDIV_SIZES for P in (2, 4, 8) if N // b >= P]


@pytest.mark.parametrize("cplx,sym,N,b,P", CASES)
def test_reference_test_matrices(pdiv_golden, cplx, sym, N, b, P):
    A, (d, u, l) = banded_case(N, b, cplx, sym)
    G = pdiv_lm.pdiv(A, b, P)
    gd, gu, gl = matu.convertDenseToBlkTridiag(G, b)
    R = dense.inv_selected(d, u, l)
    assert all(np.allclose(g, r) for g, r in zip((gd, gu, gl), R))   # pdiv_test.py:134-136
    key = f"pdiv_c{int(cplx)}_s{int(sym)}_N{N}_b{b}_P{P}"
    ref = [pdiv_golden[key + s] for s in ("_d", "_u", "_l")]
    assert _worst((gd, gu, gl), R) <= 10 * _worst(ref, R) + 1e-10


@pytest.mark.parametrize("cplx,sym,N,b,P", [c for c in CASES if c[2] == 128])
def test_per_process_outputs(pdiv_golden, cplx, sym, N, b, P):
    """pdiv_localmap_all gives what pdiv_localmap returns on every process."""
    A, _ = banded_case(N, b, cplx, sym)
    starts, sizes = pdiv_u.divide_matrix(A, P, b)
    K_i, Bu_i, Bl_i = pdiv_u.partition_subdomain(A, starts, sizes, b)
    out = pdiv_lm.pdiv_localmap_all(K_i, Bu_i, Bl_i, b)
    key = f"pdiv_c{int(cplx)}_s{int(sym)}_N{N}_b{b}_P{P}"
    rd, ru, rl = (pdiv_golden[key + s] for s in ("_d", "_u", "_l"))
    n = N // b
    for p, ((Xd, Xu, Xl), s, m) in enumerate(zip(out, starts, sizes)):
        assert Xd.shape == Xu.shape == Xl.shape == (m, b, b)
        assert np.allclose(Xd, rd[s:s + m])
        e = min(s + m, n - 1)
        assert np.allclose(Xu[:e - s], ru[s:e]) and np.allclose(Xl[:e - s], rl[s:e])
        if p == P - 1:
            assert not Xu[-1].any() and not Xl[-1].any()   # pdiv_test.py:127-129


@pytest.mark.parametrize("n,b,P", [(16, 12, 1), (16, 12, 2), (16, 12, 4), (16, 12, 8), (16, 12, 16), (17, 12, 4),
                                   (23, 32, 8), (12, 64, 4), (10, 96, 2), (8, 160, 4)])
def test_dominant(n, b, P):
    d, u, l = workloads.dominant(n, b, seed=P)
    G = pdiv_lm.pdiv_blocks(d, u, l, partitions=P)
    assert _worst(G, rgf_oracle.rgf(d, u, l)) <= 1e-12
    assert _worst(G, pdiv_oracle.pdiv(d, u, l, P)) <= 1e-12


def test_dominant_reference_outputs(pdiv_golden):
    d, u, l = workloads.dominant(16, 12, seed=0)
    for P in (2, 4, 8, 16):
        G = pdiv_lm.pdiv_blocks(d, u, l, partitions=P)
        ref = [pdiv_golden[f"dom_pdiv_P{P}" + s] for s in ("_d", "_u", "_l")]
        assert _worst(G, ref) <= 1e-12


@pytest.mark.parametrize("E", [0.4, -1.2])
@pytest.mark.parametrize("n,b,P", [(64, 32, 2), (64, 32, 8), (16, 128, 4)])
def test_tight_binding(E, n, b, P):
    d, u, l = workloads.tight_binding(n, b, E, seed=11)
    G = pdiv_lm.pdiv_blocks(d, u, l, partitions=P)
    R = dense.inv_selected(d, u, l)
    eo = _worst(pdiv_oracle.pdiv(d, u, l, P), R)
    assert _worst(G, R) <= max(10 * eo, 1e-9)


def test_large_blocks_on_the_device():
    """n = 64, b = 256 (the plain-at-scale matrix), torch tensors in and out."""
    import torch
    d, u, l = workloads.dominant(64, 256, seed=0)
    R = rgf_oracle.rgf(d, u, l)
    td, tu, tl = (torch.from_numpy(x).cuda() for x in (d, u, l))
    for P in (4, 8):
        G = pdiv_lm.pdiv_blocks(td, tu, tl, partitions=P)
        assert all(torch.is_tensor(g) and g.is_cuda for g in G)
        assert _worst([g.cpu().numpy() for g in G], R) <= 1e-12


def test_real_and_single_precision():
    d, u, l = workloads.dominant(16, 24, seed=3)
    dr, ur, lr = (x.real.copy() for x in (d, u, l))
    assert _worst(pdiv_lm.pdiv_blocks(dr, ur, lr, partitions=4), dense.inv_selected(dr, ur, lr)) <= 1e-12
    ds, us, ls = (x.astype(np.complex64) for x in (d, u, l))
    G = pdiv_lm.pdiv_blocks(ds, us, ls, partitions=4)
    assert G[0].dtype == np.complex64
    assert _worst(G, dense.inv_selected(d, u, l)) <= 1e-6


def test_limits_and_singular_block():
    d, u, l = workloads.dominant(12, 4, seed=1)
    with pytest.raises(ValueError, match="power of 2"):
        pdiv_lm.pdiv_blocks(d, u, l, partitions=3)
    with pytest.raises(ValueError, match="greater than the number of processes"):
        pdiv_lm.pdiv_blocks(d[:2], u[:1], l[:1], partitions=4)
    A = matu.convertBlkTridiagToDense(d, u, l)
    with pytest.raises(ValueError, match="multiple of the blocksize"):
        pdiv_lm.pdiv(A, 5, 2)
    d = d.copy()
    d[0] = 0.0                                   # the first partition inverts A_00 first
    with pytest.raises(np.linalg.LinAlgError):
        pdiv_lm.pdiv_blocks(d, u, l, partitions=2)
