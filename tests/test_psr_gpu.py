"""GPU parity of the PSR selected inversion (partitions as teams of one launch).

Reference: ``src/sinv/algorithms/psr/psr_seqsolve.py:20-943``.  Checked
against the reference's own outputs (``tests/golden/psr_outputs.npz``, made by
running the reference ``psr_seqsolve`` on 3 and 4 partitions), the oracle
restatement (``oracle/psr_oracle.py``) and the dense inverse.  Tolerances:

  * the reference test's ``np.allclose`` against the dense inverse
    (``tests/psr_tests/psr_test.py:67-70``) plus <= 1e-9 relative Frobenius
    against the reference output on its banded test matrices;
  * <= 1e-12 on diagonally dominant matrices;
  * tight-binding matrices: PSR inverts undamped diagonal blocks, so its
    rounding grows with their condition as the reference's does; the bound is
    10x the oracle PSR's own distance to the dense inverse plus 1e-11.
"""

import os

import numpy as np
import pytest

from oracle import dense, psr_oracle, rgf_oracle
from sinv_b200 import workloads
from sinv_b200.algorithms import psr_s
from sinv_b200.utils import matu
from tests.golden.make_golden import PSR_SIZES, PSR_VARIANTS, banded_case

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _worst(G, R):
    return max([dense.rel_fro(np.asarray(g), r) for g, r in zip(G, R) if np.asarray(r).size] or [0.0])


@pytest.fixture(scope="module")
def psr_golden():
    return np.load(os.path.join(HERE, "golden", "psr_outputs.npz"))


CASES = [(c, s, N, b, P) for c, s in PSR_VARIANTS for N, b in PSR_SIZES for P in (3, 4) if N // b >= 3 * P]


@pytest.mark.parametrize("cplx,sym,N,b,P", CASES)
def test_reference_test_matrices(psr_golden, cplx, sym, N, b, P):
    A, _ = banded_case(N, b, cplx, sym)
    G = psr_s.psr_seqsolve(A, b, partitions=P)                       # psr_test.py:65
    gd, gu, gl = matu.convertDenseToBlkTridiag(G, b)
    rd, ru, rl = matu.convertDenseToBlkTridiag(np.linalg.inv(A), b)
    assert np.allclose(gd, rd) and np.allclose(gu, ru) and np.allclose(gl, rl)   # :67-70
    key = f"psr_c{int(cplx)}_s{int(sym)}_N{N}_b{b}_P{P}"
    for g, s in zip((gd, gu, gl), ("_d", "_u", "_l")):
        assert dense.rel_fro(g, psr_golden[key + s]) <= 1e-9


@pytest.mark.parametrize("P", [3, 4, 8])
def test_dominant_matches_reference(psr_golden, P):
    d, u, l = workloads.dominant(24, 16, seed=0)
    G = psr_s.psr_blocks(d, u, l, partitions=P)
    for g, s in zip(G, ("_d", "_u", "_l")):
        assert dense.rel_fro(g, psr_golden[f"dom_psr_P{P}" + s]) <= 1e-12


@pytest.mark.parametrize("n,P", [(9, 3), (10, 3), (13, 4), (24, 8), (40, 5), (96, 32), (64, None)])
@pytest.mark.parametrize("b", [1, 3, 32, 65, 130])
@pytest.mark.parametrize("dtype", [np.complex128, np.float64])
def test_partitions_and_block_sizes(n, P, b, dtype):
    if n * b * b > 64 * 130 * 130:
        pytest.skip("kept small")
    d, u, l = workloads.dominant(n, b, seed=n * 7 + b, dtype=dtype)
    G = psr_s.psr_blocks(d, u, l, partitions=P)
    assert G[0].dtype == dtype
    Pn = psr_s.partitions_for(n, P)
    assert _worst(G, psr_oracle.psr(d, u, l, Pn)) <= 1e-12
    assert _worst(G, rgf_oracle.rgf(d, u, l)) <= 1e-12


@pytest.mark.parametrize("n,b,P", [(64, 256, None), (30, 64, 5), (48, 128, 4)])
def test_tight_binding(n, b, P):
    d, u, l = workloads.tight_binding(n, b, 0.3, seed=n + b)
    G = psr_s.psr_blocks(d, u, l, partitions=P)
    D = dense.inv_selected(d, u, l)
    ref = _worst(psr_oracle.psr(d, u, l, psr_s.partitions_for(n, P)), D)
    # measured: at most 2.8x the oracle PSR's own distance (one Newton step per block inverse)
    assert _worst(G, D) <= 4 * ref + 1e-11, (_worst(G, D), ref)


def test_torch_inputs_single_precision_and_dense_torch():
    import torch
    d, u, l = workloads.dominant(12, 24, seed=5)
    td, tu, tl = (torch.from_numpy(x).cuda() for x in (d, u, l))
    G = psr_s.psr_blocks(td, tu, tl, partitions=3)
    assert all(g.is_cuda for g in G)
    R = psr_oracle.psr(d, u, l, 3)
    assert _worst([g.cpu().numpy() for g in G], R) <= 1e-12
    G32 = psr_s.psr_blocks(d.astype(np.complex64), u.astype(np.complex64), l.astype(np.complex64), partitions=4)
    assert G32[0].dtype == np.complex64 and _worst(G32, R) <= 1e-5
    A = torch.from_numpy(matu.convertBlkTridiagToDense(d, u, l)).cuda()
    Gt = psr_s.psr_seqsolve(A, 24, partitions=3)
    assert Gt.is_cuda
    assert _worst(matu.convertDenseToBlkTridiag(Gt.cpu().numpy(), 24), R) <= 1e-12


@pytest.mark.parametrize("n,b,P,dtype", [(12, 8, 3, np.complex128), (24, 16, 4, np.complex128),
                                         (40, 64, 5, np.complex128), (30, 33, 3, np.float64),
                                         (64, 130, 6, np.complex128)])
def test_partitions_one_at_a_time_as_ranks(n, b, P, dtype):
    """The per-rank path of a multi-GPU PSR (``sinvb_psr_part_*``), its ranks run
    one after another on this GPU, each holding only its partition's rows:
    each partition reduces, the boundary slots are exchanged in-process (what
    the all-gather does across GPUs), the reduced system is solved, each
    partition produces its rows."""
    d, u, l = workloads.dominant(n, b, seed=3 * n + b, dtype=dtype)
    parts = [psr_s.PsrPart(*psr_s.local_blocks(d, u, l, P, k), n, P, k) for k in range(P)]
    slots = [p.reduce().clone() for p in parts]
    RG = parts[0].solve_reduced(*psr_s.reduced_system(slots, n, P))
    Gd, Gu, Gl = (np.zeros_like(x) for x in (d, u, l))
    for k, p in enumerate(parts):
        gs, link = psr_s.boundary_inverse(RG, k, P)
        G = [g.cpu().numpy() for g in p.produce(gs, link)]
        t, B = p.rows
        e = min(B + 1, n - 1)
        Gd[t:B + 1], Gu[t:e], Gl[t:e] = G[0], G[1], G[2]
    R = psr_oracle.psr(d, u, l, P)
    assert _worst([Gd, Gu, Gl], R) <= 1e-12
    assert _worst([Gd, Gu, Gl], rgf_oracle.rgf(d, u, l)) <= 1e-12


def test_limits_and_singular_block():
    d, u, l = workloads.dominant(8, 4, seed=1)
    with pytest.raises(ValueError):
        psr_s.psr_blocks(d, u, l)                # 8 < 3 * 3
    d, u, l = workloads.dominant(12, 4, seed=1)
    with pytest.raises(ValueError):
        psr_s.psr_blocks(d, u, l, partitions=2)  # fewer than 3 partitions
    with pytest.raises(ValueError):
        psr_s.psr_blocks(d, u, l, partitions=5)  # 12 < 3 * 5
    d = d.copy()
    d[0] = 0.0                                   # the first partition inverts A_00 first
    with pytest.raises(np.linalg.LinAlgError):
        psr_s.psr_blocks(d, u, l, partitions=3)
