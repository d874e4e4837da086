"""Two-sided RGF (``rgf2s.rgf2sided``): both halves of the block chain on one
GPU, meeting in the middle.  Checked against the oracle restatement of the
reference rgf (``src/sinv/algorithms/rgf/rgf.py:17-64``; the reference's
``rgf2sided.py`` computes the same selected inverse) and the dense inverse.
Tolerances as for rgf: 1e-12 relative Frobenius on diagonally dominant
matrices, 1e-11 on tight-binding matrices.
"""

import numpy as np
import pytest

from oracle import dense, rgf_oracle
from sinv_b200 import workloads
from sinv_b200.algorithms import rgf2s

pytestmark = pytest.mark.gpu


def _worst(G, R):
    return max(dense.rel_fro(g, r) for g, r in zip(G, R) if r.size)


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 8, 17])
@pytest.mark.parametrize("b", [8, 33, 64, 130])
def test_matches_oracle(n, b):
    d, u, l = workloads.dominant(n, b, seed=10 * n + b)
    assert _worst(rgf2s.rgf2sided(d, u, l), rgf_oracle.rgf(d, u, l)) <= 1e-12


@pytest.mark.parametrize("dtype", [np.complex128, np.float64])
@pytest.mark.parametrize("sym", [False, True])
def test_flags_and_dtypes(dtype, sym):
    d, u, l = workloads.dominant(9, 40, seed=5, dtype=dtype)
    if sym:
        d = d + np.transpose(d, (0, 2, 1))
        l = np.ascontiguousarray(np.transpose(u, (0, 2, 1)))
    ref = rgf_oracle.rgf(d, u, l, sym_mat=sym)
    assert _worst(rgf2s.rgf2sided(d, u, l, sym_mat=sym), ref) <= 1e-12
    Gd, Gu, Gl = rgf2s.rgf2sided(d, u, l, sym_mat=sym, save_off_diag=False)
    assert dense.rel_fro(Gd, ref[0]) <= 1e-12
    assert np.all(np.isnan(Gu)) and np.all(np.isnan(Gl))


@pytest.mark.parametrize("n,b", [(9, 256), (64, 64), (6, 130)])
def test_tight_binding_vs_dense(n, b):
    d, u, l = workloads.tight_binding(n, b, 0.4, seed=n)
    assert _worst(rgf2s.rgf2sided(d, u, l), dense.inv_selected(d, u, l)) <= 1e-11


def test_torch_inputs_stay_on_device():
    import torch
    d, u, l = workloads.dominant(6, 32, seed=1)
    out = rgf2s.rgf2sided(*(torch.from_numpy(x).cuda() for x in (d, u, l)))
    assert all(t.is_cuda for t in out)
    assert _worst([t.cpu().numpy() for t in out], rgf_oracle.rgf(d, u, l)) <= 1e-12
