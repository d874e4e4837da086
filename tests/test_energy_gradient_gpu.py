"""The energy-summed density-of-states gradient on the GPU (adjoint path)
against the dense formula dL/dH = -(1/pi) Im (G^2)^T summed over energies."""

import numpy as np
import pytest
import torch

from sinv_b200 import distributed, workloads
from tests.test_distributed import dense_term

pytestmark = pytest.mark.gpu


def test_energy_loss_and_grad_matches_dense():
    n, b = 5, 16
    H_on, H_cp = workloads.hamiltonian(n, b, seed=8)
    energies = [-1.2, -0.3, 0.5, 1.4]
    loss, g_on, g_cp = distributed.energy_loss_and_grad(torch.from_numpy(H_on).cuda(),
                                                        torch.from_numpy(H_cp).cuda(), energies)
    ref = [dense_term(H_on, H_cp, E) for E in energies]
    assert abs(loss.item() - sum(r[0] for r in ref)) <= 1e-9 * abs(sum(r[0] for r in ref))
    r_on = sum(r[1] for r in ref)
    r_cp = sum(r[2] for r in ref)
    assert np.linalg.norm(g_on.cpu().numpy() - r_on) <= 1e-8 * np.linalg.norm(r_on)
    assert np.linalg.norm(g_cp.cpu().numpy() - r_cp) <= 1e-8 * np.linalg.norm(r_cp)
