"""The batched adjoint (one persistent launch per direction over many
instances) against the single-instance adjoint and against torch autograd
through the dense FP64 inverse.

Tolerances: 1e-10 relative against the single-instance adjoint (same
recursion, different tile shapes and teams), 1e-9 against dense autograd
(as the single-instance tests)."""

import numpy as np
import pytest
import torch

from sinv_b200 import workloads
from sinv_b200.algorithms import rgf_autograd, rgf_batched_autograd
from tests.test_adjoint_gpu import dense_selected, loss_fn

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return (torch.linalg.norm(a - b) / torch.linalg.norm(b)).item()


def _weights(shapes, seed):
    rng = np.random.default_rng(seed)
    out = []
    for n, b in shapes:
        out.append([torch.from_numpy(rng.standard_normal(s) + 1j * rng.standard_normal(s)).cuda()
                    for s in ((n, b, b), (n - 1, b, b), (n - 1, b, b))])
    return out


@pytest.mark.parametrize("sym", [False, True])
def test_batched_adjoint_matches_single_and_dense(sym):
    shapes = [(5, 8), (1, 16), (7, 33), (4, 64), (3, 130), (10, 16), (2, 256)]
    inst = []
    for k, (n, b) in enumerate(shapes):
        d, u, l = workloads.tight_binding(n, b, 0.2 + 0.1 * k, seed=1300 + k)
        if sym:
            l = np.ascontiguousarray(np.transpose(u, (0, 2, 1)))
        inst.append(tuple(torch.from_numpy(x).cuda() for x in (d, u, l)))
    W = _weights(shapes, 5)
    leaves = [tuple(x.clone().requires_grad_(True) for x in t) for t in inst]
    outs = rgf_batched_autograd(leaves, sym_mat=sym)
    loss = sum(loss_fn(*G, *w) for G, w in zip(outs, W))
    loss.backward()
    for k, (t, w) in enumerate(zip(inst, W)):
        single = [x.clone().requires_grad_(True) for x in t]
        loss_fn(*rgf_autograd(*single, sym_mat=sym), *w).backward()
        for a, r in zip(leaves[k], single):
            if r.numel():
                assert _rel(a.grad, r.grad) <= 1e-10, (k, _rel(a.grad, r.grad))
        # with sym_mat, G_upper := G_lower^T is a different function of A off the
        # symmetric matrices, so its gradient is compared with the single adjoint only
        if not sym and shapes[k][0] * shapes[k][1] <= 1024:
            dense = [x.clone().requires_grad_(True) for x in t]
            loss_fn(*dense_selected(*dense), *w).backward()
            for a, r in zip(leaves[k], dense):
                if r.numel():
                    assert _rel(a.grad, r.grad) <= 1e-9, (k, _rel(a.grad, r.grad))


def test_batched_energy_gradient_at_the_differentiated_size():
    """n = 32, b = 128 (the differentiated workload's size), 6 energies of its
    generator: the batched density-of-states gradient against dense autograd."""
    from sinv_b200 import distributed
    from tests.test_config_sizes_gpu import _dense_selected, _dos_gradient
    energies, n, b, hseed = workloads.gradient_set_spec()
    energies = energies[:6]
    onsite, coupling = workloads.hamiltonian(n, b, hseed)
    Hd = torch.from_numpy(onsite).cuda()
    Hu = torch.from_numpy(coupling).cuda()
    loss, g_on, g_cp = distributed.energy_loss_and_grad(Hd, Hu, energies)
    ref = _dos_gradient(_dense_selected, Hd, Hu, energies, torch.complex128)
    for a, r in zip((g_on, g_cp), ref):
        assert _rel(a, r) <= 1e-9, _rel(a, r)
