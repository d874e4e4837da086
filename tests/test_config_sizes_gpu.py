"""Parity at the sizes the benchmark configurations run, not only at
oracle-friendly shrunken sizes.

* plain at scale (n = 64, b = 256, diagonally dominant, seed 0): rgf and bcr
  on the same block arrays against the oracle restatement of the reference
  rgf (``src/sinv/algorithms/rgf/rgf.py:17-64``) at 1e-12, the bar of the
  plain path;
* energy batch: one full-size tight-binding instance per block size
  (b = 64, 128, 256, 512, n >= 100, energies and Hamiltonian seeds of the
  batch's generator): batched FP64 against the oracle at 5e-11, the
  mixed-precision path at 1e-8.  At these sizes the oracle itself (LAPACK
  inverses with partial pivoting) lies 0.8e-12 (b = 64) and 2.0e-12
  (b = 128, n = 100) from the dense FP64 inverse; the pivot-free block
  inversions here land within about ten times that (1.6e-11 at b = 128);
* differentiated (n = 32, b = 128, one Hamiltonian, several energies): the
  density-of-states gradient by the adjoint against torch autograd through
  the dense FP64 inverse (N = 4096) at 1e-9 (complex128) and 1e-5
  (complex64);
* large blocks (the n = 4, b = 1024 sub-instance of the n = 256 workload):
  mixed at 1e-8 and FP64 at 1e-11 against the dense FP64 inverse.
"""

import numpy as np
import pytest
import torch

from oracle import dense, rgf_oracle
from sinv_b200 import workloads
from sinv_b200.algorithms import BatchPlan, bcr_s, rgf, rgf_autograd

pytestmark = pytest.mark.gpu


def _worst(G, R):
    return max(dense.rel_fro(np.asarray(x), np.asarray(r)) for x, r in zip(G, R) if np.asarray(r).size)


def _np(G):
    return [g.cpu().numpy() if torch.is_tensor(g) else g for g in G]


def test_plain_at_scale_rgf_and_bcr_match_oracle():
    n, b = 64, 256
    d, u, l = workloads.dominant(n, b, seed=0)
    R = rgf_oracle.rgf(d, u, l)
    td, tu, tl = (torch.from_numpy(x).cuda() for x in (d, u, l))
    assert _worst(_np(rgf.rgf_blocks(td, tu, tl)), R) <= 1e-12
    assert _worst(_np(bcr_s.bcr_blocks(td, tu, tl)), R) <= 1e-12


def _full_size_instance(b):
    """The first energy-batch instance of block size b, with n raised to >= 100."""
    for (e, n, bb, s) in workloads.energy_batch_spec():
        if bb == b:
            return workloads.tight_binding(max(n, 100), b, e, seed=s)
    raise AssertionError(b)


@pytest.mark.parametrize("b", [64, 128, 256, 512])
def test_energy_batch_full_size_instance(b):
    d, u, l = _full_size_instance(b)
    R = rgf_oracle.rgf(d, u, l)
    inst = [tuple(torch.from_numpy(x).cuda() for x in (d, u, l))]
    fp64 = BatchPlan(inst)
    fp64.run()
    fp64.check()
    err64 = _worst(_np(fp64.results()[0]), R)
    assert err64 <= 5e-11, err64
    mixed = BatchPlan(inst, precision="mixed")
    mixed.run()
    mixed.check()
    errm = _worst(_np(mixed.results()[0]), R)
    assert errm <= 1e-8, errm


def _dense_selected(d, u, l):
    n, b = d.shape[0], d.shape[1]
    A = torch.zeros((n * b, n * b), dtype=d.dtype, device=d.device)
    for i in range(n):
        A[i * b:(i + 1) * b, i * b:(i + 1) * b] = d[i]
        if i + 1 < n:
            A[i * b:(i + 1) * b, (i + 1) * b:(i + 2) * b] = u[i]
            A[(i + 1) * b:(i + 2) * b, i * b:(i + 1) * b] = l[i]
    G = torch.linalg.inv(A)
    Gd = torch.stack([G[i * b:(i + 1) * b, i * b:(i + 1) * b] for i in range(n)])
    Gu = torch.stack([G[i * b:(i + 1) * b, (i + 1) * b:(i + 2) * b] for i in range(n - 1)])
    Gl = torch.stack([G[(i + 1) * b:(i + 2) * b, i * b:(i + 1) * b] for i in range(n - 1)])
    return Gd, Gu, Gl


def _dos_gradient(fn, Hd, Hu, energies, dtype):
    """dL/dH of L = sum_k -Im Tr sum_i G_ii(E_k) / pi through `fn`."""
    hd = Hd.clone().requires_grad_(True)
    hu = Hu.clone().requires_grad_(True)
    b = Hd.shape[1]
    eye = torch.eye(b, dtype=dtype, device=Hd.device)
    loss = 0.0
    for E in energies:
        dd = (E + 1j * workloads.ETA) * eye - hd.to(dtype)
        edge = torch.zeros_like(dd)
        edge[0] = 1j * workloads.SIGMA_EDGE * eye
        edge[-1] = edge[-1] + 1j * workloads.SIGMA_EDGE * eye
        Gd, _, _ = fn(dd + edge, (-hu.to(dtype)).contiguous(), (-hu.transpose(1, 2).to(dtype)).contiguous())
        loss = loss - Gd.diagonal(0, 1, 2).imag.sum() / np.pi
    loss.backward()
    return hd.grad, hu.grad


@pytest.mark.parametrize("dtype,tol", [(torch.complex128, 1e-9), (torch.complex64, 1e-5)])
def test_differentiated_configuration_gradient(dtype, tol):
    energies, n, b, hseed = workloads.gradient_set_spec()
    energies = energies[:4]
    onsite, coupling = workloads.hamiltonian(n, b, hseed)
    Hd = torch.from_numpy(onsite).cuda()
    Hu = torch.from_numpy(coupling).cuda()
    if dtype == torch.complex64:
        Hd, Hu = Hd.float(), Hu.float()
    ours = _dos_gradient(rgf_autograd, Hd, Hu, energies, dtype)
    ref = _dos_gradient(_dense_selected, Hd.double(), Hu.double(), energies, torch.complex128)
    for a, r in zip(ours, ref):
        err = (torch.linalg.norm(a.double() - r) / torch.linalg.norm(r)).item()
        assert err <= tol, err


def test_large_block_sub_instance_against_dense_inverse():
    e, _, b, seed = workloads.large_mixed_spec(count=1)[0]
    d, u, l = workloads.tight_binding(4, b, e, seed=seed)
    inst = [tuple(torch.from_numpy(x).cuda() for x in (d, u, l))]
    ref = _np(_dense_selected(*inst[0]))
    fp64 = BatchPlan(inst)
    fp64.run()
    fp64.check()
    err64 = _worst(_np(fp64.results()[0]), ref)
    assert err64 <= 1e-11, err64
    mixed = BatchPlan(inst, precision="mixed")
    mixed.run()
    mixed.check()
    errm = _worst(_np(mixed.results()[0]), ref)
    assert errm <= 1e-8, errm
