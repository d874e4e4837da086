"""The hand-written RGF adjoint against torch autograd through a dense FP64
inverse and against central finite differences.

Tolerances: 1e-9 relative to the dense-autograd gradient (both FP64; the
adjoint goes through the pivot-free block recursion and sqrt(n)
recomputation); finite differences with h = 1e-6 agree to 1e-6 relative.
"""

import numpy as np
import pytest
import torch

from sinv_b200 import workloads
from sinv_b200.algorithms import rgf_autograd

pytestmark = pytest.mark.gpu


def dense_selected(d, u, l):
    """Differentiable reference: blocks of torch.linalg.inv of the dense matrix."""
    n, b = d.shape[0], d.shape[1]
    rows = []
    for i in range(n):
        row = []
        for j in range(n):
            if i == j:
                row.append(d[i])
            elif j == i + 1:
                row.append(u[i])
            elif i == j + 1:
                row.append(l[j])
            else:
                row.append(torch.zeros((b, b), dtype=d.dtype, device=d.device))
        rows.append(torch.cat(row, 1))
    G = torch.linalg.inv(torch.cat(rows, 0))
    Gd = torch.stack([G[i * b:(i + 1) * b, i * b:(i + 1) * b] for i in range(n)])
    Gu = torch.stack([G[i * b:(i + 1) * b, (i + 1) * b:(i + 2) * b] for i in range(n - 1)]) if n > 1 else d[:0]
    Gl = torch.stack([G[(i + 1) * b:(i + 2) * b, i * b:(i + 1) * b] for i in range(n - 1)]) if n > 1 else d[:0]
    return Gd, Gu, Gl


def loss_fn(Gd, Gu, Gl, wd, wu, wl):
    """A loss touching every selected block (real for complex G)."""
    if Gd.is_complex():
        return (wd * Gd).real.sum() + (wu * Gu).imag.sum() - 0.5 * (wl * Gl).real.sum() - Gd.diagonal(0, 1, 2).imag.sum() / np.pi
    return (wd * Gd).sum() + (wu * Gu).sum() - 0.5 * (wl * Gl).sum()


def grads(fn, d, u, l, w):
    leaves = [x.clone().requires_grad_(True) for x in (d, u, l)]
    loss = loss_fn(*fn(*leaves), *w)
    loss.backward()
    return [x.grad if x.grad is not None else torch.zeros_like(x) for x in leaves], loss.item()


def rel(a, b):
    return (torch.linalg.norm(a - b) / torch.linalg.norm(b)).item()


@pytest.mark.parametrize("n,b,team", [(1, 4, None), (2, 3, None), (5, 8, None), (10, 16, None), (7, 33, None),
                                      (9, 70, "grid"), (4, 96, None), (17, 8, "grid")])
@pytest.mark.parametrize("dtype", [torch.complex128, torch.float64])
def test_adjoint_matches_dense_autograd(n, b, team, dtype):
    rng = np.random.default_rng(n * 100 + b)
    npdt = np.complex128 if dtype.is_complex else np.float64
    d, u, l = (torch.from_numpy(x).cuda() for x in workloads.dominant(n, b, seed=n + b, dtype=npdt))
    w = []
    for cnt in (n, n - 1, n - 1):
        x = rng.standard_normal((cnt, b, b)) + (1j * rng.standard_normal((cnt, b, b)) if dtype.is_complex else 0)
        w.append(torch.from_numpy(np.asarray(x, npdt)).cuda())
    g_ours, l_ours = grads(lambda a, bb, c: rgf_autograd(a, bb, c, team=team), d, u, l, w)
    g_ref, l_ref = grads(dense_selected, d, u, l, w)
    assert abs(l_ours - l_ref) <= 1e-10 * max(1.0, abs(l_ref))
    for go, gr in zip(g_ours, g_ref):
        if gr.numel():
            assert rel(go, gr) <= 1e-9, rel(go, gr)


@pytest.mark.parametrize("sym", [False, True])
def test_adjoint_tight_binding_hamiltonian_gradient(sym):
    """dL/dH for L = sum_k sum_i -Im Tr G_ii(E_k) / pi, A_k = (E_k + i eta) I - H - Sigma."""
    n, b = 6, 24
    onsite, coupling = workloads.hamiltonian(n, b, seed=5)
    Hd = torch.from_numpy(onsite).cuda().requires_grad_(True)
    Hu = torch.from_numpy(coupling).cuda().requires_grad_(True)
    energies = [-0.7, 0.2, 1.1]
    eye = torch.eye(b, dtype=torch.complex128, device="cuda")

    def assemble(Hd, Hu, E):
        d = (E + 1e-3j) * eye - Hd.to(torch.complex128)
        d = d.clone()
        d[0] = d[0] + 0.1j * eye
        d[-1] = d[-1] + 0.1j * eye
        u = -Hu.to(torch.complex128)
        l = -Hu.transpose(1, 2).to(torch.complex128)
        return d, u, l

    def total(fn):
        loss = 0
        for E in energies:
            Gd, Gu, Gl = fn(*assemble(Hd, Hu, E))
            loss = loss - Gd.diagonal(0, 1, 2).imag.sum() / np.pi
        return loss

    for H in (Hd, Hu):
        H.grad = None
    total(lambda d, u, l: rgf_autograd(d, u, l, sym_mat=sym)).backward()
    ours = [Hd.grad.clone(), Hu.grad.clone()]
    for H in (Hd, Hu):
        H.grad = None
    total(dense_selected).backward()
    for a, r in zip(ours, [Hd.grad, Hu.grad]):
        assert rel(a, r) <= 1e-8, rel(a, r)


def test_adjoint_central_finite_differences():
    n, b, h = 6, 12, 1e-6
    d, u, l = (torch.from_numpy(x).cuda() for x in workloads.tight_binding(n, b, 0.4, seed=9))
    rng = np.random.default_rng(1)
    w = [torch.from_numpy(rng.standard_normal(s) + 1j * rng.standard_normal(s)).cuda()
         for s in ((n, b, b), (n - 1, b, b), (n - 1, b, b))]
    (gd, gu, gl), _ = grads(rgf_autograd, d, u, l, w)
    for trial in range(3):
        V = [torch.from_numpy(rng.standard_normal(x.shape) + 1j * rng.standard_normal(x.shape)).cuda()
             for x in (d, u, l)]
        with torch.no_grad():
            Lp = loss_fn(*rgf_autograd(d + h * V[0], u + h * V[1], l + h * V[2]), *w).item()
            Lm = loss_fn(*rgf_autograd(d - h * V[0], u - h * V[1], l - h * V[2]), *w).item()
        fd = (Lp - Lm) / (2 * h)
        # torch's gradient of a real loss w.r.t. a complex tensor z is 2 dL/dz*,
        # so the directional derivative along v is Re <grad, v>
        an = sum((torch.conj(g) * v).real.sum().item() for g, v in zip((gd, gu, gl), V))
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (fd, an)


def test_single_precision_gradient_dtype():
    d, u, l = (torch.from_numpy(x).cuda() for x in workloads.dominant(4, 8, seed=2, dtype=np.complex64))
    leaves = [x.clone().requires_grad_(True) for x in (d, u, l)]
    Gd, Gu, Gl = rgf_autograd(*leaves)
    (Gd.real.sum() + Gu.imag.sum()).backward()
    assert all(x.grad.dtype == torch.complex64 for x in leaves)
    ref = [x.to(torch.complex128).requires_grad_(True) for x in (d, u, l)]
    Rd, Ru, Rl = dense_selected(*ref)
    (Rd.real.sum() + Ru.imag.sum()).backward()
    for a, r in zip(leaves, ref):
        assert rel(a.grad.to(torch.complex128), r.grad) <= 1e-5
