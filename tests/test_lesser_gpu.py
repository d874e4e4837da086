"""Lesser Green's function G< = G Sigma< G^H in the RGF sweeps, checked
against the dense FP64 product (test-side numpy) and, for the retarded
blocks, the oracle restatement of the reference rgf
(``src/sinv/algorithms/rgf/rgf.py:17-64``).  Tolerances: 1e-11 relative
Frobenius per block family on tight-binding matrices, 1e-12 on diagonally
dominant ones.
"""

import numpy as np
import pytest

from oracle import dense, rgf_oracle
from sinv_b200 import workloads
from sinv_b200.algorithms import rgf_greater, rgf_lesser

pytestmark = pytest.mark.gpu


def _sigma(n, b, seed, contacts_only):
    rng = np.random.default_rng(seed)
    s = np.zeros((n, b, b), np.complex128)
    for i in range(n):
        if contacts_only and 0 < i < n - 1:
            continue
        R = rng.standard_normal((b, b)) + 1j * rng.standard_normal((b, b))
        s[i] = 1j * (R @ R.conj().T) / b  # i x (positive semidefinite): a lesser self-energy
    return s


def _dense_lesser(d, u, l, s):
    n, b = d.shape[0], d.shape[1]
    G = np.linalg.inv(dense.to_dense(d, u, l))
    S = np.zeros_like(G)
    for i in range(n):
        S[i * b:(i + 1) * b, i * b:(i + 1) * b] = s[i]
    GL = G @ S @ G.conj().T
    blk = lambda M, i, j: M[i * b:(i + 1) * b, j * b:(j + 1) * b]
    return ([blk(GL, i, i) for i in range(n)], [blk(GL, i, i + 1) for i in range(n - 1)],
            [blk(GL, i + 1, i) for i in range(n - 1)])


def _worst(A, R):
    return max([dense.rel_fro(np.asarray(a), r) for a, r in zip(A, R) if np.asarray(r).size] or [0.0])


@pytest.mark.parametrize("n,b,team", [(1, 8, None), (2, 8, None), (5, 16, None), (9, 33, None), (7, 64, "cta"),
                                      (6, 96, None), (4, 130, None), (12, 40, "grid")])
@pytest.mark.parametrize("contacts_only", [True, False])
def test_lesser_matches_dense(n, b, team, contacts_only):
    d, u, l = workloads.tight_binding(n, b, 0.2, seed=n + b)
    s = _sigma(n, b, seed=3 * n + b, contacts_only=contacts_only)
    Gd, Gu, Gl, GLd, GLu, GLl = rgf_lesser(d, u, l, s, team=team)
    Rd, Ru, Rl = _dense_lesser(d, u, l, s)
    assert _worst(GLd, Rd) <= 1e-11
    assert _worst(GLu, Ru) <= 1e-11
    assert _worst(GLl, Rl) <= 1e-11
    ref = rgf_oracle.rgf(d, u, l)
    assert _worst([Gd, Gu, Gl], ref) <= 1e-11


def test_lesser_dominant_and_torch():
    import torch
    d, u, l = workloads.dominant(8, 48, seed=4)
    s = _sigma(8, 48, seed=1, contacts_only=False)
    out = rgf_lesser(*(torch.from_numpy(x).cuda() for x in (d, u, l, s)))
    assert all(t.is_cuda for t in out)
    Rd, Ru, _ = _dense_lesser(d, u, l, s)
    assert _worst([t.cpu().numpy() for t in out[3]], Rd) <= 1e-12
    assert _worst([t.cpu().numpy() for t in out[4]], Ru) <= 1e-12


@pytest.mark.parametrize("n,b,E", [(6, 16, 0.2), (9, 64, -0.7), (4, 130, 1.1)])
def test_greater_minus_lesser_is_spectral(n, b, E):
    """Sigma< = i f Gamma, Sigma> = -i (1 - f) Gamma with Gamma = i (Sigma^R - Sigma^A)
    (the eta broadening everywhere plus the contact blocks of the tight-binding
    model): then G> - G< = G (Sigma^R - Sigma^A) G^H = G - G^H, blockwise."""
    d, u, l = workloads.tight_binding(n, b, E, seed=n * b)
    eye = np.eye(b)
    gamma = np.stack([2 * workloads.ETA * eye + (2 * workloads.SIGMA_EDGE * eye if i in (0, n - 1) else 0)
                      for i in range(n)]).astype(np.complex128)
    f = 0.3
    sl = 1j * f * gamma
    sg = -1j * (1 - f) * gamma
    Gd, Gu, Gl, Ld, Lu, Ll = rgf_lesser(d, u, l, sl)
    _, _, _, Hd, Hu, Hl = rgf_greater(d, u, l, sg)
    Rd, Ru, Rl = _dense_lesser(d, u, l, sg)
    assert _worst(Hd, Rd) <= 1e-11 and _worst(Hu, Ru) <= 1e-11 and _worst(Hl, Rl) <= 1e-11
    spec_d = Gd - np.conj(np.transpose(Gd, (0, 2, 1)))
    spec_u = Gu - np.conj(np.transpose(Gl, (0, 2, 1)))
    assert _worst([Hd - Ld], [spec_d]) <= 1e-10
    assert _worst([Hu - Lu], [spec_u]) <= 1e-10
