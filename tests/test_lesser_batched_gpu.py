"""Batched lesser / greater Green's functions (``sinvb_rgf_lesser_batched_z``)
against the single-matrix call, the dense FP64 product G Sigma< G^H and, for
the retarded blocks, the oracle restatement of the reference rgf
(``src/sinv/algorithms/rgf/rgf.py:17-64``).  Tolerances (relative Frobenius
per block family): 1e-11 on tight-binding instances (against the
single-matrix call, whose team and tiling differ above b = 48, the dense
product and the oracle), 1e-12 on diagonally dominant ones.
"""

import numpy as np
import pytest

from oracle import dense, rgf_oracle
from sinv_b200 import _lib, workloads
from sinv_b200.algorithms import rgf_greater_batched, rgf_lesser, rgf_lesser_batched

pytestmark = pytest.mark.gpu


def _sigma(n, b, seed):
    """Lesser self-energy of the two contacts: i x (positive semidefinite) on
    the first and last diagonal blocks."""
    rng = np.random.default_rng(seed)
    s = np.zeros((n, b, b), np.complex128)
    for i in sorted({0, n - 1}):
        R = rng.standard_normal((b, b)) + 1j * rng.standard_normal((b, b))
        s[i] = 1j * (R @ R.conj().T) / b
    return s


def _dense_lesser(d, u, l, s):
    n, b = d.shape[0], d.shape[1]
    G = np.linalg.inv(dense.to_dense(d, u, l))
    S = np.zeros_like(G)
    for i in range(n):
        S[i * b:(i + 1) * b, i * b:(i + 1) * b] = s[i]
    GL = G @ S @ G.conj().T
    blk = lambda M, i, j: M[i * b:(i + 1) * b, j * b:(j + 1) * b]
    return (np.array([blk(GL, i, i) for i in range(n)]), np.array([blk(GL, i, i + 1) for i in range(n - 1)]),
            np.array([blk(GL, i + 1, i) for i in range(n - 1)]))


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    if b.size == 0:
        return 0.0
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


SHAPES = [(4, 32), (6, 64), (3, 128), (2, 256), (5, 16), (1, 48), (7, 24), (2, 512)]


@pytest.mark.parametrize("team", [None, "cta"])
def test_ragged_batch_matches_single_calls_dense_and_oracle(team):
    inst = [workloads.tight_binding(n, b, -1.5 + 0.4 * k, seed=300 + k) for k, (n, b) in enumerate(SHAPES)]
    sig = [_sigma(n, b, 400 + k) for k, (n, b) in enumerate(SHAPES)]
    got = rgf_lesser_batched(inst, sig, team=team)
    for k, ((d, u, l), s, res) in enumerate(zip(inst, sig, got)):
        one = rgf_lesser(d, u, l, s)
        for g, r in zip(res, one):
            assert _rel(g, r) <= 1e-11, (k, _rel(g, r))
        GL = _dense_lesser(d, u, l, s)
        for g, r in zip(res[3:], GL):
            assert _rel(g, r) <= 1e-11, (k, _rel(g, r))
        R = rgf_oracle.rgf(d, u, l)
        for g, r in zip(res[:3], R):
            assert _rel(g, r) <= 1e-11, (k, _rel(g, r))


def test_energies_of_one_hamiltonian_share_their_coupling_blocks():
    """The energy loop: one H, many energies; the coupling blocks are the same
    device tensors in every descriptor (inputs may be shared)."""
    import torch
    n, b = 8, 64
    onsite, coupling = workloads.hamiltonian(n, b, 77)
    energies = np.linspace(-1.8, 1.8, 24)
    host = [workloads.tight_binding(n, b, e, H=(onsite, coupling)) for e in energies]
    u = torch.from_numpy(host[0][1]).cuda()
    l = torch.from_numpy(host[0][2]).cuda()
    for d_, u_, l_ in host:
        assert np.array_equal(u_, host[0][1]) and np.array_equal(l_, host[0][2])
    inst = [(torch.from_numpy(d_).cuda(), u, l) for d_, _, _ in host]
    sig = [torch.from_numpy(_sigma(n, b, 500 + k)).cuda() for k in range(len(host))]
    got = rgf_lesser_batched(inst, sig)
    for k in range(0, len(host), 5):
        one = rgf_lesser(*host[k], sig[k].cpu().numpy())
        for g, r in zip(got[k], one):
            assert _rel(g.cpu().numpy(), r) <= 1e-11, k
    # numpy inputs sharing one host array per coupling block family (moved to the device once)
    hu, hl = host[0][1], host[0][2]
    got_np = rgf_lesser_batched([(d_, hu, hl) for d_, _, _ in host], [x.cpu().numpy() for x in sig])
    for k in range(len(host)):
        for g, r in zip(got_np[k], got[k]):
            assert _rel(g, r.cpu().numpy()) == 0.0, k


def test_more_instances_than_scratch_slots():
    """200 one-CTA instances on 148 scratch slots: every slot is returned and reused."""
    shapes = [(3, 16)] * 200
    inst = [workloads.tight_binding(n, b, 0.01 * k - 1.0, seed=600 + k) for k, (n, b) in enumerate(shapes)]
    sig = [_sigma(n, b, 700 + k) for k, (n, b) in enumerate(shapes)]
    st = []
    got = rgf_lesser_batched(inst, sig, statuses=st)
    assert st == [_lib.OK] * len(shapes)
    for k in range(0, len(shapes), 23):
        for g, r in zip(got[k][3:], _dense_lesser(*inst[k], sig[k])):
            assert _rel(g, r) <= 1e-11, k


def test_a_failed_pivot_is_reported_for_its_instance_only():
    shapes = [(3, 32), (4, 32), (3, 64)]
    inst = [workloads.dominant(n, b, seed=800 + k) for k, (n, b) in enumerate(shapes)]
    d0 = inst[1][0].copy()
    d0[0] = 0.0   # the first block inverse of instance 1 meets a zero pivot
    inst[1] = (d0, inst[1][1], inst[1][2])
    sig = [_sigma(n, b, 900 + k) for k, (n, b) in enumerate(shapes)]
    st = []
    got = rgf_lesser_batched(inst, sig, check=False, statuses=st)
    assert st == [_lib.OK, _lib.STATUS_PIVOT, _lib.OK]
    for k in (0, 2):
        for g, r in zip(got[k][3:], _dense_lesser(*inst[k], sig[k])):
            assert _rel(g, r) <= 1e-12, k
    with pytest.raises(np.linalg.LinAlgError):
        rgf_lesser_batched(inst, sig)


def test_greater_minus_lesser_is_G_minus_G_dagger_for_every_energy():
    """Sigma< = i f Gamma, Sigma> = -i (1 - f) Gamma with Gamma = i (Sigma^R - Sigma^A)
    (the eta broadening everywhere plus the contact blocks of the tight-binding
    model): the batched results obey G> - G< = G - G^H on the diagonal blocks."""
    shapes = [(5, 32), (4, 64), (3, 128)]
    inst, sl, sg = [], [], []
    eye = lambda b: np.eye(b)
    for k, (n, b) in enumerate(shapes):
        d, u, l = workloads.tight_binding(n, b, -0.7 + 0.5 * k, seed=1000 + k)
        gamma = np.stack([2 * workloads.ETA * eye(b) + (2 * workloads.SIGMA_EDGE * eye(b) if i in (0, n - 1) else 0)
                          for i in range(n)]).astype(np.complex128)
        f = 0.3 + 0.1 * k
        inst.append((d, u, l))
        sl.append(1j * f * gamma)
        sg.append(-1j * (1 - f) * gamma)
    les = rgf_lesser_batched(inst, sl)
    gre = rgf_greater_batched(inst, sg)
    for k in range(len(shapes)):
        Gd = les[k][0]
        lhs = gre[k][3] - les[k][3]
        rhs = Gd - np.conj(np.transpose(Gd, (0, 2, 1)))
        assert _rel(lhs, rhs) <= 1e-10, (k, _rel(lhs, rhs))


def test_sharded_form_on_one_process_runs_the_batched_call():
    """distributed.rgf_lesser_batched_sharded with no process group: this
    process's share is every instance, computed by the batched call."""
    from sinv_b200 import distributed
    shapes = [(3, 32), (5, 64), (2, 16)]
    inst = [workloads.tight_binding(n, b, 0.2 * k, seed=1100 + k) for k, (n, b) in enumerate(shapes)]
    sig = [_sigma(n, b, 1200 + k) for k, (n, b) in enumerate(shapes)]
    got = distributed.rgf_lesser_batched_sharded(inst, sig)
    ref = rgf_lesser_batched(inst, sig)
    assert sorted(got) == [0, 1, 2]
    for k in range(3):
        for g, r in zip(got[k], ref[k]):
            assert _rel(g, r) == 0.0
