"""Multi-rank host logic on CPU: the cost-balanced energy sharding and the
gradient all-reduce, run as two ``gloo`` ranks (no GPU).

The per-energy term here is a dense numpy evaluation of
L(E) = -Im Tr G(E) / pi and its gradient with respect to H (test code only);
on GPUs the same function runs the batched adjoint.
"""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from sinv_b200 import distributed, workloads

N, B = 4, 5
ENERGIES = [-1.5, -0.4, 0.1, 0.7, 1.3]


def dense_term(H_onsite, H_coupling, E, eta=1e-3, sigma=0.1):
    """(loss, dL/dH_onsite, dL/dH_coupling) from a dense inverse."""
    n, b = H_onsite.shape[0], H_onsite.shape[1]
    H = np.zeros((n * b, n * b))
    for i in range(n):
        H[i * b:(i + 1) * b, i * b:(i + 1) * b] = H_onsite[i]
        if i < n - 1:
            H[i * b:(i + 1) * b, (i + 1) * b:(i + 2) * b] = H_coupling[i]
            H[(i + 1) * b:(i + 2) * b, i * b:(i + 1) * b] = H_coupling[i].T
    S = np.zeros((n * b, n * b), complex)
    S[:b, :b] -= 1j * sigma * np.eye(b)
    S[-b:, -b:] -= 1j * sigma * np.eye(b)
    A = (E + 1j * eta) * np.eye(n * b) - H - S
    G = np.linalg.inv(A)
    loss = -np.trace(G).imag / np.pi
    # dL/dH_jk = -(1/pi) Im (G^2)_kj  (A depends on -H)
    dH = -(G @ G).T.imag / np.pi
    g_on = np.stack([dH[i * b:(i + 1) * b, i * b:(i + 1) * b] for i in range(n)])
    g_cp = np.stack([dH[i * b:(i + 1) * b, (i + 1) * b:(i + 2) * b]
                     + dH[(i + 1) * b:(i + 2) * b, i * b:(i + 1) * b].T for i in range(n - 1)])
    return loss, g_on, g_cp


def _term_fn(H_on, H_cp):
    def term(E):
        l, go, gc = dense_term(H_on, H_cp, E)
        return (torch.tensor(l, dtype=torch.float64), torch.from_numpy(go), torch.from_numpy(gc))
    return term


def _rank_main(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        H_on, H_cp = workloads.hamiltonian(N, B, seed=4)
        loss, g_on, g_cp = distributed.energy_loss_and_grad(
            torch.from_numpy(H_on), torch.from_numpy(H_cp), ENERGIES, compute=_term_fn(H_on, H_cp))
        np.savez(os.path.join(out_dir, "rank%d.npz" % rank), loss=loss.numpy(), g_on=g_on.numpy(),
                 g_cp=g_cp.numpy())
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_gradient_allreduce_two_gloo_ranks(tmp_path):
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    H_on, H_cp = workloads.hamiltonian(N, B, seed=4)
    ref = [dense_term(H_on, H_cp, E) for E in ENERGIES]
    ref_loss = sum(r[0] for r in ref)
    ref_on = sum(r[1] for r in ref)
    ref_cp = sum(r[2] for r in ref)
    outs = [np.load(tmp_path / ("rank%d.npz" % r)) for r in range(world)]
    for o in outs:  # every rank holds the full sum
        assert np.allclose(o["loss"], ref_loss, rtol=1e-12)
        assert np.allclose(o["g_on"], ref_on, rtol=1e-10, atol=1e-12)
        assert np.allclose(o["g_cp"], ref_cp, rtol=1e-10, atol=1e-12)


def test_dense_gradient_matches_finite_differences():
    """The CPU stand-in itself: central differences on one coupling entry."""
    H_on, H_cp = workloads.hamiltonian(3, 3, seed=2)
    _, _, gc = dense_term(H_on, H_cp, 0.3)
    h = 1e-6
    Hp, Hm = H_cp.copy(), H_cp.copy()
    Hp[1, 0, 2] += h
    Hm[1, 0, 2] -= h
    fd = (dense_term(H_on, Hp, 0.3)[0] - dense_term(H_on, Hm, 0.3)[0]) / (2 * h)
    assert abs(fd - gc[1, 0, 2]) <= 1e-5 * max(1.0, abs(fd))


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_shard_by_cost_partitions_and_balances(world):
    spec = workloads.energy_batch_spec()
    costs = [distributed.instance_cost(n, b) for (_, n, b, _) in spec]
    bins = distributed.shard_by_cost(costs, world)
    flat = sorted(k for b in bins for k in b)
    assert flat == list(range(len(spec)))
    assert bins == distributed.shard_by_cost(costs, world)       # deterministic
    assert all(distributed.shard_by_cost(costs, world, r) == bins[r] for r in range(world))
    loads = [sum(costs[k] for k in b) for b in bins]
    assert max(loads) <= 1.05 * sum(loads) / world + max(costs)  # LPT bound


def test_single_process_fallback_sums_locally():
    H_on, H_cp = workloads.hamiltonian(N, B, seed=4)
    loss, g_on, _ = distributed.energy_loss_and_grad(torch.from_numpy(H_on), torch.from_numpy(H_cp), ENERGIES,
                                                     compute=_term_fn(H_on, H_cp))
    ref = sum(dense_term(H_on, H_cp, E)[0] for E in ENERGIES)
    assert abs(loss.item() - ref) <= 1e-12 * abs(ref)


def _dense_lesser_all(inst, sigs):
    """The six block families of G and G< = G Sigma< G^H per instance (dense, test code)."""
    res = []
    for (d, u, l), s in zip(inst, sigs):
        n, b = d.shape[0], d.shape[1]
        A = np.zeros((n * b, n * b), complex)
        S = np.zeros_like(A)
        for i in range(n):
            A[i * b:(i + 1) * b, i * b:(i + 1) * b] = d[i]
            S[i * b:(i + 1) * b, i * b:(i + 1) * b] = s[i]
            if i < n - 1:
                A[i * b:(i + 1) * b, (i + 1) * b:(i + 2) * b] = u[i]
                A[(i + 1) * b:(i + 2) * b, i * b:(i + 1) * b] = l[i]
        G = np.linalg.inv(A)
        GL = G @ S @ G.conj().T
        blk = lambda M, i, j: M[i * b:(i + 1) * b, j * b:(j + 1) * b]
        fam = lambda M: (np.array([blk(M, i, i) for i in range(n)]),
                         np.array([blk(M, i, i + 1) for i in range(n - 1)]),
                         np.array([blk(M, i + 1, i) for i in range(n - 1)]))
        res.append(fam(G) + fam(GL))
    return res


def _lesser_problem():
    shapes = [(3, 4), (5, 3), (2, 6), (4, 4), (3, 5), (6, 2), (2, 3)]
    inst = [workloads.tight_binding(n, b, -1.0 + 0.3 * k, seed=60 + k) for k, (n, b) in enumerate(shapes)]
    sigs = []
    for (n, b) in shapes:
        s = np.zeros((n, b, b), complex)
        s[0] = s[-1] = 0.2j * np.eye(b)
        sigs.append(s)
    return inst, sigs


def _lesser_rank_main(rank, world, port, out_dir):
    import pickle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        inst, sigs = _lesser_problem()
        mine = distributed.rgf_lesser_batched_sharded(inst, sigs, compute=_dense_lesser_all)
        every = distributed.rgf_lesser_batched_sharded(inst, sigs, gather=True, compute=_dense_lesser_all)
        with open(os.path.join(out_dir, "lesser%d.pkl" % rank), "wb") as f:
            pickle.dump((sorted(mine), every), f)
    finally:
        dist.destroy_process_group()


def test_lesser_energies_sharded_over_two_gloo_ranks(tmp_path):
    """Each rank computes its cost-balanced share of the energies; the shares
    cover every instance once, and the gathered results are every instance's
    on every rank."""
    import pickle
    world = 2
    mp.spawn(_lesser_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    inst, sigs = _lesser_problem()
    ref = _dense_lesser_all(inst, sigs)
    got = [pickle.load(open(tmp_path / ("lesser%d.pkl" % r), "rb")) for r in range(world)]
    shares = [set(m) for m, _ in got]
    assert shares[0].isdisjoint(shares[1]) and shares[0] | shares[1] == set(range(len(inst)))
    assert all(shares)
    for _, every in got:
        assert sorted(every) == list(range(len(inst)))
        for k in range(len(inst)):
            for g, r in zip(every[k], ref[k]):
                assert np.allclose(g, r, rtol=1e-12, atol=1e-14)
