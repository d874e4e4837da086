"""Multi-rank PSR host logic on CPU: ``distributed.psr_distributed`` run as 3 and
4 ``gloo`` ranks, one partition per rank (the reference's layout,
``src/sinv/algorithms/psr/psr_seqsolve.py:20-73``).

Each rank's compute here is a stand-in built from the oracle's partition
functions (test code only); on GPUs the same host logic drives ``PsrPart``
(``sinvb_psr_part_*``).  Each rank passes only its partition's rows.  What is
under test: the boundary slots each rank contributes, the one all-gather, the
reduced system every rank assembles and solves, the boundary blocks and
coupling each rank takes back, and the final gather of the rows.  The result must equal the oracle PSR on the same
partitions and the dense inverse.
"""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import dense, psr_oracle, rgf_oracle
from sinv_b200 import distributed, workloads


class OraclePart:
    """The per-rank compute of ``psr_distributed`` on the CPU, from the oracle
    (it reads the whole matrix, test code only; the slots and outputs follow
    the ``PsrPart`` contract)."""

    def __init__(self, d, u, l, P, part):
        self.dn, self.un, self.ln = d, u, l
        self.n, self.b = d.shape[0], d.shape[1]
        self.u, self.l = torch.from_numpy(u), torch.from_numpy(l)
        self.P, self.part = P, part
        starts, sizes = psr_oracle.divide(self.n, P)
        self.s, self.m = starts[part], sizes[part]
        self.rows = (self.s, self.s + self.m - 1)

    def _kind(self, red, cen, last):
        return red if self.part == 0 else last if self.part == self.P - 1 else cen

    def reduce(self):
        self.A = psr_oracle._blocks(self.dn, self.un, self.ln)
        self.L, self.U, self.Dinv = {}, {}, {}
        f = self._kind(psr_oracle.reduce_topleft, psr_oracle.reduce_central, psr_oracle.reduce_bottomright)
        f(self.A, self.L, self.U, self.Dinv, self.s, self.m)
        t, B = self.rows
        z = np.zeros_like(self.dn[0])
        if self.part == 0:
            slots = [self.A[(B, B)], z, z, z]
        elif self.part == self.P - 1:
            slots = [self.A[(t, t)], z, z, z]
        else:
            slots = [self.A[(t, t)], self.A[(B, B)], self.A[(t, B)], self.A[(B, t)]]
        link = [self.un[B], self.ln[B]] if self.part < self.P - 1 else [z, z]
        return torch.from_numpy(np.stack(slots + link))

    def solve_reduced(self, Rd, Ru, Rl):
        return tuple(torch.from_numpy(x) for x in rgf_oracle.rgf(Rd.numpy(), Ru.numpy(), Rl.numpy()))

    def produce(self, slots, link):
        t, B = self.rows
        sl = slots.numpy()
        G = {}
        if self.part == 0:
            G[(B, B)] = sl[0]
        elif self.part == self.P - 1:
            G[(t, t)] = sl[0]
        else:
            G[(t, t)], G[(B, B)], G[(t, B)], G[(B, t)] = sl[0], sl[1], sl[2], sl[3]
        f = self._kind(psr_oracle.produce_topleft, psr_oracle.produce_central, psr_oracle.produce_bottomright)
        f(self.A, self.L, self.U, self.Dinv, G, self.s, self.m)
        b = self.b
        m = B - t + 1
        mc = m if self.part < self.P - 1 else m - 1
        Gd = np.zeros((m, b, b), self.dn.dtype)
        Gu = np.zeros((mc, b, b), self.dn.dtype)
        Gl = np.zeros((mc, b, b), self.dn.dtype)
        for i in range(t, B + 1):
            Gd[i - t] = G[(i, i)]
            if i < B:
                Gu[i - t], Gl[i - t] = G[(i, i + 1)], G[(i + 1, i)]
        if link is not None:
            Gu[m - 1], Gl[m - 1] = link[0].numpy(), link[1].numpy()
        return torch.from_numpy(Gd), torch.from_numpy(Gu), torch.from_numpy(Gl)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir, n, b, gather):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from sinv_b200.algorithms.psr_seqsolve import local_blocks
        d, u, l = workloads.dominant(n, b, seed=n + b)
        ld, lu, ll = local_blocks(d, u, l, world, rank)
        G = distributed.psr_distributed(ld, lu, ll, n, gather=gather,
                                        make_part=lambda: OraclePart(d, u, l, world, rank))
        np.savez(os.path.join(out_dir, "r%d.npz" % rank), *[g.numpy() for g in G])
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,n,b", [(3, 9, 4), (3, 14, 3), (4, 17, 5)])
def test_psr_ranks_match_oracle(tmp_path, world, n, b):
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path), n, b, True), nprocs=world, join=True)
    d, u, l = workloads.dominant(n, b, seed=n + b)
    R = psr_oracle.psr(d, u, l, world)
    D = dense.inv_selected(d, u, l)
    for r in range(world):
        z = np.load(os.path.join(tmp_path, "r%d.npz" % r))
        G = [z["arr_%d" % k] for k in range(3)]
        for g, x, y in zip(G, R, D):
            assert dense.rel_fro(g, x) <= 1e-13
            assert dense.rel_fro(g, y) <= 1e-12


def test_psr_ranks_without_gather_own_their_rows(tmp_path):
    world, n, b = 3, 11, 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path), n, b, False), nprocs=world, join=True)
    d, u, l = workloads.dominant(n, b, seed=n + b)
    R = psr_oracle.psr(d, u, l, world)
    starts, sizes = psr_oracle.divide(n, world)
    for r in range(world):
        z = np.load(os.path.join(tmp_path, "r%d.npz" % r))
        t, B = starts[r], starts[r] + sizes[r] - 1
        e = min(B + 1, n - 1)
        assert z["arr_0"].shape[0] == B + 1 - t and z["arr_1"].shape[0] == e - t
        assert dense.rel_fro(z["arr_0"], R[0][t:B + 1]) <= 1e-13
        assert dense.rel_fro(z["arr_1"], R[1][t:e]) <= 1e-13
        assert dense.rel_fro(z["arr_2"], R[2][t:e]) <= 1e-13
