"""Mixed-precision batched RGF: block products on the int8 tensor cores.

The mixed path computes the block products of both sweeps with the Ozaki
scheme on tcgen05 (int8 slices, exact int32 sums, FP64 reconstruction) for
blocks of b >= 256, FP64 DMMA products for smaller blocks, and every block
inverse in FP64.  It is checked against the FP64 batched path and
the oracle restatement of the reference rgf
(``src/sinv/algorithms/rgf/rgf.py:17-64``).

Tolerances (relative Frobenius, per output array):
  * 1e-8 on tight-binding instances, the accuracy bar of the mixed mode;
  * 1e-9 on diagonally dominant instances with 6 digits;
  * each extra digit must not make the error worse, and 8 digits reach 5e-12
    (b = 256 tight-binding blocks).
"""

import numpy as np
import pytest

from oracle import dense, rgf_oracle
from sinv_b200 import workloads
from sinv_b200.algorithms import BatchPlan, rgf_batched

pytestmark = pytest.mark.gpu


def _worst(G, R):
    return max(dense.rel_fro(x, r) for x, r in zip(G, R) if r.size)


RAGGED = [(1, 8), (3, 33), (4, 64), (2, 65), (5, 100), (3, 128), (2, 130), (6, 16), (3, 256), (2, 300), (1, 512)]


def test_mixed_ragged_dominant():
    inst = [workloads.dominant(n, b, seed=300 + k) for k, (n, b) in enumerate(RAGGED)]
    mixed = rgf_batched(inst, precision="mixed")
    for (d, u, l), G in zip(inst, mixed):
        assert _worst(G, rgf_oracle.rgf(d, u, l)) <= 1e-9


def test_mixed_tight_binding_meets_1e8():
    spec = workloads.energy_batch_spec(count=64)[:8]
    inst = [workloads.tight_binding(min(n, 16), b, e, seed=s) for (e, n, b, s) in spec]
    fp64 = rgf_batched(inst)
    mixed = rgf_batched(inst, precision="mixed")
    for (d, u, l), G, R in zip(inst, mixed, fp64):
        assert _worst(G, R) <= 1e-8, _worst(G, R)
    d, u, l = inst[0]
    assert _worst(mixed[0][:1], dense.inv_selected(d, u, l)[:1]) <= 1e-8


def test_mixed_digits_trade_accuracy():
    inst = [workloads.tight_binding(4, 256, 0.3 + 0.1 * k, seed=40 + k) for k in range(3)]
    ref = rgf_batched(inst)
    errs = []
    for digits in (5, 6, 7, 8):
        out = rgf_batched(inst, precision="mixed", digits=digits)
        errs.append(max(_worst(G, R) for G, R in zip(out, ref)))
    for a, b in zip(errs, errs[1:]):
        assert b <= a * 1.5 + 1e-15, errs
    assert errs[-1] <= 5e-12, errs
    assert errs[0] <= 1e-5, errs


@pytest.mark.parametrize("inplace", [False, True])
def test_mixed_teams_and_in_place(inplace):
    """b = 256 / 512 run on teams of 2 / 4 CTAs sharing the tile work of each product."""
    import torch
    shapes = [(3, 512), (2, 256), (4, 64), (3, 192)]
    inst = [workloads.dominant(n, b, seed=500 + k) for k, (n, b) in enumerate(shapes)]
    tinst = [tuple(torch.from_numpy(x).cuda() for x in t) for t in inst]
    plan = BatchPlan(tinst, precision="mixed", inplace=inplace)
    plan.run()
    plan.check()
    for (d, u, l), G in zip(inst, plan.results()):
        assert _worst([g.cpu().numpy() for g in G], rgf_oracle.rgf(d, u, l)) <= 1e-9
    single = BatchPlan([tuple(torch.from_numpy(x).cuda() for x in t) for t in inst], precision="mixed",
                       team="cta")
    single.run()
    single.check()
    for G1, G2 in zip(plan.results(), single.results()):
        for a, b in zip(G1, G2):
            assert dense.rel_fro(a.cpu().numpy(), b.cpu().numpy()) <= 1e-9


@pytest.mark.parametrize("sym", [False, True])
def test_mixed_flags(sym):
    inst = []
    for k, (n, b) in enumerate([(4, 8), (6, 70), (3, 256), (2, 260)]):
        d, u, l = workloads.dominant(n, b, seed=k)
        if sym:
            d = d + np.transpose(d, (0, 2, 1))
            l = np.ascontiguousarray(np.transpose(u, (0, 2, 1)))
        inst.append((d, u, l))
    out = rgf_batched(inst, sym_mat=sym, precision="mixed")
    for (d, u, l), G in zip(inst, out):
        assert _worst(G, rgf_oracle.rgf(d, u, l, sym_mat=sym)) <= 1e-9
    out = rgf_batched(inst, sym_mat=sym, save_off_diag=False, precision="mixed")
    for (d, u, l), G in zip(inst, out):
        assert _worst(G[:1], rgf_oracle.rgf(d, u, l, sym_mat=sym)[:1]) <= 1e-9


def test_mixed_rerun_is_deterministic():
    import torch
    inst = [workloads.dominant(n, b, seed=9 + n) for n, b in [(5, 64), (3, 256)]]
    tinst = [tuple(torch.from_numpy(x).cuda() for x in t) for t in inst]
    plan = BatchPlan(tinst, precision="mixed")
    plan.run()
    first = [tuple(g.clone() for g in G) for G in plan.results()]
    plan.run()
    plan.check()
    for G0, G1 in zip(first, plan.results()):
        for a, b in zip(G0, G1):
            assert torch.equal(a, b)
