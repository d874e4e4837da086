"""GPU parity of the batched RGF (one persistent launch over many matrices).

Every instance is checked against the CPU oracle restatement of the reference
rgf (``src/sinv/algorithms/rgf/rgf.py:17-64``), one matrix at a time.
Tolerance: 1e-12 relative Frobenius for diagonally dominant instances; for
tight-binding instances (condition numbers ~1e3 at eta = 1e-3) 1e-11.
"""

import numpy as np
import pytest

from oracle import dense, rgf_oracle
from sinv_b200 import workloads
from sinv_b200.algorithms import BatchPlan, rgf_batched

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return dense.rel_fro(a, b)


def _check(G, R, tol):
    for x, r in zip(G, R):
        if r.size:
            assert _rel(x, r) <= tol, (_rel(x, r), tol)


RAGGED = [(1, 1), (3, 3), (4, 16), (2, 32), (7, 33), (5, 64), (3, 65), (6, 128), (1, 40), (9, 8), (2, 130),
          (12, 24)]


@pytest.mark.parametrize("dtype", [np.complex128, np.float64])
def test_ragged_batch_matches_oracle(dtype):
    inst = [workloads.dominant(n, b, seed=100 + k, dtype=dtype) for k, (n, b) in enumerate(RAGGED)]
    out = rgf_batched(inst)
    assert len(out) == len(inst)
    for (d, u, l), G in zip(inst, out):
        _check(G, rgf_oracle.rgf(d, u, l), 1e-12)


@pytest.mark.parametrize("sym", [False, True])
def test_batch_flags(sym):
    inst = []
    for k, (n, b) in enumerate([(4, 8), (6, 70), (3, 33)]):
        d, u, l = workloads.dominant(n, b, seed=k)
        if sym:
            d = d + np.transpose(d, (0, 2, 1))
            l = np.ascontiguousarray(np.transpose(u, (0, 2, 1)))
        inst.append((d, u, l))
    out = rgf_batched(inst, sym_mat=sym)
    for (d, u, l), G in zip(inst, out):
        _check(G, rgf_oracle.rgf(d, u, l, sym_mat=sym), 1e-12)
    out = rgf_batched(inst, sym_mat=sym, save_off_diag=False)
    for (d, u, l), G in zip(inst, out):
        _check(G[:1], rgf_oracle.rgf(d, u, l, sym_mat=sym)[:1], 1e-12)
        assert np.all(np.isnan(G[1])) and np.all(np.isnan(G[2]))


def test_tight_binding_energy_batch_subset():
    spec = [(e, n, b, s) for (e, n, b, s) in workloads.energy_batch_spec(count=64)][:10]
    # shrink to oracle-friendly sizes, keep the generator and energies
    inst = [workloads.tight_binding(min(n, 12), min(b, 64), e, seed=s) for (e, n, b, s) in spec]
    out = rgf_batched(inst)
    for (d, u, l), G in zip(inst, out):
        _check(G, rgf_oracle.rgf(d, u, l), 1e-11)
        _check(G[:1], dense.inv_selected(d, u, l)[:1], 1e-11)


def test_rerun_is_deterministic_and_inputs_untouched():
    import torch
    inst = [workloads.dominant(n, b, seed=7 + n) for n, b in [(5, 64), (8, 32), (3, 100)]]
    tinst = [tuple(torch.from_numpy(x).cuda() for x in t) for t in inst]
    plan = BatchPlan(tinst)
    plan.run()
    first = [tuple(g.clone() for g in G) for G in plan.results()]
    plan.run()
    plan.run()
    plan.check()
    for G0, G1 in zip(first, plan.results()):
        for a, b in zip(G0, G1):
            assert torch.equal(a, b)
    for (d, u, l), (td, tu, tl) in zip(inst, tinst):
        assert np.array_equal(td.cpu().numpy(), d)


def test_singular_instance_reported_by_index():
    inst = [workloads.dominant(n, b, seed=n) for n, b in [(3, 8), (4, 8), (3, 16), (2, 8)]]
    d, u, l = inst[2]
    d = d.copy()
    u = u.copy()
    d[1] = 0.0
    u[0] = 0.0
    inst[2] = (d, u, l)
    plan = BatchPlan(inst)
    plan.run()
    st = plan.statuses()
    assert st[2] == 1 and st[0] == 0 and st[1] == 0 and st[3] == 0
    with pytest.raises(np.linalg.LinAlgError, match="instance 2"):
        plan.check()
    good = plan.results(like=inst[0][0])
    for k in (0, 1, 3):
        _check(good[k], rgf_oracle.rgf(*inst[k]), 1e-12)


@pytest.mark.parametrize("inplace", [False, True])
def test_teams_for_large_blocks_and_in_place(inplace):
    """b = 256 / 512 instances run on teams of 2 / 4 CTAs; optionally in place."""
    import torch
    shapes = [(3, 512), (2, 256), (4, 64), (3, 256), (1, 512), (5, 32)]
    inst = [workloads.dominant(n, b, seed=200 + k) for k, (n, b) in enumerate(shapes)]
    tinst = [tuple(torch.from_numpy(x).cuda() for x in t) for t in inst]
    plan = BatchPlan(tinst, inplace=inplace)
    plan.run()
    plan.check()
    for (d, u, l), G in zip(inst, plan.results()):
        _check([g.cpu().numpy() for g in G], rgf_oracle.rgf(d, u, l), 1e-12)
    if inplace:
        assert plan.results()[0][0].data_ptr() == tinst[0][0].data_ptr()
    single = BatchPlan([tuple(torch.from_numpy(x).cuda() for x in t) for t in inst], team="cta")
    single.run()
    for G1, G2 in zip(plan.results(), single.results()):
        for a, b in zip(G1, G2):
            assert _rel(a.cpu().numpy(), b.cpu().numpy()) <= 1e-12


@pytest.mark.parametrize("wave_bytes", [6 * 2 ** 20, None])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_host_streamed_batch_matches_device_batch(precision, wave_bytes):
    """rgf_batched_host, results written over the host inputs: waves of a few
    instances (buffer reuse across waves), or (wave_bytes=None, the batch fits)
    one launch whose teams wait for each instance's copy-in flag while the
    host copies out finished instances."""
    import torch
    from sinv_b200.algorithms import rgf_batched_host
    shapes = [(3, 256), (5, 64), (2, 130), (4, 32), (3, 300), (6, 16), (2, 64)]
    inst = [workloads.tight_binding(n, b, 0.2 + 0.05 * k, seed=600 + k) for k, (n, b) in enumerate(shapes)]
    host = [tuple(torch.from_numpy(x.copy()).pin_memory() for x in t) for t in inst]
    ref = rgf_batched(inst, precision=precision)
    out = rgf_batched_host(host, outputs=host, precision=precision, wave_bytes=wave_bytes)
    assert out is host
    for (d, u, l), G, R in zip(inst, out, ref):
        for g, r in zip(G, R):
            if r.size:
                assert _rel(g.numpy(), r) <= 1e-12, _rel(g.numpy(), r)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_host_streamed_batch_with_a_schedule(precision):
    """One streamed launch with a schedule (sinvb_rgf_batched_stream_sched_*):
    teams larger than the rule's and a queue order that is not b^3 n; the
    host copies in the schedule's order (BatchPlan.queue_order) and the
    results match the device batch."""
    import torch
    from sinv_b200.algorithms import rgf_batched_host
    shapes = [(3, 256), (5, 64), (2, 130), (4, 32), (3, 300), (6, 16), (2, 64)]
    inst = [workloads.tight_binding(n, b, 0.2 + 0.05 * k, seed=650 + k) for k, (n, b) in enumerate(shapes)]
    host = [tuple(torch.from_numpy(x.copy()).pin_memory() for x in t) for t in inst]
    sched = {"team": [4, 1, 2, 1, 4, 1, 1], "priority": [float(k) for k in range(len(shapes))]}
    plan = BatchPlan([tuple(torch.from_numpy(x).cuda() for x in t) for t in inst], schedule=sched)
    assert plan.queue_order() == list(range(len(shapes)))[::-1]
    ref = rgf_batched(inst, precision=precision)
    out = rgf_batched_host(host, outputs=host, precision=precision, schedule=sched)
    for G, R in zip(out, ref):
        for g, r in zip(G, R):
            if r.size:
                assert _rel(g.numpy(), r) <= 1e-12, _rel(g.numpy(), r)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_rerun_captured_in_cuda_graph(precision):
    """BatchPlan.capture(): the re-run (memsets + persistent cooperative launch)
    as a CUDA graph; replays reproduce the eager results bit for bit and follow
    new input values."""
    import torch
    shapes = [(4, 256), (3, 64), (5, 32), (2, 300)]
    inst = [workloads.tight_binding(n, b, 0.1 * k, seed=700 + k) for k, (n, b) in enumerate(shapes)]
    tinst = [tuple(torch.from_numpy(x).cuda() for x in t) for t in inst]
    plan = BatchPlan(tinst, precision=precision)
    plan.run()
    plan.check()
    eager = [tuple(g.clone() for g in G) for G in plan.results()]
    graph = plan.capture()
    for G in plan.results():
        for g in G:
            g.zero_()
    graph.replay()
    graph.replay()
    torch.cuda.synchronize()
    plan.check()
    for G0, G1 in zip(eager, plan.results()):
        for a, b in zip(G0, G1):
            assert torch.equal(a, b)
    # new inputs in the same tensors: the replay follows them
    new = workloads.tight_binding(4, 256, 0.55, seed=777)
    for dst, src in zip(tinst[0], new):
        dst.copy_(torch.from_numpy(src))
    graph.replay()
    torch.cuda.synchronize()
    ref = rgf_batched([new], precision=precision)[0]
    for g, r in zip(plan.results()[0], ref):
        assert _rel(g.cpu().numpy(), r) <= 1e-12


def test_failed_pivots_release_their_scratch_slots():
    """More singular instances than scratch slots (one slot per concurrent
    team: 148 on a B200 for b < 256), then healthy ones.  A failed pivot must
    not keep its slot: every healthy instance gets one and finishes OK, with
    no instance timing out.  The wait bound is lowered to 5 s so a regression
    shows as SINVB_STATUS_TIMEOUT instead of minutes of waiting."""
    from sinv_b200 import _lib
    singular, healthy = 200, 40
    inst = []
    for k in range(singular + healthy):
        d, u, l = workloads.dominant(3, 16, seed=900 + k)
        if k < singular:
            d = d.copy()
            d[0] = 0.0  # the first block inverse meets a zero pivot
        inst.append((d, u, l))
    plan = BatchPlan(inst, wait_limit=5.0)
    plan.run()
    st = plan.statuses()
    assert np.all(st[:singular] == _lib.STATUS_PIVOT), np.unique(st[:singular], return_counts=True)
    assert np.all(st[singular:] == _lib.OK), np.unique(st[singular:], return_counts=True)
    res = plan.results(like=inst[0][0])
    for k in range(singular, singular + healthy, 7):
        _check(res[k], rgf_oracle.rgf(*inst[k]), 1e-12)


@pytest.mark.parametrize("shapes", [[(4, 32)] * 6, [(2, 64), (3, 256), (2, 64)]])
def test_streamed_wait_runs_out_for_a_missing_instance(shapes):
    """A streamed batch whose ready word for one instance is never written:
    that instance's bounded wait (lowered to 50 ms) runs out, it reports
    SINVB_STATUS_TIMEOUT and is skipped, the launch returns, and every other
    instance is correct.  No fault, no trap: a device wait that gives up."""
    import torch
    from sinv_b200 import _lib
    inst = [workloads.tight_binding(n, b, 0.3 + 0.1 * k, seed=950 + k) for k, (n, b) in enumerate(shapes)]
    tinst = [tuple(torch.from_numpy(x).cuda() for x in t) for t in inst]
    missing = len(inst) // 2
    count = len(inst)
    gen = 7
    ready = torch.full((count,), gen, dtype=torch.int32, device="cuda")
    ready[missing] = 0
    done = torch.zeros(count, dtype=torch.int32, device="cuda")
    plan = BatchPlan(tinst, wait_limit=0.05)
    plan.run_streamed(ready, done, gen)
    torch.cuda.synchronize()  # the launch ends although one instance never became ready
    st = plan.statuses()
    assert st[missing] == _lib.STATUS_TIMEOUT
    assert all(st[k] == _lib.OK for k in range(count) if k != missing), st
    assert torch.all(done == gen)  # the skipped instance is signalled done too
    res = plan.results()
    for k in range(count):
        if k != missing:
            _check([g.cpu().numpy() for g in res[k]], rgf_oracle.rgf(*inst[k]), 1e-11)
    # the same plan, all inputs ready, default bound: every instance is OK again
    plan.set_wait_limit(60.0)
    ready.fill_(gen + 1)
    plan.run_streamed(ready, done, gen + 1)
    plan.check()
