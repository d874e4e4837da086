"""The autotuner on the GPU: measured tables, and tuned batches against the
oracle restatement of the reference rgf (``src/sinv/algorithms/rgf/rgf.py:17-64``)
and against the library's fixed rule.

Tolerances as in the other batched tests: 1e-12 (dominant, FP64), 1e-9
(dominant, mixed).  A tuned plan may not be slower than the fixed rule by
more than timing noise (25 %, best of three) on a small mixed batch."""

import numpy as np
import pytest

from oracle import dense, rgf_oracle
from sinv_b200 import autotune, workloads
from sinv_b200.algorithms import BatchPlan

pytestmark = pytest.mark.gpu


def _worst(G, R):
    return max(dense.rel_fro(np.asarray(x), np.asarray(r)) for x, r in zip(G, R) if np.asarray(r).size)


@pytest.fixture(scope="module")
def tune_cache(tmp_path_factory):
    import os
    path = str(tmp_path_factory.mktemp("tune") / "autotune.json")
    old = os.environ.get("SINVB_TUNE_CACHE")
    os.environ["SINVB_TUNE_CACHE"] = path
    yield path
    if old is None:
        os.environ.pop("SINVB_TUNE_CACHE")
    else:
        os.environ["SINVB_TUNE_CACHE"] = old


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tuned_batch_matches_oracle(tune_cache, precision):
    import torch
    shapes = [(3, 256), (6, 64), (2, 300), (5, 32), (4, 128), (1, 256)]
    inst = [workloads.dominant(n, b, seed=1200 + k) for k, (n, b) in enumerate(shapes)]
    tinst = [tuple(torch.from_numpy(x).cuda() for x in t) for t in inst]
    plan = BatchPlan(tinst, precision=precision, tune=True)
    assert plan.schedule is not None and len(plan.schedule["team"]) == len(shapes)
    plan.run()
    plan.check()
    tol = 1e-12 if precision == "fp64" else 1e-9
    for (d, u, l), G in zip(inst, plan.results()):
        assert _worst([g.cpu().numpy() for g in G], rgf_oracle.rgf(d, u, l)) <= tol
    table = autotune.load_or_measure([64, 256], precision, 7)
    assert set(table) >= {"64", "256"}


def _best_ms(plan, reps=3):
    import torch
    best = 1e30
    plan.run()
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
        e0.record()
        plan.run()
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    plan.check()
    return best


def test_tuned_batch_not_slower_than_fixed_rule(tune_cache):
    import torch
    spec = [(e, min(n, 24), b, s) for (e, n, b, s) in workloads.energy_batch_spec(count=160) if b <= 256]
    inst = [workloads.tight_binding_device(n, b, e, s, device="cuda") for (e, n, b, s) in spec]
    fixed = BatchPlan(inst, precision="mixed")
    tuned = BatchPlan(inst, precision="mixed", tune=True)
    t_fixed = _best_ms(fixed)
    t_tuned = _best_ms(tuned)
    assert t_tuned <= 1.25 * t_fixed, (t_tuned, t_fixed, tuned.schedule["mixed_min_b"])
    for G, R in zip(tuned.results()[:8], fixed.results()[:8]):
        for a, r in zip(G, R):
            assert (torch.linalg.vector_norm(a - r) / torch.linalg.vector_norm(r)).item() <= 1e-8
