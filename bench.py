#!/usr/bin/env python
"""Throughput of batched selected inversion (RGF) on B200.

Workload ("energy_batch_512"): 512 independent tight-binding instances
A_k = (E_k + i 1e-3) I - H_k - Sigma_k, E_k ~ U[-2, 2], block counts
U{16..128}, block sizes from {64, 128, 256, 512}, complex128 (169 GB of
input, 338 GB with the outputs).  That exceeds one GPU's HBM, so the batch is
processed in waves: each wave's inputs are generated on the device (untimed)
and one persistent launch inverts the whole wave (timed with CUDA events on
the launching stream).  A step is one pass over all 512 instances.  Inputs are
larger than L2 (126 MB) in every wave.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl sinvb|reference]
                    [--precision mixed|fp64] [--count 512]
                    [--workload energy_batch|plain_large|gradient_set|large_mixed|bcr_batch]

The default workload is the energy batch in mixed precision (block products
on the int8 tensor cores for b >= 256, FP64 inverses).  The other workloads:
plain_large (one n=64, b=256 matrix through the single-matrix FP64 path, and
bcr, the two-sided RGF and PSR over 3-12 partitions), gradient_set (loss and
dL/dH over 128 energies through the adjoint, forward and backward timed
apart), large_mixed (n=256, b=1024 instances in
one in-place wave, mixed vs FP64 and the error on a 4-block sub-instance) and
bcr_batch (256 small matrices through the batched BCR, beside one BCR call
per matrix and the batched FP64 RGF).  At one GPU the default energy-batch
line also carries the plain_large, gradient_set, lesser_batch and one wave of
the large_mixed results under
"other_workloads" (--no-legs leaves them out).

Metric: matrices/s of the whole batch (all ranks).  Under torchrun every rank
processes its own 512-instance batch (different Hamiltonian seeds): weak
scaling, no collective on the data path.  Rank 0 prints one JSON line.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RGF matrices/s batched+mixed vs plain FP64, same B200 @rel err≤1e-8; % TC peak"
UNIT = "matrices/s"
WORKLOAD = "energy_batch_512"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="sinvb", choices=["sinvb", "reference"])
    ap.add_argument("--workload", default="energy_batch",
                    choices=["energy_batch", "plain_large", "gradient_set", "large_mixed", "bcr_batch",
                             "lesser_batch"])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--digits", type=int, default=7, help="int8 slices per value of the mixed products")
    ap.add_argument("--count", type=int, default=0, help="instances (0: the workload's default)")
    ap.add_argument("--shape", default=None, help="n,b: uniform batch of that shape instead of the energy batch")
    ap.add_argument("--wave-gb", type=float, default=0.0, help="input GB per wave (0: as much as HBM holds)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-per-b", type=int, default=PER_B,
                    help="CPU sample: the first this many instances of each block size")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-legs", action="store_true",
                    help="energy batch only: skip the single-matrix and gradient workloads appended to its line")
    ap.add_argument("--only", default=None, choices=["rgf", "bcr", "rgf2s", "psr", "pdiv"],
                    help="plain_large: time only this algorithm (a short run for a profiler)")
    ap.add_argument("--tune", dest="tune", action="store_true", default=True,
                    help="teams, int8 cut-over and queue order from the autotuner (default)")
    ap.add_argument("--no-tune", dest="tune", action="store_false", help="the library's fixed rule instead")
    return ap.parse_args()


# --------------------------------------------------------------------------- helpers
def batch_spec(count, rank, shape=None):
    """Instances (E, n, b, seed) of this rank's batch: the energy batch, or with
    ``shape`` = (n, b) a uniform batch of that shape (small profiling cases)."""
    from sinv_b200 import workloads
    spec = workloads.energy_batch_spec(count=count)
    if shape is not None:
        spec = [(e, shape[0], shape[1], s) for (e, _, _, s) in spec]
    if rank:
        spec = [(e, n, b, s + 100000 * rank) for (e, n, b, s) in spec]
    return spec


def in_elems(n, b):
    return (3 * n - 2) * b * b


def make_waves(spec, budget_elems):
    waves, cur, used = [], [], 0
    for k, (e, n, b, s) in enumerate(spec):
        need = in_elems(n, b)
        if cur and used + need > budget_elems:
            waves.append(cur)
            cur, used = [], 0
        cur.append(k)
        used += need
    if cur:
        waves.append(cur)
    return waves


def carve(pool, spec, idx):
    """Views (diag, upper, lower) for instances idx, packed back to back in pool."""
    views, off = [], 0
    for k in idx:
        _, n, b, _ = spec[k]
        bb = b * b
        d = pool[off:off + n * bb].view(n, b, b); off += n * bb
        u = pool[off:off + (n - 1) * bb].view(n - 1, b, b); off += (n - 1) * bb
        l = pool[off:off + (n - 1) * bb].view(n - 1, b, b); off += (n - 1) * bb
        views.append((d, u, l))
    return views


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.idx = device_index
        self.proc = None
        # the raw samples of the last timed region (the line carries their summary)
        self.path = os.environ.get("SINVB_BENCH_CLOCKS", os.path.join(tempfile.gettempdir(), "sinvb_bench_clocks.csv"))

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                                          "-i", str(self.idx), "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sms, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm, smax = float(parts[1]), float(parts[2])
            except ValueError:
                continue
            mx = max(mx, smax)
            sms.append(sm)
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sms:
            return None
        loaded = [s for s in sms if s > 0.5 * mx] or sms
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sms)}


def fp64_peak_tflops(torch):
    """Measured FP64 tensor peak on this GPU: cuBLAS DGEMM 8192^3, best of 5."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    (a @ b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
        e0.record()
        a @ b
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def dmma_peak_tflops(torch):
    """Measured FP64 tensor-core (DMMA) peak of this GPU, best of 3 probe runs."""
    import ctypes
    from sinv_b200 import _lib
    lib = _lib.load()
    best = 0.0
    for _ in range(3):
        v = ctypes.c_double(0.0)
        _lib.check(lib.sinvb_fp64_mma_peak(1 << 16, ctypes.byref(v),
                                           ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)),
                   "sinvb_fp64_mma_peak")
        best = max(best, v.value)
    return best


# The CPU baseline's fixed sample: the first PER_B instances of each block
# size in the batch's order (same seeds and energies as the GPU run), 32
# instances of the 512.
PER_B = 8


def cpu_sample(spec, per_b=PER_B):
    """Stratified fixed sample of the batch: the first ``per_b`` instances of
    each block size, in batch order."""
    seen, idx = {}, []
    for k, (_, _, b, _) in enumerate(spec):
        if seen.get(b, 0) < per_b:
            seen[b] = seen.get(b, 0) + 1
            idx.append(k)
    return idx


def _cpu_env():
    """Host threads the BLAS uses, and the host's core count."""
    return {"blas_threads": _blas_threads(), "nproc": os.cpu_count() or 1,
            "OPENBLAS_NUM_THREADS": os.environ.get("OPENBLAS_NUM_THREADS", "unset")}


def _extrapolate(spec, spf_by_b):
    """Seconds for the whole batch from seconds-per-canonical-flop per block size."""
    from sinv_b200 import workloads
    return sum(workloads.rgf_flops(n, b) * spf_by_b[b] for (_, n, b, _) in spec)


def cpu_baseline(spec, reps=3, per_b=PER_B):
    """The reference RGF (numpy restatement of src/sinv/algorithms/rgf/rgf.py,
    the same numpy / OpenBLAS calls in the same order) on the host cores: the
    fixed stratified sample (two instances per block size), each timed
    ``reps`` times after one untimed warm-up, median per instance; the batch
    time is extrapolated from the median seconds per canonical flop of each
    block size (marked as extrapolated)."""
    from oracle import rgf_oracle
    from sinv_b200 import workloads
    idx = cpu_sample(spec, per_b)
    spf = {}
    timed, sampled = 0.0, []
    warm = workloads.tight_binding(*spec[idx[0]][1:3], spec[idx[0]][0], seed=spec[idx[0]][3])
    rgf_oracle.rgf(*warm)
    for k in idx:
        e, n, b, s = spec[k]
        d, u, l = workloads.tight_binding(n, b, e, seed=s)
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            rgf_oracle.rgf(d, u, l)
            ts.append(time.perf_counter() - t0)
        timed += sum(ts)
        med = statistics.median(ts)
        spf.setdefault(b, []).append(med / workloads.rgf_flops(n, b))
        sampled.append("n=%d,b=%d:%.3fs" % (n, b, med))
    spf_med = {b: statistics.median(v) for b, v in spf.items()}
    t_batch = _extrapolate(spec, spf_med)
    env = _cpu_env()
    return {"value": len(spec) / t_batch, "unit": UNIT, "cores": env["blas_threads"], "kind": "port",
            "sample": "reference rgf (numpy/OpenBLAS restatement) on a fixed stratified sample (the first %d "
                      "instances of each block size: %s), median of %d timed runs each after a warm-up; "
                      "batch time extrapolated from the median seconds per canonical flop of each block size"
                      % (per_b, ", ".join(sampled), reps),
            "extrapolated": True, "timed_seconds": timed,
            "spread_seconds_per_flop": {str(b): [min(v), max(v)] for b, v in sorted(spf.items())}, **env}


# Smallest block size whose products the mixed kernel runs on the int8 tensor
# cores (the library's cut-over; smaller blocks keep FP64 DMMA products).
MIXED_MIN_B = 256
INT8_PEAK_TOPS = 4500.0  # nominal dense int8 rate of a B200 (no measured figure on this pool)
# DRAM bytes (read + write) per canonical flop of the batched kernel, from ncu
# captures of n = 8, b = 512 batches: mixed, 74 instances on two-CTA teams
# (the autotuned schedule), 320.7 GB per launch for 5.09e12 canonical flops;
# FP64, 37 instances on four-CTA teams, 101.9 GB for 2.54e12.  The operand
# re-reads per output tile grow like b^3, as the flops do, so the launch's
# traffic is estimated as this ratio times its canonical flops.
TRAFFIC_BYTES_PER_FLOP = {"mixed": 320.7e9 / 5.085e12, "fp64": 101.9e9 / 2.54e12}


def tensor_work(spec, precision, digits, mixed_min_b=None):
    """Work the batched schedule issues per pass, by pipe: int8 tensor-core ops
    of the Ozaki products (S(S+1)/2 digit pairs, each a real (2b) x b x (2b)
    product, 2 ops per multiply-add; 6 (n-1) products per instance), and FP64
    flops on DMMA (every block inverse, b^3 complex multiply-adds, and the
    products of blocks the mixed path leaves in FP64)."""
    int8, fp64 = 0.0, 0.0
    pairs = digits * (digits + 1) // 2
    cut = MIXED_MIN_B if mixed_min_b is None else mixed_min_b
    for (_, n, b, _) in spec:
        prods = 6 * (n - 1)
        fp64 += 8.0 * n * b ** 3
        if precision == "mixed" and b >= cut:
            int8 += prods * pairs * 2.0 * (2 * b) * b * (2 * b)
        else:
            fp64 += prods * 8.0 * b ** 3
    return int8, fp64


# --------------------------------------------------------------------------- arms
def schedule_summary(sched, shapes=None, table=None):
    """The autotuner's choices for the bench line: the winning candidate, the
    teams used per block size, the int8 cut-over and the estimate, and the
    measured block-row latency (ms, GPU full) of every (block size, team,
    product path) it chose from."""
    if not sched:
        return "fixed rule (teams by block size, int8 products from b=256)"
    out = {"candidate": sched.get("candidate"), "int8_cutover_b": sched.get("int8_cutover"),
           "estimate_ms": round(sched["estimate_ms"], 1), "teams_used": sorted({int(t) for t in sched["team"]})}
    if shapes is not None and len(shapes) == len(sched["team"]):
        by_b = {}
        for (_, b), t in zip(shapes, sched["team"]):
            by_b.setdefault(str(b), set()).add(int(t))
        out["teams_by_b"] = {b: sorted(v) for b, v in sorted(by_b.items(), key=lambda kv: int(kv[0]))}
    if table:
        out["row_ms"] = {b: {t: {path: round(c["row_ms"], 3) for path, c in paths.items()}
                             for t, paths in teams.items()} for b, teams in table.items()}
    return out


def pipe_rates(spec, args, ms, dmma_peak, mixed_min_b=None):
    """Average rates of the two tensor pipes over one pass (counted work /
    device time of the pass); ``mixed_min_b``: the smallest block size whose
    products ran on the int8 pipe (the schedule's cut-over)."""
    if ms <= 0:
        return None
    int8, fp64 = tensor_work(spec, args.precision, args.digits, mixed_min_b)
    sec = ms * 1e-3
    out = {"dmma": {"tflops": fp64 / sec / 1e12, "frac_of_dmma_peak": fp64 / sec / 1e12 / dmma_peak,
                    "work": "every block inverse (b^3 complex multiply-adds) and the products left in FP64"}}
    if int8:
        out["int8"] = {"tops": int8 / sec / 1e12, "peak_tops": INT8_PEAK_TOPS,
                       "frac": int8 / sec / 1e12 / INT8_PEAK_TOPS, "peak_source": "nominal dense int8",
                       "work": "Ozaki digit-pair products, %d pairs of a (2b) x b x (2b) real product each"
                               % (args.digits * (args.digits + 1) // 2)}
    return out


def run_reference(args, rank, world):
    """CPU reference arm: the reference RGF on the host cores.  A step is one
    pass over the fixed stratified sample (the first PER_B instances of each
    block size), timed on the wall clock; ``ms_per_step`` is the median pass.
    The matrices/s of the whole batch is extrapolated from the median seconds
    per canonical flop of each block size over the timed passes."""
    if rank != 0:
        return
    from oracle import rgf_oracle
    from sinv_b200 import workloads
    shape = tuple(int(x) for x in args.shape.split(",")) if args.shape else None
    spec = batch_spec(args.count, 0, shape)
    idx = cpu_sample(spec, args.cpu_per_b)
    inst = {k: workloads.tight_binding(spec[k][1], spec[k][2], spec[k][0], seed=spec[k][3]) for k in idx}
    spf, steps_ms = {}, []
    for step in range(args.warmup + args.steps):
        t_step = 0.0
        for k in idx:
            e, n, b, s = spec[k]
            t0 = time.perf_counter()
            rgf_oracle.rgf(*inst[k])
            t = time.perf_counter() - t0
            t_step += t
            if step >= args.warmup:
                spf.setdefault(b, []).append(t / workloads.rgf_flops(n, b))
        if step >= args.warmup:
            steps_ms.append(1e3 * t_step)
    spf_med = {b: statistics.median(v) for b, v in spf.items()}
    v = len(spec) / _extrapolate(spec, spf_med)
    env = _cpu_env()
    sample = ", ".join("n=%d,b=%d" % (spec[k][1], spec[k][2]) for k in idx)
    cb = {"value": v, "unit": UNIT, "cores": env["blas_threads"], "kind": "port",
          "sample": "reference rgf (numpy/OpenBLAS restatement of rgf.py, the reference itself cannot run "
                    "without its sources) on the fixed stratified sample (the first %d instances of each block "
                    "size: %s), one pass over the sample per step, %d timed steps after %d warm-up steps; the "
                    "batch's matrices/s extrapolated from the median seconds per canonical flop of each block size"
                    % (args.cpu_per_b, sample, args.steps, args.warmup),
          "extrapolated": True,
          "spread_seconds_per_flop": {str(b): [min(x), max(x)] for b, x in sorted(spf.items())}, **env}
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": statistics.median(steps_ms),
            "ms_per_step_meaning": "median wall time of one timed step: one pass over the %d-instance sample, "
                                   "not over the batch" % len(idx),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": "synthetic", "config": {"workload": WORKLOAD, "count": args.count,
                                            "block_sizes": [64, 128, 256, 512], "n_range": [16, 128]},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_sinvb(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from sinv_b200 import workloads
    from sinv_b200.algorithms import BatchPlan, rgf

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    shape = tuple(int(x) for x in args.shape.split(",")) if args.shape else None
    spec = batch_spec(args.count, rank, shape)
    dgemm_peak = fp64_peak_tflops(torch)
    peak = dmma_peak_tflops(torch)

    tune_table = None
    if args.tune:  # measure (or load) the autotuner's table before the input pool takes HBM
        from sinv_b200 import autotune
        for prec in {args.precision, "fp64"}:
            tab = autotune.load_or_measure(sorted({b for (_, _, b, _) in spec}), prec, args.digits, dev)
            if prec == args.precision:
                tune_table = tab
        torch.cuda.empty_cache()
    free, _ = torch.cuda.mem_get_info()
    # In place (results over the inputs): the whole batch fits in HBM as one
    # wave; the per-CTA scratch slots need ~3 GB more.
    if args.wave_gb > 0:
        budget = int(args.wave_gb * 1e9 / 16)
    else:
        budget = int((free - 6e9) / 16)
    max_inst = max(in_elems(n, b) for (_, n, b, _) in spec)
    budget = max(budget, max_inst)
    waves = make_waves(spec, budget)
    pool_elems = max(sum(in_elems(spec[k][1], spec[k][2]) for k in w) for w in waves)
    pin = torch.empty(pool_elems, dtype=torch.complex128, device=dev)
    views = [carve(pin, spec, w) for w in waves]
    plans = [BatchPlan(v, precision=args.precision, inplace=True, digits=args.digits, tune=args.tune)
             for v in views]
    flops = [sum(workloads.rgf_flops(spec[k][1], spec[k][2]) for k in w) for w in waves]

    def generate(wi):
        for k, (d, u, l) in zip(waves[wi], views[wi]):
            e, n, b, s = spec[k]
            workloads.tight_binding_device(n, b, e, s, device=dev, out=(d, u, l))

    stream = torch.cuda.current_stream()
    clocks = Clocks(local_rank) if rank == 0 else None
    step_ms, kern_ms, kern_flops = [], [], []
    for step in range(args.warmup + args.steps):
        timed = step >= args.warmup
        if timed and step == args.warmup and clocks:
            clocks.start()
        total = 0.0
        for wi, plan in enumerate(plans):
            generate(wi)           # in place: every launch starts from fresh inputs (untimed)
            if world > 1:
                dist.barrier()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
            e0.record(stream)
            plan.run(stream)
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            if world > 1:
                t = torch.tensor([ms], dtype=torch.float64, device=dev)
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
                ms = float(t.item())
            total += ms
            if timed:
                kern_ms.append(ms)
                kern_flops.append(flops[wi])
        if timed:
            step_ms.append(total)
    clk = clocks.stop() if clocks else None
    for plan in plans:
        plan.check()
    ms_step = statistics.mean(step_ms)
    value = args.count * world / (ms_step * 1e-3)
    achieved = sum(kern_flops) / (sum(kern_ms) * 1e-3) / 1e12

    workload = WORKLOAD if shape is None else "uniform_%dx(n=%d,b=%d)" % (args.count, shape[0], shape[1])
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "c128" if args.precision == "fp64" else "c128 (mixed products)",
           "data": "synthetic",
           "config": {"workload": workload, "count": args.count, "block_sizes": [64, 128, 256, 512],
                      "n_range": [16, 128], "precision": args.precision, "path": "batched persistent",
                      "waves": len(waves), "wave_input_gb": round(pool_elems * 16 / 1e9, 2),
                      "in_place": True, "schedule": schedule_summary(plans[0].schedule, [(spec[k][1], spec[k][2]) for k in waves[0]],
                                                   tune_table),
                      "l2": "inputs larger than L2 in every wave", "parallelism": "replicas%d" % world},
           "gpu_launches": len(plans) * args.steps,
           "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                        "frac": achieved / peak,
                        "traffic": TRAFFIC_BYTES_PER_FLOP[args.precision] * sum(flops) / len(flops),
                        "traffic_source": "ncu dram__bytes read+write of an n=8 b=512 launch (mixed: 74 "
                                          "instances on two-CTA teams; FP64: 37 on four-CTA teams), scaled to "
                                          "this launch by canonical flops",
                        "algorithmic_bytes": sum(workloads.rgf_bytes(n, b) for (_, n, b, _) in spec) / len(flops),
                        "kernel": "rgf_batched_kernel", "flops": "canonical 8 b^3 (8(n-1)+n) per instance",
                        "frac_meaning": "FP64-equivalent: canonical flops per second over the FP64 DMMA peak; "
                                        "the tensor pipes actually used are in pipes",
                        "peak_source": "FP64 tensor-core (DMMA) rate measured at start on this GPU by "
                                       "sinvb_fp64_mma_peak (MEASURED_PEAKS.json has no FP64 figure)",
                        "peak_dgemm_cublas": dgemm_peak,
                        "pipes": pipe_rates(spec, args, sum(kern_ms) / max(1, args.steps), peak,
                                             (plans[0].schedule or {}).get("mixed_min_b"))},
           "clocks": clk}

    # the plain per-matrix FP64 path (one library call per instance, the whole
    # GPU on each matrix) over the same batch, one pass, same in-place inputs
    if not args.no_plain:
        plain_ms = plain_pass(torch, rgf, views, generate, stream)
        plain = args.count / (plain_ms * 1e-3)
        out["vs_plain_fp64"] = {"batched": value / world, "plain_per_matrix_fp64": plain,
                                "ratio": value / world / plain, "sample": "the whole batch, one pass"}
    # the batched FP64 path over the same batch, one pass (for the mixed line)
    if args.precision != "fp64":
        del plans
        plans = [BatchPlan(v, precision="fp64", inplace=True, tune=args.tune) for v in views]
        f_ms = 0.0
        for wi, plan in enumerate(plans):
            generate(wi)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
            e0.record(stream)
            plan.run(stream)
            e1.record(stream)
            e1.synchronize()
            f_ms += e0.elapsed_time(e1)
            plan.check()
        out["batched_fp64"] = {"value": args.count / (f_ms * 1e-3), "unit": UNIT,
                               "mixed_over_fp64": value / world / (args.count / (f_ms * 1e-3)),
                               "sample": "the whole batch, one pass"}

    del pin, views, plans, plan, generate   # loop variables and `generate` hold the pool too
    torch.cuda.empty_cache()
    # accuracy of this precision against the FP64 path, on a sample of the batch
    if args.precision != "fp64":
        out["rel_err_vs_fp64"] = mixed_accuracy(torch, spec, args, dev)
    # the reference's rgf run per matrix on the GPU through library calls
    # (cuBLAS products, cuSOLVER inverses), on the CPU baseline's sample
    if not args.no_plain:
        lib = library_per_block(torch, spec, dev, stream)
        lib["ratio"] = value / world / lib["matrices_per_s"]
        out["vs_library_per_block_rgf"] = lib
    # e2e on a stratified sample (every 16th instance)
    if not args.no_e2e:
        try:
            out["e2e"] = e2e_streamed(torch, spec, args, dev, world)
        except RuntimeError as err:  # pinned host memory refused
            out["e2e"] = e2e_sample(torch, spec, args, dev, world)
            out["e2e"]["streamed_unavailable"] = str(err)[:200]
    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_baseline(spec, per_b=args.cpu_per_b)
    return out


def library_rgf(torch, d, u, l):
    """The reference rgf (src/sinv/algorithms/rgf/rgf.py:40-64) with torch
    operations on the GPU: one cuSOLVER inverse and cuBLAS complex products
    per block, 8 products per block row as the reference writes them."""
    n = d.shape[0]
    inv, mm = torch.linalg.inv, torch.matmul
    g = [None] * n
    g[0] = inv(d[0])
    for i in range(1, n):
        g[i] = inv(d[i] - mm(mm(l[i - 1], g[i - 1]), u[i - 1]))
    Gd, Gu, Gl = [None] * n, [None] * (n - 1), [None] * (n - 1)
    Gd[n - 1] = g[n - 1]
    for i in range(n - 2, -1, -1):
        lf = mm(mm(Gd[i + 1], l[i]), g[i])
        Gl[i] = -lf
        Gu[i] = -mm(mm(g[i], u[i]), Gd[i + 1])
        Gd[i] = g[i] + mm(mm(g[i], u[i]), lf)
    return Gd, Gu, Gl


def library_per_block(torch, spec, dev, stream):
    """matrices/s of library_rgf over the batch: the fixed stratified sample
    (two instances per block size), one untimed call then the median of 3
    timed calls per instance (CUDA events), extrapolated to the batch by the
    median seconds per canonical flop of each block size."""
    from sinv_b200 import workloads
    spf = {}
    for k in cpu_sample(spec, per_b=2):
        e, n, b, s = spec[k]
        d, u, l = workloads.tight_binding_device(n, b, e, s, device=dev)
        library_rgf(torch, d, u, l)
        ts = [_events_ms(torch, lambda: library_rgf(torch, d, u, l), stream) for _ in range(3)]
        spf.setdefault(b, []).append(statistics.median(ts) * 1e-3 / workloads.rgf_flops(n, b))
        del d, u, l
    med = {b: statistics.median(v) for b, v in spf.items()}
    return {"matrices_per_s": len(spec) / _extrapolate(spec, med), "extrapolated": True,
            "sample": "the reference rgf with torch ops on the GPU (cuSOLVER inverse, cuBLAS products, 8 products "
                      "per block row), fixed stratified sample of 2 instances per block size, median of 3 calls each"}


def plain_pass(torch, rgf, views, generate, stream):
    """Device ms of one pass of the plain per-matrix FP64 path (one library call
    per instance, the whole GPU on each matrix) over the batch, in place on
    freshly generated inputs.  A function of its own so that no loop variable
    outlives it holding a view of the input pool."""
    plain_ms = 0.0
    for wi, wave in enumerate(views):
        generate(wi)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
        e0.record(stream)
        for (d, u, l) in wave:
            rgf.rgf_blocks(d, u, l, check=False, overwrite_a=True)
        e1.record(stream)
        e1.synchronize()
        plain_ms += e0.elapsed_time(e1)
    return plain_ms


def mixed_accuracy(torch, spec, args, dev):
    """Relative Frobenius error of the mixed path against the FP64 path, per
    output array (G_diag, G_upper, G_lower) of every 32nd instance."""
    from sinv_b200 import workloads
    from sinv_b200.algorithms import BatchPlan

    idx = list(range(0, len(spec), 32))
    inst = [workloads.tight_binding_device(spec[k][1], spec[k][2], spec[k][0], spec[k][3], device=dev)
            for k in idx]
    ref = BatchPlan(inst)
    mix = BatchPlan(inst, precision=args.precision, digits=args.digits)
    ref.run()
    mix.run()
    ref.check()
    mix.check()
    errs = []
    for G, R in zip(mix.results(), ref.results()):
        for a, r in zip(G, R):
            if r.numel():
                errs.append(float(torch.linalg.vector_norm(a - r) / torch.linalg.vector_norm(r)))
    del ref, mix, inst
    torch.cuda.empty_cache()
    return {"max": max(errs), "median": statistics.median(errs), "digits": args.digits,
            "bar": 1e-8, "sample": "every 32nd instance (%d), each of G_diag/G_upper/G_lower" % len(idx)}


def e2e_streamed(torch, spec, args, dev, world):
    """End to end over the whole batch through the public host-streamed call
    (rgf_batched_host): pinned host inputs in, results back over them, every
    host-to-device and device-to-host copy inside the timed region (they
    overlap the sweeps of other waves).  Inputs are regenerated between steps
    (untimed).  Falls back to a quarter of the batch when host memory is short."""
    import psutil
    import torch.distributed as dist
    from sinv_b200 import workloads
    from sinv_b200.algorithms import rgf_batched_host

    need = sum(in_elems(n, b) for (_, n, b, _) in spec) * 16
    idx = list(range(len(spec)))
    for stride in (2, 4, 8):  # whole batch, else every 2nd / 4th / 8th instance, as host memory allows
        if psutil.virtual_memory().available >= 1.5 * sum(in_elems(spec[k][1], spec[k][2]) for k in idx) * 16:
            break
        idx = list(range(0, len(spec), stride))
    host = []
    for k in idx:
        _, n, b, _ = spec[k]
        host.append(tuple(torch.empty((rows, b, b), dtype=torch.complex128, pin_memory=True)
                          for rows in (n, n - 1, n - 1)))

    def regen():
        for k, h in zip(idx, host):
            e, n, b, s = spec[k]
            for dst, src in zip(h, workloads.tight_binding_device(n, b, e, s, device=dev)):
                dst.copy_(src)

    sched, sched_note = None, ""
    if args.tune:  # teams and queue order for a streamed batch (the table is cached by now)
        from sinv_b200 import autotune
        shapes = [(spec[k][1], spec[k][2]) for k in idx]
        table = autotune.load_or_measure(sorted({b for _, b in shapes}), args.precision, args.digits, dev)
        sched = autotune.stream_schedule(shapes, table, torch.cuda.get_device_properties(dev).multi_processor_count,
                                         args.precision)
        by_b = {}
        for (_, b), t in zip(shapes, sched["team"]):
            by_b.setdefault(b, set()).add(int(t))
        sched_note = (", teams and queue order from autotune.stream_schedule (%s; teams by b %s; simulated %.0f ms)"
                      % (sched["candidate"], {b: sorted(v) for b, v in sorted(by_b.items())}, sched["estimate_ms"]))
    times = []
    for step in range(args.warmup + args.steps):
        regen()
        torch.cuda.empty_cache()  # the generator's temporaries (untimed)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rgf_batched_host(host, outputs=host, precision=args.precision, digits=args.digits, device=dev,
                         schedule=sched)
        t = time.perf_counter() - t0
        if world > 1:
            tt = torch.tensor([t], dtype=torch.float64, device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t = float(tt.item())
        if step >= args.warmup:
            times.append(t)
    bytes_step = sum(in_elems(spec[k][1], spec[k][2]) for k in idx) * 16
    from sinv_b200.algorithms.batched import _available_bytes
    mode = ("one launch, teams waiting for each instance's copy-in"
            if bytes_step + (8 << 30) <= _available_bytes(torch, dev) else "waves in two device buffers")
    del host
    return {"value": len(idx) * world / statistics.median(times), "unit": UNIT,
            "h2d_bytes_per_step": bytes_step, "d2h_bytes_per_step": bytes_step,
            "sample": ("the whole batch" if len(idx) == len(spec) else
                       "every %dth instance (%d)" % (len(spec) // len(idx), len(idx)))
                      + ", %.0f GB each way through pinned host memory; rgf_batched_host (%s%s) overlaps the "
                        "copies with the sweeps; wall clock around the call"
                      % (bytes_step / 1e9, mode, sched_note)}


def e2e_sample(torch, spec, args, dev, world):
    """End-to-end (pinned host buffers, copies inside the timed region) through the
    public BatchPlan API, and the plain per-matrix FP64 path on the same sample."""
    import torch.distributed as dist
    from sinv_b200 import workloads
    from sinv_b200.algorithms import BatchPlan, rgf

    idx = list(range(0, len(spec), 16))
    tot = sum(in_elems(spec[k][1], spec[k][2]) for k in idx)
    pin_dev = torch.empty(tot, dtype=torch.complex128, device=dev)
    pout_dev = torch.empty(tot, dtype=torch.complex128, device=dev)
    ins = carve(pin_dev, spec, idx)
    outs = carve(pout_dev, spec, idx)
    for k, (d, u, l) in zip(idx, ins):
        e, n, b, s = spec[k]
        workloads.tight_binding_device(n, b, e, s, device=dev, out=(d, u, l))
    host_in = torch.empty(tot, dtype=torch.complex128, pin_memory=True)
    host_out = torch.empty(tot, dtype=torch.complex128, pin_memory=True)
    host_in.copy_(pin_dev)
    plan = BatchPlan(ins, outputs=outs, precision=args.precision, digits=args.digits)
    stream = torch.cuda.current_stream()
    times = []
    for step in range(args.warmup + args.steps):
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
        e0.record(stream)
        pin_dev.copy_(host_in, non_blocking=True)
        plan.run(stream)
        host_out.copy_(pout_dev, non_blocking=True)
        e1.record(stream)
        e1.synchronize()
        if step >= args.warmup:
            times.append(e0.elapsed_time(e1))
    plan.check()
    ms = statistics.mean(times)
    # the same sample device-only, for comparison with the e2e figure
    dev_t = []
    for step in range(2):
        e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
        e0.record(stream)
        plan.run(stream)
        e1.record(stream)
        e1.synchronize()
        dev_t.append(e0.elapsed_time(e1))
    bytes_step = tot * 16
    e2e = {"value": len(idx) * world / (ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": bytes_step,
           "d2h_bytes_per_step": bytes_step,
           "sample": "every 16th instance of the batch (%d instances, %.1f GB in), pinned host buffers, "
                     "copies inside the timed region" % (len(idx), bytes_step / 1e9),
           "device_only_value_same_sample": len(idx) / (min(dev_t) * 1e-3)}
    del host_in, host_out, pin_dev, pout_dev, plan
    return e2e


# --------------------------------------------------------------------------- other workloads
def _events_ms(torch, fn, stream):
    e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
    e0.record(stream)
    fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def _max_over_ranks(torch, world, dev, ms):
    if world == 1:
        return ms
    import torch.distributed as dist
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_plain_large(args, rank, world, local_rank):
    """One matrix n=64, b=256 (diagonally dominant generator, seed 0) through the
    plain single-matrix FP64 path: rgf, and bcr on the same block arrays.  A step
    is one selected inversion; every rank inverts its own copy (replicas)."""
    import torch
    from sinv_b200 import workloads
    from sinv_b200.algorithms import bcr_s, pdiv_lm, psr_s, rgf, rgf2s
    from oracle import rgf_oracle
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    n, b = 64, 256
    psr_parts = [0, 3, 4, 8, 12]  # 0: the automatic choice
    pdiv_parts = [2, 4, 8, 16]
    dn, un, ln = workloads.dominant(n, b, seed=0)
    d, u, l = (torch.from_numpy(x).to(dev) for x in (dn, un, ln))
    peak = dmma_peak_tflops(torch)
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # 256 MB > L2
    clocks = Clocks(local_rank) if rank == 0 else None
    ts, tb, t2 = [], [], []
    tp = {P: [] for P in psr_parts}
    tq = {P: [] for P in pdiv_parts}
    if args.only:
        calls = {"rgf": lambda: rgf.rgf_blocks(d, u, l, check=False),
                 "bcr": lambda: bcr_s.bcr_blocks(d, u, l, check=False),
                 "rgf2s": lambda: rgf2s.rgf2sided(d, u, l, check=False),
                 "psr": lambda: psr_s.psr_blocks(d, u, l, partitions=4, check=False),
                 "pdiv": lambda: pdiv_lm.pdiv_blocks(d, u, l, partitions=4, check=False)}
        ts = []
        for step in range(args.warmup + args.steps):
            flush.zero_()
            m = _events_ms(torch, calls[args.only], stream)
            if step >= args.warmup:
                ts.append(m)
        return {"metric": "%s ms, one matrix n=64 b=256 (profiling run)" % args.only, "value": statistics.median(ts),
                "unit": "ms", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": statistics.median(ts), "higher_is_better": False,
                "config": {"workload": "plain_large(n=64,b=256)", "only": args.only,
                           "partitions": 4 if args.only in ("psr", "pdiv") else None}}
    for step in range(args.warmup + args.steps):
        if step == args.warmup and clocks:
            clocks.start()
        flush.zero_()
        ms = _events_ms(torch, lambda: rgf.rgf_blocks(d, u, l, check=False), stream)
        flush.zero_()
        mb = _events_ms(torch, lambda: bcr_s.bcr_blocks(d, u, l, check=False), stream)
        flush.zero_()
        m2 = _events_ms(torch, lambda: rgf2s.rgf2sided(d, u, l, check=False), stream)
        mp = {}
        for P in psr_parts:
            flush.zero_()
            mp[P] = _events_ms(torch, lambda: psr_s.psr_blocks(d, u, l, partitions=P or None, check=False), stream)
        mq = {}
        for P in pdiv_parts:
            flush.zero_()
            mq[P] = _events_ms(torch, lambda: pdiv_lm.pdiv_blocks(d, u, l, partitions=P, check=False), stream)
        if step >= args.warmup:
            for P in psr_parts:
                tp[P].append(_max_over_ranks(torch, world, dev, mp[P]))
            for P in pdiv_parts:
                tq[P].append(_max_over_ranks(torch, world, dev, mq[P]))
            ts.append(_max_over_ranks(torch, world, dev, ms))
            tb.append(_max_over_ranks(torch, world, dev, mb))
            t2.append(_max_over_ranks(torch, world, dev, m2))
    clk = clocks.stop() if clocks else None
    G = rgf.rgf_blocks(d, u, l)
    R = rgf_oracle.rgf(dn, un, ln)
    err = max(float(np.linalg.norm(g.cpu().numpy() - r) / np.linalg.norm(r)) for g, r in zip(G, R))
    ms = statistics.median(ts)
    F = workloads.rgf_flops(n, b)
    # e2e: host (pinned) inputs in, host outputs back, through the public call
    hd, hu, hl = (torch.from_numpy(x).pin_memory() for x in (dn, un, ln))
    outs = [torch.empty_like(x).pin_memory() for x in (hd, hu, hl)]   # the caller's pinned result buffers
    te = []
    for step in range(args.warmup + args.steps):
        def e2e():
            G = rgf.rgf_blocks(hd.to(dev, non_blocking=True), hu.to(dev, non_blocking=True),
                               hl.to(dev, non_blocking=True), check=False)
            for o, g in zip(outs, G):
                o.copy_(g, non_blocking=True)
            torch.cuda.current_stream().synchronize()
            return outs
        m = _events_ms(torch, e2e, stream)
        if step >= args.warmup:
            te.append(m)
    bytes_in = sum(x.nbytes for x in (dn, un, ln))
    out = {"metric": "RGF matrices/s, one matrix, plain FP64 path", "value": world / (ms * 1e-3),
           "unit": "matrices/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
           "data": "synthetic", "config": {"workload": "plain_large(n=64,b=256)", "n": n, "b": b,
                                           "generator": "diagonally dominant, seed 0",
                                           "l2": "256 MB buffer written between timed calls",
                                           "parallelism": "replicas%d" % world},
           "gpu_launches": args.steps, "rel_err_vs_oracle": err,
           "roofline": {"bound": "tensor", "achieved": F / (ms * 1e-3) / 1e12, "peak": peak, "unit": "TFLOP/s",
                        "frac": F / (ms * 1e-3) / 1e12 / peak, "traffic": None, "kernel": "rgf_grid_kernel",
                        "flops": "canonical 8 b^3 (8(n-1)+n)", "peak_source": "sinvb_fp64_mma_peak (DMMA)"},
           "bcr": {"ms": statistics.median(tb), "matrices_per_s": world / (statistics.median(tb) * 1e-3),
                   "rel_err_vs_oracle": max(float(np.linalg.norm(g.cpu().numpy() - r) / np.linalg.norm(r))
                                            for g, r in zip(bcr_s.bcr_blocks(d, u, l), R))},
           "rgf2sided": {"ms": statistics.median(t2), "matrices_per_s": world / (statistics.median(t2) * 1e-3),
                         "rel_err_vs_oracle": max(float(np.linalg.norm(g.cpu().numpy() - r) / np.linalg.norm(r))
                                                  for g, r in zip(rgf2s.rgf2sided(d, u, l), R))},
           "psr": {"partitions_auto": psr_s.partitions_for(n),
                   "ms_by_partitions": {str(P or psr_s.partitions_for(n)): statistics.median(tp[P])
                                        for P in psr_parts},
                   "rel_err_vs_oracle": max(float(np.linalg.norm(g.cpu().numpy() - r) / np.linalg.norm(r))
                                            for g, r in zip(psr_s.psr_blocks(d, u, l), R))},
           "pdiv": {"ms_by_partitions": {str(P): statistics.median(tq[P]) for P in pdiv_parts},
                    "rel_err_vs_oracle": {str(P): max(float(np.linalg.norm(g.cpu().numpy() - r) / np.linalg.norm(r))
                                                      for g, r in zip(pdiv_lm.pdiv_blocks(d, u, l, partitions=P), R))
                                          for P in pdiv_parts}},
           "clocks": clk,
           "e2e": {"value": world / (statistics.median(te) * 1e-3), "unit": "matrices/s",
                   "h2d_bytes_per_step": bytes_in, "d2h_bytes_per_step": bytes_in}}
    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"] = plain_cpu(dn, un, ln)
    return out


def run_bcr_batch(args, rank, world, local_rank):
    """A batch of small tight-binding matrices (n in [8, 64], b in {32, 64, 128})
    through the batched BCR: one launch runs phase k of every matrix's
    reduction / production schedule between the same grid barriers.  Beside it,
    on the same matrices: one single-matrix BCR call per matrix, and the
    batched FP64 RGF.  A step is one pass over the batch; every rank inverts
    its own copy (replicas)."""
    import torch
    from sinv_b200 import workloads
    from sinv_b200.algorithms import BatchPlan, BcrBatchPlan, bcr_batched, bcr_s
    from oracle import bcr_oracle
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    spec = workloads.bcr_batch_spec(args.count)
    host = [workloads.tight_binding(n, b, e, seed=s) for (e, n, b, s) in spec]
    inst = [tuple(torch.from_numpy(x).to(dev) for x in t) for t in host]
    peak = dmma_peak_tflops(torch)
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # 256 MB > L2
    plan = BcrBatchPlan(inst)
    rgfp = BatchPlan(inst)
    clocks = Clocks(local_rank) if rank == 0 else None
    tb, tr, tl = [], [], []
    for step in range(args.warmup + args.steps):
        if step == args.warmup and clocks:
            clocks.start()
        flush.zero_()
        mb = _events_ms(torch, lambda: plan.run(stream), stream)
        flush.zero_()
        mr = _events_ms(torch, lambda: rgfp.run(stream), stream)
        if step >= args.warmup:
            tb.append(_max_over_ranks(torch, world, dev, mb))
            tr.append(_max_over_ranks(torch, world, dev, mr))
    clk = clocks.stop() if clocks else None
    plan.check()
    rgfp.check()
    # one single-matrix BCR call per matrix (untimed by the clock sampler; a few steps)
    for step in range(1 + min(args.steps, 2)):
        flush.zero_()
        m = _events_ms(torch, lambda: [bcr_s.bcr_blocks(*t, check=False) for t in inst], stream)
        if step >= 1:
            tl.append(_max_over_ranks(torch, world, dev, m))
    errs = []
    for k in range(0, len(inst), max(1, len(inst) // 8)):
        G = plan.results()[k]
        R = rgfp.results()[k]
        errs.append(max(float(torch.linalg.norm(g - r) / torch.linalg.norm(r)) for g, r in zip(G, R) if r.numel()))
    ms = statistics.median(tb)
    F = sum(workloads.rgf_flops(n, b) for (_, n, b, _) in spec)
    count = len(spec)
    del plan, rgfp
    torch.cuda.empty_cache()
    # e2e: numpy inputs in, numpy results back, through the public call (schedule build and upload included)
    te = []
    bytes_in = sum(x.nbytes for t in host for x in t)
    for step in range(1 + min(args.steps, 2)):
        m = _events_ms(torch, lambda: bcr_batched(host, check=False), stream)
        if step >= 1:
            te.append(_max_over_ranks(torch, world, dev, m))
    out = {"metric": "BCR matrices/s, batch of small matrices, FP64", "value": world * count / (ms * 1e-3),
           "unit": "matrices/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
           "data": "synthetic",
           "config": {"workload": "bcr_batch(%d matrices, n 8-64, b 32/64/128)" % count, "count": count,
                      "generator": "tight-binding A(E), energies in [-2, 2], seed 5",
                      "l2": "256 MB buffer written between timed calls",
                      "parallelism": "replicas%d" % world},
           "gpu_launches": args.steps, "rel_err_vs_batched_rgf": max(errs),
           "roofline": {"bound": "tensor", "achieved": F / (ms * 1e-3) / 1e12, "peak": peak, "unit": "TFLOP/s",
                        "frac": F / (ms * 1e-3) / 1e12 / peak, "traffic": None, "kernel": "bcr_kernel",
                        "flops": "canonical RGF count 8 b^3 (8(n-1)+n) per matrix (BCR itself does more)",
                        "peak_source": "sinvb_fp64_mma_peak (DMMA)"},
           "bcr_per_matrix_calls": {"ms": statistics.median(tl),
                                    "matrices_per_s": world * count / (statistics.median(tl) * 1e-3)},
           "rgf_batched_fp64": {"ms": statistics.median(tr),
                                "matrices_per_s": world * count / (statistics.median(tr) * 1e-3)},
           "clocks": clk,
           "e2e": {"value": world * count / (statistics.median(te) * 1e-3), "unit": "matrices/s",
                   "h2d_bytes_per_step": bytes_in, "d2h_bytes_per_step": bytes_in}}
    if rank == 0 and world == 1 and not args.no_cpu:
        sample = host[:4]
        t0 = time.perf_counter()
        for d, u, l in sample:
            bcr_oracle.bcr_blocks(d, u, l)
        t = time.perf_counter() - t0
        fs = sum(workloads.rgf_flops(n, b) for (_, n, b, _) in spec[:4])
        v = (fs / t) / (F / count)
        out["cpu_baseline"] = {"value": v, "unit": "matrices/s", "cores": _blas_threads(), "kind": "port",
                               "sample": "the first 4 matrices, scaled to the batch's mean size by canonical flops"}
    return out


def plain_cpu(dn, un, ln):
    from oracle import rgf_oracle
    t0 = time.perf_counter()
    rgf_oracle.rgf(dn, un, ln)
    t = time.perf_counter() - t0
    return {"value": 1.0 / t, "unit": "matrices/s", "cores": _blas_threads(), "kind": "port",
            "sample": "the whole matrix once (reference rgf restated in numpy/OpenBLAS)"}


def _blas_threads():
    try:
        from threadpoolctl import threadpool_info
        return max([i.get("num_threads", 1) for i in threadpool_info() if i.get("user_api") == "blas"] or [1])
    except Exception:
        return os.cpu_count() or 1


def run_gradient_set(args, rank, world, local_rank):
    """Loss L = sum_k -Im Tr sum_i G_ii(E_k) / pi over 128 energies of one shared
    tight-binding H (n=32, b=128) and dL/dH by the hand-written adjoint.  A step
    evaluates the loss and the gradient over all energies; energies are split
    over ranks and one all-reduce sums the gradient (strong scaling).  Forward
    and backward device times are reported separately."""
    import torch
    from sinv_b200 import distributed, workloads
    from sinv_b200.algorithms import rgf_autograd, rgf_batched_autograd
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    energies, n, b, hseed = workloads.gradient_set_spec(count=args.count)
    onsite, coupling = workloads.hamiltonian(n, b, hseed)
    Hd = torch.from_numpy(onsite).to(dev)
    Hu = torch.from_numpy(coupling).to(dev)
    mine = distributed.shard_by_cost([1.0] * len(energies), world, rank)
    eye = torch.eye(b, dtype=torch.complex128, device=dev)
    stream = torch.cuda.current_stream()
    peak = dmma_peak_tflops(torch)

    def step():
        """Loss and dL/dH over this rank's energies: one batched forward
        launch (with adjoint checkpoints) and one batched adjoint launch."""
        from sinv_b200.distributed import _energy_matrix
        hd = Hd.clone().requires_grad_(True)
        hu = Hu.clone().requires_grad_(True)
        e0, e1, e2 = (torch.cuda.Event(True) for _ in range(3))
        e0.record(stream)
        inst = [_energy_matrix(hd, hu, energies[k], workloads.ETA, workloads.SIGMA_EDGE) for k in mine]
        out = rgf_batched_autograd(inst)
        loss = sum(-Gd.diagonal(0, 1, 2).imag.sum() / np.pi for (Gd, _, _) in out)
        e1.record(stream)
        loss.backward()
        e2.record(stream)
        e2.synchronize()
        if world > 1:
            import torch.distributed as dist
            flat = torch.cat([loss.detach().reshape(1), hd.grad.reshape(-1), hu.grad.reshape(-1)])
            dist.all_reduce(flat)
        return e0.elapsed_time(e1), e1.elapsed_time(e2)

    def sequential_pass():
        """The same energies one rgf_autograd call each (the single-instance
        adjoint), for comparison."""
        fwd = bwd = 0.0
        for k in mine:
            hd = Hd.clone().requires_grad_(True)
            hu = Hu.clone().requires_grad_(True)
            e0, e1, e2 = (torch.cuda.Event(True) for _ in range(3))
            e0.record(stream)
            from sinv_b200.distributed import _energy_matrix
            Gd, _, _ = rgf_autograd(*_energy_matrix(hd, hu, energies[k], workloads.ETA, workloads.SIGMA_EDGE))
            lk = -Gd.diagonal(0, 1, 2).imag.sum() / np.pi
            e1.record(stream)
            lk.backward()
            e2.record(stream)
            e2.synchronize()
            fwd += e0.elapsed_time(e1)
            bwd += e1.elapsed_time(e2)
        return fwd, bwd

    clocks = Clocks(local_rank) if rank == 0 else None
    fw, bw, tot = [], [], []
    for s_ in range(args.warmup + args.steps):
        if s_ == args.warmup and clocks:
            clocks.start()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
        e0.record(stream)
        f, bk = step()
        e1.record(stream)
        e1.synchronize()
        if s_ >= args.warmup:
            fw.append(f)
            bw.append(bk)
            tot.append(_max_over_ranks(torch, world, dev, e0.elapsed_time(e1)))
    clk = clocks.stop() if clocks else None
    ms = statistics.median(tot)
    f_ms, b_ms = statistics.median(fw), statistics.median(bw)
    sf, sb = sequential_pass()  # one rgf_autograd call per energy, for comparison
    F = workloads.rgf_flops(n, b) * len(mine)
    return {"metric": "energy-gradient evaluations/s (loss and dL/dH per energy)", "value": len(energies) / (ms * 1e-3),
            "unit": "energies/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"workload": "gradient_set(128 energies, n=32, b=128)", "energies": len(energies), "n": n,
                       "b": b, "parallelism": "energies sharded over %d rank(s), one all-reduce" % world},
            "gpu_launches": 2 * args.steps,
            "path": "batched forward with checkpoints + batched adjoint (one persistent launch each)",
            "forward_ms": f_ms, "backward_ms": b_ms, "backward_over_forward": b_ms / f_ms,
            "one_call_per_energy": {"forward_ms": sf, "backward_ms": sb, "batched_speedup": (sf + sb) / (f_ms + b_ms)},
            "roofline": {"bound": "tensor", "achieved": F / (f_ms * 1e-3) / 1e12, "peak": peak, "unit": "TFLOP/s",
                         "frac": F / (f_ms * 1e-3) / 1e12 / peak, "traffic": None,
                         "kernel": "batched rgf forward with checkpoints (forward only)",
                         "flops": "canonical 8 b^3 (8(n-1)+n) per energy"},
            "clocks": clk}


# DRAM bytes per energy of the batched lesser kernel at n=32, b=128 (ncu
# dram__bytes_read.sum + dram__bytes_write.sum of a 32-energy launch: 1.89 + 4.26 GB)
LESSER_TRAFFIC_PER_ENERGY = 6.145e9 / 32


def run_lesser_batch(args, rank, world, local_rank):
    """Retarded and lesser Green's functions over 128 energies of one shared
    tight-binding H (n=32, b=128), Sigma< = i f Gamma with Gamma the eta
    broadening plus the contacts: one batched call (one persistent launch)
    against one rgf_lesser call per energy, both through the public Python
    calls with inputs resident on the device.  Every rank runs its own batch
    (replicas)."""
    import torch
    from sinv_b200 import workloads
    from sinv_b200.algorithms import rgf_lesser, rgf_lesser_batched
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    energies, n, b, hseed = workloads.gradient_set_spec(count=args.count)
    H = workloads.hamiltonian(n, b, hseed)
    host = [workloads.tight_binding(n, b, e, H=H) for e in energies]
    u = torch.from_numpy(host[0][1]).to(dev)
    l = torch.from_numpy(host[0][2]).to(dev)
    inst = [(torch.from_numpy(d).to(dev), u, l) for d, _, _ in host]
    eye = np.eye(b)
    gamma = np.stack([2 * workloads.ETA * eye + (2 * workloads.SIGMA_EDGE * eye if i in (0, n - 1) else 0)
                      for i in range(n)])
    sig = torch.from_numpy((1j * 0.4 * gamma).astype(np.complex128)).to(dev)
    sigs = [sig] * len(inst)
    stream = torch.cuda.current_stream()
    clocks = Clocks(local_rank) if rank == 0 else None
    tb, ts = [], []
    for step in range(args.warmup + args.steps):
        if step == args.warmup and clocks:
            clocks.start()
        torch.cuda.synchronize()
        mb = _events_ms(torch, lambda: rgf_lesser_batched(inst, sigs), stream)
        ms = _events_ms(torch, lambda: [rgf_lesser(d, uu, ll, sig) for d, uu, ll in inst], stream)
        if step >= args.warmup:
            tb.append(_max_over_ranks(torch, world, dev, mb))
            ts.append(_max_over_ranks(torch, world, dev, ms))
    clk = clocks.stop() if clocks else None
    got = rgf_lesser_batched(inst, sigs)
    err = 0.0
    for k in range(0, len(inst), 32):
        one = rgf_lesser(*inst[k], sig)
        err = max(err, max(float(torch.linalg.norm(g - r) / torch.linalg.norm(r)) for g, r in zip(got[k], one)))
    mb, ms = statistics.median(tb), statistics.median(ts)
    count = len(inst)
    # the sweep pair's work: 16 complex b x b products per block row and one
    # block inversion (8 b^3 flops each, as the canonical RGF count)
    F = 17 * 8.0 * b ** 3 * n * count
    peak = dmma_peak_tflops(torch)
    return {"metric": "lesser Green's function evaluations/s (G and G< per energy)",
            "value": world * count / (mb * 1e-3), "unit": "energies/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": mb, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"workload": "lesser_batch(%d energies, n=%d, b=%d, shared H)" % (count, n, b),
                       "parallelism": "replicas%d" % world},
            "gpu_launches": args.steps, "path": "rgf_lesser_batched: one persistent launch",
            "one_call_per_energy": {"ms": ms, "energies_per_s": world * count / (ms * 1e-3),
                                    "batched_speedup": ms / mb},
            "rel_err_vs_single_call": err, "clocks": clk,
            "roofline": {"bound": "tensor", "achieved": F / (mb * 1e-3) / 1e12, "peak": peak, "unit": "TFLOP/s",
                         "frac": F / (mb * 1e-3) / 1e12 / peak,
                         "traffic": LESSER_TRAFFIC_PER_ENERGY * count * (n * b * b) / (32 * 128 * 128),
                         "traffic_source": "ncu dram__bytes read+write of a 32-energy n=32 b=128 launch (6.15 GB), "
                                           "per energy, scaled by n b^2",
                         "kernel": "lesser_batched_kernel",
                         "flops": "17 complex b^3 products (8 b^3 flops each) per block row and energy",
                         "peak_source": "sinvb_fp64_mma_peak (DMMA)"}}


def run_large_mixed(args, rank, world, local_rank):
    """Instances n=256, b=1024 (12.85 GB of input each), tight-binding generator,
    mixed precision: 64 instances streamed through HBM in waves (equal waves of
    at most what fits in place beside the workspace: 11 on a B200); each wave's inputs are generated on the
    device (untimed) and one persistent launch inverts the wave (timed).  A
    step is one pass over all instances.  The FP64 path runs the first wave
    once for comparison.  Error of the mixed path on a 4-block sub-instance
    (n=4, b=1024) against the FP64 path and the dense FP64 inverse."""
    import torch
    from sinv_b200 import workloads
    from sinv_b200.algorithms import BatchPlan
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    spec = workloads.large_mixed_spec(count=args.count)
    if rank:
        spec = [(e, n, b, s + 100000 * rank) for (e, n, b, s) in spec]
    peak = dmma_peak_tflops(torch)
    free, _ = torch.cuda.mem_get_info()
    per = in_elems(spec[0][1], spec[0][2])
    # headroom: the plan's workspace (scratch slots, digit planes) and the generator's temporaries
    most = max(1, min(len(spec), int((free - 16e9) / 16) // per))
    nwaves = -(-len(spec) // most)
    wave = -(-len(spec) // nwaves)  # equal waves, the last one possibly shorter
    waves = [list(range(i, min(i + wave, len(spec)))) for i in range(0, len(spec), wave)]
    pool = torch.empty(wave * per, dtype=torch.complex128, device=dev)
    views = carve(pool, [spec[0]] * wave, list(range(wave)))
    plans = {}

    def plan_for(w, precision):
        key = (len(w), precision)
        if key not in plans:
            plans.clear()  # one plan (and workspace) at a time
            torch.cuda.empty_cache()
            plans[key] = BatchPlan(views[:len(w)], precision=precision, inplace=True, digits=args.digits)
        return plans[key]

    def generate(w):
        for k, (d, u, l) in zip(w, views):
            e, n, b, s = spec[k]
            workloads.tight_binding_device(n, b, e, s, device=dev, out=(d, u, l))

    stream = torch.cuda.current_stream()
    clocks = Clocks(local_rank) if rank == 0 else None
    tm = []
    for step in range(args.warmup + args.steps):
        if step == args.warmup and clocks:
            clocks.start()
        total = 0.0
        for w in waves:
            generate(w)
            torch.cuda.synchronize()
            p = plan_for(w, "mixed")
            ms = _events_ms(torch, lambda: p.run(stream), stream)
            p.check()
            total += _max_over_ranks(torch, world, dev, ms)
        if step >= args.warmup:
            tm.append(total)
    clk = clocks.stop() if clocks else None
    plans.clear()
    p64 = BatchPlan(views[:len(waves[0])], precision="fp64", inplace=True)
    generate(waves[0])
    torch.cuda.synchronize()
    t64 = _events_ms(torch, lambda: p64.run(stream), stream)
    p64.check()
    t64_per_inst = t64 / len(waves[0])
    del p64, views, pool
    torch.cuda.empty_cache()
    # error on the 4-block sub-instance
    e, _, b, sd = spec[0]
    sub = workloads.tight_binding_device(4, b, e, sd, device=dev)
    Gm = BatchPlan([sub], precision="mixed", digits=args.digits)
    Gf = BatchPlan([sub])
    Gm.run()
    Gf.run()
    Gm.check()
    Gf.check()
    dense = torch.zeros((4 * b, 4 * b), dtype=torch.complex128, device=dev)
    d, u, l = sub
    for i in range(4):
        dense[i * b:(i + 1) * b, i * b:(i + 1) * b] = d[i]
        if i < 3:
            dense[i * b:(i + 1) * b, (i + 1) * b:(i + 2) * b] = u[i]
            dense[(i + 1) * b:(i + 2) * b, i * b:(i + 1) * b] = l[i]
    inv = torch.linalg.inv(dense)
    ref_diag = torch.stack([inv[i * b:(i + 1) * b, i * b:(i + 1) * b] for i in range(4)])

    def rel(a, r):
        return float(torch.linalg.vector_norm(a - r) / torch.linalg.vector_norm(r))

    err_fp64 = max(rel(a, r) for a, r in zip(Gm.results()[0], Gf.results()[0]) if r.numel())
    err_dense = rel(Gm.results()[0][0], ref_diag)
    ms = statistics.median(tm)
    F = sum(workloads.rgf_flops(n, b) for (_, n, b, _) in spec)
    return {"metric": "RGF matrices/s, n=256 b=1024 instances, mixed precision", "value": len(spec) * world / (ms * 1e-3),
            "unit": "matrices/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128 (mixed products)",
            "data": "synthetic",
            "config": {"workload": "large_mixed_%dx(n=256,b=1024)" % len(spec), "count": len(spec),
                       "input_gb": round(sum(in_elems(n, b) for (_, n, b, _) in spec) * 16 / 1e9, 1),
                       "waves": len(waves), "wave_instances": wave,
                       "in_place": True, "digits": args.digits, "parallelism": "replicas%d" % world},
            "gpu_launches": args.steps * len(waves),
            "fp64_first_wave": {"ms": t64, "instances": len(waves[0]), "matrices_per_s": 1e3 / t64_per_inst,
                                "mixed_over_fp64": t64_per_inst / (ms / len(spec))},
            "rel_err": {"mixed_vs_fp64_sub_instance": err_fp64, "mixed_diag_vs_dense_fp64_inverse": err_dense,
                        "sub_instance": "n=4, b=1024, first instance's generator"},
            "roofline": {"bound": "tensor", "achieved": F / (ms * 1e-3) / 1e12, "peak": peak, "unit": "TFLOP/s (FP64-equivalent)",
                         "frac": F / (ms * 1e-3) / 1e12 / peak, "traffic": None, "kernel": "rgf_batched_kernel (mixed)",
                         "flops": "canonical 8 b^3 (8(n-1)+n)", "peak_source": "sinvb_fp64_mma_peak (DMMA)"},
            "clocks": clk}


def reference_other(args, world):
    """Reference arm of the non-default workloads (rank 0, host cores)."""
    from sinv_b200 import workloads
    from oracle import rgf_oracle
    base = {"impl": "reference", "n_gpus": world, "steps": args.steps, "warmup": args.warmup}
    if args.workload == "plain_large":
        dn, un, ln = workloads.dominant(64, 256, seed=0)
        ts = []
        for _ in range(max(1, args.steps)):
            t0 = time.perf_counter()
            rgf_oracle.rgf(dn, un, ln)
            ts.append(time.perf_counter() - t0)
        v = 1.0 / statistics.median(ts)
        base.update({"metric": "RGF matrices/s, one matrix, plain FP64 path", "value": v, "unit": "matrices/s",
                     "higher_is_better": True, "config": {"workload": "plain_large(n=64,b=256)"},
                     "cpu_baseline": {"value": v, "unit": "matrices/s", "cores": _blas_threads(), "kind": "port",
                                      "sample": "the whole matrix per step"},
                     "e2e": {"value": v, "unit": "matrices/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
        return base
    if args.workload == "large_mixed":
        e, _, b, sd = workloads.large_mixed_spec(count=1)[0]
        d, u, l = workloads.tight_binding(4, b, e, seed=sd)
        t0 = time.perf_counter()
        rgf_oracle.rgf(d, u, l)
        t = (time.perf_counter() - t0) * workloads.rgf_flops(256, b) / workloads.rgf_flops(4, b)
        v = 1.0 / t
        base.update({"metric": "RGF matrices/s, n=256 b=1024 instances, mixed precision", "value": v,
                     "unit": "matrices/s", "higher_is_better": True,
                     "config": {"workload": "large_mixed(n=256,b=1024)"},
                     "cpu_baseline": {"value": v, "unit": "matrices/s", "cores": _blas_threads(), "kind": "port",
                                      "sample": "a 4-block sub-instance (n=4, b=1024) in FP64, extrapolated to "
                                                "n=256 by the canonical flop count"},
                     "e2e": {"value": v, "unit": "matrices/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
        return base
    if args.workload == "bcr_batch":
        from oracle import bcr_oracle
        spec = workloads.bcr_batch_spec(args.count)
        sample = spec[:8]
        ts = []
        for _ in range(max(1, args.steps)):
            t0 = time.perf_counter()
            for (e, n, b, sd) in sample:
                bcr_oracle.bcr_blocks(*workloads.tight_binding(n, b, e, seed=sd))
            ts.append(time.perf_counter() - t0)
        fs = sum(workloads.rgf_flops(n, b) for (_, n, b, _) in sample)
        F = sum(workloads.rgf_flops(n, b) for (_, n, b, _) in spec)
        v = (fs / statistics.median(ts)) / (F / len(spec))
        base.update({"metric": "BCR matrices/s, batch of small matrices, FP64", "value": v, "unit": "matrices/s",
                     "higher_is_better": True,
                     "config": {"workload": "bcr_batch(%d matrices, n 8-64, b 32/64/128)" % len(spec)},
                     "cpu_baseline": {"value": v, "unit": "matrices/s", "cores": _blas_threads(), "kind": "port",
                                      "sample": "the first 8 matrices per step (reference bcr_serial restated in "
                                                "numpy), scaled to the batch's mean size by canonical flops"},
                     "e2e": {"value": v, "unit": "matrices/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
        return base
    if args.workload == "lesser_batch":
        base.update({"unavailable": "the reference computes no lesser Green's function (only rgf's retarded blocks)"})
        return base
    base.update({"unavailable": "the reference computes no derivatives (no adjoint of rgf exists in it)"})
    return base


def other_workloads(args, rank, world, local_rank):
    """The single-matrix workload (one n=64, b=256 matrix: rgf, bcr, two-sided
    RGF, PSR, PDIV, errors against the oracle, e2e, CPU baseline) and the
    gradient workload (128 energies, n=32, b=128: loss and dL/dH through the
    batched adjoint), the lesser workload (the same energies' G and G< in
    one batched call) and one in-place wave (11 instances) of the large mixed
    workload (n=256, b=1024) measured after the energy batch in the same process, each
    with its own warm-up, CUDA-event timing and clock samples, so that one
    default run records them all.  A leg that fails is reported by its error;
    the energy-batch figures stand."""
    import copy
    import torch
    legs = {}
    # (workload, function, instances, timed steps, warm-up steps); the large
    # mixed workload runs one in-place wave of its n=256, b=1024 instances
    legs_spec = (("plain_large", run_plain_large, 1, 5, 3), ("gradient_set", run_gradient_set, 128, 5, 3),
                 ("lesser_batch", run_lesser_batch, 128, 5, 3), ("large_mixed", run_large_mixed, 11, 1, 1))
    for name, fn, count, steps, warmup in legs_spec:
        torch.cuda.empty_cache()
        a = copy.copy(args)
        a.workload, a.count, a.steps, a.warmup, a.only = name, count, steps, warmup, None
        try:
            legs[name] = fn(a, rank, world, local_rank)
        except Exception as err:  # noqa: BLE001 -- the headline line still prints
            legs[name] = {"error": "%s: %s" % (type(err).__name__, str(err)[:300])}
    return legs


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if not args.count:
        args.count = {"energy_batch": 512, "gradient_set": 128, "large_mixed": 64, "plain_large": 1,
                      "bcr_batch": 256, "lesser_batch": 128}[args.workload]
    if args.impl == "reference":
        if args.workload == "energy_batch":
            run_reference(args, rank, world)
        elif rank == 0:
            print(json.dumps(reference_other(args, world)), flush=True)
        return
    import datetime
    import torch
    import torch.distributed as dist
    if world > 1:
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        fn = {"energy_batch": run_sinvb, "plain_large": run_plain_large, "gradient_set": run_gradient_set,
              "large_mixed": run_large_mixed, "bcr_batch": run_bcr_batch,
              "lesser_batch": run_lesser_batch}[args.workload]
        out = fn(args, rank, world, local_rank)
        if args.workload == "energy_batch" and world == 1 and not args.shape and not args.no_legs:
            out["other_workloads"] = other_workloads(args, rank, world, local_rank)
        if rank == 0:
            print(json.dumps(out), flush=True)
    finally:
        if world > 1:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
