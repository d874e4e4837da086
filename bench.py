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
                    [--precision fp64|mixed] [--count 512]

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
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--digits", type=int, default=7, help="int8 slices per value of the mixed products")
    ap.add_argument("--count", type=int, default=512)
    ap.add_argument("--shape", default=None, help="n,b: uniform batch of that shape instead of the energy batch")
    ap.add_argument("--wave-gb", type=float, default=0.0, help="input GB per wave (0: as much as HBM holds)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
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
        self.path = os.path.join(ROOT, "gpurun_out", "bench_clocks.csv") if os.path.isdir(
            os.path.join(ROOT, "gpurun_out")) else "/tmp/sinvb_bench_clocks.csv"

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


def cpu_sample(spec):
    """Stratified CPU sample: the first instance of each block size."""
    seen, idx = set(), []
    for k, (_, _, b, _) in enumerate(spec):
        if b not in seen:
            seen.add(b)
            idx.append(k)
    return idx


def cpu_baseline(spec, reps=1):
    """The reference RGF (numpy restatement of src/sinv/algorithms/rgf/rgf.py) on host
    cores, on one instance per block size; extrapolated to the whole batch by the
    canonical flop count per block-size class."""
    from oracle import rgf_oracle
    from sinv_b200 import workloads
    try:
        from threadpoolctl import threadpool_info
        cores = max([i.get("num_threads", 1) for i in threadpool_info() if i.get("user_api") == "blas"] or [1])
    except Exception:
        cores = os.cpu_count() or 1
    spf, sampled = {}, []
    t_total = 0.0
    for k in cpu_sample(spec):
        e, n, b, s = spec[k]
        d, u, l = workloads.tight_binding(n, b, e, seed=s)
        best = 1e30
        for _ in range(reps):
            t0 = time.perf_counter()
            rgf_oracle.rgf(d, u, l)
            best = min(best, time.perf_counter() - t0)
        t_total += best
        spf[b] = best / workloads.rgf_flops(n, b)
        sampled.append("n=%d,b=%d:%.2fs" % (n, b, best))
    t_batch = sum(workloads.rgf_flops(n, b) * spf[b] for (_, n, b, _) in spec)
    return {"value": len(spec) / t_batch, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": "reference rgf (numpy/OpenBLAS restatement) on one instance per block size [%s], "
                      "extrapolated to the %d-instance batch by the canonical flop count per block size"
                      % (", ".join(sampled), len(spec)),
            "sample_seconds": t_total}


# --------------------------------------------------------------------------- arms
def run_reference(args, rank, world):
    if rank != 0:
        return
    shape = tuple(int(x) for x in args.shape.split(",")) if args.shape else None
    spec = batch_spec(args.count, 0, shape)
    vals = []
    for step in range(args.warmup + args.steps):
        cb = cpu_baseline(spec)
        if step >= args.warmup:
            vals.append(cb["value"])
    v = statistics.median(vals)
    cb["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * args.count / v,
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
    plans = []
    for w in waves:
        plans.append(BatchPlan(carve(pin, spec, w), precision=args.precision, inplace=True,
                               digits=args.digits))
    flops = [sum(workloads.rgf_flops(spec[k][1], spec[k][2]) for k in w) for w in waves]

    def generate(wi):
        for k, (d, u, l) in zip(waves[wi], plans[wi].inputs):
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
                      "in_place": True,
                      "l2": "inputs larger than L2 in every wave", "parallelism": "replicas%d" % world},
           "gpu_launches": len(plans) * args.steps,
           "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                        "frac": achieved / peak, "traffic": None,
                        "kernel": "rgf_batched_kernel", "flops": "canonical 8 b^3 (8(n-1)+n) per instance",
                        "peak_source": "FP64 tensor-core (DMMA) rate measured at start on this GPU by "
                                       "sinvb_fp64_mma_peak (MEASURED_PEAKS.json has no FP64 figure)",
                        "peak_dgemm_cublas": dgemm_peak},
           "clocks": clk}

    # the plain per-matrix FP64 path (one library call per instance, the whole
    # GPU on each matrix) over the same batch, one pass, same in-place inputs
    if not args.no_plain:
        plain_ms = plain_pass(torch, rgf, plans, generate, stream)
        plain = args.count / (plain_ms * 1e-3)
        out["vs_plain_fp64"] = {"batched": value / world, "plain_per_matrix_fp64": plain,
                                "ratio": value / world / plain, "sample": "the whole batch, one pass"}

    del pin, plans, plan, generate   # `plan` (loop variable) and `generate` hold the pool too
    torch.cuda.empty_cache()
    # accuracy of this precision against the FP64 path, on a sample of the batch
    if args.precision != "fp64":
        out["rel_err_vs_fp64"] = mixed_accuracy(torch, spec, args, dev)
    # e2e on a stratified sample (every 16th instance)
    if not args.no_e2e:
        out["e2e"] = e2e_sample(torch, spec, args, dev, world)
    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_baseline(spec)
    return out


def plain_pass(torch, rgf, plans, generate, stream):
    """Device ms of one pass of the plain per-matrix FP64 path (one library call
    per instance, the whole GPU on each matrix) over the batch, in place on
    freshly generated inputs.  A function of its own so that no loop variable
    outlives it holding a view of the input pool."""
    plain_ms = 0.0
    for wi, plan in enumerate(plans):
        generate(wi)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
        e0.record(stream)
        for (d, u, l) in plan.inputs:
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


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import datetime
    import torch
    import torch.distributed as dist
    if world > 1:
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        out = run_sinvb(args, rank, world, local_rank)
        if rank == 0:
            print(json.dumps(out), flush=True)
    finally:
        if world > 1:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
