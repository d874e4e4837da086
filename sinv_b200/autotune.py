"""Autotuner of the batched persistent RGF: per block size, which team size
(CTAs per instance) and which product path (int8 tensor cores or FP64 DMMA)
run fastest on this GPU, measured and cached; and per batch, the team of
every instance and the queue order that minimise the estimated makespan.

The reference inverts one matrix per ``rgf`` call
(``src/sinv/algorithms/rgf/rgf.py:17-64``) and has nothing to tune; the
batched kernel walks the same 6-product sweep per block row
(``rgf.py:47-62``) on a team of CTAs, and the cost of a block row depends on
the block size, the team and the product path:

* a larger team shortens an instance's chain (each product's tiles and each
  inversion panel's column blocks are split over more CTAs) but costs more
  SM time per block row (barriers, pivot blocks inverted by every member);
* int8 products pay digit slicing and pipeline fill, which small blocks do
  not amortise.

``measure`` times uniform batches that fill the GPU (one instance per team
slot) and records, per (block size, team, path), the block-row latency with
the GPU full and the SM time per block row.  ``schedule`` turns that table
into a ``sinvb_batch_schedule``: every instance starts on its cheapest team
(least SM time per row); while the longest estimated chain exceeds the
work bound (total SM time / SMs), that instance moves to the next larger
team that shortens it; instances are queued longest first.  The int8
cut-over is the smallest block size whose int8 rows beat its FP64 rows.

The GEMM tile shape follows the block size (32 x 32 tiles for b <= 32,
64 x 64 above: one tile column per 64-wide inversion panel), so it is not a
free knob here.

Cache: JSON at ``$SINVB_TUNE_CACHE`` (default
``~/.cache/sinv_b200/autotune.json``), keyed by device name, SM count,
library version, precision and digits.
"""

import json
import os
import time

TEAMS = (1, 2, 4, 8)
FORMAT = 1


def cache_path():
    return os.environ.get("SINVB_TUNE_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "sinv_b200",
                                                              "autotune.json")


def cache_key(device_name, sms, version, precision, digits):
    return "%s|sm%d|v%d|%s|d%d" % (device_name, sms, version, precision, digits if precision == "mixed" else 0)


def load_cache(path=None):
    path = path or cache_path()
    try:
        with open(path) as f:
            data = json.load(f)
        if data.get("format") != FORMAT:
            return {"format": FORMAT, "entries": {}}
        return data
    except (OSError, ValueError):
        return {"format": FORMAT, "entries": {}}


def save_cache(data, path=None):
    path = path or cache_path()
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def validate_table(table):
    """A measured table: {"b": {"<team>": {"fp64": {...}, "int8": {...}}}} with
    row_ms and sm_ms per entry.  Raises ValueError when malformed."""
    if not isinstance(table, dict) or not table:
        raise ValueError("empty table")
    for b, teams in table.items():
        int(b)
        if not isinstance(teams, dict) or not teams:
            raise ValueError("block size %s has no teams" % b)
        for t, paths in teams.items():
            if int(t) < 1:
                raise ValueError("team %s" % t)
            for path, v in paths.items():
                if path not in ("fp64", "int8"):
                    raise ValueError("path %s" % path)
                if not (v["row_ms"] > 0 and v["sm_ms"] > 0):
                    raise ValueError("costs of b=%s team=%s %s" % (b, t, path))
    return table


def _rows(b):
    return 12 if b >= 512 else 16 if b >= 256 else 24


def measure(block_sizes, precision="mixed", digits=7, device=None, teams=TEAMS, int8_from=128, log=None):
    """Measure the block-row costs of every (block size, team, path) on the GPU.

    For each combination a uniform tight-binding batch of grid / team
    instances (n = 12..24 blocks) runs once untimed and once timed (CUDA
    events); row_ms = time / n (a block row of one instance with the GPU
    full), sm_ms = row_ms * team."""
    import torch

    from . import _lib, workloads
    from .algorithms import BatchPlan

    device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    table = {}
    for b in sorted(block_sizes):
        n = _rows(b)
        table[str(b)] = {}
        for t in teams:
            if t > 1 and t > max(1, b // 64):
                continue  # more CTAs than 64-wide column blocks: no work for the extra members
            count = max(1, sms // t)
            paths = ["fp64"]
            if precision == "mixed" and b >= int8_from:
                paths.append("int8")
            entry = {}
            for path in paths:
                inst = [workloads.tight_binding_device(n, b, 0.3 + 0.01 * k, 5000 + k, device=device)
                        for k in range(count)]
                # in a mixed batch FP64-product instances run in the mixed kernel:
                # measure them there (int8 cut-over above b)
                sched = {"team": [t] * count, "mixed_min_b": (b if path == "int8" else b + 1)}
                plan = BatchPlan(inst, precision=precision, inplace=True, digits=digits, schedule=sched)
                plan.run()
                torch.cuda.synchronize(device)
                plan.check()
                for k, (d, u, l) in enumerate(inst):
                    workloads.tight_binding_device(n, b, 0.3 + 0.01 * k, 5000 + k, device=device, out=(d, u, l))
                e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
                e0.record()
                plan.run()
                e1.record()
                e1.synchronize()
                plan.check()
                ms = e0.elapsed_time(e1)
                entry[path] = {"row_ms": ms / n, "sm_ms": ms / n * t, "count": count, "n": n}
                if log:
                    log("tune b=%d team=%d %s: %.3f ms/row, %.2f SM-ms/row" % (b, t, path, ms / n, ms / n * t))
                del plan, inst
                torch.cuda.empty_cache()
            table[str(b)][str(t)] = entry
    _ = _lib  # the library is loaded by BatchPlan
    return validate_table(table)


def load_or_measure(block_sizes, precision="mixed", digits=7, device=None, path=None, log=None):
    """The cached table for this GPU / library / precision, measuring the
    block sizes it lacks."""
    import torch

    from . import _lib

    device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    props = torch.cuda.get_device_properties(device)
    key = cache_key(props.name, props.multi_processor_count, int(_lib.load().sinvb_version()), precision, digits)
    data = load_cache(path)
    table = dict(data["entries"].get(key, {}).get("table", {}))
    missing = [b for b in block_sizes if str(b) not in table]
    if missing:
        t0 = time.time()
        table.update(measure(missing, precision, digits, device, log=log))
        data["entries"][key] = {"table": table, "measured_at": time.time(), "seconds": time.time() - t0}
        save_cache(data, path)
    return validate_table(table)


def _best_path(costs):
    """(path, costs) of the cheaper product path of one team entry."""
    return min(costs.items(), key=lambda kv: kv[1]["row_ms"])


def mixed_cutover(table):
    """Smallest block size whose int8 rows beat its FP64 rows on its cheapest team."""
    best = None
    for b in sorted(table, key=int):
        teams = table[b]
        t = min(teams, key=lambda t: _best_path(teams[t])[1]["sm_ms"])
        paths = teams[t]
        if "int8" in paths and paths["int8"]["row_ms"] < paths["fp64"]["row_ms"]:
            best = int(b) if best is None else best
        elif best is not None:
            best = None  # int8 must win for every larger block size too
    return best


def _nearest(table, b):
    keys = sorted(int(x) for x in table)
    return str(min(keys, key=lambda x: (abs(x - b), x)))


def simulate(durations, teams, priority, sms):
    """Makespan (ms) of the persistent kernel's queue for given per-instance
    durations (ms with its team), teams and priorities: instances in
    descending priority, their member slots handed out in order to whichever
    CTA is free first; an instance starts when its last member has arrived
    (members that arrive early wait) and holds all its members until it
    ends."""
    import heapq
    order = sorted(range(len(durations)), key=lambda k: -priority[k])
    free = [(0.0, c) for c in range(sms)]
    heapq.heapify(free)
    end = 0.0
    for k in order:
        members = [heapq.heappop(free) for _ in range(min(teams[k], sms))]
        start = max(t for t, _ in members)
        finish = start + durations[k]
        end = max(end, finish)
        for _, c in members:
            heapq.heappush(free, (finish, c))
    return end


def fixed_rule_teams(shapes, sms):
    """The library's own team rule (sinvb_rgf_batched_* without a schedule)."""
    t = [8 if b >= 1024 else 4 if b >= 512 else 2 if b >= 256 else 1 for _, b in shapes]
    if sum(t) < sms:
        share = sms // len(shapes)
        t = [max(x, min(share, b // 64, 16)) if b >= 256 else x for x, (_, b) in zip(t, shapes)]
    return t


def schedule(shapes, table, sms, precision="mixed"):
    """Teams, queue priorities (estimated ms) and the int8 cut-over for a batch
    of (n, b) shapes, from a measured table (``measure``).

    Candidates: the library's fixed rule, every instance on its SM-cheapest
    team, and the greedy assignment that moves the longest estimated chain to
    a larger team while it exceeds a fraction of the work bound (several
    fractions); the candidate with the smallest simulated makespan
    (``simulate``) wins.  Returns {"team": [...], "priority": [...],
    "mixed_min_b": int, "int8_cutover": b or None, "estimate_ms": float,
    "work_ms": float, "chain_ms": float, "candidate": str}."""
    cut = mixed_cutover(table) if precision == "mixed" else None
    mixed_min_b = cut if cut is not None else 1 << 30

    def costs(b, t):
        row = table[_nearest(table, b)]
        key = str(t) if str(t) in row else min(row, key=lambda x: abs(int(x) - t))
        c = row[key]
        path = "int8" if (precision == "mixed" and b >= mixed_min_b and "int8" in c) else "fp64"
        return c[path]

    rows = [(n - 1) if n > 1 else 1 for n, _ in shapes]

    def durations(team):
        return [r * costs(b, t)["row_ms"] for r, (_, b), t in zip(rows, shapes, team)]

    def work(team):
        return sum(r * costs(b, t)["sm_ms"] for r, (_, b), t in zip(rows, shapes, team)) / sms

    choices = []
    for n, b in shapes:
        row = table[_nearest(table, b)]
        choices.append(sorted(t for t in (int(x) for x in row) if t <= sms))
    cheapest = [min(ts, key=lambda t: costs(b, t)["sm_ms"]) for ts, (_, b) in zip(choices, shapes)]

    def greedy(frac):
        team = list(cheapest)
        for _ in range(4 * len(shapes)):
            d = durations(team)
            k = max(range(len(shapes)), key=lambda i: d[i])
            if d[k] <= frac * work(team):
                break
            b = shapes[k][1]
            bigger = [t for t in choices[k] if t > team[k] and costs(b, t)["row_ms"] < costs(b, team[k])["row_ms"]]
            if not bigger:
                break
            team[k] = min(bigger)
        return team

    cands = {"fixed rule": fixed_rule_teams(shapes, sms), "cheapest": cheapest}
    for frac in (0.5, 0.7, 0.85, 1.0):
        cands["greedy %.2f" % frac] = greedy(frac)
    best = None
    for name, team in cands.items():
        d = durations(team)
        span = simulate(d, team, d, sms)
        if best is None or span < best[0]:
            best = (span, name, team, d)
    span, name, team, durs = best
    never = 1 << 30  # int8 products for no block size
    return {"team": team, "priority": durs,
            "mixed_min_b": (int(cut) if cut is not None else never) if precision == "mixed" else 0,
            "int8_cutover": cut, "estimate_ms": span, "work_ms": work(team), "chain_ms": max(durs),
            "candidate": name}


def simulate_stream(durations, teams, order, in_bytes, sms, h2d_gbs=55.0, d2h_gbs=55.0):
    """Wall time (ms) of a host-streamed batch (rgf_batched_host, one launch):
    inputs copied in queue order at ``h2d_gbs``; an instance starts when its
    inputs have arrived and its team's members are free (members handed to
    the first free CTAs, as ``simulate``); results copied out one after
    another at ``d2h_gbs`` in the order instances finish.  ``in_bytes``: the
    input (= output) bytes of each instance."""
    import heapq
    free = [(0.0, c) for c in range(sms)]
    heapq.heapify(free)
    arrive, t = {}, 0.0
    for k in order:
        t += in_bytes[k] / (h2d_gbs * 1e6)
        arrive[k] = t
    finish = []
    for k in order:
        members = [heapq.heappop(free) for _ in range(min(teams[k], sms))]
        start = max([arrive[k]] + [f for f, _ in members])
        end = start + durations[k]
        finish.append((end, k))
        for _, c in members:
            heapq.heappush(free, (end, c))
    out = 0.0
    for end, k in sorted(finish):
        out = max(out, end) + in_bytes[k] / (d2h_gbs * 1e6)
    return out


_stream_memo = {}


def stream_schedule(shapes, table, sms, precision="mixed", elem_bytes=16, h2d_gbs=55.0, d2h_gbs=55.0,
                    order_moves=1000):
    """``_stream_schedule``, remembered for the last few distinct arguments:
    an energy loop that streams batches of the same shapes on the same table
    pays for the order search once.  Returns a fresh copy of the schedule."""
    key = (tuple((int(n), int(b)) for n, b in shapes), json.dumps(table, sort_keys=True), int(sms), precision,
           int(elem_bytes), float(h2d_gbs), float(d2h_gbs), int(order_moves))
    if key not in _stream_memo:
        if len(_stream_memo) >= 8:
            _stream_memo.pop(next(iter(_stream_memo)))
        _stream_memo[key] = _stream_schedule(shapes, table, sms, precision, elem_bytes, h2d_gbs, d2h_gbs, order_moves)
    out = _stream_memo[key]
    return {k: (list(v) if isinstance(v, list) else v) for k, v in out.items()}


def _stream_schedule(shapes, table, sms, precision="mixed", elem_bytes=16, h2d_gbs=55.0, d2h_gbs=55.0,
                     order_moves=1000):
    """Teams and queue order for a host-streamed batch: the candidates of
    ``schedule`` plus every instance on its fastest team (shortest chain) and
    that for the largest block size only, each queued longest first, compared
    by ``simulate_stream`` (copy-in, sweeps and copy-out overlapped).  Copies
    make late finishers expensive: an instance that ends after the last input
    has arrived still has its results to copy out, so shorter chains can win
    over the device-resident makespan choice.  The winner's copy / queue order
    then comes from ``stream_order`` (``order_moves`` local-search moves; its
    priorities rank that order).  Returns the ``schedule`` dict with
    "estimate_ms" the simulated wall time."""
    base = schedule(shapes, table, sms, precision)
    mixed_min_b = base["mixed_min_b"]

    def costs(b, t):
        row = table[_nearest(table, b)]
        key = str(t) if str(t) in row else min(row, key=lambda x: abs(int(x) - t))
        c = row[key]
        path = "int8" if (precision == "mixed" and b >= mixed_min_b and "int8" in c) else "fp64"
        return c[path]

    rows = [(n - 1) if n > 1 else 1 for n, _ in shapes]
    in_bytes = [(3 * n - 2) * b * b * elem_bytes for n, b in shapes]
    choices = [sorted(t for t in (int(x) for x in table[_nearest(table, b)]) if t <= sms) for _, b in shapes]
    fastest = [min(ts, key=lambda t: costs(b, t)["row_ms"]) for ts, (_, b) in zip(choices, shapes)]
    bmax = max(b for _, b in shapes)
    bases = {"tuned " + base["candidate"]: base["team"], "fixed rule": fixed_rule_teams(shapes, sms)}
    cands = dict(bases)
    cands["fastest"] = fastest
    for name, team in bases.items():
        cands[name + ", fastest for b=%d" % bmax] = [f if b == bmax else t
                                                     for f, t, (_, b) in zip(fastest, team, shapes)]
    best = None
    for name, team in cands.items():
        d = [r * costs(b, t)["row_ms"] for r, (_, b), t in zip(rows, shapes, team)]
        order = sorted(range(len(shapes)), key=lambda k: -d[k])
        wall = simulate_stream(d, team, order, in_bytes, sms, h2d_gbs, d2h_gbs)
        if best is None or wall < best[0]:
            best = (wall, name, team, d)
    wall, name, team, d = best
    # the order: longest first makes the first results wait for a long chain
    # while copy-out idles; search for one that keeps the copy-out busy
    order, searched = stream_order(d, team, in_bytes, sms, h2d_gbs, d2h_gbs, moves=order_moves)
    if searched < wall:
        wall, name = searched, name + ", order searched"
        prio = [0.0] * len(shapes)
        for pos, k in enumerate(order):
            prio[k] = float(len(shapes) - pos)
    else:
        prio = d
    out = dict(base)
    out.update({"team": team, "priority": prio, "estimate_ms": wall, "candidate": name, "chain_ms": max(d)})
    return out


def stream_order(durations, teams, in_bytes, sms, h2d_gbs=55.0, d2h_gbs=55.0, moves=1000, seed=0):
    """Copy-in (= queue) order of a host-streamed batch, by local search on
    ``simulate_stream``: start from the better of longest chain first and
    most bytes per chain-ms first, then ``moves`` times move one instance to
    another position and keep the move unless the simulated wall time grows
    (fixed seed: the same inputs give the same order).  About 1.5 ms of host
    time per move for 256 instances.  Returns (order, wall_ms)."""
    import random
    count = len(durations)
    starts = [sorted(range(count), key=lambda k: -durations[k]),
              sorted(range(count), key=lambda k: -in_bytes[k] / max(durations[k], 1e-9))]
    walls = [simulate_stream(durations, teams, o, in_bytes, sms, h2d_gbs, d2h_gbs) for o in starts]
    cur, best = (starts[0], walls[0]) if walls[0] <= walls[1] else (starts[1], walls[1])
    cur = list(cur)
    rnd = random.Random(seed)
    for _ in range(moves if count > 1 else 0):
        i, j = rnd.randrange(count), rnd.randrange(count)
        if i == j:
            continue
        cur.insert(j, cur.pop(i))
        v = simulate_stream(durations, teams, cur, in_bytes, sms, h2d_gbs, d2h_gbs)
        if v <= best:
            best = v
        else:
            cur.insert(i, cur.pop(j))
    return cur, best
