"""The autotuner's host logic (no GPU): cache format, table validation, the
int8 cut-over and the makespan-driven team assignment."""

import json

import pytest

from sinv_b200 import autotune


def _table():
    # b=64: one team only; b=512: team 1 cheapest per SM, team 4 shortest chain
    return {
        "64": {"1": {"fp64": {"row_ms": 0.05, "sm_ms": 0.05}}},
        "256": {"1": {"fp64": {"row_ms": 1.0, "sm_ms": 1.0}, "int8": {"row_ms": 0.9, "sm_ms": 0.9}},
                "2": {"fp64": {"row_ms": 0.55, "sm_ms": 1.1}, "int8": {"row_ms": 0.5, "sm_ms": 1.0}}},
        "512": {"1": {"fp64": {"row_ms": 40.0, "sm_ms": 40.0}, "int8": {"row_ms": 34.0, "sm_ms": 34.0}},
                "2": {"fp64": {"row_ms": 21.0, "sm_ms": 42.0}, "int8": {"row_ms": 17.5, "sm_ms": 35.0}},
                "4": {"fp64": {"row_ms": 11.0, "sm_ms": 44.0}, "int8": {"row_ms": 9.0, "sm_ms": 36.0}}},
    }


def test_cache_round_trip(tmp_path):
    path = str(tmp_path / "tune.json")
    data = autotune.load_cache(path)
    assert data == {"format": autotune.FORMAT, "entries": {}}
    key = autotune.cache_key("NVIDIA B200", 148, 110, "mixed", 7)
    data["entries"][key] = {"table": _table(), "measured_at": 0.0, "seconds": 1.0}
    autotune.save_cache(data, path)
    again = autotune.load_cache(path)
    assert autotune.validate_table(again["entries"][key]["table"]) == _table()
    # a file of another format is ignored, not trusted
    with open(path, "w") as f:
        json.dump({"format": 999, "entries": {key: {}}}, f)
    assert autotune.load_cache(path)["entries"] == {}


@pytest.mark.parametrize("bad", [{}, {"64": {}}, {"64": {"0": {"fp64": {"row_ms": 1, "sm_ms": 1}}}},
                                 {"64": {"1": {"tf32": {"row_ms": 1, "sm_ms": 1}}}},
                                 {"64": {"1": {"fp64": {"row_ms": 0, "sm_ms": 1}}}}])
def test_validate_rejects_malformed(bad):
    with pytest.raises((ValueError, KeyError)):
        autotune.validate_table(bad)


def test_int8_cutover_is_the_smallest_winning_block_size():
    assert autotune.mixed_cutover(_table()) == 256
    t = _table()
    t["512"]["1"]["int8"]["row_ms"] = 50.0  # int8 loses at 512: no cut-over covers every larger size
    t["512"]["2"]["int8"]["row_ms"] = 50.0
    t["512"]["4"]["int8"]["row_ms"] = 50.0
    assert autotune.mixed_cutover(t) is None


def test_schedule_moves_long_chains_to_larger_teams():
    shapes = [(128, 512)] + [(16, 512)] * 30 + [(64, 64)] * 20 + [(32, 256)] * 10
    s = autotune.schedule(shapes, _table(), sms=148, precision="mixed")
    assert len(s["team"]) == len(shapes) and len(s["priority"]) == len(shapes)
    # the long b=512 chain leaves its cheapest team (1) for a shorter one
    assert s["team"][0] > 1
    # whichever candidate wins, its simulated makespan is the smallest
    assert s["candidate"] in ("fixed rule", "cheapest") or s["candidate"].startswith("greedy")
    assert s["mixed_min_b"] == 256
    # the simulated makespan is at least the work and chain bounds
    assert s["estimate_ms"] >= max(s["work_ms"], s["chain_ms"]) * (1 - 1e-12)
    # queue order: the long chain first
    assert max(range(len(shapes)), key=lambda k: s["priority"][k]) == 0


def test_schedule_fp64_has_no_cutover():
    s = autotune.schedule([(10, 256), (10, 512)], _table(), sms=148, precision="fp64")
    assert s["mixed_min_b"] == 0


def test_simulation_models_team_formation():
    # two 1-CTA instances of 10 ms then a 2-CTA instance of 5 ms on 2 SMs: 15 ms
    assert autotune.simulate([10.0, 10.0, 5.0], [1, 1, 2], [3.0, 2.0, 1.0], sms=2) == pytest.approx(15.0)
    # a 2-CTA instance waits for its second member: 10 + 5 on 2 SMs even when queued after one 1-CTA job
    assert autotune.simulate([10.0, 5.0], [1, 2], [2.0, 1.0], sms=2) == pytest.approx(15.0)
    assert autotune.simulate([4.0] * 8, [1] * 8, [1.0] * 8, sms=4) == pytest.approx(8.0)


def test_schedule_never_worse_than_fixed_rule_in_simulation():
    shapes = [(n, b) for n, b in zip(range(16, 129, 7), [512, 256, 64, 128] * 5)]
    t = _table()
    t["128"] = {"1": {"fp64": {"row_ms": 0.3, "sm_ms": 0.3}}}
    s = autotune.schedule(shapes, t, sms=16, precision="mixed")
    fixed = autotune.fixed_rule_teams(shapes, 16)

    def dur(team):
        out = []
        for (n, b), tt in zip(shapes, team):
            row = t[autotune._nearest(t, b)]
            key = str(tt) if str(tt) in row else min(row, key=lambda x: abs(int(x) - tt))
            c = row[key]
            path = "int8" if b >= s["mixed_min_b"] and "int8" in c else "fp64"
            out.append((n - 1) * c[path]["row_ms"])
        return out
    d = dur(fixed)
    assert s["estimate_ms"] <= autotune.simulate(d, fixed, d, 16) + 1e-9


def test_simulate_stream_one_instance():
    # 1 GB in at 10 GB/s (100 ms), 50 ms of sweeps, 1 GB out (100 ms)
    wall = autotune.simulate_stream([50.0], [1], [0], [1e9], 4, h2d_gbs=10.0, d2h_gbs=10.0)
    assert abs(wall - 250.0) < 1e-9


def test_simulate_stream_overlaps_copies():
    # two instances on two CTAs: the second copy-in overlaps the first sweep,
    # the first copy-out overlaps the second sweep
    wall = autotune.simulate_stream([100.0, 100.0], [1, 1], [0, 1], [1e9, 1e9], 2, h2d_gbs=10.0, d2h_gbs=10.0)
    assert abs(wall - 400.0) < 1e-9   # in 0-100, 100-200; sweeps 100-200, 200-300; out 200-300, 300-400


def test_stream_schedule_prefers_short_chains_when_copies_dominate():
    # b = 512: team 8 halves the chain at a 30 % SM-time premium; with the
    # copies in the way, the streamed choice takes the short chains while the
    # device-resident makespan choice keeps the cheaper teams
    tab = {"512": {"2": {"fp64": {"row_ms": 16.0, "sm_ms": 32.0}}, "4": {"fp64": {"row_ms": 8.5, "sm_ms": 34.0}},
                   "8": {"fp64": {"row_ms": 5.2, "sm_ms": 41.6}}},
           "64": {"1": {"fp64": {"row_ms": 0.05, "sm_ms": 0.05}}}}
    shapes = [(100, 512)] * 40 + [(60, 64)] * 200
    s = autotune.stream_schedule(shapes, tab, 148, "fp64")
    assert len(s["team"]) == len(shapes) and len(s["priority"]) == len(shapes)
    assert all(t in (1, 2, 4, 8) for t in s["team"])
    walls = {}
    for name, team in (("cheap", [2] * 40 + [1] * 200), ("short", [8] * 40 + [1] * 200)):
        d = [99 * (16.0 if t == 2 else 5.2) for t in team[:40]] + [59 * 0.05] * 200
        order = sorted(range(len(d)), key=lambda k: -d[k])
        walls[name] = autotune.simulate_stream(d, team, order, [(3 * n - 2) * b * b * 16 for n, b in shapes], 148)
    assert walls["short"] < walls["cheap"]
    assert s["estimate_ms"] <= walls["short"] + 1e-6


def test_stream_order_search_keeps_copy_out_busy():
    """Longest-first makes the first results wait for a long chain while the
    copy-out idles; the searched order is never worse, is the same on every
    call, and the schedule's priorities rank exactly that order."""
    tab = {"512": {"8": {"int8": {"row_ms": 4.6, "sm_ms": 36.8}, "fp64": {"row_ms": 6.2, "sm_ms": 49.6}}},
           "256": {"4": {"fp64": {"row_ms": 1.8, "sm_ms": 7.2}}},
           "64": {"1": {"fp64": {"row_ms": 0.17, "sm_ms": 0.17}}}}
    import numpy as np
    rng = np.random.default_rng(5)
    shapes = [(int(rng.integers(16, 129)), int(rng.choice([64, 256, 512]))) for _ in range(60)]
    in_bytes = [(3 * n - 2) * b * b * 16 for n, b in shapes]
    team = [8 if b == 512 else 4 if b == 256 else 1 for _, b in shapes]
    d = [(n - 1) * (4.6 if b == 512 else 1.8 if b == 256 else 0.17) for n, b in shapes]
    longest = sorted(range(len(d)), key=lambda k: -d[k])
    base = autotune.simulate_stream(d, team, longest, in_bytes, 148)
    o1, w1 = autotune.stream_order(d, team, in_bytes, 148, moves=300)
    o2, w2 = autotune.stream_order(d, team, in_bytes, 148, moves=300)
    assert o1 == o2 and w1 == w2 and sorted(o1) == list(range(len(d)))
    assert w1 <= base and w1 == autotune.simulate_stream(d, team, o1, in_bytes, 148)
    s = autotune.stream_schedule(shapes, tab, 148, "mixed", order_moves=300)
    order = sorted(range(len(shapes)), key=lambda k: -s["priority"][k])
    def row_ms(b, t):   # the nearest measured team, as the autotuner looks it up
        row = tab[str(b)]
        c = row[str(t) if str(t) in row else min(row, key=lambda x: abs(int(x) - t))]
        return c["int8" if (b >= s["mixed_min_b"] and "int8" in c) else "fp64"]["row_ms"]
    ds = [(n - 1) * row_ms(b, t) for (n, b), t in zip(shapes, s["team"])]
    assert abs(autotune.simulate_stream(ds, s["team"], order, in_bytes, 148) - s["estimate_ms"]) < 1e-6


def test_stream_schedule_is_remembered_for_the_same_batch(monkeypatch):
    """The same shapes on the same table: the order search runs once, and each
    call gets its own copy of the schedule."""
    tab = {"256": {"4": {"fp64": {"row_ms": 1.8, "sm_ms": 7.2}}}, "64": {"1": {"fp64": {"row_ms": 0.17, "sm_ms": 0.17}}}}
    shapes = [(20 + k, 256 if k % 3 else 64) for k in range(30)]
    calls = []
    real = autotune.stream_order

    def counting(*a, **k):
        calls.append(1)
        return real(*a, **k)

    monkeypatch.setattr(autotune, "stream_order", counting)
    autotune._stream_memo.clear()
    s1 = autotune.stream_schedule(shapes, tab, 148, "fp64", order_moves=50)
    s2 = autotune.stream_schedule(shapes, tab, 148, "fp64", order_moves=50)
    assert len(calls) == 1 and s1 == s2 and s1["team"] is not s2["team"]
    s2["team"][0] = -1
    assert autotune.stream_schedule(shapes, tab, 148, "fp64", order_moves=50)["team"][0] != -1
    autotune.stream_schedule(shapes[:-1], tab, 148, "fp64", order_moves=50)
    assert len(calls) == 2
