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
    # short b=512 instances stay on the SM-cheapest team
    assert all(t == 1 for t in s["team"][1:31])
    assert s["mixed_min_b"] == 256
    # the estimate is the larger of the work and chain bounds
    assert s["estimate_ms"] == pytest.approx(max(s["work_ms"], s["chain_ms"]))
    # queue order: the long chain first
    assert max(range(len(shapes)), key=lambda k: s["priority"][k]) == 0


def test_schedule_fp64_has_no_cutover():
    s = autotune.schedule([(10, 256), (10, 512)], _table(), sms=148, precision="fp64")
    assert s["mixed_min_b"] == 0
