"""The launch-shape autotuner's host logic (dvc_b200.autotune) on the CPU:
the settings tried, the choice, the parity guard across settings, the saved
file and its application, and the workload's cross-stream reference indices.
The timing itself runs on a GPU (python -m dvc_b200.autotune)."""
import json

import numpy as np
import pytest

from dvc_b200 import autotune as at


def fake_outputs(n, seed=0, bp_seed=None):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        planes = rng.integers(0, 30, (6, 4)).astype(np.int32)
        if bp_seed is not None:  # BP work differs between settings, the rest may not
            planes[:, 3] = np.random.default_rng(bp_seed).integers(0, 1000, 6)
        out.append((rng.integers(0, 256, (4, 6), dtype=np.uint8), int(rng.integers(0, 5000)), planes))
    return out


def test_space_covers_threads_and_floors():
    s = at.space()
    assert len(s) == len(at.THREADS) * len(at.SPEC_FLOORS)
    assert {d[at.ENV_THREADS] for d in s} == {"512", "1024"}
    assert {int(d[at.ENV_FLOOR]) for d in s} == {int(x) for x in at.SPEC_FLOORS}
    assert all(set(d) == set(at.ENV_ALL) for d in s)


def test_tune_picks_fastest_median_and_restores_env():
    env = {at.ENV_FLOOR: "3"}
    speed = {"512": 1.3, "1024": 1.0}
    seen = []

    def measure(st):
        seen.append((env[at.ENV_THREADS], env[at.ENV_FLOOR]))  # the setting is in env while it runs
        k = int(st[at.ENV_FLOOR])
        base = 100.0 * speed[st[at.ENV_THREADS]] * (1.0 + abs(k - 8) / 40.0)
        return [base + 5, base, base - 1, base + 50], fake_outputs(3, bp_seed=k)

    best, results = at.tune(measure, at.space(), env)
    assert best["setting"] == dict(at.defaults(), **{at.ENV_THREADS: "1024", at.ENV_FLOOR: "8"})
    assert len(results) == len(at.space()) and len(seen) == len(results)
    assert seen[0] == ("1024", "1")
    assert env == {at.ENV_FLOOR: "3"}  # restored: the variable set before, the others removed


def test_coordinate_search_finds_each_knobs_best_value():
    """A step time with a separate best value per knob: the coordinate search
    reaches it, tries each setting once, and leaves the environment as it was."""
    want = {at.ENV_THREADS: "1024", at.ENV_THREADS_QCIF: "512", at.ENV_FLOOR: "12", at.ENV_SI: "64",
            at.ENV_FME: "512"}
    env = {}

    def measure(st):
        assert all(env[k] == v for k, v in st.items())
        t = 100.0 + sum(5.0 * (st[k] != v) + 0.0001 * int(st[k]) for k, v in want.items())
        return [t, t + 1, t - 1], fake_outputs(2, bp_seed=len(st[at.ENV_FLOOR]))

    best, results = at.tune_coordinates(measure, env=env)
    assert best["setting"] == want
    assert len(results) == 1 + sum(len(v) - 1 for _, v in at.KNOBS)
    assert env == {}


def test_tune_refuses_settings_that_decode_differently():
    calls = []

    def measure(st):
        calls.append(st)
        return [1.0], fake_outputs(2, seed=len(calls) // 2)  # the third setting decodes other frames

    with pytest.raises(RuntimeError, match="decoded differently"):
        at.tune(measure, at.space()[:4], {})


def test_save_and_apply(tmp_path):
    best = {"setting": {at.ENV_THREADS: "1024", at.ENV_FLOOR: "12", at.ENV_SI: "64"}, "ms": [3.0, 2.0, 4.0]}
    p = tmp_path / "tuning.json"
    at.save(str(p), best, [best], "test device")
    doc = json.loads(p.read_text())
    assert doc["best"] == best["setting"] and doc["median_ms"] == 3.0 and doc["device"] == "test device"
    env = {}
    got = at.apply(str(p), env)
    assert {k: v for k, v in got.items() if v is not None} == best["setting"]
    env = {at.ENV_FLOOR: "4"}  # a value the caller set wins
    got = at.apply(str(p), env)
    assert got[at.ENV_FLOOR] == "4" and got[at.ENV_THREADS] == "1024" and got[at.ENV_SI] == "64"


def test_workload_references_stay_within_each_stream():
    items = at.workload(n_streams=2, n_frames=9)
    assert len(items) == 2 * 6  # per stream: 9 frames, GOP 4 -> 6 WZ frames
    seen_ref = 0
    for i, it in enumerate(items):
        for name in ("past_from", "future_from"):
            j = it.get(name)
            if j is not None:
                seen_ref += 1
                assert 0 <= j < i and (j < 6) == (i < 6), (i, name, j)  # earlier item, same stream
                assert it[name[:-5]] is None
    assert seen_ref > 0
    assert items[0]["qindex"] == 1 and items[6]["qindex"] == 8
