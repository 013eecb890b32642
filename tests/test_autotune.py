"""Host logic of the autotuner (no GPU): the constrained pick of the
operating point, the tuned-file loader, and the committed tuned point that
bench.py reads."""
import json

from fastrrt_b200 import autotune


def _trial(slots, pps, succ):
    return {"slots": slots, "check_every": 2, "mix": 1.0, "plans_per_s": pps, "success_rate": succ}


def test_pick_takes_the_fastest_trial_that_meets_the_success_bar():
    trials = [_trial(256, 9000.0, 0.99), _trial(512, 15000.0, 0.975), _trial(1024, 20000.0, 0.95)]
    best = autotune.pick(trials, 0.969)
    # the 1024-slot trial is faster but below the bar
    assert best["slots"] == 512
    assert autotune.pick(trials, 0.98)["slots"] == 256
    # the bar is inclusive
    assert autotune.pick([_trial(768, 1.0, 0.969)], 0.969)["slots"] == 768


def test_pick_returns_none_when_no_trial_meets_the_bar():
    assert autotune.pick([_trial(256, 9000.0, 0.90)], 0.969) is None
    assert autotune.pick([], 0.969) is None


def test_load_reads_best_and_tolerates_missing_or_broken_files(tmp_path):
    assert autotune.load(str(tmp_path / "absent.json")) is None
    broken = tmp_path / "broken.json"
    broken.write_text("{not json")
    assert autotune.load(str(broken)) is None
    nobest = tmp_path / "nobest.json"
    nobest.write_text(json.dumps({"trials": []}))
    assert autotune.load(str(nobest)) is None
    good = tmp_path / "good.json"
    good.write_text(json.dumps({"best": {"slots": 640}}))
    assert autotune.load(str(good)) == {"slots": 640}


def test_committed_operating_point_is_complete_and_meets_the_bar():
    """the file bench.py reads: every key it uses, values inside the grids
    the tuner searched, and the success bar the pick enforced"""
    with open(autotune.DEFAULT_OUT) as f:
        tuned = json.load(f)
    best = tuned["best"]
    for key in ("slots", "check_every", "mix", "sweep_blocks_per_sm", "work_blocks_per_sm",
                "serving_check_every", "c2_launch"):
        assert key in best, key
    assert best["slots"] in autotune.GRID["slots"]
    assert best["check_every"] in autotune.GRID["check_every"]
    assert best["mix"] in autotune.GRID["mix"]
    assert best["serving_check_every"] in autotune.SERVING["check_every"]
    assert best["c2_launch"]["sweep_blocks_per_sm"] in autotune.C2_GRID["sweep_blocks_per_sm"]
    assert best["c2_launch"]["work_blocks_per_sm"] in autotune.C2_GRID["work_blocks_per_sm"]
    assert best["success_rate"] >= tuned["min_success"] >= autotune.MIN_SUCCESS - 1e-9
    # the pick over the recorded trials reproduces the recorded best
    again = autotune.pick(tuned["trials"], tuned["min_success"])
    assert again is not None
    assert (again["slots"], again["check_every"], again["mix"]) == (best["slots"], best["check_every"],
                                                                     best["mix"])
