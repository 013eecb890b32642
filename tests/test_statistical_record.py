"""The committed whole-planner statistics against the reference planner
(oracle/compare_success.py, run on a B200 with the reference's own FastRRT
compiled from its sources): the record covers 1000 seeds and sits within the
target, success rate within one point and mean path cost within 1 %."""
import json
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load(name):
    with open(os.path.join(ROOT, "oracle", name)) as f:
        return json.load(f)


def test_c0_record_is_within_one_point_and_one_percent():
    d = load("compare_success_c0.json")
    assert d["seeds"] == [0, 999]
    assert abs(d["success_mine"] - d["success_reference"]) <= 0.01 + 1e-12
    assert abs(d["success_diff_points"] - 100 * (d["success_mine"] - d["success_reference"])) < 1e-9
    rel = d["mean_path_cost_mine"] / d["mean_path_cost_reference"] - 1
    assert abs(rel - d["path_cost_rel_diff"]) < 1e-12
    assert abs(rel) <= 0.01
    assert abs(d["mean_path_len_mine"] / d["mean_path_len_reference"] - 1) <= 0.01
    # paths counted for this library passed its device validator
    assert "validate" in d["mine_validated_by"]
    assert d["both_solved"] >= 900


def test_mixed_size_record_agrees_within_its_confidence_interval():
    """200 seeds of the mixed-size generator: most requests are not solvable
    within 100 loops by either planner; the two success rates agree within
    the 95 % interval of the sample"""
    d = load("compare_success_c2.json")
    assert abs(d["success_mine"] - d["success_reference"]) <= max(d["success_ci95"])
