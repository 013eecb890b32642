"""Generates tests/golden/curve_quality.npz from the reference's own Python
curve-quality code (tests/python_dataset/curve_quality.py, class
CurveAssessment), imported from the reference tree.

    python tests/golden/make_curve_quality.py [/path/to/FastRRT]

The module imports matplotlib and cv2 for its plotting helpers only; a stub
stands in for matplotlib when it is absent (nothing here plots).  The
curves are integer cell sequences of the kinds interpolated paths have:
rounded Hermite curves between seeded poses, random walks with one-cell
steps (some with repeated cells), zigzags with sharp turns, and short
curves down to two cells, where the reference's window arithmetic raises.
For each curve the fixture keeps the reference's length, jerk and
tangential-discontinuity flag (window 4, threshold 15 deg, the headings
computed from the cells), or a marker where the reference raised.
"""
import math
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import build_oracle  # noqa: E402


def load_reference(reference):
    if "matplotlib" not in sys.modules:
        try:
            import matplotlib  # noqa: F401
        except ImportError:
            mpl = types.ModuleType("matplotlib")
            mpl.pyplot = types.ModuleType("matplotlib.pyplot")
            sys.modules["matplotlib"] = mpl
            sys.modules["matplotlib.pyplot"] = mpl.pyplot
    sys.path.insert(0, os.path.join(reference, "tests", "python_dataset"))
    import curve_quality
    return curve_quality.CurveAssessment


def hermite_cells(rng, n_samples, upward=False):
    """cells of a rounded Hermite curve; `upward`: from the bottom band to the
    top band with end headings near 0 (heading 0 points to -z, as in the
    planner's frames), else between two random poses"""
    if upward:
        x0, z0 = rng.integers(60, 196), rng.integers(200, 240)
        x1, z1 = rng.integers(60, 196), rng.integers(10, 60)
        h0, h1 = rng.uniform(-0.6, 0.6, 2)
    else:
        x0, z0 = rng.integers(20, 236, 2)
        x1, z1 = rng.integers(20, 236, 2)
        h0, h1 = rng.uniform(-math.pi, math.pi, 2)
    d = math.hypot(x1 - x0, z1 - z0)
    t = np.linspace(0.0, 1.0, n_samples)
    h00 = 2 * t**3 - 3 * t**2 + 1
    h10 = t**3 - 2 * t**2 + t
    h01 = -2 * t**3 + 3 * t**2
    h11 = t**3 - t**2
    px = h00 * x0 + h10 * d * math.sin(h0) + h01 * x1 + h11 * d * math.sin(h1)
    pz = h00 * z0 - h10 * d * math.cos(h0) + h01 * z1 - h11 * d * math.cos(h1)
    cells = np.stack([np.round(px), np.round(pz)], 1).astype(np.int64)
    keep = np.ones(len(cells), bool)
    keep[1:] = np.any(cells[1:] != cells[:-1], axis=1)
    return cells[keep]


def random_walk(rng, n, repeats):
    steps = rng.integers(-1, 2, (n - 1, 2))
    if not repeats:
        zero = ~np.any(steps != 0, axis=1)
        steps[zero, 1] = -1
    start = np.array([[128, 200]])
    return np.concatenate([start, start + np.cumsum(steps, 0)]).astype(np.int64)


def zigzag(rng, n):
    pts = [[128, 220]]
    dx = 1
    for k in range(1, n):
        if rng.random() < 0.15:
            dx = -dx
        pts.append([pts[-1][0] + dx, pts[-1][1] - 1])
    return np.array(pts, np.int64)


def curves():
    rng = np.random.default_rng(2024)
    out = []
    for k in range(48):
        out.append(hermite_cells(rng, int(rng.integers(40, 400)), upward=True))
    for k in range(16):
        out.append(hermite_cells(rng, int(rng.integers(20, 400))))
    for k in range(16):
        out.append(random_walk(rng, int(rng.integers(5, 120)), repeats=k % 3 == 0))
    for k in range(12):
        out.append(zigzag(rng, int(rng.integers(8, 80))))
    for n in (2, 3, 4, 5, 6, 7, 8, 9):
        out.append(hermite_cells(rng, 400, upward=True)[:n])
    out.append(np.array([[100, 100], [100, 99], [100, 98], [100, 97], [100, 96], [100, 95]], np.int64))
    return [c for c in out if len(c) >= 2]


def first_heading(c):
    """the direction of the curve's first cells in the curve-quality heading
    convention (0 towards -z, positive towards +x)"""
    b = c[min(4, len(c) - 1)]
    return math.pi / 2 - math.atan2(-(b[1] - c[0][1]), b[0] - c[0][0])


def main(reference=None):
    reference = reference or build_oracle.reference_root()
    CA = load_reference(reference)
    ca = CA(256, 256)
    rng = np.random.default_rng(7)
    cs = curves()
    n = len(cs)
    lengths = np.array([len(c) for c in cs], np.int32)
    flat = np.concatenate(cs).astype(np.int32)
    # start headings near the curve's first direction (within or beyond the
    # 15 deg threshold) for most curves, the planner's 0 for the rest
    start_heading = np.array([first_heading(c) + rng.uniform(-0.4, 0.4) if k % 4 else 0.0
                              for k, c in enumerate(cs)])
    total_length = np.zeros(n)
    jerk = np.full(n, np.nan)
    tan = np.full(n, -1, np.int8)  # -1: the reference raised
    for k, c in enumerate(cs):
        total_length[k] = CA._CurveAssessment__compute_curve_length(c)
        try:
            jerk[k] = ca._CurveAssessment__compute_jerk(c)
        except (IndexError, ZeroDivisionError):
            pass
        try:
            tan[k] = int(ca._CurveAssessment__tangential_discontinuity(
                c, window_side=4, threshold=15, start_heading=float(start_heading[k]), compute_heading=True))
        except (IndexError, ZeroDivisionError):
            pass
    np.savez_compressed(os.path.join(HERE, "curve_quality.npz"), lengths=lengths, cells=flat,
                        start_heading=start_heading, total_length=total_length, jerk=jerk, tan=tan)
    print(f"{n} curves, {int(np.isnan(jerk).sum())} where the reference's jerk raised, "
          f"{int((tan == 1).sum())} with a tangential discontinuity; written to {HERE}")


if __name__ == "__main__":
    main(*sys.argv[1:])
