"""CPU restatement of the reference's curve-quality metrics
(tests/python_dataset/curve_quality.py, class CurveAssessment) for interpolated
paths.  TEST INFRASTRUCTURE ONLY: the GPU kernel of the product is checked
against it.

A curve is an (n, 2+) array of cells (x, z, ...).  The reference computes in
float64 Python; so does this restatement.  Its window arithmetic indexes the
curve with negative positions on short curves (Python wraps them); the
restatement does the same and returns NaN where the reference would raise an
IndexError (positions below -n).  Pinned against the reference's own
CurveAssessment by tests/golden/curve_quality.npz (generated by
tests/golden/make_curve_quality.py, which imports the reference module).
"""
import math

import numpy as np

WINDOW = 4          # window_side of assess_curve (curve_quality.py:110-124)
THRESHOLD_DEG = 15  # threshold of __tangential_discontinuity (curve_quality.py:227)


def _at(curve, k):
    n = len(curve)
    if k < -n:
        raise IndexError(k)
    return curve[k]


def curve_length(curve):
    """__compute_curve_length (curve_quality.py:92-99)"""
    s = 0.0
    for i in range(1, len(curve)):
        s += math.sqrt((curve[i][0] - curve[i - 1][0]) ** 2 + (curve[i][1] - curve[i - 1][1]) ** 2)
    return s


def _window(n, pos, w):
    """the window bounds of __curve_mean_heading / __derivate_curve_p
    (curve_quality.py:191-201, 248-258)"""
    i, j = pos - w, pos + w
    if i < 0:
        j = j - i
        i = 0
    if j >= n:
        i = i - (j - n) - 1
        j = n - 1
    return i, j


def _heading(p1, p2):
    """__curve_heading (curve_quality.py:179-189): (heading, valid)"""
    if p1[0] == p2[0] and p1[1] == p2[1]:
        return 0.0, False
    h = math.pi / 2 - math.atan2(-(p2[1] - p1[1]), p2[0] - p1[0])
    if h > math.pi:
        h -= 2 * math.pi
    return h, True


def _mean_heading(curve, pos, w):
    """__curve_mean_heading (curve_quality.py:191-225), debug off: invalid
    pairs count as 0"""
    i, j = _window(len(curve), pos, w)
    h, count = 0.0, 0
    for k in range(i, pos):
        h += _heading(_at(curve, k), curve[pos])[0]
        count += 1
    for k in range(pos + 1, j + 1):
        h += _heading(curve[pos], _at(curve, k))[0]
        count += 1
    return h / count


def tangential_discontinuity(curve, start_heading, w=WINDOW, threshold_deg=THRESHOLD_DEG):
    """__tangential_discontinuity (curve_quality.py:227-241), compute_heading on"""
    a_before = start_heading
    thr = math.radians(threshold_deg)
    for i in range(1, len(curve)):
        a = _mean_heading(curve, i, w)
        if abs(a - a_before) > thr:
            return True
        a_before = a
    return False


def _derivate_curve(curve, pos, w):
    """__derivate_p / __derivate_curve_p (curve_quality.py:243-276)"""
    i, j = _window(len(curve), pos, w)
    h, count = 0.0, 0
    for k in range(i, pos):
        a = _at(curve, k)
        h += math.atan2(curve[pos][1] - a[1], curve[pos][0] - a[0])
        count += 1
    for k in range(pos + 1, j + 1):
        b = _at(curve, k)
        h += math.atan2(b[1] - curve[pos][1], b[0] - curve[pos][0])
        count += 1
    return h / count


def jerk(curve, w=WINDOW):
    """__compute_jerk (curve_quality.py:290-294): |sum| np.gradient twice| of
    the windowed direction"""
    v = [_derivate_curve(curve, i, w) for i in range(len(curve))]
    a = np.gradient(np.asarray(v, np.float64), 1)
    j = np.gradient(a, 1)
    return float(abs(np.sum(np.abs(j))))


def assess(curve, start_heading):
    """(length, jerk, tangential discontinuity) of a curve; NaN / None where
    the reference's arithmetic would fail"""
    curve = [tuple(float(c) for c in p[:2]) for p in np.asarray(curve)]
    length = curve_length(curve)
    if len(curve) < 3:
        return length, float("nan"), None
    try:
        return length, jerk(curve), tangential_discontinuity(curve, start_heading)
    except (IndexError, ZeroDivisionError):
        return length, float("nan"), None
