"""Generates tests/golden/interpolation.npz from the reference's own
interpolate() (src/interpolation.cpp), compiled with g++ from the reference
tree together with interp_harness.cpp and the driveless stand-ins of
oracle/ref/shim (the reference includes driveless headers that are not in
its tree).

    python tests/golden/make_interpolation.py [/path/to/FastRRT]

The control-point paths are seeded: planned-path-like chains from the
bottom of a 256x256 frame towards its top (steps of 5-40 cells, headings
near the chain's direction), chains with sharp turns, chains that leave the
frame (their out-of-frame samples are skipped), two-point paths and
repeated points.  For each path the fixture keeps the reference's cells and
headings.
"""
import math
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import build_oracle  # noqa: E402

W = H = 256


def build(reference, tmp):
    exe = os.path.join(tmp, "interp")
    cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "oracle", "ref", "shim"),
                    "-I", cuda_inc, os.path.join(reference, "src", "interpolation.cpp"),
                    os.path.join(HERE, "interp_harness.cpp"), "-o", exe], check=True)
    return exe


def chain(rng, n, jitter, start=(128, 230)):
    pts = [(start[0], start[1], 0.0)]
    h = rng.uniform(-0.3, 0.3)
    for _ in range(n - 1):
        h += rng.normal(0, jitter)
        step = rng.uniform(5, 40)
        x = int(round(pts[-1][0] + step * math.sin(h)))
        z = int(round(pts[-1][1] - step * math.cos(h)))
        pts.append((x, z, float(np.float32(h + rng.normal(0, 0.05)))))
    return np.array(pts, np.float32)


def paths():
    rng = np.random.default_rng(77)
    out = []
    for _ in range(40):
        out.append(chain(rng, int(rng.integers(2, 12)), 0.25))
    for _ in range(12):
        out.append(chain(rng, int(rng.integers(3, 9)), 1.2))          # sharp turns
    for _ in range(8):
        out.append(chain(rng, int(rng.integers(6, 14)), 0.4, start=(10, 240)))  # may leave the frame
    out.append(np.array([[128, 128, 0.0], [128, 0, 0.0]], np.float32))
    out.append(np.array([[128, 128, 0.0], [128, 128, 0.0], [140, 100, 0.3]], np.float32))  # repeat
    out.append(np.array([[0, 255, -1.2], [255, 0, 1.0]], np.float32))
    return out


def run(exe, path):
    inp = f"{W} {H} {len(path)}\n" + "".join(f"{int(p[0])} {int(p[1])} {float(p[2]):.9g}\n" for p in path)
    lines = subprocess.run([exe], input=inp, capture_output=True, text=True, check=True).stdout.split("\n")
    m = int(lines[0])
    rows = [lines[1 + k].split() for k in range(m)]
    return np.array([[float(r[0]), float(r[1]), float(r[2])] for r in rows], np.float32).reshape(m, 3)


def main(reference=None):
    reference = reference or build_oracle.reference_root()
    if shutil.which("g++") is None:
        raise SystemExit("g++ is needed")
    tmp = tempfile.mkdtemp()
    try:
        exe = build(reference, tmp)
        ps = paths()
        outs = [run(exe, p) for p in ps]
    finally:
        shutil.rmtree(tmp)
    np.savez_compressed(os.path.join(HERE, "interpolation.npz"),
                        n_in=np.array([len(p) for p in ps], np.int32), paths=np.concatenate(ps),
                        n_out=np.array([len(o) for o in outs], np.int32),
                        out=np.concatenate(outs) if outs else np.zeros((0, 3), np.float32),
                        width=W, height=H)
    print(f"{len(ps)} paths, {sum(len(o) for o in outs)} interpolated points; written to {HERE}")


if __name__ == "__main__":
    main(*sys.argv[1:])
