"""Generates the golden fixtures in this directory from the reference's own
code (oracle/_ref/libfastrrt_ref.so, built by oracle/ref/Makefile from the
reference tree) and the reference's unit-test data files.

    python tests/golden/make_golden.py [/path/to/FastRRT]

Outputs (small .npz files, committed):
  kinematic_c0.npz  check_kinematic_new_path on 2048 seeded candidates of a
                    seeded 256x256 frame (reference host build)
  hermite_c0.npz    checkDirectConnectionToGoal on 1024 seeded pose pairs
  feasible_c0.npz   __computeFeasibleForAngle on 2048 seeded (cell, angle)
  graph_dumps.npz   the node lists of unittests/src/test_data/*.txt
"""
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from fastrrt_b200 import synth  # noqa: E402
from oracle import build_oracle, oracle as O  # noqa: E402

W = H = 256
MAX_STEER = math.radians(40.0)
LR = 5.4 / 2


def main(reference=None):
    reference = reference or build_oracle.reference_root()
    build_oracle.build_ref(reference)
    if O.ref_lib() is None:
        raise SystemExit("oracle/_ref not built")
    cls, _, _ = synth.c0_request(3)
    frame = O.Frame(cls, synth.CLASS_COSTS)
    heading, sx, sz, steer, seg = synth.candidates(2048, W, H, 11)
    rc = O.RefCase(frame, heading=heading, max_steer_rad=MAX_STEER, lr=LR, mdx=11, mdz=20)
    out = rc.kinematic(sx, sz, steer, seg, 2.0)
    np.savez_compressed(os.path.join(HERE, "kinematic_c0.npz"), cls=cls, heading=heading, sx=sx,
                        sz=sz, steer=steer, length=seg, velocity=np.float32(2.0),
                        max_steer=np.float64(MAX_STEER), lr=np.float64(LR), mdx=11, mdz=20, out=out)
    x, z, lh, gx, gz, gh = synth.hermite_pairs(1024, W, H, 5, num_points=40)
    hout = rc.direct(0.8, x, z, lh, gx, gz, gh)
    np.savez_compressed(os.path.join(HERE, "hermite_c0.npz"), cls=cls, x=x, z=z, lh=lh, gx=gx, gz=gz,
                        gh=gh, max_curvature=np.float32(0.8), mdx=11, mdz=20, out=hout)
    rng = np.random.default_rng(17)
    fx = rng.integers(0, W, 2048).astype(np.int32)
    fz = rng.integers(0, H, 2048).astype(np.int32)
    fa = rng.uniform(-math.pi, math.pi, 2048).astype(np.float32)
    fout = rc.feasible(fx, fz, fa)
    np.savez_compressed(os.path.join(HERE, "feasible_c0.npz"), cls=cls, x=fx, z=fz, a=fa, mdx=11,
                        mdz=20, out=fout)
    dumps = {}
    data_dir = os.path.join(reference, "unittests", "src", "test_data")
    for name in sorted(os.listdir(data_dir)):
        rows = [list(map(float, line.split())) for line in open(os.path.join(data_dir, name))
                if line.strip()]
        dumps[name.replace(".txt", "")] = np.array(rows, np.float64)
    np.savez_compressed(os.path.join(HERE, "graph_dumps.npz"), **dumps)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main(*sys.argv[1:])
