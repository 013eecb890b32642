"""Seeded synthetic BEV frames and planning requests.

The workloads measured by this project use no dataset: every frame is drawn
from a seeded generator with the shapes, sizes and value distributions of
the benchmark configurations.

  * 256 x 256 (or 128 / 512) uint8 class-id grid at 0.135 m/px;
  * a road corridor of class 0 (cost 0) from the bottom to the top;
  * axis-aligned rectangles and disks (radius 4-20 px) of class 3 (cost -1,
    an obstacle), 40% of them inside the corridor so that the direct route
    is usually blocked; by default 12 rectangles and 6 disks, or as many as
    needed to reach a requested obstacle coverage;
  * elsewhere a blocky mix of class 1 (low cost) and class 2 (high cost);
  * start and goal neighbourhoods are kept free of obstacles.
"""
import math

import numpy as np

CLASS_ROAD, CLASS_LOW, CLASS_HIGH, CLASS_OBSTACLE = 0, 1, 2, 3
CLASS_COSTS = np.array([0.0, 1.0, 4.0, -1.0], dtype=np.float32)
M_PER_PX = 0.135


def _clear_box(cls, cx, cz, hx, hz, value=CLASS_ROAD):
    H, W = cls.shape
    x0, x1 = max(0, cx - hx), min(W, cx + hx + 1)
    z0, z1 = max(0, cz - hz), min(H, cz + hz + 1)
    cls[z0:z1, x0:x1] = np.where(cls[z0:z1, x0:x1] == CLASS_OBSTACLE, value, cls[z0:z1, x0:x1])


def make_frame(seed, size=256, n_rect=12, n_disk=6, coverage=None, start=None, goal=None,
               keep_clear=(24, 44)):
    """One class-id frame.  With `coverage` set, rectangles and disks are
    added (two rectangles per disk) until that obstacle fraction is reached."""
    rng = np.random.default_rng(np.uint64(seed) + np.uint64(0x5EED))
    W = H = int(size)
    blk = 8
    mix = rng.random(((H + blk - 1) // blk, (W + blk - 1) // blk)) < 0.5
    cls = np.where(np.kron(mix, np.ones((blk, blk), bool))[:H, :W], CLASS_HIGH, CLASS_LOW)
    cls = cls.astype(np.uint8)
    half = max(12, int(0.18 * W))
    cx = W // 2 + int(rng.integers(-W // 16, W // 16 + 1))
    cls[:, max(0, cx - half):min(W, cx + half)] = CLASS_ROAD

    def centre_x():
        # 40% of the obstacles land inside the corridor, so that the direct
        # route from start to goal is usually blocked
        if rng.random() < 0.4:
            return float(rng.uniform(cx - half, cx + half))
        return float(rng.uniform(0, W))

    def add_rect():
        w = int(rng.integers(4, max(6, W // 10)))
        h = int(rng.integers(4, max(6, H // 10)))
        x = int(min(max(0, centre_x() - w / 2), W - w))
        z = int(rng.integers(0, H - h))
        cls[z:z + h, x:x + w] = CLASS_OBSTACLE

    zz, xx = np.mgrid[0:H, 0:W]

    def add_disk():
        r = float(rng.uniform(4, 20))
        x = centre_x()
        z = float(rng.uniform(0, H))
        cls[(xx - x) ** 2 + (zz - z) ** 2 <= r * r] = CLASS_OBSTACLE

    if coverage is None:
        for _ in range(n_rect):
            add_rect()
        for _ in range(n_disk):
            add_disk()
    else:
        # coverage counts only obstacles outside the start / goal neighbourhoods,
        # which are cleared afterwards
        keep = np.ones((H, W), bool)
        for p in (start, goal):
            if p is not None:
                keep[max(0, p[1] - keep_clear[1]):p[1] + keep_clear[1] + 1,
                     max(0, p[0] - keep_clear[0]):p[0] + keep_clear[0] + 1] = False
        k = 0
        while ((cls == CLASS_OBSTACLE) & keep).mean() < coverage and k < 10000:
            add_rect() if k % 3 != 2 else add_disk()
            k += 1
    if start is not None:
        _clear_box(cls, start[0], start[1], *keep_clear)
    if goal is not None:
        _clear_box(cls, goal[0], goal[1], *keep_clear)
    return cls


def c0_request(seed, size=256):
    """The single-instance workload: start (W/2, H/2, 0), goal (W/2, 0, 0)."""
    W = size
    start = (W // 2, W // 2, 0.0)
    goal = (W // 2, 0, 0.0)
    cls = make_frame(seed, size, start=start, goal=goal)
    return cls, start, goal


def batch_request(seed, sizes=(128, 256, 512), coverage=(0.05, 0.30), steer_deg=(30.0, 45.0)):
    """One request of the batched workload: frame size drawn from `sizes`,
    obstacle coverage U(coverage), start near the bottom centre with heading
    U(-0.3, 0.3) rad, goal anywhere on the top band, steering limit
    U(steer_deg)."""
    rng = np.random.default_rng(np.uint64(seed) + np.uint64(0xBA7C4))
    size = int(sizes[int(rng.integers(0, len(sizes)))])
    cov = float(rng.uniform(*coverage))
    start = (size // 2 + int(rng.integers(-size // 16, size // 16 + 1)),
             size - 1 - int(rng.integers(size // 16, size // 8 + 1)),
             float(np.float32(rng.uniform(-0.3, 0.3))))
    goal = (int(rng.integers(size // 8, size - size // 8)), int(rng.integers(0, size // 16 + 1)),
            0.0)
    cls = make_frame(seed, size, coverage=cov, start=start, goal=goal)
    steer = float(rng.uniform(*steer_deg))
    return cls, start, goal, steer, cov


def candidates(n, W, H, seed, max_steer_deg=40.0, length=(5.0, 40.0)):
    """Per-candidate workload: parent cell uniform in the frame, steering
    U(-max, max), segment length U(length).  The parent heading U(-pi, pi) is
    drawn per cell (one heading per node-grid cell)."""
    rng = np.random.default_rng(np.uint64(seed) + np.uint64(0xCA7D))
    heading = rng.uniform(-math.pi, math.pi, W * H).astype(np.float32)
    sx = rng.integers(0, W, n).astype(np.int32)
    sz = rng.integers(0, H, n).astype(np.int32)
    ms = math.radians(max_steer_deg)
    steer = rng.uniform(-ms, ms, n).astype(np.float32)
    seg = rng.uniform(length[0], length[1], n).astype(np.float32)
    return heading, sx, sz, steer, seg


def hermite_pairs(n, W, H, seed, num_points=64):
    """Hermite pose pairs whose integer distance truncates to `num_points`
    (the reference samples TO_INT(distance) points per curve)."""
    rng = np.random.default_rng(np.uint64(seed) + np.uint64(0x4E41))
    xs, zs, gxs, gzs = [], [], [], []
    need = n
    while need > 0:
        m = need * 2
        x = rng.integers(0, W, m)
        z = rng.integers(0, H, m)
        a = rng.uniform(-math.pi, math.pi, m)
        r = rng.uniform(num_points, num_points + 1, m)
        gx = np.rint(x + r * np.cos(a)).astype(np.int64)
        gz = np.rint(z + r * np.sin(a)).astype(np.int64)
        d = np.sqrt(((gx - x) ** 2 + (gz - z) ** 2).astype(np.float32))
        ok = (gx >= 0) & (gx < W) & (gz >= 0) & (gz < H) & (d.astype(np.int64) == num_points)
        idx = np.nonzero(ok)[0][:need]
        xs.append(x[idx]); zs.append(z[idx]); gxs.append(gx[idx]); gzs.append(gz[idx])
        need -= len(idx)
    x = np.concatenate(xs).astype(np.int32)
    z = np.concatenate(zs).astype(np.int32)
    gx = np.concatenate(gxs).astype(np.int32)
    gz = np.concatenate(gzs).astype(np.int32)
    lh = rng.uniform(-math.pi, math.pi, n).astype(np.float32)
    gh = rng.uniform(-math.pi, math.pi, n).astype(np.float32)
    return x, z, lh, gx, gz, gh
