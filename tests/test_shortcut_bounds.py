"""The exactness arguments behind the footprint and curvature shortcuts of
the curve and expansion kernels (fastrrt_b200/csrc/frrt_device.cuh), checked
on the CPU with the reference's float32 probe arithmetic
(path_feasible.cu:18-78: cell = (int)(j c - i s + x), (int)(j s + i c + z),
with and without the fused multiply-add a compiler may form):

- box_feasible: every probed cell lies within ceil(mdx |c| + mdz |s| + 1e-3)
  cells of the centre in x (and the transposed bound in z), so an
  obstacle-free box means an obstacle-free footprint;
- rows_clear_warp: every probed cell lies inside the x interval that the
  row-interval test computes for its row, so clear intervals mean a clear
  footprint;
- the clear mask: every probe at any heading lies within Chebyshev radius
  floor(sqrt(mdx^2 + mdz^2)) + 2, so a clear cell needs no probe;
- HermTask::ref_over: outside the 1e-6 band around the curvature limit the
  comparison of num^2 with limit^2 s2^3 gives the reference's
  (float)(num / pow(s2, 1.5)) > limit.
"""
import math

import numpy as np

f32 = np.float32
SIZES = [(11, 20), (22, 40), (5, 9), (1, 1), (30, 12)]  # (mdx, mdz): half-extents in cells


def probe_cells(x, z, c, s, mdx, mdz, fused):
    """every cell the reference's probe loop visits, in float32"""
    i, j = np.meshgrid(np.arange(-mdz, mdz + 1), np.arange(-mdx, mdx + 1), indexing="ij")
    i = i.astype(f32).ravel()
    j = j.astype(f32).ravel()
    if fused:
        # j*c - i*s as fma(j, c, -(i*s)) and j*s + i*c as fma(j, s, i*c)
        xo = (j.astype(np.float64) * c - (i * s).astype(np.float64)).astype(f32)
        zo = (j.astype(np.float64) * s + (i * c).astype(np.float64)).astype(f32)
    else:
        xo = (j * c) - (i * s)
        zo = (j * s) + (i * c)
    xl = np.trunc(xo + f32(x)).astype(np.int64)
    zl = np.trunc(zo + f32(z)).astype(np.int64)
    return xl, zl


def angles(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.uniform(-math.pi, math.pi, n)
    # and the axis directions, where a sine or cosine is (nearly) zero
    a[:16] = np.repeat([0.0, math.pi / 2, -math.pi / 2, math.pi], 4)
    return a


def test_box_bound_holds_for_every_probe():
    for mdx, mdz in SIZES:
        for a in angles(400, mdx * 100 + mdz):
            c = f32(math.cos(a))
            s = f32(math.sin(a))
            for fused in (False, True):
                for x, z in ((100, 100), (0, 0), (3, 250)):
                    xl, zl = probe_cells(x, z, c, s, mdx, mdz, fused)
                    # the box's direction is computed another way on the
                    # device (from the curve's derivative): perturb it
                    for da in (0.0, 1e-6, -1e-6):
                        ac = f32(abs(math.cos(a + da)))
                        as_ = f32(abs(math.sin(a + da)))
                        ex = math.ceil(f32(mdx * ac + mdz * as_ + f32(1e-3)))
                        ez = math.ceil(f32(mdx * as_ + mdz * ac + f32(1e-3)))
                        assert np.abs(xl - x).max() <= ex, (mdx, mdz, a, fused)
                        assert np.abs(zl - z).max() <= ez, (mdx, mdz, a, fused)


def row_intervals(x, z, c, s, mdx, mdz, H):
    """the row-interval test's x interval per row (float32, as the device)"""
    ac, as_ = abs(c), abs(s)
    ez = f32(f32(mdx) * as_ + f32(mdz) * ac)
    z0 = max(0, int(math.floor(f32(z) - ez)) - 1)
    z1 = min(H - 1, int(math.floor(f32(z) + ez)) + 1)
    use1, use2 = ac > f32(1e-6), as_ > f32(1e-6)
    ic = f32(1.0) / c if use1 else f32(0)
    is_ = f32(1.0) / s if use2 else f32(0)
    h1, h2 = f32(mdx) * abs(ic), f32(mdz) * abs(is_)
    sic, cis = s * ic, c * is_
    out = {}
    for zr in range(z0, z1 + 1):
        za = f32(zr - z) - (f32(1.001) if zr == 0 else f32(0.001))
        zb = f32(zr - z + 1) + f32(0.001)
        lo, hi = f32(-1e30), f32(1e30)
        if use1:
            pa, pb = -za * sic, -zb * sic
            lo = max(lo, min(pa, pb) - h1)
            hi = min(hi, max(pa, pb) + h1)
        if use2:
            qa, qb = za * cis, zb * cis
            lo = max(lo, min(qa, qb) - h2)
            hi = min(hi, max(qa, qb) + h2)
        if not lo <= hi:
            continue
        xa = max(0, int(math.floor(f32(x) + lo - f32(1e-3))))
        xb = int(f32(x) + hi + f32(1e-3))
        out[zr] = (xa, xb)
    return out


def test_row_intervals_cover_every_probe():
    W = H = 256
    for mdx, mdz in SIZES[:3]:
        for a in angles(150, 7 + mdx):
            c = f32(math.cos(a))
            s = f32(math.sin(a))
            for x, z in ((128, 128), (2, 1), (250, 60)):
                iv = row_intervals(x, z, c, s, mdx, mdz, H)
                for fused in (False, True):
                    xl, zl = probe_cells(x, z, c, s, mdx, mdz, fused)
                    inside = (xl >= 0) & (xl < W) & (zl >= 0) & (zl < H)
                    for px, pz in zip(xl[inside], zl[inside]):
                        assert pz in iv, (mdx, mdz, a, x, z, px, pz)
                        xa, xb = iv[pz]
                        assert xa <= px <= xb, (mdx, mdz, a, x, z, px, pz, xa, xb)


def test_curvature_band_decides_as_the_reference():
    rng = np.random.default_rng(5)
    n = 200000
    limit = f32(0.35)
    ddx = rng.normal(0, 30, n)
    ddz = rng.normal(0, 30, n)
    s2 = ddx * ddx + ddz * ddz
    # numerators spread around the limit, many within a few 1e-6 of it
    k = float(limit) * (1 + rng.choice([1e-3, 1e-5, 2e-6, 1e-7, 0.0], n) * rng.choice([-1, 1], n))
    num = k * s2 ** 1.5 * (1 + rng.normal(0, 1e-9, n))
    khi = float(limit) * (1 + 1e-6)
    klo = float(limit) * (1 - 1e-6)
    n2 = num * num
    s6 = s2 * s2 * s2
    over = n2 > khi * khi * s6
    under = n2 < klo * klo * s6
    ref = (num / np.power(s2, 1.5)).astype(f32) > limit
    assert over.sum() > 1000 and under.sum() > 1000 and (~over & ~under).sum() > 100
    assert not (over & under).any()
    assert np.array_equal(ref[over], np.ones(over.sum(), bool))
    assert np.array_equal(ref[under], np.zeros(under.sum(), bool))


def test_clear_radius_bounds_every_probe():
    """the clear mask marks cells with no obstacle within Chebyshev radius
    floor(sqrt(mdx^2 + mdz^2)) + 2: every probe of the footprint at any
    heading lies within it, so a clear cell is feasible at every heading"""
    for mdx, mdz in SIZES:
        rc = int(math.floor(math.sqrt(mdx * mdx + mdz * mdz))) + 2
        for a in angles(300, 31 + mdz):
            c = f32(math.cos(a))
            s = f32(math.sin(a))
            for fused in (False, True):
                for x, z in ((100, 100), (0, 0)):
                    xl, zl = probe_cells(x, z, c, s, mdx, mdz, fused)
                    assert max(np.abs(xl - x).max(), np.abs(zl - z).max()) <= rc, (mdx, mdz, a)


def test_summed_area_boxes_stay_below_the_count_modulus():
    """the summed-area table holds obstacle counts mod 2^16, so a box count
    is exact only for boxes of fewer than 65536 cells; the box test is used
    only when mdx + mdz <= 120, where the largest box at any heading
    ((2 ex + 1) x (2 ez + 1), ex and ez at most ceil(sqrt(mdx^2 + mdz^2) +
    1e-3)) stays below that"""
    worst = 0
    for mdx in range(0, 121):
        for mdz in range(0, 121 - mdx):
            e = math.ceil(math.sqrt(mdx * mdx + mdz * mdz) + 1e-3)
            worst = max(worst, (2 * e + 1) ** 2)
    assert worst < 65536
    # and the bound on e holds at every heading
    for mdx, mdz in SIZES:
        for a in angles(200, 3):
            e = mdx * abs(math.cos(a)) + mdz * abs(math.sin(a))
            assert e <= math.sqrt(mdx * mdx + mdz * mdz) + 1e-9
