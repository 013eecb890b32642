import numpy as np

from fastrrt_b200 import synth


def test_c0_frames_are_seeded_and_clear_at_endpoints():
    a, s, g = synth.c0_request(5)
    b, _, _ = synth.c0_request(5)
    assert np.array_equal(a, b) and a.shape == (256, 256) and a.dtype == np.uint8
    assert s == (128, 128, 0.0) and g == (128, 0, 0.0)
    assert not np.any(a[128 - 44:128 + 45, 128 - 24:128 + 25] == synth.CLASS_OBSTACLE)
    assert 0.02 < (a == synth.CLASS_OBSTACLE).mean() < 0.25
    assert set(np.unique(a)) <= {0, 1, 2, 3}


def test_batch_requests_cover_sizes_and_coverage():
    sizes = set()
    for k in range(40):
        cls, st, gl, steer, cov = synth.batch_request(k)
        sizes.add(cls.shape[0])
        assert 30 <= steer <= 45 and 0.05 <= cov <= 0.30
        assert (cls == synth.CLASS_OBSTACLE).mean() >= cov - 1e-9
        assert 0 <= gl[1] < cls.shape[0] // 8
    assert sizes == {128, 256, 512}


def test_hermite_pairs_have_requested_sample_count():
    x, z, lh, gx, gz, gh = synth.hermite_pairs(500, 256, 256, 1, num_points=64)
    d = np.sqrt(((gx - x) ** 2 + (gz - z) ** 2).astype(np.float32)).astype(np.int64)
    assert np.all(d == 64)
