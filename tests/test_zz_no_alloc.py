"""fastrrt_candidates_kinematic_noalloc: the kinematic candidate check for
callers that cannot allocate device memory (memory reserved up front, pool
policies that forbid new allocations, code that must stay out of the
driver's allocator).  Through the C ABI it must return what the allocating
entry point (a candidates context + fastrrt_candidates_kinematic_device)
returns on the same inputs, on two calls in a row with different frames, so
that nothing one call leaves in the shared device array leaks into the next.
This file is collected last on purpose."""
import ctypes as C
import math

import numpy as np
import pytest

from fastrrt_b200 import synth

pytestmark = pytest.mark.gpu
MS = math.radians(40.0)
LR = 5.4 / 2


def case(seed, size, coverage):
    cls = synth.make_frame(seed, size, coverage=coverage)
    heading, sx, sz, steer, seg = synth.candidates(8192, size, size, seed)
    cost = np.random.default_rng(seed).uniform(0, 50, size * size).astype(np.float32)
    return cls, heading, cost, sx, sz, steer, seg


def via_context(F, torch, cls, heading, cost, sx, sz, steer, seg):
    fr = F.SearchFrame(class_ids=cls, class_costs=synth.CLASS_COSTS)
    ctx = F.Candidates(fr, min_dist=(22, 40), max_steering_rad=MS, lr_m=LR, heading_grid=heading,
                       cost_grid=cost)
    d = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (sx, sz, steer, seg)]
    out = torch.zeros((len(sx), 4), dtype=torch.float32, device="cuda")
    pr = torch.zeros(1, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    ctx.kinematic_device(*d, 2.0, out, pr)
    torch.cuda.synchronize()
    return out.cpu().numpy(), int(pr.item())


class NoAllocCall:
    """device copies of one case's inputs and outputs; call() runs the entry
    point on them and returns (rc, error text)"""

    def __init__(self, F, torch, cls, heading, cost, sx, sz, steer, seg, costs=synth.CLASS_COSTS):
        self.F, self.torch = F, torch
        self.H, self.W = cls.shape
        dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
        self.dcls, self.dcost_tab = dev(cls.astype(np.uint8)), dev(costs)
        self.n_classes = len(costs)
        self.dh, self.dc = dev(heading), dev(cost)
        self.dsx, self.dsz, self.dst, self.dln = dev(sx), dev(sz), dev(steer), dev(seg)
        self.n = len(sx)
        self.out = torch.full((self.n, 4), 7.0, dtype=torch.float32, device="cuda")
        self.pr = torch.zeros(1, dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()

    def call(self):
        rc = self.F.lib().fastrrt_candidates_kinematic_noalloc(
            self.W, self.H, self.dcls.data_ptr(), self.dcost_tab.data_ptr(), self.n_classes,
            self.dh.data_ptr(), self.dc.data_ptr(), 22, 40, -1, -1, -1, -1, MS, LR, self.n,
            self.dsx.data_ptr(), self.dsz.data_ptr(), self.dst.data_ptr(), self.dln.data_ptr(), 2.0,
            self.out.data_ptr(), self.pr.data_ptr(), None)
        return rc, (self.F._lib.last_error() if rc else "")


def via_noalloc(F, torch, *args):
    c = NoAllocCall(F, torch, *args)
    rc, err = c.call()
    assert rc == 0, err
    torch.cuda.synchronize()
    return c.out.cpu().numpy(), int(c.pr.item())


@pytest.fixture(scope="module")
def torch_gpu(gpu):
    import torch
    return torch


def test_noalloc_matches_allocating_entry_point_twice(gpu, torch_gpu):
    # two calls in a row: a 256 x 256 frame at 30% obstacles, then a
    # 128 x 128 frame at 5% (smaller masks over the same array)
    for seed, size, cov in ((11, 256, 0.30), (12, 128, 0.05)):
        args = case(seed, size, cov)
        want, want_pr = via_context(gpu, torch_gpu, *args)
        got, got_pr = via_noalloc(gpu, torch_gpu, *args)
        # the same kernels on the same inputs: bit-exact
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (seed, size)
        assert got_pr == want_pr and got_pr > 0
        assert 0.0 < float((got[:, 0] >= 0).mean()) < 1.0


def test_noalloc_rejects_oversized_frames(gpu):
    L = gpu.lib()
    one = C.c_void_p(1)
    rc = L.fastrrt_candidates_kinematic_noalloc(
        1025, 64, one, one, 4, one, one, 22, 40, -1, -1, -1, -1, MS, LR, 1, one, one, one, one,
        2.0, one, None, None)
    assert rc < 0
    assert "1024" in gpu._lib.last_error()


def test_noalloc_allocates_no_device_memory(gpu, torch_gpu):
    # after a warm-up call (module load, first launches) a further call leaves
    # the device's free memory unchanged: nothing was allocated or kept
    torch = torch_gpu
    c = NoAllocCall(gpu, torch, *case(13, 256, 0.15))
    assert c.call()[0] == 0
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    rc, err = c.call()
    torch.cuda.synchronize()
    assert rc == 0, err
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_rejects_bad_class_ids_and_cells(gpu, torch_gpu):
    torch = torch_gpu
    cls, heading, cost, sx, sz, steer, seg = case(14, 128, 0.15)
    # a class id beyond the cost table
    bad = cls.copy()
    bad[5, 7] = 9
    rc, err = NoAllocCall(gpu, torch, bad, heading, cost, sx, sz, steer, seg, costs=synth.CLASS_COSTS[:4]).call()
    assert rc < 0 and "class id" in err
    # one candidate whose start cell lies outside the frame: its row is the
    # rejected row, the others match the allocating entry point, and the call
    # reports the cell
    sx2 = sx.copy()
    sx2[3] = 128
    c = NoAllocCall(gpu, torch, cls, heading, cost, sx2, sz, steer, seg)
    rc, err = c.call()
    assert rc < 0 and "outside the frame" in err
    torch.cuda.synchronize()
    got = c.out.cpu().numpy()
    assert np.array_equal(got[3], [-1.0, -1.0, 0.0, 0.0])
    want, _ = via_context(gpu, torch, cls, heading, cost, sx, sz, steer, seg)
    keep = np.arange(len(sx)) != 3
    assert np.array_equal(got[keep].view(np.uint32), want[keep].view(np.uint32))
    # the next good call succeeds: the flags start at zero on every call
    assert via_noalloc(gpu, torch, cls, heading, cost, sx, sz, steer, seg)[1] > 0
