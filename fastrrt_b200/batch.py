"""Batched planner: many planning requests advance together, one CUDA graph
launch per loop() over every live slot (fastrrt_batch_* in the C ABI)."""
import math

import numpy as np

from . import _lib


def make_request(cls, class_costs, start, goal, *, perception_m=None, m_per_px=0.135,
                 max_steering_deg=40.0, vehicle_length_m=5.4, max_curvature=-1.0,
                 velocity_m_s=2.0, min_dist=(22, 40), max_path_size=40.0, dist_to_goal_tol=20.0,
                 heading_tol_rad=None, seed=0, smart=False, max_iterations=0,
                 lower_bound=(-1, -1), upper_bound=(-1, -1), timeout_ms=0):
    """A fastrrt_request; the returned object keeps its arrays alive."""
    cls = np.ascontiguousarray(cls, np.uint8)
    costs = np.ascontiguousarray(class_costs, np.float32)
    H, W = cls.shape
    if perception_m is None:
        perception_m = (W * m_per_px, H * m_per_px)
    if heading_tol_rad is None:
        heading_tol_rad = math.radians(10.0)
    r = _lib.Request()
    r.width, r.height = W, H
    r.class_ids = cls.ctypes.data_as(_lib.C.POINTER(_lib.C.c_uint8))
    r.class_costs = costs.ctypes.data_as(_lib.C.POINTER(_lib.C.c_float))
    r.n_classes = len(costs)
    r.perception_w_m, r.perception_h_m = perception_m
    r.max_steering_deg = max_steering_deg
    r.vehicle_length_m = vehicle_length_m
    r.max_curvature = max_curvature
    r.lb_x, r.lb_z = lower_bound
    r.ub_x, r.ub_z = upper_bound
    r.start_x, r.start_z, r.start_heading = int(start[0]), int(start[1]), float(start[2])
    r.goal_x, r.goal_z, r.goal_heading = int(goal[0]), int(goal[1]), float(goal[2])
    r.velocity_m_s = velocity_m_s
    r.min_dist_x, r.min_dist_z = min_dist
    r.max_path_size = max_path_size
    r.dist_to_goal_tol = dist_to_goal_tol
    r.heading_tol_rad = heading_tol_rad
    r.seed = int(seed)
    r.smart = int(bool(smart))
    r.max_iterations = int(max_iterations)
    r.class_ids_on_device = 0
    r.timeout_ms = int(timeout_ms)
    r._keep = (cls, costs)
    return r


def device_request(r, device_ptr):
    """A copy of request `r` whose class ids are read from device memory
    (e.g. a torch.uint8 tensor's data_ptr())."""
    d = _lib.Request()
    _lib.C.pointer(d)[0] = r
    d.class_ids = _lib.C.cast(_lib.C.c_void_p(device_ptr), _lib.C.POINTER(_lib.C.c_uint8))
    d.class_ids_on_device = 1
    d._keep = getattr(r, "_keep", None)
    return d


def slot_bytes(width, height):
    """device memory of one planning slot's storage for a width x height frame"""
    return int(_lib.lib().fastrrt_slot_bytes(int(width), int(height)))


class BatchPlanner:
    """Many planning requests in one CUDA graph launch per iteration.

    Without `budget_bytes` every one of the n_slots slots holds storage for
    a max_width x max_height frame.  With it, n_slots is the most requests
    planned at once and each admitted request takes storage sized by its own
    frame from an arena of budget_bytes; admission waits (serve) or fails
    (admit) while the arena has no room."""

    def __init__(self, n_slots, max_width, max_height, budget_bytes=0):
        L = _lib.lib()
        if budget_bytes:
            h = L.fastrrt_batch_create_budget(n_slots, max_width, max_height, int(budget_bytes))
        else:
            h = L.fastrrt_batch_create(n_slots, max_width, max_height)
        if not h:
            raise _lib.FastRRTError("batch_create: " + _lib.last_error())
        self._h = h
        self.n_slots = n_slots

    def memory(self):
        """(budget, bytes held now, most bytes held) of the slots' storage"""
        b, u, p = _lib.C.c_uint64(), _lib.C.c_uint64(), _lib.C.c_uint64()
        _lib.check(_lib.lib().fastrrt_batch_memory(self._h, _lib.C.byref(b), _lib.C.byref(u),
                                                   _lib.C.byref(p)), "batch_memory")
        return b.value, u.value, p.value

    def __del__(self):
        try:
            if getattr(self, "_h", None) and _lib._lib is not None:
                _lib.lib().fastrrt_batch_destroy(self._h)
                self._h = None
        except (AttributeError, TypeError):
            pass  # interpreter shutdown

    def admit_many(self, requests, timeout_ms=0):
        arr = (_lib.Request * len(requests))(*requests)
        self._keep = requests
        _lib.check(_lib.lib().fastrrt_batch_admit_many(self._h, len(requests), arr, timeout_ms),
                   "batch_admit_many")

    def admit(self, slot, request, timeout_ms=0):
        _lib.check(_lib.lib().fastrrt_batch_admit(self._h, slot, _lib.C.byref(request), timeout_ms),
                   "batch_admit")

    def run(self, max_launches=1000, check_every=1):
        return _lib.check(_lib.lib().fastrrt_batch_run(self._h, max_launches, check_every),
                          "batch_run")

    def step(self):
        _lib.check(_lib.lib().fastrrt_batch_step(self._h), "batch_step")

    def last_ms(self):
        return float(_lib.lib().fastrrt_batch_last_ms(self._h))

    def status(self):
        done = np.zeros(self.n_slots, np.int32)
        goal = np.zeros(self.n_slots, np.int32)
        loops = np.zeros(self.n_slots, np.int32)
        _lib.check(_lib.lib().fastrrt_batch_status(self._h, done, goal, loops), "batch_status")
        return done, goal, loops

    def collect(self, slots):
        slots = np.ascontiguousarray(slots, np.int32)
        n = len(slots)
        valid = np.zeros(n, np.int32)
        length = np.zeros(n, np.float32)
        path_n = np.zeros(n, np.int32)
        _lib.check(_lib.lib().fastrrt_batch_collect(self._h, n, slots, valid, length, path_n),
                   "batch_collect")
        return valid, length, path_n

    def interpolate(self, cap=8192):
        """GPU interpolation of the last collected paths and their curve
        quality: (length, jerk, tangential discontinuity) arrays"""
        L = _lib.lib()
        n = self.n_slots  # the last list has at most this many paths
        length = np.zeros(n, np.float32)
        jerk = np.zeros(n, np.float32)
        disc = np.zeros(n, np.int32)
        m = _lib.check(L.fastrrt_batch_interpolate(self._h, int(cap), length.ctypes.data, jerk.ctypes.data,
                                                   disc.ctypes.data), "batch_interpolate")
        self._interp_cap = cap
        return length[:m], jerk[:m], disc[:m]

    def interpolated_path(self, k):
        cap = getattr(self, "_interp_cap", 8192)
        buf = np.zeros(3 * cap, np.float32)
        m = _lib.check(_lib.lib().fastrrt_batch_interpolated_path(self._h, k, buf, cap),
                       "batch_interpolated_path")
        return buf[:3 * m].reshape(m, 3)

    def path(self, k, cap=1024):
        buf = np.zeros(3 * cap, np.float32)
        m = _lib.check(_lib.lib().fastrrt_batch_path(self._h, k, buf, cap), "batch_path")
        return buf[:3 * m].reshape(m, 3).copy()

    def plan(self, requests, max_launches=1000, check_every=4):
        """admit + loop until done + validate; returns (valid, length,
        latency_ms, device_ms)"""
        n = len(requests)
        arr = (_lib.Request * n)(*requests)
        valid = np.zeros(n, np.int32)
        length = np.zeros(n, np.float32)
        lat = np.zeros(n, np.float32)
        dev = _lib.C.c_float(0)
        _lib.check(_lib.lib().fastrrt_batch_plan(self._h, n, arr, max_launches, check_every, valid,
                                                 length, lat, _lib.C.byref(dev)), "batch_plan")
        return valid, length, lat, dev.value

    def serve(self, requests, arrival_ms=None, timeout_ms=100, check_every=2):
        """Continuous batching over `requests` (admitted as they arrive and
        slots free up); returns a dict of per-request arrays (valid, length,
        latency_ms from arrival to the device-clock finish, service_ms from
        admission to finish, result_ms from arrival until the validated path
        is on the host, loops) and the wall and device (CUDA event) time of
        the call in ms."""
        n = len(requests)
        arr = (_lib.Request * n)(*requests) if n else None
        out = {"valid": np.zeros(n, np.int32), "length": np.zeros(n, np.float32),
               "latency_ms": np.zeros(n, np.float32), "service_ms": np.zeros(n, np.float32),
               "loops": np.zeros(n, np.int32), "result_ms": np.zeros(n, np.float32)}
        arrival = None
        if arrival_ms is not None:
            arrival = np.ascontiguousarray(arrival_ms, np.float64)
        wall = _lib.C.c_double(0)
        dev = _lib.C.c_float(0)
        _lib.check(_lib.lib().fastrrt_batch_serve(
            self._h, n, arr, None if arrival is None else arrival.ctypes.data, int(timeout_ms),
            int(check_every), out["valid"], out["length"], out["latency_ms"], out["service_ms"],
            out["loops"], _lib.C.byref(wall), _lib.C.byref(dev), out["result_ms"]), "batch_serve")
        out["wall_ms"] = wall.value
        out["device_ms"] = dev.value
        return out

    def set_launch(self, sweep_blocks_per_sm=8, work_blocks_per_sm=2):
        _lib.check(_lib.lib().fastrrt_batch_set_launch(self._h, int(sweep_blocks_per_sm),
                                                       int(work_blocks_per_sm)), "batch_set_launch")

    def set_proposal(self, net, mix=0.5, cap=131072):
        """attach a ProposalNet (None detaches): each candidate's expansion is
        sampled from the network with probability mix, uniformly otherwise"""
        self._net = net
        _lib.check(_lib.lib().fastrrt_batch_set_proposal(self._h, net.handle if net else None,
                                                         float(mix), int(cap)), "batch_set_proposal")

    def proposal_attached(self):
        """whether a network is attached (set_proposal with a net)"""
        return getattr(self, "_net", None) is not None

    def log_paths(self, X_dev, labels_dev, offset, cap):
        """training rows of the last collected list's valid paths into device
        tensors (X: rows of 1040 bf16, labels: int32); returns rows written"""
        return _lib.check(_lib.lib().fastrrt_batch_log_paths(self._h, X_dev.data_ptr(),
                                                             labels_dev.data_ptr(), int(offset),
                                                             int(cap)), "batch_log_paths")

    def log_nodes(self, X_dev, labels_dev, offset, cap):
        """training rows of every accepted expansion (node of the final graph
        but the start) of the last collected list's solved requests"""
        return _lib.check(_lib.lib().fastrrt_batch_log_nodes(self._h, X_dev.data_ptr(),
                                                             labels_dev.data_ptr(), int(offset),
                                                             int(cap)), "batch_log_nodes")

    def profile(self, on=True):
        _lib.check(_lib.lib().fastrrt_batch_profile(self._h, int(on)), "batch_profile")

    def kernel_times(self):
        L = _lib.lib()
        k = L.fastrrt_kernel_count()
        ms = np.zeros(k, np.float64)
        n = np.zeros(k, np.int64)
        _lib.check(L.fastrrt_batch_kernel_times(self._h, ms, n), "kernel_times")
        return {L.fastrrt_kernel_name(i).decode(): (float(ms[i]), int(n[i])) for i in range(k)}

    def probes(self):
        a, g, p = _lib.C.c_uint64(), _lib.C.c_uint64(), _lib.C.c_uint64()
        _lib.check(_lib.lib().fastrrt_batch_probes(self._h, _lib.C.byref(a), _lib.C.byref(g),
                                                   _lib.C.byref(p)), "batch_probes")
        return {"k_expand": a.value, "k_goal": g.value, "k_gd_eval": p.value}

    def direct_connections(self, slot, W, H):
        """the goal direct connections of `slot`'s W x H cells evaluated so
        far: (flag uint8, 0 / 1 or 255 = not evaluated, cost, heading)"""
        flag = np.zeros(W * H, np.uint8)
        cost = np.zeros(W * H, np.float32)
        heading = np.zeros(W * H, np.float32)
        _lib.check(_lib.lib().fastrrt_batch_direct_connections(
            self._h, int(slot), flag.ctypes.data, cost.ctypes.data, heading.ctypes.data),
            "batch_direct_connections")
        return flag, cost, heading

    def release(self, slot):
        _lib.check(_lib.lib().fastrrt_batch_release(self._h, slot), "batch_release")
