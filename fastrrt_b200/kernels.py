"""Per-candidate kernels of the planner behind the C ABI: kinematic expansion
(check_kinematic_new_path), Hermite connection (checkDirectConnectionToGoal)
and the footprint check (__computeFeasibleForAngle), over one frame."""
import ctypes as C

import numpy as np

from . import _lib


class Candidates:
    def __init__(self, frame, min_dist=(0, 0), lower_bound=(-1, -1), upper_bound=(-1, -1),
                 max_steering_rad=0.6981317007977318, lr_m=5.412658773 / 2, heading_grid=None,
                 cost_grid=None):
        self.frame = frame
        self._hg = None if heading_grid is None else np.ascontiguousarray(heading_grid, np.float32)
        self._cg = None if cost_grid is None else np.ascontiguousarray(cost_grid, np.float32)
        h = _lib.lib().fastrrt_candidates_create(
            frame.get_cuda_ptr(), int(min_dist[0]), int(min_dist[1]), int(lower_bound[0]),
            int(lower_bound[1]), int(upper_bound[0]), int(upper_bound[1]), float(max_steering_rad),
            float(lr_m), None if self._hg is None else self._hg.ctypes.data,
            None if self._cg is None else self._cg.ctypes.data)
        if not h:
            raise _lib.FastRRTError("candidates: " + _lib.last_error())
        self._h = h

    def __del__(self):
        try:
            if getattr(self, "_h", None) and _lib._lib is not None:
                _lib.lib().fastrrt_candidates_destroy(self._h)
                self._h = None
        except (AttributeError, TypeError):
            pass  # interpreter shutdown

    def kinematic(self, sx, sz, steer, length, velocity):
        n = len(sx)
        out = np.zeros(4 * n, np.float32)
        pr = C.c_uint64(0)
        _lib.check(_lib.lib().fastrrt_candidates_kinematic(
            self._h, n, np.ascontiguousarray(sx, np.int32), np.ascontiguousarray(sz, np.int32),
            np.ascontiguousarray(steer, np.float32), np.ascontiguousarray(length, np.float32),
            float(velocity), out, C.byref(pr)), "candidates_kinematic")
        return out.reshape(n, 4), pr.value

    def kinematic_device(self, sx, sz, steer, length, velocity, out, probes, stream=0):
        """Device pointers (e.g. torch tensors' data_ptr())."""
        return _lib.check(_lib.lib().fastrrt_candidates_kinematic_device(
            self._h, int(len_of(sx)), ptr(sx), ptr(sz), ptr(steer), ptr(length), float(velocity),
            ptr(out), ptr(probes), stream or None), "candidates_kinematic_device")

    def hermite(self, x, z, local_heading, gx, gz, goal_heading, max_curvature, safe=0):
        n = len(x)
        out = np.zeros(n, np.float32)
        pr = C.c_uint64(0)
        _lib.check(_lib.lib().fastrrt_candidates_hermite(
            self._h, n, np.ascontiguousarray(x, np.int32), np.ascontiguousarray(z, np.int32),
            np.ascontiguousarray(local_heading, np.float32), np.ascontiguousarray(gx, np.int32),
            np.ascontiguousarray(gz, np.int32), np.ascontiguousarray(goal_heading, np.float32),
            float(max_curvature), int(safe), out, C.byref(pr)), "candidates_hermite")
        return out, pr.value

    def hermite_device(self, x, z, local_heading, gx, gz, goal_heading, max_curvature, out, probes,
                       safe=0, stream=0):
        return _lib.check(_lib.lib().fastrrt_candidates_hermite_device(
            self._h, int(len_of(x)), ptr(x), ptr(z), ptr(local_heading), ptr(gx), ptr(gz),
            ptr(goal_heading), float(max_curvature), int(safe), ptr(out), ptr(probes),
            stream or None), "candidates_hermite_device")

    def feasible(self, x, z, angle_rad):
        n = len(x)
        out = np.zeros(n, np.int32)
        pr = C.c_uint64(0)
        _lib.check(_lib.lib().fastrrt_candidates_feasible(
            self._h, n, np.ascontiguousarray(x, np.int32), np.ascontiguousarray(z, np.int32),
            np.ascontiguousarray(angle_rad, np.float32), out, C.byref(pr)), "candidates_feasible")
        return out, pr.value


def ptr(t):
    return None if t is None else t.data_ptr()


def len_of(t):
    return t.numel() if hasattr(t, "numel") else len(t)
