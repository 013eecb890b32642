"""FastRRT planner: the reference's Python API (python_bind/app/pyfastrrt/src/
fastrrt.py:7-290) over libfastrrt_b200.so.

Two constructor forms are accepted:
  FastRRT(ego_params)                                   (pyfastrrt)
  FastRRT(search_frame=..., perception_width_m=..., perception_height_m=...,
          max_steering_angle_deg=..., vehicle_length_m=..., timeout_ms=...,
          min_dist_x=..., min_dist_z=..., path_costs=...)   (README.md:24-48)
and set_plan_data takes either a SearchParams or (cuda_ptr, start, goal,
velocity_m_s).
"""
import ctypes as C

import numpy as np

from . import _lib
from .driveless import EgoParams, SearchFrame, SearchParams, Waypoint, angle


class FastRRT:
    def __init__(self, ego_params=None, *, search_frame=None, perception_width_m=None,
                 perception_height_m=None, max_steering_angle_deg=None, vehicle_length_m=None,
                 timeout_ms=-1, min_dist_x=0, min_dist_z=0, path_costs=None,
                 lower_bound=(-1, -1), upper_bound=(-1, -1), max_curvature=-1.0,
                 max_path_size_px=40.0, dist_to_goal_tolerance_px=20.0,
                 heading_error_tolerance_deg=10.0, seed=None):
        L = _lib.lib()
        self._ptr = None
        if ego_params is None:
            if search_frame is None:
                raise _lib.FastRRTError("FastRRT needs ego_params or search_frame")
            ego_params = (EgoParams.init(search_frame.width, search_frame.height)
                          .with_search_physical_size(perception_width_m, perception_height_m)
                          .with_max_steering_angle(angle.new_deg(max_steering_angle_deg))
                          .with_vehicle_length(vehicle_length_m)
                          .with_ego_lower_bound(lower_bound)
                          .with_ego_upper_bound(upper_bound)
                          .with_max_curvature(max_curvature)
                          .with_segmentation_class_costs(
                              path_costs if path_costs is not None else search_frame.class_costs)
                          .build())
        self._ego = ego_params
        self._defaults = dict(timeout_ms=timeout_ms, min_distance=(min_dist_x, min_dist_z),
                              max_path_size_px=max_path_size_px,
                              dist_to_goal_tolerance_px=dist_to_goal_tolerance_px,
                              heading_error_tolerance=angle.new_deg(heading_error_tolerance_deg))
        path_costs = np.asarray(ego_params.segmentation_class_costs, np.float32)
        costs = np.ascontiguousarray(np.concatenate(([len(path_costs)], path_costs)),
                                     dtype=np.float32)
        w, h = ego_params.search_frame_dimensions
        pw, ph = ego_params.search_frame_physical_dimensions
        lb, ub = ego_params.ego_lower_bound, ego_params.ego_upper_bound
        ptr = L.fastrrt_initialize(w, h, pw, ph, ego_params.max_steering_angle.deg(),
                                   ego_params.vehicle_length_m, lb[0], lb[1], ub[0], ub[1], costs,
                                   ego_params.max_curvature)
        if not ptr:
            raise _lib.FastRRTError("fastrrt_initialize: " + _lib.last_error())
        self._ptr = ptr
        self._frame = None
        if seed is not None:
            self.set_seed(seed)

    def __del__(self):
        if getattr(self, "_ptr", None) and _lib._lib is not None:
            _lib.lib().fastrrt_destroy(self._ptr)
            self._ptr = None

    # -- planner API (fastrrt.py:172-290) --------------------------------------
    def set_frame_preprocessing(self, use=True):
        """the goal direct connections follow the frame's preprocessing flags
        (distance channel, safe zone) from the next set_plan_data on"""
        _lib.check(_lib.lib().fastrrt_set_frame_preprocessing(self._ptr, int(bool(use))),
                   "set_frame_preprocessing")

    def set_seed(self, seed):
        _lib.check(_lib.lib().fastrrt_set_seed(self._ptr, int(seed)), "set_seed")

    def set_plan_data(self, search_params=None, start=None, goal=None, velocity_m_s=None, *,
                      cuda_ptr=None):
        if search_params is None or not isinstance(search_params, SearchParams):
            if search_params is not None:       # README form: (cuda_ptr, start, goal, velocity)
                cuda_ptr = search_params
            d = self._defaults
            sp = (SearchParams.init(_wp(start), _wp(goal))
                  .with_velocity(velocity_m_s).with_min_distance(d["min_distance"])
                  .with_timeout(d["timeout_ms"]).with_max_path_size(d["max_path_size_px"])
                  .with_distance_to_goal_tolerance(d["dist_to_goal_tolerance_px"])
                  .with_heading_error_tolerance(d["heading_error_tolerance"])
                  .with_frame(cuda_ptr).build())
            search_params = sp
        frame = search_params.frame
        self._frame = frame            # keeps the device frame alive
        handle = frame.get_cuda_ptr() if isinstance(frame, SearchFrame) else frame
        s, g = search_params.start, search_params.goal
        md = search_params.min_distance
        _lib.lib().set_plan_data(self._ptr, handle, s.x, s.z, s.heading.rad(), g.x, g.z,
                                 g.heading.rad(), search_params.velocity_m_s, md[0], md[1],
                                 search_params.timeout_ms, search_params.max_path_size_px,
                                 search_params.distance_to_goal_tolerance_px,
                                 search_params.heading_error_tolerance.rad())
        err = _lib.last_error()
        if err:
            raise _lib.FastRRTError("set_plan_data: " + err)
        return True

    def search_init(self, copy_intrinsic_costs_from_frame=False):
        _lib.lib().search_init(self._ptr, copy_intrinsic_costs_from_frame)

    def loop(self, smart=False):
        return bool(_lib.lib().loop(self._ptr, smart))

    def path_optimize(self):
        return bool(_lib.lib().path_optimize(self._ptr))

    def goal_reached(self):
        return bool(_lib.lib().goal_reached(self._ptr))

    def get_planned_path(self, interpolate=False):
        L = _lib.lib()
        ptr = L.interpolate_planned_path(self._ptr) if interpolate else L.get_planned_path(self._ptr)
        if not ptr:
            raise _lib.FastRRTError("get_planned_path: " + _lib.last_error())
        res = _convert_path(ptr)
        L.release_planned_path_data(ptr)
        return res

    def get_planned_path_array(self, interpolate=False):
        """(n, 3) float32 array of (x, z, heading), empty when there is no path."""
        L = _lib.lib()
        ptr = L.interpolate_planned_path(self._ptr) if interpolate else L.get_planned_path(self._ptr)
        if not ptr:
            raise _lib.FastRRTError("get_planned_path: " + _lib.last_error())
        n = int(ptr[0])
        arr = np.ctypeslib.as_array(ptr, (3 * n + 1,))[1:].reshape(n, 3).copy()
        L.release_planned_path_data(ptr)
        return arr

    def interpolate_planned_path_p(self, path):
        path = np.ascontiguousarray(path, np.float32).reshape(-1)
        L = _lib.lib()
        ptr = L.interpolate_planned_path_p(self._ptr, path, len(path))
        res = _convert_path(ptr)
        L.release_planned_path_data(ptr)
        return res

    def build_ideal_curve(self, goal_x, goal_z, goal_heading):
        L = _lib.lib()
        ptr = L.ideal_curve(self._ptr, goal_x, goal_z, goal_heading)
        res = _convert_path(ptr)
        L.release_planned_path_data(ptr)
        return res

    def export_graph_nodes(self):
        L = _lib.lib()
        ptr = L.export_graph_nodes(self._ptr)
        size = ptr[0]
        if size == 0:
            L.release_export_graph_nodes(ptr)
            return None
        nodes = np.ctypeslib.as_array(ptr, (3 * size + 1,))[1:].reshape(size, 3).astype(np.int32)
        L.release_export_graph_nodes(ptr)
        return nodes

    def compute_region_debug_performance(self):
        _lib.lib().compute_region_debug_performance(self._ptr)

    def save_current_graph_state(self, filename):
        _lib.lib().save_current_graph_state(self._ptr, filename.encode("utf-8"))

    def load_graph_state(self, filename):
        _lib.lib().load_graph_state(self._ptr, filename.encode("utf-8"))

    # -- artificial potential fields (on the device) ---------------------------
    def compute_apf_repulsion(self, search_frame, kr, radius):
        """the repulsive field of the frame's obstacles added to the intrinsic costs"""
        _lib.check(_lib.lib().fastrrt_apf_repulsion(self._ptr, search_frame.get_cuda_ptr(), float(kr),
                                                    int(radius)), "apf_repulsion")

    def compute_apf_attraction(self, search_frame, ka, goal_x, goal_z):
        """the goal's attractive field added to the intrinsic costs"""
        _lib.check(_lib.lib().fastrrt_apf_attraction(self._ptr, search_frame.get_cuda_ptr(), float(ka),
                                                     int(goal_x), int(goal_z)), "apf_attraction")

    def get_intrinsic_costs(self):
        w, h = self._ego.search_frame_dimensions
        out = np.zeros(w * h, np.float32)
        _lib.check(_lib.lib().fastrrt_intrinsic_costs(self._ptr, out), "intrinsic_costs")
        return out.reshape(h, w)

    # -- validation (on the device) --------------------------------------------
    def check_graph_is_consistent(self):
        """CudaGraph::checkGraphIsConsistent of the planner's graph"""
        return bool(_lib.check(_lib.lib().fastrrt_check_graph_consistent(self._ptr),
                               "check_graph_consistent"))

    def validate_path(self, path):
        """the device path validator on an (n, 3) array of (x, z, heading)"""
        p = np.ascontiguousarray(np.asarray(path, np.float32).reshape(-1, 3))
        return bool(_lib.check(_lib.lib().fastrrt_validate_path(self._ptr, p.reshape(-1), len(p)),
                               "validate_path"))

    # -- instrumentation -------------------------------------------------------
    def probe_count(self):
        v = C.c_uint64(0)
        _lib.check(_lib.lib().fastrrt_probe_count(self._ptr, C.byref(v)), "probe_count")
        return v.value

    def loop_count(self):
        return _lib.check(_lib.lib().fastrrt_loop_count(self._ptr), "loop_count")


def _wp(v):
    if isinstance(v, Waypoint):
        return v
    return Waypoint(v[0], v[1], angle.new_rad(v[2] if len(v) > 2 else 0.0))


def _convert_path(ptr):
    """fastrrt.py:225-237: None when empty, else a list of Waypoint."""
    size = int(ptr[0])
    if size == 0:
        return None
    return [Waypoint(x=int(ptr[3 * i + 1]), z=int(ptr[3 * i + 2]), heading=angle.new_rad(ptr[3 * i + 3]))
            for i in range(size)]
