"""Stand-ins for the pydriveless types the reference's Python layer takes
(angle, Waypoint, EgoParams, SearchParams, SearchFrame), with the builder
methods the reference's scripts call.  The driveless library itself is not
part of the reference tree; these classes carry exactly the fields that the
planner reads.
"""
import math

import numpy as np

from . import _lib


class angle:
    def __init__(self, rad=0.0):
        self._rad = float(rad)

    @staticmethod
    def new_rad(v):
        return angle(v)

    @staticmethod
    def new_deg(v):
        return angle(math.radians(v))

    def rad(self):
        return self._rad

    def deg(self):
        return math.degrees(self._rad)

    def __eq__(self, other):
        return isinstance(other, angle) and abs(self._rad - other._rad) < 1e-5

    def __repr__(self):
        return f"angle({self.deg():.4f} deg)"


class Waypoint:
    def __init__(self, x, z, heading=None):
        self.x = int(x)
        self.z = int(z)
        if heading is None:
            heading = angle(0.0)
        elif not isinstance(heading, angle):
            heading = angle(float(heading))
        self.heading = heading

    @staticmethod
    def distance_between(a, b):
        return math.hypot(b.x - a.x, b.z - a.z)

    def __repr__(self):
        return f"Waypoint({self.x}, {self.z}, {self.heading.rad():.4f})"


class SearchFrame:
    """A BEV frame on the GPU: class ids (H x W) and class costs (< 0 =
    obstacle), optionally traversability bits (the third SearchFrame
    channel)."""

    def __init__(self, width=None, height=None, class_ids=None, class_costs=None, trav=None):
        self._handle = None
        self.width = width
        self.height = height
        self.class_costs = None if class_costs is None else np.asarray(class_costs, np.float32)
        if class_ids is not None:
            self.set_class_ids(class_ids, trav)

    def set_class_costs(self, costs):
        self.class_costs = np.ascontiguousarray(costs, np.float32)

    def set_class_ids(self, class_ids, trav=None):
        cls = np.ascontiguousarray(class_ids, np.uint8)
        if self.class_costs is None:
            raise _lib.FastRRTError("SearchFrame needs class costs before its data")
        self.height, self.width = cls.shape
        self._release()
        t = None if trav is None else np.ascontiguousarray(trav, np.int32)
        h = _lib.lib().fastrrt_frame_create(self.width, self.height, cls.reshape(-1),
                                            self.class_costs, len(self.class_costs),
                                            None if t is None else t.ctypes.data)
        if not h:
            raise _lib.FastRRTError("frame: " + _lib.last_error())
        self._handle = h

    def set_frame_data(self, img):
        """The reference's float3 layout (H x W x 3): class id, distance, bits."""
        xyz = np.ascontiguousarray(img, np.float32)
        self.height, self.width = xyz.shape[:2]
        self._release()
        h = _lib.lib().fastrrt_frame_create_f3(self.width, self.height, xyz.reshape(-1),
                                               self.class_costs, len(self.class_costs))
        if not h:
            raise _lib.FastRRTError("frame: " + _lib.last_error())
        self._handle = h

    def get_cuda_ptr(self):
        if self._handle is None:
            raise _lib.FastRRTError("SearchFrame has no data")
        return self._handle

    # -- preprocessing (the driveless SearchFrame's, on the device) -------------
    def process_distance_to_goal(self, goal_x, goal_z):
        """fills the distance channel with every cell's distance to the goal"""
        _lib.check(_lib.lib().fastrrt_frame_process_distance_to_goal(self.get_cuda_ptr(), int(goal_x),
                                                                     int(goal_z)),
                   "process_distance_to_goal")

    def process_safe_distance_zone(self, min_dist):
        """sets traversability bit 0x100 where the (min_dist_x, min_dist_z)
        footprint holds no obstacle at any heading"""
        _lib.check(_lib.lib().fastrrt_frame_process_safe_zone(self.get_cuda_ptr(), int(min_dist[0]),
                                                              int(min_dist[1])),
                   "process_safe_distance_zone")

    def _flags(self):
        a, b = _lib.C.c_int(), _lib.C.c_int()
        _lib.check(_lib.lib().fastrrt_frame_flags(self.get_cuda_ptr(), _lib.C.byref(a), _lib.C.byref(b)),
                   "frame_flags")
        return bool(a.value), bool(b.value)

    def is_safe_zone_checked(self):
        return self._flags()[0]

    def is_distance_to_goal_processed(self):
        return self._flags()[1]

    def channels(self):
        """(distance, traversability) host copies, H x W each"""
        d = np.zeros((self.height, self.width), np.float32)
        t = np.zeros((self.height, self.width), np.int32)
        _lib.check(_lib.lib().fastrrt_frame_channels(self.get_cuda_ptr(), d.ctypes.data, t.ctypes.data),
                   "frame_channels")
        return d, t

    def _release(self):
        if self._handle is not None and _lib._lib is not None:
            _lib.lib().fastrrt_frame_destroy(self._handle)
        self._handle = None

    def __del__(self):
        try:
            self._release()
        except Exception:
            pass


class EgoParams:
    def __init__(self):
        self.search_frame_dimensions = (0, 0)
        self.search_frame_physical_dimensions = (1.0, 1.0)
        self.max_steering_angle = angle.new_deg(40)
        self.vehicle_length_m = 5.412658773
        self.max_curvature = -1.0
        self.ego_lower_bound = (-1, -1)
        self.ego_upper_bound = (-1, -1)
        self.segmentation_class_costs = np.zeros(0, np.float32)
        self.segmentation_class_colors = None

    @staticmethod
    def init(width, height):
        e = EgoParams()
        e.search_frame_dimensions = (int(width), int(height))
        return e

    def with_segmentation_class_costs(self, costs):
        self.segmentation_class_costs = np.asarray(costs, np.float32)
        return self

    def with_segmentation_class_colors(self, colors):
        self.segmentation_class_colors = colors
        return self

    def with_ego_lower_bound(self, v):
        self.ego_lower_bound = tuple(v)
        return self

    def with_ego_upper_bound(self, v):
        self.ego_upper_bound = tuple(v)
        return self

    def with_max_steering_angle(self, a):
        self.max_steering_angle = a
        return self

    def with_max_curvature(self, c):
        self.max_curvature = float(c)
        return self

    def with_search_physical_size(self, w, h):
        self.search_frame_physical_dimensions = (float(w), float(h))
        return self

    def with_vehicle_length(self, v):
        self.vehicle_length_m = float(v)
        return self

    def build(self):
        return self

    def new_search_frame(self):
        w, h = self.search_frame_dimensions
        return SearchFrame(w, h, class_costs=self.segmentation_class_costs)

    def new_search_params(self, start, goal):
        return SearchParams.init(start, goal)


class SearchParams:
    def __init__(self):
        self.start = Waypoint(0, 0)
        self.goal = Waypoint(0, 0)
        self.velocity_m_s = 1.0
        self.min_distance = (0, 0)
        self.timeout_ms = -1
        self.max_path_size_px = 40.0
        self.distance_to_goal_tolerance_px = 20.0
        self.heading_error_tolerance = angle.new_deg(10)
        self.frame = None

    @staticmethod
    def init(start, goal):
        p = SearchParams()
        p.start = start
        p.goal = goal
        return p

    def with_velocity(self, v):
        self.velocity_m_s = float(v)
        return self

    def with_min_distance(self, v):
        self.min_distance = tuple(v)
        return self

    def with_timeout(self, ms):
        self.timeout_ms = int(ms)
        return self

    def with_max_path_size(self, v):
        self.max_path_size_px = float(v)
        return self

    def with_distance_to_goal_tolerance(self, v):
        self.distance_to_goal_tolerance_px = float(v)
        return self

    def with_heading_error_tolerance(self, a):
        self.heading_error_tolerance = a
        return self

    def with_frame(self, f):
        self.frame = f
        return self

    def build(self):
        return self
