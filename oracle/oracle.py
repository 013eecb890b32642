"""ctypes bindings for the CPU oracle (liboracle.so) and for the reference's
own sources compiled by oracle/ref/Makefile (oracle/_ref/libfastrrt_ref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product package.
"""
import ctypes as C
import os

import numpy as np

from . import build_oracle

HERE = os.path.dirname(os.path.abspath(__file__))

NULL, NODE, TEMP, PROCESSING, COLLISION, CONNECT_TO_GOAL = range(6)
FP_HOST, FP_DEVICE = 0, 1


class OrcFrame(C.Structure):
    _fields_ = [("W", C.c_int), ("H", C.c_int), ("cls", C.POINTER(C.c_uint8)),
                ("class_costs", C.POINTER(C.c_float)), ("n_classes", C.c_int),
                ("trav", C.POINTER(C.c_int32)), ("dist", C.POINTER(C.c_float))]


class OrcSearch(C.Structure):
    _fields_ = [("W", C.c_int), ("H", C.c_int), ("mdx", C.c_int), ("mdz", C.c_int),
                ("lbx", C.c_int), ("lbz", C.c_int), ("ubx", C.c_int), ("ubz", C.c_int)]


class OrcPhysical(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("rate_w", "inv_rate_w", "rate_h", "inv_rate_h",
                                           "max_steer_rad", "max_steer_deg", "lr",
                                           "max_curvature")]


class OrcGraph(C.Structure):
    _fields_ = [("W", C.c_int), ("H", C.c_int),
                ("px", C.POINTER(C.c_int32)), ("pz", C.POINTER(C.c_int32)),
                ("type", C.POINTER(C.c_int32)), ("child", C.POINTER(C.c_int32)),
                ("heading", C.POINTER(C.c_float)), ("cost", C.POINTER(C.c_float)),
                ("intrinsic", C.POINTER(C.c_float)), ("direct", C.POINTER(C.c_float)),
                ("gd_flag", C.POINTER(C.c_float)), ("gd_heading", C.POINTER(C.c_float)),
                ("gd_cost", C.POINTER(C.c_float)),
                ("og_x", C.c_float), ("og_z", C.c_float), ("og_h", C.c_float),
                ("goal_reached", C.c_int), ("node_collision", C.c_int),
                ("density_w", C.c_int), ("density_h", C.c_int), ("density_size", C.c_int),
                ("region_count", C.POINTER(C.c_uint32)),
                ("sp", OrcSearch), ("pp", OrcPhysical), ("has_pp", C.c_int)]


class OrcF4(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float), ("w", C.c_float)]


class OrcPlanParams(C.Structure):
    _fields_ = [("start_x", C.c_int), ("start_z", C.c_int), ("start_heading", C.c_float),
                ("goal_x", C.c_int), ("goal_z", C.c_int), ("goal_heading", C.c_float),
                ("velocity", C.c_float), ("max_path_size", C.c_float),
                ("dist_tol", C.c_float), ("heading_tol", C.c_float), ("seed", C.c_uint64)]


class OrcPlanner(C.Structure):
    _fields_ = [("g", C.POINTER(OrcGraph)), ("f", C.POINTER(OrcFrame)), ("pp", OrcPlanParams),
                ("last_expanded", C.c_int), ("iter", C.c_uint32), ("smart", C.c_int),
                ("has_plan", C.c_int), ("probes", C.c_longlong), ("probes_goal", C.c_longlong),
                ("probes_pre", C.c_longlong)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = build_oracle.ORACLE_SO
        if not os.path.exists(path):
            build_oracle.build_oracle()
        L = C.CDLL(path)
        P = C.POINTER
        i32p = np.ctypeslib.ndpointer(np.int32, flags="C")
        f32p = np.ctypeslib.ndpointer(np.float32, flags="C")
        i64p = np.ctypeslib.ndpointer(np.int64, flags="C")
        u8p = np.ctypeslib.ndpointer(np.uint8, flags="C")
        u64p = np.ctypeslib.ndpointer(np.uint64, flags="C")
        f64p = np.ctypeslib.ndpointer(np.float64, flags="C")
        sig = {
            "orc_set_fp_mode": (None, [C.c_int]),
            "orc_get_fp_mode": (C.c_int, []),
            "orc_philox4x32": (None, [C.c_uint32] * 6 + [P(C.c_uint32)]),
            "orc_u01": (C.c_float, [C.c_uint32]),
            "orc_draw_expansion": (None, [C.c_uint64, C.c_uint32, C.c_uint32, C.c_float,
                                          C.c_float, P(C.c_float), P(C.c_float)]),
            "orc_physical_params": (None, [P(OrcPhysical), C.c_int, C.c_int, C.c_float,
                                           C.c_float, C.c_double, C.c_float, C.c_float]),
            "orc_search_params": (None, [P(OrcSearch)] + [C.c_int] * 8),
            "orc_feasible": (C.c_int, [P(OrcFrame), P(OrcSearch), C.c_int, C.c_int, C.c_float,
                                       P(C.c_longlong)]),
            "orc_kinematic_path": (OrcF4, [P(OrcGraph), P(OrcFrame), C.c_int, C.c_int, C.c_float,
                                           C.c_float, C.c_float, P(C.c_longlong), P(C.c_int)]),
            "orc_kinematic_f64_pose": (None, [P(OrcGraph), C.c_int, C.c_int, C.c_float, C.c_float,
                                              C.c_int, P(C.c_double)]),
            "orc_kinematic_f32_pose": (None, [P(OrcGraph), C.c_int, C.c_int, C.c_float, C.c_float,
                                              C.c_int, P(C.c_double)]),
            "orc_direct_connection": (C.c_float, [P(OrcGraph), P(OrcFrame), P(OrcSearch),
                                                  C.c_float, C.c_int, C.c_int, C.c_float,
                                                  C.c_int, C.c_int, C.c_float, C.c_int,
                                                  P(C.c_longlong)]),
            "orc_hermite_test": (C.c_float, [P(OrcGraph), P(OrcFrame), P(C.c_float), C.c_int,
                                             C.c_int, C.c_int, C.c_int, C.c_float, C.c_int,
                                             C.c_float, P(C.c_longlong)]),
            "orc_compute_heading": (C.c_double, [C.c_int] * 4),
            "orc_kinematic_connection": (C.c_int, [P(OrcGraph), P(OrcFrame), C.c_int, C.c_int,
                                                   C.c_int, C.c_int, C.c_float, P(C.c_double),
                                                   P(C.c_double)]),
            "orc_max_curvature_default": (C.c_float, [C.c_float, C.c_float]),
            "orc_graph_new": (P(OrcGraph), [C.c_int, C.c_int]),
            "orc_graph_free": (None, [P(OrcGraph)]),
            "orc_graph_set_coordinate_start": (None, [P(OrcGraph), C.c_int, C.c_int, C.c_float]),
            "orc_graph_add": (None, [P(OrcGraph), C.c_int, C.c_int, C.c_float, C.c_int, C.c_int,
                                     C.c_float]),
            "orc_graph_add_temporary": (None, [P(OrcGraph), C.c_int, C.c_int, C.c_float, C.c_int,
                                               C.c_int, C.c_float]),
            "orc_graph_remove": (None, [P(OrcGraph), C.c_int, C.c_int]),
            "orc_graph_clear": (None, [P(OrcGraph)]),
            "orc_graph_count": (C.c_uint32, [P(OrcGraph), C.c_int]),
            "orc_graph_count_all": (C.c_uint32, [P(OrcGraph)]),
            "orc_graph_set_collision": (None, [P(OrcGraph), C.c_int, C.c_int, C.c_int, C.c_int,
                                               C.c_float, C.c_float]),
            "orc_graph_get_parent": (None, [P(OrcGraph), C.c_int, C.c_int, P(C.c_int),
                                            P(C.c_int)]),
            "orc_graph_solve_collisions": (None, [P(OrcGraph)]),
            "orc_graph_accept": (None, [P(OrcGraph)]),
            "orc_graph_density": (None, [P(OrcGraph)]),
            "orc_graph_check_goal_reached": (C.c_int, [P(OrcGraph), P(OrcFrame), C.c_int, C.c_int,
                                                       C.c_float, C.c_float, C.c_float]),
            "orc_graph_find_best_node": (C.c_int, [P(OrcGraph), P(OrcFrame), C.c_float, C.c_float,
                                                   C.c_int, C.c_int, C.c_float, P(C.c_int),
                                                   P(C.c_int)]),
            "orc_graph_is_consistent": (C.c_int, [P(OrcGraph)]),
            "orc_graph_process_direct_goal": (None, [P(OrcGraph), P(OrcFrame), P(OrcSearch),
                                                     C.c_int, C.c_int, C.c_float, C.c_float,
                                                     P(C.c_longlong)]),
            "orc_graph_best_goal_connection": (C.c_int, [P(OrcGraph), P(OrcFrame), C.c_float,
                                                         C.c_int, P(OrcF4), P(C.c_longlong)]),
            "orc_graph_expand": (C.c_int, [P(OrcGraph), P(OrcFrame), C.c_uint64, C.c_uint32,
                                           C.c_float, C.c_float, C.c_int, C.c_int, C.c_int,
                                           P(C.c_longlong)]),
            "orc_planner_new": (P(OrcPlanner), [C.c_int, C.c_int, C.c_float, C.c_float, C.c_float,
                                                C.c_float, C.c_int, C.c_int, C.c_int, C.c_int,
                                                C.c_float]),
            "orc_planner_free": (None, [P(OrcPlanner)]),
            "orc_planner_set_plan_data": (None, [P(OrcPlanner), P(OrcFrame), P(OrcPlanParams),
                                                 C.c_int, C.c_int]),
            "orc_planner_search_init": (None, [P(OrcPlanner)]),
            "orc_planner_loop": (C.c_int, [P(OrcPlanner), C.c_int]),
            "orc_planner_goal_reached": (C.c_int, [P(OrcPlanner)]),
            "orc_planner_path": (C.c_int, [P(OrcPlanner), f32p, C.c_int]),
            "orc_planner_optimize": (C.c_int, [P(OrcPlanner)]),
            "orc_interpolate": (C.c_int, [f32p, C.c_int, C.c_int, C.c_int, f32p, C.c_int]),
            "orc_plan": (C.c_int, [P(OrcPlanner), C.c_int, C.c_int, P(C.c_int)]),
            "orc_validate_path": (C.c_int, [P(OrcPlanner), f32p, C.c_int]),
            "orc_validate_waypoints": (C.c_int, [P(OrcPlanner), f32p, C.c_int]),
            "orc_kinematic_batch": (None, [P(OrcGraph), P(OrcFrame), C.c_int, i32p, i32p, f32p,
                                           f32p, C.c_float, f32p, i64p, i32p]),
            "orc_feasible_batch": (None, [P(OrcFrame), P(OrcSearch), C.c_int, i32p, i32p, f32p,
                                          i32p, i64p]),
            "orc_direct_batch": (None, [P(OrcGraph), P(OrcFrame), P(OrcSearch), C.c_float, C.c_int,
                                        i32p, i32p, f32p, i32p, i32p, f32p, C.c_int, f32p, i64p]),
            "orc_plan_batch": (C.c_int, [C.c_int, C.c_int, C.c_int, u8p, f32p, C.c_int, i32p, u64p,
                                         C.c_float, C.c_float, C.c_float, C.c_float, C.c_int,
                                         C.c_int, C.c_float, C.c_float, C.c_float, C.c_float,
                                         C.c_int, C.c_int, C.c_int, C.c_int, i32p, i32p, f32p,
                                         f64p]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def set_fp_mode(mode):
    lib().orc_set_fp_mode(mode)


class Frame:
    """Class-id frame + class-cost table (+ optional traversability bits)."""

    def __init__(self, cls, class_costs, trav=None, dist=None):
        self.cls = np.ascontiguousarray(cls, dtype=np.uint8)
        self.H, self.W = self.cls.shape
        self.costs = np.ascontiguousarray(class_costs, dtype=np.float32)
        self.trav = None if trav is None else np.ascontiguousarray(trav, dtype=np.int32)
        self.dist = None if dist is None else np.ascontiguousarray(dist, dtype=np.float32)
        self.s = OrcFrame(self.W, self.H, self.cls.ctypes.data_as(C.POINTER(C.c_uint8)),
                          self.costs.ctypes.data_as(C.POINTER(C.c_float)), len(self.costs),
                          None if self.trav is None else
                          self.trav.ctypes.data_as(C.POINTER(C.c_int32)),
                          None if self.dist is None else
                          self.dist.ctypes.data_as(C.POINTER(C.c_float)))

    def xyz(self):
        """float3 frame as the reference's SearchFrame stores it"""
        out = np.zeros((self.H, self.W, 3), np.float32)
        out[..., 0] = self.cls
        if self.dist is not None:
            out[..., 1] = self.dist.reshape(self.H, self.W)
        if self.trav is not None:
            out[..., 2] = self.trav.reshape(self.H, self.W)
        return out


def search(W, H, min_dist_x, min_dist_z, lb=(-1, -1), ub=(-1, -1)):
    sp = OrcSearch()
    lib().orc_search_params(C.byref(sp), W, H, min_dist_x, min_dist_z, lb[0], lb[1], ub[0], ub[1])
    return sp


class Graph:
    """Owning wrapper of an orc_graph with numpy views of its arrays."""

    def __init__(self, W, H, pw_m=None, ph_m=None, max_steer_deg=40.0, vehicle_len=5.412658773,
                 max_curvature=-1.0, min_dist=(0, 0), lb=(-1, -1), ub=(-1, -1)):
        L = lib()
        self.p = L.orc_graph_new(W, H)
        self.g = self.p.contents
        self.W, self.H = W, H
        if pw_m is not None:
            L.orc_physical_params(C.byref(self.g.pp), W, H, pw_m, ph_m,
                                  float(np.float32(max_steer_deg)) * np.pi / 180.0,
                                  vehicle_len, max_curvature)
            self.g.has_pp = 1
        L.orc_search_params(C.byref(self.g.sp), W, H, min_dist[0], min_dist[1], lb[0], lb[1],
                            ub[0], ub[1])
        n = W * H
        self.px = np.ctypeslib.as_array(self.g.px, (n,))
        self.pz = np.ctypeslib.as_array(self.g.pz, (n,))
        self.type = np.ctypeslib.as_array(self.g.type, (n,))
        self.child = np.ctypeslib.as_array(self.g.child, (n,))
        self.heading = np.ctypeslib.as_array(self.g.heading, (n,))
        self.cost = np.ctypeslib.as_array(self.g.cost, (n,))
        self.intrinsic = np.ctypeslib.as_array(self.g.intrinsic, (n,))
        self.gd_flag = np.ctypeslib.as_array(self.g.gd_flag, (n,))
        self.gd_heading = np.ctypeslib.as_array(self.g.gd_heading, (n,))
        self.gd_cost = np.ctypeslib.as_array(self.g.gd_cost, (n,))

    def __del__(self):
        if getattr(self, "p", None):
            lib().orc_graph_free(self.p)
            self.p = None

    def add(self, x, z, heading, ppx, ppz, cost):
        lib().orc_graph_add(self.p, x, z, heading, ppx, ppz, cost)

    def add_temporary(self, x, z, heading, ppx, ppz, cost):
        lib().orc_graph_add_temporary(self.p, x, z, heading, ppx, ppz, cost)

    def set_collision(self, x, z, npx, npz, heading, cost):
        lib().orc_graph_set_collision(self.p, x, z, npx, npz, heading, cost)

    def solve_collisions(self):
        lib().orc_graph_solve_collisions(self.p)

    def accept(self):
        lib().orc_graph_accept(self.p)

    def clear(self):
        lib().orc_graph_clear(self.p)

    def count(self, t=NODE):
        return lib().orc_graph_count(self.p, t)

    def count_all(self):
        return lib().orc_graph_count_all(self.p)

    def parent(self, x, z):
        a, b = C.c_int(), C.c_int()
        lib().orc_graph_get_parent(self.p, x, z, C.byref(a), C.byref(b))
        return a.value, b.value

    def type_at(self, x, z):
        return int(self.type[z * self.W + x])

    def child_at(self, x, z):
        return int(self.child[z * self.W + x])

    def heading_at(self, x, z):
        return float(self.heading[z * self.W + x])

    def consistent(self):
        return bool(lib().orc_graph_is_consistent(self.p))

    def goal_reached(self, frame, gx, gz, gh, tol, max_err):
        return bool(lib().orc_graph_check_goal_reached(self.p, C.byref(frame.s), gx, gz, gh, tol,
                                                       max_err))

    def best_node(self, frame, heading, radius, x, z, max_err):
        a, b = C.c_int(), C.c_int()
        lib().orc_graph_find_best_node(self.p, C.byref(frame.s), heading, radius, x, z, max_err,
                                       C.byref(a), C.byref(b))
        return a.value, b.value

    def derive(self, frame, x, z, steering, path_size, velocity):
        """CudaGraph::derivateNode (graph_expansion.cu:224-244) for one node"""
        return lib().orc_kinematic_path(self.p, C.byref(frame.s), x, z, steering, path_size,
                                        velocity, None, None)

    def process_direct_goal(self, frame, gx, gz, gh, max_curvature=-1.0, sp=None):
        pr = C.c_longlong(0)
        lib().orc_graph_process_direct_goal(self.p, C.byref(frame.s),
                                            C.byref(sp if sp is not None else self.g.sp),
                                            gx, gz, gh, max_curvature, C.byref(pr))
        return pr.value

    def kinematic_batch(self, frame, sx, sz, steer, length, velocity):
        n = len(sx)
        out = np.zeros((n, 4), np.float32)
        probes = np.zeros(n, np.int64)
        steps = np.zeros(n, np.int32)
        lib().orc_kinematic_batch(self.p, C.byref(frame.s), n, np.ascontiguousarray(sx, np.int32),
                                  np.ascontiguousarray(sz, np.int32),
                                  np.ascontiguousarray(steer, np.float32),
                                  np.ascontiguousarray(length, np.float32), velocity,
                                  out.reshape(-1), probes, steps)
        return out, probes, steps

    def direct_batch(self, frame, maxc, x, z, lh, gx, gz, gh, safe=0, sp=None):
        n = len(x)
        out = np.zeros(n, np.float32)
        probes = np.zeros(n, np.int64)
        lib().orc_direct_batch(self.p, C.byref(frame.s), C.byref(sp if sp is not None else self.g.sp),
                               maxc, n, np.ascontiguousarray(x, np.int32),
                               np.ascontiguousarray(z, np.int32), np.ascontiguousarray(lh, np.float32),
                               np.ascontiguousarray(gx, np.int32), np.ascontiguousarray(gz, np.int32),
                               np.ascontiguousarray(gh, np.float32), safe, out, probes)
        return out, probes


def feasible_batch(frame, sp, x, z, a):
    n = len(x)
    out = np.zeros(n, np.int32)
    probes = np.zeros(n, np.int64)
    lib().orc_feasible_batch(C.byref(frame.s), C.byref(sp), n, np.ascontiguousarray(x, np.int32),
                             np.ascontiguousarray(z, np.int32), np.ascontiguousarray(a, np.float32),
                             out, probes)
    return out, probes


def draw_expansion(seed, pos, it, max_steer, max_path):
    s, l = C.c_float(), C.c_float()
    lib().orc_draw_expansion(seed, pos, it, max_steer, max_path, C.byref(s), C.byref(l))
    return s.value, l.value


class Planner:
    """Oracle FastRRT (fastrrt.cpp:35-232) on one frame."""

    def __init__(self, frame, pw_m=34.56, ph_m=34.56, max_steer_deg=40.0, vehicle_len=5.4,
                 lb=(-1, -1), ub=(-1, -1), max_curvature=-1.0):
        self.frame = frame
        self.p = lib().orc_planner_new(frame.W, frame.H, pw_m, ph_m, max_steer_deg, vehicle_len,
                                       lb[0], lb[1], ub[0], ub[1], max_curvature)
        g = self.p.contents.g.contents
        n = frame.W * frame.H
        self.type = np.ctypeslib.as_array(g.type, (n,))
        self.heading = np.ctypeslib.as_array(g.heading, (n,))
        self.cost = np.ctypeslib.as_array(g.cost, (n,))
        self.px = np.ctypeslib.as_array(g.px, (n,))
        self.pz = np.ctypeslib.as_array(g.pz, (n,))
        self.child = np.ctypeslib.as_array(g.child, (n,))
        self.intrinsic = np.ctypeslib.as_array(g.intrinsic, (n,))
        self.gd_flag = np.ctypeslib.as_array(g.gd_flag, (n,))
        self.gd_heading = np.ctypeslib.as_array(g.gd_heading, (n,))
        self.gd_cost = np.ctypeslib.as_array(g.gd_cost, (n,))

    def __del__(self):
        if getattr(self, "p", None):
            lib().orc_planner_free(self.p)
            self.p = None

    def set_plan_data(self, start, goal, velocity, min_dist, max_path=40.0, dist_tol=20.0,
                      heading_tol=None, seed=0):
        if heading_tol is None:
            heading_tol = float(np.float32(10.0 * np.pi / 180.0))
        self.pp = OrcPlanParams(start[0], start[1], start[2], goal[0], goal[1], goal[2], velocity,
                                max_path, dist_tol, heading_tol, seed)
        lib().orc_planner_set_plan_data(self.p, C.byref(self.frame.s), C.byref(self.pp),
                                        min_dist[0], min_dist[1])

    def search_init(self):
        lib().orc_planner_search_init(self.p)

    def loop(self, smart=False):
        return bool(lib().orc_planner_loop(self.p, int(smart)))

    def goal_reached(self):
        return bool(lib().orc_planner_goal_reached(self.p))

    def path(self, cap=4096):
        buf = np.zeros(3 * cap, np.float32)
        n = lib().orc_planner_path(self.p, buf, cap)
        return buf[:3 * n].reshape(n, 3).copy()

    def optimize(self):
        return bool(lib().orc_planner_optimize(self.p))

    def validate(self, path):
        path = np.ascontiguousarray(path, np.float32).reshape(-1)
        return bool(lib().orc_validate_path(self.p, path, len(path) // 3))

    def validate_waypoints(self, path):
        """the validator's checks that do not read this planner's graph"""
        path = np.ascontiguousarray(path, np.float32).reshape(-1)
        return bool(lib().orc_validate_waypoints(self.p, path, len(path) // 3))

    def plan(self, smart=False, max_iter=1000):
        it = C.c_int(0)
        ok = lib().orc_plan(self.p, int(smart), max_iter, C.byref(it))
        return bool(ok), it.value

    @property
    def probes(self):
        c = self.p.contents
        return c.probes + c.probes_goal + c.probes_pre

    @property
    def probes_by_phase(self):
        """expansion (+ optimisation), goal-connection search, precompute"""
        c = self.p.contents
        return {"expand": c.probes, "goal": c.probes_goal, "pre": c.probes_pre}

    @property
    def iterations(self):
        return self.p.contents.iter


def interpolate(path, W, H, cap=1 << 16):
    path = np.ascontiguousarray(path, np.float32).reshape(-1)
    out = np.zeros(3 * cap, np.float32)
    m = lib().orc_interpolate(path, len(path) // 3, W, H, out, cap)
    return out[:3 * m].reshape(m, 3).copy()


def plan_batch(cls, class_costs, start_goal, seeds, *, pw_m, ph_m, max_steer_deg, vehicle_len,
               min_dist, velocity, max_path, dist_tol, heading_tol, timeout_ms, max_iter,
               smart=False, threads=0):
    """CPU baseline: plans len(seeds) frames with OpenMP; start_goal rows are
    (sx, sz, sh*1e6, gx, gz, gh*1e6) int32."""
    cls = np.ascontiguousarray(cls, np.uint8)
    n, H, W = cls.shape
    ok = np.zeros(n, np.int32)
    iters = np.zeros(n, np.int32)
    cost = np.zeros(n, np.float32)
    ms = np.zeros(n, np.float64)
    lib().orc_plan_batch(n, W, H, cls.reshape(-1), np.ascontiguousarray(class_costs, np.float32),
                         len(class_costs), np.ascontiguousarray(start_goal, np.int32).reshape(-1),
                         np.ascontiguousarray(seeds, np.uint64), pw_m, ph_m, max_steer_deg,
                         vehicle_len, min_dist[0], min_dist[1], velocity, max_path, dist_tol,
                         heading_tol, timeout_ms, max_iter, int(smart), threads, ok, iters, cost, ms)
    return ok, iters, cost, ms


# --------------------------------------------------------------------------
# the reference's own sources (oracle/_ref), host and device entry points
# --------------------------------------------------------------------------
_ref = None


def ref_lib():
    """Loads oracle/_ref/libfastrrt_ref.so, or returns None when absent."""
    global _ref
    if _ref is None:
        path = build_oracle.REF_SO
        if not os.path.exists(path):
            return None
        L = C.CDLL(path)
        f32p = np.ctypeslib.ndpointer(np.float32, flags="C")
        i32p = np.ctypeslib.ndpointer(np.int32, flags="C")
        common = [C.c_int, C.c_int, f32p, f32p, C.c_int, f32p, f32p, C.c_double, C.c_double] + \
            [C.c_int] * 6 + [C.c_float, C.c_float]
        for pre in ("ref_h_", "ref_d_"):
            getattr(L, pre + "kinematic").argtypes = common + [C.c_int, i32p, i32p, f32p, f32p,
                                                               C.c_float, f32p]
            getattr(L, pre + "kinematic").restype = C.c_int
            getattr(L, pre + "feasible").argtypes = common + [C.c_int, i32p, i32p, f32p, i32p]
            getattr(L, pre + "feasible").restype = C.c_int
            getattr(L, pre + "direct").argtypes = common + [C.c_float, C.c_int, i32p, i32p, f32p,
                                                            i32p, i32p, f32p, C.c_int, f32p]
            getattr(L, pre + "direct").restype = C.c_int
        L.ref_h_compute_heading.argtypes = [C.c_int] * 4
        L.ref_h_compute_heading.restype = C.c_float
        L.ref_d_compute_heading.argtypes = [C.c_int, i32p, i32p, i32p, i32p, f32p]
        L.ref_d_compute_heading.restype = C.c_int
        L.ref_frame_new.argtypes = [C.c_int, C.c_int, f32p, f32p, C.c_int] + [C.c_int] * 6
        L.ref_frame_new.restype = C.c_void_p
        L.ref_frame_free.argtypes = [C.c_void_p]
        L.ref_frame_free.restype = None
        _ref = L
    return _ref


class RefCase:
    """Inputs shared by the reference per-candidate entry points."""

    def __init__(self, frame, heading=None, cost=None, max_steer_rad=None, lr=None, mdx=0, mdz=0,
                 lb=(-1, -1), ub=(-1, -1), og=None):
        self.W, self.H = frame.W, frame.H
        self.xyz = np.ascontiguousarray(frame.xyz().reshape(-1))
        self.costs = frame.costs
        n = self.W * self.H
        self.heading = np.zeros(n, np.float32) if heading is None else \
            np.ascontiguousarray(heading, np.float32).reshape(-1)
        self.cost = np.zeros(n, np.float32) if cost is None else \
            np.ascontiguousarray(cost, np.float32).reshape(-1)
        self.max_steer = float(max_steer_rad or 0.0)
        self.lr = float(lr or 1.0)
        self.md = (mdx, mdz)
        self.lb, self.ub = lb, ub
        self.og = og if og is not None else (float(self.W // 2), float(self.H // 2))

    def args(self):
        return (self.W, self.H, self.xyz, self.costs, len(self.costs), self.heading, self.cost,
                self.max_steer, self.lr, self.md[0], self.md[1], self.lb[0], self.lb[1],
                self.ub[0], self.ub[1], self.og[0], self.og[1])

    def kinematic(self, sx, sz, steer, length, velocity, device=False):
        L = ref_lib()
        n = len(sx)
        out = np.zeros(4 * n, np.float32)
        fn = L.ref_d_kinematic if device else L.ref_h_kinematic
        rc = fn(*self.args(), n, np.ascontiguousarray(sx, np.int32),
                np.ascontiguousarray(sz, np.int32), np.ascontiguousarray(steer, np.float32),
                np.ascontiguousarray(length, np.float32), velocity, out)
        if rc != 0:
            raise RuntimeError("reference kinematic entry point failed")
        return out.reshape(n, 4)

    def feasible(self, x, z, a, device=False):
        L = ref_lib()
        n = len(x)
        out = np.zeros(n, np.int32)
        fn = L.ref_d_feasible if device else L.ref_h_feasible
        rc = fn(*self.args(), n, np.ascontiguousarray(x, np.int32), np.ascontiguousarray(z, np.int32),
                np.ascontiguousarray(a, np.float32), out)
        if rc != 0:
            raise RuntimeError("reference feasibility entry point failed")
        return out

    def direct(self, maxc, x, z, lh, gx, gz, gh, safe=0, device=False):
        L = ref_lib()
        n = len(x)
        out = np.zeros(n, np.float32)
        fn = L.ref_d_direct if device else L.ref_h_direct
        rc = fn(*self.args(), maxc, n, np.ascontiguousarray(x, np.int32),
                np.ascontiguousarray(z, np.int32), np.ascontiguousarray(lh, np.float32),
                np.ascontiguousarray(gx, np.int32), np.ascontiguousarray(gz, np.int32),
                np.ascontiguousarray(gh, np.float32), safe, out)
        if rc != 0:
            raise RuntimeError("reference direct-connection entry point failed")
        return out


class RefPlanner:
    """The reference's own FastRRT (src/fastrrt.cpp) through its C ABI
    (src/python_bind.cpp) in oracle/_ref, on the GPU.  Its RNG is seeded from
    the wall clock (random_number_gen.cu:40), so runs are not repeatable."""

    def __init__(self, cls, class_costs, pw_m, ph_m, max_steer_deg, vehicle_len,
                 lb=(-1, -1), ub=(-1, -1), max_curvature=-1.0):
        L = ref_lib()
        self.L = L
        for name, res, args in [
            ("fastrrt_initialize", C.c_void_p, [C.c_int, C.c_int, C.c_float, C.c_float, C.c_float,
                                                C.c_float, C.c_int, C.c_int, C.c_int, C.c_int,
                                                C.c_void_p, C.c_float]),
            ("fastrrt_destroy", None, [C.c_void_p]),
            ("set_plan_data", None, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_int,
                                     C.c_int, C.c_float, C.c_float, C.c_int, C.c_int, C.c_int,
                                     C.c_float, C.c_float, C.c_float]),
            ("goal_reached", C.c_bool, [C.c_void_p]),
            ("search_init", None, [C.c_void_p, C.c_bool]),
            ("loop", C.c_bool, [C.c_void_p, C.c_bool]),
            ("path_optimize", C.c_bool, [C.c_void_p]),
            ("get_planned_path", C.POINTER(C.c_float), [C.c_void_p]),
            ("release_planned_path_data", None, [C.POINTER(C.c_float)]),
            ("save_current_graph_state", None, [C.c_void_p, C.c_char_p])]:
            getattr(L, name).restype = res
            getattr(L, name).argtypes = args
        cls = np.ascontiguousarray(cls, np.uint8)
        self.H, self.W = cls.shape
        xyz = np.zeros((self.H, self.W, 3), np.float32)
        xyz[..., 0] = cls
        self.costs = np.ascontiguousarray(class_costs, np.float32)
        self._xyz = np.ascontiguousarray(xyz.reshape(-1))
        self.lb, self.ub = lb, ub
        head = np.ascontiguousarray(np.concatenate(([len(self.costs)], self.costs)), np.float32)
        self.p = L.fastrrt_initialize(self.W, self.H, pw_m, ph_m, max_steer_deg, vehicle_len,
                                      lb[0], lb[1], ub[0], ub[1], head.ctypes.data, max_curvature)
        self.frame = None

    def set_plan_data(self, start, goal, velocity, min_dist, timeout_ms=-1, max_path=40.0,
                      dist_tol=20.0, heading_tol=None):
        if heading_tol is None:
            heading_tol = float(np.float32(np.radians(10.0)))
        mdx, mdz = int(float(np.float32(min_dist[0]) / 2)), int(float(np.float32(min_dist[1]) / 2))
        if self.frame is not None:
            self.L.ref_frame_free(self.frame)
        self.frame = self.L.ref_frame_new(self.W, self.H, self._xyz, self.costs, len(self.costs),
                                          self.lb[0], self.lb[1], self.ub[0], self.ub[1], mdx, mdz)
        self.L.set_plan_data(self.p, self.frame, start[0], start[1], start[2], goal[0], goal[1],
                             goal[2], velocity, min_dist[0], min_dist[1], timeout_ms, max_path,
                             dist_tol, heading_tol)

    def plan(self, smart=False, max_iter=1000):
        self.L.search_init(self.p, False)
        it = 0
        while not self.L.goal_reached(self.p) and it < max_iter:
            it += 1
            if not self.L.loop(self.p, smart):
                break
        return bool(self.L.goal_reached(self.p)), it

    def save_graph(self, filename):
        """the reference's graph dump (CudaGraph::dumpGraph, graph.cu:496-520)"""
        self.L.save_current_graph_state(self.p, filename.encode("utf-8"))

    def path(self):
        ptr = self.L.get_planned_path(self.p)
        n = int(ptr[0])
        arr = np.array([ptr[1 + i] for i in range(3 * n)], np.float32).reshape(n, 3)
        self.L.release_planned_path_data(ptr)
        return arr

    def __del__(self):
        try:
            if self.frame is not None:
                self.L.ref_frame_free(self.frame)
            self.L.fastrrt_destroy(self.p)
        except Exception:
            pass
