"""Loads libfastrrt_b200.so and declares its C ABI (include/fastrrt_b200.h).

The library is the only implementation: when it is missing or fails to load
every call raises; there is no CPU fallback.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfastrrt_b200.so")

_lib = None


class FastRRTError(RuntimeError):
    pass


class Request(C.Structure):
    """fastrrt_request (include/fastrrt_b200.h)."""
    _fields_ = [("width", C.c_int), ("height", C.c_int),
                ("class_ids", C.POINTER(C.c_uint8)), ("class_costs", C.POINTER(C.c_float)),
                ("n_classes", C.c_int),
                ("perception_w_m", C.c_float), ("perception_h_m", C.c_float),
                ("max_steering_deg", C.c_float), ("vehicle_length_m", C.c_float),
                ("max_curvature", C.c_float),
                ("lb_x", C.c_int), ("lb_z", C.c_int), ("ub_x", C.c_int), ("ub_z", C.c_int),
                ("start_x", C.c_int), ("start_z", C.c_int), ("start_heading", C.c_float),
                ("goal_x", C.c_int), ("goal_z", C.c_int), ("goal_heading", C.c_float),
                ("velocity_m_s", C.c_float), ("min_dist_x", C.c_int), ("min_dist_z", C.c_int),
                ("max_path_size", C.c_float), ("dist_to_goal_tol", C.c_float),
                ("heading_tol_rad", C.c_float), ("seed", C.c_uint64), ("smart", C.c_int),
                ("max_iterations", C.c_int), ("class_ids_on_device", C.c_int),
                ("timeout_ms", C.c_int)]


EXPORTS = [
    # reference planner ABI (src/python_bind.cpp)
    "fastrrt_initialize", "fastrrt_destroy", "set_plan_data", "goal_reached", "search_init",
    "loop", "path_optimize", "export_graph_nodes", "release_export_graph_nodes",
    "get_planned_path", "interpolate_planned_path", "release_planned_path_data",
    "interpolate_planned_path_p", "ideal_curve", "compute_region_debug_performance",
    "save_current_graph_state", "load_graph_state", "fastrrt_apf_repulsion", "fastrrt_apf_attraction",
    "fastrrt_intrinsic_costs", "fastrrt_check_graph_consistent",
    "fastrrt_validate_path",
    # frames, seeding, errors
    "fastrrt_last_error", "fastrrt_frame_create", "fastrrt_frame_create_f3",
    "fastrrt_frame_destroy", "fastrrt_frame_process_distance_to_goal",
    "fastrrt_frame_process_safe_zone", "fastrrt_frame_flags", "fastrrt_frame_channels",
    "fastrrt_set_frame_preprocessing", "fastrrt_set_seed", "fastrrt_probe_count", "fastrrt_loop_count",
    # per-candidate kernels
    "fastrrt_candidates_create", "fastrrt_candidates_destroy", "fastrrt_candidates_kinematic",
    "fastrrt_candidates_kinematic_device", "fastrrt_candidates_hermite",
    "fastrrt_candidates_hermite_device", "fastrrt_candidates_feasible",
    "fastrrt_candidates_kinematic_noalloc", "fastrrt_debug_set_stage_wait_limit",
    "fastrrt_debug_stage_timeouts",
    # batched planner
    "fastrrt_batch_create", "fastrrt_batch_create_budget", "fastrrt_slot_bytes",
    "fastrrt_batch_memory", "fastrrt_batch_destroy", "fastrrt_batch_admit",
    "fastrrt_batch_admit_many", "fastrrt_batch_run", "fastrrt_batch_step", "fastrrt_batch_status",
    "fastrrt_batch_collect", "fastrrt_batch_path", "fastrrt_batch_release",
    "fastrrt_batch_last_ms", "fastrrt_batch_plan", "fastrrt_batch_profile",
    "fastrrt_batch_kernel_times", "fastrrt_kernel_count", "fastrrt_kernel_name",
    "fastrrt_batch_probes", "fastrrt_batch_interpolate", "fastrrt_batch_interpolated_path",
    "fastrrt_batch_direct_connections", "fastrrt_batch_serve",
    # learned expansion proposal
    "fastrrt_mlp_create", "fastrrt_mlp_destroy", "fastrrt_mlp_get_weights",
    "fastrrt_mlp_set_weights", "fastrrt_mlp_forward", "fastrrt_mlp_gradients", "fastrrt_mlp_train",
    "fastrrt_batch_set_proposal", "fastrrt_batch_log_paths", "fastrrt_batch_set_launch",
    "fastrrt_gemm_bf16", "fastrrt_batch_log_nodes",
]


def lib():
    """The loaded library; raises FastRRTError when it cannot be loaded."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FastRRTError(f"{LIB_PATH} is missing: build it with `python -m fastrrt_b200.build`")
    try:
        L = C.CDLL(LIB_PATH)
    except OSError as e:
        raise FastRRTError(f"cannot load {LIB_PATH}: {e}") from e
    P = C.POINTER
    f32p = np.ctypeslib.ndpointer(np.float32, flags="C")
    i32p = np.ctypeslib.ndpointer(np.int32, flags="C")
    u8p = np.ctypeslib.ndpointer(np.uint8, flags="C")
    vp = C.c_void_p
    sig = {
        "fastrrt_initialize": (vp, [C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float,
                                    C.c_int, C.c_int, C.c_int, C.c_int, f32p, C.c_float]),
        "fastrrt_destroy": (None, [vp]),
        "set_plan_data": (None, [vp, vp, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int, C.c_float,
                                 C.c_float, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                 C.c_float]),
        "goal_reached": (C.c_bool, [vp]),
        "search_init": (None, [vp, C.c_bool]),
        "loop": (C.c_bool, [vp, C.c_bool]),
        "path_optimize": (C.c_bool, [vp]),
        "export_graph_nodes": (P(C.c_int), [vp]),
        "release_export_graph_nodes": (None, [P(C.c_int)]),
        "get_planned_path": (P(C.c_float), [vp]),
        "interpolate_planned_path": (P(C.c_float), [vp]),
        "release_planned_path_data": (None, [P(C.c_float)]),
        "interpolate_planned_path_p": (P(C.c_float), [vp, f32p, C.c_int]),
        "ideal_curve": (P(C.c_float), [vp, C.c_int, C.c_int, C.c_float]),
        "compute_region_debug_performance": (None, [vp]),
        "save_current_graph_state": (None, [vp, C.c_char_p]),
        "load_graph_state": (None, [vp, C.c_char_p]),
        "fastrrt_apf_repulsion": (C.c_int, [vp, vp, C.c_float, C.c_int]),
        "fastrrt_apf_attraction": (C.c_int, [vp, vp, C.c_float, C.c_int, C.c_int]),
        "fastrrt_intrinsic_costs": (C.c_int, [vp, f32p]),
        "fastrrt_check_graph_consistent": (C.c_int, [vp]),
        "fastrrt_validate_path": (C.c_int, [vp, f32p, C.c_int]),
        "fastrrt_last_error": (C.c_char_p, []),
        "fastrrt_frame_create": (vp, [C.c_int, C.c_int, u8p, f32p, C.c_int, vp]),
        "fastrrt_frame_create_f3": (vp, [C.c_int, C.c_int, f32p, f32p, C.c_int]),
        "fastrrt_frame_destroy": (None, [vp]),
        "fastrrt_frame_process_distance_to_goal": (C.c_int, [vp, C.c_int, C.c_int]),
        "fastrrt_frame_process_safe_zone": (C.c_int, [vp, C.c_int, C.c_int]),
        "fastrrt_frame_flags": (C.c_int, [vp, P(C.c_int), P(C.c_int)]),
        "fastrrt_frame_channels": (C.c_int, [vp, vp, vp]),
        "fastrrt_set_frame_preprocessing": (C.c_int, [vp, C.c_int]),
        "fastrrt_set_seed": (C.c_int, [vp, C.c_uint64]),
        "fastrrt_probe_count": (C.c_int, [vp, P(C.c_uint64)]),
        "fastrrt_loop_count": (C.c_int, [vp]),
        "fastrrt_candidates_create": (vp, [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                           C.c_double, C.c_double, vp, vp]),
        "fastrrt_candidates_destroy": (None, [vp]),
        "fastrrt_candidates_kinematic": (C.c_int, [vp, C.c_int, i32p, i32p, f32p, f32p, C.c_float,
                                                   f32p, P(C.c_uint64)]),
        "fastrrt_candidates_kinematic_device": (C.c_int, [vp, C.c_int, vp, vp, vp, vp, C.c_float,
                                                          vp, vp, vp]),
        "fastrrt_candidates_hermite": (C.c_int, [vp, C.c_int, i32p, i32p, f32p, i32p, i32p, f32p,
                                                 C.c_float, C.c_int, f32p, P(C.c_uint64)]),
        "fastrrt_candidates_hermite_device": (C.c_int, [vp, C.c_int, vp, vp, vp, vp, vp, vp,
                                                        C.c_float, C.c_int, vp, vp, vp]),
        "fastrrt_candidates_feasible": (C.c_int, [vp, C.c_int, i32p, i32p, f32p, i32p,
                                                  P(C.c_uint64)]),
        "fastrrt_candidates_kinematic_noalloc": (C.c_int, [C.c_int, C.c_int, vp, vp, C.c_int, vp,
                                                           vp, C.c_int, C.c_int, C.c_int, C.c_int,
                                                           C.c_int, C.c_int, C.c_double,
                                                           C.c_double, C.c_int, vp, vp, vp, vp,
                                                           C.c_float, vp, vp, vp]),
        "fastrrt_debug_set_stage_wait_limit": (C.c_int, [C.c_int64]),
        "fastrrt_debug_stage_timeouts": (C.c_int, [P(C.c_uint64)]),
        "fastrrt_batch_create": (vp, [C.c_int, C.c_int, C.c_int]),
        "fastrrt_batch_create_budget": (vp, [C.c_int, C.c_int, C.c_int, C.c_uint64]),
        "fastrrt_slot_bytes": (C.c_uint64, [C.c_int, C.c_int]),
        "fastrrt_batch_memory": (C.c_int, [vp, P(C.c_uint64), P(C.c_uint64), P(C.c_uint64)]),
        "fastrrt_batch_destroy": (None, [vp]),
        "fastrrt_batch_admit": (C.c_int, [vp, C.c_int, P(Request), C.c_int]),
        "fastrrt_batch_admit_many": (C.c_int, [vp, C.c_int, P(Request), C.c_int]),
        "fastrrt_batch_run": (C.c_int, [vp, C.c_int, C.c_int]),
        "fastrrt_batch_step": (C.c_int, [vp]),
        "fastrrt_batch_status": (C.c_int, [vp, i32p, i32p, i32p]),
        "fastrrt_batch_collect": (C.c_int, [vp, C.c_int, i32p, i32p, f32p, i32p]),
        "fastrrt_batch_path": (C.c_int, [vp, C.c_int, f32p, C.c_int]),
        "fastrrt_batch_release": (C.c_int, [vp, C.c_int]),
        "fastrrt_batch_last_ms": (C.c_float, [vp]),
        "fastrrt_batch_plan": (C.c_int, [vp, C.c_int, P(Request), C.c_int, C.c_int, i32p, f32p,
                                         f32p, P(C.c_float)]),
        "fastrrt_batch_profile": (C.c_int, [vp, C.c_int]),
        "fastrrt_batch_kernel_times": (C.c_int, [vp, np.ctypeslib.ndpointer(np.float64, flags="C"),
                                                 np.ctypeslib.ndpointer(np.int64, flags="C")]),
        "fastrrt_kernel_count": (C.c_int, []),
        "fastrrt_kernel_name": (C.c_char_p, [C.c_int]),
        "fastrrt_batch_probes": (C.c_int, [vp, P(C.c_uint64), P(C.c_uint64), P(C.c_uint64)]),
        "fastrrt_batch_interpolate": (C.c_int, [vp, C.c_int, vp, vp, vp]),
        "fastrrt_batch_interpolated_path": (C.c_int, [vp, C.c_int, f32p, C.c_int]),
        "fastrrt_batch_direct_connections": (C.c_int, [vp, C.c_int, vp, vp, vp]),
        "fastrrt_mlp_create": (vp, [C.c_uint64, C.c_int]),
        "fastrrt_mlp_destroy": (None, [vp]),
        "fastrrt_mlp_get_weights": (C.c_int, [vp] + [f32p] * 6),
        "fastrrt_mlp_set_weights": (C.c_int, [vp] + [f32p] * 6),
        "fastrrt_mlp_forward": (C.c_int, [vp, C.c_int, f32p, f32p]),
        "fastrrt_mlp_gradients": (C.c_int, [vp, C.c_int, f32p, i32p] + [f32p] * 6 + [P(C.c_float)]),
        "fastrrt_mlp_train": (C.c_int, [vp, vp, vp, C.c_int, C.c_int, C.c_int, C.c_float, C.c_uint64,
                                        P(C.c_float)]),
        "fastrrt_batch_set_proposal": (C.c_int, [vp, vp, C.c_float, C.c_int]),
        "fastrrt_gemm_bf16": (C.c_int, [C.c_int, C.c_int, C.c_int, vp, C.c_int, C.c_int, vp, C.c_int,
                                        C.c_int, vp, C.c_int, vp, C.c_int, vp, vp, C.c_int, vp, vp,
                                        C.c_uint64, vp]),
        "fastrrt_batch_set_launch": (C.c_int, [vp, C.c_int, C.c_int]),
        "fastrrt_batch_log_paths": (C.c_int, [vp, vp, vp, C.c_int, C.c_int]),
        "fastrrt_batch_log_nodes": (C.c_int, [vp, vp, vp, C.c_int, C.c_int]),
        "fastrrt_batch_serve": (C.c_int, [vp, C.c_int, P(Request), vp, C.c_int, C.c_int, i32p, f32p,
                                          f32p, f32p, i32p, P(C.c_double), P(C.c_float), f32p]),
    }
    for name in EXPORTS:
        fn = getattr(L, name)
        res, args = sig[name]
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return _lib


def last_error():
    msg = lib().fastrrt_last_error()
    return msg.decode() if msg else ""


def check(rc, what):
    if rc is None or (isinstance(rc, int) and rc < 0):
        raise FastRRTError(f"{what}: {last_error()}")
    return rc


def require_cuda():
    """Raises unless a CUDA device is visible (the planner has no CPU path)."""
    import torch
    if not torch.cuda.is_available():
        raise FastRRTError("fastrrt_b200 needs a CUDA device; none is visible")
