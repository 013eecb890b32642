"""The C ABI library loads without a GPU and exports every symbol that
include/fastrrt_b200.h declares; the Python layer mirrors pyfastrrt."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "fastrrt_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\([^;{]*\)\s*;", text)
    return sorted(set(n for n in names if n not in ("if", "while", "for")))


def test_library_exports_every_declared_symbol():
    from fastrrt_b200 import _lib
    L = _lib.lib()
    names = declared_functions()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) == set(_lib.EXPORTS)


def test_reference_abi_names_present():
    # every extern "C" name of the reference's src/python_bind.cpp
    names = declared_functions()
    for n in ["fastrrt_initialize", "fastrrt_destroy", "set_plan_data", "goal_reached",
              "search_init", "loop", "path_optimize", "export_graph_nodes",
              "release_export_graph_nodes", "get_planned_path", "interpolate_planned_path",
              "release_planned_path_data", "interpolate_planned_path_p", "ideal_curve",
              "compute_region_debug_performance", "save_current_graph_state", "load_graph_state"]:
        assert n in names


def test_python_api_surface():
    import fastrrt_b200 as F
    for m in ["set_plan_data", "search_init", "loop", "path_optimize", "goal_reached",
              "get_planned_path", "export_graph_nodes", "compute_region_debug_performance",
              "save_current_graph_state", "load_graph_state", "build_ideal_curve",
              "interpolate_planned_path_p"]:
        assert hasattr(F.FastRRT, m)


def test_errors_without_gpu_are_loud():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    import fastrrt_b200 as F
    import numpy as np
    with pytest.raises(F.FastRRTError):
        F.SearchFrame(class_ids=np.zeros((8, 8), np.uint8), class_costs=np.zeros(1, np.float32))
