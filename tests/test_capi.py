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


def test_slot_storage_sizes():
    """per-request storage of the budget arena (fastrrt_slot_bytes, host
    arithmetic): 256-byte aligned, growing with the frame, about 122 bytes
    per cell (node grid 22 B, goal connections, memo, scratch, frame copy,
    masks and summed-area table), and the sizes the serving benchmark
    reports for 128 / 256 / 512 frames"""
    from fastrrt_b200 import batch
    sizes = {s: batch.slot_bytes(s, s) for s in (64, 100, 128, 256, 512, 1000)}
    assert (sizes[128], sizes[256], sizes[512]) == (2002944, 7974912, 31862784)
    assert all(v % 256 == 0 for v in sizes.values())
    keys = sorted(sizes)
    assert all(sizes[a] < sizes[b] for a, b in zip(keys, keys[1:]))
    for s in (256, 512, 1000):
        assert 110 < sizes[s] / (s * s) < 130
    # a wide frame and a tall one of the same cells take the same storage
    # up to row padding of the bit masks
    assert abs(batch.slot_bytes(512, 128) - batch.slot_bytes(128, 512)) < 0.01 * batch.slot_bytes(512, 128)


def declared_arity():
    """parameter count of every function the header declares"""
    text = open(os.path.join(ROOT, "include", "fastrrt_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    out = {}
    for name, params in re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(([^;{()]*)\)\s*;", text):
        p = " ".join(params.split())
        out[name] = 0 if p in ("", "void") else p.count(",") + 1
    return out


def test_binding_argument_counts_match_the_header():
    """the ctypes layer declares as many arguments as the header for every
    entry point (a mismatch would pass garbage through the ABI)"""
    from fastrrt_b200 import _lib
    L = _lib.lib()
    arity = declared_arity()
    assert set(arity) == set(_lib.EXPORTS)
    wrong = {n: (arity[n], len(getattr(L, n).argtypes)) for n in arity
             if len(getattr(L, n).argtypes) != arity[n]}
    assert not wrong, wrong


def test_request_struct_layout_matches_the_header(tmp_path):
    """ctypes' Request against the C compiler's layout of fastrrt_request
    (offset of every field and the size), from a tiny program built against
    include/fastrrt_b200.h"""
    import shutil
    import subprocess

    from fastrrt_b200 import _lib
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    names = [f[0] for f in _lib.Request._fields_]
    src = tmp_path / "layout.c"
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "fastrrt_b200.h"\nint main(void) {\n'
                   + "".join(f'    printf("{n} %zu\\n", offsetof(fastrrt_request, {n}));\n' for n in names)
                   + '    printf("sizeof %zu\\n", sizeof(fastrrt_request));\n    return 0;\n}\n')
    exe = str(tmp_path / "layout")
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", exe], check=True)
    got = dict(line.split() for line in subprocess.run([exe], capture_output=True, text=True,
                                                       check=True).stdout.splitlines())
    for n in names:
        assert int(got[n]) == getattr(_lib.Request, n).offset, n
    assert int(got["sizeof"]) == __import__("ctypes").sizeof(_lib.Request)
