"""The C ABI library: it loads, exports every declared entry point and rejects bad input."""
import ctypes as C
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "delta_ray_b200.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"DR_API\s+[\w\s\*]+?\b(dr_\w+)\s*\(", text)))


def test_header_declares_the_entry_points():
    names = declared_functions()
    for n in ("dr_scene_create", "dr_scene_update", "dr_scene_destroy", "dr_render_forward",
              "dr_render_backward", "dr_last_error", "dr_scene_grad_layout", "dr_trace_rays"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from delta_ray_b200 import _lib
    L = _lib.lib()
    for n in declared_functions():
        assert hasattr(L, n), n
    assert L.dr_abi_version() == 2


def test_null_arguments_are_rejected_without_a_device():
    from delta_ray_b200 import _abi, _lib
    L = _lib.lib()
    rd = _abi.render_desc(8, 8, 1, 1, 0)
    st = L.dr_render_forward(None, C.byref(rd), None, None)
    assert st == 1  # DR_ERR_INVALID_ARGUMENT
    assert "NULL" in _lib.last_error()
    with pytest.raises(_lib.DrError):
        _lib.check(L.dr_scene_grad_layout(None, None))
    assert L.dr_set_item_queue_limit(-1) == 1
    assert L.dr_set_item_queue_limit(0) == 0
    t = _abi.dr_tuning(64, 3, 0, 0, 0)
    assert L.dr_scene_set_tuning(None, C.byref(t)) == 1
    assert L.dr_scene_get_tuning(None, C.byref(t)) == 1
    rep = _abi.dr_tune_report()
    assert L.dr_scene_autotune(None, C.byref(rd), None, None, 4, C.byref(rep), None) == 1


def test_tuning_structs_match_header():
    from delta_ray_b200 import _abi
    assert C.sizeof(_abi.dr_tuning) == 24
    assert C.sizeof(_abi.dr_tune_report) == 24 + 4 + 4 + 4 + 4  # padded to 8 bytes


def test_render_desc_layout_matches_header():
    from delta_ray_b200 import _abi
    # int width,height,spp,max_bounces; uint64 seed; int64 pes; int dp_mode, flags; int reserved[7]
    assert C.sizeof(_abi.dr_render_desc) == 4 * 4 + 8 + 8 + 4 + 32 + 4  # padded to 8 bytes
