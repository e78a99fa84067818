"""The C-ABI library loads on a host without a GPU and exports every declared symbol."""
import ctypes
import os
import re

import pytest

from rtb200 import native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(ROOT, "include", "rtb200.h")).read()
    return sorted(set(re.findall(r"RTB_API\s+[\w\s\*]+?\b(rtb_\w+)\s*\(", text)))


def test_header_declares_the_boundary():
    names = _declared()
    for required in ("rtb_context_create", "rtb_scene_upload", "rtb_scene_build", "rtb_trace_replay",
                     "rtb_render_sample", "rtb_last_frame_stats", "rtb_status_string"):
        assert required in names


def test_library_exports_every_declared_symbol():
    lib = native.lib()
    for name in _declared():
        assert hasattr(lib, name), name
        assert name in native.SIGNATURES, name


def test_status_strings():
    lib = native.lib()
    assert lib.rtb_status_string(0) == b"ok"
    assert b"argument" in lib.rtb_status_string(1)


def test_context_create_reports_unavailable_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = native.lib()
    h = ctypes.c_void_p()
    assert lib.rtb_context_create(0, ctypes.byref(h)) == 2  # RTB_ERR_UNAVAILABLE
