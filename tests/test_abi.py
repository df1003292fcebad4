"""CPU checks of the C ABI: the library loads, exports every function the
header declares, struct layouts agree, and calls fail cleanly (no crash) on
a machine without a GPU.  No compute calls."""
import ctypes as C
import os
import re

import pytest

from swiftbwa_b200 import abi
from swiftbwa_b200.build import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "swb_cuda.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(swb_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    build()
    return abi.load_library()


def test_header_declares_what_python_binds():
    assert header_functions() == sorted(abi.EXPORTED_SYMBOLS)


def test_library_exports_every_declared_symbol(lib):
    missing = [s for s in header_functions() if not hasattr(lib, s)]
    assert not missing


def test_struct_sizes_match_header():
    assert C.sizeof(abi.ExtTask) == 40
    assert C.sizeof(abi.GlobalTask) == 40
    assert C.sizeof(abi.LocalTask) == 32
    assert C.sizeof(abi.ExtResult) == 24
    assert C.sizeof(abi.LocalResult) == 24
    assert C.sizeof(abi.GlobalResult) == 24
    assert C.sizeof(abi.Scoring) == 44


def test_scoring_default_matches_reference(lib):
    s = abi.Scoring()
    lib.swb_scoring_default(C.byref(s))
    # ScoringParameters.swift:3-28 defaults
    assert (s.a, s.b, s.o_ins, s.e_ins, s.o_del, s.e_del, s.zdrop, s.pen_clip5, s.pen_clip3,
            s.band_width, s.min_seed_len) == (1, 4, 6, 1, 6, 1, 100, 5, 5, 100, 19)
    assert abi.Scoring.default().a == 1


def test_strerror_names_every_status(lib):
    for code in range(0, -10, -1):
        assert lib.swb_strerror(code) and lib.swb_strerror(code) != b"unknown status"
    assert lib.swb_strerror(-99) == b"unknown status"


def test_null_arguments_are_rejected_without_crash(lib):
    assert lib.swb_init(0, 0, None) == abi.SWB_ERR_INVALID_ARG
    sc = abi.Scoring.default()
    assert lib.swb_ext_batch(None, C.byref(sc), None, 0, None, 0, None) == abi.SWB_ERR_INVALID_ARG
    assert lib.swb_last_batch_stats(None, None, None) == abi.SWB_ERR_INVALID_ARG
    assert lib.swb_kernel_launches(None) == 0
    v = C.c_double()
    assert lib.swb_int_alu_peak(None, C.byref(v)) == abi.SWB_ERR_INVALID_ARG
    assert lib.swb_int16x2_alu_peak(None, C.byref(v)) == abi.SWB_ERR_INVALID_ARG
    q = (C.c_int32 * 2)(32, 64)
    assert lib.swb_set_ext_bins(None, q, 2) == abi.SWB_ERR_INVALID_ARG
    assert lib.swb_get_ext_bins(None, q, 2, C.byref(C.c_int())) == abi.SWB_ERR_INVALID_ARG
    assert lib.swb_tune_ext_bins(None, C.byref(sc), None, 0, None, 0, None, 0, None, None, None) == abi.SWB_ERR_INVALID_ARG
    lib.swb_destroy(None)


def test_init_without_gpu_reports_no_device(lib):
    h = C.c_void_p()
    rc = lib.swb_init(0, 0, C.byref(h))
    if rc == abi.SWB_OK:
        lib.swb_destroy(h)
        pytest.skip("a GPU is visible here")
    assert rc == abi.SWB_ERR_NO_DEVICE
    assert b"device" in lib.swb_last_error_message()


def test_cigar_caps_follow_the_header_rule():
    """Engine.cigar_caps sizes swb_cigar_batch's outputs by the header's rule:
    cigar_cap = sum(qlen + rlen + 2) words, md_cap = sum(6*(qlen+rlen)+8) bytes
    (one spare entry each)."""
    import numpy as np
    from swiftbwa_b200.alignment import Engine
    rng = np.random.default_rng(3)
    t = np.zeros(1000, abi.CIGAR_TASK_DTYPE)
    t["qlen"] = rng.integers(0, 300, t.size)
    t["rlen"] = rng.integers(0, 400, t.size)
    q, r = t["qlen"].astype(np.int64), t["rlen"].astype(np.int64)
    assert Engine.cigar_caps(t) == (int((q + r + 2).sum()) + 1, int((6 * (q + r) + 8).sum()) + 1)
    assert Engine.cigar_caps(t[:0]) == (1, 1)
