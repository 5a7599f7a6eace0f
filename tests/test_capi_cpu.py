"""The C ABI library without a GPU: it loads, exports every symbol include/*.h declares, and its
host-only entry points behave."""
import ctypes
import glob
import os
import re

import pytest

from conftest import ROOT, cuda_available


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        with open(h) as f:
            text = f.read()
        names |= set(re.findall(r"QMIV_API\s+[\w\s\*]+?\b(qmiv_\w+)\s*\(", text))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    for n in ["qmiv_ctx_create", "qmiv_calc_create", "qmiv_frame_pair_compute", "qmiv_calc_scp", "qmiv_batch_compute"]:
        assert n in names


def test_library_loads_and_exports_every_declared_symbol():
    import qmiv_b200
    from qmiv_b200 import _lib
    lib = qmiv_b200.library()
    for name in declared_symbols():
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"


def test_status_strings_and_version():
    import qmiv_b200
    lib = qmiv_b200.library()
    assert lib.qmiv_api_version() == 1
    assert lib.qmiv_status_string(0) == b"ok"
    assert lib.qmiv_status_string(6) == b"HBM budget exceeded"
    assert lib.qmiv_status_string(99) == b"unknown status"


def test_params_default_match_reference_defaults():
    """xCorrespPixelShiftPrms.h:22-24, xGlobClrDiff.h:20, xSSIM.h:35-37."""
    import qmiv_b200
    p = qmiv_b200.make_params()
    assert p.search_range == 2
    assert list(p.cws) == [4, 1, 1, 0] and list(p.cwa) == [4, 1, 1, 0]
    assert [round(x, 6) for x in p.unc] == [0.01, 0.01, 0.01, 0.0]
    assert (p.ssim_window, p.ssim_stride) == (8, 4)
    assert (p.ssim_mode, p.ssim_border) == (qmiv_b200.SSM_BLOCK_AVERAGED, qmiv_b200.BRD_NONE)
    assert p.invalid_pel_action == qmiv_b200.PEL_STOP
    # the regular modes take 11x11 windows unless told otherwise
    q = qmiv_b200.make_params(ssim_mode=qmiv_b200.SSM_REGULAR_GAUSSIAN_FLT, ssim_stride=1)
    assert (q.ssim_mode, q.ssim_window, q.ssim_stride) == (0, 11, 1)


@pytest.mark.skipif(cuda_available(), reason="checks the no-GPU error path")
def test_ctx_create_without_gpu_fails_cleanly():
    import qmiv_b200
    with pytest.raises(qmiv_b200.QmivError) as ei:
        qmiv_b200.Context(0)
    assert ei.value.status in (1, 3)


def test_null_arguments_are_rejected():
    import qmiv_b200
    lib = qmiv_b200.library()
    assert lib.qmiv_ctx_create(0, 0, None) == 1
    assert lib.qmiv_calc_create(None, 64, 64, 8, 420, None, None) == 1
    assert lib.qmiv_frame_pair_compute(None, None, None, 0, None) == 1
    assert lib.qmiv_calc_destroy(None) == 1
    assert lib.qmiv_batch_destroy(None) == 1


def test_every_handle_entry_point_rejects_null():
    """Each entry point checks its handle and pointers before any device work: a null handle gives
    QMIV_ERR_INVALID_ARG (1) and a message, never a crash (the reference asserts instead)."""
    import ctypes
    import qmiv_b200
    lib = qmiv_b200.library()
    ms, nl, g4 = (ctypes.c_double * 8)(), (ctypes.c_uint64 * 8)(), (ctypes.c_int32 * 4)()
    calls = {
        "qmiv_ctx_destroy": lambda: lib.qmiv_ctx_destroy(None),
        "qmiv_ctx_memory": lambda: lib.qmiv_ctx_memory(None, None, None),
        "qmiv_ctx_set_profiling": lambda: lib.qmiv_ctx_set_profiling(None, 1),
        "qmiv_ctx_stage_times": lambda: lib.qmiv_ctx_stage_times(None, ms, nl, 0),
        "qmiv_frame_pair_submit": lambda: lib.qmiv_frame_pair_submit(None, None, None, 0),
        "qmiv_frame_pair_wait": lambda: lib.qmiv_frame_pair_wait(None, 0, None),
        "qmiv_frame_pair_compute_masked": lambda: lib.qmiv_frame_pair_compute_masked(None, None, None, None, 8, 0, None, None),
        "qmiv_calc_set_color_space": lambda: lib.qmiv_calc_set_color_space(None, 0, 0),
        "qmiv_calc_gcd": lambda: lib.qmiv_calc_gcd(None, None, None, g4),
        "qmiv_calc_scp": lambda: lib.qmiv_calc_scp(None, None, None, None, None, None, 0),
        "qmiv_calc_set_gcd": lambda: lib.qmiv_calc_set_gcd(None, None),
        "qmiv_calc_cps_rows": lambda: lib.qmiv_calc_cps_rows(None, None, None),
        "qmiv_calc_stream": lambda: lib.qmiv_calc_stream(None, None),
        "qmiv_frame_pair_compute_static": lambda: lib.qmiv_frame_pair_compute_static(None, None, 64, 64, 8, 420, None, 1,
                                                                                      None, None),
        "qmiv_batch_create": lambda: lib.qmiv_batch_create(None, 4, 1 << 20, None, 0, None),
        "qmiv_batch_compute": lambda: lib.qmiv_batch_compute(None, None, 0, None),
        "qmiv_batch_submit": lambda: lib.qmiv_batch_submit(None, None, 0, None),
        "qmiv_batch_wait": lambda: lib.qmiv_batch_wait(None, 0, None),
        "qmiv_batch_stream": lambda: lib.qmiv_batch_stream(None, None),
        "qmiv_batch_tuning": lambda: lib.qmiv_batch_tuning(None, 64, 64, 8, 2, None, None, None),
        "qmiv_server_create": lambda: lib.qmiv_server_create(None, None, 4, 1 << 20, 1, None),
        "qmiv_server_destroy": lambda: lib.qmiv_server_destroy(None),
        "qmiv_server_submit": lambda: lib.qmiv_server_submit(None, None, None),
        "qmiv_server_wait": lambda: lib.qmiv_server_wait(None, 0, 0, None, None),
        "qmiv_server_stats": lambda: lib.qmiv_server_stats(None, None, None, None, None, 0),
    }
    for name, call in calls.items():
        assert call() == 1, name
        assert lib.qmiv_last_error(), name
