"""ctypes declarations of include/qmiv_gpu.h and the loader of the in-tree libqmiv_b200.so.

There is no fallback: if the CUDA library is missing or cannot be loaded, importing fails.
"""
from __future__ import annotations

import ctypes
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libqmiv_b200.so")

# status codes
OK, ERR_INVALID_ARG, ERR_UNSUPPORTED, ERR_CUDA, ERR_OUT_OF_MEMORY, ERR_INVALID_PIXEL, ERR_BUDGET, \
    ERR_TIMEOUT, ERR_NOT_READY, ERR_CANCELLED, ERR_BUSY = range(11)

# metric bits
PSNR, WSPSNR, IVPSNR, SSIM, MSSSIM, IVSSIM, IVMSSSIM = 1, 2, 4, 8, 16, 32, 64
ALL = 0x7F
METRIC_BITS = {"PSNR": PSNR, "WSPSNR": WSPSNR, "IVPSNR": IVPSNR, "SSIM": SSIM, "MSSSIM": MSSSIM,
               "IVSSIM": IVSSIM, "IVMSSSIM": IVMSSSIM}

MEM_HOST, MEM_DEVICE = 0, 1
STAGES = ["h2d", "prepass", "reduce", "cps", "ssim_win", "ssim_rows", "finalize", "d2h"]
PEL_SKIP, PEL_WARN, PEL_STOP, PEL_CNCL = 0, 1, 2, 3
# colour spaces (ColorSpaceInput / ColorSpaceMetric), apps/QMIV/src/xUtilsQMIV.h:12-27
CS_RGB, CS_BGR, CS_GBR, CS_YCBCR = 2, 3, 4, 16
CS_BT601, CS_SMPTE170M, CS_BT709, CS_SMPTE240M, CS_BT2020 = 17, 18, 19, 20, 21
# structural similarity modes (StructSimMode, xSSIM::eMode) and border extensions (StructSimBrdExt, eMrgExt)
SSM_REGULAR_GAUSSIAN_FLT, SSM_REGULAR_GAUSSIAN_INT, SSM_REGULAR_AVERAGED, SSM_BLOCK_GAUSSIAN_INT, SSM_BLOCK_AVERAGED = 0, 1, 2, 3, 4
BRD_NONE, BRD_NEAREST, BRD_REFLECT, BRD_MIRROR, BRD_CONSTANT, BRD_ZERO = 0, 1, 2, 3, 4, 5


class QmivParams(ctypes.Structure):
    _fields_ = [
        ("search_range", ctypes.c_int32), ("cws", ctypes.c_int32 * 4), ("cwa", ctypes.c_int32 * 4),
        ("unc", ctypes.c_float * 4), ("erp", ctypes.c_int32), ("lon_range_deg", ctypes.c_int32),
        ("lat_range_deg", ctypes.c_int32), ("ssim_window", ctypes.c_int32), ("ssim_stride", ctypes.c_int32),
        ("invalid_pel_action", ctypes.c_int32), ("ssim_mode", ctypes.c_int32), ("ssim_border", ctypes.c_int32),
    ]


class QmivFrame(ctypes.Structure):
    _fields_ = [("plane", ctypes.c_void_p * 3), ("pitch", ctypes.c_int64 * 3), ("mem", ctypes.c_int32)]


class QmivResult(ctypes.Structure):
    _fields_ = [
        ("gcd_r2t", ctypes.c_int32 * 4), ("exact", ctypes.c_int32 * 4), ("invalid_pel", ctypes.c_int32 * 2),
        ("ssd", ctypes.c_uint64 * 4), ("cps_sse_r2t", ctypes.c_uint64 * 4), ("cps_sse_t2r", ctypes.c_uint64 * 4),
        ("psnr", ctypes.c_double * 4), ("psnr_pic", ctypes.c_double),
        ("wspsnr", ctypes.c_double * 4), ("wspsnr_pic", ctypes.c_double),
        ("ivpsnr", ctypes.c_double), ("ivpsnr_r2t", ctypes.c_double), ("ivpsnr_t2r", ctypes.c_double),
        ("ssim", ctypes.c_double * 4), ("ssim_pic", ctypes.c_double),
        ("msssim", ctypes.c_double * 4), ("msssim_pic", ctypes.c_double),
        ("ivssim", ctypes.c_double), ("ivssim_r2t", ctypes.c_double), ("ivssim_t2r", ctypes.c_double),
        ("ivmsssim", ctypes.c_double), ("ivmsssim_r2t", ctypes.c_double), ("ivmsssim_t2r", ctypes.c_double),
    ]

    def as_dict(self):
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            d[name] = list(v) if hasattr(v, "__len__") else v
        return d


class QmivPairDesc(ctypes.Structure):
    _fields_ = [("in0", QmivFrame), ("in1", QmivFrame), ("width", ctypes.c_int32), ("height", ctypes.c_int32),
                ("bitdepth", ctypes.c_int32), ("chroma_format", ctypes.c_int32), ("search_range", ctypes.c_int32),
                ("metric_mask", ctypes.c_uint32)]


class QmivRequest(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int32), ("height", ctypes.c_int32), ("bitdepth", ctypes.c_int32),
                ("chroma_format", ctypes.c_int32), ("search_range", ctypes.c_int32), ("metric_mask", ctypes.c_uint32),
                ("num_pairs", ctypes.c_int32), ("in0", ctypes.POINTER(QmivFrame)), ("in1", ctypes.POINTER(QmivFrame))]


class QmivRequestStats(ctypes.Structure):
    _fields_ = [("submit_ms", ctypes.c_double), ("admit_ms", ctypes.c_double), ("done_ms", ctypes.c_double),
                ("latency_ms", ctypes.c_double), ("batches", ctypes.c_int32),
                ("mean_psnr_pic", ctypes.c_double), ("mean_wspsnr_pic", ctypes.c_double),
                ("mean_ivpsnr", ctypes.c_double), ("mean_ssim_pic", ctypes.c_double),
                ("mean_msssim_pic", ctypes.c_double), ("mean_ivssim", ctypes.c_double),
                ("mean_ivmsssim", ctypes.c_double)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


# name -> (restype, argtypes); every symbol include/qmiv_gpu.h declares
_P = ctypes.c_void_p
_PP = ctypes.POINTER(ctypes.c_void_p)
SIGNATURES = {
    "qmiv_api_version": (ctypes.c_int32, []),
    "qmiv_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "qmiv_last_error": (ctypes.c_char_p, []),
    "qmiv_params_default": (None, [ctypes.POINTER(QmivParams)]),
    "qmiv_ctx_create": (ctypes.c_int, [ctypes.c_int32, ctypes.c_uint64, _PP]),
    "qmiv_ctx_destroy": (ctypes.c_int, [_P]),
    "qmiv_ctx_memory": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]),
    "qmiv_ctx_set_profiling": (ctypes.c_int, [_P, ctypes.c_int32]),
    "qmiv_ctx_stage_times": (ctypes.c_int, [_P, ctypes.c_double * 8, ctypes.c_uint64 * 8, ctypes.c_int32]),
    "qmiv_calc_create": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                        ctypes.POINTER(QmivParams), _PP]),
    "qmiv_calc_destroy": (ctypes.c_int, [_P]),
    "qmiv_frame_pair_compute": (ctypes.c_int, [_P, ctypes.POINTER(QmivFrame), ctypes.POINTER(QmivFrame),
                                               ctypes.c_uint32, ctypes.POINTER(QmivResult)]),
    "qmiv_frame_pair_compute_masked": (ctypes.c_int, [_P, ctypes.POINTER(QmivFrame), ctypes.POINTER(QmivFrame),
                                                      ctypes.POINTER(QmivFrame), ctypes.c_int32, ctypes.c_uint32,
                                                      ctypes.POINTER(QmivResult), ctypes.POINTER(ctypes.c_int32)]),
    "qmiv_frame_pair_submit": (ctypes.c_int, [_P, ctypes.POINTER(QmivFrame), ctypes.POINTER(QmivFrame), ctypes.c_uint32]),
    "qmiv_frame_pair_wait": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.POINTER(QmivResult)]),
    "qmiv_calc_gcd": (ctypes.c_int, [_P, ctypes.POINTER(QmivFrame), ctypes.POINTER(QmivFrame), ctypes.c_int32 * 4]),
    "qmiv_calc_scp": (ctypes.c_int, [_P, ctypes.POINTER(QmivFrame), ctypes.POINTER(QmivFrame),
                                     ctypes.POINTER(ctypes.c_int32), _P, _P, ctypes.c_int32]),
    "qmiv_calc_set_gcd": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int32)]),
    "qmiv_calc_set_color_space": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32]),
    "qmiv_calc_cps_rows": (ctypes.c_int, [_P, _P, _P]),
    "qmiv_calc_stream": (ctypes.c_int, [_P, _PP]),
    "qmiv_frame_pair_compute_static": (ctypes.c_int, [ctypes.POINTER(QmivFrame), ctypes.POINTER(QmivFrame),
                                                      ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                                      ctypes.POINTER(QmivParams), ctypes.c_uint32, _P,
                                                      ctypes.POINTER(QmivResult)]),
    "qmiv_batch_create": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int64, ctypes.POINTER(QmivParams),
                                         ctypes.c_int32, _PP]),
    "qmiv_probe_int32_peak": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_double)]),
    "qmiv_probe_fp32_peak": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_double)]),
    "qmiv_probe_fp64_peak": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_double)]),
    "qmiv_batch_destroy": (ctypes.c_int, [_P]),
    "qmiv_batch_stream": (ctypes.c_int, [_P, _PP]),
    "qmiv_batch_compute": (ctypes.c_int, [_P, ctypes.POINTER(QmivPairDesc), ctypes.c_int32, ctypes.POINTER(QmivResult)]),
    "qmiv_batch_compute_masked": (ctypes.c_int, [_P, ctypes.POINTER(QmivPairDesc), ctypes.POINTER(QmivFrame),
                                                 ctypes.POINTER(ctypes.c_int32), ctypes.c_int32, ctypes.POINTER(QmivResult),
                                                 ctypes.POINTER(ctypes.c_int32)]),
    "qmiv_batch_submit": (ctypes.c_int, [_P, ctypes.POINTER(QmivPairDesc), ctypes.c_int32, ctypes.POINTER(ctypes.c_uint64)]),
    "qmiv_batch_wait": (ctypes.c_int, [_P, ctypes.c_uint64, ctypes.POINTER(QmivResult)]),
    "qmiv_batch_tuning": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                         ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32),
                                         ctypes.POINTER(ctypes.c_int32)]),
    "qmiv_server_create": (ctypes.c_int, [_P, ctypes.POINTER(QmivParams), ctypes.c_int32, ctypes.c_int64, ctypes.c_int32,
                                          _PP]),
    "qmiv_server_destroy": (ctypes.c_int, [_P]),
    "qmiv_server_submit": (ctypes.c_int, [_P, ctypes.POINTER(QmivRequest), ctypes.POINTER(ctypes.c_uint64)]),
    "qmiv_server_wait": (ctypes.c_int, [_P, ctypes.c_uint64, ctypes.c_int32, ctypes.POINTER(QmivResult),
                                        ctypes.POINTER(QmivRequestStats)]),
    "qmiv_server_stats": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                         ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64), ctypes.c_int32]),
}

_lib = None


def load(path: str | None = None):
    """Load libqmiv_b200.so (building it first if it is missing and nvcc is available)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        from . import build as _build
        _build.build()
    lib = ctypes.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)  # AttributeError = symbol missing: fail loudly
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


class QmivError(RuntimeError):
    def __init__(self, status: int, where: str):
        lib = load()
        msg = lib.qmiv_last_error().decode(errors="replace")
        super().__init__(f"{where}: {lib.qmiv_status_string(status).decode()} ({status}): {msg}")
        self.status = status


def check(status: int, where: str):
    if status != OK:
        raise QmivError(status, where)
