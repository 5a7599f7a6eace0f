"""qmiv_b200 — the QMIV metric hot path (GCD, CPS search, PSNR / WS-PSNR / IV-PSNR, SSIM / MS-SSIM /
IV-SSIM / IV-MS-SSIM) on B200 GPUs, through the C ABI of libqmiv_b200.so (include/qmiv_gpu.h).

The Python classes mirror the reference's pmbb-ivqm processors:

    reference (libs/pmbb-ivqm/src)                     here
    xGlobClrDiffProc::CalcGlobalColorDiff(T, R)        Calc.calc_global_color_diff(f0, f1)
    xShftCompPicProc::GenShftCompPics(...)             Calc.gen_shft_comp_pics(f0, f1)
    xPSNR::calcPicPSNR / xWSPSNR::calcPicWSPSNR        Calc.calc_pic_psnr / calc_pic_wspsnr
    xIVPSNR::calcPicIVPSNR(T, R, GCD)                  Calc.calc_pic_ivpsnr(f0, f1)
    xSSIM::calcPicSSIM / calcPicMSSSIM                 Calc.calc_pic_ssim / calc_pic_msssim
    xIVSSIM::calcPicIVSSIM / calcPicIVMSSSIM           Calc.calc_pic_ivssim / calc_pic_ivmsssim
    one frame of xAppQMIV::processAllFrames            Calc.compute(f0, f1, metrics)

A frame is a sequence of three planes (Y, Cb, Cr): numpy arrays (host memory) or CUDA tensors /
objects exposing __cuda_array_interface__ (device memory), uint8 for bit depth <= 8, else uint16.
"""
from __future__ import annotations

import ctypes
from typing import Iterable, Sequence

import numpy as np

from . import _lib
from ._lib import (ALL, IVMSSSIM, IVPSNR, IVSSIM, METRIC_BITS, MSSSIM, PSNR, SSIM, WSPSNR, PEL_CNCL, PEL_SKIP,
                   CS_RGB, CS_BGR, CS_GBR, CS_YCBCR, CS_BT601, CS_SMPTE170M, CS_BT709, CS_SMPTE240M, CS_BT2020,
                   PEL_STOP, PEL_WARN, QmivError, check, SSM_REGULAR_GAUSSIAN_FLT, SSM_REGULAR_GAUSSIAN_INT,
                   SSM_REGULAR_AVERAGED, SSM_BLOCK_GAUSSIAN_INT, SSM_BLOCK_AVERAGED, BRD_NONE, BRD_NEAREST, BRD_REFLECT,
                   BRD_MIRROR, BRD_CONSTANT, BRD_ZERO)

__all__ = ["Context", "Calc", "Batch", "make_params", "metric_mask", "QmivError", "library", "frame_from_raw",
           "raw_frame_bytes",
           "PSNR", "WSPSNR", "IVPSNR", "SSIM", "MSSSIM", "IVSSIM", "IVMSSSIM", "ALL", "Server"]


def library():
    """The loaded libqmiv_b200.so (ctypes.CDLL)."""
    return _lib.load()


def metric_mask(metrics) -> int:
    if metrics is None:
        return ALL
    if isinstance(metrics, int):
        return metrics
    if isinstance(metrics, str):
        metrics = [m.strip() for m in metrics.split(",") if m.strip()]
    m = 0
    for name in metrics:
        key = name.upper().replace("-", "").replace("_", "")
        if key not in METRIC_BITS:
            raise ValueError(f"unknown metric {name!r}")
        m |= METRIC_BITS[key]
    return m


def make_params(search_range=2, cws=(4, 1, 1, 0), cwa=(4, 1, 1, 0), unc=(0.01, 0.01, 0.01, 0.0), erp=False,
                lon_range=360, lat_range=180, invalid_pel_action=PEL_STOP, ssim_mode=SSM_BLOCK_AVERAGED,
                ssim_border=BRD_NONE, ssim_window=None, ssim_stride=4) -> _lib.QmivParams:
    """Processor parameters; the SSIM options are the app's StructSimMode / StructSimBrdExt /
    StructSimWindow / StructSimStride (ssim_window defaults to 11 for the regular modes, else 8)."""
    p = _lib.QmivParams()
    library().qmiv_params_default(ctypes.byref(p))
    p.search_range = search_range
    p.cws = (ctypes.c_int32 * 4)(*cws)
    p.cwa = (ctypes.c_int32 * 4)(*cwa)
    p.unc = (ctypes.c_float * 4)(*unc)
    p.erp = int(bool(erp))
    p.lon_range_deg = lon_range
    p.lat_range_deg = lat_range
    p.invalid_pel_action = invalid_pel_action
    p.ssim_mode = ssim_mode
    p.ssim_border = ssim_border
    p.ssim_window = ssim_window if ssim_window is not None else (11 if ssim_mode <= SSM_REGULAR_AVERAGED else 8)
    p.ssim_stride = ssim_stride
    return p


def _plane_info(plane):
    """(pointer, pitch in bytes, mem kind, keep-alive object) of one plane."""
    cai = getattr(plane, "__cuda_array_interface__", None)
    if cai is not None:
        shape, strides = cai["shape"], cai.get("strides")
        itemsize = np.dtype(cai["typestr"]).itemsize
        if strides is None:
            pitch = shape[1] * itemsize if len(shape) > 1 else shape[0] * itemsize
        else:
            if len(strides) > 1 and strides[1] != itemsize:
                raise ValueError("device plane rows must be contiguous")
            pitch = strides[0]
        return cai["data"][0], pitch, _lib.MEM_DEVICE, plane
    arr = np.asarray(plane)
    if arr.ndim != 2:
        raise ValueError("a plane must be 2-D")
    if arr.strides[1] != arr.itemsize:
        arr = np.ascontiguousarray(arr)
    return arr.ctypes.data, arr.strides[0], _lib.MEM_HOST, arr


def raw_frame_bytes(width: int, height: int, bitdepth: int, chroma_format: int = 420) -> int:
    """Bytes of one frame in a raw planar YUV file (xSeq's layout: Y, Cb, Cr; 1 byte per sample up
    to 8 bits, else 2 bytes little endian)."""
    esz = 1 if bitdepth <= 8 else 2
    cw = width if chroma_format == 444 else width // 2
    ch = height // 2 if chroma_format == 420 else height
    return esz * (width * height + 2 * cw * ch)


def frame_from_raw(buffer, width: int, height: int, bitdepth: int, chroma_format: int = 420, index: int = 0):
    """The three planes of frame `index` of a raw planar YUV file held in `buffer` (1-D bytes: a numpy
    uint8 array in host memory or a torch uint8 tensor on the device), as views with no copy and no
    conversion: the kernels read 8-bit samples as bytes and deeper ones as 16-bit words, and never
    upsample chroma (the reference's xSeqPic::xUnpackFrame, libs/pmbb-core/src/xSeq.cpp:231-290,
    is not needed)."""
    esz = 1 if bitdepth <= 8 else 2
    cw = width if chroma_format == 444 else width // 2
    ch = height // 2 if chroma_format == 420 else height
    sizes = [(height, width), (ch, cw), (ch, cw)]
    off = index * raw_frame_bytes(width, height, bitdepth, chroma_format)
    planes = []
    for h, w in sizes:
        n = h * w * esz
        seg = buffer[off:off + n]
        if len(seg) != n:
            raise ValueError("buffer shorter than the frame")
        if hasattr(seg, "__cuda_array_interface__"):
            import torch
            planes.append(seg.view(torch.uint16 if esz == 2 else torch.uint8).view(h, w))
        else:
            planes.append(np.asarray(seg).view(np.uint16 if esz == 2 else np.uint8).reshape(h, w))
        off += n
    return tuple(planes)


def make_frame(planes: Sequence) -> tuple[_lib.QmivFrame, list]:
    if len(planes) != 3:
        raise ValueError("a frame has three planes (Y, Cb, Cr)")
    f = _lib.QmivFrame()
    keep, mems = [], set()
    for c, pl in enumerate(planes):
        ptr, pitch, mem, k = _plane_info(pl)
        f.plane[c] = ptr
        f.pitch[c] = pitch
        mems.add(mem)
        keep.append(k)
    if len(mems) != 1:
        raise ValueError("all planes of a frame must live in the same memory")
    f.mem = mems.pop()
    return f, keep


class Context:
    """Device + HBM budget (qmiv_ctx_create)."""

    def __init__(self, device: int = 0, hbm_budget: int = 0):
        self._lib = library()
        h = ctypes.c_void_p()
        check(self._lib.qmiv_ctx_create(device, hbm_budget, ctypes.byref(h)), "qmiv_ctx_create")
        self.handle = h
        self.device = device

    def memory(self):
        used, budget = ctypes.c_uint64(), ctypes.c_uint64()
        check(self._lib.qmiv_ctx_memory(self.handle, ctypes.byref(used), ctypes.byref(budget)), "qmiv_ctx_memory")
        return used.value, budget.value

    def set_profiling(self, enable: bool = True):
        check(self._lib.qmiv_ctx_set_profiling(self.handle, int(bool(enable))), "qmiv_ctx_set_profiling")

    def stage_times(self, reset: bool = False) -> dict:
        """{stage: (milliseconds, launches)} accumulated while profiling was on."""
        ms, n = (ctypes.c_double * 8)(), (ctypes.c_uint64 * 8)()
        check(self._lib.qmiv_ctx_stage_times(self.handle, ms, n, int(bool(reset))), "qmiv_ctx_stage_times")
        return {name: (ms[i], n[i]) for i, name in enumerate(_lib.STAGES)}

    def close(self):
        if self.handle:
            check(self._lib.qmiv_ctx_destroy(self.handle), "qmiv_ctx_destroy")
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Calc:
    """A metric calculator for one picture shape (qmiv_calc_create)."""

    def __init__(self, ctx: Context, width: int, height: int, bitdepth: int, chroma_format: int = 420, **params):
        self._lib = library()
        self.ctx = ctx
        self.width, self.height, self.bitdepth, self.chroma_format = width, height, bitdepth, chroma_format
        self.params = make_params(**params)
        h = ctypes.c_void_p()
        check(self._lib.qmiv_calc_create(ctx.handle, width, height, bitdepth, chroma_format,
                                         ctypes.byref(self.params), ctypes.byref(h)), "qmiv_calc_create")
        self.handle = h

    def close(self):
        if self.handle:
            check(self._lib.qmiv_calc_destroy(self.handle), "qmiv_calc_destroy")
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- full pipeline -------------------------------------------------------------------------
    def compute(self, frame0, frame1, metrics=None) -> dict:
        f0, k0 = make_frame(frame0)
        f1, k1 = make_frame(frame1)
        res = _lib.QmivResult()
        check(self._lib.qmiv_frame_pair_compute(self.handle, ctypes.byref(f0), ctypes.byref(f1),
                                                metric_mask(metrics), ctypes.byref(res)), "qmiv_frame_pair_compute")
        return res.as_dict()

    def set_color_space(self, color_space_input: int, color_space_metric: int):
        """Colour-space conversion before the metrics (qmiv_calc_set_color_space), codes CS_*."""
        check(self._lib.qmiv_calc_set_color_space(self.handle, color_space_input, color_space_metric),
              "qmiv_calc_set_color_space")

    def compute_masked(self, frame0, frame1, mask, mask_bitdepth: int, metrics=None):
        """Mask mode (qmiv_frame_pair_compute_masked): mask is the mask picture's luma plane (H x W;
        uint8 for mask_bitdepth 8, else uint16; host array or CUDA tensor). Returns (result dict,
        number of non-zero mask samples)."""
        f0, k0 = make_frame(frame0)
        f1, k1 = make_frame(frame1)
        fm, km = make_frame((mask, mask, mask))
        res = _lib.QmivResult()
        nnm = ctypes.c_int32()
        m = metric_mask(metrics) if metrics is not None else PSNR | WSPSNR | IVPSNR
        check(self._lib.qmiv_frame_pair_compute_masked(self.handle, ctypes.byref(f0), ctypes.byref(f1), ctypes.byref(fm),
                                                       mask_bitdepth, m, ctypes.byref(res), ctypes.byref(nnm)),
              "qmiv_frame_pair_compute_masked")
        return res.as_dict(), int(nnm.value)

    def submit(self, frame0, frame1, metrics=None):
        f0, k0 = make_frame(frame0)
        f1, k1 = make_frame(frame1)
        self._inflight = (k0, k1)
        check(self._lib.qmiv_frame_pair_submit(self.handle, ctypes.byref(f0), ctypes.byref(f1), metric_mask(metrics)),
              "qmiv_frame_pair_submit")

    def wait(self, timeout_ms: int = -1) -> dict:
        res = _lib.QmivResult()
        check(self._lib.qmiv_frame_pair_wait(self.handle, timeout_ms, ctypes.byref(res)), "qmiv_frame_pair_wait")
        self._inflight = None
        return res.as_dict()

    # ---- processor-style calls -----------------------------------------------------------------
    def calc_global_color_diff(self, frame0, frame1) -> list:
        f0, k0 = make_frame(frame0)
        f1, k1 = make_frame(frame1)
        out = (ctypes.c_int32 * 4)()
        check(self._lib.qmiv_calc_gcd(self.handle, ctypes.byref(f0), ctypes.byref(f1), out), "qmiv_calc_gcd")
        return list(out)

    def gen_shft_comp_pics(self, frame0, frame1):
        """(SCP0, SCP1) as host uint16 arrays of shape (3, H, W)."""
        f0, k0 = make_frame(frame0)
        f1, k1 = make_frame(frame1)
        shp = (3, self.height, self.width)
        s0, s1 = np.zeros(shp, np.uint16), np.zeros(shp, np.uint16)
        check(self._lib.qmiv_calc_scp(self.handle, ctypes.byref(f0), ctypes.byref(f1), None,
                                      s0.ctypes.data_as(ctypes.c_void_p), s1.ctypes.data_as(ctypes.c_void_p),
                                      _lib.MEM_HOST), "qmiv_calc_scp")
        return s0, s1

    def set_gcd(self, gcd_r2t=None):
        """Use a given GCD (R2T convention) for later calls, as calcPicIVPSNR(Tst, Ref, GCD); None clears."""
        arg = None if gcd_r2t is None else (ctypes.c_int32 * 4)(*gcd_r2t)
        check(self._lib.qmiv_calc_set_gcd(self.handle, arg), "qmiv_calc_set_gcd")

    def cps_rows(self):
        """Per-row CPS SSE (H, 3) of the last computed pair, (R2T, T2R)."""
        a = np.zeros((self.height, 3), np.uint64)
        b = np.zeros((self.height, 3), np.uint64)
        check(self._lib.qmiv_calc_cps_rows(self.handle, a.ctypes.data_as(ctypes.c_void_p),
                                           b.ctypes.data_as(ctypes.c_void_p)), "qmiv_calc_cps_rows")
        return a, b

    def calc_pic_psnr(self, frame0, frame1):
        r = self.compute(frame0, frame1, PSNR)
        return r["psnr"][:3]

    def calc_pic_wspsnr(self, frame0, frame1):
        r = self.compute(frame0, frame1, WSPSNR)
        return r["wspsnr"][:3]

    def calc_pic_ivpsnr(self, frame0, frame1):
        return self.compute(frame0, frame1, IVPSNR)["ivpsnr"]

    def calc_pic_ssim(self, frame0, frame1):
        return self.compute(frame0, frame1, SSIM)["ssim"][:3]

    def calc_pic_msssim(self, frame0, frame1):
        return self.compute(frame0, frame1, MSSSIM)["msssim"][:3]

    def calc_pic_ivssim(self, frame0, frame1):
        return self.compute(frame0, frame1, IVSSIM)["ivssim"]

    def calc_pic_ivmsssim(self, frame0, frame1):
        return self.compute(frame0, frame1, IVMSSSIM)["ivmsssim"]


class Batch:
    """Many frame pairs of uneven shape per call (qmiv_batch_*)."""

    GRAPH, AUTOTUNE = 1, 4

    def __init__(self, ctx: Context, max_pairs: int, max_pixels: int, graph: bool = False, autotune: bool = False,
                 **params):
        self._lib = library()
        self.ctx = ctx
        self.params = make_params(**params)
        flags = (self.GRAPH if graph else 0) | (self.AUTOTUNE if autotune else 0)
        h = ctypes.c_void_p()
        check(self._lib.qmiv_batch_create(ctx.handle, max_pairs, max_pixels, ctypes.byref(self.params),
                                          flags, ctypes.byref(h)), "qmiv_batch_create")
        self.handle = h
        self._inflight = {}

    def close(self):
        if self.handle:
            check(self._lib.qmiv_batch_destroy(self.handle), "qmiv_batch_destroy")
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @staticmethod
    def _descs(pairs):
        descs = (_lib.QmivPairDesc * max(1, len(pairs)))()
        keep = []
        for i, p in enumerate(pairs):
            f0, k0 = make_frame(p["frame0"])
            f1, k1 = make_frame(p["frame1"])
            keep += [k0, k1]
            d = descs[i]
            d.in0, d.in1 = f0, f1
            d.width, d.height, d.bitdepth = p["width"], p["height"], p["bitdepth"]
            d.chroma_format = p.get("chroma_format", 420)
            d.search_range = p.get("search_range", 2)
            d.metric_mask = metric_mask(p.get("metrics"))
        return descs, keep

    def compute(self, pairs: Iterable[dict]) -> list[dict]:
        """pairs: dicts with frame0, frame1, width, height, bitdepth, chroma_format, search_range, metrics."""
        pairs = list(pairs)
        descs, keep = self._descs(pairs)
        out = (_lib.QmivResult * max(1, len(pairs)))()
        check(self._lib.qmiv_batch_compute(self.handle, descs, len(pairs), out), "qmiv_batch_compute")
        return [out[i].as_dict() for i in range(len(pairs))]

    def compute_masked(self, pairs: Iterable[dict], masks, mask_bitdepths) -> tuple[list[dict], list[int]]:
        """Mask mode for many pairs (qmiv_batch_compute_masked): pairs as for compute() (metrics from
        PSNR, WSPSNR, IVPSNR), masks the mask pictures' luma planes (uint8 for bit depth 8, else uint16;
        host arrays or CUDA tensors), mask_bitdepths one per pair. Returns (result dicts, numbers of
        non-zero mask samples)."""
        pairs = list(pairs)
        n = len(pairs)
        descs, keep = self._descs(pairs)
        fm = (_lib.QmivFrame * max(1, n))()
        for i, m in enumerate(masks):
            fm[i], k = make_frame((m, m, m))
            keep.append(k)
        bds = (ctypes.c_int32 * max(1, n))(*mask_bitdepths)
        out = (_lib.QmivResult * max(1, n))()
        nnm = (ctypes.c_int32 * max(1, n))()
        check(self._lib.qmiv_batch_compute_masked(self.handle, descs, fm, bds, n, out, nnm), "qmiv_batch_compute_masked")
        return [out[i].as_dict() for i in range(n)], [int(nnm[i]) for i in range(n)]

    def submit(self, pairs: Iterable[dict]) -> int:
        """Asynchronous compute (qmiv_batch_submit): returns a ticket for wait(); up to two in flight.
        The frames must stay alive and unchanged until the wait."""
        pairs = list(pairs)
        descs, keep = self._descs(pairs)
        t = ctypes.c_uint64()
        check(self._lib.qmiv_batch_submit(self.handle, descs, len(pairs), ctypes.byref(t)), "qmiv_batch_submit")
        self._inflight[t.value] = (len(pairs), pairs, keep)
        return t.value

    def wait(self, ticket: int) -> list[dict]:
        n = self._inflight[ticket][0] if ticket in self._inflight else 0
        out = (_lib.QmivResult * max(1, n))()
        try:
            check(self._lib.qmiv_batch_wait(self.handle, ctypes.c_uint64(ticket), out), "qmiv_batch_wait")
        finally:
            self._inflight.pop(ticket, None)
        return [out[i].as_dict() for i in range(n)]

    def stream(self) -> int:
        """cudaStream_t of the batch, as an integer (for torch.cuda.ExternalStream)."""
        p = ctypes.c_void_p()
        check(self._lib.qmiv_batch_stream(self.handle, ctypes.byref(p)), "qmiv_batch_stream")
        return p.value or 0

    def tuning(self, width, height, bitdepth, search_range):
        """(tile width, tile height, rows per thread) of the CPS work list for pairs of this kind."""
        tw, th, p = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        check(self._lib.qmiv_batch_tuning(self.handle, width, height, bitdepth, search_range, ctypes.byref(tw),
                                          ctypes.byref(th), ctypes.byref(p)), "qmiv_batch_tuning")
        return tw.value, th.value, p.value


class Server:
    """Serving loop (qmiv_server_*): sequences of frame pairs admitted by HBM budget and continuously
    batched over `workers` engines. Frames handed to submit() must stay alive until wait() returns."""

    def __init__(self, ctx: Context, max_batch_pairs: int = 64, max_batch_pixels: int = 64 * 4096 * 2048,
                 workers: int = 2, **params):
        self._lib = library()
        self.ctx = ctx
        self.params = make_params(**params)
        h = ctypes.c_void_p()
        check(self._lib.qmiv_server_create(ctx.handle, ctypes.byref(self.params), max_batch_pairs, max_batch_pixels,
                                           workers, ctypes.byref(h)), "qmiv_server_create")
        self.handle = h
        self._keep = {}

    def close(self):
        if self.handle:
            check(self._lib.qmiv_server_destroy(self.handle), "qmiv_server_destroy")
            self.handle = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, pairs, width, height, bitdepth, chroma_format=420, search_range=2, metrics=None) -> int:
        """pairs: list of (frame0, frame1); every frame a tuple of three planes (numpy or CUDA arrays)."""
        pairs = list(pairs)
        n = len(pairs)
        a0, a1 = (_lib.QmivFrame * max(1, n))(), (_lib.QmivFrame * max(1, n))()
        keep = [a0, a1]
        for i, (f0, f1) in enumerate(pairs):
            a0[i], k0 = make_frame(f0)
            a1[i], k1 = make_frame(f1)
            keep += [k0, k1]
        req = _lib.QmivRequest(width, height, bitdepth, chroma_format, search_range, metric_mask(metrics), n,
                               ctypes.cast(a0, ctypes.POINTER(_lib.QmivFrame)),
                               ctypes.cast(a1, ctypes.POINTER(_lib.QmivFrame)))
        t = ctypes.c_uint64()
        check(self._lib.qmiv_server_submit(self.handle, ctypes.byref(req), ctypes.byref(t)), "qmiv_server_submit")
        self._keep[t.value] = (keep, n)
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1):
        """(per-pair result dicts, request statistics dict)."""
        entry = self._keep.get(ticket)
        n = entry[1] if entry else 0
        out = (_lib.QmivResult * max(1, n))()
        st = _lib.QmivRequestStats()
        check(self._lib.qmiv_server_wait(self.handle, ticket, timeout_ms, out if n else None, ctypes.byref(st)),
              "qmiv_server_wait")
        self._keep.pop(ticket, None)
        return [out[i].as_dict() for i in range(n)], st.as_dict()

    def stats(self, reset: bool = False) -> dict:
        p50, p99, pps = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        done = ctypes.c_int64()
        check(self._lib.qmiv_server_stats(self.handle, ctypes.byref(p50), ctypes.byref(p99), ctypes.byref(pps),
                                          ctypes.byref(done), int(bool(reset))), "qmiv_server_stats")
        return {"p50_ms": p50.value, "p99_ms": p99.value, "pairs_per_s": pps.value, "completed": done.value}
