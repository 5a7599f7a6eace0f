"""CPU checkers for the QMIV metric hot path.

TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
``--impl reference`` legs may import this package, and only to check or to time the reference
side. The product library (qmiv_b200) never imports it.

Two checkers are wrapped here:

* ``Oracle``    -- oracle/libqmiv_oracle.so, the plain-C restatement (qmiv_oracle.c).
* ``Reference`` -- oracle/_ref/<arch>/libqmivref.so, the QMIV reference library itself, compiled
                   from its own sources by oracle/Makefile (only present where it was built).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

PSNR, WSPSNR, IVPSNR, SSIM, MSSSIM, IVSSIM, IVMSSSIM = 1, 2, 4, 8, 16, 32, 64
ALL = 127
# colour spaces of the app's -csi / -csm options (apps/QMIV/src/xUtilsQMIV.h:12-27)
CS_RGB, CS_BGR, CS_GBR, CS_YCBCR = 2, 3, 4, 16
CS_BT601, CS_SMPTE170M, CS_BT709, CS_SMPTE240M, CS_BT2020 = 17, 18, 19, 20, 21
# structural similarity modes (xSSIM::eMode) and margin extension modes (eMrgExt) of the app's -ssm / -ssb
SSM_REGULAR_GAUSSIAN_FLT, SSM_REGULAR_GAUSSIAN_INT, SSM_REGULAR_AVERAGED, SSM_BLOCK_GAUSSIAN_INT, SSM_BLOCK_AVERAGED = 0, 1, 2, 3, 4
BRD_NONE, BRD_NEAREST, BRD_REFLECT, BRD_MIRROR, BRD_CONSTANT, BRD_ZERO = 0, 1, 2, 3, 4, 5


class SsimCfg(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int32), ("border", ctypes.c_int32), ("window", ctypes.c_int32), ("stride", ctypes.c_int32)]


class Params(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_int32), ("height", ctypes.c_int32), ("bitdepth", ctypes.c_int32),
        ("chroma_format", ctypes.c_int32), ("search_range", ctypes.c_int32),
        ("cws", ctypes.c_int32 * 4), ("cwa", ctypes.c_int32 * 4), ("unc", ctypes.c_float * 4),
        ("erp", ctypes.c_int32), ("lon_range", ctypes.c_int32), ("lat_range", ctypes.c_int32),
        ("num_threads", ctypes.c_int32),
    ]


class Result(ctypes.Structure):
    _fields_ = [
        ("gcd_r2t", ctypes.c_int32 * 4), ("exact", ctypes.c_int32 * 4),
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


def make_params(width, height, bitdepth, chroma_format=420, search_range=2, cws=(4, 1, 1, 0), cwa=(4, 1, 1, 0),
                unc=(0.01, 0.01, 0.01, 0.0), erp=False, lon_range=360, lat_range=180, num_threads=0):
    return Params(width, height, bitdepth, chroma_format, search_range, tuple(cws), tuple(cwa), tuple(unc),
                  int(bool(erp)), lon_range, lat_range, num_threads)


def _planes(frame):
    arrs = [np.ascontiguousarray(p) for p in frame]
    return arrs, (ctypes.c_void_p * 3)(*[a.ctypes.data for a in arrs])


def _u16(a):
    return np.ascontiguousarray(a, dtype=np.uint16)


class _Lib:
    def __init__(self, path):
        self.path = path
        self.lib = ctypes.CDLL(path)


class Oracle(_Lib):
    """The plain-C restatement."""

    def __init__(self, path=None):
        path = path or os.path.join(HERE, "libqmiv_oracle.so")
        if not os.path.exists(path):
            build_oracle()
        super().__init__(path)
        L = self.lib
        L.qo_compute_pair.restype = ctypes.c_int
        L.qo_num_scales.restype = ctypes.c_int32

    def compute_pair(self, params: Params, frame0, frame1, mask=ALL, want_scp=False):
        a0, p0 = _planes(frame0)
        a1, p1 = _planes(frame1)
        res = Result()
        n = params.width * params.height * 3
        scp0 = np.zeros(n, np.uint16) if want_scp else None
        scp1 = np.zeros(n, np.uint16) if want_scp else None
        rc = self.lib.qo_compute_pair(ctypes.byref(params), p0, p1, ctypes.c_uint32(mask), ctypes.byref(res),
                                      scp0.ctypes.data_as(ctypes.c_void_p) if want_scp else None,
                                      scp1.ctypes.data_as(ctypes.c_void_p) if want_scp else None)
        if rc != 0:
            raise RuntimeError(f"qo_compute_pair failed ({rc})")
        out = res.as_dict()
        if want_scp:
            shp = (3, params.height, params.width)
            out["scp0"], out["scp1"] = scp0.reshape(shp), scp1.reshape(shp)
        return out

    def compute_pair_cs(self, params: Params, frame0, frame1, cs_in, cs_metric, mask=ALL & ~(MSSSIM | IVMSSSIM)):
        """The pipeline after the app's colour-space conversion (-csi cs_in, -csm cs_metric)."""
        a0, p0 = _planes(frame0)
        a1, p1 = _planes(frame1)
        res = Result()
        rc = self.lib.qo_compute_pair_cs(ctypes.byref(params), p0, p1, ctypes.c_uint32(mask), ctypes.c_int32(cs_in),
                                         ctypes.c_int32(cs_metric), ctypes.byref(res))
        if rc != 0:
            raise RuntimeError(f"qo_compute_pair_cs failed ({rc})")
        return res.as_dict()

    def compute_pair_ssim(self, params: Params, frame0, frame1, mode, border, window, stride, mask=ALL):
        """The pipeline with the app's structural similarity options (-ssm, -ssb, -ssw, -sss)."""
        a0, p0 = _planes(frame0)
        a1, p1 = _planes(frame1)
        res = Result()
        cfg = SsimCfg(mode, border, window, stride)
        rc = self.lib.qo_compute_pair_ssim(ctypes.byref(params), p0, p1, ctypes.c_uint32(mask), ctypes.byref(cfg),
                                           ctypes.byref(res))
        if rc != 0:
            raise RuntimeError(f"qo_compute_pair_ssim failed ({rc})")
        return res.as_dict()

    def compute_pair_masked(self, params: Params, frame0, frame1, mask_plane, mask_bitdepth, mask=PSNR | WSPSNR | IVPSNR):
        """Mask mode (GCD-M, PSNR-M, WS-PSNR-M, IV-PSNR-M); returns (result dict, NumNonMasked)."""
        a0, p0 = _planes(frame0)
        a1, p1 = _planes(frame1)
        m = np.ascontiguousarray(mask_plane, np.uint8 if mask_bitdepth <= 8 else np.uint16)
        res = Result()
        nnm = ctypes.c_int32()
        rc = self.lib.qo_compute_pair_masked(ctypes.byref(params), p0, p1, m.ctypes.data_as(ctypes.c_void_p),
                                             ctypes.c_int32(mask_bitdepth), ctypes.c_uint32(mask), ctypes.byref(res),
                                             ctypes.byref(nnm))
        if rc != 0:
            raise RuntimeError(f"qo_compute_pair_masked failed ({rc})")
        return res.as_dict(), int(nnm.value)

    def unpack444(self, frame, width, height, bitdepth, chroma_format):
        a, p = _planes(frame)
        dst = np.zeros((3, height, width), np.uint16)
        self.lib.qo_unpack444(p, width, height, bitdepth, chroma_format, dst.ctypes.data_as(ctypes.c_void_p))
        return dst

    def gcd(self, tst444, ref444, bitdepth, coef=(0.01, 0.01, 0.01, 0.0)):
        t, r = _u16(tst444), _u16(ref444)
        out = (ctypes.c_int32 * 4)()
        self.lib.qo_gcd(t.ctypes.data_as(ctypes.c_void_p), r.ctypes.data_as(ctypes.c_void_p), t.shape[2], t.shape[1],
                        bitdepth, (ctypes.c_float * 4)(*coef), out)
        return list(out)

    def cps(self, tst444, ref444, bitdepth, gcd, search_range=2, cws=(4, 1, 1, 0), want_scp=True):
        t, r = _u16(tst444), _u16(ref444)
        H, W = t.shape[1], t.shape[2]
        rows = np.zeros((H, 3), np.uint64)
        scp = np.zeros((3, H, W), np.uint16) if want_scp else None
        self.lib.qo_cps(t.ctypes.data_as(ctypes.c_void_p), r.ctypes.data_as(ctypes.c_void_p), W, H, bitdepth,
                        (ctypes.c_int32 * 4)(*gcd), search_range, (ctypes.c_int32 * 4)(*cws),
                        rows.ctypes.data_as(ctypes.c_void_p), scp.ctypes.data_as(ctypes.c_void_p) if want_scp else None)
        return rows, scp

    def cps_rows_std(self, tst444, ref444, gcd, search_range=2, cws=(4, 1, 1, 0)):
        t, r = _u16(tst444), _u16(ref444)
        H, W = t.shape[1], t.shape[2]
        rows = np.zeros((H, 3), np.uint64)
        self.lib.qo_cps_rows_std(t.ctypes.data_as(ctypes.c_void_p), r.ctypes.data_as(ctypes.c_void_p), W, H,
                                 (ctypes.c_int32 * 4)(*gcd), search_range, (ctypes.c_int32 * 4)(*cws),
                                 rows.ctypes.data_as(ctypes.c_void_p))
        return rows

    def ws_weights(self, height, lat_range=180):
        w = np.zeros(height, np.float64)
        corr = ctypes.c_double()
        self.lib.qo_ws_weights(height, lat_range, w.ctypes.data_as(ctypes.c_void_p), ctypes.byref(corr))
        return w, corr.value

    def ssim_pic(self, tst444, ref444, bitdepth, calc_l=True, ws_weights=None):
        t, r = _u16(tst444), _u16(ref444)
        out = (ctypes.c_double * 3)()
        wp = None
        if ws_weights is not None:
            ws_weights = np.ascontiguousarray(ws_weights, np.float64)
            wp = ws_weights.ctypes.data_as(ctypes.c_void_p)
        self.lib.qo_ssim_pic(t.ctypes.data_as(ctypes.c_void_p), r.ctypes.data_as(ctypes.c_void_p), t.shape[2],
                             t.shape[1], bitdepth, int(calc_l), wp, out)
        return list(out)

    def msssim_pic(self, tst444, ref444, bitdepth):
        t, r = _u16(tst444), _u16(ref444)
        out = (ctypes.c_double * 3)()
        rc = self.lib.qo_msssim_pic(t.ctypes.data_as(ctypes.c_void_p), r.ctypes.data_as(ctypes.c_void_p),
                                    t.shape[2], t.shape[1], bitdepth, out)
        if rc != 0:
            raise ValueError("picture too small for MS-SSIM")
        return list(out)

    def num_scales(self, width, height):
        return int(self.lib.qo_num_scales(width, height))


def host_arch():
    """Best micro-architecture level this host's CPU runs (x86-64-v4/v3/v2)."""
    flags = set()
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    flags = set(line.split(":", 1)[1].split())
                    break
    except OSError:
        pass
    if {"avx512f", "avx512bw", "avx512dq", "avx512vl"} <= flags:
        return "x86-64-v4"
    if {"avx2", "fma", "bmi2"} <= flags:
        return "x86-64-v3"
    return "x86-64-v2"


def reference_dir(arch=None):
    return os.path.join(HERE, "_ref", arch or host_arch())


def reference_available(arch=None):
    d = reference_dir(arch)
    return os.path.exists(os.path.join(d, "libqmivref.so"))


class Reference(_Lib):
    """The QMIV reference library compiled from its own sources (oracle/_ref)."""

    def __init__(self, arch=None):
        path = os.path.join(reference_dir(arch), "libqmivref.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        super().__init__(path)
        L = self.lib
        L.ref_compute_pair.restype = ctypes.c_int
        L.ref_ssim_block.restype = ctypes.c_double
        L.ref_xorshift32.restype = ctypes.c_uint32
        L.ref_xorshift32.argtypes = [ctypes.c_uint32]
        L.ref_add_block_noise.restype = ctypes.c_uint32

    def compute_pair(self, params: Params, frame0, frame1, mask=ALL, want_scp=False):
        a0, p0 = _planes(frame0)
        a1, p1 = _planes(frame1)
        res = Result()
        n = params.width * params.height * 3
        scp0 = np.zeros(n, np.uint16) if want_scp else None
        scp1 = np.zeros(n, np.uint16) if want_scp else None
        rc = self.lib.ref_compute_pair(ctypes.byref(params), p0, p1, ctypes.c_uint32(mask), ctypes.byref(res),
                                       scp0.ctypes.data_as(ctypes.c_void_p) if want_scp else None,
                                       scp1.ctypes.data_as(ctypes.c_void_p) if want_scp else None)
        if rc != 0:
            raise RuntimeError(f"ref_compute_pair failed ({rc})")
        out = res.as_dict()
        if want_scp:
            shp = (3, params.height, params.width)
            out["scp0"], out["scp1"] = scp0.reshape(shp), scp1.reshape(shp)
        return out

    def compute_pair_cs(self, params: Params, frame0, frame1, cs_in, cs_metric, mask=ALL & ~(MSSSIM | IVMSSSIM)):
        """The pipeline with the app's colour-space conversion (-csi cs_in, -csm cs_metric)."""
        a0, p0 = _planes(frame0)
        a1, p1 = _planes(frame1)
        res = Result()
        rc = self.lib.ref_compute_pair_cs(ctypes.byref(params), p0, p1, ctypes.c_uint32(mask), ctypes.c_int32(cs_in),
                                          ctypes.c_int32(cs_metric), ctypes.byref(res))
        if rc != 0:
            raise RuntimeError(f"ref_compute_pair_cs failed ({rc})")
        return res.as_dict()

    def compute_pair_ssim(self, params: Params, frame0, frame1, mode, border, window, stride, mask=ALL):
        """The pipeline with the app's structural similarity options (-ssm, -ssb, -ssw, -sss)."""
        a0, p0 = _planes(frame0)
        a1, p1 = _planes(frame1)
        res = Result()
        cfg = SsimCfg(mode, border, window, stride)
        rc = self.lib.ref_compute_pair_ssim(ctypes.byref(params), p0, p1, ctypes.c_uint32(mask), ctypes.byref(cfg),
                                            ctypes.byref(res))
        if rc != 0:
            raise RuntimeError(f"ref_compute_pair_ssim failed ({rc})")
        return res.as_dict()

    def compute_pair_masked(self, params: Params, frame0, frame1, mask_plane, mask_bitdepth, mask=PSNR | WSPSNR | IVPSNR):
        """The app's mask mode (GCD-M, PSNR-M, WS-PSNR-M, IV-PSNR-M); returns (result dict, NumNonMasked)."""
        a0, p0 = _planes(frame0)
        a1, p1 = _planes(frame1)
        m = np.ascontiguousarray(mask_plane, np.uint8 if mask_bitdepth <= 8 else np.uint16)
        res = Result()
        nnm = ctypes.c_int32()
        rc = self.lib.ref_compute_pair_masked(ctypes.byref(params), p0, p1, m.ctypes.data_as(ctypes.c_void_p),
                                              ctypes.c_int32(mask_bitdepth), ctypes.c_uint32(mask), ctypes.byref(res),
                                              ctypes.byref(nnm))
        if rc != 0:
            raise RuntimeError(f"ref_compute_pair_masked failed ({rc})")
        return res.as_dict(), int(nnm.value)

    def cps_rows(self, tst444, ref444, bitdepth, gcd, search_range=2, cws=(4, 1, 1, 0)):
        t, r = _u16(tst444), _u16(ref444)
        H, W = t.shape[1], t.shape[2]
        a = np.zeros((H, 3), np.uint64)
        b = np.zeros((H, 3), np.uint64)
        self.lib.ref_cps_rows(t.ctypes.data_as(ctypes.c_void_p), r.ctypes.data_as(ctypes.c_void_p), W, H, bitdepth,
                              (ctypes.c_int32 * 4)(*gcd), search_range, (ctypes.c_int32 * 4)(*cws),
                              a.ctypes.data_as(ctypes.c_void_p), b.ctypes.data_as(ctypes.c_void_p))
        return a, b

    def gcd(self, tst444, ref444, bitdepth, coef=(0.01, 0.01, 0.01, 0.0)):
        t, r = _u16(tst444), _u16(ref444)
        out = (ctypes.c_int32 * 4)()
        self.lib.ref_gcd(t.ctypes.data_as(ctypes.c_void_p), r.ctypes.data_as(ctypes.c_void_p), t.shape[2], t.shape[1],
                         bitdepth, (ctypes.c_float * 4)(*coef), out)
        return list(out)

    def xorshift32(self, state):
        return int(self.lib.ref_xorshift32(ctypes.c_uint32(state)))

    def fill_perlin(self, height, width, bitdepth, headroom, seed):
        dst = np.zeros((height, width), np.uint16)
        self.lib.ref_fill_perlin(dst.ctypes.data_as(ctypes.c_void_p), width, width, height, bitdepth, headroom,
                                 ctypes.c_uint32(seed))
        return dst

    def add_block_noise(self, src_padded, margin, width, height, bitdepth, state):
        """src_padded: (H+2m, W+2m) uint16 with an edge-replicated margin. Returns (dst, state)."""
        src = np.ascontiguousarray(src_padded, np.uint16)
        dst = np.zeros((height, width), np.uint16)
        stride = src.shape[1]
        origin = src.ctypes.data + (margin * stride + margin) * 2
        st = self.lib.ref_add_block_noise(dst.ctypes.data_as(ctypes.c_void_p), ctypes.c_void_p(origin), width, stride,
                                          width, height, bitdepth, ctypes.c_uint32(state))
        return dst, int(st)


def build_oracle():
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def build_reference(ref_root=None, jobs=8):
    """Compile the reference from its own sources into oracle/_ref (only where they exist).

    ref_root: the reference's source tree; QMIV_REFERENCE_ROOT is read when it is not given. Without
    either, nothing is built."""
    ref_root = ref_root or os.environ.get("QMIV_REFERENCE_ROOT")
    if not ref_root or not os.path.isdir(ref_root):
        return False
    subprocess.run(["make", "-s", "-C", HERE, f"-j{jobs}", "ref", f"REF={ref_root}"], check=True)
    if os.path.exists(os.path.join(os.path.dirname(HERE), "qmiv_b200", "libqmiv_b200.so")):
        subprocess.run(["make", "-s", "-C", HERE, f"-j{jobs}", "shimcheck", f"REF={ref_root}"], check=True)
    return True


def shim_check_path(arch=None):
    """The drop-in adapter's check program (oracle/Makefile shimcheck), or None where it is not built."""
    p = os.path.join(reference_dir(arch), "shim_check")
    return p if os.path.exists(p) else None
