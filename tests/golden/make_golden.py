"""Generates the golden fixtures in tests/golden/ by running the QMIV reference itself.

The reference is compiled from its own sources by oracle/Makefile into oracle/_ref/<arch>/; this
script only runs where that build exists (the development container). The GPU box never runs it:
tests read the committed JSON / npz files.

The x86-64-v3 (AVX2) build is used: the x86-64-v4 (AVX-512) build of the reference mis-converts
8-bit 4:2:0 chroma when the picture width is 64 modulo 128 (xPixelOpsAVX512.cpp CvtUpsampleHV builds
a store mask with a 64-bit shift by 64), which the portable and AVX2 builds do not.

    python tests/golden/make_golden.py            # golden.json
    python tests/golden/make_golden.py masked     # golden_masked.json (mask mode)
    python tests/golden/make_golden.py colour     # golden_colour.json (colour-space conversion)
    python tests/golden/make_golden.py ssim_modes # golden_ssim_modes.json (structural similarity options)

The structural similarity option fixtures come from the x86-64-v2 build. GCC contracts a*b+c into
fused multiply-adds by default in C++ (-ffp-contract=fast) wherever the target has FMA (x86-64-v3 and
up), which moves the last bits of the non-power-of-two-scaled window formulas; the v2 build evaluates
the arithmetic as written. The v3 values are stored beside them to bound that difference.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import oracle  # noqa: E402
from detgen import det_mask, det_pair, hash32, to444  # noqa: E402

ARCH = "x86-64-v3"

# (width, height, bitdepth, chroma_format, R, erp, seed, extra params)
PIPELINE_CASES = [
    (64, 64, 8, 420, 2, False, 1, {}),
    (96, 64, 10, 420, 2, True, 2, {}),
    (128, 96, 8, 444, 2, False, 3, {}),
    (130, 66, 10, 422, 4, True, 4, {}),
    (256, 128, 10, 420, 2, True, 5, {}),
    (200, 100, 8, 420, 3, False, 6, {}),
    (320, 192, 10, 420, 5, True, 7, {}),
    (66, 34, 8, 420, 1, False, 8, {}),
    (512, 256, 10, 420, 2, True, 9, {}),
    (1024, 512, 8, 420, 4, False, 10, {}),
    (1920, 1080, 8, 420, 2, False, 11, {}),
    (96, 96, 14, 444, 2, False, 12, {}),
    (128, 64, 12, 420, 2, True, 13, {}),
    (64, 64, 10, 420, 2, False, 14, {"cws": (2, 1, 1, 0), "cwa": (6, 1, 1, 0)}),
    (128, 128, 10, 420, 3, True, 15, {"unc": (0.02, 0.02, 0.02, 0.0)}),
    (192, 64, 8, 420, 2, False, 16, {"lat_range": 120}),
    (96, 64, 10, 420, 2, True, 17, {"variant": "exact_chroma"}),
    (64, 48, 8, 420, 2, False, 18, {"variant": "identical"}),
]

CPS_SIZES = [(64, 64)]
CPS_BITDEPTHS = [8, 10, 14]
CPS_GCDS = [(0, 0, 0, 0), (1, 1, 1, 0), (-1, -1, -1, 0), (-1, 1, 1, 0)]


def fhex(v):
    return float(v).hex()


def case_frames(W, H, bd, cf, seed, variant=None):
    f0, f1 = det_pair(W, H, bd, seed, cf)
    if variant == "exact_chroma":
        f1 = (f1[0], f0[1].copy(), f0[2].copy())
    elif variant == "identical":
        f1 = tuple(p.copy() for p in f0)
    return f0, f1


def make_pipeline(ref):
    out = []
    for (W, H, bd, cf, R, erp, seed, extra) in PIPELINE_CASES:
        extra = dict(extra)
        variant = extra.pop("variant", None)
        kw = dict(search_range=R, erp=erp, num_threads=8)
        kw.update({k: v for k, v in extra.items() if k in ("cws", "cwa", "unc", "lat_range")})
        p = oracle.make_params(W, H, bd, cf, **kw)
        f0, f1 = case_frames(W, H, bd, cf, seed, variant)
        mask = oracle.ALL
        if oracle.Oracle().num_scales(W, H) < 1:
            mask &= ~(oracle.MSSSIM | oracle.IVMSSSIM)
        r = ref.compute_pair(p, f0, f1, mask, want_scp=True)
        t0, t1 = to444(f0, cf), to444(f1, cf)
        g = r["gcd_r2t"]
        rows_r2t, _ = ref.cps_rows(t0, t1, bd, g, R, kw.get("cws", (4, 1, 1, 0)))
        rows_t2r, _ = ref.cps_rows(t1, t0, bd, [-x for x in g], R, kw.get("cws", (4, 1, 1, 0)))
        exp = {}
        for k, v in r.items():
            if k.startswith("scp"):
                exp[k + "_sha256"] = hashlib.sha256(np.ascontiguousarray(v).tobytes()).hexdigest()
            elif isinstance(v, list):
                exp[k] = [fhex(x) if isinstance(x, float) else int(x) for x in v]
            else:
                exp[k] = fhex(v) if isinstance(v, float) else int(v)
        out.append(dict(width=W, height=H, bitdepth=bd, chroma_format=cf, search_range=R, erp=erp, seed=seed,
                        variant=variant, params={k: list(v) if isinstance(v, tuple) else v
                                                 for k, v in kw.items() if k != "num_threads"},
                        mask=mask, expected=exp,
                        cps_rows_r2t=rows_r2t.astype(np.int64).tolist(),
                        cps_rows_t2r=rows_t2r.astype(np.int64).tolist()))
        print("pipeline", W, H, bd, cf, R, erp, variant, r["ivpsnr"])
    return out


def make_cps(ref):
    """Fixtures in the manner of libs/pmbb-ivqm/test/test-xCorrespPixelShift.cpp: Perlin-noise originals
    (xPerlinNoise::fillPerlinNoiseI), block-noise modifications (xTestUtilsIVQM::addBlockNoise) on all
    three components, margin 8 edge-replicated, R = 2, weights 4:1:1, GCD in {0, +1, -1, (-1,+1,+1)}."""
    state = 666  # xTestUtils::c_XorShiftSeed
    arrays, cases = {}, []
    margin = 8
    for (W, H) in CPS_SIZES:
        for bd in CPS_BITDEPTHS:
            org = np.zeros((3, H, W), np.uint16)
            for c in range(3):
                org[c] = ref.fill_perlin(H, W, bd, 8, state)
                state = ref.xorshift32(state)
            mod = np.zeros_like(org)
            for c in range(3):
                pad = np.pad(org[c], margin, mode="edge")
                mod[c], state = ref.add_block_noise(pad, margin, W, H, bd, state)
            key = f"{W}x{H}_{bd}"
            arrays[key + "_org"], arrays[key + "_mod"] = org, mod
            for g in CPS_GCDS:
                a, b = ref.cps_rows(mod, org, bd, g, 2, (4, 1, 1, 0))
                cases.append(dict(key=key, width=W, height=H, bitdepth=bd, gcd=list(g),
                                  rows_interleaved=a.astype(np.int64).tolist(), rows_planar=b.astype(np.int64).tolist()))
            print("cps", key, int(org.max()), int(mod.max()))
    np.savez_compressed(os.path.join(HERE, "cps_fixtures.npz"), **arrays)
    return cases


def make_gcd(ref):
    """xGlobClrDiff::CalcGlobalColorDiff on deterministic pictures, default and unit coefficients."""
    cases = []
    for (W, H, bd, seed) in [(128, 128, 8, 1), (256, 128, 10, 2), (128, 256, 12, 3), (256, 256, 14, 4)]:
        f0, f1 = det_pair(W, H, bd, seed, 444, offset=(5, -7, 1))
        t0, t1 = to444(f0, 444), to444(f1, 444)
        for coef in [(0.01, 0.01, 0.01, 0.0), (1.0, 1.0, 1.0, 1.0), (0.003, 0.02, 0.5, 0.0)]:
            cases.append(dict(width=W, height=H, bitdepth=bd, seed=seed, coef=list(coef),
                              gcd_10=ref.gcd(t1, t0, bd, coef), gcd_01=ref.gcd(t0, t1, bd, coef)))
    return cases


def make_ssim_windows(ref):
    """xStructSim::CalcBlckAvg (dispatched) and xStructSimSTD::CalcBlckAvg on 8x8 windows."""
    import ctypes
    cases = []
    for bd in (8, 10, 12, 14):
        maxv = (1 << bd) - 1
        for k in range(8):
            h = hash32(np.arange(128, dtype=np.uint32) + np.uint32(bd * 1000 + k * 7919))
            t = (h[:64] % (maxv + 1)).astype(np.uint16).reshape(8, 8)
            r = (h[64:] % (maxv + 1)).astype(np.uint16).reshape(8, 8)
            if k % 2:
                r = np.clip(t.astype(np.int64) + (h[64:].reshape(8, 8) % 21).astype(np.int64) - 10, 0, maxv).astype(np.uint16)
            tt, rr = np.ascontiguousarray(t), np.ascontiguousarray(r)
            vals = {}
            for calc_l in (0, 1):
                for std in (0, 1):
                    v = ref.lib.ref_ssim_block(tt.ctypes.data_as(ctypes.c_void_p), rr.ctypes.data_as(ctypes.c_void_p),
                                               8, 8, bd, calc_l, std)
                    vals[f"l{calc_l}_std{std}"] = fhex(v)
            cases.append(dict(bitdepth=bd, k=k, tst=t.tolist(), ref=r.tolist(), values=vals))
    return cases


# mask mode: (width, height, bitdepth, chroma_format, R, erp, seed, mask bit depth, mask kind)
MASKED_CASES = [
    (64, 64, 10, 420, 2, True, 21, 8, "binary"),
    (64, 48, 8, 444, 3, False, 22, 10, "weights"),
    (96, 64, 10, 422, 2, True, 23, 14, "weights"),
    (130, 66, 8, 420, 1, False, 24, 8, "sparse"),
    (128, 64, 12, 420, 2, True, 25, 10, "binary"),
    (64, 64, 10, 420, 4, False, 26, 8, "ones"),
    (256, 128, 10, 420, 2, True, 27, 8, "region"),
    (200, 100, 8, 420, 5, False, 28, 12, "weights"),
    (66, 34, 10, 420, 2, True, 29, 8, "binary"),
    (1920, 1080, 8, 420, 2, False, 30, 8, "binary"),
]


def make_masked(ref):
    """The app's mask mode (xAppQMIV.cpp:900-1030) run by the compiled reference: GCD-M, PSNR-M,
    WS-PSNR-M, IV-PSNR-M and the number of non-masked samples. Frames and masks come from detgen."""
    out = []
    for (W, H, bd, cf, R, erp, seed, mbd, kind) in MASKED_CASES:
        p = oracle.make_params(W, H, bd, cf, search_range=R, erp=erp, num_threads=8)
        f0, f1 = det_pair(W, H, bd, seed, cf)
        m = det_mask(W, H, mbd, seed, kind)
        r, nnm = ref.compute_pair_masked(p, f0, f1, m, mbd)
        keys = ["gcd_r2t", "exact", "psnr", "psnr_pic", "wspsnr", "wspsnr_pic", "ivpsnr", "ivpsnr_r2t", "ivpsnr_t2r"]
        exp = {k: ([fhex(x) if isinstance(x, float) else int(x) for x in r[k]] if isinstance(r[k], list)
                   else fhex(r[k])) for k in keys}
        exp["num_non_masked"] = nnm
        out.append(dict(width=W, height=H, bitdepth=bd, chroma_format=cf, search_range=R, erp=erp, seed=seed,
                        mask_bitdepth=mbd, mask_kind=kind, expected=exp))
        print("masked", W, H, bd, cf, R, erp, mbd, kind, nnm, r["ivpsnr"])
    return out


def main_masked():
    ref = oracle.Reference(ARCH)
    data = dict(generator="tests/golden/make_golden.py masked", reference_build=ARCH, masked=make_masked(ref))
    with open(os.path.join(HERE, "golden_masked.json"), "w") as f:
        json.dump(data, f, separators=(",", ":"))
    print("wrote", os.path.join(HERE, "golden_masked.json"))


# colour-space conversion: (width, height, bitdepth, chroma_format, R, erp, seed, -csi, -csm)
COLOUR_CASES = [
    (64, 48, 8, 420, 2, False, 41, 19, 2),      # YCbCr BT.709 -> RGB
    (64, 48, 10, 444, 2, True, 42, 2, 17),      # RGB -> YCbCr BT.601
    (96, 64, 10, 444, 3, False, 43, 3, 2),      # BGR reordered to RGB
    (96, 64, 8, 444, 2, True, 44, 4, 2),        # GBR reordered to RGB
    (128, 64, 10, 420, 2, True, 45, 21, 2),     # YCbCr BT.2020 -> RGB
    (64, 64, 12, 444, 2, False, 46, 2, 20),     # RGB -> YCbCr SMPTE 240M
    (66, 34, 8, 444, 1, False, 47, 4, 21),      # GBR -> YCbCr BT.2020 (no reordering)
    (64, 48, 10, 420, 4, True, 48, 18, 3),      # YCbCr SMPTE 170M -> BGR (plain RGB order)
    (256, 128, 10, 444, 2, True, 49, 2, 19),    # RGB -> YCbCr BT.709
]


def make_colour(ref):
    """The pipeline after the app's colour-space conversion (xAppQMIV.cpp:853-891), all metrics but the
    multi-scale ones, run by the compiled reference. Frames come from detgen."""
    out = []
    mask = oracle.ALL & ~(oracle.MSSSIM | oracle.IVMSSSIM)
    for (W, H, bd, cf, R, erp, seed, cs_in, cs_metric) in COLOUR_CASES:
        p = oracle.make_params(W, H, bd, cf, search_range=R, erp=erp, num_threads=8)
        f0, f1 = det_pair(W, H, bd, seed, cf)
        r = ref.compute_pair_cs(p, f0, f1, cs_in, cs_metric, mask)
        exp = {k: ([fhex(x) if isinstance(x, float) else int(x) for x in v] if isinstance(v, list)
                   else (fhex(v) if isinstance(v, float) else int(v))) for k, v in r.items()}
        out.append(dict(width=W, height=H, bitdepth=bd, chroma_format=cf, search_range=R, erp=erp, seed=seed,
                        cs_in=cs_in, cs_metric=cs_metric, mask=mask, expected=exp))
        print("colour", W, H, bd, cf, R, erp, cs_in, cs_metric, r["ivpsnr"])
    return out


def main_colour():
    ref = oracle.Reference(ARCH)
    data = dict(generator="tests/golden/make_golden.py colour", reference_build=ARCH, colour=make_colour(ref))
    with open(os.path.join(HERE, "golden_colour.json"), "w") as f:
        json.dump(data, f, separators=(",", ":"))
    print("wrote", os.path.join(HERE, "golden_colour.json"))


# structural similarity options: (width, height, bitdepth, chroma_format, R, erp, seed, -ssm, -ssb, -ssw, -sss)
SSM_FLT, SSM_INT, SSM_AVG, SSM_BGI, SSM_BAVG = 0, 1, 2, 3, 4
SSIM_MODE_CASES = [
    (64, 48, 10, 420, 2, True, 61, SSM_FLT, 0, 11, 1),      # the original paper's setting
    (96, 64, 8, 420, 2, False, 62, SSM_FLT, 0, 11, 4),
    (72, 40, 10, 444, 3, True, 63, SSM_FLT, 1, 11, 1),      # Nearest
    (66, 34, 8, 422, 1, False, 64, SSM_FLT, 2, 11, 3),      # Reflect
    (64, 64, 12, 420, 2, True, 65, SSM_FLT, 3, 11, 2),      # Mirror
    (48, 40, 10, 444, 2, False, 66, SSM_FLT, 4, 11, 5),     # Constant (65535)
    (64, 48, 8, 420, 5, True, 67, SSM_FLT, 5, 11, 11),      # Zero
    (128, 64, 10, 420, 2, True, 68, SSM_INT, 0, 11, 1),
    (80, 48, 14, 444, 2, False, 69, SSM_INT, 1, 11, 4),
    (64, 64, 10, 420, 4, True, 70, SSM_INT, 4, 11, 3),
    (96, 64, 10, 420, 2, True, 71, SSM_AVG, 0, 11, 1),
    (64, 48, 8, 444, 2, False, 72, SSM_AVG, 3, 11, 2),
    (130, 66, 10, 422, 2, True, 73, SSM_AVG, 5, 11, 4),
    (64, 64, 10, 420, 2, True, 74, SSM_BGI, 0, 8, 4),
    (96, 64, 8, 420, 3, False, 75, SSM_BGI, 0, 8, 8),
    (128, 96, 10, 444, 2, True, 76, SSM_BGI, 0, 16, 4),
    (64, 48, 12, 420, 2, False, 77, SSM_BGI, 0, 16, 1),
    (64, 64, 10, 420, 2, True, 78, SSM_BAVG, 0, 8, 1),
    (96, 64, 8, 420, 2, False, 79, SSM_BAVG, 0, 8, 8),
    (72, 56, 10, 444, 2, True, 80, SSM_BAVG, 0, 8, 3),
    (128, 96, 10, 420, 2, True, 81, SSM_BAVG, 0, 16, 4),
    (96, 64, 14, 444, 2, False, 82, SSM_BAVG, 0, 16, 16),
    (160, 96, 10, 420, 2, True, 83, SSM_BAVG, 0, 32, 4),
    (130, 70, 8, 422, 2, False, 84, SSM_BAVG, 0, 32, 7),
    (256, 128, 10, 420, 2, True, 85, SSM_FLT, 0, 11, 1),
    # 15- and 16-bit pictures: the regular Gaussian windows sum in double / int64 in the reference, so
    # plain SSIM is defined there (not MS-SSIM: the SIMD downsampling adds in signed 16-bit lanes; not the
    # IV metrics: the search's int32 errors overflow)
    (64, 48, 16, 444, 2, False, 86, SSM_FLT, 0, 11, 1, 1 | 8),
    (96, 64, 15, 420, 2, True, 87, SSM_INT, 1, 11, 2, 1 | 2 | 8),
    (72, 72, 16, 422, 2, False, 88, SSM_FLT, 4, 11, 3, 8),
]
SSIM_KEYS = ("ssim", "ssim_pic", "msssim", "msssim_pic", "ivssim", "ivssim_r2t", "ivssim_t2r", "ivmsssim", "ivmsssim_r2t",
             "ivmsssim_t2r")


def make_ssim_modes(ref, ref_fma):
    """Every metric of the pipeline under the app's -ssm / -ssb / -ssw / -sss options, run by the
    compiled reference (xSSIM::setStructSimParams, xAppQMIV.cpp:722; border extension of the pictures
    and the SCPs, :798 and :918-926). Frames come from detgen."""
    out = []
    for case in SSIM_MODE_CASES:
        (W, H, bd, cf, R, erp, seed, mode, border, window, stride), extra = case[:11], case[11:]
        p = oracle.make_params(W, H, bd, cf, search_range=R, erp=erp, num_threads=8)
        f0, f1 = det_pair(W, H, bd, seed, cf)
        mask = extra[0] if extra else oracle.ALL
        if oracle.Oracle().num_scales(W, H) < 1:
            mask &= ~(oracle.MSSSIM | oracle.IVMSSSIM)
        r = ref.compute_pair_ssim(p, f0, f1, mode, border, window, stride, mask)
        r3 = ref_fma.compute_pair_ssim(p, f0, f1, mode, border, window, stride, mask)
        enc = lambda d: {k: ([fhex(x) if isinstance(x, float) else int(x) for x in v] if isinstance(v, list)
                             else (fhex(v) if isinstance(v, float) else int(v))) for k, v in d.items()}
        out.append(dict(width=W, height=H, bitdepth=bd, chroma_format=cf, search_range=R, erp=erp, seed=seed,
                        ssim_mode=mode, ssim_border=border, ssim_window=window, ssim_stride=stride, mask=mask,
                        expected=enc(r), expected_fma_build={k: v for k, v in enc(r3).items() if k in SSIM_KEYS}))
        dev = max(abs(a - b) for k in SSIM_KEYS for a, b in zip(r[k] if isinstance(r[k], list) else [r[k]],
                                                                 r3[k] if isinstance(r3[k], list) else [r3[k]]))
        print("ssim_modes", W, H, bd, cf, R, erp, mode, border, window, stride, r["ssim_pic"], r["ivssim"], "v3 dev", dev)
    return out


def main_ssim_modes():
    ref = oracle.Reference("x86-64-v2")
    ref_fma = oracle.Reference("x86-64-v3")
    data = dict(generator="tests/golden/make_golden.py ssim_modes", reference_build="x86-64-v2",
                fma_build="x86-64-v3", ssim_modes=make_ssim_modes(ref, ref_fma))
    with open(os.path.join(HERE, "golden_ssim_modes.json"), "w") as f:
        json.dump(data, f, separators=(",", ":"))
    print("wrote", os.path.join(HERE, "golden_ssim_modes.json"))


def main():
    ref = oracle.Reference(ARCH)
    data = dict(generator="tests/golden/make_golden.py", reference_build=ARCH,
                pipeline=make_pipeline(ref), cps=make_cps(ref), gcd=make_gcd(ref), ssim_windows=make_ssim_windows(ref))
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(data, f, separators=(",", ":"))
    print("wrote", os.path.join(HERE, "golden.json"))


if __name__ == "__main__":
    if sys.argv[1:] == ["masked"]:
        main_masked()
    elif sys.argv[1:] == ["colour"]:
        main_colour()
    elif sys.argv[1:] == ["ssim_modes"]:
        main_ssim_modes()
    else:
        main()
