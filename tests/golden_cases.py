"""Helpers shared by the tests: rebuild the golden cases' frames and compare result dicts."""
import hashlib

import numpy as np

from detgen import det_pair

RESULT_FLOAT_KEYS = ["psnr", "psnr_pic", "wspsnr", "wspsnr_pic", "ivpsnr", "ivpsnr_r2t", "ivpsnr_t2r", "ssim",
                     "ssim_pic", "msssim", "msssim_pic", "ivssim", "ivssim_r2t", "ivssim_t2r", "ivmsssim",
                     "ivmsssim_r2t", "ivmsssim_t2r"]
METRIC_OF_KEY = {"psnr": 1, "wspsnr": 2, "ivpsnr": 4, "ssim": 8, "msssim": 16, "ivssim": 32, "ivmsssim": 64}


def case_frames(case):
    f0, f1 = det_pair(case["width"], case["height"], case["bitdepth"], case["seed"], case["chroma_format"])
    if case.get("variant") == "exact_chroma":
        f1 = (f1[0], f0[1].copy(), f0[2].copy())
    elif case.get("variant") == "identical":
        f1 = tuple(p.copy() for p in f0)
    return f0, f1


def case_params(case):
    p = dict(case["params"])
    for k in ("cws", "cwa", "unc"):
        if k in p:
            p[k] = tuple(p[k])
    return p


def unhex(v):
    if isinstance(v, list):
        return [float.fromhex(x) if isinstance(x, str) else x for x in v]
    return float.fromhex(v) if isinstance(v, str) else v


def metric_enabled(key, mask):
    base = key.split("_")[0]
    return bool(METRIC_OF_KEY.get(base, 0) & mask)


def compare_result(got, expected, mask, ignore=()):
    """Bit-exact comparison of a result dict against a golden 'expected' block. Returns mismatches."""
    bad = []
    for k in ["gcd_r2t", "exact"]:
        if k in ignore:
            continue
        if list(got[k][:3]) != list(expected[k][:3]):
            bad.append((k, got[k], expected[k]))
    for k in RESULT_FLOAT_KEYS:
        if k in ignore or not metric_enabled(k, mask):
            continue
        e = unhex(expected[k])
        g = got[k]
        if isinstance(e, list):
            if [float(x) for x in g[:3]] != [float(x) for x in e[:3]]:
                bad.append((k, g[:3], e[:3]))
        elif float(g) != float(e):
            bad.append((k, g, e))
    return bad


SSIM_KEYS = ["ssim", "ssim_pic", "msssim", "msssim_pic", "ivssim", "ivssim_r2t", "ivssim_t2r", "ivmsssim", "ivmsssim_r2t",
             "ivmsssim_t2r"]


def ssim_mode_ids():
    import json, os
    with open(os.path.join(os.path.dirname(__file__), "golden", "golden_ssim_modes.json")) as f:
        g = json.load(f)["ssim_modes"]
    names = {0: "RglrFlt", 1: "RglrInt", 2: "RglrAvg", 3: "BlckInt", 4: "BlckAvg"}
    return [f"{names[c['ssim_mode']]}_b{c['ssim_border']}_w{c['ssim_window']}_s{c['ssim_stride']}_{c['width']}x{c['height']}_"
            f"{c['bitdepth']}b_{c['chroma_format']}{'_erp' if c['erp'] else ''}" for c in g]


def max_ssim_deviation(got, expected, mask):
    """Largest absolute difference over the SSIM-family values of a result dict and a golden block."""
    dev = 0.0
    for k in SSIM_KEYS:
        if not metric_enabled(k, mask) or k not in expected:
            continue
        e, g = unhex(expected[k]), got[k]
        es, gs = (e[:3], g[:3]) if isinstance(e, list) else ([e], [g])
        dev = max(dev, max(abs(float(a) - float(b)) for a, b in zip(gs, es)))
    return dev


def sha256(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def masked_case_inputs(case):
    """Frames and mask of a golden mask-mode case (detgen)."""
    from detgen import det_mask
    f0, f1 = det_pair(case["width"], case["height"], case["bitdepth"], case["seed"], case["chroma_format"])
    m = det_mask(case["width"], case["height"], case["mask_bitdepth"], case["seed"], case["mask_kind"])
    return f0, f1, m


MASKED_METRICS = 1 | 2 | 4


def compare_masked(got, nnm, expected):
    """Bit-exact comparison of a mask-mode result against its golden block. Returns mismatches."""
    bad = compare_result(got, expected, MASKED_METRICS)
    if nnm != expected["num_non_masked"]:
        bad.append(("num_non_masked", nnm, expected["num_non_masked"]))
    return bad
