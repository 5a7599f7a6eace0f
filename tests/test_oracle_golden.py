"""Pins the C restatement (oracle/qmiv_oracle.c) to the golden fixtures produced by the compiled QMIV
reference (tests/golden/make_golden.py). Everything here runs on the CPU."""
import numpy as np
import pytest

import oracle
from golden_cases import ssim_mode_ids, max_ssim_deviation, case_frames, case_params, compare_result, sha256, unhex


def _pipeline_ids(golden_json=None):
    import json, os
    with open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")) as f:
        g = json.load(f)
    return [f"{c['width']}x{c['height']}_{c['bitdepth']}b_{c['chroma_format']}_R{c['search_range']}"
            f"{'_erp' if c['erp'] else ''}{'_' + c['variant'] if c.get('variant') else ''}" for c in g["pipeline"]]


@pytest.mark.parametrize("idx", range(len(_pipeline_ids())), ids=_pipeline_ids())
def test_pipeline_matches_reference(idx, golden, oracle_lib):
    case = golden["pipeline"][idx]
    f0, f1 = case_frames(case)
    p = oracle.make_params(case["width"], case["height"], case["bitdepth"], case["chroma_format"], **case_params(case))
    got = oracle_lib.compute_pair(p, f0, f1, case["mask"], want_scp=True)
    exp = case["expected"]
    assert compare_result(got, exp, case["mask"]) == []
    assert sha256(got["scp0"]) == exp["scp0_sha256"]
    assert sha256(got["scp1"]) == exp["scp1_sha256"]


@pytest.mark.parametrize("idx", range(len(_pipeline_ids())), ids=_pipeline_ids())
def test_cps_rows_match_reference(idx, golden, oracle_lib):
    case = golden["pipeline"][idx]
    f0, f1 = case_frames(case)
    cf, bd, R = case["chroma_format"], case["bitdepth"], case["search_range"]
    t0 = oracle_lib.unpack444(f0, case["width"], case["height"], bd, cf)
    t1 = oracle_lib.unpack444(f1, case["width"], case["height"], bd, cf)
    g = unhex(case["expected"]["gcd_r2t"])
    cws = tuple(case["params"].get("cws", (4, 1, 1, 0)))
    r2t, _ = oracle_lib.cps(t0, t1, bd, g, R, cws, want_scp=False)
    t2r, _ = oracle_lib.cps(t1, t0, bd, [-x for x in g], R, cws, want_scp=False)
    assert r2t.astype(np.int64).tolist() == case["cps_rows_r2t"]
    assert t2r.astype(np.int64).tolist() == case["cps_rows_t2r"]


def test_cps_unit_fixtures(golden, cps_arrays, oracle_lib):
    """libs/pmbb-ivqm/test/test-xCorrespPixelShift.cpp style: Perlin originals, block noise, 4 GCDs."""
    for case in golden["cps"]:
        org, mod = cps_arrays[case["key"] + "_org"], cps_arrays[case["key"] + "_mod"]
        rows, scp = oracle_lib.cps(mod, org, case["bitdepth"], case["gcd"], 2, (4, 1, 1, 0), want_scp=True)
        assert rows.astype(np.int64).tolist() == case["rows_interleaved"]
        std = oracle_lib.cps_rows_std(mod, org, case["gcd"], 2, (4, 1, 1, 0))
        assert std.astype(np.int64).tolist() == case["rows_planar"]
        # SSD(Tst, SCP) == CPS SSE when no clipping happens (test-xCorrespPixelShift.cpp:155-179)
        g = np.array(case["gcd"][:3], np.int64)[:, None, None]
        d = mod.astype(np.int64) + g - (scp.astype(np.int64) + g)
        maxv = (1 << case["bitdepth"]) - 1
        unclipped = (scp.astype(np.int64) > 0) & (scp.astype(np.int64) < maxv)
        if unclipped.all():
            assert (d ** 2).reshape(3, -1).sum(axis=1).tolist() == rows.sum(axis=0).tolist()


def test_gcd_matches_reference(golden, oracle_lib):
    from detgen import det_pair, to444
    for case in golden["gcd"]:
        f0, f1 = det_pair(case["width"], case["height"], case["bitdepth"], case["seed"], 444, offset=(5, -7, 1))
        t0, t1 = to444(f0, 444), to444(f1, 444)
        assert oracle_lib.gcd(t1, t0, case["bitdepth"], case["coef"]) == case["gcd_10"]
        assert oracle_lib.gcd(t0, t1, case["bitdepth"], case["coef"]) == case["gcd_01"]


@pytest.mark.parametrize("bd", [8, 10, 12, 14])
@pytest.mark.parametrize("size", [(128, 128), (256, 128), (128, 256), (256, 256)])
def test_gcd_known_answers(bd, size, oracle_lib):
    """libs/pmbb-ivqm/test/test-xGlobClrDiff.cpp:45-87 with coefficient 1.0."""
    W, H = size
    maxv = (1 << bd) - 1
    one = (1.0, 1.0, 1.0, 1.0)
    ref = np.zeros((3, H, W), np.uint16)
    for fill, expect in [(0, 0), (1, 1), (maxv, maxv)]:
        mod = np.full((3, H, W), fill, np.uint16)
        assert oracle_lib.gcd(mod, ref, bd, one)[:3] == [expect] * 3
        assert oracle_lib.gcd(ref, mod, bd, one)[:3] == [-expect] * 3
    rng = np.random.default_rng(bd * 7 + W)
    ref = rng.integers(0, maxv - 8, (3, H, W)).astype(np.uint16)
    mod = ref + np.array([4, 3, 2], np.uint16)[:, None, None]
    assert oracle_lib.gcd(mod, ref, bd, one)[:3] == [4, 3, 2]
    assert oracle_lib.gcd(ref, mod, bd, one)[:3] == [-4, -3, -2]
    assert oracle_lib.gcd(ref, ref, bd, one)[:3] == [0, 0, 0]


def test_ssim_windows_match_reference(golden, oracle_lib):
    for case in golden["ssim_windows"]:
        t = np.array(case["tst"], np.uint16)
        r = np.array(case["ref"], np.uint16)
        vals = case["values"]
        # the dispatched (SIMD) and portable reference windows agree (test-xStructSim.cpp:169-170)
        assert vals["l0_std0"] == vals["l0_std1"] and vals["l1_std0"] == vals["l1_std1"]
        for calc_l in (0, 1):
            got = oracle_lib.ssim_pic(np.stack([t] * 3), np.stack([r] * 3), case["bitdepth"], calc_l)
            assert got == [float.fromhex(vals[f"l{calc_l}_std1"])] * 3


def test_window_counts():
    """xSSIM::xCalcNumBlocks against brute force, as libs/pmbb-ivqm/test/test-xSSIM.cpp:29-51."""
    for length in range(100, 4097, 27):
        cnt = len(range(0, length - 8 + 1, 4))
        assert cnt == (length - 8) // 4 + 1


def test_num_scales(oracle_lib):
    assert oracle_lib.num_scales(2048, 2048) == 5
    assert oracle_lib.num_scales(256, 128) == 3
    assert oracle_lib.num_scales(31, 500) == 0
    assert oracle_lib.num_scales(4096, 2048) == 5


def _masked_ids():
    import json, os
    with open(os.path.join(os.path.dirname(__file__), "golden", "golden_masked.json")) as f:
        g = json.load(f)["masked"]
    return [f"{c['width']}x{c['height']}_{c['bitdepth']}b_{c['chroma_format']}_R{c['search_range']}"
            f"{'_erp' if c['erp'] else ''}_m{c['mask_bitdepth']}{c['mask_kind']}" for c in g]


@pytest.mark.parametrize("idx", range(len(_masked_ids())), ids=_masked_ids())
def test_masked_pipeline_matches_reference(idx, golden_masked, oracle_lib):
    """Mask mode (GCD-M, CPS-M, PSNR-M, WS-PSNR-M, IV-PSNR-M) of the restatement against the compiled
    reference's outputs, bit for bit, including the reference's bit-depth choice in PSNR-M and its
    direction labels in IV-PSNR-M."""
    import oracle
    from golden_cases import compare_masked, masked_case_inputs
    case = golden_masked[idx]
    f0, f1, m = masked_case_inputs(case)
    p = oracle.make_params(case["width"], case["height"], case["bitdepth"], case["chroma_format"],
                           search_range=case["search_range"], erp=case["erp"])
    got, nnm = oracle_lib.compute_pair_masked(p, f0, f1, m, case["mask_bitdepth"])
    assert compare_masked(got, nnm, case["expected"]) == []


def test_masked_refuses_ssim(oracle_lib):
    import numpy as np
    import oracle
    from detgen import det_mask, det_pair
    f0, f1 = det_pair(32, 32, 8, 1, 420)
    p = oracle.make_params(32, 32, 8, 420)
    with pytest.raises(RuntimeError):
        oracle_lib.compute_pair_masked(p, f0, f1, det_mask(32, 32, 8, 1), 8, oracle.IVSSIM)


def _colour_ids():
    import json, os
    with open(os.path.join(os.path.dirname(__file__), "golden", "golden_colour.json")) as f:
        g = json.load(f)["colour"]
    return [f"{c['width']}x{c['height']}_{c['bitdepth']}b_{c['chroma_format']}_cs{c['cs_in']}to{c['cs_metric']}" for c in g]


@pytest.mark.parametrize("idx", range(len(_colour_ids())), ids=_colour_ids())
def test_colour_pipeline_matches_reference(idx, golden_colour, oracle_lib):
    """Colour-space conversion before the metrics (YCbCr <-> RGB in four standards, BGR/GBR reordering)
    of the restatement against the compiled reference, bit for bit."""
    import oracle
    case = golden_colour[idx]
    f0, f1 = case_frames(case)
    p = oracle.make_params(case["width"], case["height"], case["bitdepth"], case["chroma_format"],
                           search_range=case["search_range"], erp=case["erp"])
    got = oracle_lib.compute_pair_cs(p, f0, f1, case["cs_in"], case["cs_metric"], case["mask"])
    assert compare_result(got, case["expected"], case["mask"]) == []


def test_colour_refused_combinations(oracle_lib):
    import oracle
    from detgen import det_pair
    f0, f1 = det_pair(32, 32, 8, 1, 444)
    p = oracle.make_params(32, 32, 8, 444)
    for cs_in, cs_metric in [(oracle.CS_BT601, oracle.CS_BT709), (oracle.CS_YCBCR, oracle.CS_RGB), (oracle.CS_RGB, oracle.CS_YCBCR)]:
        with pytest.raises(RuntimeError):
            oracle_lib.compute_pair_cs(p, f0, f1, cs_in, cs_metric)


@pytest.mark.parametrize("idx", range(len(ssim_mode_ids())), ids=ssim_mode_ids())
def test_ssim_modes_match_reference(idx, golden_ssim_modes, oracle_lib):
    """Every metric under the app's structural similarity options (regular 11x11 Gaussian float /
    Gaussian integer / averaged windows with the five border extensions, block Gaussian integer 8/16 and
    averaged 8/16/32 windows, strides 1..window) of the restatement against the compiled reference's
    portable-arithmetic build, bit for bit, and within 1e-14 of its FMA-contracted build."""
    import oracle
    case = golden_ssim_modes[idx]
    f0, f1 = case_frames(case)
    p = oracle.make_params(case["width"], case["height"], case["bitdepth"], case["chroma_format"],
                           search_range=case["search_range"], erp=case["erp"])
    got = oracle_lib.compute_pair_ssim(p, f0, f1, case["ssim_mode"], case["ssim_border"], case["ssim_window"],
                                       case["ssim_stride"], case["mask"])
    assert compare_result(got, case["expected"], case["mask"]) == []
    assert max_ssim_deviation(got, case["expected_fma_build"], case["mask"]) < 1e-14


def test_ssim_mode_refusals(oracle_lib):
    """Option sets the reference cannot evaluate: regular windows other than 11, Gaussian 32x32 blocks
    (CalcBlckInt returns NaN), stride 0 or above the window, the averaged 11x11 window over the constant
    65535 margin (32-bit overflow), pictures smaller than the window."""
    import oracle
    from detgen import det_pair
    f0, f1 = det_pair(48, 48, 8, 1, 444)
    p = oracle.make_params(48, 48, 8, 444)
    for cfg in [(0, 0, 8, 1), (3, 0, 32, 4), (4, 0, 8, 0), (4, 0, 8, 9), (2, 4, 11, 1), (4, 0, 64, 4), (7, 0, 8, 4),
                (0, 6, 11, 1)]:
        with pytest.raises(RuntimeError):
            oracle_lib.compute_pair_ssim(p, f0, f1, *cfg, mask=oracle.SSIM)


def test_oracle_masked_ssd_wraps_like_the_reference(oracle_lib):
    """The reference forms a masked squared difference as an int32 product that wraps (two's
    complement) before widening to 64 bits (xDistortionSTD.cpp:62). The C restatement does the same in
    defined arithmetic: one luma difference of 50000 (its square above 2^31) gives the SSD of the wrapped
    product read as uint64, checked through PSNR-M = K - 10 log10(SSD) with K taken from a difference
    of 46340, whose square does not wrap."""
    import math
    import numpy as np
    W, H = 16, 8
    p = oracle.make_params(W, H, 10, 420, search_range=1, erp=False)
    m = np.ones((H, W), np.uint8)

    def psnr_y(d):
        f0 = tuple(np.zeros((h, w), np.uint16) for h, w in ((H, W), (H // 2, W // 2), (H // 2, W // 2)))
        f1 = tuple(np.array(pl, copy=True) for pl in f0)
        f1[0][2, 3] = d
        r, _ = oracle_lib.compute_pair_masked(p, f0, f1, m, 8)
        return r["psnr"][0]

    k = psnr_y(46340) + 10.0 * math.log10(46340 * 46340)
    sq = (50000 * 50000) & 0xffffffff                          # the int32 product's bits
    wrapped = (sq - (1 << 32)) % (1 << 64) if sq >= (1 << 31) else sq   # sign-extended, read as uint64
    assert math.isclose(psnr_y(50000), k - 10.0 * math.log10(wrapped), rel_tol=1e-12, abs_tol=1e-9)
