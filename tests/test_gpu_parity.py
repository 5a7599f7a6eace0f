"""Parity of the CUDA library (through its C ABI) with the reference: bit-exact on the golden
fixtures, and against the C restatement on seeded inputs up to the full 4096x2048 workload."""
import numpy as np
import pytest

import oracle
from golden_cases import case_frames, case_params, compare_result, sha256, unhex

pytestmark = pytest.mark.gpu


def _ids():
    import json, os
    with open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")) as f:
        g = json.load(f)
    return [f"{c['width']}x{c['height']}_{c['bitdepth']}b_{c['chroma_format']}_R{c['search_range']}"
            f"{'_erp' if c['erp'] else ''}{'_' + c['variant'] if c.get('variant') else ''}" for c in g["pipeline"]]


def _calc(qctx, case, **over):
    import qmiv_b200
    kw = case_params(case)
    kw.update(over)
    kw.pop("lon_range", None)
    return qmiv_b200.Calc(qctx, case["width"], case["height"], case["bitdepth"], case["chroma_format"], **kw)


def _device(frame):
    import torch
    return tuple(torch.from_numpy(np.ascontiguousarray(p)).cuda() for p in frame)


@pytest.mark.parametrize("idx", range(len(_ids())), ids=_ids())
def test_pipeline_golden_host_frames(idx, golden, qctx):
    case = golden["pipeline"][idx]
    f0, f1 = case_frames(case)
    with _calc(qctx, case) as calc:
        got = calc.compute(f0, f1, case["mask"])
        assert compare_result(got, case["expected"], case["mask"]) == []
        r2t, t2r = calc.cps_rows()
        assert r2t.astype(np.int64).tolist() == case["cps_rows_r2t"]
        assert t2r.astype(np.int64).tolist() == case["cps_rows_t2r"]
        s0, s1 = calc.gen_shft_comp_pics(f0, f1)
        assert sha256(s0) == case["expected"]["scp0_sha256"]
        assert sha256(s1) == case["expected"]["scp1_sha256"]


@pytest.mark.parametrize("idx", [0, 1, 4, 10], ids=[_ids()[i] for i in [0, 1, 4, 10]])
def test_pipeline_golden_device_frames(idx, golden, qctx):
    case = golden["pipeline"][idx]
    f0, f1 = case_frames(case)
    with _calc(qctx, case) as calc:
        got = calc.compute(_device(f0), _device(f1), case["mask"])
        assert compare_result(got, case["expected"], case["mask"]) == []


def test_cps_unit_fixtures(golden, cps_arrays, qctx):
    """test-xCorrespPixelShift.cpp style fixtures, explicit GCDs, 4:4:4 input (R2T = (Tst=Mod, Ref=Org))."""
    import qmiv_b200
    for case in golden["cps"]:
        org, mod = cps_arrays[case["key"] + "_org"], cps_arrays[case["key"] + "_mod"]
        W, H, bd = case["width"], case["height"], case["bitdepth"]
        with qmiv_b200.Calc(qctx, W, H, bd, 444, invalid_pel_action=qmiv_b200.PEL_SKIP) as calc:
            calc.set_gcd(case["gcd"])
            mod_f = tuple(mod[c].astype(np.uint8 if bd <= 8 else np.uint16) for c in range(3))
            org_f = tuple(org[c].astype(np.uint8 if bd <= 8 else np.uint16) for c in range(3))
            calc.compute(mod_f, org_f, qmiv_b200.IVPSNR)
            r2t, _ = calc.cps_rows()
            assert r2t.astype(np.int64).tolist() == case["rows_interleaved"], (case["key"], case["gcd"])


@pytest.mark.parametrize("bd", [8, 10, 12, 14])
def test_gcd_known_answers(bd, qctx):
    """libs/pmbb-ivqm/test/test-xGlobClrDiff.cpp:45-87: fills 0/1/Max and constant offsets, coef 1.0."""
    import qmiv_b200
    W, H = 128, 128
    maxv = (1 << bd) - 1
    dt = np.uint8 if bd <= 8 else np.uint16
    with qmiv_b200.Calc(qctx, W, H, bd, 444, unc=(1.0, 1.0, 1.0, 1.0)) as calc:
        zero = tuple(np.zeros((H, W), dt) for _ in range(3))
        for fill in (0, 1, maxv):
            mod = tuple(np.full((H, W), fill, dt) for _ in range(3))
            # qmiv_calc_gcd(In0, In1) = round(mean(In1 - In0)); the reference's CalcGlobalColorDiff(Mod, Ref)
            assert calc.calc_global_color_diff(zero, mod)[:3] == [fill] * 3
            assert calc.calc_global_color_diff(mod, zero)[:3] == [-fill] * 3
        rng = np.random.default_rng(bd)
        ref = tuple(rng.integers(0, maxv - 8, (H, W)).astype(dt) for _ in range(3))
        mod = tuple((ref[c].astype(np.int64) + (4, 3, 2)[c]).astype(dt) for c in range(3))
        assert calc.calc_global_color_diff(ref, mod)[:3] == [4, 3, 2]
        assert calc.calc_global_color_diff(mod, ref)[:3] == [-4, -3, -2]


def test_gcd_golden(golden, qctx):
    import qmiv_b200
    from detgen import det_pair
    for case in golden["gcd"]:
        f0, f1 = det_pair(case["width"], case["height"], case["bitdepth"], case["seed"], 444, offset=(5, -7, 1))
        with qmiv_b200.Calc(qctx, case["width"], case["height"], case["bitdepth"], 444, unc=tuple(case["coef"])) as calc:
            assert calc.calc_global_color_diff(f0, f1) == case["gcd_10"]
            assert calc.calc_global_color_diff(f1, f0) == case["gcd_01"]


def test_ssim_windows_golden(golden, qctx):
    import qmiv_b200
    for case in golden["ssim_windows"]:
        bd = case["bitdepth"]
        dt = np.uint8 if bd <= 8 else np.uint16
        t = np.array(case["tst"], dt)
        r = np.array(case["ref"], dt)
        with qmiv_b200.Calc(qctx, 8, 8, bd, 444) as calc:
            got = calc.calc_pic_ssim((t, t, t), (r, r, r))
            assert got == [float.fromhex(case["values"]["l1_std1"])] * 3


@pytest.mark.parametrize("shape", [(640, 360, 8, 420, 2, False), (416, 240, 10, 420, 4, True),
                                   (352, 288, 10, 422, 3, False), (258, 130, 8, 444, 1, True),
                                   (1280, 720, 10, 420, 2, True), (320, 240, 14, 420, 2, False),
                                   (200, 120, 13, 444, 3, True)])
def test_against_oracle_seeded(shape, qctx, oracle_lib):
    import qmiv_b200
    from qmiv_b200 import synth
    W, H, bd, cf, R, erp = shape
    f0, f1 = synth.make_pair(W, H, bd, seed=W * 7 + H, chroma_format=cf)
    p = oracle.make_params(W, H, bd, cf, search_range=R, erp=erp)
    exp = oracle_lib.compute_pair(p, f0, f1, oracle.ALL, want_scp=True)
    with qmiv_b200.Calc(qctx, W, H, bd, cf, search_range=R, erp=erp) as calc:
        got = calc.compute(f0, f1, qmiv_b200.ALL)
        for k in exp:
            if k.startswith("scp"):
                continue
            assert got[k][:3] == exp[k][:3] if isinstance(exp[k], list) else got[k] == exp[k], k
        s0, s1 = calc.gen_shft_comp_pics(f0, f1)
        assert np.array_equal(s0, exp["scp0"]) and np.array_equal(s1, exp["scp1"])


def test_ssim_family_rejected_above_14_bits(qctx):
    """The SSIM family's exact 32-bit sub-block moments need bit depth <= 14; deeper pictures are
    refused for those metrics and still served for the PSNR family."""
    import qmiv_b200
    from qmiv_b200 import synth
    f0, f1 = synth.make_pair(64, 48, 15, seed=3)
    with qmiv_b200.Calc(qctx, 64, 48, 15) as calc:
        with pytest.raises(qmiv_b200.QmivError) as ei:
            calc.compute(f0, f1, qmiv_b200.IVSSIM)
        assert "bit depth" in str(ei.value)
        assert calc.compute(f0, f1, qmiv_b200.IVPSNR | qmiv_b200.PSNR)["ivpsnr"] > 0


def test_full_size_erp_4096x2048_10bit(qctx, oracle_lib):
    """The headline workload shape, one pair, all metrics: bit-exact against the C restatement."""
    import qmiv_b200
    from qmiv_b200 import synth
    W, H = 4096, 2048
    f0, f1 = synth.make_pair(W, H, 10, seed=12345)
    mask = qmiv_b200.IVPSNR | qmiv_b200.WSPSNR | qmiv_b200.IVSSIM | qmiv_b200.PSNR
    p = oracle.make_params(W, H, 10, 420, erp=True)
    exp = oracle_lib.compute_pair(p, f0, f1, mask)
    with qmiv_b200.Calc(qctx, W, H, 10, 420, erp=True) as calc:
        got = calc.compute(f0, f1, mask)
    for k in ["gcd_r2t", "psnr", "psnr_pic", "wspsnr", "wspsnr_pic", "ivpsnr", "ivpsnr_r2t", "ivpsnr_t2r",
              "ivssim", "ivssim_r2t", "ivssim_t2r"]:
        assert got[k] == exp[k], k


def test_msssim_workload_2048_blurred(qctx, oracle_lib):
    """The MS-SSIM workload's shape: 2048x2048 10-bit 4:2:0 pairs with a seeded blur, 5 scales,
    MS-SSIM and IV-MS-SSIM through the plain and the batched form, bit-exact against the C restatement
    and, where it is built here, the compiled reference library."""
    import qmiv_b200
    from qmiv_b200 import synth
    W = H = 2048
    pairs = [synth.make_pair(W, H, 10, seed=2000 + i, blur_sigma=s) for i, s in enumerate((0.7, 1.8))]
    mask = qmiv_b200.MSSSIM | qmiv_b200.IVMSSSIM
    keys = ["gcd_r2t", "msssim", "msssim_pic", "ivmsssim", "ivmsssim_r2t", "ivmsssim_t2r"]
    p = oracle.make_params(W, H, 10, 420)
    exp = [oracle_lib.compute_pair(p, a, b, mask) for a, b in pairs]
    with qmiv_b200.Calc(qctx, W, H, 10, 420) as calc:
        plain = [calc.compute(a, b, mask) for a, b in pairs]
    descs = [dict(frame0=a, frame1=b, width=W, height=H, bitdepth=10, search_range=2, metrics=mask) for a, b in pairs]
    with qmiv_b200.Batch(qctx, 2, 2 * W * H, graph=True, autotune=True) as batch:
        batched = batch.compute(descs)
    for k in keys:
        for i in range(len(pairs)):
            assert plain[i][k] == exp[i][k], (i, k)
            assert batched[i][k] == exp[i][k], (i, k)
    if oracle.reference_available():
        ref = oracle.Reference().compute_pair(p, *pairs[0], mask)
        for k in keys:
            assert plain[0][k] == ref[k], k


def test_full_size_properties(qctx):
    """Size-independent properties at 4096x2048: identical frames give SSE 0, GCD 0, SSIM 1, and the
    result does not depend on the order the pairs are computed in."""
    import qmiv_b200
    from qmiv_b200 import synth
    W, H = 4096, 2048
    f0, f1 = synth.make_pair(W, H, 10, seed=7)
    with qmiv_b200.Calc(qctx, W, H, 10, 420, erp=True) as calc:
        same = calc.compute(f0, f0, qmiv_b200.ALL)
        assert same["gcd_r2t"][:3] == [0, 0, 0]
        assert same["cps_sse_r2t"][:3] == [0, 0, 0] and same["cps_sse_t2r"][:3] == [0, 0, 0]
        assert same["ssim"][:3] == [1.0, 1.0, 1.0] and same["ivssim"] == 1.0
        assert same["exact"][:3] == [1, 1, 1]
        a = calc.compute(f0, f1, qmiv_b200.ALL)
        b = calc.compute(f1, f0, qmiv_b200.ALL)
        a2 = calc.compute(f0, f1, qmiv_b200.ALL)
        assert a == a2
        # swapping the inputs negates the GCD and swaps the two search directions
        assert b["gcd_r2t"][:3] == [-x for x in a["gcd_r2t"][:3]]
        assert b["ivpsnr_r2t"] == a["ivpsnr_t2r"] and b["ivpsnr_t2r"] == a["ivpsnr_r2t"]
        assert b["ivssim_r2t"] == a["ivssim_t2r"] and b["ivssim_t2r"] == a["ivssim_r2t"]
        assert a["psnr"] == b["psnr"] and a["ssim"] == b["ssim"]


def test_cps_tma_and_plain_tile_loads_agree(qctx, oracle_lib):
    """Device planes with 16-byte row pitches reach the search through TMA tile loads, planes with an
    odd pitch through plain loads; host frames are staged with aligned pitches. All equal the oracle."""
    import torch
    import qmiv_b200
    from qmiv_b200 import synth
    W, H, bd = 640, 360, 10
    f0, f1 = synth.make_pair(W, H, bd, seed=99)
    mask = qmiv_b200.IVPSNR | qmiv_b200.IVSSIM | qmiv_b200.PSNR | qmiv_b200.WSPSNR
    exp = oracle_lib.compute_pair(oracle.make_params(W, H, bd, 420, erp=True), f0, f1, mask)

    def strided(frame, extra):
        views = []
        for pl in frame:
            h, w = pl.shape
            big = np.zeros((h, w + extra), dtype=pl.dtype)
            big[:, :w] = pl
            views.append(torch.from_numpy(big).cuda()[:, :w])
        return tuple(views)

    keys = ["gcd_r2t", "psnr", "wspsnr", "ivpsnr", "ivpsnr_r2t", "ivpsnr_t2r", "ivssim", "ivssim_r2t", "ivssim_t2r"]
    with qmiv_b200.Calc(qctx, W, H, bd, 420, erp=True) as calc:
        for a, b in [(f0, f1), (_device(f0), _device(f1)), (strided(f0, 3), strided(f1, 3)),
                     (strided(f0, 8), strided(f1, 5))]:
            got = calc.compute(a, b, mask)
            for k in keys:
                assert got[k] == exp[k], k
