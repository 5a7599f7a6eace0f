"""Colour-space conversion before the metrics (qmiv_calc_set_color_space): YCbCr <-> RGB in the four
standards and BGR / GBR reordering, on 4:2:0 and 4:4:4 inputs, bit-exact against the compiled
reference's fixtures and the C restatement."""
import numpy as np
import pytest

import oracle
from golden_cases import case_frames, compare_result

pytestmark = pytest.mark.gpu


def _ids():
    import json, os
    with open(os.path.join(os.path.dirname(__file__), "golden", "golden_colour.json")) as f:
        g = json.load(f)["colour"]
    return [f"{c['width']}x{c['height']}_{c['bitdepth']}b_{c['chroma_format']}_cs{c['cs_in']}to{c['cs_metric']}" for c in g]


@pytest.mark.parametrize("idx", range(len(_ids())), ids=_ids())
def test_colour_golden(idx, golden_colour, qctx):
    import qmiv_b200
    case = golden_colour[idx]
    f0, f1 = case_frames(case)
    with qmiv_b200.Calc(qctx, case["width"], case["height"], case["bitdepth"], case["chroma_format"],
                        search_range=case["search_range"], erp=case["erp"]) as calc:
        calc.set_color_space(case["cs_in"], case["cs_metric"])
        got = calc.compute(f0, f1, case["mask"])
    assert compare_result(got, case["expected"], case["mask"]) == []


@pytest.mark.parametrize("shape", [(1920, 1080, 10, 420, oracle.CS_BT709, oracle.CS_RGB),
                                   (640, 360, 8, 444, oracle.CS_RGB, oracle.CS_BT2020),
                                   (352, 288, 10, 444, oracle.CS_GBR, oracle.CS_RGB)])
def test_colour_against_oracle_device_frames(shape, qctx, oracle_lib):
    import torch
    import qmiv_b200
    from qmiv_b200 import synth
    W, H, bd, cf, cs_in, cs_m = shape
    f0, f1 = synth.make_pair(W, H, bd, seed=W, chroma_format=cf)
    mask = qmiv_b200.IVPSNR | qmiv_b200.PSNR | qmiv_b200.IVSSIM | qmiv_b200.SSIM | qmiv_b200.WSPSNR
    exp = oracle_lib.compute_pair_cs(oracle.make_params(W, H, bd, cf), f0, f1, cs_in, cs_m, mask)
    d0 = tuple(torch.from_numpy(np.ascontiguousarray(p)).cuda() for p in f0)
    d1 = tuple(torch.from_numpy(np.ascontiguousarray(p)).cuda() for p in f1)
    with qmiv_b200.Calc(qctx, W, H, bd, cf) as calc:
        calc.set_color_space(cs_in, cs_m)
        got = calc.compute(d0, d1, mask)
        # back to no conversion: the plain results again
        calc.set_color_space(qmiv_b200.CS_YCBCR, qmiv_b200.CS_YCBCR)
        plain = calc.compute(d0, d1, mask)
    for k in ["gcd_r2t", "exact", "psnr", "wspsnr", "ivpsnr", "ivpsnr_r2t", "ivpsnr_t2r", "ssim", "ivssim"]:
        assert got[k] == exp[k], k
    assert plain == qmiv_b200.Calc(qctx, W, H, bd, cf).compute(d0, d1, mask)


def test_colour_refusals_and_invalid_pixels(qctx, oracle_lib):
    import qmiv_b200
    from qmiv_b200 import synth
    W, H, bd = 128, 64, 10
    f0, f1 = synth.make_pair(W, H, bd, seed=2, chroma_format=444)
    with qmiv_b200.Calc(qctx, W, H, bd, 444) as calc:
        with pytest.raises(qmiv_b200.QmivError) as ei:
            calc.set_color_space(qmiv_b200.CS_BT601, qmiv_b200.CS_BT709)
        assert ei.value.status == 2
        with pytest.raises(qmiv_b200.QmivError) as ei:
            calc.set_color_space(qmiv_b200.CS_YCBCR, qmiv_b200.CS_RGB)
        assert ei.value.status == 1
        calc.set_color_space(qmiv_b200.CS_RGB, qmiv_b200.CS_BT601)
        with pytest.raises(qmiv_b200.QmivError) as ei:
            calc.calc_global_color_diff(f0, f1)
        assert ei.value.status == 2
        bad = tuple(p.copy() for p in f1)
        bad[1][3, 4] = 1023 + 7
        with pytest.raises(qmiv_b200.QmivError) as ei:
            calc.compute(f0, bad, qmiv_b200.PSNR)
        assert ei.value.status == 5                           # checked before the conversion
    with qmiv_b200.Calc(qctx, W, H, bd, 444, invalid_pel_action=qmiv_b200.PEL_CNCL) as calc:
        calc.set_color_space(qmiv_b200.CS_RGB, qmiv_b200.CS_BT601)
        got = calc.compute(f0, bad, qmiv_b200.PSNR | qmiv_b200.IVPSNR)
    clipped = tuple(np.minimum(p, 1023) for p in bad)
    exp = oracle_lib.compute_pair_cs(oracle.make_params(W, H, bd, 444), f0, clipped, oracle.CS_RGB, oracle.CS_BT601,
                                     oracle.PSNR | oracle.IVPSNR)
    assert got["invalid_pel"] == [0, 1]
    for k in ["psnr", "ivpsnr", "gcd_r2t"]:
        assert got[k] == exp[k], k
