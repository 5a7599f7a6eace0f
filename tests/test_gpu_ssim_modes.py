"""Structural similarity options (qmiv_params.ssim_mode / ssim_border / ssim_window / ssim_stride): regular
11x11 Gaussian float, Gaussian integer and averaged windows with every border extension, block Gaussian
integer and averaged windows of every size and stride, through SSIM, MS-SSIM, IV-SSIM and IV-MS-SSIM,
bit-exact against the compiled reference's fixtures and the C restatement."""
import numpy as np
import pytest

import oracle
from golden_cases import case_frames, compare_result, max_ssim_deviation, ssim_mode_ids

pytestmark = pytest.mark.gpu


def _calc(qctx, case, **kw):
    import qmiv_b200
    return qmiv_b200.Calc(qctx, case["width"], case["height"], case["bitdepth"], case["chroma_format"],
                          search_range=case["search_range"], erp=case["erp"], ssim_mode=case["ssim_mode"],
                          ssim_border=case["ssim_border"], ssim_window=case["ssim_window"],
                          ssim_stride=case["ssim_stride"], **kw)


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("idx", range(len(ssim_mode_ids())), ids=ssim_mode_ids())
def test_ssim_modes_golden(idx, golden_ssim_modes, qctx):
    case = golden_ssim_modes[idx]
    f0, f1 = case_frames(case)
    with _calc(qctx, case) as calc:
        got = calc.compute(f0, f1, case["mask"])
    assert compare_result(got, case["expected"], case["mask"]) == []
    # the reference's FMA-contracted build moves only the last bits
    assert max_ssim_deviation(got, case["expected_fma_build"], case["mask"]) < 1e-14


@pytest.mark.parametrize("idx", [0, 3, 8, 15, 22], ids=[ssim_mode_ids()[i] for i in [0, 3, 8, 15, 22]])
def test_ssim_modes_golden_device_frames(idx, golden_ssim_modes, qctx):
    case = golden_ssim_modes[idx]
    f0, f1 = case_frames(case)
    with _calc(qctx, case) as calc:
        got = calc.compute(tuple(_dev(p) for p in f0), tuple(_dev(p) for p in f1), case["mask"])
    assert compare_result(got, case["expected"], case["mask"]) == []


@pytest.mark.parametrize("shape", [
    # (W, H, bitdepth, chroma, R, erp, mode, border, window, stride, metrics)
    (640, 360, 10, 420, 2, True, 0, 0, 11, 1, oracle.ALL),                       # the paper's setting
    (1920, 1080, 8, 420, 2, False, 0, 0, 11, 4, oracle.SSIM | oracle.MSSSIM),
    (352, 288, 10, 422, 3, True, 1, 2, 11, 2, oracle.SSIM | oracle.IVSSIM),
    (500, 260, 12, 444, 2, True, 2, 3, 11, 1, oracle.SSIM | oracle.IVSSIM),
    (720, 480, 10, 420, 2, False, 3, 0, 16, 3, oracle.SSIM | oracle.IVMSSSIM),
    (1280, 720, 10, 420, 2, True, 4, 0, 32, 4, oracle.SSIM | oracle.IVSSIM | oracle.MSSSIM),
    (300, 200, 14, 444, 2, False, 0, 4, 11, 11, oracle.SSIM | oracle.IVSSIM),
    (256, 256, 8, 420, 1, True, 4, 0, 8, 1, oracle.ALL),
    # averaged windows at strides 1, 2, 4 take the box-sum kernel: 14-bit samples (the largest sums),
    # partial tiles at odd sizes, margins, MS-SSIM scales
    (320, 180, 14, 444, 2, False, 4, 0, 32, 1, oracle.SSIM | oracle.IVSSIM),
    (510, 254, 10, 420, 2, True, 4, 0, 16, 2, oracle.SSIM | oracle.IVSSIM),
    (333, 111, 12, 444, 2, False, 2, 1, 11, 4, oracle.SSIM | oracle.MSSSIM),
    (300, 170, 14, 420, 2, True, 2, 5, 11, 2, oracle.SSIM | oracle.IVSSIM),
])
def test_ssim_modes_against_oracle_seeded(shape, qctx, oracle_lib):
    """Seeded synthetic frames (the bench's generator) at sizes beyond the fixtures."""
    import qmiv_b200
    from qmiv_b200 import synth
    W, H, bd, cf, R, erp, mode, brd, win, st, mask = shape
    f0, f1 = synth.make_pair(W, H, bd, seed=W * 7 + H, chroma_format=cf)
    p = oracle.make_params(W, H, bd, cf, search_range=R, erp=erp)
    exp = oracle_lib.compute_pair_ssim(p, f0, f1, mode, brd, win, st, mask)
    with qmiv_b200.Calc(qctx, W, H, bd, cf, search_range=R, erp=erp, ssim_mode=mode, ssim_border=brd, ssim_window=win,
                        ssim_stride=st) as calc:
        got = calc.compute(f0, f1, mask)
    exp_enc = {k: ([float(x).hex() for x in v] if isinstance(v, list) and v and isinstance(v[0], float)
                   else (float(v).hex() if isinstance(v, float) else v)) for k, v in exp.items()}
    assert compare_result(got, exp_enc, mask) == []


@pytest.mark.parametrize("mode,border,window,stride", [(0, 0, 11, 1), (1, 3, 11, 4), (2, 1, 11, 2), (3, 0, 16, 4),
                                                       (4, 0, 32, 8)])
def test_ssim_modes_identical_full_size(mode, border, window, stride, qctx):
    """4096x2048 10-bit 4:2:0 (the IV-PSNR benchmark picture): a picture against itself gives SSIM and
    MS-SSIM of exactly 1 under every option (each window's numerators equal its denominators, and the
    compensated sums count the windows exactly); the ERP-weighted IV-SSIM divides a weighted sum by the
    weight mean times the window count, which rounds to within a few ulp of 1."""
    import qmiv_b200
    from qmiv_b200 import synth
    W, H = 4096, 2048
    f0, _ = synth.make_pair(W, H, 10, seed=11)
    f0d = tuple(_dev(p) for p in f0)
    with qmiv_b200.Calc(qctx, W, H, 10, 420, erp=True, ssim_mode=mode, ssim_border=border, ssim_window=window,
                        ssim_stride=stride) as calc:
        got = calc.compute(f0d, f0d, qmiv_b200.SSIM | qmiv_b200.IVSSIM | qmiv_b200.MSSSIM)
    assert list(got["ssim"][:3]) == [1.0, 1.0, 1.0]
    assert got["msssim_pic"] == 1.0
    assert abs(got["ivssim"] - 1.0) < 1e-15


def test_ssim_mode_refusals(qctx):
    import qmiv_b200
    bad = [dict(ssim_mode=0, ssim_window=8), dict(ssim_mode=3, ssim_window=32), dict(ssim_mode=4, ssim_window=8, ssim_stride=0),
           dict(ssim_mode=4, ssim_window=16, ssim_stride=17), dict(ssim_mode=2, ssim_border=4), dict(ssim_mode=4, ssim_window=12),
           dict(ssim_mode=5), dict(ssim_mode=0, ssim_border=6)]
    for kw in bad:
        with pytest.raises(qmiv_b200.QmivError):
            qmiv_b200.Calc(qctx, 64, 64, 10, 420, **kw)
    # a picture smaller than the window
    with qmiv_b200.Calc(qctx, 40, 24, 8, 420, ssim_mode=4, ssim_window=32) as calc:
        from qmiv_b200 import synth
        f0, f1 = synth.make_pair(40, 24, 8, seed=1)
        with pytest.raises(qmiv_b200.QmivError):
            calc.compute(f0, f1, qmiv_b200.SSIM)
        got = calc.compute(f0, f1, qmiv_b200.PSNR)   # the calc still works for the other metrics
        assert got["psnr_pic"] > 0
    # above 14 bits: plain SSIM under the regular Gaussian windows only
    f0, f1 = synth.make_pair(64, 48, 16, seed=2, chroma_format=444)
    with qmiv_b200.Calc(qctx, 64, 48, 16, 444, ssim_mode=0, ssim_stride=1) as calc:
        assert 0.0 < calc.compute(f0, f1, qmiv_b200.SSIM)["ssim_pic"] <= 1.0
        for m in (qmiv_b200.MSSSIM, qmiv_b200.IVSSIM, qmiv_b200.IVMSSSIM):
            with pytest.raises(qmiv_b200.QmivError):
                calc.compute(f0, f1, m)
    with qmiv_b200.Calc(qctx, 64, 48, 15, 420, ssim_mode=2) as calc:
        with pytest.raises(qmiv_b200.QmivError):
            calc.compute(*synth.make_pair(64, 48, 15, seed=3), qmiv_b200.SSIM)


@pytest.mark.parametrize("mode,border,window,stride", [(0, 0, 11, 1), (1, 2, 11, 4), (3, 0, 16, 4)])
def test_batched_and_serving_forms_take_ssim_options(mode, border, window, stride, qctx):
    """The batched form (synchronous and submit / wait) and the serving loop give, under other
    structural similarity options, the same results as the plain form: the SSIM metrics of such pairs
    are computed pair by pair after the batch, the others in the batch."""
    import qmiv_b200
    from qmiv_b200 import synth
    opts = dict(ssim_mode=mode, ssim_border=border, ssim_window=window, ssim_stride=stride, erp=True)
    shapes = [(128, 64, 10, 420, 2), (96, 96, 8, 444, 3), (160, 96, 10, 422, 2)]
    frames = [synth.make_pair(W, H, bd, seed=W + bd, chroma_format=cf) for (W, H, bd, cf, R) in shapes]
    masks = [qmiv_b200.ALL, qmiv_b200.SSIM | qmiv_b200.IVSSIM, qmiv_b200.PSNR | qmiv_b200.IVPSNR | qmiv_b200.MSSSIM]
    plain = []
    for (W, H, bd, cf, R), (f0, f1), m in zip(shapes, frames, masks):
        with qmiv_b200.Calc(qctx, W, H, bd, cf, search_range=R, **opts) as calc:
            plain.append(calc.compute(f0, f1, m))
    descs = [dict(frame0=f0, frame1=f1, width=W, height=H, bitdepth=bd, chroma_format=cf, search_range=R, metrics=m)
             for (W, H, bd, cf, R), (f0, f1), m in zip(shapes, frames, masks)]
    px = sum(W * H for (W, H, _, _, _) in shapes)
    with qmiv_b200.Batch(qctx, max_pairs=len(descs), max_pixels=px, **opts) as b:
        assert b.compute(descs) == plain
        t0, t1 = b.submit(descs), b.submit(descs)
        assert b.wait(t0) == plain and b.wait(t1) == plain
    with qmiv_b200.Server(qctx, max_batch_pairs=4, max_batch_pixels=px, **opts) as srv:
        tickets = [srv.submit([fr], W, H, bd, cf, search_range=R, metrics=m)
                   for (W, H, bd, cf, R), fr, m in zip(shapes, frames, masks)]
        got = [srv.wait(t)[0][0] for t in tickets]
    assert got == plain
