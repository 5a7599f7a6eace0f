"""Behaviour of the C ABI around the metric path: error statuses, invalid pixels, the HBM budget,
asynchronous submission, the batched form against the plain form."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _pair(W=256, H=128, bd=10, seed=3, cf=420):
    from qmiv_b200 import synth
    return synth.make_pair(W, H, bd, seed=seed, chroma_format=cf)


def test_invalid_pixel_stop_and_conceal(qctx, oracle_lib):
    """InvalidPelActn (apps/QMIV/src/xAppQMIV.cpp:834-852): STOP fails, CNCL clips to the bit depth."""
    import qmiv_b200
    f0, f1 = _pair()
    bad = tuple(p.copy() for p in f1)
    bad[0][5, 7] = 1023 + 40
    bad[2][3, 3] = 2000
    with qmiv_b200.Calc(qctx, 256, 128, 10) as calc:
        with pytest.raises(qmiv_b200.QmivError) as ei:
            calc.compute(f0, bad, qmiv_b200.ALL)
        assert ei.value.status == 5  # QMIV_ERR_INVALID_PIXEL
    with qmiv_b200.Calc(qctx, 256, 128, 10, invalid_pel_action=qmiv_b200.PEL_CNCL) as calc:
        got = calc.compute(f0, bad, qmiv_b200.ALL)
        assert got["invalid_pel"] == [0, 1]
    clipped = tuple(np.minimum(p, 1023) for p in bad)
    exp = oracle_lib.compute_pair(oracle.make_params(256, 128, 10, 420), f0, clipped, oracle.ALL)
    for k in ["gcd_r2t", "psnr", "ivpsnr", "ivssim", "ssim", "msssim", "ivmsssim"]:
        assert got[k] == exp[k], k


def test_invalid_pixel_skip_uses_exact_integer_search(qctx, oracle_lib):
    """SKIP keeps out-of-range samples; the search falls back to the int32 path and stays exact."""
    import qmiv_b200
    f0, f1 = _pair(seed=9)
    bad = tuple(p.copy() for p in f1)
    bad[0][10:14, 20:24] = 5000
    with qmiv_b200.Calc(qctx, 256, 128, 10, invalid_pel_action=qmiv_b200.PEL_SKIP) as calc:
        got = calc.compute(f0, bad, qmiv_b200.IVPSNR | qmiv_b200.PSNR)
    exp = oracle_lib.compute_pair(oracle.make_params(256, 128, 10, 420), f0, bad, oracle.IVPSNR | oracle.PSNR)
    for k in ["gcd_r2t", "psnr", "ivpsnr", "ivpsnr_r2t", "ivpsnr_t2r"]:
        assert got[k] == exp[k], k


def test_bad_arguments(qctx):
    import qmiv_b200
    with pytest.raises(qmiv_b200.QmivError) as ei:
        qmiv_b200.Calc(qctx, 255, 128, 10, 420)  # odd width with 4:2:0
    assert ei.value.status == 1
    with pytest.raises(qmiv_b200.QmivError) as ei:
        qmiv_b200.Calc(qctx, 256, 128, 10, 420, search_range=7)
    assert ei.value.status == 2
    with qmiv_b200.Calc(qctx, 256, 128, 10) as calc:
        f0, f1 = _pair()
        with pytest.raises(ValueError):
            calc.compute(f0[:2], f1)


def test_hbm_budget(qctx):
    import qmiv_b200
    with qmiv_b200.Context(0, hbm_budget=1 << 20) as small:
        calc = qmiv_b200.Calc(small, 1024, 512, 10)
        f0, f1 = _pair(1024, 512)
        with pytest.raises(qmiv_b200.QmivError) as ei:
            calc.compute(f0, f1, qmiv_b200.ALL)
        assert ei.value.status == 6  # QMIV_ERR_BUDGET
        calc.close()
        assert small.memory()[0] == 0


def test_async_submit_wait_and_timeout(qctx):
    import qmiv_b200
    f0, f1 = _pair(1024, 512, seed=5)
    with qmiv_b200.Calc(qctx, 1024, 512, 10) as calc:
        sync = calc.compute(f0, f1, qmiv_b200.ALL)
        calc.submit(f0, f1, qmiv_b200.ALL)
        with pytest.raises(qmiv_b200.QmivError) as ei:
            calc.submit(f0, f1, qmiv_b200.ALL)
        assert ei.value.status == 10  # busy: one submission in flight
        got = None
        try:
            got = calc.wait(0)
        except qmiv_b200.QmivError as e:
            assert e.status == 7  # timeout with zero wait; the work is still in flight
        if got is None:
            got = calc.wait(-1)
        assert got == sync


def test_batch_matches_plain(qctx):
    import qmiv_b200
    shapes = [(256, 128, 10, 2), (192, 96, 8, 4), (256, 128, 10, 4), (320, 240, 8, 2)]
    pairs, plain = [], []
    for i, (W, H, bd, R) in enumerate(shapes):
        f0, f1 = _pair(W, H, bd, seed=100 + i)
        pairs.append(dict(frame0=f0, frame1=f1, width=W, height=H, bitdepth=bd, search_range=R,
                          metrics=qmiv_b200.IVPSNR | qmiv_b200.PSNR | qmiv_b200.IVSSIM))
        with qmiv_b200.Calc(qctx, W, H, bd, search_range=R) as calc:
            plain.append(calc.compute(f0, f1, pairs[-1]["metrics"]))
    with qmiv_b200.Batch(qctx, max_pairs=8, max_pixels=1 << 22) as batch:
        for _ in range(2):
            got = batch.compute(pairs)
            assert got == plain
