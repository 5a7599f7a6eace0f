"""The batched form (qmiv_batch_*, one launch per stage for all pairs, CPS as one persistent work list
per search range and sample size) against the plain one-pair form: identical results for uneven
shapes, bit depths, search ranges, chroma formats and metric sets, with host or device frames, on
eager runs, captured CUDA graphs and replays, with and without the tile-shape autotuner, and
independently of the other pairs in the batch."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ALL_METRICS = ["PSNR", "WSPSNR", "IVPSNR", "SSIM", "MSSSIM", "IVSSIM", "IVMSSSIM"]


def _specs():
    # (W, H, bd, cf, R, metrics)
    return [
        (256, 128, 10, 420, 2, ALL_METRICS),
        (192, 96, 8, 420, 4, ["IVPSNR", "PSNR", "IVSSIM"]),
        (130, 66, 10, 422, 3, ["IVPSNR", "SSIM", "WSPSNR"]),
        (320, 240, 8, 444, 1, ["IVPSNR", "IVMSSSIM"]),
        (128, 128, 12, 420, 5, ["IVPSNR", "MSSSIM", "IVSSIM"]),
        (64, 48, 8, 420, 2, ["PSNR", "WSPSNR"]),
        (640, 360, 10, 420, 4, ["IVPSNR", "PSNR", "IVSSIM"]),
        (258, 130, 8, 420, 2, ALL_METRICS),
    ]


def _frames(spec, seed, device=False, extra_pitch=0):
    import torch
    from qmiv_b200 import synth
    W, H, bd, cf, R, _ = spec
    f0, f1 = synth.make_pair(W, H, bd, seed=seed, chroma_format=cf)
    if not device:
        return f0, f1

    def dev(fr):
        out = []
        for p in fr:
            if extra_pitch:
                big = np.zeros((p.shape[0], p.shape[1] + extra_pitch), dtype=p.dtype)
                big[:, :p.shape[1]] = p
                out.append(torch.from_numpy(big).cuda()[:, :p.shape[1]])
            else:
                out.append(torch.from_numpy(np.ascontiguousarray(p)).cuda())
        return tuple(out)
    return dev(f0), dev(f1)


def _plain(qctx, spec, f0, f1, erp):
    import qmiv_b200
    W, H, bd, cf, R, metrics = spec
    with qmiv_b200.Calc(qctx, W, H, bd, cf, search_range=R, erp=erp) as calc:
        return calc.compute(f0, f1, qmiv_b200.metric_mask(metrics))


def _desc(spec, f0, f1):
    import qmiv_b200
    W, H, bd, cf, R, metrics = spec
    return dict(frame0=f0, frame1=f1, width=W, height=H, bitdepth=bd, chroma_format=cf, search_range=R,
                metrics=qmiv_b200.metric_mask(metrics))


@pytest.mark.parametrize("erp", [False, True])
def test_batch_uneven_set_matches_plain(qctx, erp):
    import qmiv_b200
    specs = _specs()
    frames = [_frames(s, 500 + i, device=(i % 2 == 1), extra_pitch=(3 if i == 3 else 0)) for i, s in enumerate(specs)]
    plain = [_plain(qctx, s, *f, erp) for s, f in zip(specs, frames)]
    px = sum(s[0] * s[1] for s in specs)
    with qmiv_b200.Batch(qctx, max_pairs=len(specs), max_pixels=px, erp=erp) as batch:
        got = batch.compute([_desc(s, *f) for s, f in zip(specs, frames)])
    for i, (g, p) in enumerate(zip(got, plain)):
        assert g == p, (i, specs[i])


def test_batch_graph_capture_and_replay(qctx):
    """Same signature four times with different frames: eager run, capture, replays."""
    import qmiv_b200
    specs = _specs()[:5]
    px = sum(s[0] * s[1] for s in specs)
    with qmiv_b200.Batch(qctx, max_pairs=8, max_pixels=px, graph=True) as batch:
        for rnd in range(4):
            frames = [_frames(s, 900 + 10 * rnd + i, device=True) for i, s in enumerate(specs)]
            plain = [_plain(qctx, s, *f, False) for s, f in zip(specs, frames)]
            got = batch.compute([_desc(s, *f) for s, f in zip(specs, frames)])
            assert got == plain, rnd


def test_batch_host_frames_in_sub_batches(qctx):
    """Host frames large enough to be uploaded in several sub-batches, overlapping compute."""
    import qmiv_b200
    spec = (4096, 2048, 10, 420, 2, ["IVPSNR", "PSNR", "IVSSIM", "WSPSNR"])
    frames = [_frames(spec, 60 + i) for i in range(3)]
    plain = [_plain(qctx, spec, *f, True) for f in frames]
    with qmiv_b200.Batch(qctx, max_pairs=3, max_pixels=3 * 4096 * 2048, erp=True) as batch:
        assert batch.compute([_desc(spec, *f) for f in frames]) == plain


def test_batch_autotune(qctx):
    import qmiv_b200
    specs = [(640, 360, 10, 420, 2, ["IVPSNR", "IVSSIM"]), (640, 360, 8, 420, 4, ["IVPSNR"]),
             (320, 240, 10, 444, 5, ["IVPSNR"])]
    frames = [_frames(s, 40 + i, device=True) for i, s in enumerate(specs)]
    plain = [_plain(qctx, s, *f, False) for s, f in zip(specs, frames)]
    with qmiv_b200.Batch(qctx, max_pairs=4, max_pixels=1 << 22, autotune=True) as batch:
        for _ in range(2):
            assert batch.compute([_desc(s, *f) for s, f in zip(specs, frames)]) == plain
        for W, H, bd, cf, R, _ in specs:
            tw, th, rows = batch.tuning(W, H, bd, R)
            assert tw == 128 and th in (16, 24, 32) and rows == 4
            if R == 5:
                assert th == 16
        with pytest.raises(qmiv_b200.QmivError):
            batch.tuning(100, 100, 8, 2)


def test_batch_result_independent_of_the_mix(qctx):
    """A pair's result is the same alone, in any position, and beside any other pairs."""
    import qmiv_b200
    specs = _specs()
    frames = [_frames(s, 700 + i, device=True) for i, s in enumerate(specs)]
    descs = [_desc(s, *f) for s, f in zip(specs, frames)]
    px = sum(s[0] * s[1] for s in specs)
    with qmiv_b200.Batch(qctx, max_pairs=len(specs), max_pixels=px) as batch:
        alone = [batch.compute([d])[0] for d in descs]
        mixed = batch.compute(descs)
        rev = batch.compute(descs[::-1])[::-1]
        sub = batch.compute(descs[1::2])
    assert mixed == alone and rev == alone
    assert sub == alone[1::2]


def test_batch_limits(qctx):
    import qmiv_b200
    s = _specs()[0]
    f0, f1 = _frames(s, 1, device=True)
    with qmiv_b200.Batch(qctx, max_pairs=1, max_pixels=s[0] * s[1]) as batch:
        with pytest.raises(qmiv_b200.QmivError):
            batch.compute([_desc(s, f0, f1)] * 2)
    with qmiv_b200.Batch(qctx, max_pairs=4, max_pixels=s[0] * s[1]) as batch:
        with pytest.raises(qmiv_b200.QmivError):
            batch.compute([_desc(s, f0, f1)] * 2)
        assert batch.compute([]) == []


def test_batch_submit_wait_two_in_flight(qctx):
    """Asynchronous submissions (qmiv_batch_submit / qmiv_batch_wait): two calls in flight, host and
    device frames, each call's results equal to the synchronous form; a third submission and a
    synchronous call while the first slot is held are refused."""
    import qmiv_b200
    specs = _specs()[:4]
    fa = [_frames(s, 1100 + i, device=(i % 2 == 0)) for i, s in enumerate(specs)]
    fb = [_frames(s, 1200 + i) for i, s in enumerate(specs)]
    px = sum(s[0] * s[1] for s in specs)
    with qmiv_b200.Batch(qctx, max_pairs=len(specs), max_pixels=px, autotune=True) as batch:
        da = [_desc(s, *f) for s, f in zip(specs, fa)]
        db = [_desc(s, *f) for s, f in zip(specs, fb)]
        exp_a, exp_b = batch.compute(da), batch.compute(db)
        for _ in range(3):
            ta = batch.submit(da)
            tb = batch.submit(db)
            with pytest.raises(qmiv_b200.QmivError) as ei:
                batch.submit(da)
            assert ei.value.status == 10  # QMIV_ERR_BUSY
            with pytest.raises(qmiv_b200.QmivError):
                batch.compute(da)
            assert batch.wait(tb) == exp_b
            assert batch.wait(ta) == exp_a
        with pytest.raises(qmiv_b200.QmivError):
            batch.wait(ta)
        ta = batch.submit(da)   # left in flight: destroying the batch waits for it
