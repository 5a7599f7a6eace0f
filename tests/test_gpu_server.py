"""The serving loop (qmiv_server_*): requests of uneven shape, search range and metric set admitted by HBM
budget and continuously batched. Every request's results are the same alone, in a concurrent mix and in
the plain one-pair form; sequence means follow the reference's compensated average; admission waits for
memory and rejects what can never fit; latency statistics are reported."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _req_frames(W, H, bd, n, seed, device):
    import torch
    from qmiv_b200 import synth
    out = []
    for i in range(n):
        f0, f1 = synth.make_pair(W, H, bd, seed=seed + i)
        if device:
            f0 = tuple(torch.from_numpy(p).cuda() for p in f0)
            f1 = tuple(torch.from_numpy(p).cuda() for p in f1)
        out.append((f0, f1))
    return out


def _requests():
    # (W, H, bd, R, metrics, pairs, device frames)
    return [
        (640, 360, 10, 2, ["IVPSNR", "PSNR", "IVSSIM"], 5, True),
        (320, 240, 8, 4, ["IVPSNR"], 3, False),
        (256, 128, 10, 3, ["IVPSNR", "PSNR", "IVSSIM", "SSIM", "MSSSIM", "IVMSSSIM", "WSPSNR"], 4, True),
        (1280, 720, 8, 2, ["IVPSNR", "PSNR"], 2, False),
        (416, 240, 10, 5, ["IVPSNR", "IVSSIM"], 6, True),
    ]


def _kbns_mean(vals):
    s = c = 0.0
    for v in vals:
        t = s + v
        c += ((s - t) + v) if abs(s) >= abs(v) else ((v - t) + s)
        s = t
    return (s + c) / len(vals)


def test_server_results_alone_mixed_and_plain(qctx):
    import qmiv_b200
    reqs = _requests()
    frames = [_req_frames(W, H, bd, n, 100 * k, dev) for k, (W, H, bd, R, m, n, dev) in enumerate(reqs)]
    plain = []
    for (W, H, bd, R, m, n, dev), fr in zip(reqs, frames):
        with qmiv_b200.Calc(qctx, W, H, bd, search_range=R) as calc:
            plain.append([calc.compute(a, b, qmiv_b200.metric_mask(m)) for a, b in fr])
    with qmiv_b200.Server(qctx, max_batch_pairs=8, max_batch_pixels=8 * 1280 * 720, workers=2) as srv:
        alone = []
        for (W, H, bd, R, m, n, dev), fr in zip(reqs, frames):
            t = srv.submit(fr, W, H, bd, search_range=R, metrics=m)
            alone.append(srv.wait(t))
        tickets = [srv.submit(fr, W, H, bd, search_range=R, metrics=m)
                   for (W, H, bd, R, m, n, dev), fr in zip(reqs, frames)]
        mixed = [srv.wait(t) for t in tickets[::-1]][::-1]
        st = srv.stats()
    for k in range(len(reqs)):
        assert alone[k][0] == plain[k], k
        assert mixed[k][0] == plain[k], k
        stats = mixed[k][1]
        assert stats["mean_ivpsnr"] == _kbns_mean([r["ivpsnr"] for r in plain[k]])
        assert stats["latency_ms"] > 0 and stats["done_ms"] >= stats["admit_ms"] >= stats["submit_ms"]
        assert stats["batches"] >= 1
    assert st["completed"] == 2 * len(reqs)
    assert 0 < st["p50_ms"] <= st["p99_ms"] and st["pairs_per_s"] > 0


def test_server_admission_by_budget():
    import qmiv_b200
    W, H, bd = 640, 360, 10
    # staged bytes of one 640x360 10-bit 4:2:0 frame: 640*2*360 + 2 * 320*2*180 = 691200
    frame = 691200
    one = 2 * 8 * frame                       # resident frames of one 8-pair request
    ctx = qmiv_b200.Context(0, hbm_budget=int(1.5 * one) + (1 << 20))   # one fits, two do not
    try:
        fr = _req_frames(W, H, bd, 8, 7, device=False)
        with qmiv_b200.Server(ctx, max_batch_pairs=4, max_batch_pixels=4 * W * H, workers=1) as srv:
            with pytest.raises(qmiv_b200.QmivError) as ei:
                srv.submit(fr * 3, W, H, bd, metrics=["IVPSNR"])   # 24 pairs: more than the whole budget
            assert ei.value.status == 6
            t1 = srv.submit(fr, W, H, bd, metrics=["IVPSNR", "PSNR"])
            t2 = srv.submit(fr[::-1], W, H, bd, metrics=["IVPSNR", "PSNR"])
            r1, s1 = srv.wait(t1)
            r2, s2 = srv.wait(t2)
        # the second request's frames fit only after the first one's were released
        assert s2["admit_ms"] >= s1["done_ms"]
        assert r2 == r1[::-1]
        used, budget = ctx.memory()
        assert used <= budget
    finally:
        ctx.close()


def test_server_waits_and_timeouts(qctx):
    import qmiv_b200
    fr = _req_frames(256, 128, 10, 2, 3, device=True)
    with qmiv_b200.Server(qctx, max_batch_pairs=2, max_batch_pixels=2 * 256 * 128, workers=1) as srv:
        t = srv.submit(fr, 256, 128, 10, metrics=["IVPSNR"])
        res, st = srv.wait(t, timeout_ms=60000)
        assert len(res) == 2 and math.isfinite(st["mean_ivpsnr"])
        with pytest.raises(qmiv_b200.QmivError):
            srv.wait(t)   # released by the successful wait
        pending = [srv.submit(fr, 256, 128, 10, metrics=["IVPSNR"]) for _ in range(3)]
    # destroy waited for the pending requests; their tickets are gone with the server
    assert len(pending) == 3
