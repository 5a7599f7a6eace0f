"""Mask mode (qmiv_frame_pair_compute_masked): GCD-M, CPS-M, PSNR-M, WS-PSNR-M and IV-PSNR-M against
the compiled reference's fixtures and the C restatement, bit for bit, with host and device frames."""
import numpy as np
import pytest

import oracle
from golden_cases import compare_masked, masked_case_inputs

pytestmark = pytest.mark.gpu


def _ids():
    import json, os
    with open(os.path.join(os.path.dirname(__file__), "golden", "golden_masked.json")) as f:
        g = json.load(f)["masked"]
    return [f"{c['width']}x{c['height']}_{c['bitdepth']}b_{c['chroma_format']}_R{c['search_range']}"
            f"{'_erp' if c['erp'] else ''}_m{c['mask_bitdepth']}{c['mask_kind']}" for c in g]


def _calc(qctx, case):
    import qmiv_b200
    return qmiv_b200.Calc(qctx, case["width"], case["height"], case["bitdepth"], case["chroma_format"],
                          search_range=case["search_range"], erp=case["erp"])


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("idx", range(len(_ids())), ids=_ids())
def test_masked_golden_host_frames(idx, golden_masked, qctx):
    case = golden_masked[idx]
    f0, f1, m = masked_case_inputs(case)
    with _calc(qctx, case) as calc:
        got, nnm = calc.compute_masked(f0, f1, m, case["mask_bitdepth"])
    assert compare_masked(got, nnm, case["expected"]) == []


@pytest.mark.parametrize("idx", [0, 2, 6, 9], ids=[_ids()[i] for i in [0, 2, 6, 9]])
def test_masked_golden_device_frames(idx, golden_masked, qctx):
    case = golden_masked[idx]
    f0, f1, m = masked_case_inputs(case)
    with _calc(qctx, case) as calc:
        got, nnm = calc.compute_masked(tuple(_dev(p) for p in f0), tuple(_dev(p) for p in f1), _dev(m),
                                       case["mask_bitdepth"])
    assert compare_masked(got, nnm, case["expected"]) == []


@pytest.mark.parametrize("shape", [(640, 360, 10, 420, 2, True, 8, "weights"), (352, 288, 8, 422, 5, False, 10, "binary"),
                                   (258, 130, 10, 444, 3, True, 12, "sparse"),
                                   (4096, 2048, 10, 420, 2, True, 8, "binary")])
def test_masked_against_oracle_seeded(shape, qctx, oracle_lib):
    """Seeded synthetic frames (the bench's generator) with detgen masks, up to the 4096x2048 workload."""
    import qmiv_b200
    from qmiv_b200 import synth
    from detgen import det_mask
    W, H, bd, cf, R, erp, mbd, kind = shape
    f0, f1 = synth.make_pair(W, H, bd, seed=W + H, chroma_format=cf)
    m = det_mask(W, H, mbd, W * 3 + H, kind)
    p = oracle.make_params(W, H, bd, cf, search_range=R, erp=erp)
    exp, n_exp = oracle_lib.compute_pair_masked(p, f0, f1, m, mbd)
    with qmiv_b200.Calc(qctx, W, H, bd, cf, search_range=R, erp=erp) as calc:
        got, nnm = calc.compute_masked(f0, f1, m, mbd)
    assert nnm == n_exp
    for k in ["gcd_r2t", "psnr", "wspsnr"]:
        assert list(got[k][:3]) == list(exp[k][:3]), k
    for k in ["psnr_pic", "wspsnr_pic", "ivpsnr", "ivpsnr_r2t", "ivpsnr_t2r"]:
        assert got[k] == exp[k], k


def test_masked_ones_equals_plain_ivpsnr(qctx):
    """With every mask sample at its maximum, IV-PSNR-M is the plain IV-PSNR (the weights and the
    non-masked count cancel), while PSNR-M shows the reference's use of the mask's bit depth."""
    import qmiv_b200
    from qmiv_b200 import synth
    W, H, bd = 320, 240, 10
    f0, f1 = synth.make_pair(W, H, bd, seed=5)
    ones = np.full((H, W), 255, np.uint8)
    with qmiv_b200.Calc(qctx, W, H, bd) as calc:
        plain = calc.compute(f0, f1, qmiv_b200.IVPSNR | qmiv_b200.PSNR)
        got, nnm = calc.compute_masked(f0, f1, ones, 8)
    assert nnm == W * H
    assert got["ivpsnr"] == plain["ivpsnr"]
    assert got["gcd_r2t"] == plain["gcd_r2t"]
    # 10 log10(1023^2 / 255^2) apart
    assert abs((plain["psnr"][0] - got["psnr"][0]) - 20 * np.log10(1023 / 255)) < 1e-9


def test_masked_errors(qctx):
    import qmiv_b200
    from qmiv_b200 import synth
    from detgen import det_mask
    W, H = 64, 48
    f0, f1 = synth.make_pair(W, H, 8, seed=1)
    m = det_mask(W, H, 8, 1)
    with qmiv_b200.Calc(qctx, W, H, 8) as calc:
        with pytest.raises(qmiv_b200.QmivError) as ei:
            calc.compute_masked(f0, f1, m, 8, qmiv_b200.IVSSIM)
        assert ei.value.status == 2  # QMIV_ERR_UNSUPPORTED
        with pytest.raises(qmiv_b200.QmivError):
            calc.compute_masked(f0, f1, np.zeros((H, W), np.uint8), 8)
        with pytest.raises(qmiv_b200.QmivError):
            calc.compute_masked(f0, f1, m, 7)
        # the calc still works after the refusals
        got, nnm = calc.compute_masked(f0, f1, m, 8)
        assert nnm == int((m != 0).sum())


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(640, 360, 10, 420, 2, 8, "weights"), (352, 288, 8, 444, 5, 10, "binary"),
                                   (258, 130, 10, 422, 4, 12, "sparse"), (200, 100, 10, 420, 1, 8, "weights")])
def test_masked_search_forms_agree(shape, qctx, oracle_lib):
    """The masked search has two kernels: exact integer keys, four pixels per thread, where the bit
    depth, weights and GCD range bound every error and samples are in range (STOP, CNCL), and the
    plain per-candidate integer loop otherwise (SKIP, WARN). On in-range frames every action gives
    the same values, and both equal the C restatement."""
    import qmiv_b200
    from qmiv_b200 import synth
    from detgen import det_mask
    W, H, bd, cf, R, mbd, kind = shape
    f0, f1 = synth.make_pair(W, H, bd, seed=W * 7 + R, chroma_format=cf)
    m = det_mask(W, H, mbd, W + 11 * H, kind)
    p = oracle.make_params(W, H, bd, cf, search_range=R, erp=True)
    exp, n_exp = oracle_lib.compute_pair_masked(p, f0, f1, m, mbd)
    sse = []
    for act in (qmiv_b200.PEL_STOP, qmiv_b200.PEL_CNCL, qmiv_b200.PEL_SKIP, qmiv_b200.PEL_WARN):
        with qmiv_b200.Calc(qctx, W, H, bd, cf, search_range=R, erp=True, invalid_pel_action=act) as calc:
            got, nnm = calc.compute_masked(f0, f1, m, mbd)
        assert nnm == n_exp
        for k in ["gcd_r2t", "psnr", "wspsnr"]:
            assert list(got[k][:3]) == list(exp[k][:3]), (act, k)
        for k in ["psnr_pic", "wspsnr_pic", "ivpsnr", "ivpsnr_r2t", "ivpsnr_t2r"]:
            assert got[k] == exp[k], (act, k)
        sse.append((list(got["cps_sse_r2t"][:3]), list(got["cps_sse_t2r"][:3])))
    assert all(v == sse[0] for v in sse), sse      # the per-direction uint64 search sums of both kernels


@pytest.mark.gpu
def test_masked_out_of_range_samples_skip(qctx, oracle_lib):
    """Under SKIP, samples above the bit depth's maximum are searched as they are (the integer-loop
    kernel); the results equal the C restatement's on the same frames."""
    import qmiv_b200
    from qmiv_b200 import synth
    from detgen import det_mask
    W, H, bd = 160, 96, 10
    f0, f1 = synth.make_pair(W, H, bd, seed=99)
    f1 = tuple(np.array(pl, copy=True) for pl in f1)
    f1[0][10, 17] = 1500
    f1[1][5, 9] = 1200
    m = det_mask(W, H, 8, 5, "weights")
    p = oracle.make_params(W, H, bd, 420, search_range=2, erp=False)   # the restatement computes on raw samples
    exp, n_exp = oracle_lib.compute_pair_masked(p, f0, f1, m, 8)
    with qmiv_b200.Calc(qctx, W, H, bd, search_range=2, invalid_pel_action=qmiv_b200.PEL_SKIP) as calc:
        got, nnm = calc.compute_masked(f0, f1, m, 8)
    assert nnm == n_exp
    for k in ["gcd_r2t", "psnr"]:
        assert list(got[k][:3]) == list(exp[k][:3]), k
    for k in ["psnr_pic", "ivpsnr", "ivpsnr_r2t", "ivpsnr_t2r"]:
        assert got[k] == exp[k], k


@pytest.mark.parametrize("erp", [False, True])
def test_masked_batched_equals_one_pair_calls(erp, golden_masked, qctx):
    """The batched mask mode (qmiv_batch_compute_masked) on an uneven set: every golden case (8/10/12-bit
    pictures, 8-14-bit masks, R 1-5, 4:2:0/4:2:2/4:4:4 as the fixtures have them) plus seeded
    1920x1080 and 4096x2048 pairs, host and device frames mixed, in one call. Each pair's result
    equals the one-pair call's; the golden cases also equal the compiled reference's fixtures."""
    import qmiv_b200
    from qmiv_b200 import synth
    from detgen import det_mask
    cases = [c for c in golden_masked if bool(c["erp"]) == erp]
    items = []
    for k, c in enumerate(cases):
        f0, f1, m = masked_case_inputs(c)
        if k % 2:
            f0, f1, m = tuple(_dev(p) for p in f0), tuple(_dev(p) for p in f1), _dev(m)
        items.append((c["width"], c["height"], c["bitdepth"], c["chroma_format"], c["search_range"], f0, f1, m,
                      c["mask_bitdepth"], c))
    for W, H, bd, R, mbd in [(1920, 1080, 8, 2, 8), (4096, 2048, 10, 2, 10)]:
        f0, f1 = synth.make_pair(W, H, bd, seed=W + bd)
        m = det_mask(W, H, mbd, W + H, "weights")
        items.append((W, H, bd, 420, R, tuple(_dev(p) for p in f0), tuple(_dev(p) for p in f1), _dev(m), mbd, None))
    mask = qmiv_b200.PSNR | qmiv_b200.WSPSNR | qmiv_b200.IVPSNR
    pairs = [dict(frame0=f0, frame1=f1, width=W, height=H, bitdepth=bd, chroma_format=cf, search_range=R, metrics=mask)
             for W, H, bd, cf, R, f0, f1, m, mbd, c in items]
    with qmiv_b200.Batch(qctx, len(pairs), sum(p["width"] * p["height"] for p in pairs), erp=erp) as batch:
        for _ in range(2):   # the second call reuses the batch's arena
            got, nnm = batch.compute_masked(pairs, [it[7] for it in items], [it[8] for it in items])
            for i, (W, H, bd, cf, R, f0, f1, m, mbd, c) in enumerate(items):
                with qmiv_b200.Calc(qctx, W, H, bd, cf, search_range=R, erp=erp) as calc:
                    one, one_nnm = calc.compute_masked(f0, f1, m, mbd)
                assert got[i] == one and nnm[i] == one_nnm, (i, W, H, bd, R)
                if c is not None:
                    assert compare_masked(got[i], nnm[i], c["expected"]) == []


@pytest.mark.gpu
@pytest.mark.parametrize("bd", [10, 14])
def test_masked_prepass_large_samples(bd, qctx, oracle_lib):
    """The aligned 4:2:0 prepass with an 8-bit mask sums pairs of 16-bit samples in 32-bit words while
    every sample of a thread's step is below 2^15, and sample by sample with the reference's int32
    products otherwise. Frames with raw samples of 2^15 and above under SKIP give the C restatement's
    sums at 10 bits and at 14 bits (the deepest mask mode takes); rows of 320 groups leave threads with
    and without a large sample in the same row."""
    import qmiv_b200
    from qmiv_b200 import synth
    from detgen import det_mask
    W, H = 1280, 64
    f0, f1 = synth.make_pair(W, H, bd, seed=5 + bd)
    f0 = tuple(np.array(pl, copy=True) for pl in f0)
    f1 = tuple(np.array(pl, copy=True) for pl in f1)
    f1[0][3, 100] = 40000
    f1[0][7, W - 1] = 65535
    f1[2][10, 33] = 32768
    f0[1][20, 600] = 50000
    m = det_mask(W, H, 8, 17, "weights")
    p = oracle.make_params(W, H, bd, 420, search_range=2, erp=True)
    exp, n_exp = oracle_lib.compute_pair_masked(p, f0, f1, m, 8)
    with qmiv_b200.Calc(qctx, W, H, bd, search_range=2, erp=True, invalid_pel_action=qmiv_b200.PEL_SKIP) as calc:
        got, nnm = calc.compute_masked(f0, f1, m, 8)
    assert nnm == n_exp
    for k in ["gcd_r2t", "psnr", "wspsnr"]:
        assert list(got[k][:3]) == list(exp[k][:3]), k
    for k in ["psnr_pic", "wspsnr_pic", "ivpsnr", "ivpsnr_r2t", "ivpsnr_t2r"]:
        assert got[k] == exp[k], k


@pytest.mark.gpu
@pytest.mark.parametrize("erp", [False, True])
def test_masked_staged_prepass_against_oracle(erp, qctx, oracle_lib):
    """Aligned 4:2:0 pairs with 8-bit masks and widths divisible by 32 take the staged prepass: persistent
    CTAs over the row pairs of every pair of a launch, each CTA's contiguous range crossing from one
    pair into the next. Pairs of four widths (stage slots of different sizes), host and device frames,
    in one batched call and one by one, give the C restatement's values."""
    import qmiv_b200
    from qmiv_b200 import synth
    from detgen import det_mask
    shapes = [(640, 360, 10, 2), (1280, 96, 8, 1), (2048, 130, 10, 3), (96, 34, 10, 2), (4096, 64, 8, 2)]
    items = []
    for k, (W, H, bd, R) in enumerate(shapes):
        f0, f1 = synth.make_pair(W, H, bd, seed=31 * k + W)
        m = det_mask(W, H, 8, 7 * k + H, "weights" if k % 2 else "sparse")
        p = oracle.make_params(W, H, bd, 420, search_range=R, erp=erp)
        exp, n_exp = oracle_lib.compute_pair_masked(p, f0, f1, m, 8)
        if k % 2:
            f0, f1, m = tuple(_dev(x) for x in f0), tuple(_dev(x) for x in f1), _dev(m)
        items.append((W, H, bd, R, f0, f1, m, exp, n_exp))
    keys3 = ["gcd_r2t", "psnr", "wspsnr"]
    keys = ["psnr_pic", "wspsnr_pic", "ivpsnr", "ivpsnr_r2t", "ivpsnr_t2r"]
    pairs = [dict(frame0=f0, frame1=f1, width=W, height=H, bitdepth=bd, search_range=R,
                  metrics=qmiv_b200.PSNR | qmiv_b200.WSPSNR | qmiv_b200.IVPSNR) for W, H, bd, R, f0, f1, m, e, n in items]
    with qmiv_b200.Batch(qctx, len(pairs), sum(W * H for W, H, *_ in items), erp=erp) as batch:
        got, nnm = batch.compute_masked(pairs, [it[6] for it in items], [8] * len(items))
    for i, (W, H, bd, R, f0, f1, m, exp, n_exp) in enumerate(items):
        assert nnm[i] == n_exp, (W, H)
        for k in keys3:
            assert list(got[i][k][:3]) == list(exp[k][:3]), (W, H, k)
        for k in keys:
            assert got[i][k] == exp[k], (W, H, k)
        with qmiv_b200.Calc(qctx, W, H, bd, search_range=R, erp=erp) as calc:
            one, one_nnm = calc.compute_masked(f0, f1, m, 8)
        assert one == got[i] and one_nnm == n_exp, (W, H)


@pytest.mark.gpu
def test_masked_batched_more_pairs_than_one_pack(qctx):
    """A batched mask-mode call passes each launch group's arguments in packs of up to 32 pairs: 40
    pairs of two sample sizes and two search ranges (groups that span two packs and groups that fit
    one) equal their one-pair calls."""
    import qmiv_b200
    from qmiv_b200 import synth
    from detgen import det_mask
    shapes = [(64 + 32 * (i % 3), 32 + 16 * (i % 2), 8 if i % 4 else 10, 2 if i % 5 else 3) for i in range(40)]
    items = []
    for i, (W, H, bd, R) in enumerate(shapes):
        f0, f1 = synth.make_pair(W, H, bd, seed=300 + i)
        m = det_mask(W, H, 8, 5 + i, "weights" if i % 2 else "binary")
        if i % 3 == 0:
            f0, f1, m = tuple(_dev(x) for x in f0), tuple(_dev(x) for x in f1), _dev(m)
        items.append((W, H, bd, R, f0, f1, m))
    pairs = [dict(frame0=f0, frame1=f1, width=W, height=H, bitdepth=bd, search_range=R,
                  metrics=qmiv_b200.PSNR | qmiv_b200.WSPSNR | qmiv_b200.IVPSNR) for W, H, bd, R, f0, f1, m in items]
    with qmiv_b200.Batch(qctx, len(pairs), sum(W * H for W, H, *_ in items), erp=True) as batch:
        got, nnm = batch.compute_masked(pairs, [it[6] for it in items], [8] * len(items))
    for i, (W, H, bd, R, f0, f1, m) in enumerate(items):
        with qmiv_b200.Calc(qctx, W, H, bd, search_range=R, erp=True) as calc:
            one, one_nnm = calc.compute_masked(f0, f1, m, 8)
        assert got[i] == one and nnm[i] == one_nnm, (i, W, H, bd, R)


@pytest.mark.gpu
def test_masked_stage_timers(qctx):
    """With the context's profiling on, a mask-mode call (one pair, then a batch of three) times each of
    its stages once per call on the stream it runs on: prepass, reduce, search, finalize and read-back."""
    import qmiv_b200
    from qmiv_b200 import synth
    from detgen import det_mask
    W, H = 320, 192
    f0, f1 = synth.make_pair(W, H, 10, seed=41)
    m = det_mask(W, H, 8, 3, "weights")
    stages = ("prepass", "reduce", "cps", "finalize", "d2h")
    with qmiv_b200.Calc(qctx, W, H, 10, search_range=2, erp=True) as calc:
        calc.compute_masked(f0, f1, m, 8)
        qctx.stage_times(reset=True)
        qctx.set_profiling(True)
        try:
            calc.compute_masked(f0, f1, m, 8)
        finally:
            qctx.set_profiling(False)
        st = qctx.stage_times(reset=True)
    for k in stages:
        assert st[k][1] == 1 and st[k][0] > 0.0, (k, st[k])
    pairs = [dict(frame0=f0, frame1=f1, width=W, height=H, bitdepth=10, search_range=2,
                  metrics=qmiv_b200.PSNR | qmiv_b200.WSPSNR | qmiv_b200.IVPSNR)] * 3
    with qmiv_b200.Batch(qctx, 3, 3 * W * H, erp=True) as batch:
        batch.compute_masked(pairs, [m] * 3, [8] * 3)
        qctx.stage_times(reset=True)
        qctx.set_profiling(True)
        try:
            batch.compute_masked(pairs, [m] * 3, [8] * 3)
        finally:
            qctx.set_profiling(False)
        st = qctx.stage_times(reset=True)
    for k in stages:
        assert st[k][1] == 1 and st[k][0] > 0.0, (k, st[k])
