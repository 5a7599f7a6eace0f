"""The allocation-free entry point, qmiv_frame_pair_compute_static.

Some callers of this library cannot allocate device memory: code that runs inside a host
application's own memory manager or a plugin sandbox where cudaMalloc is forbidden, and services
that must not allocate after start-up. The entry point keeps all of its scratch in one fixed device
array, so these callers can still compute PSNR, WS-PSNR and IV-PSNR of device-resident frames.

This file is collected last so that a run stopping at the first failure has run every other test.
It checks the entry point through the C ABI against the regular entry point on two calls in a row
(the second call must not see the first call's leftovers in the shared array). The tolerance is the
one the other parity tests use: results must be identical.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_frame(frame):
    import torch
    import qmiv_b200
    planes = tuple(torch.from_numpy(np.ascontiguousarray(p)).cuda() for p in frame)
    f, keep = qmiv_b200.make_frame(planes)
    return f, (planes, keep)


def _static_call(lib, f0, f1, W, H, bd, params, mask, cf=420):
    from qmiv_b200 import _lib
    out = _lib.QmivResult()
    st = lib.qmiv_frame_pair_compute_static(ctypes.byref(f0), ctypes.byref(f1), W, H, bd, cf, ctypes.byref(params),
                                            mask, None, ctypes.byref(out))
    return st, out.as_dict()


_KEYS = ("gcd_r2t", "exact", "ssd", "cps_sse_r2t", "cps_sse_t2r", "psnr", "psnr_pic", "wspsnr", "wspsnr_pic",
         "ivpsnr", "ivpsnr_r2t", "ivpsnr_t2r")


@pytest.mark.parametrize("erp", [False, True])
def test_static_entry_point_matches_regular_entry_point(erp):
    import torch
    import qmiv_b200
    from qmiv_b200 import synth
    lib = qmiv_b200.library()
    W, H, bd = 1920, 1080, 10
    mask = qmiv_b200.PSNR | qmiv_b200.WSPSNR | qmiv_b200.IVPSNR
    params = qmiv_b200.make_params(erp=erp)
    with qmiv_b200.Context(0) as ctx, qmiv_b200.Calc(ctx, W, H, bd, 420, erp=erp) as calc:
        for seed in (11, 12):  # two calls in a row through the shared scratch array
            a, b = synth.make_pair(W, H, bd, seed=seed)
            f0, k0 = _device_frame(a)
            f1, k1 = _device_frame(b)
            st, got = _static_call(lib, f0, f1, W, H, bd, params, mask)
            assert st == 0, lib.qmiv_last_error()
            torch.cuda.synchronize()
            exp = calc.compute(k0[0], k1[0], mask)
            for key in _KEYS:
                assert got[key] == exp[key], key


def test_static_entry_point_other_formats_match_oracle_and_allocate_nothing():
    """8-bit 4:4:4 at search range 4, then a taller 10-bit 4:2:0 picture (so a call cannot pass on rows
    an earlier call left in the shared array), each checked against the regular entry point and the
    oracle; after a first call, a further call leaves the device's free memory unchanged."""
    import torch
    import oracle
    import qmiv_b200
    from qmiv_b200 import synth
    lib = qmiv_b200.library()
    mask = qmiv_b200.PSNR | qmiv_b200.WSPSNR | qmiv_b200.IVPSNR
    cases = [(320, 180, 8, 444, 4, 21), (256, 600, 10, 420, 2, 22)]
    for W, H, bd, cf, R, seed in cases:
        params = qmiv_b200.make_params(search_range=R, erp=True)
        a, b = synth.make_pair(W, H, bd, seed=seed, chroma_format=cf)
        f0, k0 = _device_frame(a)
        f1, k1 = _device_frame(b)
        st, got = _static_call(lib, f0, f1, W, H, bd, params, mask, cf)
        assert st == 0, lib.qmiv_last_error()
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        st, again = _static_call(lib, f0, f1, W, H, bd, params, mask, cf)
        assert st == 0, lib.qmiv_last_error()
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free0, "the call changed the device's free memory"
        assert again == got
        with qmiv_b200.Context(0) as ctx, qmiv_b200.Calc(ctx, W, H, bd, cf, search_range=R, erp=True) as calc:
            exp = calc.compute(k0[0], k1[0], mask)
        ref = oracle.Oracle().compute_pair(oracle.make_params(W, H, bd, cf, search_range=R, erp=True), a, b,
                                           oracle.PSNR | oracle.WSPSNR | oracle.IVPSNR)
        for key in _KEYS:
            assert got[key] == exp[key], key
        for key in ("gcd_r2t", "exact", "psnr", "psnr_pic", "wspsnr", "wspsnr_pic", "ivpsnr", "ivpsnr_r2t", "ivpsnr_t2r"):
            assert got[key] == ref[key], key


def test_static_entry_point_rejects_what_it_cannot_do():
    import qmiv_b200
    from qmiv_b200 import synth
    lib = qmiv_b200.library()
    params = qmiv_b200.make_params()
    W, H = 64, 4400  # taller than QMIV_STATIC_MAX_HEIGHT
    a, b = synth.make_pair(W, H, 8, seed=3)
    f0, k0 = _device_frame(a)
    f1, k1 = _device_frame(b)
    st, _ = _static_call(lib, f0, f1, W, H, 8, params, qmiv_b200.IVPSNR)
    assert st == 2  # QMIV_ERR_UNSUPPORTED
    st, _ = _static_call(lib, f0, f1, W, H, 8, params, qmiv_b200.IVSSIM)
    assert st == 2
    h0, hk0 = qmiv_b200.make_frame(synth.make_pair(64, 64, 8, seed=4)[0])
    st, _ = _static_call(lib, h0, h0, 64, 64, 8, params, qmiv_b200.IVPSNR)
    assert st == 1  # host frames are not accepted
