"""The drop-in adapter (qmiv_b200/shim/xQmivGpu.cpp): a QMIV host's own 4:4:4 xPicP pictures handed to
the library through the adapter, compiled against the reference's headers and objects
(oracle/shim_check.cpp, oracle/Makefile shimcheck). Every metric equals the compiled reference
library's on the same frames (apps/QMIV/src/xAppQMIV.cpp:927-1108 processor calls) and the library's
own 4:2:0 path."""
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

KEYS = ["gcd_r2t", "psnr", "psnr_pic", "wspsnr", "wspsnr_pic", "ivpsnr", "ivpsnr_r2t", "ivpsnr_t2r", "ssim", "ssim_pic",
        "msssim", "msssim_pic", "ivssim", "ivssim_r2t", "ivssim_t2r", "ivmsssim", "ivmsssim_r2t", "ivmsssim_t2r"]


def _decode(v):
    if isinstance(v, list):
        return [_decode(x) for x in v]
    return float.fromhex(v) if isinstance(v, str) else v


@pytest.mark.parametrize("W,H,bd,R,erp", [(320, 240, 10, 2, True), (256, 192, 8, 3, False)])
def test_adapter_on_reference_pictures(W, H, bd, R, erp, qctx):
    import qmiv_b200
    from qmiv_b200 import synth
    exe = oracle.shim_check_path()
    if exe is None or not oracle.reference_available():
        pytest.skip("the adapter's check program is built where the reference's sources are (oracle/Makefile shimcheck)")
    f0, f1 = synth.make_pair(W, H, bd, seed=900 + bd)
    mask = oracle.ALL
    with tempfile.TemporaryDirectory() as tmp:
        paths = []
        for k, fr in enumerate((f0, f1)):
            p = os.path.join(tmp, f"in{k}.yuv")
            with open(p, "wb") as f:
                for plane in fr:
                    f.write(np.ascontiguousarray(plane).tobytes())
            paths.append(p)
        out = subprocess.run([exe, str(W), str(H), str(bd), "420", str(R), str(int(erp)), str(mask), *paths],
                             capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    got = {k: _decode(v) for k, v in json.loads(out.stdout).items()}
    ref = oracle.Reference().compute_pair(oracle.make_params(W, H, bd, 420, search_range=R, erp=erp), f0, f1, mask)
    with qmiv_b200.Calc(qctx, W, H, bd, 420, search_range=R, erp=erp) as calc:
        lib420 = calc.compute(f0, f1, mask)
    for k in KEYS:
        g = got[k][:3] if isinstance(got[k], list) else got[k]
        r = ref[k][:3] if isinstance(ref[k], list) else ref[k]
        l420 = lib420[k][:3] if isinstance(lib420[k], list) else lib420[k]
        assert g == r, k
        assert g == l420, k
    # the adapter's single-metric calls agree with its one-pass call
    assert got["one_psnr_y"] == got["psnr"][0] and got["one_ssim_y"] == got["ssim"][0]
    assert got["one_ivpsnr"] == got["ivpsnr"] and got["one_ivssim"] == got["ivssim"]
