"""On-device ingest: raw YUV file bytes (planar, 1 byte per sample up to 8 bits, else 2 bytes little
endian) are consumed as they are stored, on the host or copied to the device in one block, with no
unpacking or chroma upsampling, and give the results of the unpacked frames; invalid samples are
checked and concealed on the device (xAppQMIV.cpp:834-852) and identical components flagged
(:894-897)."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _raw(frames):
    return np.frombuffer(b"".join(np.ascontiguousarray(p).tobytes() for f in frames for p in f), np.uint8).copy()


@pytest.mark.parametrize("shape", [(640, 360, 10, 420), (320, 240, 8, 420), (256, 128, 10, 422), (192, 96, 8, 444)])
def test_raw_file_bytes_host_and_device(shape, qctx, oracle_lib):
    import torch
    import qmiv_b200
    from qmiv_b200 import synth
    W, H, bd, cf = shape
    seq0, seq1 = [], []
    for k in range(3):
        a, b = synth.make_pair(W, H, bd, seed=40 + k, chroma_format=cf)
        seq0.append(a); seq1.append(b)
    raw0, raw1 = _raw(seq0), _raw(seq1)
    assert raw0.size == 3 * qmiv_b200.raw_frame_bytes(W, H, bd, cf)
    dev0, dev1 = torch.from_numpy(raw0).cuda(), torch.from_numpy(raw1).cuda()   # one upload per file
    mask = qmiv_b200.IVPSNR | qmiv_b200.PSNR | qmiv_b200.IVSSIM
    with qmiv_b200.Calc(qctx, W, H, bd, cf) as calc:
        for k in range(3):
            exp = calc.compute(seq0[k], seq1[k], mask)
            host = calc.compute(qmiv_b200.frame_from_raw(raw0, W, H, bd, cf, k),
                                qmiv_b200.frame_from_raw(raw1, W, H, bd, cf, k), mask)
            dev = calc.compute(qmiv_b200.frame_from_raw(dev0, W, H, bd, cf, k),
                               qmiv_b200.frame_from_raw(dev1, W, H, bd, cf, k), mask)
            assert host == exp and dev == exp, k
            ref = oracle_lib.compute_pair(oracle.make_params(W, H, bd, cf), seq0[k], seq1[k], mask)
            assert exp["ivpsnr"] == ref["ivpsnr"] and exp["ivssim"] == ref["ivssim"]


def test_raw_ingest_checks_and_flags(qctx, oracle_lib):
    """A raw frame with samples above the bit depth: refused under STOP, clipped under CNCL; a
    component identical in both frames gets the reference's fake PSNR."""
    import torch
    import qmiv_b200
    from qmiv_b200 import synth
    W, H, bd = 256, 128, 10
    a, b = synth.make_pair(W, H, bd, seed=3)
    b = (b[0].copy(), a[1].copy(), b[2].copy())          # Cb identical
    b[0][7, 9] = 1023 + 100
    raw0, raw1 = _raw([a]), _raw([b])
    d0, d1 = torch.from_numpy(raw0).cuda(), torch.from_numpy(raw1).cuda()
    f0, f1 = qmiv_b200.frame_from_raw(d0, W, H, bd), qmiv_b200.frame_from_raw(d1, W, H, bd)
    with qmiv_b200.Calc(qctx, W, H, bd) as calc:
        with pytest.raises(qmiv_b200.QmivError) as ei:
            calc.compute(f0, f1, qmiv_b200.PSNR)
        assert ei.value.status == 5
    with qmiv_b200.Calc(qctx, W, H, bd, invalid_pel_action=qmiv_b200.PEL_CNCL) as calc:
        got = calc.compute(f0, f1, qmiv_b200.PSNR | qmiv_b200.IVPSNR)
    clipped = tuple(np.minimum(p, 1023) for p in b)
    exp = oracle_lib.compute_pair(oracle.make_params(W, H, bd, 420), a, clipped, oracle.PSNR | oracle.IVPSNR)
    assert got["exact"][:3] == [0, 1, 0] and got["invalid_pel"] == [0, 1]
    for k in ["psnr", "ivpsnr", "gcd_r2t"]:
        assert got[k] == exp[k], k
