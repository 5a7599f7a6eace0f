"""Host-side logic that needs no GPU: metric selection, frame descriptors, synthetic workloads, the
deterministic fixture generator, and the fp32 exactness bound of the CPS search keys."""
import numpy as np
import pytest

import qmiv_b200
from qmiv_b200 import synth
from detgen import det_pair, hash32


def test_metric_mask_parsing():
    assert qmiv_b200.metric_mask(None) == qmiv_b200.ALL
    assert qmiv_b200.metric_mask("IVPSNR, WS-PSNR") == qmiv_b200.IVPSNR | qmiv_b200.WSPSNR
    assert qmiv_b200.metric_mask(["psnr", "IV_SSIM"]) == qmiv_b200.PSNR | qmiv_b200.IVSSIM
    with pytest.raises(ValueError):
        qmiv_b200.metric_mask("VMAF")


def test_make_frame_host_planes():
    f0, _ = synth.make_pair(64, 32, 10, seed=1)
    fr, keep = qmiv_b200.make_frame(f0)
    assert fr.mem == 0
    assert [fr.pitch[c] for c in range(3)] == [128, 64, 64]
    with pytest.raises(ValueError):
        qmiv_b200.make_frame(f0[:2])


@pytest.mark.parametrize("cf", [420, 422, 444])
def test_synth_shapes_and_ranges(cf):
    f0, f1 = synth.make_pair(128, 64, 10, seed=3, chroma_format=cf)
    cw = 128 if cf == 444 else 64
    ch = 32 if cf == 420 else 64
    assert f0[0].shape == (64, 128) and f0[1].shape == (ch, cw) and f1[2].shape == (ch, cw)
    assert all(p.dtype == np.uint16 and p.max() <= 1023 for p in f0 + f1)
    g0, g1 = synth.make_pair(512, 256, 8, seed=3)
    assert g0[0].dtype == np.uint8
    # the distorted frame carries the global offset (+3, -2, +2 in 8-bit units)
    d = [float(g1[c].astype(float).mean() - g0[c].astype(float).mean()) for c in range(3)]
    assert d[0] > 2.0 and d[1] < -1.0 and d[2] > 1.0


def test_config_specs():
    specs = synth.config3_specs(64, seed=3)
    assert len(specs) == 64
    assert {(s["width"], s["height"]) for s in specs} <= set(synth.CONFIG3_RESOLUTIONS)
    assert {s["bitdepth"] for s in specs} <= {8, 10} and {s["search_range"] for s in specs} <= {2, 4}
    reqs = synth.config4_requests(duration_s=0.5, rate=200.0, seed=4)
    assert 60 <= len(reqs) <= 140
    assert all(1 <= len(r.specs) <= 32 for r in reqs)
    assert all(b.arrival_s > a.arrival_s for a, b in zip(reqs, reqs[1:]))


def test_detgen_is_deterministic():
    assert hash32(np.array([0, 1, 2], np.uint32)).tolist() == [0, 1753845952, 3507691905]
    a = det_pair(64, 32, 10, 5)
    b = det_pair(64, 32, 10, 5)
    assert all(np.array_equal(x, y) for x, y in zip(a[0] + a[1], b[0] + b[1]))


def cps_fp32_exact(maxv, w, maxdiff):
    """Python statement of the kernel's exactness test (qmiv_kernels.cu, cps_fp32_exact)."""
    bias, lim = 1 << 23, 1 << 24
    e = sum(w[c] * (maxv + maxdiff[c]) ** 2 for c in range(3))
    q = sum(w[c] * maxv * maxv for c in range(3))
    up = sum(2 * w[c] * maxdiff[c] * maxv for c in range(3))
    lo = sum(2 * w[c] * (maxv + maxdiff[c]) * maxv for c in range(3))
    return bias - e >= (1 << 20) and bias + e < lim and bias + q + up < lim and bias - lo > -lim


def test_fp32_key_bound_covers_default_8_and_10_bit():
    assert cps_fp32_exact(255, (4, 1, 1), (3, 3, 3))
    assert cps_fp32_exact(1023, (4, 1, 1), (10, 10, 10))
    assert not cps_fp32_exact(4095, (4, 1, 1), (41, 41, 41))


@pytest.mark.parametrize("bd,w,g", [(8, (4, 1, 1), (3, 3, 3)), (10, (4, 1, 1), (10, 10, 10)), (10, (2, 1, 1), (10, 10, 10))])
def test_fp32_keys_order_like_int32_errors(bd, w, g):
    """Within the bound, the three-FFMA biased error is exact and its key orders candidates exactly as
    (int32 error, raster index) -- checked exhaustively over random candidates in float32 numpy."""
    rng = np.random.default_rng(bd)
    maxv = (1 << bd) - 1
    n = 20000
    s = rng.integers(-g[0], maxv + g[0] + 1, (n, 3)).astype(np.int64)
    r = rng.integers(0, maxv + 1, (n, 25, 3)).astype(np.int64)
    r[:, 7] = r[:, 3]  # force ties
    wi = np.array(w, np.int64)
    err = ((s[:, None, :] - r) ** 2 * wi).sum(-1)
    best_ref = np.argmin(err, axis=1)  # first minimum in index order
    f32 = np.float32
    q = (wi[0] * r[..., 0] ** 2 + wi[1] * r[..., 1] ** 2 + wi[2] * r[..., 2] ** 2 + (1 << 23)).astype(f32)
    a = (-2 * wi * s).astype(f32)
    e = q
    for c in range(3):
        e = (a[:, None, c] * r[..., c].astype(f32) + e).astype(f32)
    assert np.array_equal(e.astype(np.int64), err - (wi * s * s).sum(-1)[:, None] + (1 << 23))
    bits = e.view(np.uint32).astype(np.uint64)
    key = ((bits - 0x49800000) << 7) + np.arange(25, dtype=np.uint64)[None, :]
    assert np.array_equal(np.argmin(key, axis=1), best_ref)


@pytest.mark.parametrize("bd,w,g,R", [(10, (4, 1, 1), 10, 2), (8, (4, 1, 1), 3, 5), (10, (4, 1, 1), 10, 4),
                                      (9, (6, 2, 3), 5, 3)])
def test_masked_integer_keys_order_like_int32_errors(bd, w, g, R):
    """The masked search's key form: t = B + sum w r^2 + sum (-2 w s) r in uint32 is the error shifted
    by a per-pixel constant into [0, 2B]; t * 128 + raster index, with masked candidates staged as
    (0, 0, 0, 2^25 - 1), picks the reference's first strict minimum over unmasked candidates. The row-sum
    split of d^2 M into 16 low bits and the rest sums exactly in 32 bits over 32 pixels."""
    rng = np.random.default_rng(bd * 31 + R)
    maxv = (1 << bd) - 1
    D = 2 * R + 1
    n = 8000
    wi = np.array(w, np.int64)
    B = int((wi * (maxv + g) ** 2).sum())
    assert 2 * B < (1 << 25) - 1 and (maxv + g) ** 2 < (1 << 24)    # the host's condition for this form
    s = rng.integers(-g, maxv + g + 1, (n, 3)).astype(np.int64)
    r = rng.integers(0, maxv + 1, (n, D * D, 3)).astype(np.int64)
    r[:, 5] = r[:, 1]                                                  # ties
    masked = rng.random((n, D * D)) < 0.4
    masked[:, (D * D) // 2] = False                                    # the centre of a searched pixel is unmasked
    err = ((s[:, None, :] - r) ** 2 * wi).sum(-1)
    best_ref = np.argmin(np.where(masked, np.iinfo(np.int64).max, err), axis=1)   # first strict minimum
    u32 = np.uint64(0xffffffff)
    q = (B + (wi * r * r).sum(-1)).astype(np.uint64)
    a = (-2 * wi * s).astype(np.int64)
    t = q.copy()
    for c in range(3):
        t = (t + ((a[:, None, c] * r[..., c]) & 0xffffffff).astype(np.uint64)) & u32
    t = np.where(masked, np.uint64((1 << 25) - 1), t)
    real = ~masked
    assert t[real].max() <= 2 * B and np.array_equal(t[real].astype(np.int64), (err + B - (wi * s * s).sum(-1)[:, None])[real])
    key = (t * np.uint64(128) + np.arange(D * D, dtype=np.uint64)[None, :]) & u32
    assert np.array_equal(np.argmin(key, axis=1), best_ref)
    # row sums: d^2 M split into low 16 bits and the rest, each summed over 32 pixels in 32 bits
    m = rng.integers(0, 1 << 14, (n // 32, 32)).astype(np.uint64)
    d2 = rng.integers(0, (maxv + g) ** 2 + 1, (n // 32, 32)).astype(np.uint64)
    v = d2 * m
    lo = (v & np.uint64(0xffff)).sum(1)
    hi = (v >> np.uint64(16)).sum(1)
    assert lo.max() < (1 << 32) and hi.max() < (1 << 32)
    assert np.array_equal((hi << np.uint64(16)) + lo, v.sum(1))


def test_pair_difference_decomposition():
    """The mask prepass forms two sample differences from one 32-bit subtraction of 16-bit pairs below
    2^15: the low half of the word difference, sign-extended, is the low difference, and the rest
    shifted down (arithmetically) is the high one; the word difference is zero exactly when both are."""
    import numpy as np
    rng = np.random.default_rng(11)
    v = rng.integers(0, 1 << 15, size=(200000, 4), dtype=np.int64)
    v[:8] = [[0, 0, 0, 0], [0x7fff, 0, 0, 0x7fff], [0, 0x7fff, 0x7fff, 0], [5, 5, 5, 5],
             [0x7fff, 0x7fff, 0, 0], [0, 0, 0x7fff, 0x7fff], [1, 0, 0, 1], [0, 1, 1, 0]]
    w0 = v[:, 0] | (v[:, 1] << 16)
    w1 = v[:, 2] | (v[:, 3] << 16)
    dw = (w1 - w0) & 0xffffffff
    dlo = ((dw & 0xffff) ^ 0x8000) - 0x8000
    rest = (dw - dlo) & 0xffffffff
    dhi = np.where(rest >= (1 << 31), rest - (1 << 32), rest) >> 16
    assert np.array_equal(dlo, v[:, 2] - v[:, 0])
    assert np.array_equal(dhi, v[:, 3] - v[:, 1])
    assert np.array_equal(dw == 0, (v[:, 2] == v[:, 0]) & (v[:, 3] == v[:, 1]))


def test_row_sum_split_of_squared_terms():
    """The masked key search sums 32 terms d^2 M below 2^38 per row and component with 32-bit warp
    reductions: the parts from bit 11 up stay below 2^27 (their sum below 2^32) and two low 11-bit parts
    share one word (each sum below 2^16); the recombined sums are exact."""
    import numpy as np
    rng = np.random.default_rng(12)
    for _ in range(200):
        t = rng.integers(0, 1 << 38, size=(32, 2), dtype=np.uint64)
        t[rng.integers(0, 32)] = (1 << 38) - 1
        hi = (t >> np.uint64(11)).sum(axis=0)
        lo_a, lo_b = (t[:, 0] & np.uint64(0x7ff)), (t[:, 1] & np.uint64(0x7ff))
        packed = (lo_a | (lo_b << np.uint64(16))).sum()
        assert int(hi.max()) < (1 << 32) and int(packed) < (1 << 32)
        lo = [int(packed) & 0xffff, int(packed) >> 16]
        for k in range(2):
            assert (int(hi[k]) << 11) + lo[k] == int(t[:, k].sum())


def test_fast2sum_with_select_equals_twosum_and_the_reference_branch():
    """The compensated sums add the rounding error of s + v formed as (big - t) + small with the larger
    operand chosen by a compare (xKBNS.h:36-43 branches on |s| >= |v|); Knuth's TwoSum yields the same
    exactly representable error. Over mixed magnitudes, signs, ties and cancellations, both errors and
    whole ordered sums agree bit for bit (IEEE double, round to nearest)."""
    import numpy as np
    rng = np.random.default_rng(13)
    n = 20000
    s = rng.standard_normal(n) * 10.0 ** rng.integers(-12, 13, n)
    v = rng.standard_normal(n) * 10.0 ** rng.integers(-12, 13, n)
    s[:6] = [1.0, -1.0, 1e16, 0.0, 3.0, -2.5]
    v[:6] = [-1.0, 1e-16, 1.0, 0.0, 3.0, 2.5]
    t = s + v
    sb = np.abs(s) >= np.abs(v)
    big, small = np.where(sb, s, v), np.where(sb, v, s)
    e_fast = (big - t) + small
    bv = t - s
    e_two = (s - (t - bv)) + (v - bv)
    assert np.array_equal(e_fast.view(np.int64), e_two.view(np.int64))

    def kbns(vals, select):
        acc, comp = 0.0, 0.0
        for x in vals:
            tt = acc + x
            if select:
                b, sm = (acc, x) if abs(acc) >= abs(x) else (x, acc)
                comp += (b - tt) + sm
            else:
                bb = tt - acc
                comp += (acc - (tt - bb)) + (x - bb)
            acc = tt
        return acc + comp
    for k in range(20):
        vals = (rng.standard_normal(300) * 10.0 ** rng.integers(-6, 7, 300)).tolist()
        assert kbns(vals, True) == kbns(vals, False)


def test_mask_byte_count_and_or_flag():
    """Two shortcuts of the mask prepass: the non-zero bytes of a 32-bit word of four 8-bit mask samples
    are counted as popc((((m & 0x7f7f7f7f) + 0x7f7f7f7f) | m) & 0x80808080), and a picture holds a
    sample above its maximum 2^bd - 1 exactly when the OR of all its samples exceeds that maximum."""
    import numpy as np
    rng = np.random.default_rng(14)
    m = rng.integers(0, 1 << 32, size=100000, dtype=np.uint64)
    m[:5] = [0, 0x80000000, 0x00ff0001, 0xffffffff, 0x01010100]
    bits = ((((m & 0x7f7f7f7f) + 0x7f7f7f7f) | m) & 0x80808080).astype(np.uint64)
    popc = np.array([bin(int(x)).count("1") for x in bits])
    nonzero = sum(((m >> np.uint64(8 * k)) & np.uint64(0xff)) != 0 for k in range(4))
    assert np.array_equal(popc, nonzero)
    for bd in (8, 10, 12, 14):
        maxv = (1 << bd) - 1
        for _ in range(50):
            x = rng.integers(0, maxv + 1, size=rng.integers(1, 64))
            if rng.random() < 0.5:
                x[rng.integers(0, x.size)] = rng.integers(maxv + 1, 1 << 16)
            assert (np.bitwise_or.reduce(x) > maxv) == (x.max() > maxv)
