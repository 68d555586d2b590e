"""The CPU oracle against golden vectors produced by the reference's own code
(tests/golden/make_golden.py).  This pins the oracle before it checks the GPU."""

import hashlib

import numpy as np
import pytest


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("nbits", [1, 2, 4])
@pytest.mark.parametrize("order", ["big", "little"])
def test_unpack(orc, golden, nbits, order):
    # reference KAT (tests/test_kernels.py:9-41 input [7, 23]) and a random array
    kat = orc.unpack(np.array([7, 23], np.uint8), nbits, order)
    np.testing.assert_array_equal(kat, golden[f"unpack_kat_{nbits}_{order}"])
    rnd = orc.unpack(golden["unpack_rand_in"], nbits, order)
    np.testing.assert_array_equal(rnd, golden[f"unpack_rand_{nbits}_{order}"])


@pytest.mark.parametrize("tag", ["dm50", "dm200", "dm120_fcenter"])
def test_dedisperse_u8(orc, golden, tag):
    x = golden["ded_u8_in"]
    d = golden[f"ded_u8_{tag}_delays"]
    out = orc.dedisperse(x.ravel(), d, 64, 4096)
    np.testing.assert_array_equal(out, golden[f"ded_u8_{tag}_out"])  # bit-exact


def test_dedisperse_f32(orc, golden):
    x = golden["ded_f32_in"]
    out = orc.dedisperse(x.ravel(), golden["ded_f32_delays"], 32, 2048)
    # reference uses fastmath (may reassociate the f64 sum): float32 results agree
    np.testing.assert_allclose(out, golden["ded_f32_out"], rtol=1e-6, atol=1e-6)


def test_c1_full(orc, golden, golden_meta):
    from sigpyproc3_b200 import synth

    raw = synth.c1_filterbank(1)
    assert sha(raw) == golden_meta["c1_input_sha256"]
    out = orc.dedisperse(raw, golden["c1_delays"], 256, 65536)
    np.testing.assert_array_equal(out, golden["c1_tim"])


def test_dmt_roll(orc, golden):
    blk = golden["dmt_block_in"]  # (nchans, nsamps)
    d = golden["dmt_block_delays"].astype(np.int32)
    out = orc.dmt_roll(blk.T.copy(), d, 32, 512)
    np.testing.assert_allclose(out, golden["dmt_block_out"], rtol=1e-5, atol=1e-5)
    out_i = orc.dmt_roll(golden["dmt_block_int_in"].T.copy(), d, 32, 512)
    np.testing.assert_array_equal(out_i, golden["dmt_block_int_out"])


def test_dmt_rowwise_matches_dedisperse(orc, golden):
    x = golden["ded_u8_in"]
    d = np.stack([golden["ded_u8_dm50_delays"], golden["ded_u8_dm200_delays"]])
    nvalid = 4096 - int(np.abs(d).max())
    out = orc.dmt(x.ravel(), d, 64, 4096, nvalid)
    np.testing.assert_array_equal(out[0], golden["ded_u8_dm50_out"][:nvalid])
    np.testing.assert_array_equal(out[1], golden["ded_u8_dm200_out"][:nvalid])


def test_dmt_packed(orc, golden):
    rnd = golden["unpack_rand_in"]  # 4096 bytes = 2-bit, 64 ch x 256 samples
    d = np.stack([golden["ded_u8_dm50_delays"] % 50])
    un = golden["unpack_rand_2_big"]
    nvalid = 256 - int(d.max())
    a = orc.dmt_packed(rnd, 2, "big", d, 64, 256, nvalid)
    b = orc.dmt(un, d, 64, 256, nvalid)
    np.testing.assert_array_equal(a, b)


def test_subband(orc, golden):
    x = golden["subband_in"]
    d = golden["subband_delays"]
    c2s = (np.arange(64) // 8).astype(np.int32)
    out = orc.subband(x.ravel(), d, c2s, int(np.abs(d).max()), 64, 8, 2048)
    np.testing.assert_array_equal(out, golden["subband_out"])


def test_bandpass_collapse(orc, golden):
    x = golden["ded_u8_in"]
    np.testing.assert_array_equal(orc.bandpass(x.ravel(), 64, 4096), golden["bpass_u8"])
    zf = golden["zdm_in"]
    np.testing.assert_array_equal(orc.bandpass(zf.ravel(), 48, 1024), golden["zdm_bpass"])


def test_zero_dm(orc, golden):
    out = orc.zero_dm(golden["zdm_in"].ravel(), 48, 1024, golden["zdm_bpass"])
    np.testing.assert_allclose(out.reshape(1024, 48), golden["zdm_out"], rtol=1e-6, atol=1e-5)


@pytest.mark.parametrize("f", [1, 2, 4, 7])
def test_downsample(orc, golden, f):
    np.testing.assert_array_equal(orc.downsample_mean(golden["ds_in"], f), golden[f"ds_out_{f}"])


def test_boxcar_snr_small(orc):
    rng = np.random.default_rng(3)
    x = rng.normal(0, 1, 1000).astype(np.float32)
    x[500:508] += 3.0
    snr, idx = orc.boxcar_snr(x, [1, 2], [1, 8])
    # brute-force check in float64
    for fi, f in enumerate([1, 2]):
        y = orc.downsample_mean(x, f).astype(np.float64)
        mu, sd = y.mean(), y.std()
        for wi, w in enumerate([1, 8]):
            s = np.array([y[t:t + w].sum() for t in range(y.size - w + 1)])
            assert idx[0, fi, wi] == int(np.argmax(s))
            assert np.isclose(snr[0, fi, wi], (s.max() - w * mu) / (sd * np.sqrt(w)), rtol=1e-12)


@pytest.mark.parametrize("tag", ["a", "b", "c"])
def test_fold(orc, golden, golden_meta, fold_input, tag):
    """kernels.fold through Filterbank.fold's block loop, against the reference's
    own output: sums, counts and the divided cube, bit for bit."""
    case = next(c for c in golden_meta["fold_cases"] if c["tag"] == tag)
    data = fold_input(case)
    freqs = orc.chan_freqs(case["nchans"], case["fch1"], case["foff"])
    d = np.atleast_1d(orc.dmdelays(freqs, case["dm"], case["tsamp"], case["fch1"])).astype(np.int32)
    sums, counts, cube = orc.filterbank_fold(
        data, case["nsamples"], case["nchans"], d, case["tsamp"], case["period"], case["accel"],
        case["nbins"], case["nints"], case["nbands"], case["gulp"])
    np.testing.assert_array_equal(counts, golden[f"fold_{tag}_count"])
    np.testing.assert_array_equal(sums, golden[f"fold_{tag}_sum"])
    np.testing.assert_array_equal(cube, golden[f"fold_{tag}_cube"])


def test_py_floordiv_matches_python(orc):
    """The restated float floor division (fold's subintegration and subband
    indices) equals Python's own // -- random operands and quotients that land
    on or next to integers."""
    import math

    rng = np.random.default_rng(41)
    a = np.concatenate([rng.integers(0, 2**31, 2000).astype(np.float64),
                        rng.normal(0, 1e6, 2000), np.arange(0, 5000, dtype=np.float64)])
    b = np.concatenate([rng.uniform(0.1, 5000.0, 2000), rng.normal(0, 100.0, 2000),
                        np.full(5000, 65536 / 31), ])
    b[b == 0] = 1.0
    extra = [(7.0, 0.1), (1.0, 0.1), (0.3, 0.1), (-7.0, 0.1), (6.0, 0.2), (65535.0, 65536 / 32),
             (12000.0, 12000 / 7), (9000.0 - 1, 9000 / 7), (5.0, -2.0), (-5.0, 2.0), (0.0, 3.0)]
    for x, y in list(zip(a, b)) + extra:
        got = orc.lib().orc_py_floordiv(float(x), float(y))
        want = float(x) // float(y)
        assert got == want and math.copysign(1, got) == math.copysign(1, want), (x, y, got, want)


def test_robust_zscore_matches_reference(orc, golden, golden_meta):
    """median / IQR scale of the oracle equal np.median and the reference's
    stats._scale_iqr (core/stats.py:480-502) on the recorded series."""
    for k, rec in enumerate(golden_meta["zscore"]):
        y = golden[f"zscore_in_{k}"]
        loc, scale = orc.median_iqr(y)
        assert loc == rec["median"], (k, loc, rec)
        expect = rec["iqr_scale"] if not np.isclose(rec["iqr_scale"], 0) else 1.0
        assert scale == expect, (k, scale, rec)


def test_mad_scale_matches_reference(orc, golden, golden_meta):
    """The oracle's MAD scale equals the reference's stats._scale_mad
    (core/stats.py:505-536) on the recorded series, including those whose MAD
    is 0 (mean absolute deviation instead)."""
    zero = 0
    for k, rec in enumerate(golden_meta["zscore"]):
        y = golden[f"zscore_in_{k}"]
        assert orc.mad_scale(y) == rec["mad_scale"], (k, rec)
        d = y.astype(np.float64)
        zero += bool(np.isclose(np.median(np.abs(d - np.median(d))), 0) and rec["mad_scale"] > 0)
    assert zero >= 1  # a non-zero mean absolute deviation is among the cases


def test_boxcar_snr_loc_scale_options(orc):
    """The S/N oracle's two z-scores: mean/std and median/IQR."""
    rng = np.random.default_rng(3)
    x = rng.normal(10.0, 3.0, 5000).astype(np.float32)
    x[2000:2010] += 20.0
    s1, i1, l1, c1 = orc.boxcar_snr(x, (1, 2), (1, 4, 16), return_loc_scale=True)
    s2, i2, l2, c2 = orc.boxcar_snr(x, (1, 2), (1, 4, 16), "median_iqr", return_loc_scale=True)
    assert l1[0, 0] == pytest.approx(float(np.mean(x, dtype=np.float64)))
    assert l2[0, 0] == float(np.median(x))
    y2 = orc.downsample_mean(x, 2)
    assert l2[0, 1] == float(np.median(y2))
    q = np.percentile(y2.astype(np.float64), [25, 75])
    assert c2[0, 1] == float((q[1] - q[0]) / 1.3489795003921634)
    assert np.all(i1 == i2)  # same windows win; only the normalisation differs
    assert np.all(s2 > 0) and np.all(s1 > 0)
