"""MatchedFilter on the GPU (next row N3: core/filters.py:29-365 with
kernels.convolve_templates core/kernels.py:861-906) against the oracle's
restatement (float64 FFT correlation over the series repeated to pocketfft's
good length).  The reference computes the same correlation with rocket_fft,
absent here: its own outputs are not pinned, its template bank and z-score
are (tests/test_host.py, tests/test_oracle_golden.py)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available()
    return torch


@pytest.mark.parametrize("kind", ["boxcar", "gaussian", "lorentzian"])
@pytest.mark.parametrize("loc,scale", [("median", "iqr"), ("mean", "std"), ("median", "std"),
                                       ("norm", "norm"), ("median", "mad"), ("mean", "mad")])
def test_matched_filter_vs_oracle(torch_cuda, orc, kind, loc, scale):
    from sigpyproc3_b200.filters import MatchedFilter

    rng = np.random.default_rng(len(kind) * 100 + len(loc) * 10 + len(scale))
    n = 6007
    x = rng.normal(10.0, 2.0, n).astype(np.float32)
    x[3000:3012] += 6.0 * np.hanning(12).astype(np.float32)
    mf = MatchedFilter(x, loc_method=loc, scale_method=scale, temp_kind=kind)
    z, convs, itemp, peak, snr = orc.matched_filter(x, loc, scale, kind)
    np.testing.assert_array_equal(mf.zscores.data, z)  # same float32 rounding
    assert mf.convs.shape == convs.shape
    np.testing.assert_allclose(mf.convs, convs, rtol=1e-5, atol=1e-5)
    assert (mf.best_temp.kind, mf.peak_bin) == (kind, peak)
    assert mf.temp_bank.index(mf.best_temp) == itemp
    assert mf.snr == pytest.approx(snr, rel=1e-5)
    lo, hi = mf.on_pulse
    assert lo <= peak <= hi
    assert mf.best_model.shape == (n,)


def test_matched_filter_edges(torch_cuda, orc):
    from sigpyproc3_b200.filters import MatchedFilter

    # a series shorter than the FFT length rule's smallest padding, and one whose
    # good length differs from n (13 -> 15)
    for n in (13, 40, 97):
        x = np.random.default_rng(n).normal(0, 1, n).astype(np.float32)
        mf = MatchedFilter(x, temp_kind="boxcar", nbins_max=8)
        _, convs, itemp, peak, snr = orc.matched_filter(x, "median", "iqr", "boxcar", 8)
        np.testing.assert_allclose(mf.convs, convs, rtol=1e-5, atol=1e-5)
        assert (mf.peak_bin, mf.temp_bank.index(mf.best_temp)) == (peak, itemp)
    with pytest.raises(ValueError):
        MatchedFilter(np.zeros(10, np.float32), temp_kind="gaussian", nbins_max=32)
    with pytest.raises(ValueError):
        MatchedFilter(np.zeros((2, 10), np.float32))


def test_row_loc_scale_mad_matches_reference(torch_cuda, golden, golden_meta):
    """spp_row_loc_scale method 2 on the recorded series: the float32 median
    and the reference's own stats._scale_mad values (golden) -- exact order
    statistics, so equal to the last bit; the mean-absolute-deviation branch
    (MAD 0) sums in another order than numpy, so within 1e-12 there."""
    torch = torch_cuda
    from sigpyproc3_b200 import _lib

    lib = _lib.load()
    for k, rec in enumerate(golden_meta["zscore"]):
        y = torch.from_numpy(golden[f"zscore_in_{k}"]).cuda()
        ls = torch.empty(2, dtype=torch.float64, device="cuda")
        _lib.check(lib.spp_row_loc_scale(y.data_ptr(), _lib.OUT_F32, 1, y.numel(), y.numel(), 2,
                                         ls.data_ptr(), torch.cuda.current_stream().cuda_stream))
        loc, scale = ls.cpu().numpy()
        assert loc == rec["median"], (k, loc, rec)
        expect = rec["mad_scale"] if not np.isclose(rec["mad_scale"], 0) else 1.0
        d = golden[f"zscore_in_{k}"].astype(np.float64)
        if np.isclose(np.median(np.abs(d - np.median(d))), 0) and expect != 1.0:
            assert scale == pytest.approx(expect, rel=1e-12), (k, scale, rec)
        else:
            assert scale == expect, (k, scale, rec)
