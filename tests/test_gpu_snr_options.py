"""S/N epilogue options on the GPU against the oracle (R9):

* the median / IQR z-score (the reference MatchedFilter's default
  loc_method="median", scale_method="iqr", core/filters.py:105-125 over
  stats.estimate_zscore, core/stats.py:418-502), whose order statistics the
  GPU finds by radix selection: S/N within rtol 1e-5 of the float64 oracle,
  argmax exact;
* TimeSeries.apply_boxcar (timeseries.py:296-325, stats.running_filter
  core/stats.py:200-243) against the oracle's exact-sum restatement.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-5


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available()
    return torch


def test_boxcar_snr_median_iqr(torch_cuda, orc):
    torch = torch_cuda
    from sigpyproc3_b200.search import boxcar_snr

    rng = np.random.default_rng(41)
    widths, factors = [1, 2, 3, 8, 16, 64, 256], [1, 2, 3, 4]
    rows = rng.normal(5.0, 2.0, size=(5, 20001)).astype(np.float32)
    rows[1, 7000:7040] += 3.0
    rows[4] = rows[4] * 1e-3 - 7.0  # negative values: order-preserving keys
    snr, idx = boxcar_snr(torch.from_numpy(rows).cuda(), widths=widths, factors=factors,
                          loc_scale="median_iqr")
    esnr, eidx = orc.boxcar_snr(rows, factors, widths, "median_iqr")
    np.testing.assert_allclose(snr.cpu().numpy(), esnr, rtol=RTOL)
    np.testing.assert_array_equal(idx.cpu().numpy(), eidx)
    # integer rows with many ties (the DM-time rows of integer data)
    irows = rng.integers(100, 140, size=(4, 30000)).astype(np.int32)
    irows[2, 100:300] += 25
    snr, idx = boxcar_snr(torch.from_numpy(irows).cuda(), widths=widths, factors=factors,
                          loc_scale="median_iqr")
    esnr, eidx = orc.boxcar_snr(irows.astype(np.float32), factors, widths, "median_iqr")
    np.testing.assert_allclose(snr.cpu().numpy(), esnr, rtol=RTOL)
    np.testing.assert_array_equal(idx.cpu().numpy(), eidx)


def test_boxcar_snr_median_iqr_edges(torch_cuda, orc):
    """Odd and even counts of one or two samples per factor, and a constant
    row (IQR 0: the scale falls back to 1, as np.isclose(scale, 0) does)."""
    torch = torch_cuda
    from sigpyproc3_b200.search import boxcar_snr

    rng = np.random.default_rng(42)
    for n in (1, 2, 3, 4, 9):
        rows = rng.normal(0.0, 1.0, size=(2, n)).astype(np.float32)
        rows[1] = 4.0
        facs = [f for f in (1, 2) if f <= n]
        snr, idx = boxcar_snr(torch.from_numpy(rows).cuda(), widths=[1], factors=facs,
                              loc_scale="median_iqr")
        esnr, eidx = orc.boxcar_snr(rows, facs, [1], "median_iqr")
        np.testing.assert_allclose(snr.cpu().numpy(), esnr, rtol=RTOL, atol=1e-12)
        np.testing.assert_array_equal(idx.cpu().numpy(), eidx)


def test_timeseries_snr_loc_scale(torch_cuda, orc):
    from sigpyproc3_b200 import Header, TimeSeries

    x = np.random.default_rng(43).normal(0, 1, 12345).astype(np.float32)
    ts = TimeSeries(x, Header(nchans=1, nsamples=x.size))
    for ls in ("mean_std", "median_iqr"):
        esnr, _ = orc.boxcar_snr(x, (1,), (1, 2, 4), ls)
        np.testing.assert_allclose(ts.snr(widths=(1, 2, 4), loc_scale=ls), esnr[0], rtol=RTOL)
    with pytest.raises(ValueError):
        ts.snr(loc_scale="mad")


@pytest.mark.parametrize("n,width", [(10007, 1), (10007, 2), (10007, 5), (10007, 8),
                                     (10007, 33), (10007, 256), (70000, 101), (5, 12),
                                     (1, 3)])
def test_apply_boxcar(torch_cuda, orc, n, width):
    from sigpyproc3_b200 import Header, TimeSeries

    x = np.random.default_rng(n + width).normal(0.5, 2.0, n).astype(np.float32)
    ts = TimeSeries(x, Header(nchans=1, nsamples=n))
    out = ts.apply_boxcar(width)
    assert out.nsamples == n
    np.testing.assert_allclose(out.data, orc.apply_boxcar(x, width), rtol=1e-6, atol=1e-9)


def test_apply_boxcar_errors(torch_cuda):
    from sigpyproc3_b200 import Header, TimeSeries

    ts = TimeSeries(np.zeros(10, np.float32), Header(nchans=1, nsamples=10))
    with pytest.raises(ValueError):
        ts.apply_boxcar(0)
