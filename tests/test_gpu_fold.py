"""Filterbank.fold on the GPU (spp_fold, kernels.fold core/kernels.py:403-445
via base.py:1109-1207) against the reference's own folded cubes and the
oracle."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available()
    return torch


def _fb(data, case, nbits):
    from sigpyproc3_b200 import ArrayFilterbank, Header

    h = Header(nchans=case["nchans"], fch1=case["fch1"], foff=case["foff"], tsamp=case["tsamp"],
               nbits=nbits, nsamples=case["nsamples"])
    return ArrayFilterbank(np.ascontiguousarray(data).view(np.uint8), h)


@pytest.mark.parametrize("tag", ["a", "b", "c"])
def test_fold_matches_reference(torch_cuda, golden, golden_meta, fold_input, tag):
    case = next(c for c in golden_meta["fold_cases"] if c["tag"] == tag)
    data = fold_input(case)
    nbits = 8 if case["dtype"] == "uint8" else 32
    fd = _fb(data, case, nbits).fold(case["period"], case["dm"], case["accel"], case["nbins"],
                                      case["nints"], case["nbands"], case["gulp"])
    ref = golden[f"fold_{tag}_cube"]
    assert fd.data.shape == ref.shape
    if nbits == 8:
        # integer sums: bit-identical to the reference's float32 cells
        np.testing.assert_array_equal(fd.data, ref)
    else:
        # float32 sums in another order: means within float32 rounding of the sums
        np.testing.assert_allclose(fd.data, ref, rtol=1e-5, atol=1e-6)
    assert fd.period == case["period"] and fd.dm == case["dm"]


def test_fold_packed_and_ascending_band(torch_cuda, orc):
    """2-bit packed data (unpacked on the device) and an ascending band (negative
    delays: rows before the block wrap to its end, as numba's indexing)."""
    rng = np.random.default_rng(31)
    for foff, nbits in ((-1.09, 2), (1.09, 8)):
        case = {"nchans": 64, "fch1": 1400.0, "foff": foff, "tsamp": 320e-6, "nsamples": 7000}
        vals = rng.integers(0, 1 << nbits, size=7000 * 64, dtype=np.uint8)
        if nbits == 2:
            v = vals.reshape(-1, 4)
            raw = ((v[:, 0] << 6) | (v[:, 1] << 4) | (v[:, 2] << 2) | v[:, 3]).astype(np.uint8)
        else:
            raw = vals
        fb = _fb(raw, case, nbits)
        fd = fb.fold(0.0271, 30.0, 2.0, 31, 6, 7, 1500)
        d = np.atleast_1d(fb.header.get_dmdelays(30.0)).astype(np.int32)
        _, _, cube = orc.filterbank_fold(vals, 7000, 64, d, 320e-6, 0.0271, 2.0, 31, 6, 7, 1500)
        np.testing.assert_array_equal(fd.data, cube)


def test_fold_rejects_too_many_cells(torch_cuda):
    case = {"nchans": 16, "fch1": 1400.0, "foff": -1.0, "tsamp": 1e-3, "nsamples": 1000}
    fb = _fb(np.zeros(1000 * 16, np.uint8), case, 8)
    with pytest.raises(ValueError):
        fb.fold(0.05, 1.0, nbins=50, nints=32, nbands=16)


def test_fold_8bit_cells_past_2e24_exact_and_deterministic(torch_cuda):
    """Cells whose totals pass 2^24 (constant 255 samples, one band, four bins:
    ~4e5 adds of 255 per cell) stay exact: the cube is 255 to float32 rounding
    and two runs agree bit for bit."""
    case = {"nchans": 64, "fch1": 1400.0, "foff": -1.0, "tsamp": 1e-3, "nsamples": 1 << 15}
    fb = _fb(np.full((1 << 15) * 64, 255, np.uint8), case, 8)
    a = fb.fold(0.0173, 5.0, nbins=4, nints=1, nbands=1, gulp=4096)
    b = fb.fold(0.0173, 5.0, nbins=4, nints=1, nbands=1, gulp=4096)
    np.testing.assert_array_equal(a.data, b.data)
    np.testing.assert_allclose(a.data, 255.0, rtol=2.0**-23)


def test_fold_float32_long_block(torch_cuda, orc):
    """Float32 cells fold with atomic adds in arrival order; against the
    oracle's sequential float32 cells the means agree within the rounding of
    the adds (relative 2^-24 per add into a cell, positive samples)."""
    rng = np.random.default_rng(77)
    n, nch = 60000, 32
    case = {"nchans": nch, "fch1": 1400.0, "foff": -2.0, "tsamp": 5e-4, "nsamples": n}
    vals = rng.normal(5.0, 1.0, n * nch).astype(np.float32)
    fb = _fb(vals, case, 32)
    fd = fb.fold(0.0311, 20.0, nbins=16, nints=4, nbands=4, gulp=8000)
    d = np.atleast_1d(fb.header.get_dmdelays(20.0)).astype(np.int32)
    sums, counts, cube = orc.filterbank_fold(vals, n, nch, d, 5e-4, 0.0311, 0.0, 16, 4, 4, 8000)
    adds = counts.ravel() / (nch // 4)  # one atomic add per (sample, band) into a cell
    got, ref = fd.data.ravel().astype(np.float64), cube.ravel().astype(np.float64)
    np.testing.assert_array_less(np.abs(got - ref), 2.0 * adds * 2.0**-24 * np.abs(ref) + 1e-30)
