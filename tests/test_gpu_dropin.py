"""The reference-facing API on the GPU (R1, R3, R5, R7-R11) against the
golden vectors and the oracle."""

import hashlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available()
    return torch


def _pack(vals, nbits, order):
    per = 8 // nbits
    v = vals.reshape(-1, per).astype(np.uint8)
    out = np.zeros(v.shape[0], dtype=np.uint8)
    for k in range(per):
        sh = (8 - (k + 1) * nbits) if order == "big" else k * nbits
        out |= (v[:, k] << sh).astype(np.uint8)
    return out


def _oracle_filterbank_dedisperse(orc, vals, nchans, nsamples, delays, gulp, start=0, nsamps=None):
    """Filterbank.dedisperse (base.py:400-424) restated with the oracle kernel."""
    from sigpyproc3_b200.readers import plan_blocks

    maxd = int(np.abs(delays).max())
    gulp = max(2 * maxd, gulp)
    tim = np.zeros(nsamples - maxd, np.float32)
    g, blocks = plan_blocks(nsamples, gulp, start, nsamps, maxd)
    pos = start
    for ii, nblk, skip in blocks:
        blk = vals[pos * nchans:(pos + nblk) * nchans]
        orc.dedisperse(blk, delays, nchans, nblk, out=tim, out_start=ii * (g - maxd))
        pos += nblk + skip
    return tim


def test_c1_dedisperse_bit_exact(torch_cuda, golden, golden_meta):
    from sigpyproc3_b200 import ArrayFilterbank, Header, synth

    raw = synth.c1_filterbank(1)
    assert sha(raw) == golden_meta["c1_input_sha256"]
    g = synth.C1
    h = Header(nchans=g.nchans, fch1=g.fch1, foff=g.foff, tsamp=g.tsamp, nbits=8,
               nsamples=g.nsamps)
    tim = ArrayFilterbank(raw, h).dedisperse(100.0)
    assert tim.header.dm == 100.0 and tim.header.nchans == 1
    assert tim.data.dtype == np.float32
    np.testing.assert_array_equal(tim.data, golden["c1_tim"])
    # the injected pulse is at sample 30000 at fch1
    assert abs(int(np.argmax(tim.data)) - 30000) <= 2


@pytest.mark.parametrize("nbits", [1, 2, 4, 8, 32])
@pytest.mark.parametrize("ref", ["fch1", "fcenter"])
def test_filreader_dedisperse(torch_cuda, orc, tmp_path, nbits, ref):
    from sigpyproc3_b200 import FilReader, Header

    rng = np.random.default_rng(100 + nbits)
    nchans, nsamples = 64, 6000
    h = Header(nchans=nchans, fch1=1510.0, foff=-1.09, tsamp=320e-6, nbits=nbits)
    if nbits == 32:
        vals = rng.normal(0, 1, nsamples * nchans).astype(np.float32)
        raw = vals
    else:
        vals = rng.integers(0, 1 << nbits, nsamples * nchans, dtype=np.uint8)
        order = "little" if nbits == 1 else "big"
        raw = vals if nbits == 8 else _pack(vals, nbits, order)
    p = tmp_path / f"x{nbits}.fil"
    h.write_sigproc(p, raw)
    fil = FilReader(p)
    assert fil.header.nsamples == nsamples
    dm = 60.0
    d = np.atleast_1d(fil.header.get_dmdelays(dm, ref)).astype(np.int32)
    tim = fil.dedisperse(dm, ref_freq=ref, gulp=700)
    expect = _oracle_filterbank_dedisperse(orc, vals, nchans, nsamples, d, 700)
    if nbits == 32:
        np.testing.assert_allclose(tim.data, expect, rtol=1e-5, atol=1e-6)
    else:
        np.testing.assert_array_equal(tim.data, expect)


def test_filreader_multifile_and_start(torch_cuda, orc, tmp_path):
    from sigpyproc3_b200 import FilReader, Header

    rng = np.random.default_rng(7)
    nchans, n1, n2 = 32, 3000, 2500
    h = Header(nchans=nchans, fch1=1400.0, foff=-2.0, tsamp=256e-6, nbits=8)
    a = rng.integers(0, 256, n1 * nchans, dtype=np.uint8)
    b = rng.integers(0, 256, n2 * nchans, dtype=np.uint8)
    h.write_sigproc(tmp_path / "a.fil", a)
    h.write_sigproc(tmp_path / "b.fil", b)
    fil = FilReader([tmp_path / "a.fil", tmp_path / "b.fil"])
    assert fil.header.nsamples == n1 + n2
    vals = np.concatenate([a, b])
    d = np.atleast_1d(fil.header.get_dmdelays(30.0)).astype(np.int32)
    tim = fil.dedisperse(30.0, gulp=1000, start=100, nsamps=4000)
    expect = _oracle_filterbank_dedisperse(orc, vals, nchans, n1 + n2, d, 1000, 100, 4000)
    np.testing.assert_array_equal(tim.data, expect)


def test_read_plan_matches_reference_bytes(torch_cuda, golden_meta):
    from sigpyproc3_b200 import ArrayFilterbank, Header

    for case in golden_meta["read_plan"]:
        nsamples, nchans, gulp, start, nsamps, skip = case["args"]
        if case["error"] is not None:
            continue
        raw = (np.arange(nsamples * nchans) % 251).astype(np.uint8)
        fb = ArrayFilterbank(raw, Header(nchans=nchans, nbits=8, nsamples=nsamples))
        got = [[n, ii, sha(data)] for n, ii, data in
               fb.read_plan(gulp=gulp, start=start, nsamps=nsamps, skipback=skip)]
        assert got == [[b[0], b[1], b[3]] for b in case["blocks"]]


def test_read_plan_unpacks_and_errors(torch_cuda, orc):
    from sigpyproc3_b200 import ArrayFilterbank, Header

    rng = np.random.default_rng(3)
    vals = rng.integers(0, 4, 64 * 1000, dtype=np.uint8)
    fb = ArrayFilterbank(_pack(vals, 2, "big"), Header(nchans=64, nbits=2, nsamples=1000))
    blocks = list(fb.read_plan(gulp=300))
    np.testing.assert_array_equal(np.concatenate([b[2] for b in blocks]), vals)
    with pytest.raises(ValueError, match="must be > skipback"):
        list(fb.read_plan(gulp=512, nsamps=1024, skipback=1024))
    short = ArrayFilterbank(_pack(vals, 2, "big")[:-100], Header(nchans=64, nbits=2, nsamples=1000))
    with pytest.raises(ValueError, match="Unexpected number of bytes"):
        list(short.read_plan(gulp=512))


def test_dedisperse_batch(torch_cuda, orc):
    torch = torch_cuda
    from sigpyproc3_b200 import ArrayFilterbank, Header

    rng = np.random.default_rng(11)
    nchans, nsamples = 128, 20000
    vals = rng.integers(0, 4, nsamples * nchans, dtype=np.uint8)
    h = Header(nchans=nchans, fch1=1500.0, foff=-0.5, tsamp=64e-6, nbits=2, nsamples=nsamples)
    fb = ArrayFilterbank(_pack(vals, 2, "big"), h)
    out, dms = fb.dedisperse_batch(dm=100.0, dmsteps=37, gulp=5000)
    d = np.atleast_2d(h.get_dmdelays(dms)).astype(np.int32)
    nvalid = nsamples - int(d.max())
    assert out.dtype == torch.int32 and out.shape == (37, nvalid)
    np.testing.assert_array_equal(out.cpu().numpy(), orc.dmt(vals, d, nchans, nsamples, nvalid))


def test_block_dmt_transform_and_dedisperse(torch_cuda, golden):
    from sigpyproc3_b200 import FilterbankBlock, Header

    blk = golden["dmt_block_in"]
    h = Header(nchans=32, fch1=1400.0, foff=-2.0, tsamp=256e-6, nsamples=512)
    fb = FilterbankBlock(blk, h)
    dmt = fb.dmt_transform(10.0, 16)
    assert dmt.ndms == 16 and dmt.nsamples == 512
    np.testing.assert_allclose(dmt.data, golden["dmt_block_out"], rtol=1e-5, atol=1e-5)
    # FilterbankBlock.dedisperse direction (test_blocks.py:100-132 pattern)
    data = np.zeros((32, 512), np.float32)
    data[:, 256] = 1.0
    b = FilterbankBlock(data, h)
    dd = b.dedisperse(50.0)
    assert dd.data[:, 257:].sum() == 0
    np.testing.assert_array_equal(dd.data.mean(1), data.mean(1))
    vv = b.dedisperse(50.0, only_valid_samples=True)
    assert vv.nsamples == 512 - h.get_dmdelays(50.0).max()


def test_bandpass_collapse_zero_dm(torch_cuda, golden, orc):
    torch = torch_cuda
    from sigpyproc3_b200 import ArrayFilterbank, Header, _lib

    x = golden["ded_u8_in"]
    fb = ArrayFilterbank(x, Header(nchans=64, nbits=8, nsamples=4096))
    np.testing.assert_array_equal(fb.bandpass(gulp=1000).data, golden["bpass_u8"])  # bit-exact
    np.testing.assert_array_equal(fb.collapse(gulp=4096).data, golden["collapse_u8"])
    zf = golden["zdm_in"]
    fz = ArrayFilterbank(zf, Header(nchans=48, nbits=32, nsamples=1024))
    bp = fz.bandpass(gulp=300).data
    np.testing.assert_array_equal(bp, golden["zdm_bpass"])
    chanwts = (bp / bp.sum()).astype(np.float32)
    xin = torch.from_numpy(zf.ravel()).cuda()
    out = torch.empty_like(xin)
    bp_d = torch.from_numpy(bp).cuda()
    w_d = torch.from_numpy(chanwts).cuda()
    _lib.call("spp_zero_dm", xin.data_ptr(), out.data_ptr(), 48, 1024, bp_d.data_ptr(),
              w_d.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    # the reference (fastmath) may contract the multiply-add: 1 ulp of the output
    np.testing.assert_allclose(out.cpu().numpy().reshape(1024, 48), golden["zdm_out"],
                               rtol=1e-6, atol=1e-5)
    # the oracle adds each spectrum's channels in order, as the reference loop
    # is written, and rounds each operation: identical bits
    np.testing.assert_array_equal(out.cpu().numpy(), orc.zero_dm(zf.ravel(), 48, 1024, bp))


def test_subband_stage1(torch_cuda, golden):
    torch = torch_cuda
    from sigpyproc3_b200 import _lib

    x = torch.from_numpy(golden["subband_in"].ravel()).cuda()
    d = golden["subband_delays"]
    maxd = int(np.abs(d).max())
    c2s = torch.from_numpy((np.arange(64) // 8).astype(np.int32)).cuda()
    out = torch.empty((2048 - maxd) * 8, dtype=torch.float32, device="cuda")
    d_d = torch.from_numpy(d).cuda()
    _lib.call("spp_subband", x.data_ptr(), 8, 0, 64, 2048, d_d.data_ptr(),
              maxd, c2s.data_ptr(), 8, out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    np.testing.assert_array_equal(out.cpu().numpy(), golden["subband_out"])


@pytest.mark.parametrize("f", [1, 2, 4, 7])
def test_timeseries_downsample(torch_cuda, golden, f):
    from sigpyproc3_b200 import Header, TimeSeries

    ts = TimeSeries(golden["ds_in"], Header(nchans=1, nsamples=golden["ds_in"].size))
    np.testing.assert_array_equal(ts.downsample(f).data, golden[f"ds_out_{f}"])


def test_boxcar_snr(torch_cuda, orc):
    torch = torch_cuda
    from sigpyproc3_b200.search import boxcar_snr

    rng = np.random.default_rng(4)
    rows = rng.normal(0, 1, size=(7, 9000)).astype(np.float32)
    rows[3, 4000:4032] += 2.0
    widths, factors = [1, 2, 4, 8, 16, 32, 64, 256], [1, 2, 4]
    snr, idx = boxcar_snr(torch.from_numpy(rows).cuda(), widths=widths, factors=factors)
    esnr, eidx = orc.boxcar_snr(rows, factors, widths)
    np.testing.assert_allclose(snr.cpu().numpy(), esnr, rtol=1e-5)
    np.testing.assert_array_equal(idx.cpu().numpy(), eidx)
    # integer rows (exact sums)
    irows = rng.integers(0, 1000, size=(3, 5000)).astype(np.int32)
    snr, idx = boxcar_snr(torch.from_numpy(irows).cuda(), widths=widths, factors=factors)
    esnr, eidx = orc.boxcar_snr(irows.astype(np.float32), factors, widths)
    np.testing.assert_allclose(snr.cpu().numpy(), esnr, rtol=1e-5)
    np.testing.assert_array_equal(idx.cpu().numpy(), eidx)
