"""PulseExtractor (readers.py:353-478) and FilterbankBlock.pad_samples
(block.py:108-146): the window arithmetic and median/mean padding restated
with numpy, against the GPU reader on a written sigproc file."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available()
    return torch


def _expected(raw, nsamples, nchans, fch1, foff, tsamp, toa, width, dm, min_nsamps, toa_freq,
              sub_nchans, pad_mode, orc):
    toa_freq = toa_freq or fch1
    sub_nchans = sub_nchans or nchans
    freqs = orc.chan_freqs(sub_nchans, toa_freq, foff)
    delays = np.atleast_1d(orc.dmdelays(freqs, dm, tsamp, toa_freq))
    disp = int(np.max(np.abs(delays))) + width * 5
    tdec = max(1, width // 2)
    bdel = ((disp // tdec) + 1) * tdec
    n = max(2 * bdel, min_nsamps * tdec)
    nstart = toa - n // 2
    s0 = max(0, nstart)
    ns = min(n + min(0, nstart), nsamples - max(0, nstart))
    c0 = int((toa_freq - fch1) / foff)
    blk = raw.reshape(nsamples, nchans)[s0:s0 + ns, c0:c0 + sub_nchans].T.astype(np.float32)
    if nstart < 0 or nstart + n > nsamples:
        pad = getattr(np, pad_mode)(blk, axis=1)
        out = np.ones((sub_nchans, n), dtype=np.float32)
        out *= pad[:, None]
        off = abs(min(0, nstart))
        out[:, off:off + blk.shape[1]] = blk
        blk = out
    return blk, n


@pytest.mark.parametrize("toa,toa_freq,sub,pad", [
    (3000, None, None, "median"),      # well inside the file
    (40, None, None, "median"),        # starts before the file: padded at the front
    (5950, 1480.0, 16, "mean"),        # runs past the end, a channel subset
])
def test_pulse_extractor(torch_cuda, orc, tmp_path, toa, toa_freq, sub, pad):
    from sigpyproc3_b200 import Header
    from sigpyproc3_b200.readers import PulseExtractor

    nsamples, nchans, fch1, foff, tsamp = 6000, 64, 1510.0, -1.0, 320e-6
    rng = np.random.default_rng(toa)
    raw = rng.integers(0, 256, size=nsamples * nchans, dtype=np.uint8)
    h = Header(nchans=nchans, fch1=fch1, foff=foff, tsamp=tsamp, nbits=8, nsamples=nsamples)
    path = tmp_path / "pulse.fil"
    h.write_sigproc(path, raw)
    pe = PulseExtractor(str(path), toa, 8, 30.0, min_nsamps=64, toa_freq=toa_freq, nchans=sub)
    blk = pe.get_data(pad_mode=pad)
    exp, n = _expected(raw, nsamples, nchans, fch1, foff, tsamp, toa, 8, 30.0, 64, toa_freq, sub,
                       pad, orc)
    assert pe.nsamps == n and blk.header.nsamples == n
    np.testing.assert_array_equal(blk.data, exp)
    assert pe.pulse_toa_block == toa - pe.nstart
    with pytest.raises(ValueError):
        blk.pad_samples(n + 4, 0, pad_mode="max")
