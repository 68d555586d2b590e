"""DM-batch parity at the headline geometry: 4096 channels, the
dmt_transform(1000, 1024) trial grid (DM 0-2000, max delay 32 402 samples),
a window of output samples plus the maximum delay, bit-exact against the
oracle's row-wise restatement of kernels.dedisperse
(src/sigpyproc/core/kernels.py:340-362).

The small-channel tests elsewhere keep every sum below 512; these reach the
upper levels of the bit-sliced counters (1- and 2-bit sums up to 3 x 4096 =
12 288, bit 13), the 8-bit SIMD lanes' periodic widening (sums up to
255 x 4096) and the tile spreads of config 2 (about 222 samples across 8
adjacent trials at the bottom of the band)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NCHANS = 4096
WINDOW = 1 << 16


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available(), "GPU tests need CUDA"
    return torch


def _pack(vals, nbits, order):
    per = 8 // nbits
    v = vals.reshape(-1, per).astype(np.uint8)
    out = np.zeros(v.shape[0], dtype=np.uint8)
    for k in range(per):
        sh = (8 - (k + 1) * nbits) if order == "big" else k * nbits
        out |= (v[:, k] << sh).astype(np.uint8)
    return out


def _unpack2(packed):
    vals = np.empty((packed.shape[0], packed.shape[1] * 4), dtype=np.uint8)
    for k in range(4):
        vals[:, k::4] = (packed >> (6 - 2 * k)) & 3
    return vals


def _grid_delays():
    from sigpyproc3_b200 import synth

    dms = synth.dm_grid(1000.0, 1024)
    return np.atleast_2d(synth.C2.delays(dms)).astype(np.int32)


def _subset(kind):
    d = _grid_delays()
    if kind == "top":  # the 48 highest trials (DM ~1906-2000): widest spreads
        return d[-48:]
    return d[np.linspace(0, 1023, 48).astype(int)]  # spread over the whole grid


def _run_all_variants(torch, orc, vals, raw_host, nbits, order, d, nsamps, *, min_run=2,
                      min_bit_sliced=0):
    from sigpyproc3_b200.dedisp import DMTPlan

    nvalid = nsamps - int(d.max())
    expect = orc.dmt(vals, d, NCHANS, nsamps, nvalid)
    rawd = torch.from_numpy(raw_host).cuda()
    plan = DMTPlan(d, NCHANS, nsamps, nbits=nbits, bitorder=order, out_dtype=torch.int32)
    out = torch.empty((d.shape[0], nvalid), dtype=torch.int32, device="cuda")
    ran = sliced = 0
    for v in range(plan.num_variants):
        plan.set_variant(v)
        out.fill_(-1)
        plan.execute(rawd, nsamps, out)
        got = out.cpu().numpy()
        bad = np.argwhere(got != expect)
        assert bad.size == 0, (plan.describe(), bad[:5].tolist(), int(bad.shape[0]))
        ran += 1
        sliced += plan.describe()["bit_sliced"]
    plan.close()
    assert ran >= min_run and sliced >= min_bit_sliced, (ran, sliced)
    return expect


@pytest.mark.parametrize("subset", ["top", "spread"])
def test_c2_2bit_config_input(torch_cuda, orc, subset):
    """The config-2 generator's own bytes (uniform 2-bit samples plus the DM
    1700 pulse) over a window of 2^16 outputs."""
    torch = torch_cuda
    from oracle import synth_host
    from sigpyproc3_b200 import synth

    d = _subset(subset)
    nsamps = WINDOW + int(d.max())
    start_row = 790_000  # the DM-1700 pulse at sample 800 000 sweeps through this window
    packed = synth_host.c2_filterbank_host(start_row, nsamps)
    # the device generator writes the same bytes (the bench's input)
    dev = synth.c2_filterbank_device()
    rb = NCHANS // 4
    np.testing.assert_array_equal(
        dev[start_row * rb:(start_row + nsamps) * rb].cpu().numpy(), packed.ravel())
    del dev
    vals = _unpack2(packed).ravel()
    expect = _run_all_variants(torch, orc, vals, packed.ravel(), 2, "big", d, nsamps)
    assert expect.max() > 6144  # sums in the upper counter levels


def test_c2_2bit_saturated_sums(torch_cuda, orc):
    """Mostly-3 samples with a run of all-3 spectra longer than the maximum
    delay: sums reach 12 288 = 3 x 4096 (bit 13 of the counters)."""
    torch = torch_cuda
    d = _subset("top")
    nsamps = 16384 + int(d.max())
    rng = np.random.default_rng(1202)
    vals = np.where(rng.random((nsamps, NCHANS)) < 0.03, rng.integers(0, 3, (nsamps, NCHANS)),
                    3).astype(np.uint8)
    vals[5000:5000 + 40000] = 3
    vals = vals.ravel()
    expect = _run_all_variants(torch, orc, vals, _pack(vals, 2, "big"), 2, "big", d, nsamps)
    assert expect.max() == 3 * NCHANS


@pytest.mark.parametrize("subset", ["top", "spread"])
def test_c2_1bit(torch_cuda, orc, subset):
    """1-bit data (little-endian bit order, the sigproc default), sums up to 4096."""
    torch = torch_cuda
    d = _subset(subset)
    nsamps = 16384 + int(d.max())
    rng = np.random.default_rng(1101)
    vals = (rng.random((nsamps, NCHANS)) < 0.9).astype(np.uint8)
    vals[2000:2000 + 36000] = 1
    vals = vals.ravel()
    expect = _run_all_variants(torch, orc, vals, _pack(vals, 1, "little"), 1, "little", d, nsamps)
    assert expect.max() == NCHANS


def test_c2_4bit(torch_cuda, orc):
    """4-bit samples near full scale: sums up to 15 x 4096 = 61 440 (the top
    level of the 16-level bit-sliced counter) through the SIMD and the
    bit-sliced kernels."""
    torch = torch_cuda
    d = _subset("top")
    nsamps = 8192 + int(d.max())
    rng = np.random.default_rng(1404)
    vals = rng.integers(0, 16, size=(nsamps, NCHANS), dtype=np.uint8)
    vals[1000:1000 + 34000] = 15
    vals = vals.ravel()
    expect = _run_all_variants(torch, orc, vals, _pack(vals, 4, "big"), 4, "big", d, nsamps,
                               min_bit_sliced=2)
    assert expect.max() == 15 * NCHANS


def test_c2_8bit_wide_sums(torch_cuda, orc):
    """8-bit data near full scale: the SIMD kernels' 16-bit lanes are widened
    into 32-bit sums every few slabs; 4096 channels take that path 16 times."""
    torch = torch_cuda
    d = _subset("top")
    nsamps = 8192 + int(d.max())
    rng = np.random.default_rng(1808)
    vals = rng.integers(200, 256, size=(nsamps, NCHANS), dtype=np.uint8)
    vals[1000:1000 + 34000] = 255
    vals = vals.ravel()
    expect = _run_all_variants(torch, orc, vals, vals, 8, "big", d, nsamps, min_bit_sliced=1)
    assert expect.max() == 255 * NCHANS


@pytest.mark.parametrize("nbits", [1, 2, 4, 8])
def test_c2_worklist_bit_sliced(torch_cuda, orc, nbits):
    """The persistent work-list kernels (served path) at 4096 channels."""
    torch = torch_cuda
    from sigpyproc3_b200 import _lib
    from sigpyproc3_b200.batch import WorkList, num_variants

    d = _subset("top")[-24:]
    nsamps = 12000 + int(d.max())
    rng = np.random.default_rng(1500 + nbits)
    vals = rng.integers(0, 1 << nbits, size=(nsamps, NCHANS), dtype=np.uint8)
    vals[3000:3000 + 34000] = (1 << nbits) - 1
    vals = vals.ravel()
    order = "little" if nbits == 1 else "big"
    raw = torch.from_numpy(_pack(vals, nbits, order)).cuda()
    nv = nsamps - int(d.max())
    expect = orc.dmt(vals, d, NCHANS, nsamps, nv)
    dd = torch.from_numpy(d).cuda()
    ran = 0
    for v in range(num_variants(nbits)):
        wl = WorkList(nbits, v)
        span = wl.span_of(d)
        slot = wl.slot_words(span)
        if slot < 0:
            continue
        halo, pitch, rpc = wl.layout(nv, 0, int(d.max()), slot)
        planar = torch.empty(NCHANS * rpc * pitch, dtype=torch.int32, device="cuda")
        wl.corner_turn(raw, _lib.BITORDER_LITTLE if nbits == 1 else _lib.BITORDER_BIG, NCHANS,
                       nsamps, halo, planar, pitch)
        out = torch.full((d.shape[0], nv), -1, dtype=torch.int32, device="cuda")
        wl.add_job(planar_ptr=planar.data_ptr(), pitch_w=pitch, halo=halo, nchans=NCHANS,
                   delays_dev=dd, delays_host=d, out_ptr=out.data_ptr(), out_stride=out.stride(0),
                   out_start=0, out_elem=4, nvalid=nv, out_kind=_lib.OUT_I32)
        wl.finalize(span)
        wl.launch()
        torch.cuda.synchronize()
        assert int(wl.status[0].item()) == 0
        np.testing.assert_array_equal(out.cpu().numpy(), expect, err_msg=f"variant {v}")
        ran += 1
        del planar, out
    assert ran >= 1
    assert expect.max() == ((1 << nbits) - 1) * NCHANS
