"""Host-side logic without a GPU: delay tables (R6) against the reference's own
outputs, the read_plan schedule (R5), sigproc headers (N1), and the C ABI
library's exported symbols."""

import ctypes
import hashlib
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_delays_match_reference(golden, golden_meta):
    from sigpyproc3_b200.header import Header

    for key, m in golden_meta["delays"].items():
        nch, f1, fo, ts = m["geom"]
        h = Header(nchans=nch, fch1=f1, foff=fo, tsamp=ts)
        dms = golden[f"delays_{key}_dms"]
        d = np.atleast_2d(h.get_dmdelays(dms, m["ref"])).astype(np.int32)
        assert sha(d) == m["sha256"], key
        np.testing.assert_array_equal(d[golden[f"delays_{key}_rowidx"]], golden[f"delays_{key}_rows"])


def test_delays_float_and_params(golden):
    from sigpyproc3_b200 import params

    freqs = np.arange(1000, dtype=np.float32) * (-1.0) + 1400
    sec = params.compute_dmdelays(freqs, np.linspace(0, 100, 50), 0.001, freqs[0], in_samples=False)
    assert sec.dtype == np.float32
    np.testing.assert_array_equal(sec, golden["delays_params_sec"])
    samp = params.compute_dmdelays(freqs, np.linspace(0, 100, 50), 0.001, freqs[0])
    assert samp.dtype == np.int32
    np.testing.assert_array_equal(samp, golden["delays_params_samp"])
    assert np.all(samp[:, 0] == 0)


def test_delays_float64_would_differ():
    # K2: recomputing in float64 changes some delays at the config-2 geometry
    from sigpyproc3_b200 import synth

    g = synth.C2
    dms = synth.dm_grid(1000.0, 1024)
    d32 = g.delays(dms)
    f = g.chan_freqs().astype(np.float64)
    d64 = np.rint(dms[:, None] * 4148.808 * (f**-2 - g.fch1**-2) / g.tsamp).astype(np.int32)
    assert np.count_nonzero(d32 != d64) > 0


def test_header_ref_freq_errors():
    from sigpyproc3_b200.header import Header

    h = Header(nchans=64, fch1=1510.0, foff=-1.09, tsamp=320e-6)
    with pytest.raises(ValueError):
        h.get_dmdelays(100, ref_freq="top")
    with pytest.raises(TypeError):
        h.get_dmdelays(100, ref_freq=[1.0])
    assert h.get_dmdelays(0).max() == 0


def test_read_plan_schedule(golden_meta):
    from sigpyproc3_b200.readers import plan_blocks

    for case in golden_meta["read_plan"]:
        nsamples, nchans, gulp, start, nsamps, skip = case["args"]
        g, blocks = plan_blocks(nsamples, gulp, start, nsamps, skip)
        pos = start * nchans
        ours = []
        for ii, nblk, sk in blocks:
            ours.append((nblk, ii, pos))
            pos += nblk * nchans + sk * nchans
        ref = [(b[0], b[1], b[2]) for b in case["blocks"]]
        if case["error"] is None:
            assert ours == ref
        else:
            # the reference stops where its read size check fails; the schedule
            # up to there is identical
            assert ours[: len(ref)] == ref
    for case in golden_meta["read_plan_errors"]:
        nsamples, gulp, nsamps, skip = case["args"]
        with pytest.raises(ValueError, match=re.escape(case["error"])):
            plan_blocks(nsamples, gulp, 0, nsamps, skip)


def test_sigproc_roundtrip(tmp_path):
    from sigpyproc3_b200.header import Header
    from sigpyproc3_b200.io import sigproc

    h = Header(nchans=64, fch1=1510.0, foff=-1.09, tsamp=320e-6, nbits=2, tstart=59000.5,
               source="J0000+0000")
    raw = np.arange(1000 * 16, dtype=np.uint8) % 251
    p = tmp_path / "x.fil"
    h.write_sigproc(p, raw)
    h2 = Header.from_sigproc(p)
    assert (h2.nchans, h2.nbits, h2.nsamples) == (64, 2, 1000)
    assert h2.fch1 == 1510.0 and h2.foff == -1.09 and h2.tsamp == 320e-6
    assert h2.source == "J0000+0000"
    d = sigproc.read_header(p)
    assert d["datalen"] == raw.nbytes
    with pytest.raises(OSError):
        bad = tmp_path / "bad.fil"
        bad.write_bytes(b"\x05\x00\x00\x00hello")
        sigproc.read_header(bad)


def test_reference_fixture_headers():
    # the reference's own sample files parse (only where the tree is mounted)
    data = Path("/root/reference/tests/data")
    if not data.is_dir():
        pytest.skip("reference test data not mounted")
    from sigpyproc3_b200.header import Header

    h = Header.from_sigproc(data / "parkes_4bit.fil")
    assert (h.nchans, h.nbits) == (832, 4)
    assert abs(h.get_dmdelays(100, in_samples=False).max() - 0.8) < 0.1  # test_header.py:35-41
    assert abs(h.get_dmdelays(5000, in_samples=False).max() - 40.4) < 0.1


def _header_functions():
    text = (ROOT / "include" / "sppgpu.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(spp_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from sigpyproc3_b200 import _lib

    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    names = _header_functions()
    assert len(names) > 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding covers them with signatures
    unbound = [n for n in names if n not in _lib.SIGNATURES]
    assert not unbound, unbound


def test_abi_argument_errors_without_gpu():
    from sigpyproc3_b200 import _lib

    lib = _lib.load()
    assert lib.spp_unpack(None, 10, 2, 0, None, None) == _lib.SPP_ERR_ARG
    assert b"null" in lib.spp_last_error_string()
    assert lib.spp_dedisperse_workspace_bytes(3, 64, 100, 0, 10) == -1
    assert lib.spp_dedisperse_workspace_bytes(8, 64, 4096, 0, 100) > 64 * 4096
    # nchans * nbits not a multiple of 8
    assert lib.spp_dedisperse_workspace_bytes(2, 3, 4096, 0, 10) == -1


@pytest.mark.parametrize("nchans,nbands", [(64, 8), (64, 5), (64, 6), (64, 7), (1000, 32),
                                           (4096, 30), (17, 17), (31, 4)])
def test_fold_band_start_matches_reference_assignment(orc, nchans, nbands):
    """Subband boundaries used by Filterbank.fold equal kernels.fold's
    ``ichan // (nchans / nsubs)``, here through the oracle's floor division."""
    from sigpyproc3_b200.readers import fold_band_start

    bs = fold_band_start(nchans, nbands)
    factor2 = nchans / nbands
    band = [int(orc.lib().orc_py_floordiv(float(c), factor2)) for c in range(nchans)]
    assert bs[0] == 0 and bs[-1] == nchans and len(bs) == nbands + 1
    for b in range(nbands):
        assert all(band[c] == b for c in range(bs[b], bs[b + 1]))


def test_pulse_extractor_window(tmp_path):
    """PulseExtractor's window arithmetic (readers.py:393-455), restated."""
    from sigpyproc3_b200 import Header
    from sigpyproc3_b200.readers import PulseExtractor

    h = Header(nchans=64, fch1=1510.0, foff=-1.0, tsamp=320e-6, nbits=8, nsamples=6000)
    path = tmp_path / "p.fil"
    h.write_sigproc(path, np.zeros(6000 * 64, np.uint8))
    for toa, width, dm, toa_freq, nch in ((3000, 8, 30.0, None, None), (40, 3, 10.0, 1480.0, 16),
                                          (5990, 1, 50.0, None, 32)):
        pe = PulseExtractor(str(path), toa, width, dm, min_nsamps=64, toa_freq=toa_freq,
                            nchans=nch)
        f1 = toa_freq or 1510.0
        sub = h.new_header({"fch1": f1, "nchans": nch or 64})
        disp = int(np.max(np.abs(np.atleast_1d(sub.get_dmdelays(dm))))) + 5 * width
        tdec = max(1, width // 2)
        n = max(2 * (((disp // tdec) + 1) * tdec), 64 * tdec)
        assert (pe.disp_delay, pe.t_decimate, pe.nsamps) == (disp, tdec, n)
        assert pe.nstart == toa - n // 2 and pe.nstart_file == max(0, toa - n // 2)
        assert pe.nsamps_file == min(n + min(0, pe.nstart), 6000 - max(0, pe.nstart))


def test_host_twins_follow_the_generator_definitions():
    """The test suite's numpy twins (oracle/synth_host.py) describe the same
    config-2 workload as the product's device generator: geometry, trial
    grid, delay table, pulse rows and threshold tables."""
    from oracle import synth_host
    from sigpyproc3_b200 import synth

    g = synth.C2
    assert (g.nchans, g.nsamps, g.nbits, g.tsamp, g.fch1, g.foff) == (
        synth_host.C2_NCHANS, synth_host.C2_NSAMPS, synth_host.C2_NBITS, synth_host.C2_TSAMP,
        synth_host.C2_FCH1, synth_host.C2_FOFF)
    assert synth.C2_PULSES == synth_host.C2_PULSES
    assert synth.C2_PULSE_WIDTH == synth_host.C2_PULSE_WIDTH
    dms = synth.dm_grid(1000.0, 1024)
    np.testing.assert_array_equal(dms, synth_host.dm_grid(1000.0, 1024))
    np.testing.assert_array_equal(np.atleast_2d(g.delays(dms)).astype(np.int32),
                                  synth_host.c2_delays(dms))
    for a, b in zip(synth.c2_pulse_rows(), synth_host.c2_pulse_rows()):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(synth.gauss_u8_thresholds(96.0, 12.0),
                                  synth_host.gauss_u8_thresholds(96.0, 12.0))
    x = synth_host.c2_filterbank_host(199_990, 40)
    assert x.shape == (40, 1024) and x.dtype == np.uint8


@pytest.mark.parametrize("nbits,order", [(1, "little"), (1, "big"), (2, "big"), (2, "little"),
                                         (4, "big"), (4, "little")])
def test_pack_host_inverts_unpack(orc, nbits, order):
    """Host packing for written files: the inverse of the reference's unpack."""
    from sigpyproc3_b200.io.bits import pack_host

    raw = np.random.default_rng(nbits).integers(0, 256, 999, dtype=np.uint8)
    np.testing.assert_array_equal(pack_host(orc.unpack(raw, nbits, order), nbits, order), raw)


def test_sigproc_writer_roundtrip(tmp_path):
    from sigpyproc3_b200 import Header
    from sigpyproc3_b200.io import sigproc

    h = Header(nchans=16, nbits=2, nsamples=0, fch1=1400.0, foff=-2.0, tsamp=1e-3,
               filename=str(tmp_path / "a.fil"))
    vals = np.random.default_rng(1).integers(0, 4, 16 * 40, dtype=np.uint8)
    with h.prep_outfile(tmp_path / "w.fil", updates={"foff": -4.0}) as w:
        w.cwrite(vals[:320])
        w.cwrite(vals[320:])
    hdr = sigproc.read_header(tmp_path / "w.fil")
    assert hdr["nsamples"] == 40 and hdr["foff"] == -4.0 and hdr["nbits"] == 2


def test_pulse_extractor_matches_reference_arithmetic(tmp_path, golden_meta):
    """PulseExtractor's window (readers.py:393-455) against the reference's own
    property code run on the same header values (tests/golden/make_golden.py)."""
    from sigpyproc3_b200 import Header
    from sigpyproc3_b200.readers import PulseExtractor

    for case in golden_meta["pulse_extractor"]:
        toa, width, dm, toa_freq, nch_sub, nsamples = case["args"]
        h = Header(nchans=64, fch1=1510.0, foff=-1.0, tsamp=320e-6, nbits=8, nsamples=nsamples)
        path = tmp_path / f"p{nsamples}.fil"
        if not path.exists():
            h.write_sigproc(path, np.zeros(nsamples * 64, np.uint8))
        pe = PulseExtractor(str(path), toa, width, dm, min_nsamps=64, toa_freq=toa_freq,
                            nchans=nch_sub)
        got = {n: int(getattr(pe, n)) for n in case["props"]}
        assert got == case["props"], (case["args"], got)


def test_good_size_matches_pocketfft_rule():
    """The FFT length the reference pads to (rocket_fft.good_size(n, real=True)):
    pocketfft's rule, as scipy.fft.next_fast_len(n, real=True) applies it."""
    from scipy import fft as sfft

    from sigpyproc3_b200.filters import good_size_real

    ns = list(range(1, 4000)) + [65535, 65536, 65537, 999983, 1 << 20, (1 << 21) - 1]
    assert [good_size_real(n) for n in ns] == [sfft.next_fast_len(n, real=True) for n in ns]


def test_template_bank_matches_reference(golden, golden_meta, orc):
    """Template.gen_* and get_box_width_spacing against the reference's own code
    (tests/golden/make_golden.py), for this package and for the oracle."""
    from sigpyproc3_b200.filters import MatchedFilter, Template

    np.testing.assert_array_equal(MatchedFilter.get_box_width_spacing(32, 1.5),
                                  golden_meta["box_widths_32_1p5"])
    np.testing.assert_array_equal(MatchedFilter.get_box_width_spacing(100, 1.3),
                                  golden_meta["box_widths_100_1p3"])
    by_kind = {}
    for rec in golden_meta["templates"]:
        t = getattr(Template, f"gen_{rec['kind']}")(rec["width"])
        ref = golden[f"temp_{rec['kind']}_{rec['k']}"]
        np.testing.assert_array_equal(t.data, ref)
        assert t.data.dtype == ref.dtype
        assert (t.ref_bin, t.ref) == (rec["ref_bin"], rec["ref"])
        by_kind.setdefault(rec["kind"], []).append((ref, rec["ref_bin"]))
    for kind, temps in by_kind.items():
        _, bank = orc.template_bank(kind)
        assert len(bank) == len(temps)
        for (h, rb), (ref, rrb) in zip(bank, temps):
            np.testing.assert_array_equal(np.asarray(h), ref)
            assert rb == rrb


def test_counter_fits_bounds():
    """Bit-sliced work-list kernels count below 2^14 (1-, 2-bit) or 2^16
    (4-bit); SIMD kernels take any channel count."""
    from sigpyproc3_b200.batch import counter_fits

    sliced, simd = {"planes": 1}, {"planes": 0}
    assert counter_fits(sliced, 4, 4369) and not counter_fits(sliced, 4, 4370)
    assert counter_fits(sliced, 2, 5461) and not counter_fits(sliced, 2, 5462)
    assert counter_fits(sliced, 1, 16383) and not counter_fits(sliced, 1, 16384)
    assert counter_fits(sliced, 8, 4112) and not counter_fits(sliced, 8, 4113)
    assert counter_fits(simd, 4, 1 << 20)


def test_channel_pair_regrouping_is_the_direct_sum(orc):
    """The channel-pair kernels' identity, on the CPU: with pair rows
    S_k,r[t] = x[2k][t] + x[2k+1][t + r] built once per (pair, relative
    offset) and shared by every trial, sum_k S_k,r(dm)[t + o(dm, 2k)] equals
    the oracle's direct sum over channels (kernels.dedisperse,
    core/kernels.py:340-362) for every trial; the rows per pair and the
    distinct rows per 8-trial tile are the quantities the plan checks."""
    from sigpyproc3_b200.header import Header

    nchans, nsamps = 64, 1500
    h = Header(nchans=nchans, fch1=1500.0, foff=-2.0, tsamp=64e-6)
    d = np.atleast_2d(h.get_dmdelays(np.linspace(0.0, 20.0, 24))).astype(np.int32)
    nvalid = nsamps - int(d.max())
    rng = np.random.default_rng(12)
    x = rng.integers(0, 4, size=(nsamps, nchans), dtype=np.uint8)
    expect = orc.dmt(x.ravel(), d, nchans, nsamps, nvalid)
    r = d[:, 1::2] - d[:, 0::2]
    rows = {}
    for k in range(nchans // 2):
        for rr in np.unique(r[:, k]):
            s = x[:, 2 * k].astype(np.int32).copy()
            part = np.zeros(nsamps, dtype=np.int32)
            part[:nsamps - rr] = x[rr:, 2 * k + 1]
            rows[(k, int(rr))] = s + part
    got = np.zeros_like(expect)
    for i in range(d.shape[0]):
        for k in range(nchans // 2):
            o = d[i, 2 * k]
            got[i] += rows[(k, int(r[i, k]))][o:o + nvalid]
    np.testing.assert_array_equal(got, expect)
    assert len(rows) < 12 * nchans  # the plan's row budget
    tiles = [max(len(np.unique(r[t:t + 8, k])) for k in range(nchans // 2))
             for t in range(0, d.shape[0], 8)]
    assert max(tiles) <= 3  # rows a tile of 8 trials reads per pair
