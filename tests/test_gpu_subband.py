"""Two-stage subband search (R7 + R9) against the oracle: the DM-time rows equal
a brute-force transform with the plan's effective delay table (exact integers),
and the S/N peaks match the float64 boxcar oracle."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available()
    return torch


def _beam(seed, nsamps, nchans):
    from oracle import synth_host

    th = synth_host.gauss_u8_thresholds(96.0, 12.0)
    return synth_host.gauss_u8_host(seed, 0, nsamps * nchans, th)


def test_subband_search_small(torch_cuda, orc):
    torch = torch_cuda
    from sigpyproc3_b200 import Header
    from sigpyproc3_b200.subband import SubbandPlan, SubbandSearch

    h = Header(nchans=256, fch1=1400.0, foff=-1.171875, tsamp=64e-6, nbits=8)
    dms = np.linspace(0, 100, 96)
    plan = SubbandPlan(h, dms, nsub=16, group=16)
    lens = [6000, 9000, 12000]
    factors, widths = (1, 2, 4), (1, 2, 4, 8, 16, 32, 64, 128, 256)
    from sigpyproc3_b200.batch import num_variants, variant_cfg
    from sigpyproc3_b200 import _lib

    # stage 1 through a bit-sliced kernel (eight plane rows per channel) and
    # through a SIMD one
    kinds = [variant_cfg(8, _lib.ACC_KAHAN32, v)["planes"] for v in range(num_variants(8))]
    pairs = ((kinds.index(1), 0), (kinds.index(0), 1))
    for v1, v2 in pairs:
        srch = SubbandSearch(plan, lens, factors=factors, widths=widths, variants=(v1, v2))
        data = [_beam(30 + i, n, 256) for i, n in enumerate(lens)]
        for b, x in zip(srch.beams, data):
            b.raw.copy_(torch.from_numpy(x))
        srch.run()
        torch.cuda.synchronize()
        assert srch.status_ok()
        for b, x, n in zip(srch.beams, data, lens):
            nv = plan.nvalid(n)
            expect = orc.dmt(x, plan.eff, 256, n, nv)
            np.testing.assert_array_equal(b.dmt.cpu().numpy(), expect)
            esnr, eidx = orc.boxcar_snr(expect.astype(np.float32), factors, widths)
            np.testing.assert_allclose(b.snr.cpu().numpy(), esnr, rtol=1e-5)
            np.testing.assert_array_equal(b.idx.cpu().numpy(), eidx)


def test_subband_graph_replay(torch_cuda, orc):
    torch = torch_cuda
    from sigpyproc3_b200 import Header
    from sigpyproc3_b200.subband import SubbandPlan, SubbandSearch

    h = Header(nchans=256, fch1=1400.0, foff=-1.171875, tsamp=64e-6, nbits=8)
    plan = SubbandPlan(h, np.linspace(0, 80, 40), nsub=16, group=8)
    lens = [7000, 5000]
    srch = SubbandSearch(plan, lens, factors=(1, 2), widths=(1, 4, 16))
    for i, b in enumerate(srch.beams):
        b.raw.copy_(torch.from_numpy(_beam(50 + i, lens[i], 256)))
    srch.capture()
    for rep in range(2):
        data = [_beam(60 + 10 * rep + i, n, 256) for i, n in enumerate(lens)]
        for b, x in zip(srch.beams, data):
            b.raw.copy_(torch.from_numpy(x))
        srch.replay()
        torch.cuda.synchronize()
        for b, x, n in zip(srch.beams, data, lens):
            expect = orc.dmt(x, plan.eff, 256, n, plan.nvalid(n))
            np.testing.assert_array_equal(b.dmt.cpu().numpy(), expect)


def test_subband_config3_geometry_rows(torch_cuda, orc):
    """Config-3 geometry (1024 ch, 32 subbands, 512 trials 0-1000): spot rows."""
    torch = torch_cuda
    from sigpyproc3_b200 import Header, synth
    from sigpyproc3_b200.subband import SubbandPlan, SubbandSearch

    g = synth.C3
    h = Header(nchans=g.nchans, fch1=g.fch1, foff=g.foff, tsamp=g.tsamp, nbits=8)
    plan = SubbandPlan(h, synth.dm_grid(500.0, 512), nsub=32, group=16)
    n = 1 << 16
    n += plan.max_eff
    srch = SubbandSearch(plan, [n])
    x = _beam(3, n, g.nchans)
    srch.beams[0].raw.copy_(torch.from_numpy(x))
    srch.run()
    torch.cuda.synchronize()
    rows = [0, 1, 255, 256, 511]
    nv = plan.nvalid(n)
    expect = orc.dmt(x, plan.eff[rows], g.nchans, n, nv)
    got = srch.beams[0].dmt.cpu().numpy()[rows]
    np.testing.assert_array_equal(got, expect)
    # two-stage delays stay within a few samples of the exact per-channel delays
    exact = np.atleast_2d(h.get_dmdelays(plan.dms)).astype(np.int64)
    assert np.abs(plan.eff - exact).max() <= 20
