"""The persistent work-list kernel on plain jobs against the oracle."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available()
    return torch


def _pack(vals, nbits, order="big"):
    per = 8 // nbits
    v = vals.reshape(-1, per).astype(np.uint8)
    out = np.zeros(v.shape[0], dtype=np.uint8)
    for k in range(per):
        sh = (8 - (k + 1) * nbits) if order == "big" else k * nbits
        out |= (v[:, k] << sh).astype(np.uint8)
    return out


def _delays(nchans, dms):
    from sigpyproc3_b200.header import Header

    h = Header(nchans=nchans, fch1=1510.0, foff=-1.09, tsamp=320e-6)
    return np.atleast_2d(h.get_dmdelays(dms)).astype(np.int32)


@pytest.mark.parametrize("nbits", [1, 2, 4, 8])
def test_worklist_jobs_match_oracle(torch_cuda, orc, nbits):
    torch = torch_cuda
    from sigpyproc3_b200 import _lib
    from sigpyproc3_b200.batch import WorkList, corner_turn, num_variants, planar_layout

    rng = np.random.default_rng(70 + nbits)
    jobs = []
    for nchans, nsamps, ndm in ((72 if nbits != 1 else 64, 2500, 19), (128, 4000, 9)):
        vals = rng.integers(0, 1 << nbits, size=nsamps * nchans, dtype=np.uint8)
        raw = vals if nbits == 8 else _pack(vals, nbits)
        d = _delays(nchans, np.linspace(0, 45, ndm))
        jobs.append((nchans, nsamps, vals, raw, d))
    ran = 0
    for v in range(num_variants(nbits)):
        wl = WorkList(nbits, v)
        keep = []
        span = max(wl.span_of(d) for *_, d in jobs)
        slot = wl.slot_words(span)
        if slot < 0:  # fixed-slot variant narrower than these tables
            continue
        ran += 1
        outs = []
        for nchans, nsamps, vals, raw, d in jobs:
            nv = nsamps - int(d.max())
            halo, pitch, rpc = wl.layout(nv, 0, int(d.max()), slot)
            planar = torch.empty(nchans * rpc * pitch, dtype=torch.int32, device="cuda")
            rawd = torch.from_numpy(raw).cuda()
            wl.corner_turn(rawd, _lib.BITORDER_BIG, nchans, nsamps, halo, planar, pitch)
            dd = torch.from_numpy(d).cuda()
            out = torch.full((d.shape[0], nv), -1, dtype=torch.int32, device="cuda")
            wl.add_job(planar_ptr=planar.data_ptr(), pitch_w=pitch, halo=halo, nchans=nchans,
                       delays_dev=dd, delays_host=d, out_ptr=out.data_ptr(),
                       out_stride=out.stride(0), out_start=0, out_elem=4, nvalid=nv,
                       out_kind=_lib.OUT_I32)
            keep += [planar, rawd, dd]
            outs.append(out)
        wl.finalize(span)
        wl.launch()
        torch.cuda.synchronize()
        assert int(wl.status[0].item()) == 0
        for (nchans, nsamps, vals, raw, d), out in zip(jobs, outs):
            expect = orc.dmt(vals, d, nchans, nsamps, nsamps - int(d.max()))
            np.testing.assert_array_equal(out.cpu().numpy(), expect, err_msg=f"variant {v}")
    assert ran >= 2


def test_worklist_uint16_rows(torch_cuda, orc):
    """16-bit planar rows (the subband intermediate) summed over delayed rows."""
    torch = torch_cuda
    from sigpyproc3_b200 import _lib
    from sigpyproc3_b200.batch import WorkList, num_variants

    rng = np.random.default_rng(5)
    nrows_in, n = 24, 3000
    vals = rng.integers(0, 8000, size=(nrows_in, n)).astype(np.uint16)
    d = rng.integers(0, 200, size=(13, nrows_in)).astype(np.int32)
    nv = n - int(d.max())
    for v in range(num_variants(16)):
        wl = WorkList(16, v)
        span = wl.span_of(d)
        slot = wl.slot_words(span)
        pitch = ((n + 1) // 2 + slot + 16 + 3) // 4 * 4
        rows = np.zeros((nrows_in, pitch * 2), dtype=np.uint16)
        rows[:, :n] = vals
        planar = torch.from_numpy(rows.view(np.int32).copy()).cuda()
        dd = torch.from_numpy(d).cuda()
        out = torch.empty((13, nv), dtype=torch.int32, device="cuda")
        wl.add_job(planar_ptr=planar.data_ptr(), pitch_w=pitch, halo=0, nchans=nrows_in,
                   delays_dev=dd, delays_host=d, out_ptr=out.data_ptr(), out_stride=out.stride(0),
                   out_start=0, out_elem=4, nvalid=nv, out_kind=_lib.OUT_I32)
        wl.finalize(span)
        wl.launch()
        torch.cuda.synchronize()
        # oracle: time-major layout of the rows
        expect = orc.dmt(np.ascontiguousarray(vals.T.astype(np.float32)), d, nrows_in, n, nv)
        np.testing.assert_array_equal(out.cpu().numpy(), expect.astype(np.int32),
                                      err_msg=f"variant {v}")
