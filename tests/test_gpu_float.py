"""Float32 path (config 5): zero-DM fused into the load, then the DM-time
transform, against the float64 oracle.

Two accumulators:

* SPP_ACC_F64 (the default for float32 input, as the reference's
  ``np.float64`` accumulator in kernels.dedisperse, core/kernels.py:356-362)
  adds each output's channels in channel order in float64 and rounds once:
  the same bits as the oracle, so every output is within rtol 1e-5 of the
  float64 sum (relative error <= 2^-24, the final rounding).
* SPP_ACC_KAHAN32 (faster, opt-in) sums 16-32-channel slabs in float32 and
  the slab partials with compensation.  Its error is bounded by
  ``1e-5 * |ref| + 2^-24 * sum_c |y_c|``; outputs near zero (heavy
  cancellation) can exceed a pure rtol of 1e-5, and the tests report how
  many do.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-5


def error_report(out32: np.ndarray, ref64: np.ndarray, mag: np.ndarray | None = None) -> dict:
    """Per-result relative error of float32 outputs against float64 sums."""
    out = out32.astype(np.float64)
    err = np.abs(out - ref64)
    rel = err / np.maximum(np.abs(ref64), np.finfo(np.float64).tiny)
    rep = {"max_rel": float(rel.max()), "frac_beyond_rtol": float(np.mean(rel > RTOL)),
           "n": int(rel.size)}
    if mag is not None:
        rep["max_err_over_bound"] = float((err / (RTOL * np.abs(ref64) + 2.0**-24 * mag)).max())
    return rep


def _zero_dm_case(orc, nchans, nsamps, foff, dms):
    import torch

    from sigpyproc3_b200 import _lib, synth
    from sigpyproc3_b200.header import Header

    g = synth.C5
    h = Header(nchans=nchans, fch1=g.fch1, foff=foff, tsamp=g.tsamp, nbits=32)
    d = np.atleast_2d(h.get_dmdelays(dms)).astype(np.int32)
    x = synth.gauss_f32_device(nsamps * nchans, 5)
    xh = x.cpu().numpy()
    bp = torch.zeros(nchans, dtype=torch.float32, device="cuda")
    _lib.call("spp_bandpass", x.data_ptr(), 32, 0, nchans, nsamps, bp.data_ptr(),
              torch.cuda.current_stream().cuda_stream)
    bph = orc.bandpass(xh, nchans, nsamps)
    np.testing.assert_array_equal(bp.cpu().numpy(), bph)  # bit-exact sequential float32
    w = torch.from_numpy(bph / bph.sum()).cuda()
    y = orc.zero_dm(xh, nchans, nsamps, bph)
    nv = nsamps - int(d.max())
    ref32, ref64 = orc.dmt(y, d, nchans, nsamps, nv, want64=True)
    return d, x, bp, w, y, ref32, ref64, nv


@pytest.mark.parametrize("acc", ["kahan", "f64"])
def test_zero_dm_dmt_float(orc, acc):
    from sigpyproc3_b200 import _lib, synth
    from sigpyproc3_b200.dedisp import DMTPlan

    nchans, nsamps = 512, 20000
    d, x, bp, w, y, ref32, ref64, nv = _zero_dm_case(orc, nchans, nsamps, synth.C5.foff * 8,
                                                     np.linspace(0, 300, 48))
    plan = DMTPlan(d, nchans, nsamps, nbits=32,
                   acc=_lib.ACC_KAHAN32 if acc == "kahan" else _lib.ACC_F64)
    mag = orc.dmt(np.abs(y), d, nchans, nsamps, nv).astype(np.float64)
    for v in range(plan.num_variants):
        plan.set_variant(v)
        out = plan.execute_zero_dm(x, nsamps, bp, w).cpu().numpy()
        if acc == "f64":
            np.testing.assert_array_equal(out, ref32, err_msg=str(plan.describe()))
        else:
            rep = error_report(out, ref64, mag)
            assert rep["max_err_over_bound"] <= 1.0, (v, rep)


def test_config5_geometry(orc):
    """4096 channels of N(0, 1) float32 at the config-5 band, three blocks of
    16 adjacent trials of the dmt_transform(1500, 4096) grid (DM 0-12,
    ~1494-1506 and ~2988-3000; adjacent trials, as in the full grid, keep a
    DM tile's delay spread within shared memory), a window of 8192 outputs past
    the 48 602-sample maximum delay, zero-DM fused.  The default (float64)
    accumulator reproduces the oracle's bits; the compensated float32 one is
    held to its documented bound, and both report their per-result error
    against the float64 sums."""
    from sigpyproc3_b200 import _lib, synth
    from sigpyproc3_b200.dedisp import DMTPlan

    grid = synth.dm_grid(1500.0, 4096)
    nchans = 4096
    nsamps = 8192 + 48602
    top = grid[-16:]
    d_top, x, bp, w, y, ref32, ref64, nv = _zero_dm_case(orc, nchans, nsamps, synth.C5.foff, top)
    assert int(d_top.max()) == 48602 and nv == 8192
    reports = {}
    for name, block in (("bottom", grid[:16]), ("middle", grid[2040:2056]), ("top", top)):
        d = np.atleast_2d(synth.C5.delays(block)).astype(np.int32)
        r32, r64 = orc.dmt(y, d, nchans, nsamps, nv, want64=True)
        mag = orc.dmt(np.abs(y), d, nchans, nsamps, nv).astype(np.float64)
        for acc in (_lib.ACC_F64, _lib.ACC_KAHAN32):
            plan = DMTPlan(d, nchans, nsamps, nbits=32, acc=acc)
            out_full = None
            for v in range(plan.num_variants):
                plan.set_variant(v)
                out_full = plan.execute_zero_dm(x, nsamps, bp, w).cpu().numpy()
                out = out_full[:, :nv]
                rep = error_report(out, r64, mag)
                reports[(name, acc, v)] = rep
                if acc == _lib.ACC_F64:
                    np.testing.assert_array_equal(out, r32, err_msg=str(plan.describe()))
                    assert rep["frac_beyond_rtol"] == 0.0, rep
                else:
                    assert rep["max_err_over_bound"] <= 1.0, (v, rep)
            plan.close()
    print("per-result error vs float64:", reports)


@pytest.mark.parametrize("plant", ["none", "zero", "subnormal", "inf"])
def test_f64_conversion_paths(orc, plant):
    """Float64 sums convert every other float32 by field arithmetic when the
    corner turn saw only normal floats, and through the conversion unit alone
    otherwise (a zero, a subnormal or an infinity anywhere in the block):
    both give the oracle's bits."""
    import torch

    from sigpyproc3_b200 import _lib
    from sigpyproc3_b200.dedisp import DMTPlan
    from sigpyproc3_b200.header import Header

    nchans, nsamps = 256, 6000
    h = Header(nchans=nchans, fch1=1400.0, foff=-0.5, tsamp=64e-6, nbits=32)
    d = np.atleast_2d(h.get_dmdelays(np.linspace(0, 200, 24))).astype(np.int32)
    rng = np.random.default_rng(77)
    x = rng.normal(0.0, 1.0, size=(nsamps, nchans)).astype(np.float32)
    value = {"zero": 0.0, "subnormal": 1e-40, "inf": np.inf}.get(plant)
    if value is not None:
        x[2500, 100] = np.float32(value)
    nv = nsamps - int(d.max())
    ref32 = orc.dmt(x.ravel(), d, nchans, nsamps, nv)
    plan = DMTPlan(d, nchans, nsamps, nbits=32, acc=_lib.ACC_F64)
    xd = torch.from_numpy(x.ravel()).cuda()
    for v in range(plan.num_variants):
        plan.set_variant(v)
        out = plan.execute(xd, nsamps).cpu().numpy()
        np.testing.assert_array_equal(out, ref32, err_msg=f"{plan.describe()} {plant}")
    plan.close()
