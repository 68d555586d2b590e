"""Float32 path (config-5 shape, reduced): zero-DM fused into the load, then the
DM-time transform, against the float64 oracle.

Tolerance: |gpu - oracle| <= 1e-5 * |oracle| + 2**-24 * sum_c |y_c| per output,
where y is the zero-DM'd input; the second term is the float32 resolution of
the summands themselves (the oracle sees the same float32 inputs)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("acc", ["kahan", "f64"])
def test_zero_dm_dmt_float(orc, acc):
    import torch

    from sigpyproc3_b200 import _lib, synth
    from sigpyproc3_b200.dedisp import DMTPlan
    from sigpyproc3_b200.header import Header

    g = synth.C5
    nchans, nsamps, ndm = 512, 20000, 48
    h = Header(nchans=nchans, fch1=g.fch1, foff=g.foff * 8, tsamp=g.tsamp, nbits=32)
    dms = np.linspace(0, 300, ndm)
    d = np.atleast_2d(h.get_dmdelays(dms)).astype(np.int32)
    x = synth.gauss_f32_device(nsamps * nchans, 5)
    xh = x.cpu().numpy()
    bp = torch.zeros(nchans, dtype=torch.float32, device="cuda")
    _lib.call("spp_bandpass", x.data_ptr(), 32, 0, nchans, nsamps, bp.data_ptr(),
              torch.cuda.current_stream().cuda_stream)
    bph = orc.bandpass(xh, nchans, nsamps)
    np.testing.assert_array_equal(bp.cpu().numpy(), bph)  # bit-exact sequential float32
    w = torch.from_numpy(bph / bph.sum()).cuda()
    plan = DMTPlan(d, nchans, nsamps, nbits=32,
                   acc=_lib.ACC_KAHAN32 if acc == "kahan" else _lib.ACC_F64)
    y = orc.zero_dm(xh, nchans, nsamps, bph)
    nv = nsamps - int(d.max())
    _, ref64 = orc.dmt(y, d, nchans, nsamps, nv, want64=True)
    mag = orc.dmt(np.abs(y), d, nchans, nsamps, nv).astype(np.float64)
    for v in range(plan.num_variants):
        plan.set_variant(v)
        out = plan.execute_zero_dm(x, nsamps, bp, w).cpu().numpy().astype(np.float64)
        err = np.abs(out - ref64)
        bound = 1e-5 * np.abs(ref64) + 2.0**-24 * mag
        assert np.all(err <= bound), (v, float(err.max()))
