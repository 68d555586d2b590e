"""GPU kernels against the oracle and the reference golden vectors (R2-R4)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# Float32 input: |gpu - fp64 oracle| <= RTOL * |oracle| + ATOL_UNIT * sum_c |x_c|
# (the second term is 2**-24 times the summands' magnitude: the float32
# representation scale of the inputs themselves).
RTOL = 1e-5
ATOL_UNIT = 2.0**-24


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available(), "GPU tests need CUDA"
    return torch


def _geom_delays(nchans, dm, ref="fch1", fch1=1510.0, foff=-1.09, tsamp=320e-6):
    from sigpyproc3_b200.header import Header

    h = Header(nchans=nchans, fch1=fch1, foff=foff, tsamp=tsamp)
    return np.atleast_1d(h.get_dmdelays(dm, ref)).astype(np.int32)


def _pack(vals, nbits, order):
    """Pack uint8 samples (time-major) to the sigproc layout (inverse of unpack)."""
    per = 8 // nbits
    v = vals.reshape(-1, per).astype(np.uint8)
    out = np.zeros(v.shape[0], dtype=np.uint8)
    for k in range(per):
        sh = (8 - (k + 1) * nbits) if order == "big" else k * nbits
        out |= (v[:, k] << sh).astype(np.uint8)
    return out


@pytest.mark.parametrize("nbits", [1, 2, 4])
@pytest.mark.parametrize("order", ["big", "little"])
def test_unpack_golden(torch_cuda, golden, nbits, order):
    from sigpyproc3_b200.io.bits import unpack

    out = unpack(golden["unpack_rand_in"], nbits, order).cpu().numpy()
    np.testing.assert_array_equal(out, golden[f"unpack_rand_{nbits}_{order}"])
    kat = unpack(np.array([7, 23], np.uint8), nbits, order).cpu().numpy()
    np.testing.assert_array_equal(kat, golden[f"unpack_kat_{nbits}_{order}"])


@pytest.mark.parametrize("tag", ["dm50", "dm200", "dm120_fcenter"])
def test_dedisperse_block_golden_u8(torch_cuda, golden, tag):
    torch = torch_cuda
    from sigpyproc3_b200.dedisp import dedisperse_block

    x = torch.from_numpy(golden["ded_u8_in"].ravel()).cuda()
    d = golden[f"ded_u8_{tag}_delays"]
    ref = golden[f"ded_u8_{tag}_out"]
    out = torch.full((ref.size + 7,), -1.0, device="cuda")
    n = dedisperse_block(x, d, 64, 4096, out, out_start=3)
    assert n == ref.size
    o = out.cpu().numpy()
    np.testing.assert_array_equal(o[3:3 + n], ref)  # bit-exact
    assert np.all(o[:3] == -1) and np.all(o[3 + n:] == -1)


def test_dedisperse_block_golden_f32(torch_cuda, golden):
    torch = torch_cuda
    from sigpyproc3_b200 import _lib
    from sigpyproc3_b200.dedisp import dedisperse_block

    x = golden["ded_f32_in"]
    d = golden["ded_f32_delays"]
    ref = golden["ded_f32_out"]
    for acc in (_lib.ACC_F64, _lib.ACC_KAHAN32):
        out = torch.zeros(ref.size, device="cuda")
        dedisperse_block(torch.from_numpy(x.ravel()).cuda(), d, 32, 2048, out, acc=acc)
        np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=RTOL, atol=1e-6)


@pytest.mark.parametrize("nbits,nchans", [(1, 64), (1, 136), (2, 64), (2, 100), (4, 64),
                                          (4, 98), (8, 64), (8, 200), (8, 300)])
@pytest.mark.parametrize("ref", ["fch1", "fcenter"])
def test_dedisperse_block_all_nbits(torch_cuda, orc, nbits, nchans, ref):
    torch = torch_cuda
    from sigpyproc3_b200.dedisp import dedisperse_block

    rng = np.random.default_rng(nbits * 1000 + nchans)
    nsamps = 3001
    vals = rng.integers(0, 1 << nbits, size=nsamps * nchans, dtype=np.uint8)
    raw = vals if nbits == 8 else _pack(vals, nbits, "big")
    d = _geom_delays(nchans, 40.0, ref)
    expect = orc.dedisperse(vals, d, nchans, nsamps)
    out = torch.zeros(expect.size, device="cuda")
    dedisperse_block(torch.from_numpy(raw).cuda(), d, nchans, nsamps, out, nbits=nbits,
                     bitorder="big")
    np.testing.assert_array_equal(out.cpu().numpy(), expect)


def test_dedisperse_block_edge_cases(torch_cuda, orc):
    torch = torch_cuda
    from sigpyproc3_b200.dedisp import dedisperse_block

    rng = np.random.default_rng(5)
    vals = rng.integers(0, 256, size=100 * 16, dtype=np.uint8)
    # zero delays: plain channel sum
    d = np.zeros(16, np.int32)
    out = torch.zeros(100, device="cuda")
    dedisperse_block(torch.from_numpy(vals).cuda(), d, 16, 100, out)
    np.testing.assert_array_equal(out.cpu().numpy(), vals.reshape(100, 16).sum(1).astype(np.float32))
    # max delay >= nsamps: nothing to do (reference: empty prange)
    d = np.full(16, 100, np.int32)
    assert dedisperse_block(torch.from_numpy(vals).cuda(), d, 16, 100, out) == 0
    # output too small -> ValueError, no write
    d = np.arange(16, dtype=np.int32)
    small = torch.zeros(10, device="cuda")
    with pytest.raises(ValueError):
        dedisperse_block(torch.from_numpy(vals).cuda(), d, 16, 100, small)
    # one sample valid
    d = np.full(16, 99, np.int32)
    d[0] = 0
    o1 = torch.zeros(1, device="cuda")
    assert dedisperse_block(torch.from_numpy(vals).cuda(), d, 16, 100, o1) == 1
    np.testing.assert_array_equal(o1.cpu().numpy(), orc.dedisperse(vals, d, 16, 100))


@pytest.mark.parametrize("nbits", [1, 2, 4, 8])
@pytest.mark.parametrize("wide", [True, False])
def test_dmt_plan_all_variants(torch_cuda, orc, nbits, wide):
    """Every kernel variant; 136/128 channels (5 or 4 slabs of 32, the last
    partial) and 96 channels (3 full slabs: an odd slab count)."""
    torch = torch_cuda
    from sigpyproc3_b200.dedisp import DMTPlan

    nchans = (136 if nbits != 1 else 128) if wide else 96
    nsamps, ndm = 2500, 19
    rng = np.random.default_rng(7 + nbits)
    vals = rng.integers(0, 1 << nbits, size=nsamps * nchans, dtype=np.uint8)
    raw = vals if nbits == 8 else _pack(vals, nbits, "big")
    dms = np.linspace(0, 60, ndm)
    d = np.atleast_2d(_geom_delays(nchans, dms))
    nvalid = nsamps - int(np.abs(d).max())
    expect = orc.dmt(vals, d, nchans, nsamps, nvalid)
    plan = DMTPlan(d, nchans, nsamps, nbits=nbits, out_dtype=torch.int32)
    assert plan.num_variants >= 2
    rawd = torch.from_numpy(raw).cuda()
    for v in range(plan.num_variants):
        plan.set_variant(v)
        out = plan.execute(rawd, nsamps)
        np.testing.assert_array_equal(out.cpu().numpy(), expect, err_msg=str(plan.describe()))
    plan.close()
    # float32 output of the same sums
    plan = DMTPlan(d, nchans, nsamps, nbits=nbits, out_dtype=torch.float32)
    out = plan.execute(rawd, nsamps)
    np.testing.assert_array_equal(out.cpu().numpy(), expect.astype(np.float32))


@pytest.mark.parametrize("nbits", [1, 2, 4, 8])
def test_dmt_plan_negative_delays_all_variants(torch_cuda, orc, nbits):
    """Delays referenced to the band centre (negative in its upper half, so
    samples before the block wrap as numba's negative indices) through every
    kernel variant, bit-sliced and SIMD, against the oracle; 72 channels (a
    partial last slab of 16 or 32)."""
    torch = torch_cuda
    from sigpyproc3_b200.dedisp import DMTPlan

    nchans, nsamps, ndm = 72, 3000, 21
    rng = np.random.default_rng(40 + nbits)
    vals = rng.integers(0, 1 << nbits, size=nsamps * nchans, dtype=np.uint8)
    raw = vals if nbits == 8 else _pack(vals, nbits, "big")
    d = np.atleast_2d(_geom_delays(nchans, np.linspace(0, 80, ndm), ref="fcenter"))
    assert d.min() < 0 < d.max()
    nvalid = nsamps - int(np.abs(d).max())
    expect = orc.dmt(vals, d, nchans, nsamps, nvalid)
    plan = DMTPlan(d, nchans, nsamps, nbits=nbits, out_dtype=torch.int32)
    rawd = torch.from_numpy(raw).cuda()
    sliced = 0
    for v in range(plan.num_variants):
        plan.set_variant(v)
        out = plan.execute(rawd, nsamps, check=True)
        np.testing.assert_array_equal(out.cpu().numpy(), expect, err_msg=str(plan.describe()))
        sliced += plan.describe()["bit_sliced"]
    plan.close()
    assert sliced >= 1


@pytest.mark.parametrize("nbits", [2, 4, 8])
def test_dmt_plan_roll_mode_integer(torch_cuda, orc, nbits):
    """Roll mode (kernels.dmt_block: circular shifts by +delay) on packed
    integer samples through every variant, against the oracle's float32 roll
    of the same integer values (exact)."""
    torch = torch_cuda
    from sigpyproc3_b200.dedisp import DMTPlan

    nchans, nsamps, ndm = 64, 2048, 12
    rng = np.random.default_rng(60 + nbits)
    vals = rng.integers(0, 1 << nbits, size=nsamps * nchans, dtype=np.uint8)
    raw = vals if nbits == 8 else _pack(vals, nbits, "big")
    d = np.atleast_2d(_geom_delays(nchans, np.linspace(0, 40, ndm)))
    assert int(d.max()) < nsamps
    expect = orc.dmt_roll(vals.astype(np.float32), d, nchans, nsamps)
    plan = DMTPlan(d, nchans, nsamps, nbits=nbits, mode="roll", out_dtype=torch.int32)
    rawd = torch.from_numpy(raw).cuda()
    for v in range(plan.num_variants):
        plan.set_variant(v)
        out = plan.execute(rawd, nsamps, check=True)
        np.testing.assert_array_equal(out.cpu().numpy().astype(np.float32), expect,
                                      err_msg=str(plan.describe()))
    plan.close()


def test_dmt_plan_out_stride_and_offset(torch_cuda, orc):
    torch = torch_cuda
    from sigpyproc3_b200.dedisp import DMTPlan

    rng = np.random.default_rng(9)
    nchans, nsamps = 64, 1200
    vals = rng.integers(0, 256, size=nsamps * nchans, dtype=np.uint8)
    d = np.atleast_2d(_geom_delays(nchans, np.linspace(0, 30, 5)))
    nvalid = nsamps - int(d.max())
    plan = DMTPlan(d, nchans, nsamps, nbits=8, out_dtype=torch.int32)
    out = torch.full((5, nvalid + 50), -7, dtype=torch.int32, device="cuda")
    plan.execute(torch.from_numpy(vals).cuda(), nsamps, out, out_start=20)
    o = out.cpu().numpy()
    np.testing.assert_array_equal(o[:, 20:20 + nvalid], orc.dmt(vals, d, nchans, nsamps, nvalid))
    assert np.all(o[:, :20] == -7) and np.all(o[:, 20 + nvalid:] == -7)


@pytest.mark.parametrize("acc", ["kahan", "f64"])
def test_dmt_float(torch_cuda, orc, acc):
    torch = torch_cuda
    from sigpyproc3_b200 import _lib
    from sigpyproc3_b200.dedisp import DMTPlan

    rng = np.random.default_rng(21)
    nchans, nsamps, ndm = 256, 3000, 24
    x = rng.normal(0, 1, size=(nsamps, nchans)).astype(np.float32)
    d = np.atleast_2d(_geom_delays(nchans, np.linspace(0, 50, ndm)))
    nvalid = nsamps - int(d.max())
    ref32, ref64 = orc.dmt(x.ravel(), d, nchans, nsamps, nvalid, want64=True)
    plan = DMTPlan(d, nchans, nsamps, nbits=32,
                   acc=_lib.ACC_KAHAN32 if acc == "kahan" else _lib.ACC_F64)
    xd = torch.from_numpy(x.ravel()).cuda()
    absx = np.abs(x)
    mag = orc.dmt(absx.ravel(), d, nchans, nsamps, nvalid).astype(np.float64)
    for v in range(plan.num_variants):
        plan.set_variant(v)
        out32 = plan.execute(xd, nsamps).cpu().numpy()
        if acc == "f64":
            # float64 sums in channel order, as kernels.dedisperse: the oracle's bits
            np.testing.assert_array_equal(out32, ref32, err_msg=str(plan.describe()))
            continue
        out = out32.astype(np.float64)
        err = np.abs(out - ref64)
        bound = RTOL * np.abs(ref64) + ATOL_UNIT * mag
        assert np.all(err <= bound), (v, float((err / np.maximum(np.abs(ref64), 1e-30)).max()))


def test_roll_mode_matches_dmt_block(torch_cuda, golden):
    torch = torch_cuda
    from sigpyproc3_b200 import _lib
    from sigpyproc3_b200.dedisp import DMTPlan

    blk = golden["dmt_block_in"]  # (32, 512)
    d = np.mod(golden["dmt_block_delays"], 512).astype(np.int32)
    plan = DMTPlan(d, 32, 512, nbits=32, mode="roll", acc=_lib.ACC_F64)
    out = plan.execute(torch.from_numpy(blk.T.copy().ravel()).cuda(), 512).cpu().numpy()
    np.testing.assert_allclose(out, golden["dmt_block_out"], rtol=1e-5, atol=1e-5)
    out_i = plan.execute(torch.from_numpy(golden["dmt_block_int_in"].T.copy().ravel()).cuda(), 512)
    np.testing.assert_array_equal(out_i.cpu().numpy(), golden["dmt_block_int_out"])


def test_host_streaming_execute(torch_cuda, orc):
    torch = torch_cuda
    from sigpyproc3_b200.dedisp import DMTPlan

    rng = np.random.default_rng(31)
    nchans, nsamps = 128, 20000
    vals = rng.integers(0, 4, size=nsamps * nchans, dtype=np.uint8)
    raw = _pack(vals, 2, "big")
    d = np.atleast_2d(_geom_delays(nchans, np.linspace(0, 100, 16)))
    nvalid = nsamps - int(d.max())
    plan = DMTPlan(d, nchans, nsamps, nbits=2, out_dtype=torch.int32)
    host_in = torch.from_numpy(raw).pin_memory()
    out = torch.empty((16, nvalid), dtype=torch.int32).pin_memory()
    plan.execute_host(host_in.numpy(), nsamps, out.numpy(), block_nsamps=3000)
    np.testing.assert_array_equal(out.numpy(), orc.dmt(vals, d, nchans, nsamps, nvalid))


def test_device_status_clean(torch_cuda):
    torch = torch_cuda
    from sigpyproc3_b200 import _lib
    from sigpyproc3_b200.dedisp import DMTPlan, workspace

    d = np.atleast_2d(_geom_delays(64, np.linspace(0, 20, 8)))
    plan = DMTPlan(d, 64, 2000, nbits=8)
    x = torch.zeros(2000 * 64, dtype=torch.uint8, device="cuda")
    ws = workspace(plan.workspace_bytes(2000))
    lib = _lib.load()
    _lib.check(lib.spp_status_clear(ws.data_ptr(), torch.cuda.current_stream().cuda_stream))
    plan.execute(x, 2000, ws=ws)
    words = (np.zeros(4, np.uint32))
    _lib.check(lib.spp_status_read(ws.data_ptr(), words.ctypes.data,
                                   torch.cuda.current_stream().cuda_stream))
    assert words[0] == 0
