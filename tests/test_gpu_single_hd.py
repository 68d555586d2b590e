"""Single-DM 8-bit dedispersion through spp_dedisperse_hd (offsets precomputed
from the host delay table, kernels.dedisperse core/kernels.py:340-362)
against the oracle and against the device-table path."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available()
    return torch


def _delays(nchans, dm, ref="fch1", fch1=1510.0, foff=-1.09, tsamp=320e-6):
    from sigpyproc3_b200.header import Header

    h = Header(nchans=nchans, fch1=fch1, foff=foff, tsamp=tsamp)
    return np.atleast_1d(h.get_dmdelays(dm, ref)).astype(np.int32)


def _run(torch, vals, d, nchans, nsamps, host_table, out_start=0, fill=-7.0):
    from sigpyproc3_b200 import _lib
    from sigpyproc3_b200.dedisp import dedisperse_block

    nvalid = nsamps - int(np.abs(d).max())
    out = torch.full((max(nvalid, 0) + out_start + 5,), fill, device="cuda")
    raw = torch.from_numpy(vals).cuda()
    lib = _lib.load()
    ws = torch.zeros(max(lib.spp_dedisperse_workspace_bytes(8, nchans, nsamps, int(d.min()),
                                                            int(d.max())), 256),
                     dtype=torch.uint8, device="cuda")
    n = dedisperse_block(raw, d, nchans, nsamps, out, out_start=out_start, host_table=host_table,
                         ws=ws)
    torch.cuda.synchronize()
    return n, out.cpu().numpy()


@pytest.mark.parametrize("nchans,nsamps,dm,ref", [
    (32, 700, 3.0, "fch1"), (64, 3001, 40.0, "fch1"), (64, 3001, 40.0, "fcenter"),
    (96, 20000, 25.0, "fch1"), (256, 65536, 100.0, "fch1"), (256, 9000, 60.0, "fcenter"),
    (512, 12000, 20.0, "fch1"), (1024, 6000, 4.0, "fcenter"), (256, 1400, 3.0, "fch1"),
    (256, 300000, 30.0, "fch1"),
])
def test_host_table_matches_oracle_and_device_path(torch_cuda, orc, nchans, nsamps, dm, ref):
    torch = torch_cuda
    rng = np.random.default_rng(nchans * 7 + nsamps)
    vals = rng.integers(0, 256, size=nsamps * nchans, dtype=np.uint8)
    d = _delays(nchans, dm, ref, foff=-300.0 / nchans)
    expect = orc.dedisperse(vals, d, nchans, nsamps)
    n1, o1 = _run(torch, vals, d, nchans, nsamps, True, out_start=3)
    n2, o2 = _run(torch, vals, d, nchans, nsamps, False, out_start=3)
    assert n1 == n2 == expect.size
    np.testing.assert_array_equal(o1[3:3 + n1], expect)
    np.testing.assert_array_equal(o2[3:3 + n2], expect)
    # nothing written outside [out_start, out_start + nvalid)
    assert (o1[:3] == -7.0).all() and (o1[3 + n1:] == -7.0).all()


def test_host_table_random_delays(torch_cuda, orc):
    """Arbitrary (unsorted, negative) delays: staged rows wrap at both ends."""
    torch = torch_cuda
    rng = np.random.default_rng(11)
    for nchans, nsamps in ((64, 5000), (160, 2500), (256, 4097), (256, 70001)):
        vals = rng.integers(0, 256, size=nsamps * nchans, dtype=np.uint8)
        d = rng.integers(-300, 300, size=nchans).astype(np.int32)
        expect = orc.dedisperse(vals, d, nchans, nsamps)
        n, o = _run(torch, vals, d, nchans, nsamps, True)
        np.testing.assert_array_equal(o[:n], expect)


def test_host_table_unsupported_shapes_fall_back(torch_cuda, orc):
    torch = torch_cuda
    from sigpyproc3_b200.dedisp import dedisperse_block

    rng = np.random.default_rng(3)
    nchans, nsamps = 72, 2000          # not a multiple of 32
    vals = rng.integers(0, 256, size=nsamps * nchans, dtype=np.uint8)
    d = _delays(nchans, 10.0)
    out = torch.zeros(nsamps, device="cuda")
    with pytest.raises(NotImplementedError):
        dedisperse_block(torch.from_numpy(vals).cuda(), d, nchans, nsamps, out, host_table=True)
    n, o = _run(torch, vals, d, nchans, nsamps, None)   # auto: device-table path
    np.testing.assert_array_equal(o[:n], orc.dedisperse(vals, d, nchans, nsamps))
    # a delay spread too wide for shared memory -> unsupported on the host-table path
    nchans, nsamps = 1024, 30000
    vals = rng.integers(0, 256, size=nsamps * nchans, dtype=np.uint8)
    d = ((np.arange(nchans, dtype=np.int32) * 20) % 9000).astype(np.int32)
    with pytest.raises(NotImplementedError):
        dedisperse_block(torch.from_numpy(vals).cuda(), d, nchans, nsamps,
                         torch.zeros(nsamps, device="cuda"), host_table=True)


def test_host_table_size_checks(torch_cuda):
    torch = torch_cuda
    from sigpyproc3_b200.dedisp import dedisperse_block

    vals = np.zeros(64 * 500, np.uint8)
    d = np.arange(64, dtype=np.int32)
    small = torch.zeros(10, device="cuda")
    with pytest.raises(ValueError):
        dedisperse_block(torch.from_numpy(vals).cuda(), d, 64, 500, small, host_table=True)
    # max delay >= nsamps: nothing to do
    d = np.full(64, 500, np.int32)
    assert dedisperse_block(torch.from_numpy(vals).cuda(), d, 64, 500, small, host_table=True) == 0
