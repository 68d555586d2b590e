"""The allocation-free single-DM entry point (spp_dedisperse_noalloc).

It exists for callers that may not allocate device memory while running --
a real-time pipeline that reserves its memory up front, or a host framework
whose allocator owns the device memory -- and keeps its scratch in a fixed
array inside the library.  Checked through the C ABI against the regular
spp_dedisperse (bit-exact for integer data), on two consecutive calls with
different inputs, against the oracle's restatement of kernels.dedisperse
(src/sigpyproc/core/kernels.py:340-362), for its status words (read through
spp_dedisperse_noalloc_status_read) and for its size limit.  Collected last
on purpose.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call_regular(lib, torch, x, nbits, nchans, nsamps, d_dev, dmin, dmax, out, acc):
    need = lib.spp_dedisperse_workspace_bytes(nbits, nchans, nsamps, dmin, dmax)
    ws = torch.empty(need, dtype=torch.uint8, device="cuda")
    rc = lib.spp_dedisperse(x.data_ptr(), nbits, 0, nchans, nsamps, d_dev.data_ptr(), dmin, dmax,
                            out.data_ptr(), out.numel(), 0, acc, ws.data_ptr(), ws.numel(),
                            torch.cuda.current_stream().cuda_stream)
    assert rc == 0, lib.spp_last_error_string()


def _status(lib, st):
    words = np.zeros(4, dtype=np.uint32)
    rc = lib.spp_dedisperse_noalloc_status_read(words.ctypes.data, st)
    return rc, words


def test_noalloc_matches_regular_twice(orc):
    import torch

    from sigpyproc3_b200 import _lib
    from sigpyproc3_b200.header import Header

    assert torch.cuda.is_available()
    lib = _lib.load()
    st = torch.cuda.current_stream().cuda_stream
    h = Header(nchans=256, fch1=1500.0, foff=-1.0, tsamp=64e-6, nbits=8)
    nsamps = 32768
    rng = np.random.default_rng(123)
    for call, (dm, nbits) in enumerate(((100.0, 8), (40.0, 2))):
        d = np.atleast_1d(h.get_dmdelays(dm)).astype(np.int32)
        dmin, dmax = int(d.min()), int(d.max())
        vals = rng.integers(0, 1 << nbits, size=nsamps * 256, dtype=np.uint8)
        if nbits == 2:
            packed = np.zeros(vals.size // 4, dtype=np.uint8)
            for k in range(4):
                packed |= (vals[k::4] << (6 - 2 * k)).astype(np.uint8)
            vals = packed
        expect = orc.dedisperse(vals if nbits == 8 else orc.unpack(vals, 2, "big"), d, 256,
                                nsamps)
        x = torch.from_numpy(vals).cuda()
        d_dev = torch.from_numpy(d).cuda()
        nv = nsamps - max(abs(dmin), abs(dmax))
        ref = torch.zeros(nv, device="cuda")
        _call_regular(lib, torch, x, nbits, 256, nsamps, d_dev, dmin, dmax, ref, _lib.ACC_F64)
        out = torch.full((nv,), -1.0, device="cuda")
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        rc = lib.spp_dedisperse_noalloc(x.data_ptr(), nbits, 0, 256, nsamps, d_dev.data_ptr(), dmin,
                                        dmax, out.data_ptr(), out.numel(), 0, _lib.ACC_F64, st)
        assert rc == 0, lib.spp_last_error_string()
        torch.cuda.synchronize()
        if call > 0:  # the first call looks up the scratch address; none allocates
            assert torch.cuda.mem_get_info()[0] == free0
        np.testing.assert_array_equal(out.cpu().numpy(), ref.cpu().numpy())
        np.testing.assert_array_equal(out.cpu().numpy(), expect)
        rc, words = _status(lib, st)
        assert rc == _lib.SPP_OK and words[0] == 0, words


def test_noalloc_status_reports_clamped_delays(orc):
    """A declared delay range narrower than the table: the kernel clamps the
    outliers (no access leaves the staged rows), flags them, and the status
    read reports it; the next correct call clears the flag."""
    import torch

    from sigpyproc3_b200 import _lib
    from sigpyproc3_b200.header import Header

    lib = _lib.load()
    st = torch.cuda.current_stream().cuda_stream
    h = Header(nchans=256, fch1=1500.0, foff=-1.0, tsamp=64e-6, nbits=8)
    nsamps = 16384
    d = np.atleast_1d(h.get_dmdelays(100.0)).astype(np.int32)
    vals = np.random.default_rng(7).integers(0, 256, size=nsamps * 256, dtype=np.uint8)
    x = torch.from_numpy(vals).cuda()
    d_dev = torch.from_numpy(d).cuda()
    dmin, dmax = int(d.min()), int(d.max())
    out = torch.zeros(nsamps, device="cuda")
    rc = lib.spp_dedisperse_noalloc(x.data_ptr(), 8, 0, 256, nsamps, d_dev.data_ptr(), dmin,
                                    dmax - 300, out.data_ptr(), out.numel(), 0, _lib.ACC_F64, st)
    assert rc == _lib.SPP_OK
    rc, words = _status(lib, st)
    assert rc == _lib.SPP_ERR_DEVICE and (words[0] & 2), words
    assert b"device status" in ctypes.string_at(lib.spp_last_error_string())
    rc = lib.spp_dedisperse_noalloc(x.data_ptr(), 8, 0, 256, nsamps, d_dev.data_ptr(), dmin, dmax,
                                    out.data_ptr(), out.numel(), 0, _lib.ACC_F64, st)
    assert rc == _lib.SPP_OK
    rc, words = _status(lib, st)
    assert rc == _lib.SPP_OK and words[0] == 0, words
    np.testing.assert_array_equal(out[:nsamps - dmax].cpu().numpy(),
                                  orc.dedisperse(vals, d, 256, nsamps))


def test_noalloc_rejects_oversized_block():
    import torch

    from sigpyproc3_b200 import _lib

    lib = _lib.load()
    limit = lib.spp_dedisperse_noalloc_max_bytes()
    assert limit == 32 << 20
    nchans, nsamps = 4096, 1 << 16  # planar scratch ~ 4096 * 16K words * 4 B > 32 MiB
    x = torch.zeros(nsamps * nchans, dtype=torch.uint8, device="cuda")
    d = torch.zeros(nchans, dtype=torch.int32, device="cuda")
    out = torch.zeros(nsamps, device="cuda")
    rc = lib.spp_dedisperse_noalloc(x.data_ptr(), 8, 0, nchans, nsamps, d.data_ptr(), 0, 0,
                                    out.data_ptr(), out.numel(), 0, _lib.ACC_F64,
                                    torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.SPP_ERR_SIZE
    assert b"fixed" in ctypes.string_at(lib.spp_last_error_string())
