"""Device-side failure path: a bounded wait that runs out reports through the
status word and leaves the context usable (no trap, no fault)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_reports():
    import torch

    from sigpyproc3_b200 import _lib
    from sigpyproc3_b200.dedisp import dedisperse_block

    lib = _lib.load()
    st = torch.cuda.current_stream().cuda_stream
    ws = torch.zeros(256, dtype=torch.uint8, device="cuda")
    _lib.check(lib.spp_selftest_wait_timeout(ws.data_ptr(), 5_000_000, st))  # 5 ms
    words = np.zeros(4, np.uint32)
    rc = lib.spp_status_read(ws.data_ptr(), words.ctypes.data, st)
    assert rc == _lib.SPP_ERR_DEVICE
    assert words[0] & 1  # SPP_DEV_TIMEOUT
    _lib.check(lib.spp_status_clear(ws.data_ptr(), st))
    assert lib.spp_status_read(ws.data_ptr(), words.ctypes.data, st) == 0
    # the context still runs kernels
    x = torch.arange(64 * 100, dtype=torch.int32).remainder(256).to(torch.uint8).cuda()
    out = torch.zeros(100, device="cuda")
    dedisperse_block(x, np.zeros(64, np.int32), 64, 100, out)
    np.testing.assert_array_equal(out.cpu().numpy(),
                                  x.cpu().numpy().reshape(100, 64).sum(1).astype(np.float32))
    with pytest.raises(ValueError):
        _lib.check(lib.spp_selftest_wait_timeout(ws.data_ptr(), 5_000_000_000, st))
