"""In-memory filterbanks (ArrayFilterbank) are page-locked in place on first
use and their blocks copied to the GPU straight from the array; a refused
registration falls back to staging through pinned buffers.  Both paths give
the same bits, and a refusal leaves no CUDA error behind for later calls."""

import gc

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case():
    from sigpyproc3_b200 import Header

    h = Header(nchans=256, fch1=1500.0, foff=-1.0, tsamp=64e-6, nbits=8, nsamples=40000)
    raw = np.random.default_rng(5).integers(0, 256, 40000 * 256, dtype=np.uint8)
    return h, raw


def test_registered_and_staged_paths_agree(orc):
    from sigpyproc3_b200 import _lib
    from sigpyproc3_b200.readers import ArrayFilterbank

    h, raw = _case()
    first = ArrayFilterbank(raw, h)
    a = first.dedisperse(80.0, gulp=8192).data
    assert first._registered is True
    # the same memory again: the driver refuses a second registration, so the
    # second object stages its blocks; the refusal must not poison later calls
    second = ArrayFilterbank(raw, h)
    b = second.dedisperse(80.0, gulp=8192).data
    assert second._registered is False
    np.testing.assert_array_equal(a, b)
    # staged through a caller's allocator (always honoured)
    import torch

    c = first.dedisperse(80.0, gulp=8192,
                         allocator=lambda n: torch.empty(n, dtype=torch.uint8).pin_memory()).data
    np.testing.assert_array_equal(a, c)
    d = np.atleast_1d(h.get_dmdelays(80.0)).astype(np.int32)
    np.testing.assert_array_equal(a, orc.dedisperse(raw, d, 256, 40000))
    # collecting the first object releases the memory: a new one registers it
    del first
    gc.collect()
    third = ArrayFilterbank(raw, h)
    np.testing.assert_array_equal(third.dedisperse(80.0, gulp=8192).data, a)
    assert third._registered is True
    assert _lib.load().spp_version() > 0


def test_read_only_array():
    from sigpyproc3_b200.readers import ArrayFilterbank

    h, raw = _case()
    ro = raw.copy()
    ro.flags.writeable = False
    a = ArrayFilterbank(ro, h).dedisperse(40.0).data
    b = ArrayFilterbank(raw.copy(), h).dedisperse(40.0).data
    np.testing.assert_array_equal(a, b)
