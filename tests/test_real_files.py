"""Real-file parity (the on-disk format feeding the path): the reference's own
sigproc test files (tests/data/parkes_{1,2,4}bit.fil, parkes_8bit_{1,2}.fil,
tutorial_2bit.fil), dedispersed by Filterbank.dedisperse (base.py:360-424)
through FilReader's block loop, against the reference's output recorded by
tests/golden/make_golden.py.

The files themselves are copied next to the vectors (tests/golden/_ref/, not
under version control) by the same script; every test here skips when they
are absent and checks each file's sha256 before use."""

import hashlib
from pathlib import Path

import numpy as np
import pytest

REF = Path(__file__).resolve().parent / "golden" / "_ref"
NAMES = ["parkes_1bit", "parkes_2bit", "parkes_4bit", "parkes_8bit_1", "parkes_8bit_2",
         "tutorial_2bit"]


def _path(name, golden_meta):
    p = REF / f"{name}.fil"
    if not p.is_file():
        pytest.skip(f"{p.name} not present (made by tests/golden/make_golden.py)")
    assert hashlib.sha256(p.read_bytes()).hexdigest() == golden_meta["files"][name]["sha256"]
    return p


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_reference_on_file(orc, golden, golden_meta, name):
    """The oracle's block loop over the file bytes equals the reference output."""
    from sigpyproc3_b200.io import sigproc

    p = _path(name, golden_meta)
    m = golden_meta["files"][name]
    hdr = sigproc.read_header(p)
    raw = np.frombuffer(p.read_bytes(), dtype=np.uint8)[hdr["hdrlen"]:]
    nbits, nch, nsamples = m["nbits"], m["nchans"], m["nsamples"]
    vals = raw if nbits == 8 else orc.unpack(raw, nbits, "little" if nbits == 1 else "big")
    d = golden[f"file_{name}_delays"]
    maxd = m["maxdelay"]
    tim = np.zeros(nsamples - maxd, dtype=np.float32)
    pos = 0
    for ii, nblk, skip in orc.read_plan_blocks(nsamples, m["gulp"], 0, None, maxd):
        blk = vals[pos * nch:(pos + nblk) * nch]
        orc.dedisperse(blk, d, nch, nblk, tim, ii * (m["gulp"] - maxd))
        pos += nblk + skip
    np.testing.assert_array_equal(tim, golden[f"file_{name}_tim"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_filreader_dedisperse_real_file(golden, golden_meta, name):
    import torch

    from sigpyproc3_b200 import FilReader

    assert torch.cuda.is_available()
    p = _path(name, golden_meta)
    m = golden_meta["files"][name]
    fil = FilReader(p)
    assert (fil.header.nbits, fil.header.nchans, fil.header.nsamples) == (
        m["nbits"], m["nchans"], m["nsamples"])
    np.testing.assert_array_equal(
        np.atleast_1d(fil.header.get_dmdelays(m["dm"])).astype(np.int32),
        golden[f"file_{name}_delays"])
    tim = fil.dedisperse(m["dm"])
    assert tim.header.dm == m["dm"] and tim.header.nchans == 1
    np.testing.assert_array_equal(tim.data, golden[f"file_{name}_tim"])  # bit-exact
    # a smaller gulp: more blocks, same series
    tim2 = fil.dedisperse(m["dm"], gulp=2 * m["maxdelay"] + 7)
    np.testing.assert_array_equal(tim2.data, golden[f"file_{name}_tim"])
