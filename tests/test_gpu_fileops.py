"""The reference's file-writing operations on the GPU (R7, R10, N2):
Filterbank.remove_zerodm (base.py:961-1028), Filterbank.downsample
(base.py:585-654), Filterbank.subband (base.py:1030-1107),
FilterbankBlock.downsample (block.py:215-244) and the 2-D mean kernel
(kernels.downsample_2d_mean_flat, core/kernels.py:207-252), against golden
outputs of the reference's own kernels run through its read_plan block loop
(tests/golden/make_golden.py) and against the oracle."""

import hashlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available()
    return torch


def _fop_file(tmp_path, golden_meta, tag):
    from sigpyproc3_b200 import Header

    m = golden_meta["file_ops"][tag]
    rng = np.random.default_rng(m["seed"])
    n = m["nsamples"] * m["nchans"]
    if m["nbits"] == 32:
        vals = rng.normal(5.0, 2.0, n).astype(np.float32)
    else:
        vals = rng.integers(0, 256, n, dtype=np.uint8)
    assert hashlib.sha256(vals.tobytes()).hexdigest() == m["input_sha256"]
    h = Header(nchans=m["nchans"], nbits=m["nbits"], nsamples=m["nsamples"], fch1=1500.0,
               foff=-1.0, tsamp=64e-6, filename=str(tmp_path / f"{tag}.fil"))
    h.write_sigproc(tmp_path / f"{tag}.fil", vals)
    return tmp_path / f"{tag}.fil", vals, m


def _data(path, dtype):
    from sigpyproc3_b200.io import sigproc

    hdr = sigproc.read_header(path)
    return hdr, np.frombuffer(path.read_bytes()[hdr["hdrlen"]:], dtype=dtype)


@pytest.mark.parametrize("tag", ["u8", "f32"])
def test_remove_zerodm_file(torch_cuda, golden, golden_meta, orc, tmp_path, tag):
    from sigpyproc3_b200 import FilReader

    path, vals, m = _fop_file(tmp_path, golden_meta, tag)
    out = FilReader(path).remove_zerodm(str(tmp_path / "z.fil"), gulp=m["gulp"])
    hdr, data = _data(tmp_path / "z.fil", vals.dtype)
    assert (hdr["nchans"], hdr["nbits"], hdr["nsamples"]) == (m["nchans"], m["nbits"],
                                                              m["nsamples"])
    assert out.endswith("z.fil")
    ref = golden[f"fop_{tag}_zerodm"]
    if tag == "u8":
        np.testing.assert_array_equal(data, ref)  # the reference's uint8 bytes
    else:
        # the reference (fastmath) may contract a multiply-add: a last-bit difference
        np.testing.assert_allclose(data, ref, rtol=1e-6)
        assert np.mean(data == ref) > 0.999
        bp = golden["fop_f32_zerodm_bpass"]
        np.testing.assert_array_equal(data, orc.zero_dm(vals, m["nchans"], m["nsamples"], bp))


@pytest.mark.parametrize("tag", ["u8", "f32"])
def test_downsample_file(torch_cuda, golden, golden_meta, tmp_path, tag):
    from sigpyproc3_b200 import FilReader

    path, vals, m = _fop_file(tmp_path, golden_meta, tag)
    tf, ff, nch = m["tfactor"], m["ffactor"], m["nchans"]
    fil = FilReader(path)
    fil.downsample(tf, ff, str(tmp_path / "c.fil"), gulp=m["gulp"], compat=True)
    _, data = _data(tmp_path / "c.fil", vals.dtype)
    ref = golden[f"fop_{tag}_downsample_compat"]
    if tag == "u8":
        np.testing.assert_array_equal(data, ref)
    else:
        np.testing.assert_allclose(data, ref, rtol=1e-6)
    # documented semantics: tf samples x ff channels of the time-major stream
    fil.downsample(tf, ff, str(tmp_path / "d.fil"), gulp=m["gulp"])
    hdr, data = _data(tmp_path / "d.fil", vals.dtype)
    x = vals.reshape(m["nsamples"], nch).astype(np.float64)
    g2 = int(np.ceil(m["gulp"] / tf) * tf)
    parts = []
    for b0 in range(0, m["nsamples"], g2):
        blk = x[b0:b0 + g2]
        nb = blk.shape[0] // tf
        mean = blk[:nb * tf].reshape(nb, tf, nch // ff, ff).sum(axis=(1, 3)) / (tf * ff)
        parts.append(np.trunc(mean).astype(np.uint8) if tag == "u8" else mean.astype(np.float32))
    expect = np.concatenate([p_.ravel() for p_ in parts])
    np.testing.assert_array_equal(data, expect)
    assert hdr["nchans"] == nch // ff and hdr["tsamp"] == pytest.approx(64e-6 * tf)
    assert hdr["foff"] == -1.0 * ff
    with pytest.raises(ValueError):
        fil.downsample(1, 7, str(tmp_path / "x.fil"))


def test_downsample_2d_kernel_golden(torch_cuda, golden):
    torch = torch_cuda
    from sigpyproc3_b200 import _lib

    st = torch.cuda.current_stream().cuda_stream
    for tag, fn in (("u8", "spp_downsample_2d_mean_u8"), ("f32", "spp_downsample_2d_mean")):
        x = torch.from_numpy(golden[f"ds2d_{tag}_in"].ravel()).cuda()
        for f1, f2 in ((3, 2), (4, 4), (1, 8), (7, 1)):
            ref = golden[f"ds2d_{tag}_{f1}_{f2}"]
            y = torch.empty(ref.size, dtype=x.dtype, device="cuda")
            _lib.call(fn, x.data_ptr(), 1001, 48, f1, f2, y.data_ptr(), st)
            np.testing.assert_array_equal(y.cpu().numpy(), ref, err_msg=f"{tag} {f1} {f2}")


@pytest.mark.parametrize("nbits", [8, 2])
def test_subband_file(torch_cuda, orc, tmp_path, nbits):
    from sigpyproc3_b200 import FilReader, Header
    from sigpyproc3_b200.io.bits import pack_host

    nch, n, nsub, dm = 64, 6000, 8, 60.0
    vals = np.random.default_rng(90 + nbits).integers(0, 1 << nbits, n * nch, dtype=np.uint8)
    raw = vals if nbits == 8 else pack_host(vals, nbits, "big")
    h = Header(nchans=nch, nbits=nbits, nsamples=n, fch1=1510.0, foff=-1.09, tsamp=320e-6,
               filename=str(tmp_path / "s.fil"))
    h.write_sigproc(tmp_path / "s.fil", raw)
    fil = FilReader(tmp_path / "s.fil")
    fil.subband(dm, nsub, outfile_name=str(tmp_path / "s.sub"), gulp=1500)
    hdr, data = _data(tmp_path / "s.sub", np.float32)
    new_foff = h.foff * nch // nsub
    assert hdr["nchans"] == nsub and hdr["nbits"] == 32 and hdr["refdm"] == dm
    assert hdr["foff"] == new_foff and hdr["fch1"] == h.ftop - new_foff / 2
    d = np.atleast_1d(h.get_dmdelays(dm)).astype(np.int32)
    maxd = int(d.max())
    c2s = (np.arange(nch) // (nch // nsub)).astype(np.int32)
    parts, pos = [], 0
    gulp = max(2 * maxd, 1500)
    for _ii, nblk, skip in orc.read_plan_blocks(n, gulp, 0, None, maxd):
        blk = vals[pos * nch:(pos + nblk) * nch]
        if nblk > maxd:
            parts.append(orc.subband(blk, d, c2s, maxd, nch, nsub, nblk))
        pos += nblk + skip
    np.testing.assert_array_equal(data, np.concatenate(parts))


def test_block_downsample(torch_cuda):
    from sigpyproc3_b200 import FilterbankBlock, Header

    x = np.random.default_rng(7).normal(0, 1, size=(48, 1001)).astype(np.float32)
    b = FilterbankBlock(x, Header(nchans=48, nsamples=1001, tsamp=1e-3, foff=-1.0))
    d = b.downsample(ffactor=4, tfactor=3)
    assert d.data.shape == (12, 333)
    expect = x[:, :999].reshape(12, 4, 333, 3).astype(np.float64).mean(axis=(1, 3))
    np.testing.assert_allclose(d.data, expect.astype(np.float32), rtol=1e-6, atol=1e-7)
    assert d.header.nchans == 12 and d.header.tsamp == pytest.approx(3e-3)
    assert d.header.foff == -4.0 and d.header.nsamples == 1001 // 3
    with pytest.raises(ValueError):
        b.downsample(ffactor=0)
