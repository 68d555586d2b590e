"""Streaming server (config 4): every chunk's result is the same alone and in
the batched mix, and equals the oracle over the concatenated stream."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available()
    return torch


def _pack(vals, nbits, order):
    per = 8 // nbits
    v = vals.reshape(-1, per).astype(np.uint8)
    out = np.zeros(v.shape[0], dtype=np.uint8)
    for k in range(per):
        sh = (8 - (k + 1) * nbits) if order == "big" else k * nbits
        out |= (v[:, k] << sh).astype(np.uint8)
    return out


def _beams():
    from sigpyproc3_b200 import Header
    from sigpyproc3_b200.serve import BeamSpec

    specs = []
    for b, (nchans, nbits, dmmax, ndm) in enumerate(
            [(64, 8, 60.0, 37), (128, 2, 90.0, 50), (96, 4, 40.0, 20), (128, 1, 70.0, 64)]):
        h = Header(nchans=nchans, fch1=1500.0, foff=-300.0 / nchans, tsamp=64e-6, nbits=nbits)
        specs.append(BeamSpec(b, h, np.linspace(0.0, dmmax, ndm)))
    return specs


def _streams(specs, nchunks=3, seed=8):
    rng = np.random.default_rng(seed)
    data = {}
    for sp in specs:
        h = sp.header
        lens = rng.integers(3000, 9000, size=nchunks)
        vals = [rng.integers(0, 1 << h.nbits, size=n * h.nchans, dtype=np.uint8) for n in lens]
        order = "little" if h.nbits == 1 else "big"
        raws = [v if h.nbits == 8 else _pack(v, h.nbits, order) for v in vals]
        data[sp.beam_id] = (lens, vals, raws)
    return data


def test_served_equals_alone_and_oracle(torch_cuda, orc):
    torch = torch_cuda
    from sigpyproc3_b200.serve import BeamState, Chunk, Server, plain_process

    specs = _beams()
    data = _streams(specs)
    # the mix: interleave the beams' chunks
    order = [(b, k) for k in range(3) for b in range(len(specs))]
    srv = Server(specs, hbm_budget=2 << 30, keep_dmt=True, max_inflight=2)
    chunks = {}
    for b, k in order:
        lens, _, raws = data[b]
        c = Chunk(b, k, int(lens[k]), torch.from_numpy(raws[k]).pin_memory())
        chunks[(b, k)] = c
        srv.submit(c)
        if k == 1:
            srv.step()  # let a batch start while more chunks arrive
    srv.drain()
    torch.cuda.synchronize()
    for sp in specs:
        b = sp.beam_id
        lens, vals, raws = data[b]
        # alone: a fresh beam state, plain per-call path
        st = BeamState(sp, torch.device("cuda", 0))
        stream_vals = np.concatenate(vals)
        total = int(lens.sum())
        d = st.delays
        ref = orc.dmt(stream_vals, d, sp.header.nchans, total, total - st.maxd)
        pos = 0
        for k in range(3):
            alone = plain_process(None, Chunk(b, k, int(lens[k]), torch.from_numpy(raws[k])), st,
                                  keep_dmt=True)
            mixed = chunks[(b, k)]
            assert mixed.nvalid == alone.nvalid
            np.testing.assert_array_equal(mixed.dmt.cpu().numpy(), alone.dmt.cpu().numpy())
            np.testing.assert_allclose(mixed.snr, alone.snr, rtol=1e-6)
            np.testing.assert_array_equal(mixed.dmt.cpu().numpy(), ref[:, pos:pos + mixed.nvalid])
            pos += mixed.nvalid
        assert pos == ref.shape[1]


def test_admission_respects_budget(torch_cuda):
    torch = torch_cuda
    from sigpyproc3_b200.serve import Chunk, Server

    specs = _beams()[:1]
    data = _streams(specs, nchunks=4, seed=9)
    lens, _, raws = data[0]
    srv = Server(specs, hbm_budget=1, keep_dmt=False)
    with pytest.raises(ValueError):
        srv.submit(Chunk(0, 0, int(lens[0]), torch.from_numpy(raws[0])))
    one = Server(specs, hbm_budget=0, keep_dmt=False)
    one.budget = max(one.chunk_bytes(Chunk(0, k, int(lens[k]), None)) for k in range(4))
    # room for one chunk at a time (any two exceed the budget)
    assert min(one.chunk_bytes(Chunk(0, k, int(lens[k]), None)) for k in range(4)) * 2 > one.budget
    for k in range(4):
        one.submit(Chunk(0, k, int(lens[k]), torch.from_numpy(raws[k])))
    while one.pending or one.inflight:
        one.step()
        assert one.in_use <= one.budget
        assert all(len(b.chunks) == 1 for b in one.inflight)
    assert len(one.done) == 4


def test_batch_cap_keeps_two_in_flight(torch_cuda):
    """With the whole queue fitting the budget, a batch still takes at most
    half of it (max_inflight=2), so the next batch can be admitted while the
    first runs; a chunk larger than the cap goes alone."""
    torch = torch_cuda
    from sigpyproc3_b200.serve import Chunk, Server

    specs = _beams()[:1]
    data = _streams(specs, nchunks=6, seed=11)
    lens, _, raws = data[0]
    srv = Server(specs, hbm_budget=0, keep_dmt=False, max_inflight=2)
    sizes = [srv.chunk_bytes(Chunk(0, k, int(lens[k]), None)) for k in range(6)]
    srv.budget = sum(sizes) + 1
    cap = srv.budget // 2
    for k in range(6):
        srv.submit(Chunk(0, k, int(lens[k]), torch.from_numpy(raws[k])))
    seen = []
    while srv.pending or srv.inflight:
        before = srv.batches
        srv.step()
        if srv.batches > before:
            b = srv.inflight[-1]
            seen.append(len(b.chunks))
            assert len(b.chunks) == 1 or b.bytes <= cap, (b.bytes, cap)
        assert srv.in_use <= srv.budget
    assert sum(seen) == 6 and len(seen) >= 2
    assert srv.batch_sizes == seen


def test_short_first_chunks(torch_cuda, orc):
    """Chunks shorter than the max delay: outputs start once the stream covers it."""
    torch = torch_cuda
    from sigpyproc3_b200.serve import BeamState, Chunk, Server, plain_process

    spec = _beams()[0]
    st0 = BeamState(spec, torch.device("cuda", 0))
    maxd = st0.maxd
    lens = np.array([maxd // 3, maxd // 2, 4000, 100])
    rng = np.random.default_rng(12)
    vals = [rng.integers(0, 256, size=n * spec.header.nchans, dtype=np.uint8) for n in lens]
    srv = Server([spec], hbm_budget=1 << 30, keep_dmt=True)
    chunks = [Chunk(0, k, int(n), torch.from_numpy(v)) for k, (n, v) in enumerate(zip(lens, vals))]
    for c in chunks:
        srv.submit(c)
    srv.drain()
    torch.cuda.synchronize()
    total = int(lens.sum())
    ref = orc.dmt(np.concatenate(vals), st0.delays, spec.header.nchans, total, total - maxd)
    got = [c.dmt.cpu().numpy() for c in chunks if c.nvalid > 0]
    np.testing.assert_array_equal(np.concatenate(got, axis=1), ref)
    assert chunks[0].nvalid <= 0 and chunks[1].nvalid <= 0
    st = BeamState(spec, torch.device("cuda", 0))
    alone = [plain_process(None, Chunk(0, k, int(n), torch.from_numpy(v)), st, keep_dmt=True)
             for k, (n, v) in enumerate(zip(lens, vals))]
    for a, c in zip(alone, chunks):
        assert max(a.nvalid, 0) == max(c.nvalid, 0)
        if c.nvalid > 0:
            np.testing.assert_array_equal(a.dmt.cpu().numpy(), c.dmt.cpu().numpy())


def test_served_wide_beams(torch_cuda, orc):
    """Config-4-sized beams: 4096 channels of 1- and 2-bit data, chunks of
    2^14 samples and more, each chunk the same alone, in the mix and in the
    oracle over the concatenated stream."""
    torch = torch_cuda
    from sigpyproc3_b200 import Header
    from sigpyproc3_b200.serve import BeamSpec, BeamState, Chunk, Server, plain_process

    specs = []
    for b, (nbits, dmmax, ndm) in enumerate([(2, 500.0, 64), (1, 300.0, 40)]):
        h = Header(nchans=4096, fch1=1500.0, foff=-300.0 / 4096, tsamp=64e-6, nbits=nbits)
        specs.append(BeamSpec(b, h, np.linspace(0.0, dmmax, ndm)))
    rng = np.random.default_rng(44)
    data = {}
    for sp in specs:
        h = sp.header
        lens = rng.integers(1 << 14, 20000, size=3)
        vals = [rng.integers(0, 1 << h.nbits, size=n * h.nchans, dtype=np.uint8) for n in lens]
        order = "little" if h.nbits == 1 else "big"
        data[sp.beam_id] = (lens, vals, [_pack(v, h.nbits, order) for v in vals])
    srv = Server(specs, hbm_budget=8 << 30, keep_dmt=True, max_inflight=2)
    chunks = {}
    for k in range(3):
        for sp in specs:
            lens, _, raws = data[sp.beam_id]
            c = Chunk(sp.beam_id, k, int(lens[k]), torch.from_numpy(raws[k]).pin_memory())
            chunks[(sp.beam_id, k)] = c
            srv.submit(c)
        srv.step()
    srv.drain()
    torch.cuda.synchronize()
    for sp in specs:
        b = sp.beam_id
        lens, vals, raws = data[b]
        st = BeamState(sp, torch.device("cuda", 0))
        total = int(lens.sum())
        ref = orc.dmt(np.concatenate(vals), st.delays, 4096, total, total - st.maxd)
        pos = 0
        for k in range(3):
            mixed = chunks[(b, k)]
            alone = plain_process(None, Chunk(b, k, int(lens[k]), torch.from_numpy(raws[k])), st,
                                  keep_dmt=True)
            assert mixed.nvalid == alone.nvalid
            if mixed.nvalid <= 0:
                continue
            m = mixed.dmt.cpu().numpy()
            np.testing.assert_array_equal(m, alone.dmt.cpu().numpy())
            np.testing.assert_array_equal(m, ref[:, pos:pos + mixed.nvalid])
            pos += mixed.nvalid
        assert pos == ref.shape[1]
