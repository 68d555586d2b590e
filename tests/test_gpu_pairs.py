"""Channel-pair kernels (2-bit data): the transform regrouped as sums over
channel pairs (2k, 2k+1), each pair summed once per relative delay
r = o(2k+1) - o(2k) and shared by every DM trial that uses it.  The same
integers are added in another order, so every output must equal the
oracle's restatement of kernels.dedisperse (src/sigpyproc/core/kernels.py:
340-362) and of kernels.dmt_block (core/kernels.py:1155-1168) bit for bit.

The plan offers the pair kernels only where each tile of adjacent DM trials
reads at most two distinct rows per pair; the tests use trial grids where
that holds (consecutive trials) and check that a paired variant ran."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    assert torch.cuda.is_available(), "GPU tests need CUDA"
    return torch


def _pack2(vals):
    v = vals.reshape(-1, 4).astype(np.uint8)
    out = np.zeros(v.shape[0], dtype=np.uint8)
    for k in range(4):
        out |= (v[:, k] << (6 - 2 * k)).astype(np.uint8)
    return out


def _delays(nchans, dms, fch1, foff, tsamp):
    from sigpyproc3_b200.header import Header

    h = Header(nchans=nchans, fch1=fch1, foff=foff, tsamp=tsamp)
    return np.atleast_2d(h.get_dmdelays(np.asarray(dms, dtype=np.float64))).astype(np.int32)


def _variants(torch, plan, raw, nsamps, shape, check):
    """Run every variant; return {variant: output} and the paired ones."""
    outs, paired = {}, []
    rawd = torch.from_numpy(raw).cuda()
    out = torch.empty(shape, dtype=torch.int32, device="cuda")
    for v in range(plan.num_variants):
        plan.set_variant(v)
        out.fill_(-1)
        plan.execute(rawd, nsamps, out, check=True)
        got = out.cpu().numpy().copy()
        check(got, plan.describe())
        outs[v] = got
        if plan.describe()["paired"]:
            paired.append(v)
    return outs, paired


def test_pairs_c2_full_grid(torch_cuda, orc):
    """All 1024 trials of the config-2 grid (4096 channels, DM 0-2000) over
    4096 outputs: every variant equals the oracle on 64 sampled rows and
    equals the first variant on all rows; a paired variant is offered."""
    torch = torch_cuda
    from sigpyproc3_b200 import synth
    from sigpyproc3_b200.dedisp import DMTPlan

    nchans = 4096
    d = np.atleast_2d(synth.C2.delays(synth.dm_grid(1000.0, 1024))).astype(np.int32)
    nvalid = 4096
    nsamps = nvalid + int(d.max())
    rng = np.random.default_rng(2024)
    vals = rng.integers(0, 4, size=nsamps * nchans, dtype=np.uint8)
    rows = np.unique(np.r_[np.linspace(0, 1023, 60).astype(int), 1020, 1021, 1022, 1023])
    expect = orc.dmt(vals, d[rows], nchans, nsamps, nvalid)
    plan = DMTPlan(d, nchans, nsamps, nbits=2, bitorder="big", out_dtype=torch.int32)
    # without autotuning the plan starts from a fixed-slot pair kernel here
    assert plan.describe()["paired"] == 1, plan.describe()
    first = {}

    def check(got, desc):
        bad = np.argwhere(got[rows] != expect)
        assert bad.size == 0, (desc, bad[:5].tolist())
        if "v0" in first:
            assert np.array_equal(got, first["v0"]), desc
        else:
            first["v0"] = got.copy()

    _, paired = _variants(torch, plan, _pack2(vals), nsamps, (1024, nvalid), check)
    plan.close()
    assert paired, "no channel-pair variant offered at the config-2 grid"


@pytest.mark.parametrize("nchans", [1000, 256])
def test_pairs_partial_slab(torch_cuda, orc, nchans):
    """Channel counts whose pairs do not fill the last slab (500 pairs: 4 left
    over for 8- and 16-pair slabs), consecutive trials, random samples."""
    torch = torch_cuda
    from sigpyproc3_b200.dedisp import DMTPlan

    dms = np.linspace(0.0, 30.0, 40)
    d = _delays(nchans, dms, 1500.0, -300.0 / nchans, 64e-6)
    nvalid = 3000
    nsamps = nvalid + int(d.max())
    rng = np.random.default_rng(nchans)
    vals = rng.integers(0, 4, size=nsamps * nchans, dtype=np.uint8)
    expect = orc.dmt(vals, d, nchans, nsamps, nvalid)
    plan = DMTPlan(d, nchans, nsamps, nbits=2, bitorder="big", out_dtype=torch.int32)

    def check(got, desc):
        bad = np.argwhere(got != expect)
        assert bad.size == 0, (desc, bad[:5].tolist())

    _, paired = _variants(torch, plan, _pack2(vals), nsamps, (len(dms), nvalid), check)
    plan.close()
    assert paired


def test_pairs_roll_mode(torch_cuda, orc):
    """Roll mode: offsets are -delay, so the relative offsets of pairs are <= 0
    (partner words reach back into the halo)."""
    torch = torch_cuda
    from sigpyproc3_b200.dedisp import DMTPlan

    nchans, nsamps = 128, 4096
    dms = np.linspace(0.0, 10.0, 24)
    d = _delays(nchans, dms, 1500.0, -2.0, 64e-6)
    assert int(d.max()) < nsamps
    rng = np.random.default_rng(77)
    vals = rng.integers(0, 4, size=nsamps * nchans, dtype=np.uint8)
    expect = orc.dmt_roll(vals.astype(np.float32), d, nchans, nsamps)
    plan = DMTPlan(d, nchans, nsamps, nbits=2, bitorder="big", mode="roll",
                   out_dtype=torch.int32)

    def check(got, desc):
        np.testing.assert_array_equal(got.astype(np.float32), expect, err_msg=str(desc))

    _, paired = _variants(torch, plan, _pack2(vals), nsamps, (len(dms), nsamps), check)
    plan.close()
    assert paired


def test_pairs_not_offered_for_scattered_tables(torch_cuda):
    """Random delay tables have many distinct relative delays per pair: the
    plan keeps to the per-channel kernels."""
    torch = torch_cuda
    from sigpyproc3_b200.dedisp import DMTPlan

    rng = np.random.default_rng(5)
    d = rng.integers(0, 900, size=(16, 64)).astype(np.int32)
    plan = DMTPlan(d, 64, 2048, nbits=2, out_dtype=torch.int32)
    kinds = []
    for v in range(plan.num_variants):
        plan.set_variant(v)
        kinds.append(plan.describe()["paired"])
    plan.close()
    assert not any(kinds)


def test_pairs_host_blocks(torch_cuda, orc):
    """The end-to-end blocked path (host input, host output) with a paired
    variant: pair rows are rebuilt per block from that block's channel rows."""
    torch = torch_cuda
    from sigpyproc3_b200.dedisp import DMTPlan

    nchans = 512
    dms = np.linspace(0.0, 100.0, 64)
    d = _delays(nchans, dms, 1500.0, -0.5, 64e-6)
    nvalid = 20000
    nsamps = nvalid + int(d.max())
    rng = np.random.default_rng(91)
    vals = rng.integers(0, 4, size=nsamps * nchans, dtype=np.uint8)
    expect = orc.dmt(vals, d, nchans, nsamps, nvalid)
    plan = DMTPlan(d, nchans, nsamps, nbits=2, bitorder="big", out_dtype=torch.int32)
    paired = [v for v in range(plan.num_variants)
              if (plan.set_variant(v), plan.describe()["paired"])[1]]
    assert paired
    raw = _pack2(vals)
    for v in paired[:2]:
        plan.set_variant(v)
        out = np.full((len(dms), nvalid), -1, dtype=np.int32)
        plan.execute_host(raw, nsamps, out, block_nsamps=4096)
        np.testing.assert_array_equal(out, expect, err_msg=str(plan.describe()))
    plan.close()


def test_autotune_cache_checks_shape(torch_cuda, tmp_path):
    """A cached choice counts only while the variant it names still has the
    recorded tile shape (variant lists change between builds)."""
    import json

    torch = torch_cuda
    from sigpyproc3_b200.dedisp import DMTPlan

    nchans, nsamps = 64, 4096
    d = _delays(nchans, np.linspace(0.0, 20.0, 16), 1500.0, -4.0, 64e-6)
    rng = np.random.default_rng(3)
    raw = torch.from_numpy(_pack2(rng.integers(0, 4, size=nsamps * nchans, dtype=np.uint8))).cuda()
    cache = tmp_path / "tuned.json"
    plan = DMTPlan(d, nchans, nsamps, nbits=2, out_dtype=torch.int32)
    rec = plan.autotune(raw, nsamps, reps=1, cache=str(cache))
    key = next(iter(json.loads(cache.read_text())))
    assert plan.autotune(raw, nsamps, reps=1, cache=str(cache))["ms"] == rec["ms"]  # cache hit
    table = json.loads(cache.read_text())
    table[key]["shape"] = {"stale": 1}
    table[key]["ms"] = -1.0
    cache.write_text(json.dumps(table))
    again = plan.autotune(raw, nsamps, reps=1, cache=str(cache))
    assert again["ms"] >= 0.0 and again["shape"] == plan.describe()  # re-tuned
    assert json.loads(cache.read_text())[key]["shape"] == plan.describe()
    plan.close()
