"""Benchmark workloads other than the default DM-time transform (bench.py
--workload c1|c3|c4|c5|snr|fold|dmt).  Each prints one JSON line through ``emit``;
``measure_c1`` and ``measure_c3`` also feed the secondary blocks of the
default line."""

from __future__ import annotations

import time

import numpy as np
import torch

from . import _lib, multi, synth
from .header import Header

UNIT = "DM-trial*samples/s"


def _events():
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def run(name: str, args, rank: int, world: int, local: int, emit, checks=None) -> None:
    """Run one workload; ``checks`` maps a workload name to a correctness
    checker the caller supplies (run outside the timed region)."""
    fn = {"c1": run_c1, "c3": run_c3, "c4": run_c4, "c5": run_c5, "snr": run_snr,
          "fold": run_fold, "dmt": run_dmt}[name]
    if name == "c5":
        fn(args, rank, world, local, emit, checks or {})
    else:
        fn(args, rank, world, local, emit)


def run_c1(args, rank, world, local, emit) -> None:
    """Config 1 through the single-DM drop-in kernel (kernels.dedisperse):
    uint8 65536 x 256, DM 100, 16 rotating input copies (272 MB > L2)."""
    m = measure_c1(max(args.steps, 1))
    if rank == 0:
        emit(**m)


def measure_c1(steps: int) -> dict:
    """Config-1 measurements as the fields of one bench line (see run_c1)."""
    import json
    from pathlib import Path

    from .dedisp import dedisperse_block, workspace

    g = synth.C1
    raw_h = synth.c1_filterbank(1)
    d = np.atleast_1d(g.delays(100.0)).astype(np.int32)
    nrot = 16
    raws = [torch.from_numpy(raw_h).cuda() for _ in range(nrot)]
    dd = torch.from_numpy(d).cuda()
    nv = g.nsamps - int(d.max())
    outs = [torch.empty(nv, dtype=torch.float32, device="cuda") for _ in range(nrot)]
    lib = _lib.load()
    ws = workspace(lib.spp_dedisperse_workspace_bytes(8, g.nchans, g.nsamps, 0, int(d.max())))
    for i in range(nrot):
        dedisperse_block(raws[i], d, g.nchans, g.nsamps, outs[i], delays_dev=dd, ws=ws)
    torch.cuda.synchronize()
    ref = outs[0].cpu().numpy()
    # the 16 rotating calls as one CUDA graph: device time without host launch cost
    graph = torch.cuda.CUDAGraph()
    cs = torch.cuda.Stream()
    cs.wait_stream(torch.cuda.current_stream())
    with torch.cuda.graph(graph, stream=cs):
        for i in range(nrot):
            dedisperse_block(raws[i], d, g.nchans, g.nsamps, outs[i], delays_dev=dd, ws=ws,
                             stream=cs)
    torch.cuda.current_stream().wait_stream(cs)
    for _ in range(3):
        graph.replay()
    torch.cuda.synchronize()
    e0, e1 = _events()
    reps = steps * 4
    e0.record()
    for _ in range(reps):
        graph.replay()
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / (reps * nrot)
    # the same calls issued one by one from Python (host-bound)
    e2, e3 = _events()
    e2.record()
    for r in range(nrot * 4):
        dedisperse_block(raws[r % nrot], d, g.nchans, g.nsamps, outs[r % nrot], delays_dev=dd, ws=ws)
    e3.record()
    e3.synchronize()
    ms_eager = e2.elapsed_time(e3) / (nrot * 4)
    # context, not the product: a plain device-to-device copy of each 17 MB
    # input (torch copy_, 2x the bytes this call reads), same rotation and replay
    dsts = [torch.empty_like(r) for r in raws]
    cg = torch.cuda.CUDAGraph()
    cs.wait_stream(torch.cuda.current_stream())
    with torch.cuda.graph(cg, stream=cs):
        for i in range(nrot):
            dsts[i].copy_(raws[i])
    torch.cuda.current_stream().wait_stream(cs)
    for _ in range(3):
        cg.replay()
    e4, e5 = _events()
    e4.record()
    for _ in range(reps):
        cg.replay()
    e5.record()
    e5.synchronize()
    copy_us = e4.elapsed_time(e5) * 1e3 / (reps * nrot)
    del dsts, cg
    # the same kernel on a 16x longer block (2^20 samples, 268 MB > L2): the
    # per-launch cost amortised, what the kernel streams at
    big_n = 16 * g.nsamps
    big_raw = torch.from_numpy(np.tile(raw_h, 16)).cuda()
    big_nv = big_n - int(d.max())
    big_out = torch.empty(big_nv, dtype=torch.float32, device="cuda")
    big_ws = workspace(lib.spp_dedisperse_workspace_bytes(8, g.nchans, big_n, 0, int(d.max())))
    for _ in range(2):
        dedisperse_block(big_raw, d, g.nchans, big_n, big_out, delays_dev=dd, ws=big_ws)
    e6, e7 = _events()
    e6.record()
    for _ in range(8):
        dedisperse_block(big_raw, d, g.nchans, big_n, big_out, delays_dev=dd, ws=big_ws)
    e7.record()
    e7.synchronize()
    big_ms = e6.elapsed_time(e7) / 8
    big_gbs = (big_n * g.nchans + big_nv * 4) / (big_ms / 1e3) / 1e9
    del big_raw, big_out, big_ws
    # end to end through the public API from host memory: ArrayFilterbank over
    # the host bytes, Filterbank.dedisperse(100) with the reference's block plan
    # (pinned staging, H2D per block, one kernel per block, TimeSeries to host)
    from .readers import ArrayFilterbank, plan_blocks

    h = Header(nchans=g.nchans, fch1=g.fch1, foff=g.foff, tsamp=g.tsamp, nbits=8,
               nsamples=g.nsamps)
    fb = ArrayFilterbank(raw_h, h)
    tim = fb.dedisperse(100.0)
    assert np.array_equal(tim.data, ref)
    ne = 20
    t0 = time.perf_counter()
    for _ in range(ne):
        fb.dedisperse(100.0)
    e2e_s = (time.perf_counter() - t0) / ne
    maxd = int(np.abs(d).max())
    gulp, blocks = plan_blocks(g.nsamps, max(2 * maxd, 16384), 0, None, maxd)
    h2d = sum(nblk for _, nblk, _ in blocks) * g.nchans
    alg = g.nsamps * g.nchans + nv * 4
    peaks = json.loads((Path(__file__).resolve().parents[1] / "MEASURED_PEAKS.json").read_text()) \
        if (Path(__file__).resolve().parents[1] / "MEASURED_PEAKS.json").exists() else {"hbm_gbs": 6650.0}
    gbs = alg / (ms / 1e3) / 1e9
    del raws, outs, graph
    return dict(metric="DM-trial x samples/s, config 1 (single-DM drop-in, 8-bit 256 ch)",
             value=nv / (ms / 1e3), unit=UNIT, n_gpus=1, steps=reps, warmup=1,
             ms_per_step=ms, higher_is_better=True, scaling="weak", vs_baseline=None,
             dtype="u8->f32", data="synthetic (numpy seed 1, injected DM-100 pulse)",
             config={"workload": "config 1: Filterbank.dedisperse(100) kernel path, 16 rotating "
                     "input copies (L2-cold)"},
             roofline={"bound": "hbm", "achieved": gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                       "frac": gbs / peaks["hbm_gbs"], "algorithmic_bytes": alg,
                       "note": "single-pass 8-bit kernel (spp_dedisperse_hd), one launch per "
                               "call, CUDA-graph replay"},
             reference_copy={"us_per_call": copy_us, "bytes_moved": 2 * g.nsamps * g.nchans,
                             "note": "torch copy_ of the same 17 MB input, same replay: what one "
                                     "launch moving these bytes costs at this size"},
             long_block={"nsamps": big_n, "ms_per_call": big_ms, "achieved_gbs": big_gbs,
                         "frac": big_gbs / peaks["hbm_gbs"],
                         "note": "same kernel and DM, 16x the samples (268 MB input, eager "
                                 "launches): streaming rate without the per-launch cost"},
             eager_ms_per_call=ms_eager, pulse_at=int(np.argmax(ref)),
             e2e={"value": nv / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                  "d2h_bytes_per_step": int(nv * 4), "ms_per_call": e2e_s * 1e3,
                  "path": "ArrayFilterbank(host bytes).dedisperse(100): reference block plan "
                          f"({len(blocks)} blocks of {gulp} samples), wall clock"})


def run_c3(args, rank, world, local, emit) -> None:
    """Config 3: 64 beams of uneven length, two-stage subband search (32
    subbands, 512 trials 0-1000), downsample 1/2/4, boxcar widths 1..256 ->
    S/N peaks; each batch of beams is one CUDA graph of persistent launches.
    Also times the plain per-call path (one brute-force dedispersion + S/N per
    beam and DM) on a subset."""
    m = measure_c3(max(args.steps, 1), max(args.warmup, 1), args.beams, args.batch, rank, world)
    if rank == 0:
        emit(**m)


def measure_c3(steps: int, warmup: int, beams: int, batch: int, rank: int, world: int) -> dict:
    """Config-3 measurements as the fields of one bench line (see run_c3)."""
    from .dedisp import dedisperse_block
    from .search import boxcar_snr
    from .batch import num_variants
    from .subband import SubbandPlan, SubbandSearch

    g = synth.C3
    h = Header(nchans=g.nchans, fch1=g.fch1, foff=g.foff, tsamp=g.tsamp, nbits=8)
    plan = SubbandPlan(h, synth.dm_grid(500.0, 512), nsub=32, group=16)
    rng = np.random.default_rng(3)
    nbeams = beams
    lens = rng.integers(1 << 18, (1 << 21) + 1, size=nbeams)
    lo, hi = multi.shard_range(nbeams, rank, world)
    th = synth.gauss_u8_thresholds(96.0, 12.0)
    factors, widths = (1, 2, 4), tuple(1 << k for k in range(9))
    # autotune the two stages on the first batch
    tune_lens = lens[lo:lo + batch]
    best, best_ms = (0, 0), None
    for v1 in range(num_variants(8)):  # stage 1: bit-sliced and SIMD 8-bit kernels
        v2 = 0
        try:
            srch = SubbandSearch(plan, tune_lens, factors=factors, widths=widths,
                                 variants=(v1, v2))
        except ValueError:  # fixed slot too narrow for this plan
            continue
        for b in srch.beams:
            synth.gauss_u8_device(b.raw.numel(), 99, 96.0, 12.0, out=b.raw)
        srch.run()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        srch.run(snr=False)
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        if best_ms is None or ms < best_ms:
            best, best_ms = (v1, v2), ms
        del srch
        torch.cuda.empty_cache()
    v1 = best[0]
    best_ms = None
    for v2 in range(4):
        srch = SubbandSearch(plan, tune_lens, factors=factors, widths=widths, variants=(v1, v2))
        for b in srch.beams:
            synth.gauss_u8_device(b.raw.numel(), 99, 96.0, 12.0, out=b.raw)
        srch.run()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        srch.run(snr=False)
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        if best_ms is None or ms < best_ms:
            best, best_ms = (v1, v2), ms
        del srch
        torch.cuda.empty_cache()
    total_ms, units = 0.0, 0
    peaks = []
    torch.cuda.synchronize()
    multi.barrier()
    for b0 in range(lo, hi, batch):
        blens = lens[b0:min(hi, b0 + batch)]
        srch = SubbandSearch(plan, blens, factors=factors, widths=widths, variants=best)
        for i, b in enumerate(srch.beams):
            synth.gauss_u8_device(b.raw.numel(), 3000 + b0 + i, 96.0, 12.0, out=b.raw)
        srch.capture()
        for _ in range(warmup):
            srch.replay()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            srch.replay()
        e1.record()
        e1.synchronize()
        total_ms += e0.elapsed_time(e1) / steps
        units += sum(512 * b.nvalid for b in srch.beams)
        peaks += [float(b.snr.max()) for b in srch.beams]
        assert srch.status_ok()
        del srch
        torch.cuda.empty_cache()
    ms_max = multi.max_over_ranks(total_ms)
    units_all = multi.sum_over_ranks(units)
    value = units_all / (ms_max / 1e3)
    # plain per-call path on a subset: 2 beams x 16 DMs, brute force + S/N per call
    nsub_beams, nsub_dms = 2, 16
    dms = plan.dms[np.linspace(0, 511, nsub_dms).astype(int)]
    t_plain, u_plain = 0.0, 0
    for bi in range(nsub_beams):
        n = int(lens[bi])
        raw = synth.gauss_u8_device(n * g.nchans, 3000 + bi, 96.0, 12.0)
        d_all = np.atleast_2d(h.get_dmdelays(dms)).astype(np.int32)
        tim = torch.empty(n, dtype=torch.float32, device="cuda")
        for dmi in range(nsub_dms):  # warm
            dedisperse_block(raw, d_all[dmi], g.nchans, n, tim)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for dmi in range(nsub_dms):
            d = d_all[dmi]
            nvi = dedisperse_block(raw, d, g.nchans, n, tim)
            boxcar_snr(tim[:nvi].view(1, -1), widths=widths, factors=factors)
            u_plain += nvi
        torch.cuda.synchronize()
        t_plain += time.perf_counter() - t0
    plain = u_plain / t_plain
    brute = _c3_batched_brute_force(plan, h, lens[:min(batch, nbeams)], factors, widths, g)
    return dict(metric="DM-trial x samples/s, config 3 (batched two-stage subband search + S/N)",
              value=value, unit=UNIT, n_gpus=world, steps=steps, warmup=warmup,
              ms_per_step=ms_max, higher_is_better=True, scaling="weak", vs_baseline=None,
              dtype="u8->uint16->int32 (+f32 S/N)", data="synthetic (device generator, seeded)",
              config={"workload": f"config 3: {nbeams} beams nsamps U[2^18,2^21], 1024 ch 8-bit, "
                      "32 subbands x 16-trial groups, 512 trials 0-1000, downsample 1/2/4, "
                      "widths 1..256", "batch_beams": batch, "variants": list(best),
                      "beams_total_samples": int(lens.sum())},
              plain_per_call={"value": plain, "unit": UNIT, "path": "dedisperse_block + boxcar_snr "
                              "per (beam, DM), brute force over 1024 channels",
                              "sample": f"{nsub_beams} beams x {nsub_dms} DMs"},
              served_over_plain=value / plain, max_snr=max(peaks) if peaks else None,
              batched_brute_force={**brute, "over_plain": brute["value"] / plain},
              gpu_launches=None)


def _c3_batched_brute_force(plan, h, lens, factors, widths, g) -> dict:
    """The plain path's algorithm (every trial over every channel) with the
    batching alone: all trials of a batch of beams in one persistent
    work-list launch, then S/N per beam.  Isolates what batching adds over
    per-call dedispersion; the two-stage subband search adds the rest."""
    from .batch import WorkList, num_variants, variant_cfg
    from .search import boxcar_snr

    lib = _lib.load()
    d_all = np.atleast_2d(h.get_dmdelays(plan.dms)).astype(np.int32)
    maxd = int(d_all.max())
    dd = torch.from_numpy(d_all).cuda()
    wl = None
    for v in range(num_variants(8)):  # the first kernel whose slot holds the spread
        cand = WorkList(8, v)
        slot = cand.slot_words(cand.span_of(d_all))
        if slot > 0 and lib.spp_wl_smem_bytes(8, _lib.ACC_KAHAN32, v, slot) <= 227 * 1024:
            wl = cand
            break
    span = wl.span_of(d_all)
    slot = wl.slot_words(span)
    beams = []
    for i, n in enumerate(lens):
        n = int(n)
        nv = n - maxd
        raw = synth.gauss_u8_device(n * g.nchans, 3000 + i, 96.0, 12.0)
        halo, pitch, rpc = wl.layout(nv, 0, maxd, slot)
        planar = torch.empty(g.nchans * rpc * pitch, dtype=torch.int32, device="cuda")
        out = torch.empty((d_all.shape[0], nv), dtype=torch.int32, device="cuda")
        wl.add_job(planar_ptr=planar.data_ptr(), pitch_w=pitch, halo=halo, nchans=g.nchans,
                   delays_dev=dd, delays_host=d_all, out_ptr=out.data_ptr(),
                   out_stride=out.stride(0), out_start=0, out_elem=4, nvalid=nv,
                   out_kind=_lib.OUT_I32)
        beams.append((raw, n, halo, planar, pitch, out))
    wl.finalize(span)

    def run():
        for raw, n, halo, planar, pitch, _ in beams:
            wl.corner_turn(raw, _lib.BITORDER_BIG, g.nchans, n, halo, planar, pitch)
        wl.launch()
        for *_, out in beams:
            boxcar_snr(out, widths=widths, factors=factors)

    run()
    torch.cuda.synchronize()
    e0, e1 = _events()
    e0.record()
    run()
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    assert int(wl.status[0].item()) == 0
    units = sum(d_all.shape[0] * out.shape[1] for *_, out in beams)
    return {"value": units / (ms / 1e3), "unit": UNIT, "ms": ms, "beams": len(beams),
            "kernel": variant_cfg(8, _lib.ACC_KAHAN32, wl.variant),
            "path": "corner turns + one persistent work-list launch over every beam's 512 trials "
                    "x 1024 channels + S/N per beam"}


def run_c4(args, rank, world, local, emit) -> None:
    """Config 4: served streaming search over 32 beams vs the plain per-call path."""
    m = measure_c4(args.chunks, args.budget_gb, local, world)
    if rank == 0:
        emit(**m)


def measure_c4(nchunks: int, budget_gb: float, local: int = 0, world: int = 1) -> dict:
    """Config-4 measurements as the fields of one bench line (see run_c4)."""
    from .serve import BeamState, Chunk, Server, chunk_sizes, make_beams, plain_process

    nbeams = 32
    specs = make_beams(nbeams, seed=4)
    sizes = chunk_sizes(nchunks, seed=4)
    beam_of = np.arange(nchunks) % nbeams
    maxbytes = max(int(sizes.max()) * s.header.nchans * s.header.nbits // 8 for s in specs)
    pool = torch.empty(maxbytes, dtype=torch.uint8).pin_memory()
    pool.copy_(synth.uniform_bytes_device(maxbytes, 44).cpu())

    def mk_chunks():
        seqs = {}
        out = []
        for i in range(nchunks):
            b = int(beam_of[i])
            k = seqs.get(b, 0)
            seqs[b] = k + 1
            out.append(Chunk(b, k, int(sizes[i]), pool))
        return out

    # plain per-call capacity: sequential processing of every chunk, after one
    # untimed pass over the first 16 chunks on separate beam states (first
    # allocations of the caching allocators, library and kernel set-up)
    dev = torch.device("cuda", local)
    warm = {s.beam_id: BeamState(s, dev) for s in specs}
    for c in mk_chunks()[: min(16, nchunks)]:
        plain_process(None, c, warm[c.beam_id])
    del warm
    states = {s.beam_id: BeamState(s, dev) for s in specs}
    plain_chunks = mk_chunks()
    torch.cuda.synchronize()
    lat_plain = []
    t0 = time.perf_counter()
    for c in plain_chunks:
        t1 = time.perf_counter()
        plain_process(None, c, states[c.beam_id])
        torch.cuda.synchronize()
        lat_plain.append(time.perf_counter() - t1)
    t_plain = time.perf_counter() - t0
    units = sum(states[c.beam_id].ndm * max(c.nvalid, 0) for c in plain_chunks)
    plain_rate = nchunks / t_plain
    plain_value = units / t_plain
    # served: Poisson arrivals at 4x the plain capacity
    rng = np.random.default_rng(40)
    arrivals = np.cumsum(rng.exponential(1.0 / (4.0 * plain_rate), size=nchunks))
    arrivals -= arrivals[0]
    srv = Server(specs, hbm_budget=int(budget_gb * (1 << 30)), max_inflight=2,
                 device=local)
    stats = srv.run_arrivals(mk_chunks(), arrivals)
    return dict(metric="DM-trial x samples/s, config 4 (served streaming search, continuous batching)",
             value=stats["throughput"], unit=UNIT, n_gpus=world, steps=1, warmup=0,
             ms_per_step=stats["makespan_s"] * 1e3, higher_is_better=True, scaling="weak",
             vs_baseline=None, dtype="u1/u2/u4/u8->int32 (+f32 S/N)",
             data="synthetic (uniform random bytes, seeded)",
             config={"workload": f"config 4: {nbeams} beams, nchans in 256/1024/4096, nbits "
                     f"1/2/4/8, {nchunks} chunks of 2^14..2^18 samples with carried overlap, "
                     "DM max U[500,3000] with 256-2048 trials, Poisson arrivals at 4x the plain "
                     "capacity", "hbm_budget_gb": budget_gb},
             latency_ms={"p50": stats["p50_ms"], "p99": stats["p99_ms"]},
             batches=stats["batches"], batch_chunks=stats["batch_chunks"],
             plain_per_call={"value": plain_value, "unit": UNIT,
                             "chunks_per_s": plain_rate,
                             "latency_ms": {"p50": float(np.percentile(lat_plain, 50) * 1e3),
                                            "p99": float(np.percentile(lat_plain, 99) * 1e3)},
                             "note": "service time per chunk, processed one at a time"},
             served_over_plain=stats["throughput"] / plain_value)


def run_c5(args, rank, world, local, emit, checks=None) -> None:
    """Config 5: float32 4096 x 2^21, zero-DM, 4096 trials 0-3000, boxcar 1..512."""
    from .dedisp import DMTPlan, workspace
    from .search import boxcar_snr

    g = synth.C5
    nsamps = args.nsamps or g.nsamps
    ndm = args.ndm or 4096
    lo = (4096 - ndm) // 2  # profiling cases: a contiguous block of the full grid's trials
    dms = synth.dm_grid(1500.0, 4096)[lo:lo + ndm]
    d = np.atleast_2d(g.delays(dms)).astype(np.int32)
    x = synth.gauss_f32_device(nsamps * g.nchans, 5)
    h = Header(nchans=g.nchans, fch1=g.fch1, foff=g.foff, tsamp=g.tsamp, nbits=32,
               nsamples=nsamps)
    nv = nsamps - int(d.max())
    out = torch.empty((ndm, nv), dtype=torch.float32, device="cuda")
    # float64 channel-ordered sums (the reference's accumulator; the oracle's
    # bits); --acc kahan selects the compensated float32 variants instead.
    # The tile shape is picked by timing one transform of each variant
    # (--variant fixes one, for profiling).
    acc_sel = _lib.ACC_KAHAN32 if getattr(args, "acc", "f64") == "kahan" else _lib.ACC_F64
    tune = []
    for acc in (acc_sel,) if args.variant is None else ():
        p = DMTPlan(d, g.nchans, nsamps, nbits=32, acc=acc)
        for v in range(p.num_variants):
            p.set_variant(v)
            p.execute(x, nsamps, out)
            e0, e1 = _events()
            e0.record()
            p.execute(x, nsamps, out)
            e1.record()
            e1.synchronize()
            tune.append((e0.elapsed_time(e1), acc, v))
        p.close()
    best = min(tune) if tune else (0.0, acc_sel, args.variant)
    plan = DMTPlan(d, g.nchans, nsamps, nbits=32, acc=best[1])
    plan.set_variant(best[2])
    widths = tuple(1 << k for k in range(10))
    bp = torch.zeros(g.nchans, dtype=torch.float32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream

    def step():
        bp.zero_()
        _lib.call("spp_bandpass", x.data_ptr(), 32, 0, g.nchans, nsamps, bp.data_ptr(), st)
        w = bp / bp.sum()
        plan.execute_zero_dm(x, nsamps, bp, w, out)
        return boxcar_snr(out, widths=widths, factors=(1,))

    step()
    torch.cuda.synchronize()
    plan.timing(True)
    e0, e1 = _events()
    e0.record()
    for _ in range(max(args.steps, 1)):
        snr, idx = step()
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / max(args.steps, 1)
    tk = plan.timing_read()
    dmt_ms = tk["ms_dmt"] / max(tk["n"], 1)
    adds = ndm * nv * g.nchans
    # per-result error against float64 sums, by the caller's checker (outside the timing)
    checks = checks or {}
    accuracy = checks["c5"](x, bp, out, d, g.nchans, nsamps) if "c5" in checks else None
    if rank == 0:
        emit(metric="DM-trial x samples/s, config 5 (float32 zero-DM + DM-time + boxcar S/N)",
             value=ndm * nv / (ms / 1e3), unit=UNIT, n_gpus=world, steps=args.steps, warmup=1,
             ms_per_step=ms, higher_is_better=True, scaling="weak", vs_baseline=None,
             dtype="f32 in, f64 channel-ordered sums" if best[1] == _lib.ACC_F64 else
                   "f32 (fp32 slab partials, compensated sum across slabs)",
             data="synthetic N(0,1) on device (seed 5)",
             config={"workload": f"config 5: float32 {g.nchans} ch x {nsamps}, zero-DM, {ndm} "
                     "trials 0-3000, boxcar widths 1..512", "tile": plan.describe(),
                     "accumulator": "fp64" if best[1] == _lib.ACC_F64 else
                     "fp32 slab partials + Kahan across slabs",
                     "autotune_ms": [round(t[0], 2) for t in tune]},
             kernel_ms={"dmt": dmt_ms, "corner_turn_zero_dm": tk["ms_corner_turn"] / max(tk["n"], 1)},
             adds_per_s=adds / (dmt_ms / 1e3), max_snr=float(snr.max()), accuracy=accuracy)
    plan.close()


def run_snr(args, rank, world, local, emit) -> None:
    """The boxcar S/N epilogue alone (R8 + R9) on a config-3-shaped DM-time
    block: 512 int32 rows x 2^20 samples, downsample 1/2/4, widths 1..256."""
    import json
    from pathlib import Path

    from .search import boxcar_snr

    nrows, n = args.ndm or 512, args.nsamps or (1 << 20)
    rows = synth.uniform_bytes_device(nrows * n * 4, 9).view(torch.int32).view(nrows, n)
    rows.bitwise_and_(0x3FFF)  # values of a 1024-channel 8-bit sum range
    factors, widths = (1, 2, 4), tuple(1 << k for k in range(9))
    snr = torch.empty((nrows, 3, 9), dtype=torch.float32, device="cuda")
    idx = torch.empty_like(snr, dtype=torch.int32)
    for _ in range(max(args.warmup, 1)):
        boxcar_snr(rows, widths=widths, factors=factors, out=(snr, idx))
    torch.cuda.synchronize()
    e0, e1 = _events()
    e0.record()
    for _ in range(max(args.steps, 1)):
        boxcar_snr(rows, widths=widths, factors=factors, out=(snr, idx))
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / max(args.steps, 1)
    alg = nrows * n * 4 * len(factors) + snr.numel() * 8  # each factor reads the rows once
    pk = Path(__file__).resolve().parents[1] / "MEASURED_PEAKS.json"
    peak = json.loads(pk.read_text())["hbm_gbs"] if pk.exists() else 6650.0
    if rank == 0:
        emit(metric="row-samples/s, boxcar S/N epilogue (downsample 1/2/4 x widths 1..256)",
             value=nrows * n / (ms / 1e3), unit="row-samples/s", n_gpus=world,
             steps=args.steps, warmup=args.warmup, ms_per_step=ms, higher_is_better=True,
             scaling="weak", vs_baseline=None, dtype="int32 -> f64 sums -> f32 S/N",
             data="synthetic uniform int32 rows on device (seed 9)",
             config={"workload": f"S/N epilogue: {nrows} rows x {n} samples (config-3 rows)"},
             roofline={"bound": "hbm", "achieved": alg / (ms / 1e3) / 1e9, "peak": peak,
                       "unit": "GB/s", "frac": alg / (ms / 1e3) / 1e9 / peak,
                       "algorithmic_bytes": alg})


def run_dmt(args, rank, world, local, emit) -> None:
    """DM-time transform of one block of seeded uniform samples of any width
    on the config-2 band (4096 channels from 1500 MHz down 300 MHz, 64 us):
    ``--nbits`` 1/2/4/8, ``--ndm`` trials (a contiguous block from the middle
    of the dmt_transform(1000, 1024) grid; all 1024 by default), ``--nsamps``
    output samples (2^18 by default).  Every kernel variant the plan accepts
    is timed (``--variant`` fixes one), corner turn and DM-time kernel
    separately; the line's value is the fastest kernel's channel-adds/s.
    For comparing the SIMD and bit-sliced kernels, and as the command of
    kernel captures."""
    from .dedisp import DMTPlan

    g = synth.C2
    nb = args.nbits
    ndm = args.ndm or 1024
    nout = args.nsamps or (1 << 18)
    lo = (1024 - ndm) // 2
    d = np.atleast_2d(g.delays(synth.dm_grid(1000.0, 1024)[lo:lo + ndm])).astype(np.int32)
    nsamps = nout + int(d.max())
    raw = synth.uniform_bytes_device(nsamps * g.nchans * nb // 8, 7)
    out = torch.empty((ndm, nout), dtype=torch.int32, device="cuda")
    plan = DMTPlan(d, g.nchans, nsamps, nbits=nb, bitorder="little" if nb == 1 else "big",
                   out_dtype=torch.int32)
    steps = max(args.steps, 1)
    rows = []
    for v in range(plan.num_variants) if args.variant is None else [args.variant]:
        plan.set_variant(v)
        for _ in range(max(args.warmup, 1)):
            plan.execute(raw, nsamps, out)
        torch.cuda.synchronize()
        plan.timing(True)
        for _ in range(steps):
            plan.execute(raw, nsamps, out)
        t = plan.timing_read()
        plan.timing(False)
        ms = t["ms_dmt"] / steps
        rows.append({"variant": v, "ms_dmt": ms, "ms_corner_turn": t["ms_corner_turn"] / steps,
                     "adds_per_s": ndm * nout * g.nchans / (ms / 1e3), **plan.describe()})
    plan.close()
    best = max(rows, key=lambda r: r["adds_per_s"])
    if rank == 0:
        emit(metric="channel-adds/s, DM-time kernel (kernel comparison)",
             value=best["adds_per_s"], unit="adds/s", n_gpus=world, steps=steps,
             warmup=args.warmup, ms_per_step=best["ms_dmt"], higher_is_better=True,
             scaling="weak", vs_baseline=None, dtype=f"u{nb}->int32",
             data="synthetic uniform bytes on device (seed 7)",
             config={"workload": f"DM-time transform, {nb}-bit 4096 ch x {nout} outputs, "
                     f"{ndm} trials of dmt_transform(1000, 1024) (config-2 band)",
                     "variants": rows})


def run_fold(args, rank, world, local, emit) -> None:
    """Filterbank.fold end to end from host memory: 8-bit 256 channels x 2^20
    samples (config-1 band, 16x longer), period 50.3 ms, DM 100, the reference's
    defaults (50 bins, 32 subintegrations, 32 subbands, gulp 16384)."""
    from .readers import ArrayFilterbank

    g = synth.C1
    n = 16 * g.nsamps
    raw = np.random.default_rng(7).integers(0, 256, size=n * g.nchans, dtype=np.uint8)
    h = Header(nchans=g.nchans, fch1=g.fch1, foff=g.foff, tsamp=g.tsamp, nbits=8, nsamples=n)
    fb = ArrayFilterbank(raw, h)
    for _ in range(max(args.warmup, 1)):
        fb.fold(0.0503, 100.0)
    torch.cuda.synchronize()
    reps = max(args.steps, 1)
    t0 = time.perf_counter()
    for _ in range(reps):
        fd = fb.fold(0.0503, 100.0)
    dt = (time.perf_counter() - t0) / reps
    nvalid = n - int(np.atleast_1d(h.get_dmdelays(100.0)).max())
    if rank == 0:
        emit(metric="folded samples/s (Filterbank.fold, host array in, cube out)",
             value=n / dt, unit="samples/s", n_gpus=world, steps=reps, warmup=args.warmup,
             ms_per_step=dt * 1e3, higher_is_better=True, scaling="weak", vs_baseline=None,
             dtype="u8 -> f32 cells", data="synthetic uniform bytes (numpy seed 7)",
             config={"workload": f"fold: 8-bit {g.nchans} ch x {n}, period 50.3 ms, DM 100, "
                                 "50 bins x 32 subints x 32 subbands, gulp 16384"},
             e2e={"value": n / dt, "unit": "samples/s", "h2d_bytes_per_step": int(n * g.nchans),
                  "d2h_bytes_per_step": int(fd.data.nbytes * 2), "ms_per_call": dt * 1e3,
                  "path": "ArrayFilterbank(host bytes).fold, wall clock"},
             folded_channel_samples=int(nvalid * g.nchans))
