#!/usr/bin/env python
"""Benchmark of the dedispersion path on B200: DM-trial x samples / s.

Default workload (the configuration the metric is quoted on, and the largest
that fits one GPU): fused unpack + brute-force DM-time transform of a 2-bit
filterbank, 4096 channels x 2**20 samples (tsamp 64 us, fch1 1500 MHz, foff
-0.0732421875 MHz), 1024 DM trials on the dmt_transform(1000, 1024) grid
(0-2000 pc/cm^3), exact int32 output of nsamps - max delay samples.  Seeded
synthetic data generated on the device (uniform 2-bit samples + three pulses),
bit-identical to the host twin in sigpyproc3_b200/synth.py.

One step = one DMTPlan.execute (corner turn + DM-time kernel) over the whole
input already resident in HBM.  The input (1 GiB) and output (4.2 GB) exceed
L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun each rank runs an independent replica of the workload (the
path shards without any exchange); the timed region is bracketed by a
barrier and device synchronisation, and the elapsed time is the maximum over
ranks.  --impl reference times the CPU restatement of the reference loop
(oracle/, the reference itself is Python/numba and is not installed on the
GPU host) on a bounded sample of the same workload, on rank 0 only.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from datetime import timedelta
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "DM-trial x samples/s (1 B200, bit-exact int32 DM-time transform)"
UNIT = "DM-trial*samples/s"
WORKLOAD = ("config 2: 2-bit packed filterbank, nchans=4096, nsamps=2^20, tsamp=64us, "
            "fch1=1500MHz, foff=-0.0732421875MHz, 1024 DM trials 0-2000 (dmt grid 1000+-1000), "
            "int32 DM x time output, fused unpack + brute-force transform")


def _peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"spp_clocks_{os.getpid()}.csv"

    def start(self):
        try:
            self.fp = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.fp, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fp.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        self.path.unlink(missing_ok=True)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def _dist_init():
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return rank, world, local


def _barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def _workload(args=None):
    import dataclasses

    from sigpyproc3_b200 import synth

    g = synth.C2
    ndm = 1024
    if args is not None and (args.nsamps or args.ndm):
        # reduced case for profiling captures (never a bench value)
        g = dataclasses.replace(g, nsamps=args.nsamps or g.nsamps)
        ndm = args.ndm or ndm
    # a reduced case keeps the full grid's trial spacing (a contiguous block of trials)
    lo = (1024 - ndm) // 2
    dms = synth.dm_grid(1000.0, 1024)[lo:lo + ndm]
    delays = np.atleast_2d(g.delays(dms)).astype(np.int32)
    return g, dms, delays


def cpu_sample_run(g, delays, raw_host: np.ndarray, threads: int, ndm_s: int = 64,
                   window: int = 65536) -> dict:
    """Time the CPU loop of the reference (oracle restatement) on a bounded sample:
    `ndm_s` DM trials spread over the grid, `window` output samples."""
    from oracle import oracle as orc

    orc.build()
    orc.set_threads(threads)
    maxd = int(delays.max())
    rows = window + maxd
    rb = g.nchans * g.nbits // 8
    packed = raw_host[: rows * rb]
    t0 = time.perf_counter()
    un = orc.unpack(packed, g.nbits, "big")
    t1 = time.perf_counter()
    sel = delays[np.linspace(0, delays.shape[0] - 1, ndm_s).astype(int)]
    orc.dmt_rowmajor(un, sel, g.nchans, rows, window)
    t2 = time.perf_counter()
    # the unpack is shared by all DMs; charge it pro rata to the sample's DMs
    unpack_share = (t1 - t0) * (ndm_s / delays.shape[0])
    dt = (t2 - t1) + unpack_share
    return {"value": ndm_s * window / dt, "seconds": dt, "ndm": ndm_s, "window": window}


def run_reference(args, rank, world):
    if rank != 0:
        return
    g, dms, delays = _workload()
    from sigpyproc3_b200 import synth

    rows = 65536 + int(delays.max())
    rb = g.nchans * g.nbits // 8
    raw_host = synth.c2_filterbank_host(0, rows).ravel()
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_sample_run(g, delays, raw_host, threads, ndm_s=8, window=8192)
    vals = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        vals.append(cpu_sample_run(g, delays, raw_host, threads, ndm_s=256)["value"])
    wall = time.perf_counter() - t0
    value = float(statistics.mean(vals))
    sample = "256 of 1024 DM trials (evenly spaced) x 65536 output samples per step, full 4096 channels"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * wall / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8->int32",
        "data": "synthetic (seeded, host twin of the device generator)",
        "config": {"workload": WORKLOAD, "rows_in_sample": rows},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_gpu(args, rank, world, local):
    import torch

    from sigpyproc3_b200 import synth
    from sigpyproc3_b200.dedisp import DMTPlan, workspace

    g, dms, delays = _workload(args)
    dev = torch.device("cuda", local)
    raw = synth.c2_filterbank_device(g)
    plan = DMTPlan(delays, g.nchans, g.nsamps, nbits=2, out_dtype=torch.int32)
    nvalid = plan.nvalid(g.nsamps)
    out = torch.empty((delays.shape[0], nvalid), dtype=torch.int32, device=dev)
    if args.variant is not None:
        plan.set_variant(args.variant)
        tune = {"all_ms": None, "variant": args.variant}
    else:
        tune = plan.autotune(raw, g.nsamps, out, reps=1, cache=os.environ.get("SPP_TUNE_CACHE"))
    ws = workspace(plan.workspace_bytes(g.nsamps), dev)
    for _ in range(args.warmup):
        plan.execute(raw, g.nsamps, out, ws=ws)
    torch.cuda.synchronize()
    _barrier(world)
    clocks = ClockSampler(local)
    clocks.start()
    plan.timing(True)
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    _barrier(world)
    e0.record(st)
    for _ in range(args.steps):
        plan.execute(raw, g.nsamps, out, ws=ws)
    e1.record(st)
    torch.cuda.synchronize()
    _barrier(world)
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    tk = plan.timing_read()
    plan.timing(False)
    from sigpyproc3_b200 import multi

    ms_max = multi.max_over_ranks(ms)
    units = delays.shape[0] * nvalid * args.steps
    value = world * units / (ms_max / 1e3)
    # dominant kernel roofline (DM-time kernel)
    dmt_s = tk["ms_dmt"] / max(tk["n"], 1) / 1e3
    alg_bytes = g.nsamps * g.nchans * g.nbits // 8 + delays.shape[0] * nvalid * 4
    peaks = _peaks()
    achieved = alg_bytes / dmt_s / 1e9
    traffic = None
    prof = {}
    tp = ROOT / "profiles" / "traffic.json"
    if tp.exists():
        prof = json.loads(tp.read_text())
        traffic = prof.get("k_dmt_c2_bytes_per_launch")
    adds = delays.shape[0] * nvalid * g.nchans
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
                "peak_source": peaks["source"], "kernel": "k_dmt_bits (bit-sliced)" if g.nbits <= 2 else "k_dmt",
                "kernel_ms": dmt_s * 1e3, "corner_turn_ms": tk["ms_corner_turn"] / max(tk["n"], 1),
                "int_adds_per_s": adds / dmt_s,
                # pipe utilisation of the same kernel from the committed ncu capture
                "pipes": {"alu": prof.get("alu_pipe_frac"), "lsu": prof.get("lsu_pipe_frac"),
                          "issue": prof.get("issue_active_frac"), "kernel": prof.get("kernel"),
                          "source": prof.get("pipe_source")},
                "note": "integer ALU/LSU-bound by construction (~814 adds per algorithmic byte): "
                        "the HBM fraction is low by design; the ALU-pipe fraction is the ceiling"}
    # end to end through the C ABI from pinned host buffers
    e2e = None
    cpu = None
    if rank == 0 and not args.no_e2e:
        host_in = torch.empty(raw.numel(), dtype=torch.uint8).pin_memory()
        host_in.copy_(raw.cpu())
        host_out = torch.empty((delays.shape[0], nvalid), dtype=torch.int32).pin_memory()
        blk = args.e2e_block
        hws = workspace(plan.host_workspace_bytes(blk), dev, stream=None)
        del out
        torch.cuda.empty_cache()
        plan.execute_host(host_in.numpy(), g.nsamps, host_out.numpy(), block_nsamps=blk, ws=hws)
        ne = max(1, min(args.steps, 3))
        t0 = time.perf_counter()
        for _ in range(ne):
            plan.execute_host(host_in.numpy(), g.nsamps, host_out.numpy(), block_nsamps=blk,
                              ws=hws)
        t1 = time.perf_counter()
        nblk = -(-nvalid // blk)
        h2d = sum((min(blk, nvalid - b * blk) + int(delays.max())) * g.nchans * g.nbits // 8
                  for b in range(nblk))
        e2e = {"value": delays.shape[0] * nvalid / ((t1 - t0) / ne), "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(delays.shape[0] * nvalid * 4),
               "steps": ne, "path": "spp_dmt_execute_host (C ABI), pinned host buffers"}
        # spot-check the e2e output against the device result (first row)
        if world == 1 and not args.no_cpu:
            threads = os.cpu_count() or 1
            rows = 65536 + int(delays.max())
            rb = g.nchans * g.nbits // 8
            c = cpu_sample_run(g, delays, host_in.numpy()[: rows * rb], threads, ndm_s=256)
            cpu = {"value": c["value"], "unit": UNIT, "cores": threads, "kind": "port",
                   "sample": f"{c['ndm']} of 1024 DM trials x {c['window']} output samples, "
                             f"{c['seconds']:.1f} s of CPU time"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u2->int32",
            "data": "synthetic (seeded counter-based generator on device)",
            "config": {"workload": WORKLOAD if not (args.ndm or args.nsamps) else
                       f"REDUCED profiling case ndm={args.ndm} nsamps={args.nsamps}",
                       "l2": "inputs larger than L2 (1 GiB in, 4.2 GB out)",
                       "ndm": int(delays.shape[0]), "nvalid": int(nvalid),
                       "tile": plan.describe(), "autotune_ms": tune.get("all_ms"),
                       "parallelism": f"replicas x{world}"},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": 2 * args.steps, "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    plan.close()


def _line(**kw):
    print(json.dumps(kw), flush=True)


def run_c3(args, rank, world, local):
    """Config 3: 64 beams of uneven length, two-stage subband search (32
    subbands, 512 trials 0-1000), downsample 1/2/4, boxcar widths 1..256 ->
    S/N peaks; each batch of beams is one CUDA graph of persistent launches.
    Also times the plain per-call path (one brute-force dedispersion + S/N per
    beam and DM) on a subset."""
    import torch

    from sigpyproc3_b200 import Header, multi, synth
    from sigpyproc3_b200.dedisp import dedisperse_block
    from sigpyproc3_b200.search import boxcar_snr
    from sigpyproc3_b200.subband import SubbandPlan, SubbandSearch

    g = synth.C3
    h = Header(nchans=g.nchans, fch1=g.fch1, foff=g.foff, tsamp=g.tsamp, nbits=8)
    plan = SubbandPlan(h, synth.dm_grid(500.0, 512), nsub=32, group=16)
    rng = np.random.default_rng(3)
    nbeams = args.beams
    lens = rng.integers(1 << 18, (1 << 21) + 1, size=nbeams)
    lo, hi = multi.shard_range(nbeams, rank, world)
    th = synth.gauss_u8_thresholds(96.0, 12.0)
    factors, widths = (1, 2, 4), tuple(1 << k for k in range(9))
    batch = args.batch
    # autotune the two stages on the first batch
    tune_lens = lens[lo:lo + batch]
    best, best_ms = (0, 0), None
    for v1, v2 in ((0, 0), (1, 0), (2, 0), (3, 0)):
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
    _barrier(world)
    for b0 in range(lo, hi, batch):
        blens = lens[b0:min(hi, b0 + batch)]
        srch = SubbandSearch(plan, blens, factors=factors, widths=widths, variants=best)
        for i, b in enumerate(srch.beams):
            synth.gauss_u8_device(b.raw.numel(), 3000 + b0 + i, 96.0, 12.0, out=b.raw)
        srch.capture()
        for _ in range(args.warmup):
            srch.replay()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            srch.replay()
        e1.record()
        e1.synchronize()
        total_ms += e0.elapsed_time(e1) / args.steps
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
    if rank == 0:
        _line(metric="DM-trial x samples/s, config 3 (batched two-stage subband search + S/N)",
              value=value, unit=UNIT, n_gpus=world, steps=args.steps, warmup=args.warmup,
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
              gpu_launches=None)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-block", type=int, default=65536,
                    help="output samples per host-streaming block in the e2e leg")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--variant", type=int, default=None, help="fix the kernel variant")
    ap.add_argument("--workload", choices=["c2", "c3", "c4", "c1", "c5", "snr", "fold"], default="c2")
    ap.add_argument("--beams", type=int, default=64, help="config 3: number of beams")
    ap.add_argument("--batch", type=int, default=4, help="config 3: beams per graph")
    ap.add_argument("--chunks", type=int, default=128, help="config 4: chunks served")
    ap.add_argument("--budget-gb", type=float, default=48.0, help="config 4: HBM budget")
    ap.add_argument("--ndm", type=int, default=None, help="profiling only: fewer DM trials")
    ap.add_argument("--nsamps", type=int, default=None, help="profiling only: fewer samples")
    args = ap.parse_args()
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        world = int(os.environ.get("WORLD_SIZE", "1"))
        run_reference(args, rank, world)
        return
    rank, world, local = _dist_init()
    try:
        if args.workload == "c3":
            run_c3(args, rank, world, local)
        elif args.workload == "c2":
            run_gpu(args, rank, world, local)
        else:
            from sigpyproc3_b200 import workloads

            workloads.run(args.workload, args, rank, world, local, _line)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
