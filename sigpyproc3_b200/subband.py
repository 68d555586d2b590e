"""Two-stage subband dedispersion search over many beams (R7 + R9, config 3).

Stage 1 (per DM group g with nominal DM nu_g): each subband s of consecutive
channels is dedispersed internally, relative to its highest-frequency
channel r_s:
    sub[g][s][t] = sum_{c in s} x[t + D(nu_g, c) - D(nu_g, r_s)][c]
Stage 2 (per trial DM i of group g):
    out[i][t] = sum_s sub[g][s][t + D(dm_i, r_s)]
so channel c of trial i is shifted by the effective delay
    E[i][c] = D(dm_i, r_s) + D(nu_g, c) - D(nu_g, r_s)
(D = the reference's integer delay table, params.compute_dmdelays).  The
reference has only stage 1 (kernels.subband, src/sigpyproc/core/kernels.py
:379-401, via Filterbank.subband, base.py:1030-1107); the second stage and the
DM grouping are this library's.  Integer input gives exact integer sums at
both stages (uint16 between them), so ``out`` equals a brute-force transform
with the table E -- which is how the oracle checks it.

Both stages run as persistent work-list launches covering every beam of a
batch (uneven lengths), followed by the boxcar S/N epilogue (downsample
factors x widths) per beam; the whole batch can be captured in one CUDA graph.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .batch import WorkList, planar_layout, tile_span, variant_cfg
from .header import Header
from .search import boxcar_snr


class SubbandPlan:
    def __init__(self, header: Header, dms, nsub: int = 32, group: int = 16,
                 ref_freq: str | float = "fch1"):
        h = header
        if h.nchans % nsub:
            raise ValueError(f"nchans {h.nchans} is not a multiple of nsub {nsub}")
        self.header = h
        self.nchans = h.nchans
        self.nsub = nsub
        self.cps = h.nchans // nsub
        self.dms = np.asarray(dms, dtype=np.float64)
        self.ndm = self.dms.size
        self.group = group
        self.ngroups = -(-self.ndm // group)
        freqs = h.chan_freqs
        self.ref_chan = np.array([s * self.cps + int(np.argmax(freqs[s * self.cps:(s + 1) * self.cps]))
                                  for s in range(nsub)])
        sub_of = np.arange(self.nchans) // self.cps
        nominal_idx = np.array([g * group + (min(group, self.ndm - g * group) - 1) // 2
                                for g in range(self.ngroups)])
        self.nominal = self.dms[nominal_idx]
        dn = np.atleast_2d(h.get_dmdelays(self.nominal, ref_freq)).astype(np.int64)
        rel = dn - dn[:, self.ref_chan[sub_of]]
        if rel.min() < 0:
            raise ValueError("subband reference channel is not the least-delayed channel")
        self.rel = np.ascontiguousarray(rel, dtype=np.int32)            # (ngroups, nchans)
        d = np.atleast_2d(h.get_dmdelays(self.dms, ref_freq)).astype(np.int64)
        self.dsub = np.ascontiguousarray(d[:, self.ref_chan], dtype=np.int32)  # (ndm, nsub)
        g_of = np.arange(self.ndm) // group
        self.eff = np.ascontiguousarray(self.dsub[:, sub_of].astype(np.int64) + rel[g_of],
                                        dtype=np.int32)
        self.max_rel = int(self.rel.max())
        self.max_eff = int(self.eff.max())

    def nvalid(self, nsamps: int) -> int:
        return max(0, nsamps - self.max_eff)


@dataclass
class BeamBuffers:
    raw: torch.Tensor        # raw uint8 samples (time-major)
    nsamps: int
    planar: torch.Tensor     # stage-1 planar rows
    sub: torch.Tensor        # stage-1 output rows (uint16) = stage-2 planar rows
    dmt: torch.Tensor        # (ndm, nvalid) int32
    nvalid: int
    snr: torch.Tensor | None = None
    idx: torch.Tensor | None = None


class SubbandSearch:
    """Batched search of several beams: corner turn, stage 1, stage 2, S/N."""

    def __init__(self, plan: SubbandPlan, nsamps_list, *, factors=(1, 2, 4),
                 widths=(1, 2, 4, 8, 16, 32, 64, 128, 256), nbits: int = 8,
                 variants: tuple[int, int] = (0, 0), device=None):
        if nbits != 8:
            raise NotImplementedError("subband search runs on 8-bit data")
        self.plan = plan
        self.factors = tuple(factors)
        self.widths = tuple(widths)
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.v1, self.v2 = variants
        self.cfg1 = variant_cfg(8, _lib.ACC_KAHAN32, self.v1)
        self.cfg2 = variant_cfg(16, _lib.ACC_KAHAN32, self.v2)
        p = plan
        span1 = max(tile_span(p.rel[:, s * p.cps:(s + 1) * p.cps], self.cfg1["DW"])
                    for s in range(p.nsub))
        span2 = 0
        for g in range(p.ngroups):
            span2 = max(span2, tile_span(p.dsub[g * p.group:(g + 1) * p.group], self.cfg2["DW"]))
        self.rel_dev = torch.from_numpy(p.rel).to(self.device)
        self.dsub_dev = torch.from_numpy(p.dsub).to(self.device)
        self.wl1 = WorkList(8, self.v1, device=self.device)
        self.wl2 = WorkList(16, self.v2, device=self.device)
        slot1 = self.wl1.slot_words(span1)
        slot2 = self.wl2.slot_words(span2)
        if slot1 < 0 or slot2 < 0:
            raise ValueError(f"work-list variants {variants}: a fixed slot is narrower than the "
                             "plan's tile span")
        self.beams: list[BeamBuffers] = []
        for ns in nsamps_list:
            ns = int(ns)
            nv = p.nvalid(ns)
            if nv <= 0:
                raise ValueError(f"beam of {ns} samples is shorter than the max delay {p.max_eff}")
            # stage-1 planar rows as its kernel reads them (one row per
            # channel, or eight bit-plane rows for a bit-sliced kernel)
            halo1, pitch1, rpc1 = self.wl1.layout(ns, 0, p.max_rel, slot1)
            _, pitch2 = planar_layout(16, self.cfg2["T"], nv, 0, int(p.dsub.max()), slot2)
            pitch2 = max(pitch2, int(math.ceil(ns / 2)) + 4)
            pitch2 += (-pitch2) % 4
            raw = torch.empty(ns * p.nchans, dtype=torch.uint8, device=self.device)
            planar = torch.empty(p.nchans * rpc1 * pitch1, dtype=torch.int32, device=self.device)
            sub = torch.zeros(p.ngroups * p.nsub * pitch2, dtype=torch.int32, device=self.device)
            dmt = torch.empty((p.ndm, nv), dtype=torch.int32, device=self.device)
            b = BeamBuffers(raw, ns, planar, sub, dmt, nv)
            b.halo1, b.pitch1, b.pitch2, b.rpc1 = halo1, pitch1, pitch2, rpc1
            self.beams.append(b)
            self._add_jobs(b)
        self.wl1.finalize(span1)
        self.wl2.finalize(span2)
        self.graph: torch.cuda.CUDAGraph | None = None

    def _add_jobs(self, b: BeamBuffers) -> None:
        p = self.plan
        for s in range(p.nsub):
            c0 = s * p.cps
            self.wl1.add_job(
                planar_ptr=b.planar.data_ptr() + c0 * b.rpc1 * b.pitch1 * 4, pitch_w=b.pitch1,
                halo=b.halo1,
                nchans=p.cps, delays_dev=self.rel_dev[:, c0:], delays_host=p.rel[:, c0:c0 + p.cps],
                out_ptr=b.sub.data_ptr() + s * b.pitch2 * 4, out_stride=p.nsub * b.pitch2 * 2,
                out_start=0, out_elem=2, nvalid=b.nsamps, out_kind=_lib.OUT_U16)
        for g in range(p.ngroups):
            i0, i1 = g * p.group, min(p.ndm, (g + 1) * p.group)
            self.wl2.add_job(
                planar_ptr=b.sub.data_ptr() + g * p.nsub * b.pitch2 * 4, pitch_w=b.pitch2, halo=0,
                nchans=p.nsub, delays_dev=self.dsub_dev[i0:i1], delays_host=p.dsub[i0:i1],
                out_ptr=b.dmt.data_ptr() + i0 * b.dmt.stride(0) * 4, out_stride=b.dmt.stride(0),
                out_start=0, out_elem=4, nvalid=b.nvalid, out_kind=_lib.OUT_I32)

    def run(self, stream: torch.cuda.Stream | None = None, snr: bool = True) -> None:
        """Enqueue the whole batch on `stream` (no host synchronisation)."""
        st = stream or torch.cuda.current_stream(self.device)
        p = self.plan
        for b in self.beams:
            self.wl1.corner_turn(b.raw, _lib.BITORDER_BIG, p.nchans, b.nsamps, b.halo1, b.planar,
                                 b.pitch1, stream=st)
        self.wl1.launch(st)
        self.wl2.launch(st)
        if snr:
            for b in self.beams:
                b.snr, b.idx = boxcar_snr(b.dmt, widths=self.widths, factors=self.factors,
                                          stream=st, out=(b.snr, b.idx))

    def capture(self) -> None:
        """Record the batch as one CUDA graph (after one eager run)."""
        self.run()
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.graph(g, stream=s):
            self.run(stream=s)
        torch.cuda.current_stream(self.device).wait_stream(s)
        self.graph = g

    def replay(self) -> None:
        if self.graph is None:
            self.run()
        else:
            self.graph.replay()

    def results(self) -> list[torch.Tensor]:
        return [b.snr for b in self.beams]

    def status_ok(self) -> bool:
        ok = True
        for wl in (self.wl1, self.wl2):
            ok &= int(wl.status[0].item()) == 0
        return ok
