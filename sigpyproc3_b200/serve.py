"""Streaming dedispersion server (config 4): continuous batching of chunks
from many beams on one GPU.

Each beam has its own geometry (nchans, nbits, band), DM trials and delay
table, resident in HBM for the life of the beam ("DM plan" state), and a
device-resident overlap tail: the last ``maxd`` raw rows of its stream
(right-aligned; ``hist`` of them are real once the stream is shorter than
``maxd``).  A chunk of ``n`` new samples is processed as [tail | chunk] from
the first real row, which yields ``hist + n - maxd`` new DM-time samples per
trial (``n`` once the tail is full) -- exactly the outputs of running
Filterbank.dedisperse over the concatenated stream.

The server loop admits arrived chunks in FIFO order while their working set
(raw + planar + DM-time output) fits the HBM budget, groups the admitted
chunks into one batch -- one persistent work-list launch per sample width
present -- and keeps up to ``max_inflight`` batches on the device at once on
separate streams, so chunks that arrive while others run join the next batch
as soon as a slot and memory free up.  Per chunk the boxcar S/N epilogue
reduces the DM-time rows to S/N peaks, which are the only bytes copied back.
Latency is measured from arrival to the completion event of its batch.
"""

from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .batch import WorkList, corner_turn, counter_fits, planar_layout, tile_span, variant_cfg
from .header import Header
from .search import boxcar_snr


@dataclass
class BeamSpec:
    beam_id: int
    header: Header
    dms: np.ndarray


@dataclass
class Chunk:
    beam_id: int
    seq: int
    nsamps: int
    data: np.ndarray | torch.Tensor   # raw bytes (host pinned or device)
    t_arrival: float = 0.0
    t_admit: float = 0.0
    t_done: float = 0.0
    nvalid: int = 0
    snr: np.ndarray | None = None
    dmt: torch.Tensor | None = None


class BeamState:
    def __init__(self, spec: BeamSpec, device: torch.device):
        h = spec.header
        self.spec = spec
        self.nbits = h.nbits
        self.nchans = h.nchans
        self.row_bytes = h.nchans * h.nbits // 8
        self.delays = np.atleast_2d(h.get_dmdelays(spec.dms)).astype(np.int32)
        if self.delays.min() < 0:
            raise ValueError("serving needs delays >= 0 (reference at the top of the band)")
        self.maxd = int(self.delays.max())
        self.ndm = self.delays.shape[0]
        self.delays_dev = torch.from_numpy(self.delays).to(device)
        self.tail = torch.zeros(max(self.maxd, 1) * self.row_bytes, dtype=torch.uint8, device=device)
        self.hist = 0  # real stream rows held (right-aligned) in the tail, <= maxd
        self.next_seq = 0
        self.bitorder = _lib.BITORDER_LITTLE if h.nbits == 1 else _lib.BITORDER_BIG
        self._spans: dict[int, int] = {}
        self.pick: tuple[int, int] | None = None  # (work-list variant, slot width)

    def span(self, dw: int) -> int:
        """Tile span of this beam's delay table for DM tiles of ``dw`` rows (cached)."""
        if dw not in self._spans:
            self._spans[dw] = tile_span(self.delays, dw)
        return self._spans[dw]


@dataclass
class _Batch:
    chunks: list
    stream: torch.cuda.Stream
    done: torch.cuda.Event
    bytes: int
    buffers: list = field(default_factory=list)
    worklists: list = field(default_factory=list)
    status: torch.Tensor | None = None  # pinned host copy of the work lists' status words


class Server:
    def __init__(self, beams: list[BeamSpec], *, hbm_budget: int = 40 << 30,
                 widths=(1, 2, 4, 8, 16, 32, 64, 128), max_inflight: int = 2,
                 keep_dmt: bool = False, variant: int | None = None, device=None):
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.beams = {b.beam_id: BeamState(b, self.device) for b in beams}
        self.budget = int(hbm_budget)
        self.widths = tuple(widths)
        self.max_inflight = max_inflight
        self.keep_dmt = keep_dmt
        self.variant = variant
        self.pending: deque[Chunk] = deque()
        self.inflight: list[_Batch] = []
        self.in_use = 0
        self.done: list[Chunk] = []
        self.copy_stream = torch.cuda.Stream(self.device)
        self.streams = [torch.cuda.Stream(self.device) for _ in range(max_inflight)]
        self._rr = 0
        self.batches = 0
        self.batch_sizes: list[int] = []

    # ---- sizing ----
    def _pick(self, st: BeamState) -> tuple[int, int]:
        """Work-list kernel for a beam: ``variant`` if given, else the first
        variant (fixed-slot kernels come first) whose shared-memory slot holds
        the beam's tile span within the per-CTA limit.  Returns (variant, slot)."""
        if st.pick is None:
            lib = _lib.load()
            acc = _lib.ACC_KAHAN32
            cands = [self.variant] if self.variant is not None else \
                range(lib.spp_wl_num_variants(st.nbits, acc))
            for v in cands:
                cfg = variant_cfg(st.nbits, acc, v)
                if not counter_fits(cfg, st.nbits, st.nchans):
                    continue
                dw = cfg["DW"]
                slot = int(lib.spp_wl_slot_words(st.nbits, acc, v, st.span(dw)))
                if slot > 0 and lib.spp_wl_smem_bytes(st.nbits, acc, v, slot) <= 227 * 1024:
                    st.pick = (v, slot)
                    break
            else:
                raise ValueError(f"beam {st.spec.beam_id}: no work-list kernel holds its delay "
                                 "spread")
        return st.pick

    def chunk_bytes(self, c: Chunk) -> int:
        st = self.beams[c.beam_id]
        rows = c.nsamps + st.maxd
        cfg = variant_cfg(st.nbits, _lib.ACC_KAHAN32, self._pick(st)[0])
        spw = cfg["spw"]
        planes = st.nbits if cfg["planes"] else 1
        planar = st.nchans * planes * (rows // spw + 4096) * 4
        return rows * st.row_bytes + planar + st.ndm * c.nsamps * 4

    # ---- API ----
    def submit(self, c: Chunk) -> None:
        st = self.beams[c.beam_id]
        if c.seq != st.next_seq:
            raise ValueError(f"beam {c.beam_id}: chunk {c.seq} out of order (expected {st.next_seq})")
        st.next_seq += 1
        if self.chunk_bytes(c) > self.budget:
            raise ValueError("chunk larger than the HBM budget")
        self.pending.append(c)

    def _admit(self) -> list[Chunk]:
        """FIFO admission into one batch.  A batch holds at most
        ``budget / max_inflight`` bytes (a single larger chunk goes alone), so
        that when the queue is long the next batch still fits beside the
        running one and its copies and corner turns overlap that batch's
        transform instead of waiting for it to retire."""
        batch, used = [], 0
        cap = self.budget // max(self.max_inflight, 1)
        while self.pending:
            c = self.pending[0]
            b = self.chunk_bytes(c)
            if self.in_use + used + b > self.budget or (batch and used + b > cap):
                break
            # keep chunks of one beam in order: a beam's second chunk in the
            # same batch would need the first one's tail, which is fine since
            # tails are copied in order on the copy stream
            batch.append(self.pending.popleft())
            used += b
        return batch

    def _group_key(self, st: BeamState) -> tuple[int, int, int]:
        """Chunks of one sample width and kernel whose shared-memory slots are
        within a factor 1.25 of each other share a work-list launch: each
        launch stages slots as wide as its widest item, so mixing a wide-span
        beam with narrow ones would copy (and hold) rows the narrow ones never
        read."""
        v, slot = self._pick(st)
        return st.nbits, v, int(math.ceil(math.log(max(slot, 1)) / math.log(1.25)))

    def _launch(self, chunks: list[Chunk], now: float) -> None:
        stream = self.streams[self._rr % len(self.streams)]
        self._rr += 1
        total = 0
        bufs = []
        groups: dict[int, list] = {}
        cs = self.copy_stream
        cs.wait_stream(stream)  # previous users of this stream's buffers are done
        for c in chunks:
            st = self.beams[c.beam_id]
            c.t_admit = now
            rows = c.nsamps + st.maxd
            raw = torch.empty(rows * st.row_bytes, dtype=torch.uint8, device=self.device)
            with torch.cuda.stream(cs):
                head = st.maxd * st.row_bytes
                if st.maxd:
                    raw[:head].copy_(st.tail, non_blocking=True)
                src = c.data if torch.is_tensor(c.data) else torch.from_numpy(c.data)
                raw[head:].copy_(src.view(-1)[: c.nsamps * st.row_bytes], non_blocking=True)
                if st.maxd:
                    st.tail.copy_(raw[rows * st.row_bytes - head:], non_blocking=True)
            # real rows start after the part of the tail not yet filled by the stream
            start_row = st.maxd - st.hist
            c.nvalid = st.hist + c.nsamps - st.maxd
            st.hist = min(st.maxd, st.hist + c.nsamps)
            groups.setdefault(self._group_key(st), []).append((c, st, raw, start_row))
            total += self.chunk_bytes(c)
        stream.wait_stream(cs)
        wls = []
        with torch.cuda.stream(stream):
            for (nbits, v, _), items in groups.items():
                wl = WorkList(nbits, v, device=self.device)
                span = max(st.span(wl.DW) for _, st, _, _ in items)
                slot = wl.slot_words(span)
                for c, st, raw, start_row in items:
                    if c.nvalid <= 0:
                        continue
                    rows = c.nsamps + st.maxd - start_row
                    halo, pitch, rpc = wl.layout(c.nvalid, 0, st.maxd, slot)
                    plen = st.nchans * rpc * pitch
                    planar = torch.empty(plen, dtype=torch.int32, device=self.device)
                    wl.corner_turn(raw[start_row * st.row_bytes:], st.bitorder, st.nchans, rows,
                                   halo, planar, pitch, stream=stream)
                    dmt = torch.empty((st.ndm, c.nvalid), dtype=torch.int32, device=self.device)
                    wl.add_job(planar_ptr=planar.data_ptr(), pitch_w=pitch, halo=halo,
                               nchans=st.nchans, delays_dev=st.delays_dev, delays_host=st.delays,
                               out_ptr=dmt.data_ptr(), out_stride=dmt.stride(0), out_start=0,
                               out_elem=4, nvalid=c.nvalid, out_kind=_lib.OUT_I32,
                               span=st.span(wl.DW))
                    bufs += [raw, planar, dmt]
                    c.dmt = dmt
                if wl._rows:
                    wl.finalize(span)
                    wl.launch(stream)
                    wls.append(wl)
            for c, _, _, _ in [x for v in groups.values() for x in v]:
                if c.nvalid > 0:
                    snr, _ = boxcar_snr(c.dmt, widths=self.widths, factors=(1,), stream=stream,
                                        with_index=False)
                    c._snr_dev = snr
                    c._snr_host = torch.empty(snr.shape, dtype=torch.float32).pin_memory()
                    c._snr_host.copy_(snr, non_blocking=True)
            # the work lists' device status words travel back with the batch
            status_host = torch.empty((max(len(wls), 1), 4), dtype=torch.int32).pin_memory()
            status_host.zero_()
            for i, wl in enumerate(wls):
                status_host[i].copy_(wl.status, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(stream)
        self.inflight.append(_Batch(chunks, stream, ev, total, bufs, wls, status_host))
        self.in_use += total
        self.batches += 1
        self.batch_sizes.append(len(chunks))

    def _retire(self, now_fn) -> int:
        n = 0
        keep = []
        for b in self.inflight:
            if b.done.query():
                if b.status is not None and bool((b.status[:, 0] != 0).any()):
                    w = b.status[b.status[:, 0] != 0][0].tolist()
                    raise _lib.SppError(_lib.SPP_ERR_DEVICE,
                                        f"work-list device status 0x{w[0] & 0xffffffff:x} "
                                        f"(block {w[1]}, detail 0x{w[2] & 0xffffffff:x})")
                t = now_fn()
                for c in b.chunks:
                    c.t_done = t
                    if c.nvalid > 0:
                        c.snr = c._snr_host.numpy().reshape(-1, len(self.widths))
                    if not self.keep_dmt:
                        c.dmt = None
                    self.done.append(c)
                self.in_use -= b.bytes
                n += len(b.chunks)
            else:
                keep.append(b)
        self.inflight = keep
        return n

    def step(self, now_fn=time.perf_counter) -> None:
        self._retire(now_fn)
        if self.pending and len(self.inflight) < self.max_inflight:
            batch = self._admit()
            if batch:
                self._launch(batch, now_fn())

    def drain(self, now_fn=time.perf_counter) -> None:
        while self.pending or self.inflight:
            self.step(now_fn)
            if self.inflight and not self.pending:
                self.inflight[0].done.synchronize()

    def run_arrivals(self, chunks: list[Chunk], arrivals: np.ndarray) -> dict:
        """Serve `chunks` arriving at `arrivals` (seconds from start)."""
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0  # noqa: E731
        i = 0
        n = len(chunks)
        while len(self.done) < n:
            t = now()
            while i < n and arrivals[i] <= t:
                chunks[i].t_arrival = arrivals[i]
                self.submit(chunks[i])
                i += 1
            self.step(now)
            if not self.inflight and not self.pending and i < n:
                time.sleep(max(0.0, min(1e-3, arrivals[i] - now())))
            elif self.inflight and (i >= n or arrivals[i] > now()):
                time.sleep(5e-5)
        makespan = max(c.t_done for c in chunks) - min(arrivals)
        lat = np.array([c.t_done - c.t_arrival for c in chunks])
        units = sum(self.beams[c.beam_id].ndm * max(c.nvalid, 0) for c in chunks)
        return {"throughput": units / makespan, "makespan_s": makespan,
                "p50_ms": float(np.percentile(lat, 50) * 1e3),
                "p99_ms": float(np.percentile(lat, 99) * 1e3), "batches": self.batches,
                "batch_chunks": list(self.batch_sizes), "chunks": n}


def plain_process(beams: dict[int, BeamState] | None, chunk: Chunk, st: BeamState,
                  widths=(1, 2, 4, 8, 16, 32, 64, 128), keep_dmt: bool = False,
                  device=None) -> Chunk:
    """The plain per-call path: one chunk at a time, synchronously (H2D, corner
    turn + DM-time transform via a per-call plan, S/N, D2H)."""
    from .dedisp import DMTPlan

    dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
    rows = chunk.nsamps + st.maxd
    raw = torch.empty(rows * st.row_bytes, dtype=torch.uint8, device=dev)
    head = st.maxd * st.row_bytes
    if st.maxd:
        raw[:head].copy_(st.tail)
    src = chunk.data if torch.is_tensor(chunk.data) else torch.from_numpy(chunk.data)
    raw[head:].copy_(src.view(-1)[: chunk.nsamps * st.row_bytes])
    if st.maxd:
        st.tail.copy_(raw[rows * st.row_bytes - head:])
    start_row = st.maxd - st.hist
    chunk.nvalid = st.hist + chunk.nsamps - st.maxd
    st.hist = min(st.maxd, st.hist + chunk.nsamps)
    if chunk.nvalid <= 0:
        chunk.nvalid = 0
        return chunk
    plan = DMTPlan(st.delays, st.nchans, rows, nbits=st.nbits,
                   bitorder="little" if st.nbits == 1 else "big", out_dtype=torch.int32)
    dmt = plan.execute(raw[start_row * st.row_bytes:], rows - start_row, check=True)
    assert dmt.shape[1] == chunk.nvalid
    if chunk.nvalid > 0:
        snr, _ = boxcar_snr(dmt, widths=widths, factors=(1,), with_index=False)
        chunk.snr = snr.cpu().numpy().reshape(-1, len(widths))
    if keep_dmt:
        chunk.dmt = dmt
    plan.close()
    return chunk


def make_beams(nbeams: int, seed: int = 4, nchans_choices=(256, 1024, 4096),
               nbits_choices=(1, 2, 4, 8), tsamp: float = 64e-6) -> list[BeamSpec]:
    """Config-4 beams: random nchans/nbits, DM max U[500, 3000] with 256-2048 trials."""
    rng = np.random.default_rng(seed)
    beams = []
    for b in range(nbeams):
        nchans = int(rng.choice(nchans_choices))
        nbits = int(rng.choice(nbits_choices))
        bw = 300.0
        h = Header(nchans=nchans, fch1=1500.0, foff=-bw / nchans, tsamp=tsamp, nbits=nbits)
        dm_max = float(rng.uniform(500.0, 3000.0))
        ndm = int(rng.integers(256, 2049))
        beams.append(BeamSpec(b, h, np.linspace(0.0, dm_max, ndm)))
    return beams


def chunk_sizes(nchunks: int, seed: int = 4, lo: int = 1 << 14, hi: int = 1 << 18) -> np.ndarray:
    return np.random.default_rng(seed + 1).integers(lo, hi + 1, size=nchunks)
