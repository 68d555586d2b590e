"""Batched DM-time work lists for the persistent kernel (k_dmt_wl).

A :class:`WorkList` collects DM-time jobs -- each one (planar rows of a beam
or channel group, a block of delay rows, output rows) -- cuts them into
items of DW trial rows x T samples and launches them all in one persistent
kernel.  The item layout mirrors ``spp_dmt_item`` in include/sppgpu.h.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib

ITEM_DTYPE = np.dtype({
    "names": ["planar", "pitch_w", "halo", "delays", "dpitch", "out", "out_stride", "out_start",
              "nvalid", "t0", "nchans", "nrows", "sign", "dlo", "dhi", "span_max", "out_kind",
              "reserved"],
    "formats": ["<u8", "<i8", "<i8", "<u8", "<i8", "<u8", "<i8", "<i8", "<i8", "<i8", "<i4", "<i4",
                "<i4", "<i4", "<i4", "<i4", "<i4", "<i4"],
    "offsets": [0, 8, 16, 24, 32, 40, 48, 56, 64, 72, 80, 84, 88, 92, 96, 100, 104, 108],
    "itemsize": 112,
})


def variant_cfg(nbits: int, acc: int, variant: int) -> dict:
    cfg = (ctypes.c_int32 * 8)()
    _lib.check(_lib.load().spp_wl_describe(nbits, acc, variant, cfg))
    d = dict(zip(("R", "DW", "TW", "SLAB", "STAGES", "T", "threads", "spw"), list(cfg)))
    d["planes"] = d["spw"] >> 8
    d["spw"] &= 0xFF
    return d


def counter_fits(cfg: dict, nbits: int, nchans: int) -> bool:
    """Whether a kernel variant can hold sums of ``nchans`` samples: the
    bit-sliced kernels count below 2^14 (1-, 2-bit), 2^16 (4-bit) or 2^20
    (8-bit)."""
    if not cfg["planes"]:
        return True
    levels = {4: 16, 8: 20}.get(nbits, 14)
    return nchans * ((1 << nbits) - 1) < (1 << levels)


def num_variants(nbits: int, acc: int = _lib.ACC_KAHAN32) -> int:
    return int(_lib.load().spp_wl_num_variants(nbits, acc))


def tile_span(delays: np.ndarray, dw: int) -> int:
    """Max over DW-row tiles and channels of the tile's delay spread."""
    d = np.atleast_2d(delays)
    ndm = d.shape[0]
    pad = (-ndm) % dw
    if pad:  # repeating the last row leaves the last tile's spread unchanged
        d = np.concatenate([d, np.repeat(d[-1:], pad, axis=0)])
    t = d.reshape(-1, dw, d.shape[1])
    return int((t.max(axis=1).astype(np.int64) - t.min(axis=1)).max())


class WorkList:
    """Items of one persistent launch.  Add jobs, then :meth:`finalize` once
    and :meth:`launch` as often as needed (the item array stays in HBM)."""

    def __init__(self, nbits: int, variant: int = 0, acc: int = _lib.ACC_KAHAN32,
                 device: torch.device | None = None):
        self.nbits = nbits
        self.acc = acc
        self.variant = variant
        self.cfg = variant_cfg(nbits, acc, variant)
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self._rows: list[np.ndarray] = []
        self.span = 0
        self.items_dev: torch.Tensor | None = None
        self.counter = torch.zeros(4, dtype=torch.int32, device=self.device)
        self.status = torch.zeros(4, dtype=torch.int32, device=self.device)
        self.slot_w = 0
        self.nctas = 0

    @property
    def T(self) -> int:
        return self.cfg["T"]

    @property
    def DW(self) -> int:
        return self.cfg["DW"]

    def span_of(self, delays_host: np.ndarray, sign: int = 1) -> int:
        return tile_span(sign * np.atleast_2d(delays_host), self.DW)

    def add_job(self, *, planar_ptr: int, pitch_w: int, halo: int, nchans: int,
                delays_dev: torch.Tensor, delays_host: np.ndarray, out_ptr: int, out_stride: int,
                out_start: int, out_elem: int, nvalid: int, out_kind: int, sign: int = 1,
                row_stride_out: int | None = None, span: int | None = None) -> None:
        """One DM-time job: rows of ``delays`` (ndm x >= nchans, row pitch =
        delays_dev.stride(0)) against ``nchans`` planar rows; output row r at
        out_ptr + r * out_stride * out_elem.  ``span``: the job's tile span
        (``tile_span`` of the signed delays for this variant's DW), when the
        caller has it cached."""
        if not counter_fits(self.cfg, self.nbits, nchans):
            raise ValueError(f"work-list variant {self.variant}: sums of {nchans} {self.nbits}-bit "
                             "samples overflow its bit-sliced counter")
        dh = np.atleast_2d(delays_host).astype(np.int64) * sign
        ndm = dh.shape[0]
        if delays_dev.dtype != torch.int32 or delays_dev.stride(-1) != 1:
            raise ValueError("delays_dev must be int32 with unit stride along channels")
        dpitch = delays_dev.stride(0) if delays_dev.dim() == 2 else nchans
        T, DW = self.T, self.DW
        ntiles = max(1, -(-nvalid // T))
        dlo, dhi = int(dh[:, :nchans].min()), int(dh[:, :nchans].max())
        self.span = max(self.span, tile_span(dh[:, :nchans], DW) if span is None else int(span))
        r0 = np.arange(0, ndm, DW)
        nrows = np.minimum(DW, ndm - r0)
        t0 = np.arange(ntiles, dtype=np.int64) * T
        rec = np.zeros(len(r0) * ntiles, dtype=ITEM_DTYPE)
        # time tile outer, DM tile inner: neighbouring items share planar data in L2
        tt, rr = np.meshgrid(np.arange(ntiles), np.arange(len(r0)), indexing="ij")
        tt, rr = tt.ravel(), rr.ravel()
        rec["planar"] = planar_ptr
        rec["pitch_w"] = pitch_w
        rec["halo"] = halo
        rec["delays"] = delays_dev.data_ptr() + r0[rr] * dpitch * 4
        rec["dpitch"] = dpitch
        rec["out"] = out_ptr + r0[rr] * out_stride * out_elem
        rec["out_stride"] = out_stride
        rec["out_start"] = out_start
        rec["nvalid"] = nvalid
        rec["t0"] = t0[tt]
        rec["nchans"] = nchans
        rec["nrows"] = nrows[rr]
        rec["sign"] = sign
        rec["dlo"] = dlo
        rec["dhi"] = dhi
        rec["out_kind"] = out_kind
        self._rows.append(rec)

    def layout(self, nvalid: int, omin: int, omax: int, slot_w: int | None = None):
        """(halo, pitch_w, rows per channel) of planar rows for this variant."""
        halo, pitch, rows = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        _lib.check(_lib.load().spp_wl_planar_layout(
            self.nbits, self.acc, self.variant, nvalid, omin, omax,
            self.slot_words() if slot_w is None else slot_w, ctypes.byref(halo),
            ctypes.byref(pitch), ctypes.byref(rows)))
        return halo.value, pitch.value, rows.value

    def corner_turn(self, raw: torch.Tensor, bitorder: int, nchans: int, nsamps: int, halo: int,
                    planar: torch.Tensor, pitch_w: int,
                    stream: torch.cuda.Stream | None = None) -> None:
        st = (stream or torch.cuda.current_stream(raw.device)).cuda_stream
        _lib.check(_lib.load().spp_wl_corner_turn(self.nbits, self.acc, self.variant,
                                                  raw.data_ptr(), bitorder, nchans, nsamps, halo,
                                                  planar.data_ptr(), pitch_w, st))

    def slot_words(self, span: int | None = None) -> int:
        return int(_lib.load().spp_wl_slot_words(self.nbits, self.acc, self.variant,
                                                 self.span if span is None else span))

    def finalize(self, span: int | None = None) -> None:
        items = np.concatenate(self._rows) if self._rows else np.zeros(0, ITEM_DTYPE)
        self.slot_w = self.slot_words(span)
        items["span_max"] = self.span if span is None else span
        self.nitems = int(items.size)
        self.items_host = items
        self.items_dev = torch.from_numpy(items.view(np.uint8).copy()).to(self.device)
        self.nctas = int(_lib.load().spp_wl_default_ctas(self.nbits, self.acc, self.variant,
                                                         self.slot_w))
        if self.nctas <= 0:
            _lib.check(_lib.SPP_ERR_CUDA)

    def launch(self, stream: torch.cuda.Stream | None = None) -> None:
        st = (stream or torch.cuda.current_stream(self.device)).cuda_stream
        _lib.check(_lib.load().spp_wl_launch(
            self.nbits, self.acc, self.variant, self.items_dev.data_ptr(), self.nitems,
            self.slot_w, self.counter.data_ptr(), self.status.data_ptr(), self.nctas, st))


def planar_layout(nbits: int, tile_T: int, nvalid: int, omin: int, omax: int,
                  slot_w: int) -> tuple[int, int]:
    halo, pitch = ctypes.c_int64(), ctypes.c_int64()
    _lib.check(_lib.load().spp_planar_layout(nbits, tile_T, nvalid, omin, omax, slot_w,
                                             ctypes.byref(halo), ctypes.byref(pitch)))
    return halo.value, pitch.value


def corner_turn(raw: torch.Tensor, nbits: int, bitorder: int, nchans: int, nsamps: int, halo: int,
                planar: torch.Tensor, pitch_w: int, stream: torch.cuda.Stream | None = None) -> None:
    st = (stream or torch.cuda.current_stream(raw.device)).cuda_stream
    _lib.check(_lib.load().spp_corner_turn(raw.data_ptr(), nbits, bitorder, nchans, nsamps, halo,
                                           planar.data_ptr(), pitch_w, st))
