"""GPU dedispersion operators (R2, R3) over the C ABI.

* :func:`dedisperse_block` -- one DM over one in-HBM block of raw samples;
  the drop-in for ``kernels.dedisperse`` (src/sigpyproc/core/kernels.py:340-362).
* :class:`DMTPlan` -- a DM-trial batch plan (delay table resident in HBM,
  tile shape chosen per geometry) whose :meth:`DMTPlan.execute` produces the
  DM-time array; ``mode="roll"`` reproduces ``kernels.dmt_block``
  (:1155-1168).

Tensors are torch CUDA tensors; raw filterbank data is passed exactly as it
sits in the file (time-major, packed for nbits < 8) -- unpacking is fused into
the kernels.
"""

from __future__ import annotations

import ctypes
import threading

import numpy as np
import torch

from . import _lib
from .io.bits import bitorder_code

_ws_lock = threading.Lock()
_ws_cache: dict[tuple[int, int], torch.Tensor] = {}


def stream_handle(stream: torch.cuda.Stream | None, device=None) -> int:
    if stream is None:
        stream = torch.cuda.current_stream(device)
    return stream.cuda_stream


def workspace(nbytes: int, device: torch.device | int | None = None,
              stream: torch.cuda.Stream | None = None) -> torch.Tensor:
    """Grow-only scratch buffer per (device, stream), 256-B aligned."""
    dev = torch.device("cuda", torch.cuda.current_device() if device is None else
                       (device.index if isinstance(device, torch.device) else device))
    key = (dev.index, stream_handle(stream, dev))
    with _ws_lock:
        buf = _ws_cache.get(key)
        if buf is None or buf.numel() < nbytes:
            buf = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=dev)
            _ws_cache[key] = buf
    return buf


def status_clear(ws: torch.Tensor, stream: torch.cuda.Stream | None = None) -> None:
    """Zero the device status block at the head of a workspace (stream-ordered).

    Kernels that wait on an mbarrier with a time limit, or that clamp a delay
    outside the declared range, record it in these words instead of faulting;
    a fresh workspace holds arbitrary bytes, so clear it before the calls whose
    status is to be read."""
    _lib.check(_lib.load().spp_status_clear(ws.data_ptr(), stream_handle(stream, ws.device)))


def status_check(ws: torch.Tensor, stream: torch.cuda.Stream | None = None) -> None:
    """Synchronise ``stream`` and raise :class:`SppError` (SPP_ERR_DEVICE) if any
    call since the last :func:`status_clear` on this workspace flagged a device
    error: a bounded wait that ran out (the output is incomplete) or a delay
    clamped into the declared range (the output is wrong)."""
    words = np.zeros(4, dtype=np.uint32)
    _lib.check(_lib.load().spp_status_read(ws.data_ptr(), words.ctypes.data,
                                           stream_handle(stream, ws.device)))


def _as_raw(data) -> torch.Tensor:
    if not torch.is_tensor(data):
        raise TypeError("expected a torch tensor")
    if not data.is_cuda:
        raise ValueError("expected a CUDA tensor")
    return data.contiguous()


def _nbits_of(raw: torch.Tensor, nbits: int | None) -> int:
    if nbits is not None:
        return int(nbits)
    if raw.dtype == torch.float32:
        return 32
    if raw.dtype == torch.uint8:
        return 8
    raise TypeError(f"unsupported dtype {raw.dtype}")


def dedisperse_block(raw: torch.Tensor, delays: np.ndarray, nchans: int, nsamps: int,
                     out: torch.Tensor, out_start: int = 0, *, nbits: int | None = None,
                     bitorder: str = "big", acc: int = _lib.ACC_F64,
                     delays_dev: torch.Tensor | None = None,
                     stream: torch.cuda.Stream | None = None,
                     ws: torch.Tensor | None = None, host_table: bool | None = None) -> int:
    """``out[out_start + t] = sum_c x[t + delays[c]][c]`` for ``t < nsamps - max|d|``.

    Returns the number of samples written.  ``raw`` holds ``nsamps`` spectra
    (uint8 packed or float32).  ``delays`` is the host int32 table (its range
    bounds the kernel's checks); ``delays_dev`` may carry a device copy.
    8-bit blocks go through ``spp_dedisperse_hd`` (offsets precomputed from the
    host table) when their shape allows, else through ``spp_dedisperse``;
    ``host_table`` True/False forces one of the two.
    """
    raw = _as_raw(raw)
    nb = _nbits_of(raw, nbits)
    delays = np.ascontiguousarray(delays, dtype=np.int32)
    if delays.size != nchans:
        raise ValueError(f"delays has {delays.size} entries for {nchans} channels")
    dmin, dmax = int(delays.min()), int(delays.max())
    nvalid = nsamps - max(abs(dmin), abs(dmax))
    if nvalid <= 0:
        return 0
    if out.dtype != torch.float32 or not out.is_cuda:
        raise TypeError("out must be a CUDA float32 tensor")
    lib = _lib.load()
    st = stream_handle(stream, raw.device)
    if nb == 8 and host_table is not False:
        rc = lib.spp_dedisperse_hd(raw.data_ptr(), nb, nchans, nsamps, delays.ctypes.data,
                                   out.data_ptr(), out.numel(), out_start, st)
        if rc == _lib.SPP_OK:
            return nvalid
        if rc != _lib.SPP_ERR_UNSUPPORTED or host_table:
            _lib.check(rc)
    elif host_table:
        raise NotImplementedError("the host-table path covers 8-bit data")
    need = lib.spp_dedisperse_workspace_bytes(nb, nchans, nsamps, dmin, dmax)
    if need < 0:
        _lib.check(_lib.SPP_ERR_ARG)
    if ws is None:
        ws = workspace(need, raw.device, stream)
    if delays_dev is None:
        delays_dev = torch.from_numpy(delays).to(raw.device, non_blocking=False)
    _lib.check(lib.spp_dedisperse(
        raw.data_ptr(), nb, bitorder_code(bitorder), nchans, nsamps, delays_dev.data_ptr(),
        dmin, dmax, out.data_ptr(), out.numel(), out_start, acc, ws.data_ptr(), ws.numel(), st))
    return nvalid


class DMTPlan:
    """DM-time transform plan over ``ndm x nchans`` int32 delays.

    mode "dedisperse": ``out[i][t] = sum_c x[t + D[i][c]][c]``, ``t < nsamps - max|D|``
    mode "roll":       ``out[i][t] = sum_c x[(t - D[i][c]) mod nsamps][c]``, ``t < nsamps``

    Integer input is summed exactly.  Float32 input is summed in float64 in
    channel order by default (``acc=ACC_F64``, the reference's accumulator);
    ``ACC_KAHAN32`` trades that for compensated float32 slab sums.
    """

    def __init__(self, delays: np.ndarray, nchans: int, nsamps_max: int, *, nbits: int = 8,
                 bitorder: str = "big", mode: str = "dedisperse", out_dtype=torch.float32,
                 acc: int = _lib.ACC_F64, device=None):
        delays = np.ascontiguousarray(np.atleast_2d(delays), dtype=np.int32)
        if delays.shape[1] != nchans:
            raise ValueError(f"delay table is {delays.shape}, expected (ndm, {nchans})")
        self.delays = delays
        self.ndm = delays.shape[0]
        self.nchans = int(nchans)
        self.nsamps_max = int(nsamps_max)
        self.nbits = int(nbits)
        self.bitorder = bitorder
        self.mode = mode
        self.out_dtype = out_dtype
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        out_kind = _lib.OUT_I32 if out_dtype == torch.int32 else _lib.OUT_F32
        mode_code = {"dedisperse": _lib.MODE_DEDISPERSE, "roll": _lib.MODE_ROLL}[mode]
        lib = _lib.load()
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(lib.spp_dmt_plan_create(
                ctypes.byref(h), self.nbits, bitorder_code(bitorder), self.nchans, self.nsamps_max,
                self.ndm, delays.ctypes.data, mode_code, out_kind, acc))
        self._h = h

    # -- introspection --
    def nvalid(self, nsamps: int) -> int:
        return int(_lib.load().spp_dmt_plan_nvalid(self._h, nsamps))

    def workspace_bytes(self, nsamps: int) -> int:
        return int(_lib.load().spp_dmt_plan_workspace_bytes(self._h, nsamps))

    def describe(self) -> dict:
        cfg = (ctypes.c_int32 * 8)()
        _lib.check(_lib.load().spp_dmt_plan_describe(self._h, cfg))
        keys = ("nbits", "R", "DW", "TW", "SLAB", "STAGES", "T", "smem")
        d = dict(zip(keys, list(cfg)))
        d["bit_sliced"] = (d["nbits"] >> 8) & 1
        d["paired"] = (d["nbits"] >> 9) & 1
        d["nbits"] &= 0xFF
        return d

    @property
    def num_variants(self) -> int:
        return int(_lib.load().spp_dmt_plan_num_variants(self._h))

    def set_variant(self, v: int) -> None:
        _lib.check(_lib.load().spp_dmt_plan_set_variant(self._h, int(v)))

    def timing(self, enable: bool = True) -> None:
        """Start (or stop) recording per-kernel CUDA events on each execute."""
        _lib.check(_lib.load().spp_dmt_plan_timing(self._h, int(enable)))

    def timing_read(self) -> dict:
        """Summed device milliseconds of the corner turn and the DM-time kernel."""
        a, b, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_int32()
        _lib.check(_lib.load().spp_dmt_plan_timing_read(self._h, ctypes.byref(a), ctypes.byref(b),
                                                        ctypes.byref(n)))
        return {"ms_corner_turn": a.value, "ms_dmt": b.value, "n": n.value}

    def autotune(self, raw: torch.Tensor, nsamps: int, out: torch.Tensor | None = None,
                 reps: int = 2, cache: str | None = None) -> dict:
        """Time every kernel variant on this input and keep the fastest.

        Results are cached per (nbits, nchans, ndm bucket, mode, out dtype) in
        the JSON file ``cache`` (default ``$SPP_TUNE_CACHE`` or
        ``~/.cache/sigpyproc3_b200/tuned.json``)."""
        import json
        import os
        from pathlib import Path

        path = Path(cache or os.environ.get("SPP_TUNE_CACHE",
                                            Path.home() / ".cache/sigpyproc3_b200/tuned.json"))
        key = (f"nb{self.nbits}-ch{self.nchans}-ndm{1 << max(0, (self.ndm - 1).bit_length())}"
               f"-{self.mode}-{self.out_dtype}")
        table = {}
        if path.exists():
            try:
                table = json.loads(path.read_text())
            except ValueError:
                table = {}
        if key in table and 0 <= table[key]["variant"] < self.num_variants:
            self.set_variant(table[key]["variant"])
            # an entry written by a build with another variant list names
            # another kernel: re-tune unless the recorded shape still matches
            if table[key].get("shape") == self.describe():
                return table[key]
        if out is None:
            out = torch.empty((self.ndm, self.nvalid(nsamps)), dtype=self.out_dtype,
                              device=raw.device)
        times = []
        for v in range(self.num_variants):
            self.set_variant(v)
            self.execute(raw, nsamps, out)
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            for _ in range(reps):
                self.execute(raw, nsamps, out)
            e.record()
            e.synchronize()
            times.append(s.elapsed_time(e) / reps)
        best = int(np.argmin(times))
        self.set_variant(best)
        rec = {"variant": best, "ms": times[best], "all_ms": times, "shape": self.describe()}
        table[key] = rec
        try:  # atomic replace: processes tuning at once never leave a torn file
            path.parent.mkdir(parents=True, exist_ok=True)
            tmp = path.with_name(f"{path.name}.{os.getpid()}.tmp")
            tmp.write_text(json.dumps(table, indent=1))
            os.replace(tmp, path)
        except OSError:
            pass
        return rec

    # -- execution --
    def execute(self, raw: torch.Tensor, nsamps: int | None = None, out: torch.Tensor | None = None,
                out_start: int = 0, stream: torch.cuda.Stream | None = None,
                ws: torch.Tensor | None = None, check: bool = False) -> torch.Tensor:
        """DM-time array of one block (stream-ordered).  ``check=True`` clears the
        workspace's device status first and reads it after the launch (a
        synchronisation), raising SppError if the kernel flagged an error;
        otherwise read it with :func:`status_check` after a run of calls."""
        raw = _as_raw(raw)
        if nsamps is None:
            rb = self.nchans * 4 if self.nbits == 32 else self.nchans * self.nbits // 8
            nsamps = raw.numel() * raw.element_size() // rb
        nv = self.nvalid(nsamps)
        if out is None:
            out = torch.empty((self.ndm, nv), dtype=self.out_dtype, device=raw.device)
        stride = out.stride(0) if out.dim() == 2 else out.numel()
        if ws is None:
            ws = workspace(self.workspace_bytes(nsamps), raw.device, stream)
        if check:
            status_clear(ws, stream)
        _lib.check(_lib.load().spp_dmt_execute(
            self._h, raw.data_ptr(), nsamps, out.data_ptr(), stride, out_start, ws.data_ptr(),
            ws.numel(), stream_handle(stream, raw.device)))
        if check:
            status_check(ws, stream)
        return out

    def execute_zero_dm(self, raw: torch.Tensor, nsamps: int, bpass: torch.Tensor,
                        chanwts: torch.Tensor, out: torch.Tensor | None = None, out_start: int = 0,
                        stream: torch.cuda.Stream | None = None) -> torch.Tensor:
        """Float32 input with kernels.remove_zerodm fused into the load."""
        raw = _as_raw(raw)
        lib = _lib.load()
        nv = self.nvalid(nsamps)
        if out is None:
            out = torch.empty((self.ndm, nv), dtype=self.out_dtype, device=raw.device)
        stride = out.stride(0) if out.dim() == 2 else out.numel()
        ws = workspace(int(lib.spp_dmt_plan_zero_dm_workspace_bytes(self._h, nsamps)), raw.device,
                       stream)
        bpass = bpass.contiguous()
        chanwts = chanwts.to(torch.float32).contiguous()
        _lib.check(lib.spp_dmt_execute_zero_dm(
            self._h, raw.data_ptr(), nsamps, bpass.data_ptr(), chanwts.data_ptr(), out.data_ptr(),
            stride, out_start, ws.data_ptr(), ws.numel(), stream_handle(stream, raw.device)))
        return out

    def host_workspace_bytes(self, block_nsamps: int) -> int:
        return int(_lib.load().spp_dmt_host_workspace_bytes(self._h, block_nsamps))

    def execute_host(self, raw_host: np.ndarray, nsamps: int, out_host: np.ndarray,
                     block_nsamps: int = 65536, ws: torch.Tensor | None = None) -> np.ndarray:
        """End-to-end from host memory (pinned for overlap); synchronous."""
        nv = self.nvalid(nsamps)
        if out_host.shape[0] != self.ndm or out_host.shape[1] < nv:
            raise ValueError("out_host too small")
        if ws is None:
            ws = workspace(self.host_workspace_bytes(block_nsamps), self.device)
        with torch.cuda.device(self.device):
            _lib.check(_lib.load().spp_dmt_execute_host(
                self._h, raw_host.ctypes.data, nsamps, out_host.ctypes.data, out_host.shape[1],
                block_nsamps, ws.data_ptr(), ws.numel()))
        return out_host

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _lib.load().spp_dmt_plan_destroy(h)
            self._h = ctypes.c_void_p()

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass
