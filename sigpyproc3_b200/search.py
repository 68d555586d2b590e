"""Boxcar matched-filter S/N over DM-time rows (R9) and the batched search."""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .dedisp import stream_handle, workspace

DEFAULT_WIDTHS = (1, 2, 4, 8, 16, 32, 64, 128, 256)


def boxcar_snr(rows: torch.Tensor, widths=DEFAULT_WIDTHS, factors=(1,), n: int | None = None,
               stream: torch.cuda.Stream | None = None, with_index: bool = True, out=None,
               loc_scale: str = "mean_std"):
    """S/N peak per (row, downsample factor, width) of a (nrows, >= n) CUDA tensor
    (float32 or int32): ``max_t (sum_{k<w} y[t+k] - w*loc(y)) / (scale(y)*sqrt(w))``
    with ``y = downsample_mean(row, f)``.  ``loc_scale`` "mean_std" (mean and
    population std) or "median_iqr" (median and IQR/1.349, the reference
    MatchedFilter's defaults).  Returns (snr float32, index int32)."""
    if loc_scale not in ("mean_std", "median_iqr"):
        raise ValueError(f"loc_scale must be 'mean_std' or 'median_iqr', got {loc_scale!r}")
    robust = loc_scale == "median_iqr"
    if rows.dim() == 1:
        rows = rows.view(1, -1)
    if rows.stride(1) != 1:
        rows = rows.contiguous()
    kind = {torch.float32: _lib.OUT_F32, torch.int32: _lib.OUT_I32}[rows.dtype]
    nrows = rows.shape[0]
    n = rows.shape[1] if n is None else n
    fac = np.ascontiguousarray(factors, dtype=np.int32)
    wid = np.ascontiguousarray(widths, dtype=np.int32)
    snr, idx = out if out is not None else (None, None)
    if snr is None:
        snr = torch.empty((nrows, fac.size, wid.size), dtype=torch.float32, device=rows.device)
    if idx is None and with_index:
        idx = torch.empty_like(snr, dtype=torch.int32)
    lib = _lib.load()
    sizer = lib.spp_boxcar_snr_robust_workspace_bytes if robust else \
        lib.spp_boxcar_snr_workspace_bytes
    need = sizer(nrows, n, fac.size, wid.size)
    ws = workspace(need, rows.device, stream)
    fn = lib.spp_boxcar_snr_robust if robust else lib.spp_boxcar_snr
    _lib.check(fn(rows.data_ptr(), kind, nrows, n, rows.stride(0),
                                  fac.ctypes.data, fac.size, wid.ctypes.data, wid.size,
                                  snr.data_ptr(), idx.data_ptr() if idx is not None else None,
                                  ws.data_ptr(), ws.numel(), stream_handle(stream, rows.device)))
    return snr, idx
