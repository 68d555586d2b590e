"""1-D dedispersed time series (R11), with GPU downsample (R8) and boxcar (R9).

Mirrors ``TimeSeries`` (src/sigpyproc/timeseries.py:27-132, :296-325): data
is float32 and matches ``header.nsamples``.  The samples live in HBM as a
torch CUDA tensor (``.tensor``); ``.data`` returns a host numpy copy for
drop-in use.
"""

from __future__ import annotations

import math

import numpy as np
import torch

from . import _lib
from .dedisp import stream_handle
from .header import Header


class TimeSeries:
    def __init__(self, data, header: Header):
        if torch.is_tensor(data):
            t = data.to(torch.float32)
        else:
            t = torch.as_tensor(np.asarray(data, dtype=np.float32))
        if t.dim() != 1:
            raise ValueError(f"Input data must be 1D, got {t.dim()}D")
        self._t = t
        self._header = header
        if header.nsamples != t.numel():
            self._header = header.new_header({"nsamples": int(t.numel())})

    @property
    def tensor(self) -> torch.Tensor:
        return self._t

    @property
    def data(self) -> np.ndarray:
        return self._t.detach().cpu().numpy()

    @property
    def header(self) -> Header:
        return self._header

    @property
    def nsamples(self) -> int:
        return int(self._t.numel())

    def _cuda(self) -> torch.Tensor:
        return self._t if self._t.is_cuda else self._t.cuda()

    def downsample(self, factor: int, filter_method: str = "mean") -> "TimeSeries":
        """Mean over non-overlapping windows (kernels.downsample_1d_mean)."""
        if filter_method != "mean":
            raise NotImplementedError("only filter_method='mean' runs on the GPU")
        if not isinstance(factor, int) or factor <= 0:
            raise ValueError("Factor must be a positive integer.")
        if factor == 1:
            return self
        x = self._cuda().contiguous()
        if factor > x.numel():
            raise ValueError("Factor must be less than the size of the array.")
        out = torch.empty(x.numel() // factor, dtype=torch.float32, device=x.device)
        _lib.call("spp_downsample_mean", x.data_ptr(), 1, x.numel(), x.numel(), factor,
                  out.data_ptr(), out.numel(), stream_handle(None, x.device))
        hdr = self.header.new_header({"tsamp": self.header.tsamp * factor, "nsamples": out.numel()})
        return TimeSeries(out, hdr)

    def apply_boxcar(self, width: int) -> "TimeSeries":
        """Square-normalised running mean (timeseries.py:296-325): symmetric
        padding, moving mean of ``width``, times sqrt(width), rolled so the
        reference bin matches the reference."""
        if width < 1:
            raise ValueError(f"invalid boxcar width: {width}")
        x = self._cuda().to(torch.float64)
        pad = (width // 2, width // 2) if width % 2 else (width // 2, width // 2 - 1)
        n = x.numel()
        left = x[: pad[0]].flip(0) if pad[0] else x[:0]
        right = x[n - pad[1]:].flip(0) if pad[1] else x[:0]
        xp = torch.cat([left, x, right])
        c = torch.cat([torch.zeros(1, dtype=torch.float64, device=x.device), torch.cumsum(xp, 0)])
        mean = (c[width:] - c[:-width]) / width
        out = (mean * math.sqrt(width)).to(torch.float32)
        ref_bin = -width // 2 + 1 if width % 2 else -width // 2
        return TimeSeries(torch.roll(out, ref_bin), self.header.new_header())

    def snr(self, widths=(1, 2, 4, 8, 16, 32, 64, 128, 256), factors=(1,)) -> np.ndarray:
        """Boxcar S/N peaks of this series (see :func:`search.boxcar_snr`)."""
        from .search import boxcar_snr

        snr, _ = boxcar_snr(self._cuda().view(1, -1), widths=widths, factors=factors)
        return snr[0].cpu().numpy()
