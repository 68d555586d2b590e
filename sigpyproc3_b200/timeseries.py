"""1-D dedispersed time series (R11), with GPU downsample (R8) and boxcar (R9).

Mirrors ``TimeSeries`` (src/sigpyproc/timeseries.py:27-132, :296-325): data
is float32 and matches ``header.nsamples``.  The samples live in HBM as a
torch CUDA tensor (``.tensor``); ``.data`` returns a host numpy copy for
drop-in use.
"""

from __future__ import annotations

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
        reference bin matches the reference (one kernel, ``spp_boxcar_filter``;
        window sums in float64)."""
        if width < 1:
            raise ValueError(f"invalid boxcar width: {width}")
        x = self._cuda().contiguous()
        out = torch.empty_like(x)
        _lib.call("spp_boxcar_filter", x.data_ptr(), x.numel(), int(width), out.data_ptr(),
                  stream_handle(None, x.device))
        return TimeSeries(out, self.header.new_header())

    def snr(self, widths=(1, 2, 4, 8, 16, 32, 64, 128, 256), factors=(1,),
            loc_scale: str = "mean_std") -> np.ndarray:
        """Boxcar S/N peaks of this series (see :func:`search.boxcar_snr`);
        ``loc_scale="median_iqr"`` z-scores with the median and the IQR, as
        the reference MatchedFilter does by default."""
        from .search import boxcar_snr

        snr, _ = boxcar_snr(self._cuda().view(1, -1), widths=widths, factors=factors,
                            loc_scale=loc_scale)
        return snr[0].cpu().numpy()
