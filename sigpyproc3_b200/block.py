"""In-memory 2-D blocks (R3/R11): ``FilterbankBlock`` (nchans, nsamps) and
``DMTBlock`` (ndms, nsamps), mirroring src/sigpyproc/block.py."""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .dedisp import DMTPlan
from .header import Header
from .timeseries import TimeSeries


def _to_cuda_f32(data) -> torch.Tensor:
    if torch.is_tensor(data):
        t = data
    else:
        t = torch.as_tensor(np.asarray(data, dtype=np.float32))
    if not t.is_cuda:
        t = t.cuda()
    return t.to(torch.float32)


class BaseBlock:
    def __init__(self, data, header: Header):
        self._t = _to_cuda_f32(data)
        if self._t.dim() != 2:
            raise ValueError(f"Data must be 2D, got {self._t.dim()}D")
        self._header = header

    @property
    def tensor(self) -> torch.Tensor:
        return self._t

    @property
    def data(self) -> np.ndarray:
        return self._t.cpu().numpy()

    @property
    def header(self) -> Header:
        return self._header

    @property
    def nsamples(self) -> int:
        return int(self._t.shape[1])

    def pad_samples(self, nsamps_final: int, offset: int, pad_mode: str = "median"):
        """Pad to ``nsamps_final`` samples per row with each row's median or mean,
        the block placed at ``offset`` (block.py:108-146).  The pad values come
        from numpy on the host, as in the reference, so they are the same
        float32 numbers."""
        if pad_mode not in {"mean", "median"}:
            raise ValueError(f"pad_mode must be 'mean' or 'median', got {pad_mode}")
        data = self.data
        pad_values = getattr(np, pad_mode)(data, axis=1)
        data_pad = np.ones((data.shape[0], nsamps_final), dtype=data.dtype)
        data_pad *= pad_values[:, None]
        data_pad[:, offset:offset + data.shape[1]] = data
        return self.__class__(data_pad, self.header.new_header({"nsamples": nsamps_final}))


class FilterbankBlock(BaseBlock):
    """(nchans, nsamples) float32 filterbank block held in HBM."""

    def __init__(self, data, header: Header, dm: float = 0.0):
        super().__init__(data, header)
        if self._t.shape[0] != header.nchans:
            raise ValueError(f"data has {self._t.shape[0]} channels, header {header.nchans}")
        self.dm = dm

    @property
    def nchans(self) -> int:
        return int(self._t.shape[0])

    def get_tim(self) -> TimeSeries:
        return TimeSeries(self._t.sum(0), self.header.dedispersed_header(dm=self.dm))

    def downsample(self, ffactor: int = 1, tfactor: int = 1,
                   filter_method: str = "mean") -> "FilterbankBlock":
        """Means over ``ffactor`` channels x ``tfactor`` samples (block.py:215-244,
        stats.downsample_2d core/stats.py:96-136), remainders dropped, on the
        GPU (float64 sums; the reference averages in float32, so results can
        differ in the last bit for non-integer data)."""
        if filter_method != "mean":
            raise NotImplementedError("only filter_method='mean' runs on the GPU")
        if not all(isinstance(f, int) and f > 0 for f in (ffactor, tfactor)):
            raise ValueError("Factors must be positive integers.")
        x = self._t.contiguous()
        nch, n = x.shape
        out = torch.empty((nch // ffactor, n // tfactor), dtype=torch.float32, device=x.device)
        _lib.call("spp_downsample_2d_mean", x.data_ptr(), nch, n, ffactor, tfactor,
                  out.data_ptr(), torch.cuda.current_stream(x.device).cuda_stream)
        changes = {"tsamp": self.header.tsamp * tfactor, "foff": self.header.foff * ffactor,
                   "nsamples": self.header.nsamples // tfactor,
                   "nchans": self.header.nchans // ffactor}
        return FilterbankBlock(out, self.header.new_header(changes))

    def get_bandpass(self) -> np.ndarray:
        return self._t.sum(1).cpu().numpy()

    def dedisperse(self, dm: float, ref_freq: str | float = "fch1", *,
                   only_valid_samples: bool = False) -> "FilterbankBlock":
        """Per-channel roll by -delay (block.py:267-307 / kernels.roll_block)."""
        delays = np.atleast_1d(self.header.get_dmdelays(dm, ref_freq=ref_freq)).astype(np.int64)
        n = self.nsamples
        shifts = -delays
        if only_valid_samples:
            pmax, nmin = max(0, int(shifts.max())), min(0, int(shifts.min()))
            valid = n + nmin - pmax
            if valid <= 0:
                raise ValueError(f"Not enough samples. Required at least {pmax - nmin} "
                                 f"samples, given {n}.")
            t = torch.arange(valid, device=self._t.device)
            idx = (t[None, :] + pmax - torch.as_tensor(shifts, device=self._t.device)[:, None])
        else:
            t = torch.arange(n, device=self._t.device)
            sh = torch.as_tensor(np.mod(shifts, n), device=self._t.device)
            idx = torch.remainder(t[None, :] - sh[:, None], n)
        new = torch.gather(self._t, 1, idx)
        return FilterbankBlock(new, self.header.new_header({"nsamples": new.shape[1]}), dm)

    def _time_major(self) -> torch.Tensor:
        return self._t.t().contiguous()

    def dmt_transform(self, dm: float, dmsteps: int = 512, ref_freq: str | float = "fch1", *,
                      only_valid_samples: bool = False) -> "DMTBlock":
        """DM-time transform over ``dm + linspace(-dm, dm, dmsteps)`` (block.py:309-343).

        Default: the reference's semantics (kernels.dmt_block: each channel
        circularly rolled by +delay, summed).  ``only_valid_samples`` keeps the
        columns valid for every trial (the reference raises there whenever the
        trials' largest delays differ).
        """
        dm_arr = dm + np.linspace(-dm, dm, dmsteps)
        dm_delays = np.atleast_2d(self.header.get_dmdelays(dm_arr, ref_freq=ref_freq))
        n = self.nsamples
        tm = self._time_major()
        if only_valid_samples:
            pmax = max(0, int(dm_delays.max()))
            nmin = min(0, int(dm_delays.min()))
            valid = n + nmin - pmax
            if valid <= 0:
                raise ValueError(f"Not enough samples. Required at least {pmax - nmin} "
                                 f"samples, given {n}.")
            # res[i][t] = sum_c x[c][t + pmax - D[i][c]]
            d2 = (pmax - dm_delays).astype(np.int32)
            plan = DMTPlan(d2, self.nchans, n, nbits=32, mode="dedisperse", acc=_lib.ACC_F64)
            out = torch.zeros((dmsteps, valid), dtype=torch.float32, device=self._t.device)
            full = plan.execute(tm, n)
            out.copy_(full[:, :valid])
        else:
            d = np.mod(dm_delays.astype(np.int64), n).astype(np.int32)
            plan = DMTPlan(d, self.nchans, n, nbits=32, mode="roll", acc=_lib.ACC_F64)
            out = plan.execute(tm, n)
        plan.close()
        return DMTBlock(out, self.header.new_header({"nchans": 1}), dm_arr)


class DMTBlock(BaseBlock):
    """(ndms, nsamples) DM-time block."""

    def __init__(self, data, header: Header, dms):
        super().__init__(data, header)
        self._dms = np.asarray(dms, dtype=np.float32)
        if self.ndms != self._dms.size:
            raise ValueError(f"Number of DMs ({self.ndms}) does not match number of DM values "
                             f"({self._dms.size})")

    @property
    def dms(self) -> np.ndarray:
        return self._dms

    @property
    def ndms(self) -> int:
        return int(self._t.shape[0])
