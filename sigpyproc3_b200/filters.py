"""Matched filtering of a time series with a bank of pulse templates (next row
N3 of the path): ``MatchedFilter`` and ``Template`` with the reference's API
(src/sigpyproc/core/filters.py:29-587).

The z-score, the template correlations and the peak search run on the GPU
(``spp_row_loc_scale``, ``spp_zscore``, ``spp_matched_filter``); the
template bank itself is a handful of short arrays built here with numpy, as
the reference builds it.  The reference correlates by FFT over the series
repeated to pocketfft's good length; the kernel computes the same circular
correlation directly in float64.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .dedisp import stream_handle

# astropy.stats.gaussian_fwhm_to_sigma
GAUSSIAN_FWHM_TO_SIGMA = 1.0 / (2.0 * math.sqrt(2.0 * math.log(2.0)))


def good_size_real(n: int) -> int:
    """Smallest 2^a 3^b 5^c >= n (pocketfft's good size for real transforms,
    which the reference obtains through rocket_fft.good_size(n, real=True)
    in kernels.circular_pad_goodsize, core/kernels.py:990-998); n itself for
    n <= 6."""
    n = int(n)
    if n <= 6:
        return n
    best = 2 * n
    f5 = 1
    while f5 < best:
        x = f5
        while x < n:
            x *= 2
        while True:
            if x < n:
                x *= 3
            elif x > n:
                best = min(best, x)
                if x & 1:
                    break
                x >>= 1
            else:
                return n
        f5 *= 5
    return best


@dataclass(frozen=True)
class ZScoreResult:
    data: np.ndarray
    loc: np.ndarray
    scale: np.ndarray


@dataclass(frozen=True, eq=False)
class Template:
    """A pulse template (filters.py:366-587): samples, width, reference bin.
    Templates compare by identity (their samples are arrays)."""

    data: np.ndarray
    width: float
    ref_bin: int = 0
    ref: str = "start"
    kind: str = "custom"

    def __post_init__(self):
        if not self.data.size:
            raise ValueError("Empty data array is not supported.")
        if self.data.ndim != 1:
            raise ValueError(f"Only 1D data is supported, got {self.data.ndim}.")
        if self.ref_bin >= self.data.size or self.ref_bin < 0:
            raise ValueError(f"Reference bin {self.ref_bin} is out of bounds.")
        if self.ref not in {"start", "peak"}:
            raise ValueError(f"ref must be 'start' or 'peak', got {self.ref}")

    @classmethod
    def gen_boxcar(cls, width: int) -> "Template":
        width = int(width)
        if width <= 0:
            raise ValueError(f"Width {width} must be greater than 0.")
        return cls(np.ones(width, dtype=np.float32), width, ref_bin=0, ref="start", kind="boxcar")

    @classmethod
    def gen_gaussian(cls, width: float, extent: float = 3.5) -> "Template":
        if width <= 0:
            raise ValueError(f"Width {width} must be greater than 0.")
        stddev = GAUSSIAN_FWHM_TO_SIGMA * width
        size = int(np.ceil(extent * stddev))
        x = np.arange(-size, size + 1)
        arr = np.exp(-0.5 * x**2 / stddev**2)
        return cls(arr, width, ref_bin=len(x) // 2, ref="peak", kind="gaussian")

    @classmethod
    def gen_lorentzian(cls, width: float, extent: float = 3.5) -> "Template":
        if width <= 0:
            raise ValueError(f"Width {width} must be greater than 0.")
        gamma = width / 2
        size = int(np.ceil(extent * gamma))
        x = np.arange(-size, size + 1)
        arr = gamma**2 / (x**2 + gamma**2)
        return cls(arr, width, ref_bin=len(x) // 2, ref="peak", kind="lorentzian")

    def get_model(self, peak_bin: int, nbins: int) -> np.ndarray:
        """The template zero-padded to nbins, normalised to zero mean and unit
        power, with its reference bin at peak_bin (filters.py:443-460)."""
        padded = np.pad(self.data, (0, nbins - self.data.size))
        arr = padded - np.mean(padded)
        norm = np.sqrt(np.sum(arr**2))
        if norm != 0:
            arr = arr / norm
        return np.roll(arr, peak_bin - self.ref_bin)

    def get_on_pulse(self, peak_bin: int, nbins: int) -> tuple[int, int]:
        if self.ref == "start":
            left, right = peak_bin, peak_bin + self.width
        else:
            left, right = peak_bin - round(self.width), peak_bin + round(self.width)
        return (max(0, left), int(min(nbins, right)))

    def __str__(self) -> str:
        return f"Template(size={self.data.size}, kind={self.kind}, width={self.width:.3f})"


def get_box_width_spacing(size_max: int, spacing_factor: float = 1.5) -> np.ndarray:
    """Boxcar widths 1, then max(w + 1, int(spacing * w)) up to size_max (filters.py:340-365)."""
    widths = [1]
    while widths[-1] < size_max:
        nxt = int(max(widths[-1] + 1, spacing_factor * widths[-1]))
        if nxt > size_max:
            break
        widths.append(nxt)
    return np.array(widths, dtype=np.float32)


class MatchedFilter:
    """Matched filter of a 1-D series against a template bank (filters.py:29-338):
    z-score by ``loc_method`` / ``scale_method``, correlate with every
    template, keep the best (template, sample)."""

    def __init__(self, data, loc_method: str = "median", scale_method: str = "iqr",
                 temp_kind: str = "boxcar", nbins_max: int = 32, spacing_factor: float = 1.5):
        x = data if torch.is_tensor(data) else torch.as_tensor(np.asarray(data, dtype=np.float32))
        if x.dim() != 1:
            raise ValueError(f"Data dimension {x.dim()} is not supported.")
        if loc_method not in {"median", "mean", "norm"}:
            raise ValueError(f"Method {loc_method} is not supported for estimating location.")
        if scale_method not in {"iqr", "mad", "std", "norm"}:
            raise NotImplementedError(f"scale_method {scale_method!r} is not on the GPU path "
                                      "(iqr, mad, std or norm)")
        if temp_kind not in {"boxcar", "gaussian", "lorentzian"}:
            raise ValueError(f"unknown template kind {temp_kind!r}")
        if x.numel() == 0:
            raise ValueError("Cannot estimate Z-scores from an empty array.")
        self._x = x.to(torch.float32).cuda().contiguous()
        self._temp_kind = temp_kind
        self._setup_templates(nbins_max, spacing_factor)
        self._zscore(loc_method, scale_method)
        self._compute()

    # ---- reference attributes ----
    @property
    def data(self) -> np.ndarray:
        return self._x.cpu().numpy()

    @property
    def zscores(self) -> ZScoreResult:
        return ZScoreResult(self._z.cpu().numpy(), np.asarray([self._loc]), np.asarray([self._scale]))

    @property
    def temp_kind(self) -> str:
        return self._temp_kind

    @property
    def temp_widths(self) -> np.ndarray:
        return self._temp_widths

    @property
    def temp_bank(self) -> list[Template]:
        return self._temp_bank

    @property
    def convs(self) -> np.ndarray:
        return self._convs.cpu().numpy()

    @property
    def peak_bin(self) -> int:
        return int(self._peak_bin)

    @property
    def best_temp(self) -> Template:
        return self._temp_bank[self._itemp]

    @property
    def snr(self) -> float:
        return float(self._snr)

    @property
    def best_model(self) -> np.ndarray:
        return self.best_temp.get_model(self.peak_bin, self._x.numel())

    @property
    def on_pulse(self) -> tuple[int, int]:
        return self.best_temp.get_on_pulse(self.peak_bin, self._x.numel())

    get_box_width_spacing = staticmethod(get_box_width_spacing)

    # ---- computation ----
    def _setup_templates(self, nbins_max: int, spacing_factor: float) -> None:
        if self._temp_kind == "boxcar":
            self._temp_widths = get_box_width_spacing(nbins_max, spacing_factor)
        else:
            if spacing_factor <= 1:
                raise ValueError("Spacing factor must be greater than 1 for non-boxcar templates.")
            npoints = int(np.ceil(np.log(nbins_max) / np.log(spacing_factor))) + 1
            self._temp_widths = np.geomspace(1, nbins_max, npoints)
        bank = []
        for width in self._temp_widths:
            temp = getattr(Template, f"gen_{self._temp_kind}")(width)
            if temp.data.size > self._x.numel():
                raise ValueError(f"Template size ({temp.data.size}) is larger than the data "
                                 f"size({self._x.numel()}).")
            bank.append(temp)
        self._temp_bank = bank

    def _zscore(self, loc_method: str, scale_method: str) -> None:
        lib = _lib.load()
        st = stream_handle(None, self._x.device)
        n = self._x.numel()
        ls = torch.tensor([0.0, 1.0], dtype=torch.float64, device=self._x.device)
        robust = torch.empty(2, dtype=torch.float64, device=self._x.device)
        plain = torch.empty(2, dtype=torch.float64, device=self._x.device)
        if "median" == loc_method or "iqr" == scale_method:
            _lib.check(lib.spp_row_loc_scale(self._x.data_ptr(), _lib.OUT_F32, 1, n, n, 1,
                                             robust.data_ptr(), st))
        if "mean" == loc_method or "std" == scale_method:
            _lib.check(lib.spp_row_loc_scale(self._x.data_ptr(), _lib.OUT_F32, 1, n, n, 0,
                                             plain.data_ptr(), st))
        mad = torch.empty(2, dtype=torch.float64, device=self._x.device)
        if scale_method == "mad":
            _lib.check(lib.spp_row_loc_scale(self._x.data_ptr(), _lib.OUT_F32, 1, n, n, 2,
                                             mad.data_ptr(), st))
        if loc_method != "norm":
            ls[0] = (robust if loc_method == "median" else plain)[0]
        if scale_method != "norm":
            ls[1] = {"iqr": robust, "mad": mad, "std": plain}[scale_method][1]
        self._z = torch.empty_like(self._x)
        _lib.check(lib.spp_zscore(self._x.data_ptr(), n, ls.data_ptr(), self._z.data_ptr(), st))
        host = ls.cpu().numpy()
        self._loc = np.float32(host[0]) if loc_method == "median" else host[0]
        self._scale = host[1]

    def _compute(self) -> None:
        n = self._x.numel()
        nfft = good_size_real(n)
        dev = self._x.device
        datas = [np.asarray(t.data, dtype=np.float64) for t in self._temp_bank]
        offs = np.concatenate([[0], np.cumsum([d.size for d in datas])]).astype(np.int32)
        stats = []
        for d in datas:
            s1, s2 = float(np.sum(d)), float(np.sum(d * d))
            stats += [s1 / nfft, math.sqrt(max(s2 - s1 * s1 / nfft, 0.0))]
        temps = torch.from_numpy(np.concatenate(datas)).to(dev)
        toff = torch.from_numpy(offs).to(dev)
        tref = torch.from_numpy(np.array([t.ref_bin for t in self._temp_bank], np.int32)).to(dev)
        tstat = torch.from_numpy(np.array(stats, np.float64)).to(dev)
        k = len(self._temp_bank)
        self._convs = torch.empty((k, n), dtype=torch.float32, device=dev)
        ws = torch.zeros(2, dtype=torch.float64, device=dev)
        _lib.check(_lib.load().spp_matched_filter(
            self._z.data_ptr(), n, nfft, temps.data_ptr(), toff.data_ptr(), tref.data_ptr(),
            tstat.data_ptr(), k, self._convs.data_ptr(), ws.data_ptr(), 16,
            stream_handle(None, dev)))
        key = int(ws.view(torch.int64)[1].item()) & ((1 << 64) - 1)
        flat = 0xFFFFFFFF - (key & 0xFFFFFFFF)
        self._itemp, self._peak_bin = divmod(flat, n)
        self._snr = self._convs[self._itemp, self._peak_bin].item()
