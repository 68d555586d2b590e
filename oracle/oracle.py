"""ctypes bindings for the C oracle plus numpy restatements -- TEST INFRASTRUCTURE.

Every function restates a reference routine (FRBs/sigpyproc3,
``src/sigpyproc/...``) on the CPU; the file:line it follows is given in each
docstring.  These are the checkers for the CUDA library, never the product.
The restatements are pinned against the reference's own outputs by the
fixtures in ``tests/golden/``.
"""

from __future__ import annotations

import ctypes
import math
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"

_i64 = ctypes.c_int64
_i32 = ctypes.c_int32
_p = ctypes.c_void_p


def build(force: bool = False) -> Path:
    src = HERE / "spp_oracle.c"
    if force or not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-B" if force else "-s", "-C", str(HERE), "liboracle.so"],
                       check=True)
    return LIB


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(LIB))
        sig = {
            "orc_set_threads": ([ctypes.c_int], None),
            "orc_max_threads": ([], ctypes.c_int),
            "orc_unpack": ([_p, _i64, ctypes.c_int, ctypes.c_int, _p], None),
            "orc_dedisperse_u8": ([_p, _p, _p, _i64, _i64, _i64], _i64),
            "orc_dedisperse_f32": ([_p, _p, _p, _i64, _i64, _i64], _i64),
            "orc_dmt_u8_i32": ([_p, _p, _i64, _i64, _i64, _i64, _p, _i64], None),
            "orc_dmt_f32": ([_p, _p, _i64, _i64, _i64, _i64, _p, _p, _i64], None),
            "orc_dmt_rowmajor_u8": ([_p, _p, _i64, _i64, _i64, _i64, _p, _i64], None),
            "orc_dmt_roll_f32": ([_p, _p, _i64, _i64, _i64, _p], None),
            "orc_dmt_packed_i32": ([_p, ctypes.c_int, ctypes.c_int, _p, _i64, _i64, _i64, _i64,
                                    _p, _i64], None),
            "orc_bandpass_f32": ([_p, _i64, _i64, _p], None),
            "orc_bandpass_u8": ([_p, _i64, _i64, _p], None),
            "orc_collapse_f32": ([_p, _i64, _i64, _p, _i64], None),
            "orc_zero_dm_f32": ([_p, _p, _i64, _i64, _p, _p], None),
            "orc_downsample_mean": ([_p, _i64, ctypes.c_int, _p], None),
            "orc_boxcar_snr_row": ([_p, _i64, _p, ctypes.c_int, _p, ctypes.c_int, _p, _p], None),
            "orc_boxcar_snr_row_ls": ([_p, _i64, _p, ctypes.c_int, _p, ctypes.c_int, ctypes.c_int,
                                       _p, _p, _p, _p], None),
            "orc_median_iqr": ([_p, _i64, _p, _p], None),
            "orc_subband_u8": ([_p, _p, _p, _p, _i64, _i64, _i64, _i64], None),
            "orc_py_floordiv": ([ctypes.c_double, ctypes.c_double], ctypes.c_double),
            "orc_fold_block": ([_p, ctypes.c_int, _p, _p, _p, _i32, ctypes.c_float,
                                ctypes.c_float, ctypes.c_float, _i32, _i32, _i32, _i32, _i32,
                                _i32, _i32], None),
        }
        for name, (args, res) in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def _ptr(a: np.ndarray) -> int:
    assert a.flags.c_contiguous
    return a.ctypes.data


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


# ---------------------------------------------------------------------------
# R6: delays.  params.compute_dmdelays (params.py:26-62) with
# Header.chan_freqs (header.py:228-237): float32 NumPy arithmetic, the same
# expression order, round-half-even, int32.
# ---------------------------------------------------------------------------
DM_CONSTANT_LK = 4.148808e3


def chan_freqs(nchans: int, fch1: float, foff: float) -> np.ndarray:
    return np.arange(nchans, dtype=np.float32) * foff + fch1


def dmdelays(freqs, dm, tsamp: float, ref_freq: float, *, in_samples: bool = True):
    freqs = np.atleast_1d(freqs).astype(np.float32)
    dm = np.atleast_1d(dm)[:, np.newaxis].astype(np.float32)
    delays = dm * DM_CONSTANT_LK * ((freqs**-2) - (ref_freq**-2))
    if in_samples:
        delays = (delays / tsamp).round().astype(np.int32)
    return delays.squeeze()


# ---------------------------------------------------------------------------
# kernels wrappers
# ---------------------------------------------------------------------------
def unpack(packed: np.ndarray, nbits: int, bitorder: str = "big") -> np.ndarray:
    """kernels.unpack{1,2,4}_8_{big,little} (core/kernels.py:20-69)."""
    packed = np.ascontiguousarray(packed, dtype=np.uint8)
    out = np.empty(packed.size * 8 // nbits, dtype=np.uint8)
    lib().orc_unpack(_ptr(packed), packed.size, nbits, int(bitorder == "big"), _ptr(out))
    return out


def dedisperse(data: np.ndarray, delays: np.ndarray, nchans: int, nsamps: int,
               out: np.ndarray | None = None, out_start: int = 0) -> np.ndarray:
    """kernels.dedisperse (core/kernels.py:340-362) on a flat (nsamps*nchans) block."""
    data = np.ascontiguousarray(data)
    delays = np.ascontiguousarray(delays, dtype=np.int32)
    nvalid = nsamps - int(np.max(np.abs(delays)))
    if out is None:
        out = np.zeros(max(nvalid, 0) + out_start, dtype=np.float32)
    if data.dtype == np.uint8:
        lib().orc_dedisperse_u8(_ptr(data), _ptr(out), _ptr(delays), nchans, nsamps, out_start)
    elif data.dtype == np.float32:
        lib().orc_dedisperse_f32(_ptr(data), _ptr(out), _ptr(delays), nchans, nsamps, out_start)
    else:
        raise TypeError(data.dtype)
    return out


def dmt(data: np.ndarray, delays: np.ndarray, nchans: int, nsamps: int,
        nvalid: int | None = None, want64: bool = False):
    """Row-wise DM batch: out[i] = kernels.dedisperse(data, delays[i])[:nvalid]."""
    data = np.ascontiguousarray(data)
    delays = np.ascontiguousarray(np.atleast_2d(delays), dtype=np.int32)
    ndm = delays.shape[0]
    if nvalid is None:
        nvalid = nsamps - int(np.max(np.abs(delays)))
    if data.dtype == np.uint8:
        out = np.zeros((ndm, nvalid), dtype=np.int32)
        lib().orc_dmt_u8_i32(_ptr(data), _ptr(delays), ndm, nchans, nsamps, nvalid, _ptr(out), nvalid)
        return out
    out = np.zeros((ndm, nvalid), dtype=np.float32)
    out64 = np.zeros((ndm, nvalid), dtype=np.float64) if want64 else None
    lib().orc_dmt_f32(_ptr(data), _ptr(delays), ndm, nchans, nsamps, nvalid, _ptr(out),
                      _ptr(out64) if want64 else None, nvalid)
    return (out, out64) if want64 else out


def dmt_rowmajor(data_u8: np.ndarray, delays: np.ndarray, nchans: int, nsamps: int,
                 nvalid: int) -> np.ndarray:
    """CPU baseline loop (kernels.dedisperse order per DM row, rows in parallel)."""
    data_u8 = np.ascontiguousarray(data_u8, dtype=np.uint8)
    delays = np.ascontiguousarray(np.atleast_2d(delays), dtype=np.int32)
    out = np.zeros((delays.shape[0], nvalid), dtype=np.int32)
    lib().orc_dmt_rowmajor_u8(_ptr(data_u8), _ptr(delays), delays.shape[0], nchans, nsamps, nvalid,
                              _ptr(out), nvalid)
    return out


def dmt_packed(packed: np.ndarray, nbits: int, bitorder: str, delays: np.ndarray, nchans: int,
               nsamps: int, nvalid: int) -> np.ndarray:
    packed = np.ascontiguousarray(packed, dtype=np.uint8)
    delays = np.ascontiguousarray(np.atleast_2d(delays), dtype=np.int32)
    ndm = delays.shape[0]
    out = np.zeros((ndm, nvalid), dtype=np.int32)
    lib().orc_dmt_packed_i32(_ptr(packed), nbits, int(bitorder == "big"), _ptr(delays), ndm,
                             nchans, nsamps, nvalid, _ptr(out), nvalid)
    return out


def dmt_roll(data_tm: np.ndarray, delays: np.ndarray, nchans: int, nsamps: int) -> np.ndarray:
    """kernels.dmt_block (core/kernels.py:1155-1168) on time-major float32 data."""
    data_tm = np.ascontiguousarray(data_tm, dtype=np.float32)
    delays = np.ascontiguousarray(np.atleast_2d(delays), dtype=np.int32)
    out = np.zeros((delays.shape[0], nsamps), dtype=np.float32)
    lib().orc_dmt_roll_f32(_ptr(data_tm), _ptr(delays), delays.shape[0], nchans, nsamps, _ptr(out))
    return out


def bandpass(data: np.ndarray, nchans: int, nsamps: int, bpass: np.ndarray | None = None):
    """kernels.extract_bpass (core/kernels.py:281-292), sequential float32."""
    bpass = np.zeros(nchans, np.float32) if bpass is None else bpass
    data = np.ascontiguousarray(data)
    fn = lib().orc_bandpass_u8 if data.dtype == np.uint8 else lib().orc_bandpass_f32
    fn(_ptr(data), nchans, nsamps, _ptr(bpass))
    return bpass


def collapse(data: np.ndarray, nchans: int, nsamps: int, tim: np.ndarray, out_start: int = 0):
    """kernels.extract_tim (core/kernels.py:255-278) for float32 data."""
    data = np.ascontiguousarray(data, dtype=np.float32)
    lib().orc_collapse_f32(_ptr(data), nchans, nsamps, _ptr(tim), out_start)
    return tim


def zero_dm(data: np.ndarray, nchans: int, nsamps: int, bpass: np.ndarray) -> np.ndarray:
    """kernels.remove_zerodm (core/kernels.py:465-505), float32 data."""
    data = np.ascontiguousarray(data, dtype=np.float32)
    bpass = np.ascontiguousarray(bpass, dtype=np.float32)
    chanwts = bpass / bpass.sum()
    out = np.empty_like(data)
    lib().orc_zero_dm_f32(_ptr(data), _ptr(out), nchans, nsamps, _ptr(bpass), _ptr(chanwts))
    return out


def downsample_mean(x: np.ndarray, factor: int) -> np.ndarray:
    """kernels.downsample_1d_mean (core/kernels.py:176-204)."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty(x.size // factor, dtype=np.float32)
    lib().orc_downsample_mean(_ptr(x), x.size, factor, _ptr(out))
    return out


def boxcar_snr(rows: np.ndarray, factors, widths, loc_scale: str = "mean_std",
               return_loc_scale: bool = False):
    """Boxcar S/N peaks per row (float64) and argmax indices: TimeSeries.downsample
    (timeseries.py:107-132) then a square-normalised boxcar (apply_boxcar,
    timeseries.py:296-325) over the series z-scored by stats.estimate_zscore
    (core/stats.py:418-502) with loc/scale "mean_std" or "median_iqr"."""
    rows = np.atleast_2d(rows)
    factors = np.ascontiguousarray(factors, dtype=np.int32)
    widths = np.ascontiguousarray(widths, dtype=np.int32)
    snr = np.zeros((rows.shape[0], factors.size, widths.size), dtype=np.float64)
    idx = np.zeros(snr.shape, dtype=np.int32)
    locs = np.zeros((rows.shape[0], factors.size), dtype=np.float64)
    scales = np.zeros_like(locs)
    robust = {"mean_std": 0, "median_iqr": 1}[loc_scale]
    for r in range(rows.shape[0]):
        row = np.ascontiguousarray(rows[r], dtype=np.float32)
        lib().orc_boxcar_snr_row_ls(_ptr(row), row.size, _ptr(factors), factors.size,
                                    _ptr(widths), widths.size, robust, snr[r].ctypes.data,
                                    idx[r].ctypes.data, locs[r].ctypes.data,
                                    scales[r].ctypes.data)
    if return_loc_scale:
        return snr, idx, locs, scales
    return snr, idx


def apply_boxcar(x: np.ndarray, width: int) -> np.ndarray:
    """TimeSeries.apply_boxcar (timeseries.py:296-325) over stats.running_filter
    "mean" (core/stats.py:200-243): np.pad "symmetric", window means (exact
    float64 window sums here; the reference's bottleneck keeps a float32
    running sum), times sqrt(width), np.roll by the reference bin."""
    x = np.asarray(x, dtype=np.float32)
    pad = (width // 2, width // 2) if width % 2 else (width // 2, width // 2 - 1)
    xp = np.pad(x, pad, "symmetric").astype(np.float64)
    win = np.lib.stride_tricks.sliding_window_view(xp, width)
    mean = np.fromiter((math.fsum(w_) for w_ in win), dtype=np.float64, count=win.shape[0]) / width
    out = (mean * math.sqrt(width)).astype(np.float32)
    ref_bin = -width // 2 + 1 if width % 2 else -width // 2
    return np.roll(out, ref_bin)


def median_iqr(y: np.ndarray) -> tuple[float, float]:
    """(median, IQR / 1.349) of float32 values as stats.estimate_zscore computes them."""
    y = np.ascontiguousarray(y, dtype=np.float32)
    loc, scale = ctypes.c_double(), ctypes.c_double()
    lib().orc_median_iqr(_ptr(y), y.size, ctypes.byref(loc), ctypes.byref(scale))
    return loc.value, scale.value


def subband(data: np.ndarray, delays: np.ndarray, chan_to_sub: np.ndarray, maxdelay: int,
            nchans: int, nsub: int, nsamps: int) -> np.ndarray:
    """kernels.subband (core/kernels.py:379-401) with a zeroed output."""
    data = np.ascontiguousarray(data, dtype=np.uint8)
    delays = np.ascontiguousarray(delays, dtype=np.int32)
    chan_to_sub = np.ascontiguousarray(chan_to_sub, dtype=np.int32)
    out = np.zeros((nsamps - maxdelay) * nsub, dtype=np.float32)
    lib().orc_subband_u8(_ptr(data), _ptr(out), _ptr(delays), _ptr(chan_to_sub), maxdelay,
                         nchans, nsub, nsamps)
    return out


# ---------------------------------------------------------------------------
# readers.FilReader.read_plan schedule (readers.py:182-216)
# ---------------------------------------------------------------------------
def read_plan_blocks(nsamples: int, gulp: int = 16384, start: int = 0, nsamps: int | None = None,
                     skipback: int = 0) -> list[tuple[int, int, int]]:
    """(ii, samples in block, skip) for each block, or ValueError as the reference."""
    if nsamps is None:
        nsamps = nsamples - start
    gulp = min(nsamps, gulp)
    skipback = abs(skipback)
    if skipback >= gulp:
        raise ValueError(f"readsamps ({gulp}) must be > skipback ({skipback})")
    nreads, lastread = divmod(nsamps, (gulp - skipback))
    if lastread < skipback:
        nreads -= 1
        lastread = nsamps - (nreads * (gulp - skipback))
    blocks = [(ii, gulp, -skipback) for ii in range(nreads)]
    if lastread != 0:
        blocks.append((nreads, lastread, 0))
    return blocks


# ---------------------------------------------------------------------------
# kernels.fold (core/kernels.py:403-445) and Filterbank.fold (base.py:1109-1207)
# ---------------------------------------------------------------------------
def fold_block(data: np.ndarray, fold_ar: np.ndarray, count_ar: np.ndarray, delays: np.ndarray,
               maxdelay: int, tsamp: float, period: float, accel: float, total_nsamps: int,
               nsamps: int, nchans: int, nbins: int, nints: int, nsubs: int, index: int) -> None:
    """One read_plan block of kernels.fold, accumulated into fold_ar / count_ar."""
    data = np.ascontiguousarray(data)
    delays = np.ascontiguousarray(delays, dtype=np.int32)
    if data.dtype not in (np.uint8, np.float32):
        raise TypeError(data.dtype)
    lib().orc_fold_block(_ptr(data), int(data.dtype == np.float32), _ptr(fold_ar), _ptr(count_ar),
                         _ptr(delays), maxdelay, tsamp, period, accel, total_nsamps, nsamps,
                         nchans, nbins, nints, nsubs, index)


def filterbank_fold(data: np.ndarray, nsamples: int, nchans: int, delays: np.ndarray,
                    tsamp: float, period: float, accel: float, nbins: int, nints: int,
                    nbands: int, gulp: int):
    """Filterbank.fold's block loop (base.py:1151-1206) over a time-major array:
    returns (sums, counts, cube) with the reference's final float32 division."""
    nbands = min(nbands, nchans)
    maxd = int(np.max(delays))
    gulp = max(2 * maxd, gulp)
    fold_ar = np.zeros(nbins * nints * nbands, dtype=np.float32)
    count_ar = np.zeros(nbins * nints * nbands, dtype=np.int32)
    pos = 0
    for ii, nblk, skip in read_plan_blocks(nsamples, gulp, 0, None, maxd):
        blk = data[pos * nchans:(pos + nblk) * nchans]
        fold_block(blk, fold_ar, count_ar, delays, maxd, tsamp, period, accel, nsamples, nblk,
                   nchans, nbins, nints, nbands, ii * (gulp - maxd))
        pos += nblk + skip
    sums, counts = fold_ar.copy(), count_ar.copy()
    with np.errstate(divide="ignore", invalid="ignore"):
        fold_ar /= count_ar
    return sums, counts, fold_ar.reshape(nints, nbands, nbins)


# ---------------------------------------------------------------------------
# MatchedFilter (core/filters.py:29-365) with kernels.convolve_templates
# (core/kernels.py:861-906) and normalize_template (:1008-1027), restated with
# numpy's float64 FFT over the series repeated to pocketfft's good length for
# real transforms (scipy.fft.next_fast_len(n, real=True): the same pocketfft
# rule the reference reaches through rocket_fft.good_size).
# ---------------------------------------------------------------------------
def mad_scale(x: np.ndarray) -> float:
    """stats._scale_mad (core/stats.py:505-536): the median absolute deviation
    from the float64 median over Phi^-1(3/4); when that is within 1e-8 of 0,
    the mean absolute deviation over sqrt(2/pi)."""
    d = np.asarray(x, dtype=np.float64)
    loc = np.median(d)
    mad = np.median(np.abs(d - loc)) / 0.6744897501960817
    if np.isclose(mad, 0):
        mad = np.mean(np.abs(d - loc)) / np.sqrt(2 / np.pi)
    return float(mad)


def zscore_f32(x: np.ndarray, loc_method: str, scale_method: str):
    """stats.estimate_zscore (core/stats.py:418-477) on a float32 series."""
    x = np.asarray(x, dtype=np.float32)
    if loc_method == "median":
        loc = np.median(x)
    elif loc_method == "mean":
        loc = np.mean(x, dtype=np.float64)
    else:
        loc = np.float32(0.0)
    # the scale is a float64 array in the reference (a strong type): the
    # division runs in float64 and rounds into the float32 output
    if scale_method == "iqr":
        q = np.percentile(x.astype(np.float64), [25, 75])
        scale = np.float64((q[1] - q[0]) / 1.3489795003921634)
    elif scale_method == "std":
        scale = np.float64(np.std(x.astype(np.float64)))
    elif scale_method == "mad":
        scale = np.float64(mad_scale(x))
    else:
        scale = np.float32(1.0)
    if np.isclose(scale, 0):
        scale = np.float64(1.0)
    z = np.subtract(x, loc, dtype=np.float32)
    np.divide(z, scale, out=z)
    return z, loc, float(scale)


def template_bank(kind: str, nbins_max: int = 32, spacing_factor: float = 1.5):
    """(widths, [(data, ref_bin)]) as MatchedFilter._setup_templates and the
    Template.gen_* constructors (core/filters.py:290-310, :508-579) build them."""
    if kind == "boxcar":
        widths = [1]
        while widths[-1] < nbins_max:
            nxt = int(max(widths[-1] + 1, spacing_factor * widths[-1]))
            if nxt > nbins_max:
                break
            widths.append(nxt)
        widths = np.array(widths, dtype=np.float32)
        return widths, [(np.ones(int(w), dtype=np.float32), 0) for w in widths]
    npoints = int(np.ceil(np.log(nbins_max) / np.log(spacing_factor))) + 1
    widths = np.geomspace(1, nbins_max, npoints)
    bank = []
    for w in widths:
        if kind == "gaussian":
            sd = w / (2.0 * np.sqrt(2.0 * np.log(2.0)))
            size = int(np.ceil(3.5 * sd))
            x = np.arange(-size, size + 1)
            bank.append((np.exp(-0.5 * x**2 / sd**2), len(x) // 2))
        else:
            g = w / 2
            size = int(np.ceil(3.5 * g))
            x = np.arange(-size, size + 1)
            bank.append((g**2 / (x**2 + g**2), len(x) // 2))
    return widths, bank


def matched_filter(data: np.ndarray, loc_method: str = "median", scale_method: str = "iqr",
                   kind: str = "boxcar", nbins_max: int = 32, spacing_factor: float = 1.5):
    """Returns (z, convs float64 (ntemps, n), itemp, peak_bin, snr)."""
    from scipy import fft as sfft

    z, _, _ = zscore_f32(data, loc_method, scale_method)
    n = z.size
    nfft = sfft.next_fast_len(n, real=True)
    data_pad = z[np.arange(nfft) % n].astype(np.float64)
    dfft = np.fft.rfft(data_pad)
    _, bank = template_bank(kind, nbins_max, spacing_factor)
    convs = np.empty((len(bank), n), dtype=np.float64)
    for k, (h, ref) in enumerate(bank):
        tp = np.zeros(nfft)
        tp[:h.size] = h
        tp = np.roll(tp, -ref)
        tp = np.roll(tp[::-1], 1)
        tp = tp - tp.mean()
        nrm = np.sqrt(np.sum(tp**2))
        if nrm != 0:
            tp = tp / nrm
        convs[k] = np.fft.irfft(dfft * np.fft.rfft(tp), nfft)[:n]
    itemp, peak = np.unravel_index(int(np.argmax(convs)), convs.shape)
    return z, convs, int(itemp), int(peak), float(convs[itemp, peak])
