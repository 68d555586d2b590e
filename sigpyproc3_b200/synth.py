"""Seeded synthetic filterbanks for the benchmark workloads.

No public dataset is involved: every input is generated here from a seed.

* Small (CPU-sized) inputs use ``numpy.random.default_rng(seed)``.
* Large inputs are generated on the GPU with a counter-based hash (the
  SplitMix64 finaliser of Steele, Lea & Flood 2014 applied to
  ``seed << 40 ^ index``): uniform bytes, or Gaussian-shaped uint8 through a
  256-entry CDF threshold table built here in float64.  The integer outputs
  are a pure function of (seed, index), so the test suite's numpy twins of
  these generators regenerate any slice on the host byte for byte.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import params


def gauss_u8_thresholds(mean: float, std: float) -> np.ndarray:
    """uint32 thresholds T[v] = floor(2**32 * P(round(X) <= v)), X ~ N(mean, std),
    clipped to [0, 255].  value = #{v < 255 : u >= T[v]} for a uniform u32."""
    t = np.empty(255, dtype=np.uint64)
    for v in range(255):
        p = 0.5 * (1.0 + math.erf((v + 0.5 - mean) / (std * math.sqrt(2.0))))
        t[v] = min(int(p * 2**32), 2**32 - 1)
    return t.astype(np.uint32)


# ---------------------------------------------------------------------------
# Workload descriptions
# ---------------------------------------------------------------------------
@dataclass(frozen=True)
class Geometry:
    nchans: int
    nsamps: int
    nbits: int
    tsamp: float
    fch1: float
    foff: float

    def chan_freqs(self) -> np.ndarray:
        return np.arange(self.nchans, dtype=np.float32) * self.foff + self.fch1

    def delays(self, dm, ref_freq: float | None = None) -> np.ndarray:
        fref = self.fch1 if ref_freq is None else ref_freq
        return params.compute_dmdelays(self.chan_freqs(), dm, self.tsamp, fref)


C1 = Geometry(nchans=256, nsamps=65536, nbits=8, tsamp=64e-6, fch1=1500.0, foff=-1.0)
C2 = Geometry(nchans=4096, nsamps=2**20, nbits=2, tsamp=64e-6, fch1=1500.0, foff=-0.0732421875)
C3 = Geometry(nchans=1024, nsamps=2**21, nbits=8, tsamp=64e-6, fch1=1400.0, foff=-0.29296875)
C5 = Geometry(nchans=4096, nsamps=2**21, nbits=32, tsamp=64e-6, fch1=1500.0, foff=-0.0732421875)


def dm_grid(dm: float, dmsteps: int) -> np.ndarray:
    """DM trials of FilterbankBlock.dmt_transform (block.py:337): dm + linspace(-dm, dm)."""
    return dm + np.linspace(-dm, dm, dmsteps)


def c1_filterbank(seed: int = 1) -> np.ndarray:
    """Config 1: uint8 (65536, 256), N(128, 16) rounded and clipped, plus one
    dispersed Gaussian pulse (FWHM 1 ms, +20 counts) at sample 30000 at fch1,
    DM 100.  Returns the flat time-major byte array."""
    g = C1
    rng = np.random.default_rng(seed)
    x = rng.normal(128.0, 16.0, size=(g.nsamps, g.nchans))
    d = g.delays(100.0).astype(np.int64)
    sigma = (1e-3 / g.tsamp) / (2.0 * math.sqrt(2.0 * math.log(2.0)))
    half = int(math.ceil(5 * sigma))
    k = np.arange(-half, half + 1)
    prof = 20.0 * np.exp(-0.5 * (k / sigma) ** 2)
    for c in range(g.nchans):
        rows = 30000 + d[c] + k
        ok = (rows >= 0) & (rows < g.nsamps)
        x[rows[ok], c] += prof[ok]
    return np.clip(np.rint(x), 0, 255).astype(np.uint8).ravel()


# Pulse sets injected by the device generators: (DM, sample at fch1)
C2_PULSES = ((250.0, 200_000), (900.0, 500_000), (1700.0, 800_000))
C2_PULSE_WIDTH = 31  # samples (~2 ms at 64 us)


def c2_pulse_rows(g: Geometry = C2) -> list[np.ndarray]:
    """Per pulse, the int32 start row of the pulse window for each channel."""
    return [(t + g.delays(dm)).astype(np.int64) - C2_PULSE_WIDTH // 2 for dm, t in C2_PULSES]


# ---------------------------------------------------------------------------
# Device generators (libsppgpu spp_synth_*)
# ---------------------------------------------------------------------------
def _dev_stream(stream=None) -> int:
    import torch

    return (stream or torch.cuda.current_stream()).cuda_stream


def uniform_bytes_device(n: int, seed: int, start: int = 0, out=None, stream=None):
    import torch

    from . import _lib

    if out is None:
        out = torch.empty(n, dtype=torch.uint8, device="cuda")
    _lib.call("spp_synth_uniform_bytes", out.data_ptr(), start, n, seed, _dev_stream(stream))
    return out


def gauss_u8_device(n: int, seed: int, mean: float, std: float, start: int = 0, out=None,
                    stream=None):
    import torch

    from . import _lib

    th = np.ascontiguousarray(gauss_u8_thresholds(mean, std), dtype=np.uint32)
    if out is None:
        out = torch.empty(n, dtype=torch.uint8, device="cuda")
    _lib.call("spp_synth_gauss_u8", out.data_ptr(), start, n, seed, th.ctypes.data,
              _dev_stream(stream))
    return out


def gauss_f32_device(n: int, seed: int, mean: float = 0.0, std: float = 1.0, start: int = 0,
                     out=None, stream=None):
    import torch

    from . import _lib

    if out is None:
        out = torch.empty(n, dtype=torch.float32, device="cuda")
    _lib.call("spp_synth_gauss_f32", out.data_ptr(), start, n, seed, mean, std, _dev_stream(stream))
    return out


def c2_filterbank_device(g: Geometry = C2, seed: int = 2, stream=None):
    """Config 2 on the device: uniform 2-bit packed samples + three pulses
    (+1 level over C2_PULSE_WIDTH samples, saturating at 3)."""
    import torch

    from . import _lib

    nbytes = g.nsamps * g.nchans * g.nbits // 8
    raw = uniform_bytes_device(nbytes, seed, stream=stream)
    for rows in c2_pulse_rows(g):
        r = torch.from_numpy(np.ascontiguousarray(rows, dtype=np.int64)).cuda()
        _lib.call("spp_synth_pulse_packed", raw.data_ptr(), g.nchans, g.nsamps, g.nbits,
                  _lib.BITORDER_BIG, r.data_ptr(), C2_PULSE_WIDTH, _dev_stream(stream))
        torch.cuda.current_stream().synchronize()
    return raw
