"""Host twins of the seeded synthetic generators -- TEST INFRASTRUCTURE ONLY.

The device generators (``sigpyproc3_b200.synth``, ``spp_synth_*``) hash
``seed << 40 ^ index`` with the SplitMix64 finaliser (Steele, Lea & Flood
2014) into uniform bytes, or into Gaussian-shaped uint8 through a 256-entry
threshold table.  The functions here produce the same bytes in numpy, so the
tests can regenerate any slice of a benchmark input on the host, and the CPU
baseline (``bench.py --impl reference``) can build the config-2 sample without
loading the CUDA library.  Nothing here imports the product package; the
tests pin these twins against the device generators byte for byte.
"""

from __future__ import annotations

import math

import numpy as np

from . import oracle as orc

# config 2: 2-bit packed filterbank, 4096 channels x 2**20 samples
C2_NCHANS = 4096
C2_NSAMPS = 1 << 20
C2_NBITS = 2
C2_TSAMP = 64e-6
C2_FCH1 = 1500.0
C2_FOFF = -0.0732421875
C2_SEED = 2
# injected pulses: (DM, sample at fch1), +1 level over C2_PULSE_WIDTH samples
C2_PULSES = ((250.0, 200_000), (900.0, 500_000), (1700.0, 800_000))
C2_PULSE_WIDTH = 31


def hash_u64(seed: int, index: np.ndarray) -> np.ndarray:
    """SplitMix64 finaliser of ``seed << 40 ^ index`` (uint64, vectorised)."""
    with np.errstate(over="ignore"):
        z = (np.uint64(seed) << np.uint64(40)) ^ index.astype(np.uint64)
        z = z + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def uniform_bytes_host(seed: int, start: int, count: int) -> np.ndarray:
    """Bytes [start, start + count) of the uniform-byte generator."""
    idx = np.arange(start, start + count, dtype=np.uint64)
    return (hash_u64(seed, idx) & np.uint64(0xFF)).astype(np.uint8)


def gauss_u8_thresholds(mean: float, std: float) -> np.ndarray:
    """T[v] = floor(2**32 * P(round(X) <= v)), X ~ N(mean, std), v < 255."""
    t = np.empty(255, dtype=np.uint64)
    for v in range(255):
        p = 0.5 * (1.0 + math.erf((v + 0.5 - mean) / (std * math.sqrt(2.0))))
        t[v] = min(int(p * 2**32), 2**32 - 1)
    return t.astype(np.uint32)


def gauss_u8_host(seed: int, start: int, count: int, thresholds: np.ndarray) -> np.ndarray:
    """Bytes [start, start + count) of the Gaussian-uint8 generator:
    value = #{v : u >= T[v]} for the top 32 bits u of each hash."""
    idx = np.arange(start, start + count, dtype=np.uint64)
    u = (hash_u64(seed, idx) >> np.uint64(32)).astype(np.uint32)
    return np.searchsorted(thresholds, u, side="right").astype(np.uint8)


def c2_chan_freqs() -> np.ndarray:
    return orc.chan_freqs(C2_NCHANS, C2_FCH1, C2_FOFF)


def c2_delays(dms) -> np.ndarray:
    """Config-2 delay table (ndm x nchans, int32) at the top-of-band reference."""
    return np.atleast_2d(orc.dmdelays(c2_chan_freqs(), dms, C2_TSAMP, C2_FCH1)).astype(np.int32)


def dm_grid(dm: float, dmsteps: int) -> np.ndarray:
    """FilterbankBlock.dmt_transform's trials (block.py:337): dm + linspace(-dm, dm)."""
    return dm + np.linspace(-dm, dm, dmsteps)


def c2_pulse_rows() -> list[np.ndarray]:
    """Per pulse, the first row of the pulse window in each channel."""
    out = []
    for dm, t in C2_PULSES:
        d = np.atleast_1d(orc.dmdelays(c2_chan_freqs(), dm, C2_TSAMP, C2_FCH1))
        out.append(d.astype(np.int64) + t - C2_PULSE_WIDTH // 2)
    return out


def c2_filterbank_host(start_row: int, nrows: int) -> np.ndarray:
    """Rows [start_row, start_row + nrows) of the config-2 input: uniform 2-bit
    samples plus the three pulses (+1 level, saturating at 3), packed
    big-endian, shape (nrows, nchans / 4)."""
    rb = C2_NCHANS * C2_NBITS // 8
    raw = uniform_bytes_host(C2_SEED, start_row * rb, nrows * rb).reshape(nrows, rb)
    vals = np.empty((nrows, C2_NCHANS), dtype=np.uint8)
    for k in range(4):
        vals[:, k::4] = (raw >> (6 - 2 * k)) & 3
    for p in c2_pulse_rows():
        for c in range(C2_NCHANS):
            lo = max(p[c], start_row)
            hi = min(p[c] + C2_PULSE_WIDTH, start_row + nrows)
            if lo < hi:
                sl = vals[lo - start_row:hi - start_row, c]
                vals[lo - start_row:hi - start_row, c] = np.minimum(sl + 1, 3)
    out = np.zeros((nrows, rb), dtype=np.uint8)
    for k in range(4):
        out |= vals[:, k::4] << (6 - 2 * k)
    return out
