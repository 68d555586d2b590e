"""Dispersion constants and the per-channel delay table (R6).

The delays must equal the reference's bit for bit, so they are computed
exactly as ``params.compute_dmdelays`` (src/sigpyproc/params.py:57-62) does:
float32 NumPy arithmetic in the same expression order (NumPy 2 treats the
Python-float constants as "weak" scalars, so every step stays float32),
round-half-even, int32.  A float64 evaluation or a hand-written
``1/(f*f)`` both differ in some channels at the benchmark geometries.
"""

from __future__ import annotations

import numpy as np

DM_CONSTANT_LK = 4.148808e3  # Lorimer & Kramer, Handbook of Pulsar Astronomy


def compute_dmdelays(freqs, dm, tsamp: float, ref_freq: float, *, in_samples: bool = True):
    """ISM dispersion delays of each channel for one or more DMs.

    Returns int32 samples (``in_samples``) or float32 seconds, shaped
    ``(nchans,)`` for a scalar DM and ``(ndm, nchans)`` otherwise.
    """
    freqs = np.atleast_1d(freqs).astype(np.float32)
    dm = np.atleast_1d(dm)[:, np.newaxis].astype(np.float32)
    delays = dm * DM_CONSTANT_LK * ((freqs**-2) - (ref_freq**-2))
    if in_samples:
        delays = (delays / tsamp).round().astype(np.int32)
    return delays.squeeze()
