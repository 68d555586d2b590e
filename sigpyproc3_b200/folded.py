"""Folded data cube (foldedcube.py:121-205 of the reference, the container
part): (subintegrations, subbands, phase bins) float32 with its header and the
period, DM and acceleration it was folded with."""

from __future__ import annotations

import numpy as np

from .header import Header


class FoldedData:
    def __init__(self, data: np.ndarray, header: Header, period: float, dm: float,
                 accel: float = 0.0):
        data = np.asarray(data, dtype=np.float32)
        if data.ndim != 3:
            raise ValueError(f"folded data must be 3-D (nints, nbands, nbins), got {data.shape}")
        self.data = data
        self.header = header
        self.period = period
        self.dm = dm
        self.accel = accel

    @property
    def nints(self) -> int:
        return self.data.shape[0]

    @property
    def nbands(self) -> int:
        return self.data.shape[1]

    @property
    def nbins(self) -> int:
        return self.data.shape[2]

    def get_profile(self) -> np.ndarray:
        """Profile summed over subintegrations and subbands."""
        return self.data.sum(axis=(0, 1))
