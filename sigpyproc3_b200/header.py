"""Observation metadata (R6/R11): the subset of the reference ``Header``
(src/sigpyproc/header.py) that the dedispersion path reads and writes."""

from __future__ import annotations

import dataclasses
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import params
from .io import sigproc
from .io.bits import BitsInfo


@dataclass(frozen=True)
class Header:
    filename: str = ""
    data_type: str = "filterbank"
    nchans: int = 1
    foff: float = -1.0
    fch1: float = 1400.0
    nbits: int = 8
    tsamp: float = 64e-6
    tstart: float = 60000.0
    nsamples: int = 0
    nifs: int = 1
    source: str = "synthetic"
    telescope_id: int = 0
    machine_id: int = 0
    dm: float = 0.0
    refdm: float = 0.0
    ibeam: int = 0
    nbeams: int = 1
    stream: sigproc.StreamInfo | None = field(default=None, compare=False, repr=False)

    # ---- frequency helpers (header.py:195-259) ----
    @property
    def bandwidth(self) -> float:
        return abs(self.foff) * self.nchans

    @property
    def ftop(self) -> float:
        return self.fch1 - 0.5 * self.foff

    @property
    def fbottom(self) -> float:
        return self.ftop + self.foff * self.nchans

    @property
    def fcenter(self) -> float:
        return self.ftop + 0.5 * self.foff * self.nchans

    @property
    def chan_freqs(self) -> np.ndarray:
        return np.arange(self.nchans, dtype=np.float32) * self.foff + self.fch1

    @property
    def fmax(self) -> float:
        return self.chan_freqs.max()

    @property
    def fmin(self) -> float:
        return self.chan_freqs.min()

    @property
    def bitsinfo(self) -> BitsInfo:
        return BitsInfo(self.nbits)

    @property
    def dtype(self) -> np.dtype:
        return self.bitsinfo.dtype

    @property
    def basename(self) -> str:
        return Path(self.filename).stem if self.filename else "synthetic"

    @property
    def tobs(self) -> float:
        return self.tsamp * self.nsamples

    # ---- delays (header.py:344-388) ----
    def ref_frequency(self, ref_freq: str | float = "fch1") -> float:
        if isinstance(ref_freq, str):
            if ref_freq not in {"fmax", "fmin", "fcenter", "fch1"}:
                raise ValueError(f"reference frequency {ref_freq} not defined")
            return float(getattr(self, ref_freq))
        if isinstance(ref_freq, (int, float)) and not isinstance(ref_freq, bool):
            return float(ref_freq)
        raise TypeError("ref_freq must be a string or a number")

    def get_dmdelays(self, dm, ref_freq: str | float = "fch1", *, in_samples: bool = True):
        return params.compute_dmdelays(self.chan_freqs, dm, self.tsamp,
                                       self.ref_frequency(ref_freq), in_samples=in_samples)

    # ---- derived headers (header.py:420-458) ----
    def new_header(self, update_dict: dict | None = None) -> "Header":
        names = {f.name for f in dataclasses.fields(self)}
        upd = {k: v for k, v in (update_dict or {}).items() if k in names}
        return dataclasses.replace(self, **upd)

    def dedispersed_header(self, dm: float) -> "Header":
        return self.new_header({"dm": dm, "nchans": 1, "data_type": "time series", "nbits": 32})

    def mjd_after_nsamps(self, nsamps: int) -> float:
        return self.tstart + nsamps * self.tsamp / 86400.0

    # ---- sigproc I/O ----
    @classmethod
    def from_sigproc(cls, filenames) -> "Header":
        hdr, info = sigproc.read_headers(filenames)
        return cls(
            filename=info.files[0], nchans=int(hdr["nchans"]), foff=float(hdr.get("foff", -1.0)),
            fch1=float(hdr.get("fch1", 1400.0)), nbits=int(hdr["nbits"]),
            tsamp=float(hdr.get("tsamp", 64e-6)), tstart=float(hdr.get("tstart", 0.0)),
            nsamples=int(hdr["nsamples"]), nifs=int(hdr.get("nifs", 1)),
            source=str(hdr.get("source_name", "")), telescope_id=int(hdr.get("telescope_id", 0)),
            machine_id=int(hdr.get("machine_id", 0)), refdm=float(hdr.get("refdm", 0.0)),
            ibeam=int(hdr.get("ibeam", 0)), nbeams=int(hdr.get("nbeams", 1)), stream=info,
        )

    def to_sigproc_dict(self) -> dict:
        return {
            "telescope_id": self.telescope_id, "machine_id": self.machine_id,
            "data_type": 2 if self.data_type == "time series" else 1,
            "source_name": self.source, "tstart": self.tstart, "tsamp": self.tsamp,
            "nbits": self.nbits, "fch1": self.fch1, "foff": self.foff, "nchans": self.nchans,
            "nifs": self.nifs, "refdm": self.refdm, "ibeam": self.ibeam, "nbeams": self.nbeams,
        }

    def write_sigproc(self, path, data) -> None:
        sigproc.write_filterbank(path, self.to_sigproc_dict(), data)

    def prep_outfile(self, filename, *, updates: dict | None = None,
                     nbits: int | None = None) -> sigproc.SigprocWriter:
        """A sigproc file with this header (plus ``updates``) written, ready for
        data blocks (header.py:575-619)."""
        nbits = self.nbits if nbits is None else int(nbits)
        upd = dict(updates or {})
        upd["nbits"] = nbits
        return sigproc.SigprocWriter(filename, self.new_header(upd).to_sigproc_dict(), nbits)
