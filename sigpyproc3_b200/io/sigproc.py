"""Sigproc binary header parsing and encoding (next-row N1 of the path).

Format (as read by io/sigproc.py:280-524, :655-680 of the reference): a
sequence of length-prefixed strings (uint32 little-endian length, ASCII)
between ``HEADER_START`` and ``HEADER_END``; each key is followed by its
value, encoded as uint32, float64, int8 or another length-prefixed string
depending on the key.  ``nsamples`` is derived from the data length as
``(8 * datalen) // nbits // nchans`` (and the smaller of that and a declared
``nsamples`` key).
"""

from __future__ import annotations

import struct
from dataclasses import dataclass, field
from pathlib import Path

_U32 = struct.Struct("<I")
_F64 = struct.Struct("<d")
_I8 = struct.Struct("b")

# key -> value codec ("u" uint32, "d" float64, "b" int8, "s" string)
KEY_TYPES: dict[str, str] = {
    "telescope_id": "u", "machine_id": "u", "data_type": "u", "rawdatafile": "s",
    "source_name": "s", "barycentric": "u", "pulsarcentric": "u", "az_start": "d",
    "za_start": "d", "src_raj": "d", "src_dej": "d", "tstart": "d", "tsamp": "d",
    "nbits": "u", "nsamples": "u", "fch1": "d", "foff": "d", "nchans": "u", "nifs": "u",
    "refdm": "d", "period": "d", "signed": "b", "ibeam": "u", "nbeams": "u",
}


def _read_str(fp) -> str:
    raw = fp.read(4)
    if len(raw) != 4:
        raise ValueError("truncated string length")
    (n,) = _U32.unpack(raw)
    if n > 4096:
        raise ValueError(f"implausible string length {n}")
    data = fp.read(n)
    if len(data) != n:
        raise ValueError("truncated string")
    return data.decode("ascii")


def _enc_str(s: str) -> bytes:
    b = s.encode("ascii")
    return _U32.pack(len(b)) + b


def read_header(path: str | Path) -> dict:
    """Parse one sigproc file; returns the keys plus hdrlen, datalen, nsamples."""
    path = Path(path)
    if not path.is_file():
        raise FileNotFoundError(path)
    hdr: dict = {}
    with path.open("rb") as fp:
        try:
            first = _read_str(fp)
        except (ValueError, UnicodeDecodeError) as exc:
            raise OSError(f"{path}: Header is not in sigproc format... Is file empty?.") from exc
        if first != "HEADER_START":
            raise OSError(f"{path}: Header is not in sigproc format.")
        while True:
            try:
                key = _read_str(fp)
            except (ValueError, UnicodeDecodeError) as exc:
                raise OSError(f"{path}: Header truncated while reading key.") from exc
            if key == "HEADER_END":
                break
            kind = KEY_TYPES.get(key)
            if kind is None:
                raise OSError(f"{path}: unknown header key {key!r}")
            try:
                if kind == "s":
                    hdr[key] = _read_str(fp)
                else:
                    st = {"u": _U32, "d": _F64, "b": _I8}[kind]
                    raw = fp.read(st.size)
                    if len(raw) != st.size:
                        raise ValueError
                    (hdr[key],) = st.unpack(raw)
            except (ValueError, UnicodeDecodeError) as exc:
                raise OSError(f"{path}: Header truncated while reading value for {key!r}.") from exc
        hdrlen = fp.tell()
        fp.seek(0, 2)
        filelen = fp.tell()
    if "nbits" not in hdr or "nchans" not in hdr:
        raise ValueError(f"{path}: missing nbits/nchans")
    datalen = filelen - hdrlen
    if datalen < 0:
        raise OSError(f"{path}: file shorter than its header")
    nsamp = (8 * datalen) // int(hdr["nbits"]) // int(hdr["nchans"])
    if "nsamples" in hdr:
        nsamp = min(nsamp, int(hdr["nsamples"]))
    hdr.update(hdrlen=hdrlen, filelen=filelen, datalen=datalen, nsamples=nsamp,
               filename=path.as_posix())
    return hdr


def encode_header(hdr: dict) -> bytes:
    """Encode the sigproc keys present in ``hdr`` (nsamples omitted)."""
    out = _enc_str("HEADER_START")
    for key, kind in KEY_TYPES.items():
        if key == "nsamples" or key not in hdr or hdr[key] is None:
            continue
        out += _enc_str(key)
        v = hdr[key]
        if kind == "s":
            out += _enc_str(str(v))
        elif kind == "u":
            out += _U32.pack(int(v))
        elif kind == "d":
            out += _F64.pack(float(v))
        else:
            out += _I8.pack(int(v))
    return out + _enc_str("HEADER_END")


@dataclass
class StreamInfo:
    """Data segments of a (possibly multi-file) observation."""

    files: list[str] = field(default_factory=list)
    hdrlens: list[int] = field(default_factory=list)
    datalens: list[int] = field(default_factory=list)

    @property
    def total(self) -> int:
        return sum(self.datalens)


def read_headers(paths) -> tuple[dict, StreamInfo]:
    """Parse a sequence of contiguous files; keys must agree (tstart excepted)."""
    if isinstance(paths, (str, Path)):
        paths = [paths]
    hdrs = [read_header(p) for p in paths]
    base = dict(hdrs[0])
    for h in hdrs[1:]:
        for k in KEY_TYPES:
            if k in ("tstart", "rawdatafile", "nsamples"):
                continue
            if base.get(k) != h.get(k):
                raise ValueError(f"Header key {k} mismatch in {h['filename']}")
    info = StreamInfo([h["filename"] for h in hdrs], [h["hdrlen"] for h in hdrs],
                      [h["datalen"] for h in hdrs])
    base["nsamples"] = sum(h["nsamples"] for h in hdrs)
    return base, info


def write_filterbank(path: str | Path, hdr: dict, data) -> None:
    """Write a sigproc file: header keys from ``hdr`` then the raw bytes of ``data``."""
    import numpy as np

    with Path(path).open("wb") as fp:
        fp.write(encode_header(hdr))
        fp.write(np.ascontiguousarray(data).tobytes())


class SigprocWriter:
    """Incremental sigproc writer: the header first, then data blocks
    appended in order (the role of the reference's FileWriter, io/fileio.py:
    346-412, without its optional rescaling).  Samples of nbits < 8 arrive as
    one uint8 per sample and are packed in the reference's bit order."""

    def __init__(self, path: str | Path, hdr: dict, nbits: int):
        self.path = Path(path)
        self.nbits = int(nbits)
        self._fp = self.path.open("wb")
        self._fp.write(encode_header(hdr))

    def cwrite(self, arr) -> None:
        import numpy as np

        from .bits import DEFAULT_BITORDER, pack_host

        a = np.ascontiguousarray(arr)
        if self.nbits in (1, 2, 4):
            a = pack_host(a, self.nbits, DEFAULT_BITORDER[self.nbits])
        self._fp.write(a.tobytes())

    def close(self) -> None:
        self._fp.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
