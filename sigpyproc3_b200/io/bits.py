"""Sample bit layouts (io/bits.py:127-245 of the reference) and GPU unpack (R4)."""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .. import _lib

NBITS_DTYPE = {1: np.uint8, 2: np.uint8, 4: np.uint8, 8: np.uint8, 32: np.float32}
# 1-bit data is little-endian, 2- and 4-bit big-endian (bits.py:175-182)
DEFAULT_BITORDER = {1: "little", 2: "big", 4: "big"}


@dataclass(frozen=True)
class BitsInfo:
    nbits: int

    def __post_init__(self):
        if self.nbits not in NBITS_DTYPE:
            raise ValueError(f"nbits {self.nbits} not in {sorted(NBITS_DTYPE)}")

    @property
    def dtype(self) -> np.dtype:
        return np.dtype(NBITS_DTYPE[self.nbits])

    @property
    def itemsize(self) -> int:
        return self.dtype.itemsize

    @property
    def unpack(self) -> bool:
        return self.nbits in (1, 2, 4)

    @property
    def bitfact(self) -> int:
        return 8 // self.nbits if self.unpack else 1

    @property
    def bitorder(self) -> str:
        return DEFAULT_BITORDER.get(self.nbits, "invalid")


def bitorder_code(bitorder: str) -> int:
    if bitorder in ("big", "b"):
        return _lib.BITORDER_BIG
    if bitorder in ("little", "l"):
        return _lib.BITORDER_LITTLE
    raise ValueError(f"bitorder must be 'big' or 'little', got {bitorder!r}")


def unpack(packed, nbits: int, bitorder: str = "big", out=None, stream=None):
    """Unpack 1/2/4-bit samples to one uint8 per sample on the GPU.

    ``packed`` is a CUDA uint8 tensor (or a host array, which is copied to the
    current device); returns a CUDA uint8 tensor of ``packed.numel()*8//nbits``.
    """
    import torch

    if nbits not in (1, 2, 4):
        raise ValueError(f"unpack: nbits must be 1, 2 or 4 (got {nbits})")
    if not torch.is_tensor(packed):
        packed = torch.from_numpy(np.ascontiguousarray(packed, dtype=np.uint8)).cuda()
    packed = packed.contiguous()
    n = packed.numel()
    if out is None:
        out = torch.empty(n * 8 // nbits, dtype=torch.uint8, device=packed.device)
    st = stream if stream is not None else torch.cuda.current_stream(packed.device)
    _lib.call("spp_unpack", packed.data_ptr(), n, nbits, bitorder_code(bitorder), out.data_ptr(),
              st.cuda_stream)
    return out


def pack_host(vals: np.ndarray, nbits: int, bitorder: str = "big") -> np.ndarray:
    """Pack uint8 samples (one per byte) into nbits-wide fields, ``8 // nbits``
    per byte in the reference's layout (kernels.pack{1,2,4}_8_{big,little},
    core/kernels.py:72-173): sample k of a byte sits in the high bits first
    for big order, in the low bits first for little order.  Host-side: it
    serves file writing, not the GPU path."""
    if nbits not in (1, 2, 4):
        raise ValueError(f"pack: nbits must be 1, 2 or 4 (got {nbits})")
    per = 8 // nbits
    v = np.ascontiguousarray(vals, dtype=np.uint8).reshape(-1, per)
    out = np.zeros(v.shape[0], dtype=np.uint8)
    for k in range(per):
        sh = (8 - (k + 1) * nbits) if bitorder == "big" else k * nbits
        out |= (v[:, k] << np.uint8(sh)).astype(np.uint8)
    return out
