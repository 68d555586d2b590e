"""B200-native filterbank dedispersion with the sigpyproc API.

Host code is Python over PyTorch (device memory, streams); the compute runs in
hand-written sm_100a CUDA kernels in ``libsppgpu.so`` behind the C ABI
declared in ``include/sppgpu.h``.  Importing the package loads that library
and fails if it is missing -- there is no CPU fallback.
"""

from __future__ import annotations

from . import _lib

_lib.load()

from .block import DMTBlock, FilterbankBlock  # noqa: E402
from .dedisp import DMTPlan, dedisperse_block  # noqa: E402
from .header import Header  # noqa: E402
from .readers import ArrayFilterbank, Filterbank, FilReader  # noqa: E402
from .timeseries import TimeSeries  # noqa: E402

__version__ = "0.1.0"

__all__ = [
    "ArrayFilterbank", "DMTBlock", "DMTPlan", "FilReader", "Filterbank", "FilterbankBlock",
    "Header", "TimeSeries", "dedisperse_block",
]
