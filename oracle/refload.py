"""Loader for the reference implementation's numba kernels (fixture generation only).

Test infrastructure, not product code.  It is used by
``tests/golden/make_golden.py`` in a container where the reference source tree
is mounted, to run the reference's own code on seeded inputs and record golden
vectors.  Nothing on the GPU path imports it.

The reference package cannot be imported as a whole here (astropy, bidict,
bottleneck, rocket_fft are absent), so:

* ``src/sigpyproc/core/kernels.py`` is loaded by path as
  ``sigpyproc.core.kernels`` with stub parent packages and a stub
  ``rocket_fft`` module (kernels.py:11 imports it; only the lazily compiled
  FFT helpers use it);
* single functions that only need numpy at call time
  (``params.compute_dmdelays`` params.py:26-62, ``Header.chan_freqs``
  header.py:228-237, ``FilReader.read_plan`` readers.py:171-233) are extracted
  from their source files with :mod:`ast` and executed in a namespace that
  provides numpy and small stand-ins for the names they touch.
"""

from __future__ import annotations

import ast
import importlib.util
import os
import sys
import tempfile
import types
from pathlib import Path

# the reference source tree, named by the caller; unset means "not available"
_ROOT_ENV = os.environ.get("SPP_REFERENCE_ROOT", "")
REF_ROOT = Path(_ROOT_ENV)
SRC = REF_ROOT / "src" / "sigpyproc"
TEST_DATA = REF_ROOT / "tests" / "data"


def available() -> bool:
    return bool(_ROOT_ENV) and (SRC / "core" / "kernels.py").is_file()


def load_kernels():
    """Return the reference ``sigpyproc.core.kernels`` module (numba-compiled)."""
    if "sigpyproc.core.kernels" in sys.modules:
        return sys.modules["sigpyproc.core.kernels"]
    os.environ.setdefault(
        "NUMBA_CACHE_DIR", os.path.join(tempfile.gettempdir(), "spp_ref_numba_cache")
    )
    for name in ("sigpyproc", "sigpyproc.core"):
        if name not in sys.modules:
            mod = types.ModuleType(name)
            mod.__path__ = []  # mark as package
            sys.modules[name] = mod
    if "rocket_fft" not in sys.modules:
        sys.modules["rocket_fft"] = types.ModuleType("rocket_fft")
    spec = importlib.util.spec_from_file_location(
        "sigpyproc.core.kernels", SRC / "core" / "kernels.py"
    )
    mod = importlib.util.module_from_spec(spec)
    sys.modules["sigpyproc.core.kernels"] = mod  # must precede exec (numba cache)
    spec.loader.exec_module(mod)
    return mod


def _extract(path: Path, names: set[str], class_name: str | None = None) -> str:
    tree = ast.parse(path.read_text())
    body = tree.body
    if class_name is not None:
        cls = next(
            n for n in body if isinstance(n, ast.ClassDef) and n.name == class_name
        )
        body = cls.body
    picked = []
    for node in body:
        if isinstance(node, ast.FunctionDef) and node.name in names:
            node.decorator_list = []
            picked.append(node)
        elif isinstance(node, ast.Assign):
            tgt = [t.id for t in node.targets if isinstance(t, ast.Name)]
            if any(t in names for t in tgt):
                picked.append(node)
    mod = ast.Module(body=picked, type_ignores=[])
    return ast.unparse(mod)


def load_compute_dmdelays():
    """Reference ``params.compute_dmdelays`` (params.py:26-62), executed as-is."""
    import numpy as np

    src = _extract(SRC / "params.py", {"DM_CONSTANT_LK", "compute_dmdelays"})
    ns: dict = {"np": np, "ArrayLike": object, "NDArray": object, "annotations": None}
    exec(compile("from __future__ import annotations\n" + src, "params.py", "exec"), ns)
    return ns["compute_dmdelays"], ns["DM_CONSTANT_LK"]


def load_header_freq_helpers():
    """Reference ``Header`` frequency properties (header.py:195-259) as functions."""
    import numpy as np

    names = {"ftop", "fbottom", "fcenter", "chan_freqs", "fmax", "fmin"}
    src = _extract(SRC / "header.py", names, class_name="Header")
    ns: dict = {"np": np}
    exec(compile("from __future__ import annotations\n" + src, "header.py", "exec"), ns)
    return {n: ns[n] for n in names}


def load_read_plan():
    """Reference ``FilReader.read_plan`` (readers.py:171-233) as a plain function.

    Call it with a fake ``self`` providing ``header`` (nsamples, nchans),
    ``bitsinfo`` (unpack, dtype), ``samp_stride``, ``chan_stride`` and ``_file``
    (``seek``/``creadinto``).
    """
    src = _extract(SRC / "readers.py", {"read_plan"}, class_name="FilReader")

    def _alloc(allocator, nbytes):  # io/fileio.py:25-71 contract, minimal
        if nbytes <= 0:
            raise ValueError(f"Requested buffer size ({nbytes}) is invalid")
        return allocator(nbytes)

    class _Log:
        def debug(self, *a, **k):
            pass

    import numpy as np

    ns: dict = {
        "np": np,
        "inspect": types.SimpleNamespace(stack=lambda: None),
        "get_callerfunc": lambda stack: "ref",
        "allocate_buffer": _alloc,
        "track": lambda seq, description=None, disable=False: seq,
        "logger": _Log(),
    }
    exec(compile("from __future__ import annotations\n" + src, "readers.py", "exec"), ns)
    return ns["read_plan"]


def load_scale_mad():
    """Reference ``stats._scale_mad`` (core/stats.py:505-536), executed as-is."""
    import numpy as np

    src = _extract(SRC / "core" / "stats.py", {"_scale_mad"})
    ns: dict = {"np": np, "NDArray": object}
    exec(compile("from __future__ import annotations\n" + src, "stats.py", "exec"), ns)
    return ns["_scale_mad"]


def load_scale_iqr():
    """Reference ``stats._scale_iqr`` (core/stats.py:480-502), executed as-is."""
    import numpy as np

    src = _extract(SRC / "core" / "stats.py", {"_scale_iqr"})
    ns: dict = {"np": np, "NDArray": object}
    exec(compile("from __future__ import annotations\n" + src, "stats.py", "exec"), ns)
    return ns["_scale_iqr"]
