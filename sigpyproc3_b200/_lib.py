"""ctypes binding of libsppgpu.so -- the only route from Python to the GPU kernels.

The library is loaded once; a missing or unloadable library raises
ImportError (there is no CPU fallback).  Status codes from the C ABI
(include/sppgpu.h) become Python exceptions carrying spp_last_error_string().
"""

from __future__ import annotations

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libsppgpu.so"

SPP_OK = 0
SPP_ERR_ARG = -1
SPP_ERR_SIZE = -2
SPP_ERR_ALIGN = -3
SPP_ERR_CUDA = -4
SPP_ERR_TIMEOUT = -5
SPP_ERR_UNSUPPORTED = -6
SPP_ERR_DELAY = -7
SPP_ERR_DEVICE = -8

BITORDER_BIG = 0
BITORDER_LITTLE = 1
OUT_F32 = 0
OUT_I32 = 1
OUT_U16 = 2
MODE_DEDISPERSE = 0
MODE_ROLL = 1
ACC_KAHAN32 = 0
ACC_F64 = 1

_i64 = ctypes.c_int64
_i32 = ctypes.c_int32
_int = ctypes.c_int
_p = ctypes.c_void_p

# name -> (argtypes, restype); must match include/sppgpu.h
SIGNATURES: dict[str, tuple[list, object]] = {
    "spp_last_error_string": ([], ctypes.c_char_p),
    "spp_version": ([], _int),
    "spp_status_read": ([_p, _p, _p], _int),
    "spp_status_clear": ([_p, _p], _int),
    "spp_host_register": ([_p, _i64], _int),
    "spp_host_unregister": ([_p], _int),
    "spp_unpack": ([_p, _i64, _int, _int, _p, _p], _int),
    "spp_dedisperse_workspace_bytes": ([_int, _i64, _i64, _i32, _i32], _i64),
    "spp_dedisperse": ([_p, _int, _int, _i64, _i64, _p, _i32, _i32, _p, _i64, _i64, _int, _p,
                        _i64, _p], _int),
    "spp_dedisperse_hd": ([_p, _int, _i64, _i64, _p, _p, _i64, _i64, _p], _int),
    "spp_fold": ([_p, _int, _i64, _i64, _p, _i32, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                  _i64, _i32, _i32, _i32, _i64, _p, _p, _p, _i64, _p], _int),
    "spp_fold_exact": ([_p, _i64, _i64, _p, _i32, ctypes.c_float, ctypes.c_float,
                        ctypes.c_float, _i64, _i32, _i32, _i32, _i64, _p, _p, _p, _i64, _p],
                       _int),
    "spp_dedisperse_noalloc_max_bytes": ([], _i64),
    "spp_dedisperse_noalloc": ([_p, _int, _int, _i64, _i64, _p, _i32, _i32, _p, _i64, _i64, _int,
                                _p], _int),
    "spp_dedisperse_noalloc_status_read": ([_p, _p], _int),
    "spp_dmt_plan_create": ([ctypes.POINTER(_p), _int, _int, _i64, _i64, _i64, _p, _int, _int,
                             _int], _int),
    "spp_dmt_plan_destroy": ([_p], _int),
    "spp_dmt_plan_nvalid": ([_p, _i64], _i64),
    "spp_dmt_plan_workspace_bytes": ([_p, _i64], _i64),
    "spp_dmt_plan_describe": ([_p, _p], _int),
    "spp_dmt_plan_num_variants": ([_p], _int),
    "spp_dmt_plan_set_variant": ([_p, _int], _int),
    "spp_dmt_plan_timing": ([_p, _int], _int),
    "spp_dmt_plan_timing_read": ([_p, _p, _p, _p], _int),
    "spp_dmt_execute": ([_p, _p, _i64, _p, _i64, _i64, _p, _i64, _p], _int),
    "spp_dmt_plan_zero_dm_workspace_bytes": ([_p, _i64], _i64),
    "spp_dmt_execute_zero_dm": ([_p, _p, _i64, _p, _p, _p, _i64, _i64, _p, _i64, _p], _int),
    "spp_dmt_execute_host": ([_p, _p, _i64, _p, _i64, _i64, _p, _i64], _int),
    "spp_dmt_host_workspace_bytes": ([_p, _i64], _i64),
    "spp_bandpass": ([_p, _int, _int, _i64, _i64, _p, _p], _int),
    "spp_collapse": ([_p, _int, _int, _i64, _i64, _p, _i64, _p], _int),
    "spp_zero_dm": ([_p, _p, _i64, _i64, _p, _p, _p], _int),
    "spp_zero_dm_u8": ([_p, _p, _i64, _i64, _p, _p, _p], _int),
    "spp_downsample_mean": ([_p, _i64, _i64, _i64, _int, _p, _i64, _p], _int),
    "spp_downsample_2d_mean": ([_p, _i64, _i64, _int, _int, _p, _p], _int),
    "spp_downsample_2d_mean_u8": ([_p, _i64, _i64, _int, _int, _p, _p], _int),
    "spp_boxcar_snr_workspace_bytes": ([_i64, _i64, _int, _int], _i64),
    "spp_boxcar_snr": ([_p, _int, _i64, _i64, _i64, _p, _int, _p, _int, _p, _p, _p, _i64, _p],
                       _int),
    "spp_boxcar_filter": ([_p, _i64, _int, _p, _p], _int),
    "spp_row_loc_scale": ([_p, _int, _i64, _i64, _i64, _int, _p, _p], _int),
    "spp_zscore": ([_p, _i64, _p, _p, _p], _int),
    "spp_matched_filter": ([_p, _i64, _i64, _p, _p, _p, _p, _int, _p, _p, _i64, _p], _int),
    "spp_boxcar_snr_robust_workspace_bytes": ([_i64, _i64, _int, _int], _i64),
    "spp_boxcar_snr_robust": ([_p, _int, _i64, _i64, _i64, _p, _int, _p, _int, _p, _p, _p, _i64,
                               _p], _int),
    "spp_subband": ([_p, _int, _int, _i64, _i64, _p, _i32, _p, _i64, _p, _p], _int),
    "spp_wl_num_variants": ([_int, _int], _int),
    "spp_wl_describe": ([_int, _int, _int, _p], _int),
    "spp_wl_slot_words": ([_int, _int, _int, _i32], _i32),
    "spp_wl_smem_bytes": ([_int, _int, _int, _i32], _i64),
    "spp_wl_launch": ([_int, _int, _int, _p, _i32, _i32, _p, _p, _i32, _p], _int),
    "spp_wl_default_ctas": ([_int, _int, _int, _i32], _i32),
    "spp_wl_planar_layout": ([_int, _int, _int, _i64, _i32, _i32, _i32, _p, _p, _p], _int),
    "spp_wl_corner_turn": ([_int, _int, _int, _p, _int, _i64, _i64, _i64, _p, _i64, _p], _int),
    "spp_planar_layout": ([_int, _i64, _i64, _i32, _i32, _i32, _p, _p], _int),
    "spp_corner_turn": ([_p, _int, _int, _i64, _i64, _i64, _p, _i64, _p], _int),
    "spp_selftest_wait_timeout": ([_p, ctypes.c_uint64, _p], _int),
    "spp_synth_uniform_bytes": ([_p, _i64, _i64, ctypes.c_uint64, _p], _int),
    "spp_synth_gauss_u8": ([_p, _i64, _i64, ctypes.c_uint64, _p, _p], _int),
    "spp_synth_gauss_f32": ([_p, _i64, _i64, ctypes.c_uint64, ctypes.c_float, ctypes.c_float, _p],
                            _int),
    "spp_synth_pulse_packed": ([_p, _i64, _i64, _int, _int, _p, _int, _p], _int),
}


class SppError(RuntimeError):
    """Error reported by libsppgpu."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[spp {code}] {msg}")
        self.code = code


_LIB: ctypes.CDLL | None = None


def load() -> ctypes.CDLL:
    """Load libsppgpu.so (raises ImportError if it is absent or broken)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python sigpyproc3_b200/_build.py` "
            "(there is no CPU fallback)"
        )
    try:
        lib = ctypes.CDLL(str(LIB_PATH))
    except OSError as exc:  # pragma: no cover - environment specific
        raise ImportError(f"cannot load {LIB_PATH}: {exc}") from exc
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _LIB = lib
    return lib


def last_error() -> str:
    msg = load().spp_last_error_string()
    return msg.decode() if msg else ""


def check(rc: int) -> None:
    """Raise the exception matching a non-zero status code."""
    if rc == SPP_OK:
        return
    msg = last_error()
    if rc in (SPP_ERR_ARG, SPP_ERR_SIZE, SPP_ERR_DELAY, SPP_ERR_ALIGN):
        raise ValueError(msg)
    if rc == SPP_ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    raise SppError(rc, msg)


def call(name: str, *args) -> int:
    lib = load()
    rc = getattr(lib, name)(*args)
    check(rc)
    return rc
