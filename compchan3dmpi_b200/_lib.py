"""ctypes binding of ``libchanrhs.so`` (the C ABI in include/chanrhs.h).

The shared library is built in-tree by ``compchan3dmpi_b200.build``.  There
is no fallback: if the library is missing, loading fails with an error that
says how to build it.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIBDIR = HERE / "lib"
LIBNAME = "libchanrhs.so"

CHAN_OK, CHAN_BLOWUP, CHAN_NONFINITE = 0, 1, 2
CHAN_EINVAL, CHAN_ENOMEM, CHAN_ECUDA, CHAN_ESTATE, CHAN_EIO = -1, -2, -3, -4, -5
CHAN_MIXED = 1

_D = ctypes.POINTER(ctypes.c_double)
_I32 = ctypes.POINTER(ctypes.c_int32)
_I64 = ctypes.POINTER(ctypes.c_int64)
_F = ctypes.POINTER(ctypes.c_float)


class ChanWallBCC(ctypes.Structure):
    """Mirror of ``struct chan_wall_bc``."""
    _fields_ = [
        ("velocity", ctypes.c_int32),
        ("thermal", ctypes.c_int32),
        ("Tw", ctypes.c_double),
        ("dTdz", ctypes.c_double),
        ("slip_grad", ctypes.c_double),
        ("wave", ctypes.c_double * 4),
        ("mask", ctypes.POINTER(ctypes.c_uint8)),
        ("uv", ctypes.POINTER(ctypes.c_double)),
        ("x1", ctypes.POINTER(ctypes.c_double)),
    ]


class ChanParamsC(ctypes.Structure):
    """Mirror of ``struct chan_params``."""
    _fields_ = [
        ("nP", ctypes.c_int32 * 3),
        ("istat", ctypes.c_int32),
        ("rk_scheme", ctypes.c_int32),
        ("forcing", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("flags", ctypes.c_int32),
        ("Re", ctypes.c_double),
        ("Mac", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("Pr", ctypes.c_double),
        ("gama", ctypes.c_double),
        ("Pe", ctypes.c_double * 3),
        ("Lx", ctypes.c_double),
        ("Ly", ctypes.c_double),
        ("Tw", ctypes.c_double * 2),
    ]


# every symbol declared in include/chanrhs.h: (name, restype, argtypes)
SIGNATURES = [
    ("chan_init", ctypes.c_int, [ctypes.POINTER(ChanParamsC), _D, _D, _D, ctypes.POINTER(ctypes.c_void_p)]),
    ("chan_upload", ctypes.c_int, [ctypes.c_void_p, _D, ctypes.c_int64, ctypes.c_double]),
    ("chan_stage", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("chan_step", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("chan_step_async", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("chan_check", ctypes.c_int, [ctypes.c_void_p]),
    ("chan_tau_wall", ctypes.c_int, [ctypes.c_void_p]),
    ("chan_avg_spatial", ctypes.c_int, [ctypes.c_void_p]),
    ("chan_stats", ctypes.c_int, [ctypes.c_void_p, _D, _D, _D, _D]),
    ("chan_set_forcing", ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, _D]),
    ("chan_download", ctypes.c_int, [ctypes.c_void_p, _D]),
    ("chan_status", ctypes.c_int, [ctypes.c_void_p, _I32, _I64, _D]),
    ("chan_sync", ctypes.c_int, [ctypes.c_void_p]),
    ("chan_profile", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("chan_profile_read", ctypes.c_int, [ctypes.c_void_p, _D, _I64]),
    ("chan_selftest_pow07", ctypes.c_int, [_D, _D, _D, ctypes.c_int64, ctypes.c_int32]),
    ("chan_stream", ctypes.c_void_p, [ctypes.c_void_p]),
    ("chan_device_bytes", ctypes.c_int64, [ctypes.c_void_p]),
    ("chan_last_error", ctypes.c_char_p, [ctypes.c_void_p]),
    ("chan_version", ctypes.c_char_p, []),
    ("chan_time_avg_start", ctypes.c_int, [ctypes.c_void_p]),
    ("chan_time_avg", ctypes.c_int, [ctypes.c_void_p, _D, _D, _D, _D, _I64, _D, _D]),
    ("chan_set_wall_bc", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ChanWallBCC)]),
    ("chan_diag_enable", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32), ctypes.c_int32, ctypes.c_int32,
                                        _D, ctypes.c_double, ctypes.c_int32]),
    ("chan_diag_read", ctypes.c_int, [ctypes.c_void_p, _D, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
                                      ctypes.POINTER(ctypes.c_int64)]),
    ("chan_fluctuation_q", ctypes.c_int, [ctypes.c_void_p, _D, _D, _D, _D, _D, _D]),
    ("chan_q_criterion", ctypes.c_int, [ctypes.POINTER(ctypes.c_int32), _D, _D, _D, _D, _D, _D, _D,
                                        ctypes.c_int32]),
    ("chan_debug_canaries", ctypes.c_int, [ctypes.c_void_p, _I64]),
    ("chan_checkpoint_write", ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p]),
    ("chan_checkpoint_read", ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p]),
    ("chan_deck_read", ctypes.c_int, [ctypes.c_char_p, _I32, _D, _D, _D, _D, _D, _I64, ctypes.c_int32]),
    ("chan_deck_write", ctypes.c_int, [ctypes.c_char_p, _I32, _D, _D, _D, _D, ctypes.c_double, ctypes.c_int64,
                                       ctypes.c_int32]),
    ("chan_io_last_error", ctypes.c_char_p, []),
    ("chan_avg_spatial_noalloc", ctypes.c_int, [_D, _I32, _D, _D, _D, ctypes.c_int32]),
    ("chan_free", None, [ctypes.c_void_p]),
    ("chan_set_buoyancy", ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]),
    ("chan_set_launch", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32]),
    ("chan_get_launch", ctypes.c_int, [ctypes.c_void_p, _I32, _I32, _I32]),
    ("chan_ensemble_create", ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int32,
                                            ctypes.POINTER(ctypes.c_void_p)]),
    ("chan_ensemble_size", ctypes.c_int, [ctypes.c_void_p]),
    ("chan_ensemble_block", ctypes.c_int, [ctypes.c_void_p]),
    ("chan_ensemble_step", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, _I32]),
    ("chan_ensemble_tune", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, _D]),
    ("chan_ensemble_counters", ctypes.c_int, [ctypes.c_void_p, _I64, _I64, _D]),
    ("chan_ensemble_set_mode", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    ("chan_ensemble_get_mode", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32),
                                              ctypes.POINTER(ctypes.c_char_p)]),
    ("chan_ensemble_last_error", ctypes.c_char_p, [ctypes.c_void_p]),
    ("chan_ensemble_free", None, [ctypes.c_void_p]),
    ("chan_selftest_umma", ctypes.c_int, [ctypes.POINTER(ctypes.c_uint16), ctypes.POINTER(ctypes.c_uint16),
                                          ctypes.POINTER(ctypes.c_float), ctypes.c_int32, ctypes.c_int32,
                                          ctypes.c_int32]),
    ("chan_closure_create", ctypes.c_int, [ctypes.c_int32, ctypes.c_int64, ctypes.POINTER(ctypes.c_void_p)]),
    ("chan_closure_sample", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                           ctypes.c_int32, ctypes.c_int32, _I64]),
    ("chan_closure_add_data", ctypes.c_int, [ctypes.c_void_p, _F, _F, ctypes.c_int64]),
    ("chan_closure_count", ctypes.c_int, [ctypes.c_void_p, _I64]),
    ("chan_closure_get_data", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, _F, _F]),
    ("chan_closure_fit_normalization", ctypes.c_int, [ctypes.c_void_p, _F]),
    ("chan_closure_set_normalization", ctypes.c_int, [ctypes.c_void_p, _F]),
    ("chan_closure_get_normalization", ctypes.c_int, [ctypes.c_void_p, _F]),
    ("chan_closure_nparams", ctypes.c_int, []),
    ("chan_closure_init", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    ("chan_closure_set_params", ctypes.c_int, [ctypes.c_void_p, _F]),
    ("chan_closure_get_params", ctypes.c_int, [ctypes.c_void_p, _F]),
    ("chan_closure_train", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                          ctypes.c_uint64, _D]),
    ("chan_closure_grad", ctypes.c_int, [ctypes.c_void_p, _F, _F, ctypes.c_int64, _F, _D]),
    ("chan_closure_infer", ctypes.c_int, [ctypes.c_void_p, _F, ctypes.c_int64, _F]),
    ("chan_closure_last_error", ctypes.c_char_p, [ctypes.c_void_p]),
    ("chan_closure_free", None, [ctypes.c_void_p]),
    ("chan_set_closure", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32]),
    ("chan_closure_flag", ctypes.c_int, [ctypes.c_void_p, _I32, ctypes.c_int32]),
]

CHAN_TILE_32x8 = 0
CHAN_TILE_32x4 = 1
CHAN_TILE_16x16 = 2
CHAN_TILE_32x16 = 3
CHAN_NTILES = 4
CHAN_ENSEMBLE_GRAPH = 0
CHAN_ENSEMBLE_PERSISTENT = 1
CHAN_ENSEMBLE_PERSISTENT_STALL_TEST = 2

_lib = None


def lib_path() -> Path:
    return Path(os.environ.get("CHANRHS_LIB", str(LIBDIR / LIBNAME)))


def load():
    """Load the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    p = lib_path()
    if not p.exists():
        raise RuntimeError(f"{p} not found: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
                           "or `python -m compchan3dmpi_b200.build`")
    L = ctypes.CDLL(str(p))
    for name, res, args in SIGNATURES:
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def dptr(a):
    return a.ctypes.data_as(_D)
