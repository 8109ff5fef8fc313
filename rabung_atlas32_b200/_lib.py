"""ctypes binding of librabung_census.so (include/rabung_census.h).

The library is built in-tree (rabung_atlas32_b200/build.py).  Loading fails
loudly when it is missing or no CUDA device is usable: there is no CPU
fallback in the product path.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

from .build import LIB

CZ_DENSE, CZ_SPARSE, CZ_AUTO, CZ_A4, CZ_VERIFY = 1, 2, 3, 4, 8
CZ_OK, CZ_EINVAL, CZ_ECUDA, CZ_EREFUSED, CZ_ELIMIT, CZ_EPENDING = 0, 1, 2, 3, 4, 5

u32, u64, i32 = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int32


class cz_profile(ctypes.Structure):
    _fields_ = [("p", u32), ("r", u32), ("M", u32), ("L", u32), ("witness", u32),
                ("status", u32), ("K", u64)]


class cz_profile64(ctypes.Structure):
    _fields_ = [("p", u64), ("r", u32), ("M", u32), ("L", u32), ("witness", u32),
                ("status", u32), ("reserved", u32), ("K", u64)]


class cz_config(ctypes.Structure):
    _fields_ = [("device", i32), ("sparse_min_p", u32), ("cover_n", u32), ("q_cap", u32 * 10),
                ("anchor_bits", u32), ("screen", u32), ("sparse_blocks", u32), ("use_graph", u32),
                ("cta_per_profile", u32), ("epoch_rows", u32), ("speculate", u32),
                ("spec_margin10", u32 * 10), ("plane_budget_mb", u32), ("dense_steps", u32),
                ("anchor_t", u32 * 10), ("reserved", u32 * 1)]


class cz_stats(ctypes.Structure):
    _fields_ = [("ms_setup", ctypes.c_float), ("ms_table", ctypes.c_float), ("ms_sparse", ctypes.c_float),
                ("ms_dense", ctypes.c_float), ("ms_a4", ctypes.c_float), ("ms_finalize", ctypes.c_float),
                ("ms_device", ctypes.c_float), ("ms_h2d", ctypes.c_float), ("ms_d2h", ctypes.c_float),
                ("n_primes", u32), ("n_dense", u32), ("n_sparse", u32), ("n_profiles", u32),
                ("n_fallback", u32), ("n_respec", u32), ("ms_respec", ctypes.c_float), ("waves", u32),
                ("kernels", u32), ("words", u64), ("completions", u64),
                ("tests", u64), ("h2d_bytes", u64), ("d2h_bytes", u64), ("staged_bytes", u64)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class cz_server_counters(ctypes.Structure):
    _fields_ = [("launches", u64), ("yields", u64), ("completed", u64), ("waiting", u64),
                ("respec_primes", u64), ("fallback_primes", u64), ("oversize_requests", u64),
                ("ms_drain", ctypes.c_double), ("ms_window", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


EXPORTS = ["cz_default_config", "cz_open", "cz_close", "cz_last_error", "cz_count_profiles",
           "cz_census", "cz_replay", "cz_a4", "cz_sieve", "cz_plane_bytes", "cz_mem_info", "cz_device_info",
           "cz_microbench", "cz_census_dense_noalloc", "cz_census_interval", "cz_server_open",
           "cz_server_close", "cz_submit", "cz_next_done", "cz_poll", "cz_server_info", "cz_server_stats",
           "cz_server_last_error",
           "cz_prime_count", "cz_open64", "cz_close64", "cz_last_error64", "cz_count_profiles64", "cz_census64",
           "baseline_init", "baseline_profile"]

_lib = None


def load(path: Path | str | None = None) -> ctypes.CDLL:
    """Load the shared library (raises OSError if it is not built)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else Path(os.environ.get("RABUNG_CENSUS_LIB", str(LIB)))
    if not p.exists():
        raise OSError(f"{p} is not built; run `python -m rabung_atlas32_b200.build`")
    L = ctypes.CDLL(str(p))
    H = ctypes.c_void_p
    L.cz_default_config.argtypes = [ctypes.POINTER(cz_config)]
    L.cz_default_config.restype = ctypes.c_int
    L.cz_open.argtypes = [ctypes.POINTER(cz_config), ctypes.POINTER(H)]
    L.cz_open.restype = ctypes.c_int
    L.cz_close.argtypes = [H]
    L.cz_close.restype = None
    L.cz_last_error.argtypes = [H]
    L.cz_last_error.restype = ctypes.c_char_p
    L.cz_count_profiles.argtypes = [ctypes.POINTER(u32), u32]
    L.cz_count_profiles.restype = u32
    L.cz_census.argtypes = [H, ctypes.POINTER(u32), u32, u32, ctypes.POINTER(cz_profile), u32,
                            ctypes.POINTER(u32), ctypes.POINTER(cz_stats)]
    L.cz_census.restype = ctypes.c_int
    L.cz_replay.argtypes = [H, ctypes.POINTER(cz_stats)]
    L.cz_replay.restype = ctypes.c_int
    L.cz_a4.argtypes = [H, ctypes.POINTER(u32), u32, ctypes.POINTER(u32)]
    L.cz_a4.restype = ctypes.c_int
    L.cz_plane_bytes.argtypes = [H, ctypes.POINTER(u32), u32, u32]
    L.cz_plane_bytes.restype = u64
    L.cz_device_info.argtypes = [H, ctypes.c_char_p, u32, ctypes.POINTER(u32)]
    L.cz_device_info.restype = ctypes.c_int
    L.cz_mem_info.argtypes = [H, ctypes.POINTER(u64), ctypes.POINTER(u64)]
    L.cz_mem_info.restype = ctypes.c_int
    L.cz_sieve.argtypes = [H, ctypes.POINTER(u32), ctypes.POINTER(u32), u32, ctypes.POINTER(u32),
                           ctypes.POINTER(u32)]
    L.cz_sieve.restype = ctypes.c_int
    L.cz_microbench.argtypes = [H, u32, ctypes.POINTER(ctypes.c_double)]
    L.cz_microbench.restype = ctypes.c_int
    L.cz_census_dense_noalloc.argtypes = [ctypes.POINTER(u32), u32, ctypes.POINTER(cz_profile), u32,
                                          ctypes.c_void_p]
    L.cz_census_dense_noalloc.restype = ctypes.c_int
    P32, P64 = ctypes.POINTER(u32), ctypes.POINTER(u64)
    L.cz_census_interval.argtypes = [H, u64, u64, u32, P32, u32, P32, ctypes.POINTER(cz_profile), u32, P32, P32,
                                     ctypes.POINTER(cz_stats)]
    L.cz_census_interval.restype = ctypes.c_int
    L.cz_server_open.argtypes = [ctypes.POINTER(cz_config), u32, u64, ctypes.POINTER(H)]
    L.cz_server_open.restype = ctypes.c_int
    L.cz_server_close.argtypes = [H]
    L.cz_server_close.restype = None
    L.cz_submit.argtypes = [H, u32, u32, P32, u32, P64]
    L.cz_submit.restype = ctypes.c_int
    L.cz_next_done.argtypes = [H, i32, P64]
    L.cz_next_done.restype = ctypes.c_int
    L.cz_poll.argtypes = [H, u64, i32, P32, u32, P32, ctypes.POINTER(cz_profile), u32, P32, P32]
    L.cz_poll.restype = ctypes.c_int
    L.cz_server_info.argtypes = [H, P64, P64, P64]
    L.cz_server_info.restype = ctypes.c_int
    L.cz_server_stats.argtypes = [H, ctypes.POINTER(cz_server_counters)]
    L.cz_server_stats.restype = ctypes.c_int
    L.cz_server_last_error.argtypes = [H]
    L.cz_server_last_error.restype = ctypes.c_char_p
    L.cz_open64.argtypes = [ctypes.POINTER(cz_config), ctypes.POINTER(H)]
    L.cz_open64.restype = ctypes.c_int
    L.cz_close64.argtypes = [H]
    L.cz_close64.restype = None
    L.cz_last_error64.argtypes = [H]
    L.cz_last_error64.restype = ctypes.c_char_p
    L.cz_count_profiles64.argtypes = [ctypes.POINTER(u64), u32]
    L.cz_count_profiles64.restype = u32
    L.cz_census64.argtypes = [H, ctypes.POINTER(u64), u32, u32, ctypes.POINTER(cz_profile64), u32,
                              ctypes.POINTER(u32), ctypes.POINTER(cz_stats)]
    L.cz_census64.restype = ctypes.c_int
    L.cz_prime_count.argtypes = [u64, u64]
    L.cz_prime_count.restype = u64
    L.baseline_init.argtypes = [ctypes.c_uint]
    L.baseline_init.restype = None
    L.baseline_profile.argtypes = [ctypes.c_uint, ctypes.c_uint, ctypes.POINTER(ctypes.c_uint),
                                   ctypes.POINTER(ctypes.c_uint), ctypes.c_int]
    L.baseline_profile.restype = ctypes.c_int
    if path is None:
        _lib = L
    return L
