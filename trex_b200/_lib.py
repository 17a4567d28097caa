"""ctypes binding of libtrex_b200.so (built in-tree into <repo>/build/).

The library is the only compute path: if it is missing, loading raises
``FileNotFoundError`` (the reference bridges do the same,
src/gpu_bridge_monoid_batch.py:25-31); there is no CPU fallback.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

REPO = Path(__file__).resolve().parent.parent
DEFAULT_LIB = REPO / "build" / "libtrex_b200.so"

c_u8p = ctypes.POINTER(ctypes.c_uint8)
c_u16p = ctypes.POINTER(ctypes.c_uint16)
c_i32p = ctypes.POINTER(ctypes.c_int32)
c_i64p = ctypes.POINTER(ctypes.c_int64)
c_u64p = ctypes.POINTER(ctypes.c_uint64)
c_f32p = ctypes.POINTER(ctypes.c_float)
c_f64p = ctypes.POINTER(ctypes.c_double)
c_intp = ctypes.POINTER(ctypes.c_int)
c_vp = ctypes.c_void_p

# name -> (restype, argtypes); every symbol declared in include/trex_b200.h.
SIGNATURES = {
    "trex_last_error": (ctypes.c_char_p, []),
    "trex_version": (ctypes.c_char_p, []),
    "trex_profile_begin": (ctypes.c_int, [ctypes.c_int]),
    "trex_set_wait_limits": (ctypes.c_int, [ctypes.c_int64, ctypes.c_int64]),
    "trex_profile_end": (ctypes.c_int, [c_f32p, ctypes.c_int, c_intp]),
    # reference C ABI
    "monoid_batch_engine_device_check": (ctypes.c_int, []),
    "monoid_batch_engine_init": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, c_u8p, c_u8p,
                                                c_u8p, c_u8p, ctypes.c_int, ctypes.c_int]),
    "monoid_batch_engine_set_kgram": (ctypes.c_int, [c_u8p, c_u8p, ctypes.c_int, ctypes.c_int,
                                                     ctypes.c_int]),
    "monoid_batch_engine_destroy": (None, []),
    "monoid_batch_engine_dispatch": (ctypes.c_int, [c_u8p, c_intp, c_intp, ctypes.c_int, ctypes.c_int,
                                                    c_f32p, c_f32p]),
    "monoid_batch_engine_dispatch_prefix": (ctypes.c_int, [c_u8p, c_intp, c_intp, ctypes.c_int,
                                                           ctypes.c_int, c_f32p, c_f32p]),
    "prefix_engine_device_check": (ctypes.c_int, []),
    "prefix_engine_init": (ctypes.c_int, [c_u8p, c_u8p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int]),
    "prefix_engine_dispatch": (ctypes.c_int, [c_u8p, c_intp, c_intp, ctypes.c_int, ctypes.c_int,
                                              c_f32p, c_f32p]),
    "prefix_engine_destroy": (None, []),
    "monoid_engine_init": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, c_u16p, c_u8p, ctypes.c_int,
                                          ctypes.c_int]),
    "monoid_engine_destroy": (None, []),
    "monoid_engine_dispatch_batch": (ctypes.c_int, [c_u16p, c_intp, c_intp, ctypes.c_int, ctypes.c_int,
                                                    c_f32p, c_f32p]),
    "monoid_engine_device_check": (ctypes.c_int, []),
    "nfa_tc_engine_init": (ctypes.c_int, [c_f32p, c_f32p, c_f32p, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int]),
    "nfa_tc_engine_dispatch": (ctypes.c_int, [c_u8p, c_intp, c_intp, ctypes.c_int, ctypes.c_int,
                                              c_f32p, c_f32p]),
    "nfa_tc_engine_destroy": (None, []),
    "trex_nfa_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, c_u64p, ctypes.c_uint64,
                                       ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(c_vp)]),
    "trex_nfa_destroy": (None, [c_vp]),
    "trex_nfa_run": (ctypes.c_int, [c_vp, c_vp, c_vp, ctypes.c_int64, ctypes.c_int64, c_vp, c_vp,
                                    c_vp, c_vp]),
    "trex_nfa_error": (ctypes.c_int, [c_vp, c_i32p]),
    "trex_nfa_run_multi": (ctypes.c_int, [ctypes.POINTER(c_vp), ctypes.c_int, c_i64p, c_vp, c_vp,
                                          ctypes.c_int64, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "trex_pnfa_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, c_f32p, c_f32p, c_f32p,
                                        ctypes.POINTER(c_vp)]),
    "trex_pnfa_destroy": (None, [c_vp]),
    "trex_pnfa_run": (ctypes.c_int, [c_vp, ctypes.c_int, c_vp, c_vp, ctypes.c_int64, ctypes.c_int64,
                                     c_vp, c_vp, c_vp, c_vp]),
    "trex_pnfa_error": (ctypes.c_int, [c_vp, c_i32p]),
    "trex_pnfa_set_sm_limit": (ctypes.c_int, [c_vp, ctypes.c_int]),
    "trex_scatter_strings": (ctypes.c_int, [c_vp, ctypes.c_int64, c_vp, ctypes.c_int64, c_vp,
                                            ctypes.c_int64, c_vp, c_vp, c_vp]),
    # handle API
    "trex_dfa_set_create": (ctypes.c_int, [ctypes.c_int, c_i32p, c_i32p, c_u8p, c_u8p,
                                           ctypes.POINTER(c_vp)]),
    "trex_dfa_set_destroy": (None, [c_vp]),
    "trex_dfa_batch_run_multi": (ctypes.c_int, [c_vp, c_vp, c_vp, ctypes.c_int64, ctypes.c_int64, c_vp, c_vp,
                                                c_vp, c_vp, ctypes.c_int64, ctypes.c_int32, c_vp]),
    "trex_dfa_kgram_max": (ctypes.c_int, [c_vp, ctypes.c_int, c_intp]),
    "trex_dfa_set_kgram": (ctypes.c_int, [c_vp, ctypes.c_int, ctypes.c_int]),
    "trex_dfa_get_kgram": (ctypes.c_int, [c_vp, ctypes.c_int, c_intp]),
    "trex_dfa_batch_scratch_bytes": (ctypes.c_int64, [ctypes.c_int64, ctypes.c_int64, ctypes.c_int32]),
    "trex_dfa_batch_run": (ctypes.c_int, [c_vp, c_vp, c_vp, c_vp, ctypes.c_int64, ctypes.c_int64,
                                          c_vp, c_vp, c_vp, c_vp, ctypes.c_int64, ctypes.c_int32,
                                          c_vp]),
    "trex_dfa_batch_error": (ctypes.c_int, [c_vp, c_vp, c_i32p]),
    "trex_dfa_batch_run_static": (ctypes.c_int, [c_vp, c_vp, c_vp, c_vp, ctypes.c_int64,
                                                 ctypes.c_int64, c_vp, c_vp, c_vp, ctypes.c_int32,
                                                 c_vp]),
    "trex_dfa_batch_static_error": (ctypes.c_int, [c_vp, c_i32p]),
    "trex_dfa_scan_scratch_bytes": (ctypes.c_int64, [ctypes.c_int64, ctypes.c_int64, ctypes.c_int32]),
    "trex_dfa_scan_run": (ctypes.c_int, [c_vp, ctypes.c_int, c_vp, c_vp, ctypes.c_int64,
                                         ctypes.c_int64, c_vp, c_vp, c_vp, c_vp, ctypes.c_int64,
                                         ctypes.c_int32, c_vp]),
    "trex_dfa_scan_error": (ctypes.c_int, [c_vp, ctypes.c_int64, ctypes.c_int64, ctypes.c_int32,
                                           c_i32p]),
    "trex_dfa_batch_host": (ctypes.c_int, [c_vp, c_u8p, c_i64p, c_i32p, ctypes.c_int64,
                                           ctypes.c_int64, c_u8p, c_u8p, c_i32p, ctypes.c_int32,
                                           c_f32p, c_f32p]),
}

ERRORS = {
    0: "ok", -1: "not initialised", -2: "unsupported shape or device", -3: "CUDA error",
    -4: "capacity exceeded", -5: "invalid argument", -6: "device-side error or timeout",
    -7: "device out of memory",
}

_lib = None
_lib_path = None


def lib_path() -> Path:
    return Path(os.environ.get("TREX_B200_LIB", DEFAULT_LIB))


def load(path=None):
    """Load (once) and return the ctypes library with all signatures set."""
    global _lib, _lib_path
    p = Path(path) if path else lib_path()
    if _lib is not None and (path is None or p == _lib_path):
        return _lib
    if not p.exists():
        raise FileNotFoundError(
            f"{p.name} not found at {p}. Build it with 'python -m trex_b200.build'.")
    L = ctypes.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    if path is None or _lib is None:
        _lib, _lib_path = L, p
    return L


def last_error() -> str:
    return (load().trex_last_error() or b"").decode(errors="replace")


def check(rc: int, what: str) -> None:
    if rc != 0:
        raise RuntimeError(f"{what} failed with code {rc} ({ERRORS.get(rc, '?')}): {last_error()}")


def ptr(a, ctype):
    """ctypes pointer to a numpy array's data (None for None)."""
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctype))
