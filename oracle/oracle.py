"""ctypes front of the C oracle (``oracle/oracle.c``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke``
and the CPU-baseline leg of ``bench.py`` as the checker / CPU baseline. The
product library (``trex_b200``) never imports it.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"

_lib = None


def build(force: bool = False) -> Path:
    if force or not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < (HERE / "oracle.c").stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def _p(a, ct):
    return a.ctypes.data_as(ctypes.POINTER(ct)) if a is not None else None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        u8p, i32p, i64p = (ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_int32),
                           ctypes.POINTER(ctypes.c_int64))
        u16p, u64p, f64p = (ctypes.POINTER(ctypes.c_uint16), ctypes.POINTER(ctypes.c_uint64),
                            ctypes.POINTER(ctypes.c_double))
        L.oracle_threads.restype = ctypes.c_int
        L.oracle_dfa_walk.argtypes = [u8p, i64p, i32p, i32p, u8p, i64p, u8p, i64p, i32p,
                                      ctypes.c_int64, u8p, u8p]
        L.oracle_dfa_positions.argtypes = [u8p, ctypes.c_int, ctypes.c_int, u8p,
                                           ctypes.c_int64, u8p]
        L.oracle_dfa_positions_batch.argtypes = [u8p, ctypes.c_int, ctypes.c_int, u8p, i64p,
                                                 ctypes.c_int64, u8p]
        L.oracle_monoid_walk.argtypes = [u16p, ctypes.c_int, ctypes.c_int, u8p, u16p, i64p,
                                         ctypes.c_int64, i32p]
        L.oracle_nfa_bool.argtypes = [u64p, ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64,
                                      ctypes.c_int, u8p, i64p, ctypes.c_int64, u64p, u8p]
        L.oracle_pnfa_fp64.argtypes = [f64p, ctypes.c_int, ctypes.c_int, f64p, f64p, u8p, i64p,
                                       ctypes.c_int64, f64p]
        for f in ("oracle_dfa_walk", "oracle_dfa_positions", "oracle_dfa_positions_batch",
                  "oracle_monoid_walk", "oracle_nfa_bool", "oracle_pnfa_fp64"):
            getattr(L, f).restype = None
        _lib = L
    return _lib


def threads() -> int:
    return lib().oracle_threads()


def set_threads(n: int) -> None:
    os.environ["OMP_NUM_THREADS"] = str(n)


# --- DFA ---------------------------------------------------------------------

def dfa_walk(tmaps, n_states, starts, accepts, data, offsets, dfa_id=None):
    """Final state and accept flag per string.

    tmaps: list of uint8 [256*N_d] tables; accepts: list of uint8 [N_d];
    data: uint8 bytes; offsets: int64 [B+1]; dfa_id: optional int32 [B].
    """
    tm = np.ascontiguousarray(np.concatenate(tmaps).astype(np.uint8))
    toff = np.cumsum([0] + [len(t) for t in tmaps[:-1]]).astype(np.int64)
    acc = np.ascontiguousarray(np.concatenate(accepts).astype(np.uint8))
    aoff = np.cumsum([0] + [len(a) for a in accepts[:-1]]).astype(np.int64)
    ns = np.asarray(n_states, dtype=np.int32)
    st = np.asarray(starts, dtype=np.int32)
    data = np.ascontiguousarray(data, dtype=np.uint8)
    offsets = np.ascontiguousarray(offsets, dtype=np.int64)
    B = len(offsets) - 1
    ids = None if dfa_id is None else np.ascontiguousarray(dfa_id, dtype=np.int32)
    fs = np.zeros(B, dtype=np.uint8)
    ac = np.zeros(B, dtype=np.uint8)
    lib().oracle_dfa_walk(_p(tm, ctypes.c_uint8), _p(toff, ctypes.c_int64), _p(ns, ctypes.c_int32),
                          _p(st, ctypes.c_int32), _p(acc, ctypes.c_uint8), _p(aoff, ctypes.c_int64),
                          _p(data if data.size else np.zeros(1, np.uint8), ctypes.c_uint8),
                          _p(offsets, ctypes.c_int64), _p(ids, ctypes.c_int32), B,
                          _p(fs, ctypes.c_uint8), _p(ac, ctypes.c_uint8))
    return fs, ac


def dfa_positions(tmap, N, start, data, offsets=None):
    """Per-position state stream (uint8, same length as data)."""
    data = np.ascontiguousarray(data, dtype=np.uint8)
    tmap = np.ascontiguousarray(tmap, dtype=np.uint8)
    out = np.zeros(max(data.size, 1), dtype=np.uint8)
    if offsets is None:
        lib().oracle_dfa_positions(_p(tmap, ctypes.c_uint8), N, start,
                                   _p(data if data.size else out, ctypes.c_uint8), data.size,
                                   _p(out, ctypes.c_uint8))
    else:
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        lib().oracle_dfa_positions_batch(_p(tmap, ctypes.c_uint8), N, start,
                                         _p(data if data.size else out, ctypes.c_uint8),
                                         _p(offsets, ctypes.c_int64), len(offsets) - 1,
                                         _p(out, ctypes.c_uint8))
    return out[:data.size]


def monoid_walk(compose, M, identity, accept, chars, offsets):
    compose = np.ascontiguousarray(compose, dtype=np.uint16).reshape(-1)
    accept = np.ascontiguousarray(accept, dtype=np.uint8)
    chars = np.ascontiguousarray(chars, dtype=np.uint16)
    offsets = np.ascontiguousarray(offsets, dtype=np.int64)
    B = len(offsets) - 1
    res = np.zeros(B, dtype=np.int32)
    lib().oracle_monoid_walk(_p(compose, ctypes.c_uint16), M, identity, _p(accept, ctypes.c_uint8),
                             _p(chars if chars.size else np.zeros(1, np.uint16), ctypes.c_uint16),
                             _p(offsets, ctypes.c_int64), B, _p(res, ctypes.c_int32))
    return res


# --- NFA ---------------------------------------------------------------------

def nfa_columns(T):
    """Dense Boolean T[sigma, N, N] (row = dst, col = src), N <= 64 ->
    uint64 cols[sigma * 64] with cols[c*64 + src] = destination mask."""
    T = np.asarray(T) != 0
    sigma, N, _ = T.shape
    cols = np.zeros((sigma, 64), dtype=np.uint64)
    weights = (np.uint64(1) << np.arange(N, dtype=np.uint64))
    for c in range(sigma):
        # bit dst of column src
        cols[c, :N] = (T[c].astype(np.uint64) * weights[:, None]).sum(axis=0, dtype=np.uint64)
    return np.ascontiguousarray(cols.reshape(-1))


def mask_of(vec) -> int:
    v = np.flatnonzero(np.asarray(vec))
    m = 0
    for b in v.tolist():
        m |= 1 << b
    return m


def nfa_bool(T, start_vec, accept_vec, data, offsets, unknown_rejects=True):
    T = np.asarray(T)
    sigma = T.shape[0]
    cols = nfa_columns(T)
    data = np.ascontiguousarray(data, dtype=np.uint8)
    offsets = np.ascontiguousarray(offsets, dtype=np.int64)
    B = len(offsets) - 1
    fm = np.zeros(B, dtype=np.uint64)
    ac = np.zeros(B, dtype=np.uint8)
    lib().oracle_nfa_bool(_p(cols, ctypes.c_uint64), sigma, mask_of(start_vec), mask_of(accept_vec),
                          1 if unknown_rejects else 0,
                          _p(data if data.size else np.zeros(1, np.uint8), ctypes.c_uint8),
                          _p(offsets, ctypes.c_int64), B, _p(fm, ctypes.c_uint64), _p(ac, ctypes.c_uint8))
    return fm, ac


def pnfa_fp64(T, start, accept, data, offsets):
    T = np.ascontiguousarray(T, dtype=np.float64)
    sigma, N, _ = T.shape
    start = np.ascontiguousarray(start, dtype=np.float64)
    accept = np.ascontiguousarray(accept, dtype=np.float64)
    data = np.ascontiguousarray(data, dtype=np.uint8)
    offsets = np.ascontiguousarray(offsets, dtype=np.int64)
    B = len(offsets) - 1
    ll = np.zeros(B, dtype=np.float64)
    lib().oracle_pnfa_fp64(_p(T, ctypes.c_double), sigma, N, _p(start, ctypes.c_double),
                           _p(accept, ctypes.c_double),
                           _p(data if data.size else np.zeros(1, np.uint8), ctypes.c_uint8),
                           _p(offsets, ctypes.c_int64), B, _p(ll, ctypes.c_double))
    return ll
