"""Handle-based engines over the trex_* C ABI.

``DFASet`` keeps up to 64 byte DFAs resident on the GPU and runs ragged
batches from device tensors (``run``) or host arrays (``run_host``). PyTorch
is used only to hold device memory and streams; all compute goes through
libtrex_b200.so.
"""

from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np

from . import _lib
from .workloads import ByteDFA


def _torch():
    import torch
    return torch


def _dptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream_handle(stream):
    if stream is None:
        torch = _torch()
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return ctypes.c_void_p(stream.cuda_stream)


def profile_begin(max_launches: int) -> None:
    """Bracket the main kernel of the next ``max_launches`` runs with CUDA events."""
    _lib.check(_lib.load().trex_profile_begin(max_launches), "trex_profile_begin")


def profile_end(capacity: int = 100000) -> list:
    """Stop recording; per-launch main-kernel durations in ms (synchronises)."""
    buf = np.zeros(capacity, dtype=np.float32)
    cnt = ctypes.c_int(0)
    _lib.check(_lib.load().trex_profile_end(_lib.ptr(buf, ctypes.c_float), capacity,
                                            ctypes.byref(cnt)), "trex_profile_end")
    return buf[:min(cnt.value, capacity)].tolist()


class DFASet:
    """Resident set of byte DFAs (N <= 256 each, at most 64).

    kgram: None (byte walks), an int applied to every automaton, or one int
    per automaton: K-gram width (1, 2, 4, 8, or 0 for the largest the
    automaton allows; automata that allow none keep byte walks when 0 is
    given). See kgram_max / set_kgram.
    """

    def __init__(self, dfas: Sequence[ByteDFA], kgram=None):
        self.lib = _lib.load()
        self.dfas = list(dfas)
        n = len(self.dfas)
        ns = np.array([d.n_states for d in self.dfas], dtype=np.int32)
        st = np.array([d.start for d in self.dfas], dtype=np.int32)
        tm = np.ascontiguousarray(np.concatenate([d.tmap for d in self.dfas]).astype(np.uint8))
        ac = np.ascontiguousarray(np.concatenate([d.accept for d in self.dfas]).astype(np.uint8))
        h = ctypes.c_void_p()
        rc = self.lib.trex_dfa_set_create(n, _lib.ptr(ns, ctypes.c_int32), _lib.ptr(st, ctypes.c_int32),
                                          _lib.ptr(tm, ctypes.c_uint8), _lib.ptr(ac, ctypes.c_uint8),
                                          ctypes.byref(h))
        _lib.check(rc, "trex_dfa_set_create")
        self._h = h
        if kgram is not None:
            ks = [kgram] * n if isinstance(kgram, int) else list(kgram)
            for i, k in enumerate(ks):
                if k == 0 and self.kgram_max(i) == 1:
                    continue
                self.set_kgram(i, k)

    def kgram_max(self, index: int) -> int:
        """Largest K-gram width automaton `index` allows (1: byte walks only)."""
        k = ctypes.c_int()
        _lib.check(self.lib.trex_dfa_kgram_max(self._h, index, ctypes.byref(k)), "trex_dfa_kgram_max")
        return k.value

    def set_kgram(self, index: int, k: int) -> None:
        """K-gram width of automaton `index` (1 = bytes, 2/4/8, 0 = largest); between runs."""
        _lib.check(self.lib.trex_dfa_set_kgram(self._h, index, k), "trex_dfa_set_kgram")

    def get_kgram(self, index: int) -> int:
        k = ctypes.c_int()
        _lib.check(self.lib.trex_dfa_get_kgram(self._h, index, ctypes.byref(k)), "trex_dfa_get_kgram")
        return k.value

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            self.lib.trex_dfa_set_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def scratch_bytes(n_strings: int, total_bytes: int, seg_len: int = 0) -> int:
        return int(_lib.load().trex_dfa_batch_scratch_bytes(n_strings, total_bytes, seg_len))

    def run(self, data, offsets, dfa_id=None, *, final_state=None, accept=None, accept_i32=None,
            scratch=None, seg_len: int = 0, stream=None, want=("final_state", "accept")):
        """Device run. data: uint8 CUDA tensor; offsets: int64 CUDA tensor [n+1];
        dfa_id: optional int32 CUDA tensor [n]. Missing outputs listed in
        ``want`` are allocated. Returns (final_state, accept, accept_i32)."""
        torch = _torch()
        n = offsets.numel() - 1
        dev = offsets.device
        if final_state is None and "final_state" in want:
            final_state = torch.empty(n, dtype=torch.uint8, device=dev)
        if accept is None and "accept" in want:
            accept = torch.empty(n, dtype=torch.uint8, device=dev)
        if accept_i32 is None and "accept_i32" in want:
            accept_i32 = torch.empty(n, dtype=torch.int32, device=dev)
        sc_bytes = scratch.numel() if scratch is not None else 0
        rc = self.lib.trex_dfa_batch_run(
            self._h, _dptr(data), _dptr(offsets), _dptr(dfa_id), n, data.numel(),
            _dptr(final_state), _dptr(accept), _dptr(accept_i32), _dptr(scratch), sc_bytes,
            seg_len, _stream_handle(stream))
        _lib.check(rc, "trex_dfa_batch_run")
        return final_state, accept, accept_i32

    def run_all(self, data, offsets, *, final_state=None, accept=None, scratch=None,
                seg_len: int = 0, stream=None):
        """Every string against every automaton of the set (device tensors, as run).
        Returns (final_state, accept) of shape [n_dfas, n] (automaton-major)."""
        torch = _torch()
        n = offsets.numel() - 1
        P = len(self.dfas)
        dev = offsets.device
        if final_state is None:
            final_state = torch.empty(max(P * n, 1), dtype=torch.uint8, device=dev)
        if accept is None:
            accept = torch.empty(max(P * n, 1), dtype=torch.uint8, device=dev)
        sc_bytes = scratch.numel() if scratch is not None else 0
        rc = self.lib.trex_dfa_batch_run_multi(
            self._h, _dptr(data), _dptr(offsets), n, data.numel(), _dptr(final_state), _dptr(accept),
            None, _dptr(scratch), sc_bytes, seg_len, _stream_handle(stream))
        _lib.check(rc, "trex_dfa_batch_run_multi")
        return final_state[:P * n].view(P, n), accept[:P * n].view(P, n)

    @staticmethod
    def scan_scratch_bytes(n_strings: int, total_bytes: int, tile_len: int = 0) -> int:
        return int(_lib.load().trex_dfa_scan_scratch_bytes(n_strings, total_bytes, tile_len))

    def scan(self, data, offsets, dfa_index: int = 0, *, states=None, final_state=None,
             accept=None, scratch=None, tile_len: int = 0, stream=None):
        """Per-position states of every string (device tensors). Returns
        (states[total_bytes], final_state[n], accept[n], scratch)."""
        torch = _torch()
        n = offsets.numel() - 1
        dev = offsets.device
        total = data.numel()
        if states is None:
            states = torch.empty(max(total, 1), dtype=torch.uint8, device=dev)
        if final_state is None:
            final_state = torch.empty(max(n, 1), dtype=torch.uint8, device=dev)
        if accept is None:
            accept = torch.empty(max(n, 1), dtype=torch.uint8, device=dev)
        need = self.scan_scratch_bytes(n, total, tile_len)
        if scratch is None or scratch.numel() < need:
            scratch = torch.empty(need, dtype=torch.uint8, device=dev)
        rc = self.lib.trex_dfa_scan_run(self._h, dfa_index, _dptr(data), _dptr(offsets), n, total,
                                        _dptr(states), _dptr(final_state), _dptr(accept),
                                        _dptr(scratch), scratch.numel(), tile_len,
                                        _stream_handle(stream))
        _lib.check(rc, "trex_dfa_scan_run")
        return states[:total], final_state[:n], accept[:n], scratch

    def scan_error_word(self, scratch, n_strings: int, total_bytes: int, tile_len: int = 0) -> int:
        v = ctypes.c_int32(0)
        rc = self.lib.trex_dfa_scan_error(_dptr(scratch), n_strings, total_bytes, tile_len,
                                          ctypes.byref(v))
        _lib.check(rc, "trex_dfa_scan_error")
        return v.value

    def last_error_word(self, scratch=None) -> int:
        v = ctypes.c_int32(0)
        rc = self.lib.trex_dfa_batch_error(self._h, _dptr(scratch), ctypes.byref(v))
        _lib.check(rc, "trex_dfa_batch_error")
        return v.value

    def run_host(self, data: np.ndarray, offsets: np.ndarray, dfa_id: Optional[np.ndarray] = None,
                 seg_len: int = 0, final_state=None, accept=None):
        """Host-buffer run (copies in and out). Returns (final_state, accept,
        kernel_ms, total_ms). Passing pinned numpy views makes the copies
        asynchronous DMA."""
        data = np.ascontiguousarray(data, dtype=np.uint8)
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        n = len(offsets) - 1
        ids = None if dfa_id is None else np.ascontiguousarray(dfa_id, dtype=np.int32)
        fs = final_state if final_state is not None else np.zeros(n, dtype=np.uint8)
        ac = accept if accept is not None else np.zeros(n, dtype=np.uint8)
        km, tm = ctypes.c_float(0), ctypes.c_float(0)
        rc = self.lib.trex_dfa_batch_host(
            self._h, _lib.ptr(data if data.size else np.zeros(1, np.uint8), ctypes.c_uint8),
            _lib.ptr(offsets, ctypes.c_int64), _lib.ptr(ids, ctypes.c_int32), n, data.size,
            _lib.ptr(fs, ctypes.c_uint8), _lib.ptr(ac, ctypes.c_uint8), None, seg_len,
            ctypes.byref(km), ctypes.byref(tm))
        _lib.check(rc, "trex_dfa_batch_host")
        return fs, ac, km.value, tm.value


def nfa_columns(T) -> np.ndarray:
    """Dense Boolean T[sigma, N, N] (row = destination, column = source),
    N <= 64 -> uint64 cols[sigma * 64] with cols[c*64 + src] = destination mask."""
    T = np.asarray(T) != 0
    sigma, N, _ = T.shape
    cols = np.zeros((sigma, 64), dtype=np.uint64)
    w = np.left_shift(np.uint64(1), np.arange(N, dtype=np.uint64))
    for c in range(sigma):
        cols[c, :N] = np.bitwise_or.reduce(np.where(T[c], w[:, None], np.uint64(0)), axis=0)
    return np.ascontiguousarray(cols.reshape(-1))


def mask_of(vec) -> int:
    m = 0
    for b in np.flatnonzero(np.asarray(vec)).tolist():
        m |= 1 << b
    return m


class NFA:
    """Resident Boolean NFA with at most 64 states (bit-parallel kernel)."""

    def __init__(self, T, start_vec, accept_vec, unknown_rejects: bool = True):
        self.lib = _lib.load()
        T = np.asarray(T)
        self.sigma, self.n_states, _ = T.shape
        cols = nfa_columns(T)
        h = ctypes.c_void_p()
        rc = self.lib.trex_nfa_create(self.n_states, self.sigma, _lib.ptr(cols, ctypes.c_uint64),
                                      mask_of(start_vec), mask_of(accept_vec),
                                      1 if unknown_rejects else 0, ctypes.byref(h))
        _lib.check(rc, "trex_nfa_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self.lib.trex_nfa_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, data, offsets, *, final_mask=None, accept=None, stream=None):
        """Device run: returns (final_mask int64 tensor [n] (bit pattern of the
        uint64 mask), accept uint8 tensor [n])."""
        torch = _torch()
        n = offsets.numel() - 1
        if final_mask is None:
            final_mask = torch.empty(max(n, 1), dtype=torch.int64, device=offsets.device)
        if accept is None:
            accept = torch.empty(max(n, 1), dtype=torch.uint8, device=offsets.device)
        rc = self.lib.trex_nfa_run(self._h, _dptr(data), _dptr(offsets), n, data.numel(),
                                   _dptr(final_mask), _dptr(accept), None, _stream_handle(stream))
        _lib.check(rc, "trex_nfa_run")
        return final_mask[:n], accept[:n]

    def error_word(self) -> int:
        v = ctypes.c_int32(0)
        _lib.check(self.lib.trex_nfa_error(self._h, ctypes.byref(v)), "trex_nfa_error")
        return v.value


def nfa_run_multi(nfas: Sequence["NFA"], group_first, data, offsets, *, final_mask, accept, scratch,
                  stream=None) -> None:
    """One call over strings grouped by automaton: strings group_first[g] ..
    group_first[g+1] - 1 of offsets run on nfas[g] (at most 64 groups), side by
    side. final_mask (int64) / accept (uint8) are indexed by the string's
    position; scratch is a device buffer of at least 8 * (len(nfas) + 1) bytes
    whose last word is the error word (bit 0: malformed offsets)."""
    lib = _lib.load()
    g = len(nfas)
    gf = np.ascontiguousarray(group_first, dtype=np.int64)
    if gf.size != g + 1:
        raise ValueError("group_first needs len(nfas) + 1 entries")
    hs = (ctypes.c_void_p * max(g, 1))(*[m._h.value for m in nfas])
    rc = lib.trex_nfa_run_multi(hs, g, _lib.ptr(gf, ctypes.c_int64), _dptr(data), _dptr(offsets),
                                data.numel(), _dptr(final_mask), _dptr(accept), None, _dptr(scratch),
                                _stream_handle(stream))
    _lib.check(rc, "trex_nfa_run_multi")


PNFA_MODES = {"bf16": 0, "fp16": 1, "fp32": 2, "bool": 3, "bf16cc": 4, "fp16cc": 5, "bool8": 6}


class PNFA:
    """Resident probabilistic NFA (at most 64 states): s' = T[c] s per symbol,
    result log(dot(s_L, accept)) in FP64 (reference
    cuda/nfa_tc_evolution.cu:456-610 computes only dot > 0.5).

    Modes: "bf16" / "fp16" run the tcgen05 tensor-core kernel (16-bit
    operands, FP32 accumulation, sigma <= 28); "fp32" the CUDA-core kernel.
    "bool" runs the Boolean NFA of the same tables on the tensor cores (the
    reference's FP16 WMMA nfa_tc_binary kernels, cuda/nfa_tc_evolution.cu:
    59-442): nonzero entries are edges, each product is thresholded to {0, 1}
    (exact), accept = some accepting state active; loglik is then the log of
    the number of active accepting states. Bytes >= sigma are skipped.
    "bool8": the same Boolean NFA with 0/1 int8 operands and int32 sums (tcgen05
    kind::i8, K = 32 an instruction: half the MMA instructions of "bool").
    "bf16cc" / "fp16cc": CUDA cores with the 16-bit tables in shared memory and an
    FP32 state, four warps per string: the low-latency form for few strings.
    """

    def __init__(self, T, start_vec, accept_vec):
        self.lib = _lib.load()
        T = np.ascontiguousarray(np.asarray(T, dtype=np.float32))
        if T.ndim != 3 or T.shape[1] != T.shape[2]:
            raise ValueError("T must have shape (sigma, n, n)")
        self.sigma, self.n_states, _ = T.shape
        start = np.ascontiguousarray(np.asarray(start_vec, dtype=np.float32).reshape(-1))
        acc = np.ascontiguousarray(np.asarray(accept_vec, dtype=np.float32).reshape(-1))
        if start.size != self.n_states or acc.size != self.n_states:
            raise ValueError("start and accept vectors must have n entries")
        h = ctypes.c_void_p()
        rc = self.lib.trex_pnfa_create(self.n_states, self.sigma, _lib.ptr(T, ctypes.c_float),
                                       _lib.ptr(start, ctypes.c_float), _lib.ptr(acc, ctypes.c_float),
                                       ctypes.byref(h))
        _lib.check(rc, "trex_pnfa_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self.lib.trex_pnfa_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, data, offsets, mode: str = "bf16", *, loglik=None, accept=None, stream=None):
        """Device run: returns (loglik float64 tensor [n], accept uint8 tensor [n])."""
        torch = _torch()
        if mode not in PNFA_MODES:
            raise ValueError(f"mode must be one of {sorted(PNFA_MODES)}")
        n = offsets.numel() - 1
        if loglik is None:
            loglik = torch.empty(max(n, 1), dtype=torch.float64, device=offsets.device)
        if accept is None:
            accept = torch.empty(max(n, 1), dtype=torch.uint8, device=offsets.device)
        rc = self.lib.trex_pnfa_run(self._h, PNFA_MODES[mode], _dptr(data), _dptr(offsets), n,
                                    data.numel(), _dptr(loglik), _dptr(accept), None,
                                    _stream_handle(stream))
        _lib.check(rc, "trex_pnfa_run")
        return loglik[:n], accept[:n]

    def set_sm_limit(self, max_sms: int) -> None:
        """Size later runs for at most max_sms SMs (0: all); results do not change."""
        _lib.check(self.lib.trex_pnfa_set_sm_limit(self._h, int(max_sms)), "trex_pnfa_set_sm_limit")

    def error_word(self) -> int:
        v = ctypes.c_int32(0)
        _lib.check(self.lib.trex_pnfa_error(self._h, ctypes.byref(v)), "trex_pnfa_error")
        return v.value
