"""ctypes bridge to the monoid batch engine.

Drop-in for the reference module ``src/gpu_bridge_monoid_batch.py``
(reference src/gpu_bridge_monoid_batch.py:34-237): same classes, methods,
return values and errors, including the all-empty shortcut (:108-111) and
the prefix dispatch for few long strings (:118-121). Behind it the monoid
is walked as an automaton over its M <= 255 elements by this library's
ragged batch kernel.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._batching import pack_strings
from .monoid import MonoidData, precompute_batch_tables
from .simulation import DFAMatrices


def _find_lib():
    p = _lib.lib_path()
    if p.exists():
        return str(p)
    raise FileNotFoundError(f"{p.name} not found at {p}. Run 'python -m trex_b200.build' first.")


class MonoidBatchEngine:
    def __init__(self, lib, md: MonoidData, dm: DFAMatrices, max_total_chars: int = 1 << 22,
                 max_batch: int = 1 << 18):
        self.lib = lib
        self.md = md
        t = precompute_batch_tables(md, dm)
        u8 = ctypes.c_uint8
        char_compose = np.ascontiguousarray(t["char_compose"])
        raw_char_map = np.ascontiguousarray(t["raw_char_map"])
        accept = np.ascontiguousarray(t["accept"])
        monoid_compose = np.ascontiguousarray(t["monoid_compose"])
        rc = self.lib.monoid_batch_engine_init(
            t["M"], t["sigma_ext"], t["identity_idx"], _lib.ptr(char_compose, u8),
            _lib.ptr(raw_char_map, u8), _lib.ptr(accept, u8), _lib.ptr(monoid_compose, u8),
            max_total_chars, max_batch)
        if rc != 0:
            raise RuntimeError(f"monoid_batch_engine_init failed with code {rc}")
        fused = np.ascontiguousarray(t["fused_compose"])
        kgram = t["kgram_compose"]
        rc = self.lib.monoid_batch_engine_set_kgram(
            _lib.ptr(fused, u8), _lib.ptr(kgram, u8) if kgram is not None else None,
            t["kgram_k"], t["sigma_k"], t["sigma"])
        if rc != 0:
            raise RuntimeError(f"monoid_batch_engine_set_kgram failed with code {rc}")

    def destroy(self):
        self.lib.monoid_batch_engine_destroy()

    def _run(self, strings):
        B = len(strings)
        L_max = max((len(s) for s in strings), default=0)
        if L_max == 0:
            acc = bool(self.md.accept_table[self.md.identity_idx])
            return [acc] * B, 0.0, 0.0
        data, offsets, total = pack_strings(strings)
        results = np.zeros(B, dtype=np.int32)
        kern_ms = ctypes.c_float(0)
        total_ms = ctypes.c_float(0)
        fn = (self.lib.monoid_batch_engine_dispatch_prefix if (B <= 128 and L_max > 100_000)
              else self.lib.monoid_batch_engine_dispatch)
        rc = fn(_lib.ptr(data, ctypes.c_uint8), _lib.ptr(offsets, ctypes.c_int),
                _lib.ptr(results, ctypes.c_int), B, total, ctypes.byref(kern_ms),
                ctypes.byref(total_ms))
        if rc != 0:
            raise RuntimeError(f"monoid_batch dispatch failed with code {rc}")
        return [bool(r) for r in results], kern_ms.value, total_ms.value

    def simulate_batch(self, strings: list) -> list:
        if not strings:
            return []
        return self._run(strings)[0]

    def simulate_batch_timed(self, strings: list):
        if not strings:
            return [], 0.0, 0.0
        return self._run(strings)


class MonoidBatchGPUSimulator:
    def __init__(self, lib_path: str | None = None):
        self.lib = _lib.load(lib_path or _find_lib())
        rc = self.lib.monoid_batch_engine_device_check()
        if rc == -1:
            raise RuntimeError("No CUDA device found")
        if rc == -2:
            raise RuntimeError("GPU does not support SM >= 7.x")

    def create_engine(self, md: MonoidData, dm: DFAMatrices, max_total_chars: int = 1 << 22,
                      max_batch: int = 1 << 18) -> MonoidBatchEngine:
        return MonoidBatchEngine(self.lib, md, dm, max_total_chars, max_batch)
