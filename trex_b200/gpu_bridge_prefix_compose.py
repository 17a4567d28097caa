"""ctypes bridge to the prefix-compose (byte-map DFA) engine.

Drop-in for the reference module ``src/gpu_bridge_prefix_compose.py``
(reference src/gpu_bridge_prefix_compose.py:34-168): same classes, methods,
return values and errors. The engine behind ``prefix_engine_*`` is this
library's ragged batch kernel (family a); N may be up to 256 here (the
reference fixes N = 16). Bytes outside the DFA alphabet are the identity,
as in the reference's GPU path (``precompute_tmap``).

Usage:
    sim = PrefixComposeGPUSimulator()
    engine = sim.create_engine(dm)
    results = engine.simulate_batch(["abb", "ab", "aabb"])
    results, kern_ms, total_ms = engine.simulate_batch_timed(strings)
    engine.destroy()
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._batching import pack_strings
from .simulation import DFAMatrices, precompute_tmap


def _find_lib():
    p = _lib.lib_path()
    if p.exists():
        return str(p)
    raise FileNotFoundError(f"{p.name} not found at {p}. Run 'python -m trex_b200.build' first.")


class PrefixComposeEngine:
    def __init__(self, lib, dm: DFAMatrices, max_total_chars: int = 1 << 22,
                 max_batch: int = 1 << 18):
        self.lib = lib
        self.dm = dm
        tmap = np.ascontiguousarray(precompute_tmap(dm))
        accept = np.zeros(dm.n_states, dtype=np.uint8)
        for s in dm.dfa.accept_states:
            accept[s] = 1
        rc = self.lib.prefix_engine_init(_lib.ptr(tmap, ctypes.c_uint8), _lib.ptr(accept, ctypes.c_uint8),
                                         dm.dfa.start, dm.n_states, 32, max_total_chars, max_batch)
        if rc != 0:
            raise RuntimeError(f"prefix_engine_init failed with code {rc}")

    def destroy(self):
        self.lib.prefix_engine_destroy()

    def _dispatch(self, strings):
        data, offsets, total = pack_strings(strings)
        B = len(strings)
        results = np.zeros(B, dtype=np.int32)
        kern_ms = ctypes.c_float(0)
        total_ms = ctypes.c_float(0)
        rc = self.lib.prefix_engine_dispatch(
            _lib.ptr(data, ctypes.c_uint8), _lib.ptr(offsets, ctypes.c_int),
            _lib.ptr(results, ctypes.c_int), B, total, ctypes.byref(kern_ms), ctypes.byref(total_ms))
        if rc != 0:
            raise RuntimeError(f"prefix_engine dispatch failed with code {rc}")
        return [bool(r) for r in results], kern_ms.value, total_ms.value

    def simulate_batch(self, strings: list) -> list:
        if not strings:
            return []
        return self._dispatch(strings)[0]

    def simulate_batch_timed(self, strings: list):
        if not strings:
            return [], 0.0, 0.0
        return self._dispatch(strings)


class PrefixComposeGPUSimulator:
    def __init__(self, lib_path: str | None = None):
        self.lib = _lib.load(lib_path or _find_lib())
        rc = self.lib.prefix_engine_device_check()
        if rc == -1:
            raise RuntimeError("No CUDA device found")
        if rc == -2:
            raise RuntimeError("GPU does not support SM >= 7.x")

    def create_engine(self, dm: DFAMatrices, max_total_chars: int = 1 << 22,
                      max_batch: int = 1 << 18) -> PrefixComposeEngine:
        return PrefixComposeEngine(self.lib, dm, max_total_chars, max_batch)
