"""ctypes bridge to the monoid scan engine (uint16 monoid-element streams).

Drop-in for the reference module ``src/gpu_bridge_monoid.py``
(reference src/gpu_bridge_monoid.py:33-179): characters are mapped to monoid
element indices on the host (unknown characters -> identity, :61-85) and the
engine walks ``acc = compose[c * M + acc]``.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .monoid import MonoidData
from .simulation import DFAMatrices


def _find_lib():
    p = _lib.lib_path()
    if p.exists():
        return str(p)
    raise FileNotFoundError(f"{p.name} not found at {p}. Run 'python -m trex_b200.build' first.")


class MonoidEngine:
    def __init__(self, lib, md: MonoidData, max_total_chars: int = 1 << 22,
                 max_batch: int = 1 << 18):
        self.lib = lib
        self.md = md
        compose = np.ascontiguousarray(md.compose_table.reshape(-1), dtype=np.uint16)
        accept = np.ascontiguousarray(md.accept_table.astype(np.uint8))
        rc = self.lib.monoid_engine_init(md.size, md.identity_idx, _lib.ptr(compose, ctypes.c_uint16),
                                         _lib.ptr(accept, ctypes.c_uint8), max_total_chars, max_batch)
        if rc != 0:
            raise RuntimeError(f"monoid_engine_init failed with code {rc}")
        # byte -> element lookup for latin-1 characters
        self._byte_map = np.full(256, md.identity_idx, dtype=np.uint16)
        self._wide = {}
        for ch, m in md.char_to_monoid.items():
            if ord(ch) < 256:
                self._byte_map[ord(ch)] = m
            else:
                self._wide[ch] = m

    def destroy(self):
        self.lib.monoid_engine_destroy()

    def _prepare_batch(self, strings):
        B = len(strings)
        lens = np.fromiter((len(s) for s in strings), dtype=np.int64, count=B)
        offsets = np.zeros(B + 1, dtype=np.int64)
        np.cumsum(lens, out=offsets[1:])
        total = int(offsets[-1])
        joined = "".join(strings)
        try:
            raw = np.frombuffer(joined.encode("latin-1"), dtype=np.uint8)
            chars = self._byte_map[raw] if total else np.zeros(1, dtype=np.uint16)
        except UnicodeEncodeError:
            ident = self.md.identity_idx
            c2m = self.md.char_to_monoid
            chars = np.fromiter((c2m.get(c, ident) for c in joined), dtype=np.uint16, count=total)
        return np.ascontiguousarray(chars, dtype=np.uint16), offsets.astype(np.int32), total

    def _run(self, strings):
        B = len(strings)
        chars, offsets, total = self._prepare_batch(strings)
        results = np.zeros(B, dtype=np.int32)
        kern_ms = ctypes.c_float(0)
        total_ms = ctypes.c_float(0)
        rc = self.lib.monoid_engine_dispatch_batch(
            _lib.ptr(chars, ctypes.c_uint16), _lib.ptr(offsets, ctypes.c_int),
            _lib.ptr(results, ctypes.c_int), B, total, ctypes.byref(kern_ms), ctypes.byref(total_ms))
        if rc != 0:
            raise RuntimeError(f"monoid_engine_dispatch_batch failed with code {rc}")
        return [bool(r) for r in results], kern_ms.value, total_ms.value

    def simulate_batch(self, strings: list) -> list:
        if not strings:
            return []
        return self._run(strings)[0]

    def simulate_batch_timed(self, strings: list):
        if not strings:
            return [], 0.0, 0.0
        return self._run(strings)


class MonoidGPUSimulator:
    def __init__(self, lib_path: str | None = None):
        self.lib = _lib.load(lib_path or _find_lib())
        rc = self.lib.monoid_engine_device_check()
        if rc == -1:
            raise RuntimeError("No CUDA device found")
        if rc == -2:
            raise RuntimeError("GPU does not support SM >= 7.x")

    def create_engine(self, md: MonoidData, dm: DFAMatrices, max_total_chars: int = 1 << 22,
                      max_batch: int = 1 << 18) -> MonoidEngine:
        return MonoidEngine(self.lib, md, max_total_chars, max_batch)
