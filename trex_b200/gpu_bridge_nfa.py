"""GPU bridge for Boolean NFAs (families c): ``NFAMatrices`` -> bit-parallel kernel.

The reference has a C engine for this path (``nfa_tc_engine_*``,
cuda/nfa_tc_evolution.cu:936-1015) but no Python bridge; this module gives it
one in the style of the other bridges (src/gpu_bridge_prefix_compose.py):
``NFAGPUSimulator().create_engine(nm)`` -> ``simulate_batch`` /
``simulate_batch_timed`` / ``destroy``. Semantics follow
``simulate_nfa`` (src/nfa_matrices.py:133-157): a character outside the
alphabet rejects the string.
"""

from __future__ import annotations

import numpy as np

from . import _lib
from .engine import NFA
from .nfa_matrices import NFAMatrices


class NFAEngine:
    def __init__(self, nm: NFAMatrices):
        if nm.n_states > 64:
            raise ValueError(f"NFA has {nm.n_states} states; the GPU engine handles at most 64")
        self.nm = nm
        self.sigma = len(nm.alphabet)
        if self.sigma > 255:
            raise ValueError("alphabet larger than 255 symbols")
        self.nfa = NFA(nm.matrix_stack, nm.start_vec, nm.accept_mask, unknown_rejects=True)
        # character -> symbol index; every other byte -> sigma (rejects)
        self._byte_map = np.full(256, self.sigma, dtype=np.uint8)
        self._wide = {}
        for i, ch in enumerate(nm.alphabet):
            if ord(ch) < 256:
                self._byte_map[ord(ch)] = i
            else:
                self._wide[ch] = i

    def destroy(self):
        self.nfa.close()

    def _encode(self, strings):
        B = len(strings)
        lens = np.fromiter((len(s) for s in strings), dtype=np.int64, count=B)
        off = np.zeros(B + 1, dtype=np.int64)
        np.cumsum(lens, out=off[1:])
        joined = "".join(strings)
        try:
            raw = np.frombuffer(joined.encode("latin-1"), dtype=np.uint8)
            sym = self._byte_map[raw]
        except UnicodeEncodeError:
            c2i = {**{ch: i for i, ch in enumerate(self.nm.alphabet)}}
            sym = np.fromiter((c2i.get(c, self.sigma) for c in joined), dtype=np.uint8,
                              count=len(joined))
        return np.ascontiguousarray(sym), off

    def _run(self, strings):
        import torch
        sym, off = self._encode(strings)
        d_sym = torch.from_numpy(sym if sym.size else np.zeros(1, np.uint8)).cuda()
        d_off = torch.from_numpy(off).cuda()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        _, acc = self.nfa.run(d_sym[:sym.size], d_off)
        e1.record()
        out = acc.cpu().numpy()
        return [bool(x) for x in out], e0.elapsed_time(e1)

    def simulate_batch(self, strings: list) -> list:
        if not strings:
            return []
        return self._run(strings)[0]

    def simulate_batch_timed(self, strings: list):
        if not strings:
            return [], 0.0, 0.0
        import time
        t0 = time.perf_counter()
        res, kms = self._run(strings)
        return res, kms, (time.perf_counter() - t0) * 1e3


class NFAGPUSimulator:
    def __init__(self, lib_path: str | None = None):
        self.lib = _lib.load(lib_path)

    def create_engine(self, nm: NFAMatrices) -> NFAEngine:
        return NFAEngine(nm)
