"""Multi-pattern matching: every string against every pattern.

Drop-in for the reference's ``src/packed_engine.py`` (``PackedEngine``,
:25-125 and :275-439): the same constructor, ``match_batch`` (results
``[pattern][string]``), ``match_batch_timed`` and ``config_info``. The
reference packs the patterns' DFAs block-diagonally into one NP × NP Boolean
matrix per character and evolves one state vector per string; a character
outside a pattern's alphabet (or outside every alphabet) leaves that
pattern's state unchanged (:107-110, :392-397).

Here, with ``use_gpu=True``, the patterns are byte DFAs resident in one
``DFASet`` and one multi-pattern launch of the B200 ragged kernel
(``trex_dfa_batch_run_multi``) walks every string with every automaton,
reading the input once per automaton without copying it. With
``use_gpu=False`` the same byte-map walk runs on the host, one pattern at a
time (the reference's CPU path, restated).
"""

from __future__ import annotations

import time
from typing import Sequence

import numpy as np

from .regex_to_dfa import compile_regex
from .simulation import DFAMatrices
from .workloads import dfa_from_regex_dfa

_MAX_SET = 64   # automata a DFA set holds


class PackedEngine:
    def __init__(self, regexes: list[str], use_gpu: bool = False, gpu_mode: str = "auto"):
        self._regexes = list(regexes)
        self._n_patterns = len(self._regexes)
        self._gpu_mode = gpu_mode
        self._dfas = [compile_regex(r) for r in self._regexes]
        self._dfa_matrices = [DFAMatrices(d) for d in self._dfas]
        chars: set[str] = set()
        for dm in self._dfa_matrices:
            chars.update(dm.alphabet)
        self._unified_alphabet = sorted(chars)
        self._state_counts = [dm.n_states for dm in self._dfa_matrices]
        self._offsets = list(np.concatenate([[0], np.cumsum(self._state_counts)[:-1]]).astype(int)) \
            if self._state_counts else []
        self._NP = ((sum(self._state_counts) + 15) // 16) * 16
        # byte maps: unknown bytes are the identity, as the packed matrices
        self._bdfas = [dfa_from_regex_dfa(d) for d in self._dfas]
        used = {ord(c) for c in chars if ord(c) < 256}
        # a byte outside every alphabet stands for characters above U+00FF
        self._unknown_byte = next((b for b in range(256) if b not in used), None)
        self._sets = None
        if use_gpu:
            self._init_gpu()

    # ---- GPU ---------------------------------------------------------------------------------
    def _init_gpu(self):
        from .engine import DFASet
        if any(ord(c) > 255 for c in self._unified_alphabet):
            raise ValueError("the B200 engine reads bytes: alphabet characters must be <= U+00FF")
        self._sets = [DFASet(self._bdfas[i:i + _MAX_SET]) for i in range(0, len(self._bdfas), _MAX_SET)]

    def _encode(self, strings: Sequence) -> tuple[np.ndarray, np.ndarray]:
        from ._batching import pack_strings
        try:
            data, off, _ = pack_strings(strings, offset_dtype=np.int64)
        except UnicodeEncodeError:
            if self._unknown_byte is None:
                raise ValueError("a character above U+00FF cannot be matched: the patterns use "
                                 "every byte value") from None
            u = chr(self._unknown_byte)
            fixed = ["".join(ch if ord(ch) < 256 else u for ch in s) if isinstance(s, str) else s
                     for s in strings]
            data, off, _ = pack_strings(fixed, offset_dtype=np.int64)
        return data, off

    def _match_gpu(self, strings: Sequence):
        import torch
        data, off = self._encode(strings)
        dev = torch.device("cuda", torch.cuda.current_device())
        d_data = torch.from_numpy(data).to(dev)
        d_off = torch.from_numpy(off).to(dev)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record()
        accs = [s.run_all(d_data[:int(off[-1])], d_off)[1] for s in self._sets]
        ev[1].record()
        acc = torch.cat(accs, dim=0).cpu().numpy() if accs else np.zeros((0, len(strings)), np.uint8)
        kernel_ms = ev[0].elapsed_time(ev[1])
        return [[bool(x) for x in row[:len(strings)]] for row in acc], kernel_ms

    # ---- CPU: the byte-map walk, pattern by pattern ------------------------------------------
    def _match_cpu(self, strings: Sequence):
        data, off = self._encode(strings)
        out = []
        for bd in self._bdfas:
            N = bd.n_states
            t = bd.tmap.reshape(256, N)
            row = []
            for j in range(len(strings)):
                s = bd.start
                for c in data[off[j]:off[j + 1]]:
                    s = t[c, s]
                row.append(bool(bd.accept[s]))
            out.append(row)
        return out

    # ---- public API --------------------------------------------------------------------------
    def match_batch(self, strings: list[str]) -> list[list[bool]]:
        """Match all strings against all patterns: results[pattern_idx][string_idx]."""
        if len(strings) == 0:
            return [[] for _ in range(self._n_patterns)]
        if self._sets is not None:
            return self._match_gpu(strings)[0]
        return self._match_cpu(strings)

    def match_batch_timed(self, strings: list[str]) -> tuple[list[list[bool]], dict]:
        t0 = time.perf_counter()
        kernel_ms = None
        if len(strings) == 0:
            res = [[] for _ in range(self._n_patterns)]
        elif self._sets is not None:
            res, kernel_ms = self._match_gpu(strings)
        else:
            res = self._match_cpu(strings)
        timing = {"total_ms": (time.perf_counter() - t0) * 1e3, "n_strings": len(strings),
                  "n_patterns": self._n_patterns, "NP": self._NP}
        if kernel_ms is not None:
            timing["kernel_ms"] = kernel_ms
        return res, timing

    @property
    def config_info(self) -> dict:
        return {"n_patterns": self._n_patterns, "state_counts": list(self._state_counts),
                "offsets": [int(x) for x in self._offsets], "NP": self._NP,
                "unified_alphabet_size": len(self._unified_alphabet), "regexes": list(self._regexes),
                "backend": "gpu" if self._sets is not None else "cpu"}

    def close(self):
        for s in self._sets or []:
            s.close()
        self._sets = None
