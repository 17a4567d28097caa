"""OptimizedEngine: the reference's unified matching API over the B200 kernels.

Drop-in for ``src/optimized_engine.py`` (reference src/optimized_engine.py:29-425):

* ``OptimizedEngine(regex, config=None, dfa_state_cap=64, monoid_cap=65536)``
  with the reference's config strings None, "monoid", "monoid+kgram",
  "baseline", "nfa", "monoid+gpu", "batched+gpu", "kgram+gpu",
  "monoid_batch+gpu", "prefix+gpu", "fp16_tc+gpu"; anything else raises
  ``ValueError`` (:79-111);
* the form documented in the reference README
  (``OptimizedEngine(pattern=..., config="auto").match(strings)``), which the
  reference class does not implement;
* a prebuilt automaton instead of a regex: a ``DFA``, ``DFAMatrices``,
  ``NFAMatrices`` or byte-level ``ByteDFA`` (random benchmark automata are not
  regexes);
* ``match_batch`` -> list[bool], ``match_batch_timed`` -> (list[bool], dict)
  with ``kernel_ms``/``total_ms`` for GPU configs and
  ``total_seconds``/``per_string_seconds``/``n_strings`` for CPU configs
  (:376-425), ``config_info`` with the keys representation, scan_backend,
  alphabet_size, kgram_k, selection_reason (:327-355).

Backends. "auto" (and None) picks a B200 engine: the ragged DFA kernel for a
DFA with at most ``dfa_state_cap`` states (<= 256), else the bit-parallel NFA
kernel for an NFA with at most 64 states; with no engine that fits it raises
``ValueError`` and names the CPU configs -- there is no silent CPU fallback,
and a missing library or GPU raises too. "baseline", "monoid",
"monoid+kgram" and "nfa" are the reference's CPU algorithms and run only when
asked for. "monoid+gpu", "monoid_batch+gpu" and "prefix+gpu" go through this
package's drop-in bridges (the reference's byte-map semantics: a character
outside the alphabet is the identity). "batched+gpu", "kgram+gpu" and
"fp16_tc+gpu" name reference WMMA engines that this package does not rebuild;
they run the ragged DFA kernel and say so in ``selection_reason``.

String semantics of the B200 DFA engine follow ``DFA.simulate``
(reference src/regex_to_dfa.py:224-233): a character outside the alphabet
sends the walk to the dead state, or rejects when there is none. The NFA
engine follows ``simulate_nfa`` (src/nfa_matrices.py:150-152): an unknown
character rejects.
"""

from __future__ import annotations

import time
from typing import Optional, Sequence, Union

import numpy as np

from .kgram import auto_k, precompute_kgrams, simulate_kgram_monoid
from .monoid import compute_monoid, simulate_monoid
from .nfa_matrices import NFAMatrices, compile_nfa_matrices, simulate_nfa
from .regex_to_dfa import DFA, compile_regex
from .simulation import DFAMatrices, simulate_sequential
from .workloads import ByteDFA

_CPU_CONFIGS = ("baseline", "monoid", "monoid+kgram", "nfa")
_REF_GPU_CONFIGS = ("monoid+gpu", "batched+gpu", "kgram+gpu", "monoid_batch+gpu", "prefix+gpu",
                    "fp16_tc+gpu")
_OWN_GPU_CONFIGS = ("dfa+gpu", "nfa+gpu")
_ALL_CONFIGS = (None, "auto") + _CPU_CONFIGS + _REF_GPU_CONFIGS + _OWN_GPU_CONFIGS


class _DfaEngine:
    """A DFA on the B200 ragged batch kernel (trex_dfa_batch_host)."""

    def __init__(self, bdfa: ByteDFA, unknown_byte: Optional[int], kgram: int = 1):
        from .engine import DFASet
        self.bdfa = bdfa
        self.unknown_byte = unknown_byte
        self.set = DFASet([bdfa], kgram=kgram)
        self.kgram = self.set.get_kgram(0)

    def _pack(self, strings):
        from ._batching import pack_strings
        try:
            data, off, _ = pack_strings(strings, offset_dtype=np.int64)
        except UnicodeEncodeError:
            if self.unknown_byte is None:
                raise ValueError("a character above U+00FF cannot be matched: the alphabet already "
                                 "uses every byte value") from None
            u = chr(self.unknown_byte)
            fixed = ["".join(ch if ord(ch) < 256 else u for ch in s) if isinstance(s, str) else s
                     for s in strings]
            data, off, _ = pack_strings(fixed, offset_dtype=np.int64)
        return data, off

    def run(self, strings):
        data, off = self._pack(strings)
        _, acc, kms, tms = self.set.run_host(data, off)
        return [bool(a) for a in acc[:len(strings)]], kms, tms

    def close(self):
        self.set.close()


def _byte_dfa_from_dfa(dfa: DFA) -> tuple[ByteDFA, Optional[int]]:
    """Byte transition map with ``DFA.simulate`` semantics: a byte whose
    character is not in the alphabet (or has no transition) goes to the dead
    state, or to an added rejecting sink when the DFA has none."""
    if any(ord(c) > 255 for c in dfa.alphabet):
        raise ValueError("the B200 DFA engine reads bytes: alphabet characters must be <= U+00FF; "
                         "use a CPU config")
    N = dfa.n_states
    dead = dfa.dead_state
    need_sink = dead is None and (len(dfa.alphabet) < 256 or any(
        len(dfa.transitions.get(s, {})) < len(dfa.alphabet) for s in range(N)))
    if need_sink:
        dead = N
        N += 1
    if N > 256:
        raise ValueError(f"the B200 DFA engine takes at most 256 states (this DFA needs {N})")
    tmap = np.empty((256, N), dtype=np.uint8)
    tmap[:, :] = dead
    for s in range(dfa.n_states):
        for ch, d in dfa.transitions.get(s, {}).items():
            tmap[ord(ch), s] = d
    if need_sink:
        tmap[:, dead] = dead
    accept = np.zeros(N, dtype=np.uint8)
    for s in dfa.accept_states:
        accept[s] = 1
    used = {ord(c) for c in dfa.alphabet}
    unknown = next((b for b in range(256) if b not in used), None)
    return ByteDFA(n_states=N, tmap=np.ascontiguousarray(tmap.reshape(-1)), accept=accept,
                   start=dfa.start), unknown


class OptimizedEngine:
    """Unified matching engine (see the module docstring)."""

    def __init__(self, regex: Union[str, DFA, DFAMatrices, NFAMatrices, ByteDFA, None] = None,
                 config: Optional[str] = None, dfa_state_cap: int = 64, monoid_cap: int = 65536,
                 *, pattern: Union[str, DFA, DFAMatrices, NFAMatrices, ByteDFA, None] = None):
        if regex is None:
            regex = pattern
        elif pattern is not None:
            raise TypeError("give the pattern once: positionally or as pattern=")
        if regex is None:
            raise TypeError("OptimizedEngine needs a regex (or a prebuilt automaton)")
        if config not in _ALL_CONFIGS:
            raise ValueError(f"Unknown config: {config!r}. "
                             f"Choose from None, 'auto', 'monoid', 'monoid+kgram', 'baseline', 'nfa', "
                             f"'monoid+gpu', 'batched+gpu', 'kgram+gpu', 'monoid_batch+gpu', "
                             f"'prefix+gpu', 'fp16_tc+gpu', 'dfa+gpu', 'nfa+gpu'.")
        self._source = regex
        self._regex = regex if isinstance(regex, str) else None
        self._config = config
        self._dfa_state_cap = dfa_state_cap
        self._monoid_cap = monoid_cap
        self._dfa: Optional[DFA] = None
        self._dm: Optional[DFAMatrices] = None
        self._md = None
        self._kg = None
        self._nm: Optional[NFAMatrices] = None
        self._bdfa: Optional[ByteDFA] = None
        self._gpu = None          # engine object with run(strings) -> (results, kernel_ms, total_ms)
        self._ref_gpu = None      # reference-style bridge engine (simulate_batch[_timed])
        self._representation = None
        self._scan_backend = None
        self._selection_reason = None
        self._kgram_k = None
        if isinstance(regex, ByteDFA):
            self._bdfa = regex
        elif isinstance(regex, DFA):
            self._dfa = regex
        elif isinstance(regex, DFAMatrices):
            self._dm = regex
            self._dfa = regex.dfa
        elif isinstance(regex, NFAMatrices):
            self._nm = regex
        elif not isinstance(regex, str):
            raise TypeError(f"unsupported pattern type {type(regex).__name__}")
        if config in (None, "auto"):
            self._auto_select()
        elif config in _CPU_CONFIGS:
            self._setup_cpu(config)
        else:
            self._setup_gpu(config)

    # ---- construction --------------------------------------------------------------------------
    def _build_dfa(self):
        if self._dfa is None and self._bdfa is None:
            if self._regex is None:
                raise ValueError("this pattern has no DFA (an NFAMatrices was given)")
            self._dfa = compile_regex(self._regex)
        if self._dm is None and self._dfa is not None:
            self._dm = DFAMatrices(self._dfa)

    def _build_nfa(self):
        if self._nm is None:
            if self._regex is None:
                raise ValueError("this pattern has no NFA form (give the regex or NFAMatrices)")
            self._nm = compile_nfa_matrices(self._regex)

    def _dfa_states(self) -> int:
        return self._bdfa.n_states if self._bdfa is not None else self._dfa.n_states

    def _setup_gpu_dfa(self, backend: str, reason: str, kgram: int = 1):
        if self._bdfa is None:
            self._bdfa, unknown = _byte_dfa_from_dfa(self._dfa)
        else:
            unknown = None
        self._gpu = _DfaEngine(self._bdfa, unknown, kgram)
        self._representation = "dfa"
        self._scan_backend = backend
        self._kgram_k = self._gpu.kgram
        self._selection_reason = reason

    def _setup_gpu_nfa(self, reason: str):
        from .gpu_bridge_nfa import NFAGPUSimulator
        self._build_nfa()
        self._ref_gpu = NFAGPUSimulator().create_engine(self._nm)
        self._representation = "nfa"
        self._scan_backend = "nfa+gpu"
        self._selection_reason = reason

    def _auto_select(self):
        if self._nm is not None and self._dfa is None and self._bdfa is None:
            n = self._nm.n_states_raw
            if n > 64:
                raise ValueError(f"no B200 engine for an NFA of {n} states (<= 64); use config='nfa'")
            self._setup_gpu_nfa(f"NFA with {n} states; bit-parallel NFA kernel")
            return
        self._build_dfa()
        n = self._dfa_states()
        if n <= min(self._dfa_state_cap, 256) or (self._regex is None and n <= 256):
            self._setup_gpu_dfa("dfa+gpu", f"DFA has {n} states; B200 ragged batch DFA kernel")
            return
        if self._regex is not None:
            self._build_nfa()
            m = self._nm.n_states_raw
            if m <= 64:
                self._setup_gpu_nfa(f"DFA has {n} states > cap {self._dfa_state_cap}; NFA has {m} "
                                    f"states; bit-parallel NFA kernel")
                return
            if n <= 256:
                self._setup_gpu_dfa("dfa+gpu", f"DFA has {n} states (NFA {m} > 64); B200 ragged "
                                               f"batch DFA kernel")
                return
        raise ValueError(f"no B200 engine fits (DFA {n} states > 256, NFA > 64 states); choose a CPU "
                         f"config explicitly: 'baseline', 'monoid', 'monoid+kgram' or 'nfa'")

    def _setup_cpu(self, config: str):
        if config == "nfa":
            self._build_nfa()
            self._representation = "nfa"
            self._scan_backend = "nfa"
            self._selection_reason = "forced config='nfa'"
            return
        self._build_dfa()
        if self._dfa is None:
            raise ValueError("CPU DFA configs need a regex, DFA or DFAMatrices")
        self._representation = "dfa"
        if config == "baseline":
            self._scan_backend = "sequential"
            self._selection_reason = "forced config='baseline'"
            return
        self._md = compute_monoid(self._dm, max_size=self._monoid_cap)
        if self._md is None:
            raise RuntimeError("compute_monoid returned None (monoid too large). "
                               "Increase monoid_cap or use a different config.")
        if config == "monoid":
            self._scan_backend = "monoid"
            self._selection_reason = "forced config='monoid'"
        else:
            k = auto_k(len(self._dfa.alphabet))
            self._kg = precompute_kgrams(self._dm, k, monoid=self._md)
            self._kgram_k = k
            self._scan_backend = "monoid+kgram"
            self._selection_reason = "forced config='monoid+kgram'"

    def _setup_gpu(self, config: str):
        if config == "nfa+gpu":
            self._setup_gpu_nfa("forced config='nfa+gpu'")
            return
        self._build_dfa()
        if config == "dfa+gpu":
            self._setup_gpu_dfa("dfa+gpu", "forced config='dfa+gpu'")
            return
        if self._dfa is None:
            raise ValueError(f"config {config!r} needs a regex, DFA or DFAMatrices")
        if config in ("monoid+gpu", "monoid_batch+gpu"):
            self._md = compute_monoid(self._dm, max_size=self._monoid_cap)
            if self._md is None:
                raise RuntimeError("compute_monoid returned None (monoid too large). "
                                   "Increase monoid_cap or use a different config.")
            if config == "monoid+gpu":
                from .gpu_bridge_monoid import MonoidGPUSimulator
                self._ref_gpu = MonoidGPUSimulator().create_engine(self._md, self._dm)
                self._selection_reason = "GPU monoid scan"
            else:
                if self._md.size > 255:
                    raise RuntimeError(f"Monoid size {self._md.size} > 255; use monoid+gpu instead")
                from .gpu_bridge_monoid_batch import MonoidBatchGPUSimulator
                self._ref_gpu = MonoidBatchGPUSimulator().create_engine(
                    self._md, self._dm, max_total_chars=1 << 29, max_batch=1 << 19)
                self._selection_reason = (f"GPU monoid batch (M={self._md.size}, "
                                          f"sigma={len(self._dm.alphabet)})")
        elif config == "prefix+gpu":
            from .gpu_bridge_prefix_compose import PrefixComposeGPUSimulator
            self._ref_gpu = PrefixComposeGPUSimulator().create_engine(
                self._dm, max_total_chars=1 << 29, max_batch=1 << 19)
            self._selection_reason = f"GPU prefix compose (N={self._dm.n_states})"
        elif config == "kgram+gpu":   # K-gram walking, the largest width the automaton allows
            self._setup_gpu_dfa(config, "config='kgram+gpu': B200 ragged batch DFA kernel with K-gram "
                                        "walking (largest K the alphabet allows; K=1 when none)", kgram=0)
            return
        else:   # batched+gpu, fp16_tc+gpu: the reference's WMMA engines
            self._setup_gpu_dfa(config, f"config={config!r}: the reference's WMMA engine is not "
                                        f"rebuilt; B200 ragged batch DFA kernel (byte map, K=1)")
            return
        self._representation = "dfa"
        self._scan_backend = config

    # ---- public API ----------------------------------------------------------------------------
    @property
    def config_info(self) -> dict:
        """representation, scan_backend, alphabet_size, kgram_k, selection_reason
        (+ dfa_states, monoid_size, nfa_states when known)."""
        info: dict = {
            "representation": self._representation,
            "scan_backend": self._scan_backend,
            "kgram_k": self._kgram_k,
            "selection_reason": self._selection_reason,
        }
        if self._dfa is not None:
            info["alphabet_size"] = len(self._dfa.alphabet)
            info["dfa_states"] = self._dfa.n_states
        elif self._bdfa is not None:
            info["alphabet_size"] = int(len(self._bdfa.symbols))
            info["dfa_states"] = self._bdfa.n_states
        elif self._nm is not None:
            info["alphabet_size"] = len(self._nm.alphabet)
        if self._md is not None:
            info["monoid_size"] = self._md.size
        if self._nm is not None:
            info["nfa_states"] = self._nm.n_states_raw
        return info

    def _match_cpu(self, strings) -> list:
        strs = [s.decode("latin-1") if isinstance(s, (bytes, bytearray)) else s for s in strings]
        if self._scan_backend == "nfa":
            return [simulate_nfa(self._nm, s) for s in strs]
        if self._scan_backend == "monoid+kgram":
            return [simulate_kgram_monoid(self._kg, self._md, self._dm, s) for s in strs]
        if self._scan_backend == "monoid":
            return [simulate_monoid(self._md, self._dm, s) for s in strs]
        return [simulate_sequential(self._dfa, s) for s in strs]

    def _run_gpu(self, strings):
        if self._gpu is not None:
            return self._gpu.run(strings)
        res, kms, tms = self._ref_gpu.simulate_batch_timed(list(strings))
        return [bool(r) for r in res], kms, tms

    def match_batch(self, strings: Sequence) -> list:
        """Match a list of strings (str or bytes). Returns list[bool]."""
        strings = list(strings)
        if not strings:
            return []
        if self._gpu is None and self._ref_gpu is None:
            return self._match_cpu(strings)
        return self._run_gpu(strings)[0]

    def match(self, strings):
        """The documented form: a list of strings -> list[bool], one string -> bool."""
        if isinstance(strings, (str, bytes, bytearray)):
            return self.match_batch([strings])[0]
        return self.match_batch(strings)

    def match_batch_timed(self, strings: Sequence) -> tuple:
        """(results, timing): GPU configs give kernel_ms and total_ms, CPU
        configs total_seconds, per_string_seconds and n_strings."""
        strings = list(strings)
        if self._gpu is not None or self._ref_gpu is not None:
            if not strings:
                return [], {"kernel_ms": 0.0, "total_ms": 0.0}
            res, kms, tms = self._run_gpu(strings)
            return res, {"kernel_ms": kms, "total_ms": tms}
        t0 = time.perf_counter()
        results = self.match_batch(strings)
        elapsed = time.perf_counter() - t0
        return results, {"total_seconds": elapsed,
                         "per_string_seconds": elapsed / len(strings) if strings else 0.0,
                         "n_strings": len(strings)}

    def close(self):
        if self._gpu is not None:
            self._gpu.close()
            self._gpu = None
        if self._ref_gpu is not None and hasattr(self._ref_gpu, "destroy"):
            self._ref_gpu.destroy()
            self._ref_gpu = None
