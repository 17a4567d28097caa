"""NFA -> Boolean transition matrices with the epsilon closure folded in.

Drop-in for the reference module ``src/nfa_matrices.py``
(reference src/nfa_matrices.py:40-157):

* ``T[c][dst, src] = 1`` iff ``dst`` is in the epsilon closure of the states
  reached from ``src`` by one ``c`` step;
* the start vector is the epsilon closure of the NFA start state;
* :func:`simulate_nfa` evaluates ``state = min(T[c] @ state, 1)`` per symbol
  and rejects on a symbol outside the alphabet.

:func:`nfa_from_matrices` builds an ``NFAMatrices`` directly from dense
matrices (random automata, the GPU engine's native input).
"""

from __future__ import annotations

from typing import Optional

import numpy as np

from .regex_to_dfa import EPSILON, NFA, RegexParser


def _epsilon_closure_set(nfa: NFA, states) -> set[int]:
    seen = set(states)
    todo = list(seen)
    while todo:
        s = todo.pop()
        for t in nfa.states[s].transitions.get(EPSILON, ()):
            if t not in seen:
                seen.add(t)
                todo.append(t)
    return seen


class NFAMatrices:
    """Boolean int8 matrices of an epsilon-NFA, one per alphabet symbol."""

    def __init__(self, nfa: NFA, pad_to: Optional[int] = None):
        self.nfa = nfa
        self.alphabet = sorted(nfa.alphabet)
        self.char_to_idx = {c: i for i, c in enumerate(self.alphabet)}
        self.n_states_raw = len(nfa.states)
        if pad_to is not None:
            self.n_states = max(pad_to, self.n_states_raw)
        else:
            self.n_states = -(-self.n_states_raw // 16) * 16
        self._build_matrices()
        self._build_state_vectors()

    def _build_matrices(self) -> None:
        N = self.n_states
        if not self.alphabet:
            # same failure as the reference (np.stack of an empty list)
            raise ValueError("need at least one array to stack")
        stack = np.zeros((len(self.alphabet), N, N), dtype=np.int8)
        closure_cache: dict[frozenset, set[int]] = {}
        for ci, ch in enumerate(self.alphabet):
            for src, st in self.nfa.states.items():
                direct = st.transitions.get(ch)
                if not direct:
                    continue
                key = frozenset(direct)
                reach = closure_cache.get(key)
                if reach is None:
                    reach = closure_cache[key] = _epsilon_closure_set(self.nfa, key)
                for dst in reach:
                    if dst < N and src < N:
                        stack[ci, dst, src] = 1
        self.matrix_stack = stack
        self.matrices = {ch: stack[ci] for ci, ch in enumerate(self.alphabet)}

    def _build_state_vectors(self) -> None:
        N = self.n_states
        self.start_vec = np.zeros(N, dtype=np.int8)
        for s in _epsilon_closure_set(self.nfa, {self.nfa.start}):
            if s < N:
                self.start_vec[s] = 1
        self.accept_mask = np.zeros(N, dtype=np.int8)
        for sid, st in self.nfa.states.items():
            if st.is_accept and sid < N:
                self.accept_mask[sid] = 1

    def check_accept(self, state_vec: np.ndarray) -> bool:
        n = self.n_states_raw
        return bool(np.any(state_vec[:n].astype(np.int8) & self.accept_mask[:n]))


def compile_nfa_matrices(regex: str, pad_to: Optional[int] = None) -> NFAMatrices:
    return NFAMatrices(RegexParser(regex).parse(), pad_to=pad_to)


def simulate_nfa(nm: NFAMatrices, input_str: str) -> bool:
    """Boolean matrix-vector walk; a symbol outside the alphabet rejects."""
    if not input_str:
        return nm.check_accept(nm.start_vec)
    state = nm.start_vec.astype(np.int32)
    for ch in input_str:
        ci = nm.char_to_idx.get(ch)
        if ci is None:
            return False
        state = np.minimum(nm.matrix_stack[ci].astype(np.int32) @ state, 1)
    return nm.check_accept(state.astype(np.int8))


def nfa_from_matrices(T: np.ndarray, start_vec: np.ndarray, accept_mask: np.ndarray,
                      alphabet: Optional[list] = None) -> NFAMatrices:
    """Wrap dense Boolean matrices ``T[sigma, N, N]`` (row = dst, col = src) as
    an :class:`NFAMatrices`. The default alphabet is ``chr(0) .. chr(sigma-1)``,
    i.e. symbol index == byte value. No epsilon moves are added."""
    T = np.asarray(T)
    sigma, N, _ = T.shape
    if alphabet is None:
        alphabet = [chr(i) for i in range(sigma)]
    nfa = NFA()
    for _ in range(N):
        nfa.new_state()
    nfa.start = int(np.flatnonzero(start_vec)[0]) if np.any(start_vec) else 0
    for ci, ch in enumerate(alphabet):
        dst_idx, src_idx = np.nonzero(T[ci])
        for d, s in zip(dst_idx.tolist(), src_idx.tolist()):
            nfa.add_trans(s, ch, d)
        nfa.alphabet.add(ch)
    for s in np.flatnonzero(accept_mask).tolist():
        nfa.states[s].is_accept = True
    nm = NFAMatrices.__new__(NFAMatrices)
    nm.nfa = nfa
    nm.alphabet = sorted(alphabet)
    nm.char_to_idx = {c: i for i, c in enumerate(nm.alphabet)}
    nm.n_states_raw = N
    nm.n_states = N
    order = [alphabet.index(c) for c in nm.alphabet]
    nm.matrix_stack = (np.asarray(T, dtype=np.int8)[order] != 0).astype(np.int8)
    nm.matrices = {ch: nm.matrix_stack[i] for i, ch in enumerate(nm.alphabet)}
    nm.start_vec = (np.asarray(start_vec) != 0).astype(np.int8)
    nm.accept_mask = (np.asarray(accept_mask) != 0).astype(np.int8)
    return nm
