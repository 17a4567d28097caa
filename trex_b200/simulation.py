"""DFA -> int8 transition matrices, CPU simulation back ends, and the byte
transition map consumed by the GPU kernels.

Drop-in for the reference module ``src/simulation.py``. Conventions kept from
it (reference src/simulation.py:20-100, 274-297):

* ``alphabet = sorted(dfa.alphabet)`` fixes the symbol -> index order;
* ``T[c][dst, src] = 1`` (column = source, row = destination), so
  ``next = T[c] @ cur``;
* states are padded to a multiple of 16 (or ``pad_to``) and padded states
  self-loop;
* ``precompute_tmap`` returns ``uint8 tmap[256 * N]`` with
  ``tmap[byte * N + s] = dst``; bytes outside the alphabet and padded states
  map to themselves (identity).
"""

from __future__ import annotations

from collections import defaultdict
from typing import Optional

import numpy as np

from .regex_to_dfa import DFA


class DFAMatrices:
    """A complete DFA as a stack of one-hot int8 transition matrices."""

    def __init__(self, dfa: DFA, pad_to: Optional[int] = None):
        self.dfa = dfa
        self.alphabet = sorted(dfa.alphabet)
        self.char_to_idx = {c: i for i, c in enumerate(self.alphabet)}
        self.n_states_raw = dfa.n_states
        if pad_to is not None:
            self.n_states = max(pad_to, dfa.n_states)
        else:
            self.n_states = -(-dfa.n_states // 16) * 16
        self._build_matrices()
        self._build_state_vectors()

    def _build_matrices(self) -> None:
        N, n_raw = self.n_states, self.n_states_raw
        pad = np.arange(n_raw, N)
        sigma = len(self.alphabet)
        if sigma == 0:
            # same failure as the reference (np.stack of an empty list)
            raise ValueError("need at least one array to stack")
        stack = np.zeros((sigma, N, N), dtype=np.int8)
        for ci, ch in enumerate(self.alphabet):
            for src in range(n_raw):
                dst = self.dfa.transitions.get(src, {}).get(ch)
                if dst is not None:
                    stack[ci, dst, src] = 1
            stack[ci, pad, pad] = 1
        self.matrix_stack = stack
        self.matrices = {ch: stack[ci] for ci, ch in enumerate(self.alphabet)}

    def _build_state_vectors(self) -> None:
        N = self.n_states
        self.start_vec = np.zeros(N, dtype=np.int8)
        self.start_vec[self.dfa.start] = 1
        self.accept_mask = np.zeros(N, dtype=np.int8)
        for s in self.dfa.accept_states:
            self.accept_mask[s] = 1

    def get_matrix_for_char(self, ch: str):
        return self.matrices.get(ch)

    def get_matrix_sequence(self, input_str: str) -> np.ndarray:
        """(L, N, N) matrices for ``input_str``; unknown symbols give identity."""
        N = self.n_states
        seq = np.empty((len(input_str), N, N), dtype=np.int8)
        eye = np.eye(N, dtype=np.int8)
        for i, ch in enumerate(input_str):
            ci = self.char_to_idx.get(ch)
            seq[i] = eye if ci is None else self.matrix_stack[ci]
        return seq

    def check_accept(self, state_vec: np.ndarray) -> bool:
        n = self.n_states_raw
        return bool(np.any(state_vec[:n] & self.accept_mask[:n]))

    def identity_matrix(self) -> np.ndarray:
        return np.eye(self.n_states, dtype=np.int8)

    # Extra helpers used by the engines (not in the reference API).
    def transition_table(self) -> np.ndarray:
        """``int32 [sigma, N]`` next-state table indexed by symbol index."""
        return np.argmax(self.matrix_stack, axis=1).astype(np.int32)


# --- CPU back ends ---------------------------------------------------------

def simulate_sequential(dfa: DFA, input_str: str) -> bool:
    """O(L) dictionary walk (the reference's CPU baseline)."""
    return dfa.simulate(input_str)


def simulate_matrix_sequential(dm: DFAMatrices, input_str: str) -> bool:
    """Matrix-vector walk; an unknown symbol rejects."""
    state = dm.start_vec.astype(np.int32)
    for ch in input_str:
        T = dm.get_matrix_for_char(ch)
        if T is None:
            return False
        state = T.astype(np.int32) @ state
    return dm.check_accept(state.astype(np.int8))


def _matmul_int8(A: np.ndarray, B: np.ndarray) -> np.ndarray:
    """int8 x int8 -> int32 product narrowed back to int8."""
    return (A.astype(np.int32) @ B.astype(np.int32)).astype(np.int8)


def _matmul_int32(A: np.ndarray, B: np.ndarray) -> np.ndarray:
    return A.astype(np.int32) @ B.astype(np.int32)


def prefix_scan_sequential(matrices: np.ndarray) -> np.ndarray:
    """Inclusive prefix products ``out[i] = M[i] @ ... @ M[0]``."""
    out = np.empty_like(matrices)
    if len(matrices) == 0:
        return out
    acc = matrices[0]
    out[0] = acc
    for i in range(1, len(matrices)):
        acc = _matmul_int8(matrices[i], acc)
        out[i] = acc
    return out


def prefix_scan_parallel(matrices: np.ndarray) -> np.ndarray:
    """Same result as :func:`prefix_scan_sequential` computed by log-depth
    doubling (each round composes element i with element i - stride)."""
    cur = matrices.copy()
    L = len(cur)
    stride = 1
    while stride < L:
        nxt = cur.copy()
        A = cur[stride:].astype(np.int32)
        B = cur[:-stride].astype(np.int32)
        nxt[stride:] = np.matmul(A, B).astype(np.int8)
        cur = nxt
        stride *= 2
    return cur


def simulate_prefix_scan(dm: DFAMatrices, input_str: str,
                         use_parallel: bool = True) -> bool:
    if not input_str:
        return dm.check_accept(dm.start_vec)
    seq = dm.get_matrix_sequence(input_str)
    pref = prefix_scan_parallel(seq) if use_parallel else prefix_scan_sequential(seq)
    final = pref[-1].astype(np.int32) @ dm.start_vec.astype(np.int32)
    return dm.check_accept(final.astype(np.int8))


def simulate_batch_sequential(dfa: DFA, strings: list) -> list:
    return [dfa.simulate(s) for s in strings]


def simulate_batch_matrix(dm: DFAMatrices, strings: list) -> list:
    """Batched matrix evolution: strings of equal length share one state
    matrix; columns with the same symbol at a position share one product.
    An unknown symbol zeroes the column (the string then rejects)."""
    results = [False] * len(strings)
    by_len: dict[int, list[int]] = defaultdict(list)
    for i, s in enumerate(strings):
        by_len[len(s)].append(i)
    start = dm.start_vec.astype(np.int32)
    for L, idx in by_len.items():
        if L == 0:
            acc = dm.check_accept(dm.start_vec)
            for i in idx:
                results[i] = acc
            continue
        S = np.repeat(start[:, None], len(idx), axis=1)
        for p in range(L):
            groups: dict[str, list[int]] = defaultdict(list)
            for col, i in enumerate(idx):
                groups[strings[i][p]].append(col)
            new = np.zeros_like(S)
            for ch, cols in groups.items():
                T = dm.get_matrix_for_char(ch)
                if T is not None:
                    new[:, cols] = T.astype(np.int32) @ S[:, cols]
            S = new
        for col, i in enumerate(idx):
            results[i] = dm.check_accept(S[:, col].astype(np.int8))
    return results


def precompute_tmap(dm: DFAMatrices) -> np.ndarray:
    """``uint8 tmap[256 * N]``, ``tmap[byte * N + s]`` = next state.

    Symbols are single characters whose code point is the byte value; bytes
    outside the alphabet and padded states are identity."""
    N = dm.n_states
    table = np.tile(np.arange(N, dtype=np.uint8), (256, 1))
    nxt = dm.transition_table()  # [sigma, N]
    for ci, ch in enumerate(dm.alphabet):
        b = ord(ch)
        if b > 255:
            raise ValueError(f"symbol {ch!r} does not fit in one byte")
        table[b, :dm.n_states_raw] = nxt[ci, :dm.n_states_raw]
    return table.reshape(-1)
