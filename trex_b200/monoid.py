"""Transition monoid of a DFA and the compose tables derived from it.

Drop-in for the reference module ``src/monoid.py``
(reference src/monoid.py:30-287). Semantics kept:

* the monoid holds the identity plus every product of per-symbol matrices;
  :func:`compute_monoid` returns ``None`` once it exceeds ``max_size``;
* ``compose_table[i, j]`` is the index of ``elements[i] @ elements[j]``
  (element ``i`` is applied after ``j``); the walk is
  ``acc = compose_table[c_new, acc]``;
* symbols outside the alphabet act as the identity.

Elements are enumerated as state-transformation vectors instead of int8
matrix products (a DFA matrix has one-hot columns, so the product is
function composition); ``elements`` is materialised as int8 matrices at the
end. The enumeration order is breadth-first with the identity at index 0 and
the alphabet symbols next, so indices are deterministic.
"""

from __future__ import annotations

import math
from collections import deque
from dataclasses import dataclass
from typing import Optional

import numpy as np

from .simulation import DFAMatrices


@dataclass
class MonoidData:
    elements: list               # list of (N, N) int8 arrays
    compose_table: np.ndarray    # (M, M) uint16
    char_to_monoid: dict         # symbol -> element index
    accept_table: np.ndarray     # (M,) bool
    identity_idx: int
    size: int


def _as_function(mat: np.ndarray) -> tuple:
    """One-hot-column matrix -> tuple f with f[src] = dst (N for an empty column)."""
    N = mat.shape[0]
    has = mat.any(axis=0)
    dst = np.argmax(mat, axis=0)
    return tuple(int(d) if h else N for d, h in zip(dst, has))


def compute_monoid(dm: DFAMatrices, max_size: int = 65536) -> Optional[MonoidData]:
    N = dm.n_states
    ident = tuple(range(N))
    index: dict[tuple, int] = {}
    funcs: list[tuple] = []

    def intern(f: tuple) -> int:
        i = index.get(f)
        if i is None:
            i = index[f] = len(funcs)
            funcs.append(f)
        return i

    identity_idx = intern(ident)
    gens = []
    char_to_monoid = {}
    for ch in dm.alphabet:
        g = intern(_as_function(dm.matrices[ch]))
        char_to_monoid[ch] = g
        gens.append(g)
    if len(funcs) > max_size:
        return None

    def apply(f_after: tuple, f_before: tuple) -> tuple:
        # (f_after o f_before)[s] = f_after[f_before[s]]; the sink N stays N.
        return tuple(f_after[t] if t < N else N for t in f_before)

    # Right-multiplication closure from the identity: every product of
    # generators is reachable as g_k o ... o g_1.
    queue = deque(range(len(funcs)))
    while queue:
        i = queue.popleft()
        fi = funcs[i]
        for g in gens:
            before = len(funcs)
            intern(apply(funcs[g], fi))
            if len(funcs) > before:
                if len(funcs) > max_size:
                    return None
                queue.append(len(funcs) - 1)

    M = len(funcs)
    F = np.array(funcs, dtype=np.int64)                       # [M, N], sink = N
    Fx = np.concatenate([F, np.full((M, 1), N, dtype=np.int64)], axis=1)
    compose = np.empty((M, M), dtype=np.uint16)
    lookup = index
    for i in range(M):
        prod = Fx[i][F]                                       # [M, N]: f_i o f_j
        for j in range(M):
            compose[i, j] = lookup[tuple(prod[j].tolist())]

    elements = []
    for f in funcs:
        E = np.zeros((N, N), dtype=np.int8)
        for src, dst in enumerate(f):
            if dst < N:
                E[dst, src] = 1
        elements.append(E)

    start = int(np.argmax(dm.start_vec))
    accept = np.zeros(M, dtype=bool)
    for k, f in enumerate(funcs):
        d = f[start]
        accept[k] = bool(d < dm.n_states_raw and dm.accept_mask[d])
    return MonoidData(elements=elements, compose_table=compose,
                      char_to_monoid=char_to_monoid, accept_table=accept,
                      identity_idx=identity_idx, size=M)


def simulate_monoid(md: MonoidData, dm: DFAMatrices, input_str: str) -> bool:
    acc = md.identity_idx
    ct = md.compose_table
    c2m = md.char_to_monoid
    for ch in input_str:
        acc = int(ct[c2m.get(ch, md.identity_idx), acc])
    return bool(md.accept_table[acc])


def kgram_width_for_bytes(sigma: int) -> int:
    """Largest k with sigma**k <= 256 (1 when sigma < 2)."""
    if sigma < 2:
        return 1
    k = max(int(math.log(256) / math.log(sigma)), 1)
    while sigma ** k > 256:
        k -= 1
    return k


def precompute_batch_tables(md: MonoidData, dm: DFAMatrices) -> dict:
    """uint8 tables for the monoid batch engine (reference
    src/monoid.py:195-287): ``char_compose [M*(sigma+1)]`` whose last column
    is the identity, ``raw_char_map[256]`` (unknown byte -> sigma),
    ``accept[M]``, ``monoid_compose[M*M]``, ``fused_compose[M*256]`` and the
    k-gram table ``kgram_compose[M*sigma**k]`` whose key reads the first
    symbol as the most significant digit."""
    M = md.size
    if M > 255:
        raise ValueError(f"Monoid size {M} exceeds uint8 limit (255)")
    sigma = len(dm.alphabet)
    sigma_ext = sigma + 1
    ct = md.compose_table

    sym_elem = np.array([md.char_to_monoid[ch] for ch in dm.alphabet], dtype=np.int64)
    char_compose = np.empty((M, sigma_ext), dtype=np.uint8)
    if sigma:
        char_compose[:, :sigma] = ct[sym_elem][:, :M].T      # [m, c] = ct[sym[c], m]
    char_compose[:, sigma] = np.arange(M)

    raw_char_map = np.full(256, sigma, dtype=np.uint8)
    for ci, ch in enumerate(dm.alphabet):
        raw_char_map[ord(ch)] = ci

    fused = char_compose[:, raw_char_map]                     # [M, 256]

    k = kgram_width_for_bytes(sigma)
    sigma_k = sigma ** k if sigma >= 2 else 1
    kgram = None
    if k >= 2:
        digits = np.array([[(g // sigma ** (k - 1 - p)) % sigma for p in range(k)]
                           for g in range(sigma_k)], dtype=np.int64)
        cur = np.repeat(np.arange(M)[:, None], sigma_k, axis=1)   # [M, sigma_k]
        for p in range(k):
            cur = char_compose[cur, digits[None, :, p]].astype(np.int64)
        kgram = np.ascontiguousarray(cur.astype(np.uint8).reshape(-1))

    return {
        'char_compose': np.ascontiguousarray(char_compose.reshape(-1)),
        'raw_char_map': raw_char_map,
        'accept': np.ascontiguousarray(md.accept_table.astype(np.uint8)),
        'monoid_compose': np.ascontiguousarray(ct.astype(np.uint8).reshape(-1)),
        'fused_compose': np.ascontiguousarray(fused.reshape(-1)),
        'kgram_compose': kgram,
        'M': M,
        'sigma': sigma,
        'sigma_ext': sigma_ext,
        'sigma_k': sigma_k,
        'kgram_k': k,
        'identity_idx': md.identity_idx,
    }
