"""k-gram precomposition over a DFA alphabet.

Drop-in for the reference module ``src/kgram.py``
(reference src/kgram.py:29-231). A k-gram ``(c0, ..., c_{k-1})`` has the
mixed-radix key ``c0*sigma^(k-1) + ... + c_{k-1}`` (first symbol most
significant); its entry is the monoid element (or int8 matrix) of the
k symbols composed newest-on-the-left.
"""

from __future__ import annotations

import itertools
from typing import Optional

import numpy as np

from .monoid import MonoidData
from .simulation import DFAMatrices, _matmul_int8


def auto_k(alphabet_size: int, max_entries: int = 65536) -> int:
    """Largest k >= 1 with alphabet_size**k <= max_entries (1 for sigma <= 1)."""
    if alphabet_size <= 1:
        return 1
    k = 1
    while alphabet_size ** (k + 1) <= max_entries:
        k += 1
    return k


def auto_k_for_gpu(alphabet_size: int, n_states: int,
                   max_table_bytes: int = 48_000_000) -> int:
    """Largest k >= 1 with alphabet_size**k * n_states**2 <= max_table_bytes."""
    if alphabet_size <= 1:
        return 1
    per = n_states * n_states
    k = 1
    while alphabet_size ** (k + 1) * per <= max_table_bytes:
        k += 1
    return k


class KGramTable:
    def __init__(self, k: int, alphabet: list, monoid_table: Optional[dict] = None,
                 matrix_table: Optional[dict] = None):
        self.k = k
        self.alphabet = alphabet
        self.sigma = len(alphabet)
        self.char_to_idx = {ch: i for i, ch in enumerate(alphabet)}
        self._monoid_table = monoid_table
        self._matrix_table = matrix_table

    def _gram_to_key(self, gram) -> int:
        key = 0
        for ch in gram:
            key = key * self.sigma + self.char_to_idx[ch]
        return key

    def lookup(self, gram) -> int:
        return self._monoid_table[self._gram_to_key(gram)]

    def lookup_matrix(self, gram) -> np.ndarray:
        return self._matrix_table[self._gram_to_key(gram)]


def precompute_kgrams(dm: DFAMatrices, k: int,
                      monoid: Optional[MonoidData] = None) -> KGramTable:
    alphabet = dm.alphabet
    sigma = len(alphabet)
    if monoid is not None:
        table: dict[int, int] = {}
        ct = monoid.compose_table
        sym = [monoid.char_to_monoid[ch] for ch in alphabet]
        for key, gram in enumerate(itertools.product(range(sigma), repeat=k)):
            acc = monoid.identity_idx
            for ci in gram:
                acc = int(ct[sym[ci], acc])
            table[key] = acc
        return KGramTable(k, alphabet, monoid_table=table)
    mats: dict[int, np.ndarray] = {}
    eye = dm.identity_matrix()
    for key, gram in enumerate(itertools.product(range(sigma), repeat=k)):
        acc = eye
        for ci in gram:
            acc = _matmul_int8(dm.matrix_stack[ci], acc)
        mats[key] = acc
    return KGramTable(k, alphabet, matrix_table=mats)


def simulate_kgram_monoid(kg: KGramTable, md: MonoidData, dm: DFAMatrices,
                          input_str: str) -> bool:
    """Whole k-grams via the table, the tail symbol by symbol
    (unknown tail symbols are the identity)."""
    acc = md.identity_idx
    ct = md.compose_table
    k = kg.k
    L = len(input_str)
    full = L - L % k
    for p in range(0, full, k):
        acc = int(ct[kg.lookup(input_str[p:p + k]), acc])
    for ch in input_str[full:]:
        acc = int(ct[md.char_to_monoid.get(ch, md.identity_idx), acc])
    return bool(md.accept_table[acc])
