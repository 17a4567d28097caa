"""Seeded synthetic automata and inputs for the five benchmark workloads.

All generators use ``numpy.random.default_rng(seed)`` so that host-side data
is reproducible; the large inputs can also be drawn on the device with a
seeded ``torch.Generator`` (same distributions, different stream).

Workloads (sizes are the full benchmark sizes; every generator takes
smaller sizes for tests):
  * plain DFA: N=16 over the 4 bytes "ACGT", 4096 strings x 1024 bytes;
  * ragged DFA batch: 16 DFAs (5 x N=8, 5 x N=12, 6 x N=16) over all 256
    bytes, 1M strings with log-normal lengths (median 2048, sigma 1.18,
    clipped to [16, 65536]); 10% of the strings use the sub-alphabet "ACGT";
    string i uses DFA i mod 16;
  * long-string scan: N=16 over 256 bytes, 8 strings x 256 MiB;
  * Boolean NFA: N=64, 20 symbols (bytes 0..19), per-symbol edge density
    0.05, start {0}, ~25% accepting, 256K strings x 4096;
  * probabilistic NFA: N=64, 20 symbols, rows T[c][dst, :] ~ Dirichlet(0.5)
    x 0.9 then ~30% of entries kept (no renormalisation), start e0,
    accept all-ones, 64K sequences x 2048.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .regex_to_dfa import DFA

ACGT = np.frombuffer(b"ACGT", dtype=np.uint8)


@dataclass
class ByteDFA:
    """A DFA over raw bytes: ``tmap[byte * n_states + s]`` = next state."""
    n_states: int
    tmap: np.ndarray            # uint8 [256 * n_states]
    accept: np.ndarray          # uint8 [n_states]
    start: int = 0
    symbols: np.ndarray = field(default_factory=lambda: np.arange(256, dtype=np.uint8))

    def to_dfa(self) -> DFA:
        """The same automaton as a reference-style :class:`DFA` whose symbols
        are ``chr(byte)``."""
        N = self.n_states
        t = self.tmap.reshape(256, N)
        trans = {s: {chr(int(b)): int(t[b, s]) for b in self.symbols} for s in range(N)}
        return DFA(n_states=N, start=self.start,
                   accept_states={int(s) for s in np.flatnonzero(self.accept)},
                   transitions=trans, alphabet={chr(int(b)) for b in self.symbols})


def random_dfa(n_states: int, symbols, rng: np.random.Generator,
               accept_frac: float = 0.25) -> ByteDFA:
    """Uniform random next state per (state, symbol); bytes outside
    ``symbols`` are the identity; start 0; round(accept_frac*N) (>= 1)
    accepting states chosen uniformly."""
    symbols = np.asarray(symbols, dtype=np.uint8)
    N = n_states
    t = np.tile(np.arange(N, dtype=np.uint8), (256, 1))
    t[symbols, :] = rng.integers(0, N, size=(len(symbols), N), dtype=np.uint8)
    acc = np.zeros(N, dtype=np.uint8)
    k = max(1, int(round(accept_frac * N)))
    acc[rng.choice(N, size=k, replace=False)] = 1
    return ByteDFA(n_states=N, tmap=np.ascontiguousarray(t.reshape(-1)), accept=acc,
                   start=0, symbols=symbols)


def dfa_from_regex_dfa(dfa: DFA, n_states=None) -> ByteDFA:
    """Byte-level tables of a reference-style DFA (same layout as
    ``precompute_tmap``; unknown bytes are the identity)."""
    from .simulation import DFAMatrices, precompute_tmap
    dm = DFAMatrices(dfa)
    N = dm.n_states
    acc = np.zeros(N, dtype=np.uint8)
    for s in dfa.accept_states:
        acc[s] = 1
    syms = np.array([ord(c) for c in dm.alphabet], dtype=np.uint8)
    return ByteDFA(n_states=N, tmap=precompute_tmap(dm), accept=acc, start=dfa.start,
                   symbols=syms)


# --- inputs -------------------------------------------------------------------

def uniform_strings(n_strings: int, length: int, symbols, rng) -> tuple:
    symbols = np.asarray(symbols, dtype=np.uint8)
    data = symbols[rng.integers(0, len(symbols), size=n_strings * length)]
    offsets = np.arange(n_strings + 1, dtype=np.int64) * length
    return data, offsets


def lognormal_lengths(n_strings: int, rng, median=2048, sigma=1.18, lo=16, hi=65536):
    L = np.rint(np.exp(rng.normal(np.log(median), sigma, size=n_strings)))
    return np.clip(L, lo, hi).astype(np.int64)


def ragged_batch(n_strings: int, rng, median=2048, sigma=1.18, lo=16, hi=65536,
                 sub_frac=0.10, sub_alphabet=ACGT, n_dfas=16):
    """Ragged byte strings: returns (data, offsets, dfa_id, is_sub)."""
    lens = lognormal_lengths(n_strings, rng, median, sigma, lo, hi)
    offsets = np.zeros(n_strings + 1, dtype=np.int64)
    np.cumsum(lens, out=offsets[1:])
    total = int(offsets[-1])
    data = rng.integers(0, 256, size=total, dtype=np.uint8)
    is_sub = np.zeros(n_strings, dtype=bool)
    is_sub[rng.choice(n_strings, size=int(round(sub_frac * n_strings)), replace=False)] = True
    for i in np.flatnonzero(is_sub):
        a, b = offsets[i], offsets[i + 1]
        data[a:b] = sub_alphabet[rng.integers(0, len(sub_alphabet), size=b - a)]
    dfa_id = (np.arange(n_strings) % n_dfas).astype(np.int32)
    return data, offsets, dfa_id, is_sub


def ragged_dfas(rng, sizes=(8,) * 5 + (12,) * 5 + (16,) * 6):
    return [random_dfa(n, np.arange(256), rng) for n in sizes]


# --- NFAs --------------------------------------------------------------------

def random_bool_nfa(rng, n_states=64, sigma=20, density=0.05, accept_frac=0.25):
    """Boolean T[sigma, N, N] (row = dst, col = src) with Bernoulli(density)
    entries, start {0}, round(accept_frac*N) accepting states."""
    T = (rng.random((sigma, n_states, n_states)) < density).astype(np.int8)
    start = np.zeros(n_states, dtype=np.int8)
    start[0] = 1
    acc = np.zeros(n_states, dtype=np.int8)
    acc[rng.choice(n_states, size=max(1, int(round(accept_frac * n_states))), replace=False)] = 1
    return T, start, acc


def random_prob_nfa(rng, n_states=64, sigma=20, alpha=0.5, scale=0.9, keep=0.30):
    """T[c][dst, :] ~ Dirichlet(alpha) * scale, then a seeded mask keeps ~keep
    of the entries (no renormalisation). Start e0, accept all-ones."""
    T = rng.dirichlet(np.full(n_states, alpha), size=(sigma, n_states)) * scale
    mask = rng.random(T.shape) < keep
    T = np.where(mask, T, 0.0)
    start = np.zeros(n_states)
    start[0] = 1.0
    accept = np.ones(n_states)
    return T, start, accept
