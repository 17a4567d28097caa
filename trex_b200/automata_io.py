"""Serialized compiled automata: one file holding byte DFAs, Boolean NFAs and
probabilistic NFAs in the forms the kernels load, so a server reloads its
resident tables without compiling regexes again (the reference has no such
format; it regenerates automata from JSON workload descriptions,
src/generate_data.py:290-297).

Format: a NumPy ``.npz`` archive (no pickled objects) with

    format            "trex_b200.automata", version 1
    dfa_count, nfa_count, pnfa_count
    dfa{i}_tmap       uint8 [256 * N]   next state of (byte, state): tmap[byte * N + s]
    dfa{i}_accept     uint8 [N]
    dfa{i}_meta       int64 [2]         N, start
    dfa{i}_symbols    uint8 [k]         the automaton's alphabet (informational)
    nfa{i}_T          int8  [sigma, N, N]  T[c][dst, src] in {0, 1}
    nfa{i}_start, nfa{i}_accept          int8 [N]
    pnfa{i}_T         float32 [sigma, N, N], pnfa{i}_start, pnfa{i}_accept float32 [N]
"""

from __future__ import annotations

from pathlib import Path
from typing import Sequence

import numpy as np

from .workloads import ByteDFA

FORMAT = "trex_b200.automata"
VERSION = 1


def save(path, dfas: Sequence[ByteDFA] = (), nfas: Sequence = (), pnfas: Sequence = ()) -> Path:
    """Writes the automata to ``path`` (``.npz``); returns the path written."""
    arrays = {"format": np.array(FORMAT), "version": np.array(VERSION, dtype=np.int64),
              "dfa_count": np.array(len(dfas), dtype=np.int64),
              "nfa_count": np.array(len(nfas), dtype=np.int64),
              "pnfa_count": np.array(len(pnfas), dtype=np.int64)}
    for i, d in enumerate(dfas):
        N = int(d.n_states)
        tmap = np.ascontiguousarray(np.asarray(d.tmap, dtype=np.uint8).reshape(-1))
        if tmap.size != 256 * N or int(tmap.max(initial=0)) >= N:
            raise ValueError(f"DFA {i}: tmap must hold 256 * N next states below N")
        arrays[f"dfa{i}_tmap"] = tmap
        arrays[f"dfa{i}_accept"] = np.asarray(d.accept, dtype=np.uint8).reshape(-1)
        arrays[f"dfa{i}_meta"] = np.array([N, int(d.start)], dtype=np.int64)
        arrays[f"dfa{i}_symbols"] = np.asarray(d.symbols, dtype=np.uint8).reshape(-1)
    for i, (T, s, a) in enumerate(nfas):
        arrays[f"nfa{i}_T"] = (np.asarray(T) != 0).astype(np.int8)
        arrays[f"nfa{i}_start"] = (np.asarray(s) != 0).astype(np.int8).reshape(-1)
        arrays[f"nfa{i}_accept"] = (np.asarray(a) != 0).astype(np.int8).reshape(-1)
    for i, (T, s, a) in enumerate(pnfas):
        arrays[f"pnfa{i}_T"] = np.asarray(T, dtype=np.float32)
        arrays[f"pnfa{i}_start"] = np.asarray(s, dtype=np.float32).reshape(-1)
        arrays[f"pnfa{i}_accept"] = np.asarray(a, dtype=np.float32).reshape(-1)
    path = Path(path)
    if path.suffix != ".npz":
        path = path.with_suffix(path.suffix + ".npz")
    np.savez_compressed(path, **arrays)
    return path


def load(path) -> dict:
    """Reads a file written by :func:`save`: {"dfas": [ByteDFA], "nfas": [(T, start,
    accept)], "pnfas": [(T, start, accept)]}. Raises ValueError on a file of another
    format or version."""
    with np.load(Path(path), allow_pickle=False) as z:
        if "format" not in z or str(z["format"]) != FORMAT:
            raise ValueError(f"{path}: not a {FORMAT} file")
        if int(z["version"]) != VERSION:
            raise ValueError(f"{path}: version {int(z['version'])}, this library reads {VERSION}")
        out = {"dfas": [], "nfas": [], "pnfas": []}
        for i in range(int(z["dfa_count"])):
            N, start = (int(x) for x in z[f"dfa{i}_meta"])
            tmap = z[f"dfa{i}_tmap"].astype(np.uint8)
            if tmap.size != 256 * N or (tmap.size and int(tmap.max()) >= N) or not 0 <= start < N:
                raise ValueError(f"{path}: DFA {i} is malformed")
            out["dfas"].append(ByteDFA(n_states=N, tmap=tmap, accept=z[f"dfa{i}_accept"].astype(np.uint8),
                                       start=start, symbols=z[f"dfa{i}_symbols"].astype(np.uint8)))
        for i in range(int(z["nfa_count"])):
            out["nfas"].append((z[f"nfa{i}_T"].astype(np.int8), z[f"nfa{i}_start"].astype(np.int8),
                                z[f"nfa{i}_accept"].astype(np.int8)))
        for i in range(int(z["pnfa_count"])):
            out["pnfas"].append((z[f"pnfa{i}_T"].astype(np.float32), z[f"pnfa{i}_start"].astype(np.float32),
                                 z[f"pnfa{i}_accept"].astype(np.float32)))
    return out
