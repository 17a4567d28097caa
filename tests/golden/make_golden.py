"""Generate golden vectors by importing the reference's own Python modules.

Run from the repository root, naming the reference project's checkout (the
directory that holds its ``src/`` package) on the command line or in
TREX_REFERENCE:

    python tests/golden/make_golden.py <reference checkout>

It writes ``tests/golden/reference_golden.json`` (small, committed). The
tests read only that JSON file; they never import the reference.

What is recorded (all inputs are seeded and stored, so the fixture is
self-contained):
  * regex languages: for every pattern, the reference's minimal DFA size, NFA
    size, and accept flags of ``DFA.simulate`` and ``simulate_nfa`` on seeded
    strings (reference src/regex_to_dfa.py:224, src/nfa_matrices.py:133);
  * monoid: reference ``compute_monoid`` size, ``simulate_monoid`` and
    ``simulate_kgram_monoid`` flags, ``auto_k`` values (src/monoid.py,
    src/kgram.py);
  * byte DFAs: random DFAs given to the reference's ``DFAMatrices`` /
    ``precompute_tmap`` and walked with ``DFA.simulate``; final states and
    per-position states from ``prefix_scan_sequential`` (src/simulation.py:142);
  * Boolean NFAs: random matrices built into a reference ``NFA`` and walked
    with ``simulate_nfa``; the final state vector comes from the reference
    matrices with the same clamp loop.
"""

from __future__ import annotations

import json
import os
import random
import sys
from pathlib import Path

import numpy as np

def _reference_dir() -> Path:
    arg = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TREX_REFERENCE")
    if not arg:
        sys.exit("usage: make_golden.py <reference checkout> (or set TREX_REFERENCE)")
    ref = Path(arg)
    if not (ref / "src" / "regex_to_dfa.py").exists():
        sys.exit(f"{ref} does not hold the reference's src/ package")
    return ref


REF = _reference_dir()
OUT = Path(__file__).resolve().parent / "reference_golden.json"

sys.path.insert(0, str(REF))

from src.regex_to_dfa import compile_regex, NFA, DFA  # noqa: E402
from src.simulation import (DFAMatrices, precompute_tmap,  # noqa: E402
                            prefix_scan_sequential, simulate_prefix_scan)
from src.nfa_matrices import compile_nfa_matrices, NFAMatrices, simulate_nfa  # noqa: E402
from src.monoid import compute_monoid, simulate_monoid  # noqa: E402
from src.kgram import auto_k, auto_k_for_gpu, precompute_kgrams, simulate_kgram_monoid  # noqa: E402
from src.generate_data import PATTERNS  # noqa: E402

PATTERN_LIST = [p.regex for p in PATTERNS.values()] + [
    "(a|b)*a(a|b)", "a*b*", "(ab|ba)*", "(a|b|c)*abc", "[a-z]+", "a(b|c)*d",
    "x?y+z*", "(a|)b", "[^a-y]", "a.c", "\\d+\\.\\d*", "\\w\\s\\w", "[]", "ab)c",
    "a**", "(a(b(c)))", "[a-c-e]", "(((a)))|b", "",
]

EXTRA_CHARS = "az09.@ x"


def _strings(alphabet, n, max_len, rng):
    return ["".join(rng.choice(alphabet) for _ in range(rng.randint(0, max_len)))
            for _ in range(n)]


def regex_section():
    out = []
    for k, pat in enumerate(PATTERN_LIST):
        dfa = compile_regex(pat)
        try:
            nm = compile_nfa_matrices(pat)
            DFAMatrices(dfa)
        except ValueError:
            # the reference cannot build matrices for an empty alphabet
            out.append({"pattern": pat, "dfa_states": dfa.n_states, "error": "ValueError",
                        "dfa_accept_empty": bool(dfa.simulate("")),
                        "dfa_accept_a": bool(dfa.simulate("a"))})
            continue
        alpha = "".join(sorted(dfa.alphabet)) or "ab"
        rng = random.Random(1000 + k)
        strings = _strings(alpha, 40, 14, rng) + _strings(alpha + EXTRA_CHARS, 10, 10, rng)
        rec = {
            "pattern": pat,
            "dfa_states": dfa.n_states,
            "nfa_states": nm.n_states_raw,
            "alphabet": sorted(dfa.alphabet),
            "strings": strings,
            "dfa_accept": [bool(dfa.simulate(s)) for s in strings],
            "nfa_accept": [bool(simulate_nfa(nm, s)) for s in strings],
            "prefix_scan_accept": [bool(simulate_prefix_scan(DFAMatrices(dfa), s))
                                   for s in strings[:10]],
        }
        dm = DFAMatrices(dfa)
        if dfa.n_states <= 24:
            md = compute_monoid(dm, max_size=4096)
            if md is not None:
                rec["monoid_size"] = md.size
                rec["monoid_accept"] = [bool(simulate_monoid(md, dm, s)) for s in strings]
                k_ = auto_k(len(dm.alphabet), 4096)
                kg = precompute_kgrams(dm, min(k_, 3), monoid=md)
                rec["kgram_k"] = kg.k
                rec["kgram_accept"] = [bool(simulate_kgram_monoid(kg, md, dm, s))
                                       for s in strings if all(c in dm.char_to_idx for c in s)]
        out.append(rec)
    return out


def _ref_dfa_from_table(nxt, accept, symbols):
    N = nxt.shape[1]
    trans = {s: {chr(int(b)): int(nxt[j, s]) for j, b in enumerate(symbols)} for s in range(N)}
    return DFA(n_states=N, start=0, accept_states={int(a) for a in np.flatnonzero(accept)},
               transitions=trans, alphabet={chr(int(b)) for b in symbols})


def byte_dfa_section():
    out = []
    rng = np.random.default_rng(7)
    specs = [(16, b"ACGT"), (16, bytes(range(256))), (8, bytes(range(256))),
             (12, bytes(range(256))), (5, b"ab"), (16, bytes(range(0, 256, 3)))]
    for k, (N, syms) in enumerate(specs):
        symbols = np.frombuffer(syms, dtype=np.uint8)
        nxt = rng.integers(0, N, size=(len(symbols), N))
        accept = np.zeros(N, dtype=np.uint8)
        accept[rng.choice(N, size=max(1, round(N / 4)), replace=False)] = 1
        dfa = _ref_dfa_from_table(nxt, accept, symbols)
        dm = DFAMatrices(dfa)
        tmap = precompute_tmap(dm)
        lens = [0, 1, 2, 3, 15, 16, 17, 31, 32, 33, 100, 257] + \
            rng.integers(0, 300, size=8).tolist()
        strs_bytes = []
        for L in lens:
            pool = symbols if k % 2 == 0 else np.arange(256, dtype=np.uint8)
            strs_bytes.append(bytes(pool[rng.integers(0, len(pool), size=L)].tolist()))
        strings = [b.decode("latin-1") for b in strs_bytes]
        # reference results: accept via DFA.simulate; final state and
        # positions via the matrix prefix scan (identity for unknown bytes).
        final_states, positions = [], []
        for s in strings:
            if not s:
                final_states.append(int(dfa.start))
                positions.append([])
                continue
            pref = prefix_scan_sequential(dm.get_matrix_sequence(s))
            st = (pref.astype(np.int32) @ dm.start_vec.astype(np.int32))  # [L, N]
            pos = np.argmax(st, axis=1).tolist()
            positions.append(pos)
            final_states.append(int(pos[-1]))
        out.append({
            "n_states": N,
            "symbols": symbols.tolist(),
            "padded_states": dm.n_states,
            "tmap": tmap.tolist(),
            "accept": accept.tolist(),
            "strings_hex": [b.hex() for b in strs_bytes],
            "dfa_accept": [bool(dfa.simulate(s)) for s in strings],
            "final_state": final_states,
            "positions": positions,
        })
    return out


def nfa_section():
    out = []
    rng = np.random.default_rng(11)
    for k, (N, sigma, dens) in enumerate([(64, 20, 0.05), (64, 2, 0.04), (33, 5, 0.1), (10, 3, 0.2)]):
        T = (rng.random((sigma, N, N)) < dens).astype(np.int8)
        nfa = NFA()
        for _ in range(N):
            nfa.new_state()
        nfa.start = 0
        for c in range(sigma):
            d_idx, s_idx = np.nonzero(T[c])
            for d, s in zip(d_idx.tolist(), s_idx.tolist()):
                nfa.add_trans(s, chr(c), d)
            nfa.alphabet.add(chr(c))
        acc = rng.choice(N, size=max(1, N // 4), replace=False)
        for a in acc.tolist():
            nfa.states[a].is_accept = True
        nm = NFAMatrices(nfa, pad_to=N)
        lens = [0, 1, 2, 5, 64, 200] + rng.integers(0, 400, size=10).tolist()
        strs = []
        for L in lens:
            v = rng.integers(0, sigma, size=L)
            if k == 0 and L > 3 and len(strs) % 5 == 4:
                v[L // 2] = sigma + 1   # a symbol outside the alphabet
            strs.append(bytes(v.astype(np.uint8).tolist()))
        masks = []
        for b in strs:
            s = b.decode("latin-1")
            st = nm.start_vec.astype(np.int32)
            bad = False
            for ch in s:
                ci = nm.char_to_idx.get(ch)
                if ci is None:
                    bad = True
                    break
                st = np.minimum(nm.matrix_stack[ci].astype(np.int32) @ st, 1)
            masks.append("0" if bad else format(sum(1 << int(i) for i in np.flatnonzero(st[:N])), "x"))
        out.append({
            "n_states": N, "sigma": sigma,
            "T_dst_src_hex": [np.packbits(T[c].reshape(-1)).tobytes().hex() for c in range(sigma)],
            "start": nm.start_vec[:N].tolist(),
            "accept": nm.accept_mask[:N].tolist(),
            "strings_hex": [b.hex() for b in strs],
            "nfa_accept": [bool(simulate_nfa(nm, b.decode("latin-1"))) for b in strs],
            "final_mask_hex": masks,
        })
    return out


def misc_section():
    return {
        "auto_k": {str(s): auto_k(s) for s in (1, 2, 3, 4, 16, 20, 256)},
        "auto_k_for_gpu": {f"{s},{n}": auto_k_for_gpu(s, n)
                           for s in (2, 4, 20) for n in (16, 64)},
    }


PACKED_SETS = [
    ["(a|b)*abb", "a*b*"],
    ["abc", "(a|b|c)*abc", "[a-z]+", "a(b|c)*d"],
    ["x?y+z*"],
    ["(ab|ba)*", "a.c", "\\d+\\.\\d*", "(a|b)*a(a|b)", "[^a-y]"],
]


def packed_section():
    """The reference's multi-pattern PackedEngine (src/packed_engine.py, CPU path):
    results[pattern][string] for a few pattern sets."""
    from src.packed_engine import PackedEngine
    rng = random.Random(29)
    out = []
    for regexes in PACKED_SETS:
        eng = PackedEngine(regexes)
        alpha = sorted(set("".join(eng._unified_alphabet)) | set(EXTRA_CHARS))
        strings = _strings(alpha, 120, 40, rng) + ["", "abb", "abc", "aabb", "xyyz", "1.5"]
        out.append({"regexes": regexes, "strings": strings,
                    "results": [[bool(x) for x in row] for row in eng.match_batch(strings)],
                    "NP": int(eng._NP), "state_counts": [int(n) for n in eng._state_counts]})
    return out


def main():
    if "--only-packed" in sys.argv:   # add or refresh this section only
        data = json.loads(OUT.read_text())
        data["packed"] = packed_section()
        OUT.write_text(json.dumps(data, separators=(",", ":")))
        print(f"updated the packed section of {OUT}")
        return
    data = {
        "generator": "tests/golden/make_golden.py",
        "regex": regex_section(),
        "byte_dfa": byte_dfa_section(),
        "nfa": nfa_section(),
        "misc": misc_section(),
        "packed": packed_section(),
    }
    OUT.write_text(json.dumps(data, separators=(",", ":")))
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
