"""The Python front end against golden vectors produced by the reference's own
modules (tests/golden/make_golden.py). CPU only."""

import numpy as np
import pytest

from trex_b200.kgram import auto_k, auto_k_for_gpu, precompute_kgrams, simulate_kgram_monoid
from trex_b200.monoid import compute_monoid, simulate_monoid
from trex_b200.nfa_matrices import compile_nfa_matrices, nfa_from_matrices, simulate_nfa
from trex_b200.regex_to_dfa import NFA, compile_regex
from trex_b200.simulation import DFAMatrices, precompute_tmap, simulate_prefix_scan
from trex_b200.workloads import ByteDFA


def _regex_records(golden):
    return [r for r in golden["regex"]]


def test_regex_languages_match_reference(golden):
    for r in _regex_records(golden):
        dfa = compile_regex(r["pattern"])
        assert dfa.n_states == r["dfa_states"], r["pattern"]
        if "error" in r:
            with pytest.raises(ValueError):
                compile_nfa_matrices(r["pattern"])
            with pytest.raises(ValueError):
                DFAMatrices(dfa)
            assert dfa.simulate("") == r["dfa_accept_empty"]
            assert dfa.simulate("a") == r["dfa_accept_a"]
            continue
        nm = compile_nfa_matrices(r["pattern"])
        assert nm.n_states_raw == r["nfa_states"], r["pattern"]
        assert sorted(dfa.alphabet) == r["alphabet"]
        assert [dfa.simulate(s) for s in r["strings"]] == r["dfa_accept"], r["pattern"]
        assert [simulate_nfa(nm, s) for s in r["strings"]] == r["nfa_accept"], r["pattern"]
        dm = DFAMatrices(dfa)
        assert [simulate_prefix_scan(dm, s) for s in r["strings"][:10]] == r["prefix_scan_accept"]


def test_monoid_and_kgram_match_reference(golden):
    seen = 0
    for r in _regex_records(golden):
        if "monoid_size" not in r:
            continue
        dfa = compile_regex(r["pattern"])
        dm = DFAMatrices(dfa)
        md = compute_monoid(dm, max_size=4096)
        assert md is not None and md.size == r["monoid_size"], r["pattern"]
        assert [simulate_monoid(md, dm, s) for s in r["strings"]] == r["monoid_accept"]
        kg = precompute_kgrams(dm, r["kgram_k"], monoid=md)
        ks = [s for s in r["strings"] if all(c in dm.char_to_idx for c in s)]
        assert [simulate_kgram_monoid(kg, md, dm, s) for s in ks] == r["kgram_accept"]
        seen += 1
    assert seen >= 10


def test_auto_k_values(golden):
    for s, k in golden["misc"]["auto_k"].items():
        assert auto_k(int(s)) == k
    for key, k in golden["misc"]["auto_k_for_gpu"].items():
        s, n = map(int, key.split(","))
        assert auto_k_for_gpu(s, n) == k


def _ref_style_dfa(rec):
    N = rec["n_states"]
    syms = np.array(rec["symbols"], dtype=np.uint8)
    t = np.array(rec["tmap"], dtype=np.uint8).reshape(256, rec["padded_states"])
    bd = ByteDFA(n_states=N, tmap=np.ascontiguousarray(t[:, :N]).reshape(-1),
                 accept=np.array(rec["accept"], dtype=np.uint8), symbols=syms)
    return bd


def test_tmap_matches_reference(golden):
    for rec in golden["byte_dfa"]:
        bd = _ref_style_dfa(rec)
        dfa = bd.to_dfa()
        dm = DFAMatrices(dfa)
        assert dm.n_states == rec["padded_states"]
        assert np.array_equal(precompute_tmap(dm), np.array(rec["tmap"], dtype=np.uint8))
        strings = [bytes.fromhex(h).decode("latin-1") for h in rec["strings_hex"]]
        assert [dfa.simulate(s) for s in strings] == rec["dfa_accept"]


def test_nfa_from_matrices_matches_reference(golden):
    for rec in golden["nfa"]:
        N, sigma = rec["n_states"], rec["sigma"]
        T = np.stack([np.unpackbits(np.frombuffer(bytes.fromhex(h), dtype=np.uint8))[:N * N]
                      .reshape(N, N) for h in rec["T_dst_src_hex"]]).astype(np.int8)
        nm = nfa_from_matrices(T, np.array(rec["start"]), np.array(rec["accept"]))
        strings = [bytes.fromhex(h).decode("latin-1") for h in rec["strings_hex"]]
        assert [simulate_nfa(nm, s) for s in strings] == rec["nfa_accept"]


def test_thompson_numbering_is_textbook():
    # literal: 2 states; alternation adds 2; closure adds 2
    nm = compile_nfa_matrices("a")
    assert nm.n_states_raw == 2
    assert compile_nfa_matrices("a|b").n_states_raw == 6
    assert compile_nfa_matrices("a*").n_states_raw == 4
    nfa = NFA()
    assert nfa.new_state() == 0 and nfa.new_state() == 1


def test_dfa_state_ids_are_canonical():
    d1 = compile_regex("(a|b)*abb")
    d2 = compile_regex("(a|b)*abb")
    assert d1.transitions == d2.transitions and d1.start == 0
