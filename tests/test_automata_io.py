"""Serialized automata (trex_b200.automata_io): round trip of byte DFAs, Boolean
and probabilistic NFAs; other files are refused."""

import numpy as np
import pytest

from trex_b200 import automata_io
from trex_b200.regex_to_dfa import compile_regex
from trex_b200.workloads import dfa_from_regex_dfa, random_bool_nfa, random_dfa, random_prob_nfa


def test_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    dfas = [random_dfa(16, np.arange(256), rng), random_dfa(5, np.frombuffer(b"ACGT", np.uint8), rng),
            dfa_from_regex_dfa(compile_regex("(a|b)*abb"))]
    nfas = [random_bool_nfa(rng, 64, 20)]
    pnfas = [random_prob_nfa(rng, 64, 20), random_prob_nfa(rng, 7, 3)]
    p = automata_io.save(tmp_path / "set", dfas, nfas, pnfas)
    got = automata_io.load(p)
    assert len(got["dfas"]) == 3 and len(got["nfas"]) == 1 and len(got["pnfas"]) == 2
    for a, b in zip(dfas, got["dfas"]):
        assert a.n_states == b.n_states and a.start == b.start
        assert np.array_equal(a.tmap, b.tmap) and np.array_equal(a.accept, b.accept)
    for a, b in zip(nfas, got["nfas"]):
        assert all(np.array_equal(np.asarray(x) != 0, y != 0) for x, y in zip(a, b))
    for a, b in zip(pnfas, got["pnfas"]):
        assert all(np.array_equal(np.asarray(x, np.float32), y) for x, y in zip(a, b))


def test_refuses_other_files(tmp_path):
    p = tmp_path / "x.npz"
    np.savez(p, a=np.zeros(3))
    with pytest.raises(ValueError):
        automata_io.load(p)
    q = automata_io.save(tmp_path / "v", [random_dfa(4, np.arange(256), np.random.default_rng(1))])
    z = dict(np.load(q))
    z["version"] = np.array(99)
    np.savez(tmp_path / "v99.npz", **z)
    with pytest.raises(ValueError):
        automata_io.load(tmp_path / "v99.npz")
    bad = dict(np.load(q))
    bad["dfa0_meta"] = np.array([4, 9])   # start out of range
    np.savez(tmp_path / "bad.npz", **bad)
    with pytest.raises(ValueError):
        automata_io.load(tmp_path / "bad.npz")
