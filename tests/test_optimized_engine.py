"""OptimizedEngine drop-in (reference src/optimized_engine.py, tests/test_optimized_engine.py).

CPU part: config handling, the reference's CPU configs against the golden
accept flags the reference produced (tests/golden/reference_golden.json), and
the byte-map translation used by the B200 DFA engine against DFA.simulate.
GPU part: every GPU config against the same golden flags, the README form
(pattern=..., config="auto", .match), prebuilt byte DFAs against the oracle.
"""

import random

import numpy as np
import pytest

from trex_b200.optimized_engine import OptimizedEngine, _byte_dfa_from_dfa
from trex_b200.regex_to_dfa import compile_regex
from trex_b200.workloads import random_dfa

REQUIRED = {"representation", "scan_backend", "alphabet_size", "kgram_k", "selection_reason"}


def _valid_records(golden):
    return [r for r in golden["regex"] if "error" not in r and r.get("strings")]


def _in_alphabet(rec):
    al = set(rec["alphabet"])
    return [i for i, s in enumerate(rec["strings"]) if all(c in al for c in s)]


# ---- CPU ------------------------------------------------------------------------------------------
def test_unknown_config_raises():
    with pytest.raises(ValueError):
        OptimizedEngine("(a|b)*abb", config="turbo")


def test_pattern_given_once():
    with pytest.raises(TypeError):
        OptimizedEngine("(a|b)*abb", pattern="ab")
    with pytest.raises(TypeError):
        OptimizedEngine()


@pytest.mark.parametrize("cfg", ["baseline", "monoid", "monoid+kgram", "nfa"])
def test_cpu_configs_match_reference_golden(golden, cfg):
    for rec in _valid_records(golden):
        if cfg in ("monoid", "monoid+kgram") and rec.get("monoid_size") is None:
            continue
        eng = OptimizedEngine(rec["pattern"], config=cfg)
        info = eng.config_info
        assert REQUIRED <= set(info), info
        if cfg == "monoid+kgram":   # the reference's k-gram walk needs in-alphabet strings
            idx = _in_alphabet(rec)
            got = eng.match_batch([rec["strings"][i] for i in idx])
            assert got == [rec["dfa_accept"][i] for i in idx], (rec["pattern"], cfg)
            continue
        got = eng.match_batch(rec["strings"])
        key = {"baseline": "dfa_accept", "monoid": "monoid_accept", "nfa": "nfa_accept"}[cfg]
        assert got == rec[key], (rec["pattern"], cfg)


def test_cpu_timed_dict():
    eng = OptimizedEngine("(a|b)*abb", config="baseline")
    res, timing = eng.match_batch_timed(["abb", "ab", ""])
    assert res == [True, False, False]
    assert {"total_seconds", "per_string_seconds", "n_strings"} <= set(timing)
    assert timing["n_strings"] == 3


def test_byte_map_follows_dfa_simulate(golden):
    """The byte DFA handed to the kernel walks like DFA.simulate, unknown bytes included."""
    rng = random.Random(3)
    for rec in _valid_records(golden):
        dfa = compile_regex(rec["pattern"])
        if any(ord(c) > 255 for c in dfa.alphabet):
            continue
        bdfa, _ = _byte_dfa_from_dfa(dfa)
        N = bdfa.n_states
        t = bdfa.tmap.reshape(256, N)
        alpha = sorted(dfa.alphabet) + ["#", "\x00", "\xff"]
        strings = rec["strings"] + ["".join(rng.choice(alpha) for _ in range(rng.randint(0, 12)))
                                    for _ in range(60)]
        for s in strings:
            st = bdfa.start
            for ch in s.encode("latin-1"):
                st = t[ch, st]
            assert bool(bdfa.accept[st]) == dfa.simulate(s), (rec["pattern"], s)


# ---- GPU ------------------------------------------------------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("cfg", [None, "auto", "dfa+gpu", "batched+gpu", "kgram+gpu", "fp16_tc+gpu"])
def test_gpu_dfa_configs_match_golden(cuda, golden, cfg):
    for rec in _valid_records(golden):
        eng = OptimizedEngine(rec["pattern"], config=cfg)
        assert REQUIRED <= set(eng.config_info)
        if cfg not in (None, "auto"):
            assert eng.config_info["scan_backend"] == cfg
        if eng.config_info["representation"] == "dfa":
            assert eng.match_batch(rec["strings"]) == rec["dfa_accept"], (rec["pattern"], cfg)
        else:
            assert eng.match_batch(rec["strings"]) == rec["nfa_accept"], (rec["pattern"], cfg)
        eng.close()


@pytest.mark.gpu
@pytest.mark.parametrize("cfg", ["monoid_batch+gpu", "prefix+gpu", "monoid+gpu", "nfa+gpu"])
def test_gpu_bridge_configs_match_golden(cuda, golden, cfg):
    for rec in _valid_records(golden):
        if cfg.startswith("monoid") and rec.get("monoid_size") is None:
            continue
        if cfg == "monoid_batch+gpu" and rec["monoid_size"] > 255:
            continue
        if cfg == "nfa+gpu" and rec["nfa_states"] > 64:
            continue
        eng = OptimizedEngine(rec["pattern"], config=cfg)
        assert eng.config_info["scan_backend"] == cfg
        got = eng.match_batch(rec["strings"])
        if cfg == "nfa+gpu":   # simulate_nfa semantics on every string
            assert got == rec["nfa_accept"], rec["pattern"]
        else:                  # byte-map bridges: identity for unknown characters
            idx = _in_alphabet(rec)
            assert [got[i] for i in idx] == [rec["dfa_accept"][i] for i in idx], (rec["pattern"], cfg)
        eng.close()


@pytest.mark.gpu
def test_readme_form_and_timing(cuda):
    eng = OptimizedEngine(pattern="(a|b)*abb", config="auto")
    assert eng.match(["aabb", "abab", "", "abb"]) == [True, False, False, True]
    assert eng.match("babb") is True
    res, timing = eng.match_batch_timed(["abb"] * 300)
    assert res == [True] * 300
    assert timing["kernel_ms"] >= 0.0 and timing["total_ms"] >= timing["kernel_ms"]
    # characters outside the alphabet (and above U+00FF) go to the dead state
    assert eng.match(["abb€", "ab#b", "Āabb"]) == [False, False, False]
    assert eng.match([b"aabb", bytearray(b"ab")]) == [True, False]
    eng.close()


@pytest.mark.gpu
def test_prebuilt_byte_dfa_matches_oracle(cuda, oracle):
    rng = np.random.default_rng(21)
    bdfa = random_dfa(16, np.arange(256), rng)
    strings = [bytes(rng.integers(0, 256, size=int(rng.integers(0, 3000)), dtype=np.uint8)) for _ in range(500)]
    eng = OptimizedEngine(bdfa)
    assert eng.config_info["dfa_states"] == 16
    got = eng.match_batch(strings)
    data = np.frombuffer(b"".join(strings), dtype=np.uint8).copy()
    off = np.zeros(len(strings) + 1, dtype=np.int64)
    np.cumsum([len(s) for s in strings], out=off[1:])
    _, acc = oracle.dfa_walk([bdfa.tmap], [16], [bdfa.start], [bdfa.accept], data, off,
                             np.zeros(len(strings), np.int32))
    assert got == [bool(a) for a in acc]
    eng.close()
