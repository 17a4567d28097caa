"""Multi-pattern PackedEngine (reference src/packed_engine.py): results[pattern][string]
against the reference's own outputs (tests/golden/reference_golden.json, section
"packed"), on the CPU path and on the B200 multi-pattern launch."""

import random

import numpy as np
import pytest

from trex_b200.packed_engine import PackedEngine

KEYS = {"n_patterns", "state_counts", "offsets", "NP", "unified_alphabet_size", "regexes", "backend"}


def test_cpu_matches_reference_golden(golden):
    for rec in golden["packed"]:
        eng = PackedEngine(rec["regexes"])
        assert eng.match_batch(rec["strings"]) == rec["results"], rec["regexes"]
        info = eng.config_info
        assert KEYS <= set(info) and info["backend"] == "cpu"
        assert info["NP"] == rec["NP"] and info["state_counts"] == rec["state_counts"]


def test_empty_batch_and_timed():
    eng = PackedEngine(["(a|b)*abb", "a*b*"])
    assert eng.match_batch([]) == [[], []]
    res, timing = eng.match_batch_timed(["abb", "ab"])
    assert res == [[True, False], [True, True]]
    assert {"total_ms", "n_strings", "n_patterns", "NP"} <= set(timing)


@pytest.mark.gpu
def test_gpu_matches_reference_golden(cuda, golden):
    for rec in golden["packed"]:
        eng = PackedEngine(rec["regexes"], use_gpu=True)
        assert eng.config_info["backend"] == "gpu"
        assert eng.match_batch(rec["strings"]) == rec["results"], rec["regexes"]
        eng.close()


@pytest.mark.gpu
def test_gpu_many_patterns_long_strings_match_cpu(cuda):
    # 70 patterns (two DFA sets), strings long enough to be cut into items
    rng = random.Random(5)
    pats = ["(a|b)*abb", "a*b*", "(ab|ba)*", "a(b|c)*d", "(a|b|c)*abc", "x?y+z*", "[a-c]+d"] * 10
    strings = ["".join(rng.choice("abcdxyz#") for _ in range(rng.randint(0, 6000))) for _ in range(60)]
    strings += ["", "abb", "abc€"]
    gpu = PackedEngine(pats, use_gpu=True)
    res, timing = gpu.match_batch_timed(strings)
    assert "kernel_ms" in timing
    assert res == PackedEngine(pats).match_batch(strings)
    gpu.close()
