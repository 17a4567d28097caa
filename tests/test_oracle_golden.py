"""Pins the C oracle to the reference: golden vectors generated from the
reference's Python modules and the known-answer tests in the reference's
CUDA test mains. CPU only."""

import numpy as np

from trex_b200.workloads import ByteDFA, random_prob_nfa


def _csr(byte_strings):
    data = np.frombuffer(b"".join(byte_strings), dtype=np.uint8).copy()
    off = np.zeros(len(byte_strings) + 1, dtype=np.int64)
    np.cumsum([len(s) for s in byte_strings], out=off[1:])
    return data, off


def test_oracle_dfa_walk_and_positions(golden, oracle):
    for rec in golden["byte_dfa"]:
        N = rec["n_states"]
        t = np.array(rec["tmap"], dtype=np.uint8).reshape(256, rec["padded_states"])[:, :N]
        tmap = np.ascontiguousarray(t).reshape(-1)
        acc = np.array(rec["accept"], dtype=np.uint8)
        strs = [bytes.fromhex(h) for h in rec["strings_hex"]]
        data, off = _csr(strs)
        fs, ac = oracle.dfa_walk([tmap], [N], [0], [acc], data, off)
        assert fs.tolist() == rec["final_state"]
        # accept agrees with DFA.simulate for strings inside the alphabet
        syms = set(rec["symbols"])
        for i, s in enumerate(strs):
            if all(b in syms for b in s):
                assert bool(ac[i]) == rec["dfa_accept"][i]
        pos = oracle.dfa_positions(tmap, N, 0, data, off)
        for i, s in enumerate(strs):
            assert pos[off[i]:off[i + 1]].tolist() == rec["positions"][i]


def test_oracle_nfa_matches_reference(golden, oracle):
    for rec in golden["nfa"]:
        N, sigma = rec["n_states"], rec["sigma"]
        T = np.stack([np.unpackbits(np.frombuffer(bytes.fromhex(h), dtype=np.uint8))[:N * N]
                      .reshape(N, N) for h in rec["T_dst_src_hex"]])
        strs = [bytes.fromhex(h) for h in rec["strings_hex"]]
        data, off = _csr(strs)
        fm, ac = oracle.nfa_bool(T, rec["start"], rec["accept"], data, off, unknown_rejects=True)
        assert [bool(a) for a in ac] == rec["nfa_accept"]
        assert [format(int(m), "x") for m in fm] == rec["final_mask_hex"]


def test_even_a_known_answers(oracle):
    # reference cuda/monoid_batch.cu:716-748 and :802-804 (even number of 'a')
    strings = [b"", b"a", b"aa", b"b", b"aab", b"aabb", b"abab", b"aaaa", b"aaaaa", b"bbb",
               b"aba", b"bab"]
    expected = [1, 0, 1, 1, 1, 1, 1, 1, 0, 1, 1, 0]
    t = np.tile(np.arange(2, dtype=np.uint8), (256, 1))
    t[ord("a")] = [1, 0]
    data, off = _csr(strings)
    _, ac = oracle.dfa_walk([t.reshape(-1)], [2], [0], [np.array([1, 0], np.uint8)], data, off)
    assert ac.tolist() == expected


def test_three_a_nfa_known_answers(oracle):
    # reference cuda/nfa_tc_evolution.cu:1056-1137: ">= 3 a's", symbols a=0, b=1
    N = 64
    T = np.zeros((2, N, N), dtype=np.int8)
    for i in range(3):
        T[0, i, i] = 1
        T[0, i + 1, i] = 1
    T[0, 3, 3] = 1
    for i in range(4):
        T[1, i, i] = 1
    for s in range(4, N):
        T[0, s, s] = T[1, s, s] = 1
    start = np.zeros(N); start[0] = 1
    acc = np.zeros(N); acc[3] = 1
    strs = [b"", b"\0", b"\0\0", b"\0\0\0", b"\1", b"\1\0\1", b"\0\0\0\1", b"\1\0\0\0",
            b"\0\1\0\1", b"\0\0\1\0\0"]
    expected = [0, 0, 0, 1, 0, 0, 1, 1, 0, 1]
    data, off = _csr(strs)
    for rej in (True, False):
        _, ac = oracle.nfa_bool(T, start, acc, data, off, unknown_rejects=rej)
        assert ac.tolist() == expected


def test_prefix_compose_known_answers(oracle):
    # reference cuda/prefix_compose.cu:518-544: (a|b)*a(a|b), second-to-last is 'a'
    # states track (second_to_last == a, last == a)
    nxt = {}
    for s in range(4):
        last_a = s & 1
        for ch, is_a in ((ord("a"), 1), (ord("b"), 0)):
            nxt[(ch, s)] = (last_a << 1) | is_a
    t = np.tile(np.arange(4, dtype=np.uint8), (256, 1))
    for (ch, s), d in nxt.items():
        t[ch, s] = d
    acc = np.array([0, 0, 1, 1], dtype=np.uint8)
    strs = [b"aa", b"ab", b"ba", b"bb", b"a", b"", b"bab", b"abb", b"aab"]
    exp = [1, 1, 0, 0, 0, 0, 1, 0, 1]
    data, off = _csr(strs)
    _, ac = oracle.dfa_walk([t.reshape(-1)], [4], [0], [acc], data, off)
    assert ac.tolist() == exp


def test_pnfa_oracle_matches_numpy_fp64(oracle):
    rng = np.random.default_rng(3)
    T, start, accept = random_prob_nfa(rng, n_states=16, sigma=5)
    strs = [bytes(rng.integers(0, 5, size=L).astype(np.uint8).tolist()) for L in (0, 1, 7, 300)]
    data, off = _csr(strs)
    ll = oracle.pnfa_fp64(T, start, accept, data, off)
    for i, s in enumerate(strs):
        v = start.copy()
        logscale = 0.0
        for c in s:
            v = T[c] @ v
            m = v.max()
            v /= m
            logscale += np.log(m)
        ref = np.log(accept @ v) + logscale
        assert abs(ll[i] - ref) <= 1e-9 * max(1.0, abs(ref))


def test_oracle_multi_dfa(oracle):
    rng = np.random.default_rng(5)
    from trex_b200.workloads import random_dfa
    dfas = [random_dfa(n, np.arange(256), rng) for n in (3, 16, 200)]
    strs = [bytes(rng.integers(0, 256, size=L).astype(np.uint8).tolist()) for L in (0, 5, 99, 1000)]
    data, off = _csr(strs * 3)
    ids = np.repeat(np.arange(3, dtype=np.int32), 4)
    fs, ac = oracle.dfa_walk([d.tmap for d in dfas], [d.n_states for d in dfas], [0, 0, 0],
                             [d.accept for d in dfas], data, off, ids)
    for i in range(12):
        d = dfas[ids[i]]
        s = 0
        for b in data[off[i]:off[i + 1]]:
            s = int(d.tmap[int(b) * d.n_states + int(s)])
        assert fs[i] == s and ac[i] == d.accept[s]
