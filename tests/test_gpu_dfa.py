"""Family (a) on the GPU: ragged batch DFA kernel vs the C oracle, through the
C ABI (handle API, reference singletons and the Python bridges)."""

import numpy as np
import pytest

from trex_b200.workloads import ACGT, random_dfa, ragged_batch, uniform_strings

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _run_set(torch, dfas, data, off, ids=None, seg_len=0):
    from trex_b200.engine import DFASet
    s = DFASet(dfas)
    d_data = _dev(torch, data if data.size else np.zeros(1, np.uint8))
    d_off = _dev(torch, off.astype(np.int64))
    d_ids = None if ids is None else _dev(torch, ids.astype(np.int32))
    fs, ac, _ = s.run(d_data[:data.size] if data.size else d_data[:0], d_off, d_ids, seg_len=seg_len)
    torch.cuda.synchronize()
    err = s.last_error_word()
    s.close()
    return fs.cpu().numpy(), ac.cpu().numpy(), err


@pytest.mark.parametrize("n_states", [1, 2, 5, 8, 9, 12, 16, 17, 24, 32, 48, 64, 65, 100, 255])
def test_random_dfa_matches_oracle(cuda, oracle, n_states):
    rng = np.random.default_rng(100 + n_states)
    d = random_dfa(n_states, np.arange(256), rng)
    lens = rng.integers(0, 3000, size=700)
    lens[:40] = np.arange(40)
    off = np.zeros(len(lens) + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    data = rng.integers(0, 256, size=int(off[-1]), dtype=np.uint8)
    fs, ac, err = _run_set(cuda, [d], data, off, seg_len=256)
    rfs, rac = oracle.dfa_walk([d.tmap], [d.n_states], [0], [d.accept], data, off)
    assert err == 0
    assert np.array_equal(fs, rfs)
    assert np.array_equal(ac, rac)


@pytest.mark.parametrize("seg_len", [64, 100, 1000, 8192])
def test_segment_maps_compose_exactly(cuda, oracle, seg_len):
    # Long strings are split; permutation DFAs never synchronise, so the
    # full 16-state map path is exercised too.
    rng = np.random.default_rng(seg_len)
    dfas = [random_dfa(16, np.arange(256), rng), random_dfa(8, np.arange(256), rng)]
    perm = np.stack([rng.permutation(12) for _ in range(256)]).astype(np.uint8)
    from trex_b200.workloads import ByteDFA
    acc = np.zeros(12, np.uint8); acc[[1, 5]] = 1
    dfas.append(ByteDFA(12, np.ascontiguousarray(perm.reshape(-1)), acc, start=3))
    lens = rng.integers(0, 40000, size=60)
    off = np.zeros(len(lens) + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    data = rng.integers(0, 256, size=int(off[-1]), dtype=np.uint8)
    ids = (np.arange(len(lens)) % 3).astype(np.int32)
    fs, ac, err = _run_set(cuda, dfas, data, off, ids, seg_len=seg_len)
    rfs, rac = oracle.dfa_walk([d.tmap for d in dfas], [d.n_states for d in dfas],
                               [d.start for d in dfas], [d.accept for d in dfas], data, off, ids)
    assert err == 0
    assert np.array_equal(fs, rfs)
    assert np.array_equal(ac, rac)


@pytest.mark.parametrize("n_states", [32, 64])
@pytest.mark.parametrize("seg_len", [64, 1000])
def test_split_strings_large_automata(cuda, oracle, n_states, seg_len):
    # Automata of 17 to 64 states have their strings cut too (warm-up 4 N bytes); a
    # permutation automaton of as many states never synchronises, so its fix-ups never meet
    # and the string is walked again from that item (one lane through the global byte map).
    rng = np.random.default_rng(n_states + seg_len)
    from trex_b200.workloads import ByteDFA
    perm = np.stack([rng.permutation(n_states) for _ in range(256)]).astype(np.uint8)
    acc = np.zeros(n_states, np.uint8)
    acc[[1, n_states - 2]] = 1
    dfas = [random_dfa(n_states, np.arange(256), rng),
            ByteDFA(n_states, np.ascontiguousarray(perm.reshape(-1)), acc, start=3)]
    lens = rng.integers(0, 30000, size=80)
    lens[:4] = [0, 1, 31, 33]
    off = np.zeros(len(lens) + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    data = rng.integers(0, 256, size=int(off[-1]), dtype=np.uint8)
    ids = (np.arange(len(lens)) % 2).astype(np.int32)
    fs, ac, err = _run_set(cuda, dfas, data, off, ids, seg_len=seg_len)
    rfs, rac = oracle.dfa_walk([d.tmap for d in dfas], [d.n_states for d in dfas],
                               [d.start for d in dfas], [d.accept for d in dfas], data, off, ids)
    assert err == 0
    assert np.array_equal(fs, rfs)
    assert np.array_equal(ac, rac)


def test_ragged_batch_mixed_sizes_to_64(cuda, oracle):
    rng = np.random.default_rng(64)
    sizes = (8, 12, 16, 24, 32, 48, 64, 64)
    dfas = [random_dfa(n, np.arange(256), rng) for n in sizes]
    data, off, ids, _ = ragged_batch(12000, rng, median=1024, hi=30000)
    ids = (ids % len(sizes)).astype(np.int32)
    fs, ac, err = _run_set(cuda, dfas, data, off, ids, seg_len=512)
    rfs, rac = oracle.dfa_walk([d.tmap for d in dfas], [d.n_states for d in dfas],
                               [0] * len(sizes), [d.accept for d in dfas], data, off, ids)
    assert err == 0
    assert np.array_equal(fs, rfs) and np.array_equal(ac, rac)


@pytest.mark.parametrize("n_states", [8, 12, 100])
@pytest.mark.parametrize("length", [32, 1024, 2080])
def test_whole_window_batches(cuda, oracle, n_states, length):
    # Strings whose bytes fill whole 32-byte windows: every batch but the last
    # (1000 items: not a multiple of 64) runs entirely through the unmasked
    # loop; 2080-byte strings are cut into pieces whose warm-ups end on window
    # boundaries.
    rng = np.random.default_rng(n_states * 7 + length)
    d = random_dfa(n_states, np.arange(256), rng)
    lens = np.full(1000, length, dtype=np.int64)
    off = np.zeros(len(lens) + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    data = rng.integers(0, 256, size=int(off[-1]), dtype=np.uint8)
    fs, ac, err = _run_set(cuda, [d], data, off, seg_len=1024)
    rfs, rac = oracle.dfa_walk([d.tmap], [d.n_states], [0], [d.accept], data, off)
    assert err == 0
    assert np.array_equal(fs, rfs)
    assert np.array_equal(ac, rac)


def test_ragged_multi_dfa_batch(cuda, oracle):
    rng = np.random.default_rng(42)
    sizes = (8,) * 5 + (12,) * 5 + (16,) * 6
    dfas = [random_dfa(n, np.arange(256), rng) for n in sizes]
    data, off, ids, _ = ragged_batch(20000, rng, median=512, hi=20000)
    fs, ac, err = _run_set(cuda, dfas, data, off, ids)
    rfs, rac = oracle.dfa_walk([d.tmap for d in dfas], [d.n_states for d in dfas],
                               [0] * 16, [d.accept for d in dfas], data, off, ids)
    assert err == 0
    assert np.array_equal(fs, rfs) and np.array_equal(ac, rac)


def test_unaligned_offsets_and_empty_strings(cuda, oracle):
    rng = np.random.default_rng(7)
    d = random_dfa(16, ACGT, rng)
    # strings starting at every alignment, including empty ones
    lens = np.array([0, 1, 2, 3, 15, 16, 17, 31, 32, 33, 47, 48, 49, 63, 64, 65, 0, 0, 1000, 7],
                    dtype=np.int64)
    off = np.zeros(len(lens) + 1, dtype=np.int64)
    off[1:] = np.cumsum(lens) + 3  # shift every start by 3 bytes
    off[0] = 3
    data = ACGT[rng.integers(0, 4, size=int(off[-1]) + 5)]
    fs, ac, err = _run_set(cuda, [d], data, off)
    rfs, rac = oracle.dfa_walk([d.tmap], [16], [0], [d.accept], data, off)
    assert err == 0 and np.array_equal(fs, rfs) and np.array_equal(ac, rac)


def test_malformed_offsets_are_reported(cuda):
    rng = np.random.default_rng(1)
    d = random_dfa(4, np.arange(256), rng)
    data = rng.integers(0, 256, size=100, dtype=np.uint8)
    off = np.array([0, 10, 5, 50, 200], dtype=np.int64)   # decreasing and out of range
    _, _, err = _run_set(cuda, [d], data, off)
    assert err & 1


@pytest.mark.parametrize("seg_len", [0, 64])
def test_overlapping_offsets_are_refused(cuda, seg_len):
    # [0, T) twenty times (with the reversed strings [T, 0) between them): the
    # valid strings alone hold 20 T bytes, more work items than total_bytes = T
    # allows for, so the planner refuses the whole batch (bit 2) besides
    # reporting the reversed strings (bit 0)
    rng = np.random.default_rng(2)
    d = random_dfa(8, np.arange(256), rng)
    T = 2048 * 64
    data = rng.integers(0, 256, size=T, dtype=np.uint8)
    off = np.tile(np.array([0, T], dtype=np.int64), 20)
    _, _, err = _run_set(cuda, [d], data, off, seg_len=seg_len)
    assert err & 1 and err & 4
    # the same automaton on a well-formed batch afterwards (same scratch sizes)
    ok = np.array([0, T // 2, T], dtype=np.int64)
    _, _, err = _run_set(cuda, [d], data, ok, seg_len=seg_len)
    assert err == 0


def test_golden_byte_dfas_on_gpu(cuda, golden):
    for rec in golden["byte_dfa"]:
        N = rec["n_states"]
        t = np.array(rec["tmap"], dtype=np.uint8).reshape(256, rec["padded_states"])[:, :N]
        from trex_b200.workloads import ByteDFA
        d = ByteDFA(N, np.ascontiguousarray(t).reshape(-1), np.array(rec["accept"], np.uint8))
        strs = [bytes.fromhex(h) for h in rec["strings_hex"]]
        data = np.frombuffer(b"".join(strs), dtype=np.uint8).copy()
        off = np.zeros(len(strs) + 1, dtype=np.int64)
        np.cumsum([len(s) for s in strs], out=off[1:])
        for seg in (0, 64):
            fs, _, err = _run_set(cuda, [d], data, off, seg_len=seg)
            assert err == 0 and fs.tolist() == rec["final_state"]


def test_host_entry_point(cuda, oracle):
    from trex_b200.engine import DFASet
    rng = np.random.default_rng(9)
    dfas = [random_dfa(n, np.arange(256), rng) for n in (16, 8)]
    data, off, ids, _ = ragged_batch(3000, rng, median=300, hi=5000, n_dfas=2)
    s = DFASet(dfas)
    fs, ac, km, tm = s.run_host(data, off, ids)
    s.close()
    rfs, rac = oracle.dfa_walk([d.tmap for d in dfas], [16, 8], [0, 0], [d.accept for d in dfas],
                               data, off, ids)
    assert np.array_equal(fs, rfs) and np.array_equal(ac, rac)
    assert tm >= km >= 0


# ---- reference bridges --------------------------------------------------------------

PATTERNS = ["(a|b)*abb", "(0|(1(01*0)*1))*", "(b*ab*ab*)*b*", "(ab)*", "0x[0-9a-f]+",
            "[a-z][a-z0-9]*", "(a|b)*a(a|b)", "a*b*", "(ab|ba)*", "(a|b|c)*abc",
            "(if|else|while|for|return)", "((ab|cd)(ef|gh))+"]


def _strings(alpha, n, max_len, rng):
    return ["".join(rng.choice(list(alpha), size=rng.integers(0, max_len + 1))) for _ in range(n)]


def test_prefix_compose_bridge_matches_dfa_simulate(cuda):
    from trex_b200.gpu_bridge_prefix_compose import PrefixComposeGPUSimulator
    from trex_b200.regex_to_dfa import compile_regex
    from trex_b200.simulation import DFAMatrices
    rng = np.random.default_rng(123)
    sim = PrefixComposeGPUSimulator()
    for pat in PATTERNS:
        dfa = compile_regex(pat)
        eng = sim.create_engine(DFAMatrices(dfa))
        strs = _strings(sorted(dfa.alphabet), 200, 500, rng) + [""]
        assert eng.simulate_batch(strs) == [dfa.simulate(s) for s in strs], pat
        res, km, tm = eng.simulate_batch_timed(strs[:3])
        assert res == [dfa.simulate(s) for s in strs[:3]] and km >= 0 and tm >= 0
        assert eng.simulate_batch([]) == []
        eng.destroy()


def test_monoid_batch_bridge(cuda):
    from trex_b200.gpu_bridge_monoid_batch import MonoidBatchGPUSimulator
    from trex_b200.monoid import compute_monoid, simulate_monoid
    from trex_b200.regex_to_dfa import compile_regex
    from trex_b200.simulation import DFAMatrices
    rng = np.random.default_rng(77)
    sim = MonoidBatchGPUSimulator()
    for pat in PATTERNS[:6]:
        dfa = compile_regex(pat)
        dm = DFAMatrices(dfa)
        md = compute_monoid(dm)
        eng = sim.create_engine(md, dm, max_total_chars=2_000_000)
        strs = [""] + _strings(sorted(dfa.alphabet), 499, 200, rng)
        assert eng.simulate_batch(strs) == [simulate_monoid(md, dm, s) for s in strs], pat
        assert eng.simulate_batch(["", "", ""]) == [dfa.simulate("")] * 3
        long = ["".join(rng.choice(sorted(dfa.alphabet), size=400_000)) for _ in range(2)]
        assert eng.simulate_batch(long) == [simulate_monoid(md, dm, s) for s in long]
        eng.destroy()


def test_monoid_scan_bridge(cuda):
    from trex_b200.gpu_bridge_monoid import MonoidGPUSimulator
    from trex_b200.monoid import compute_monoid, simulate_monoid
    from trex_b200.regex_to_dfa import compile_regex
    from trex_b200.simulation import DFAMatrices
    rng = np.random.default_rng(5)
    sim = MonoidGPUSimulator()
    for pat in PATTERNS[:5]:
        dfa = compile_regex(pat)
        dm = DFAMatrices(dfa)
        md = compute_monoid(dm)
        eng = sim.create_engine(md, dm)
        strs = _strings(sorted(dfa.alphabet) + ["z"], 300, 300, rng)
        assert eng.simulate_batch(strs) == [simulate_monoid(md, dm, s) for s in strs], pat
        eng.destroy()


def test_reference_abi_capacity_and_init_errors(cuda):
    from trex_b200 import _lib
    import ctypes
    L = _lib.load()
    res = np.zeros(4, dtype=np.int32)
    off = np.array([0, 1, 2, 3, 4], dtype=np.int32)
    data = np.frombuffer(b"abab", dtype=np.uint8).copy()
    L.prefix_engine_destroy()
    assert L.prefix_engine_dispatch(_lib.ptr(data, ctypes.c_uint8), _lib.ptr(off, ctypes.c_int),
                                    _lib.ptr(res, ctypes.c_int), 4, 4, None, None) == -1
    tmap = np.tile(np.arange(2, dtype=np.uint8), 256)
    acc = np.array([1, 0], dtype=np.uint8)
    assert L.prefix_engine_init(_lib.ptr(tmap, ctypes.c_uint8), _lib.ptr(acc, ctypes.c_uint8),
                                0, 2, 32, 2, 2) == 0
    rc = L.prefix_engine_dispatch(_lib.ptr(data, ctypes.c_uint8), _lib.ptr(off, ctypes.c_int),
                                  _lib.ptr(res, ctypes.c_int), 4, 4, None, None)
    assert rc == -4  # capacity (the reference would overrun its buffers)
    L.prefix_engine_destroy()
