"""Family (b) on the GPU: per-position states with the decoupled look-back
scan, against the C oracle (pinned to the reference's prefix_scan_sequential
by tests/test_oracle_golden.py)."""

import numpy as np
import pytest

from trex_b200.workloads import ByteDFA, random_dfa

pytestmark = pytest.mark.gpu


def _scan(torch, dfa, data, off, tile_len, out_shift=0):
    from trex_b200.engine import DFASet
    s = DFASet([dfa])
    d_data = torch.from_numpy(np.ascontiguousarray(data if data.size else np.zeros(1, np.uint8))).cuda()
    d_off = torch.from_numpy(off.astype(np.int64)).cuda()
    total = data.size
    states = None
    if out_shift:
        buf = torch.empty(total + out_shift + 16, dtype=torch.uint8, device="cuda")
        states = buf[out_shift:out_shift + max(total, 1)]
    st, fs, ac, sc = s.scan(d_data[:total], d_off, 0, states=states, tile_len=tile_len)
    torch.cuda.synchronize()
    err = s.scan_error_word(sc, len(off) - 1, total, tile_len)
    s.close()
    return st.cpu().numpy()[:total], fs.cpu().numpy(), ac.cpu().numpy(), err


def _check(oracle, dfa, data, off, st, fs, ac):
    ref = oracle.dfa_positions(dfa.tmap, dfa.n_states, dfa.start, data, off)
    assert np.array_equal(st, ref), f"first mismatch at {np.flatnonzero(st != ref)[:5]}"
    rfs, rac = oracle.dfa_walk([dfa.tmap], [dfa.n_states], [dfa.start], [dfa.accept], data, off)
    assert np.array_equal(fs, rfs)
    assert np.array_equal(ac, rac)


@pytest.mark.parametrize("n_states", [2, 5, 8, 12, 16])
@pytest.mark.parametrize("tile_len", [64, 1000, 8192])
def test_scan_random_dfa(cuda, oracle, n_states, tile_len):
    rng = np.random.default_rng(n_states * 100 + tile_len)
    d = random_dfa(n_states, np.arange(256), rng)
    lens = np.array([0, 1, 15, 16, 17, 100, 5000, 70000, 0, 300000, 3], dtype=np.int64)
    off = np.zeros(len(lens) + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    data = rng.integers(0, 256, size=int(off[-1]), dtype=np.uint8)
    st, fs, ac, err = _scan(cuda, d, data, off, tile_len)
    assert err == 0
    _check(oracle, d, data, off, st, fs, ac)


def test_scan_non_synchronising_dfa(cuda, oracle):
    # a permutation automaton never synchronises: every tile keeps its full map
    rng = np.random.default_rng(4)
    perm = np.stack([rng.permutation(16) for _ in range(256)]).astype(np.uint8)
    acc = np.zeros(16, np.uint8); acc[[2, 9]] = 1
    d = ByteDFA(16, np.ascontiguousarray(perm.reshape(-1)), acc, start=5)
    lens = np.array([20000, 3, 50000], dtype=np.int64)
    off = np.zeros(4, dtype=np.int64); np.cumsum(lens, out=off[1:])
    data = rng.integers(0, 256, size=int(off[-1]), dtype=np.uint8)
    st, fs, ac, err = _scan(cuda, d, data, off, 512)
    assert err == 0
    _check(oracle, d, data, off, st, fs, ac)


def test_scan_sub_alphabet_and_many_strings(cuda, oracle):
    rng = np.random.default_rng(8)
    acgt = np.frombuffer(b"ACGT", dtype=np.uint8)
    d = random_dfa(16, acgt, rng)
    lens = rng.integers(0, 3000, size=3000)
    off = np.zeros(len(lens) + 1, dtype=np.int64); np.cumsum(lens, out=off[1:])
    data = acgt[rng.integers(0, 4, size=int(off[-1]))]
    st, fs, ac, err = _scan(cuda, d, data, off, 256)
    assert err == 0
    _check(oracle, d, data, off, st, fs, ac)


def test_scan_unaligned_output_and_offsets(cuda, oracle):
    rng = np.random.default_rng(9)
    d = random_dfa(12, np.arange(256), rng)
    off = np.array([5, 1000, 1001, 90000], dtype=np.int64)
    data = rng.integers(0, 256, size=90003, dtype=np.uint8)
    st, fs, ac, err = _scan(cuda, d, data, off, 333, out_shift=3)
    assert err == 0
    ref = oracle.dfa_positions(d.tmap, d.n_states, 0, data, np.concatenate([[0], off]))
    # bytes before the first string are not written; compare the strings only
    assert np.array_equal(st[5:90000], ref[5:90000])
    rfs, rac = oracle.dfa_walk([d.tmap], [12], [0], [d.accept], data, off)
    assert np.array_equal(fs, rfs) and np.array_equal(ac, rac)


def test_scan_golden_positions(cuda, golden):
    for rec in golden["byte_dfa"]:
        N = rec["n_states"]
        if N > 16:
            continue
        t = np.array(rec["tmap"], dtype=np.uint8).reshape(256, rec["padded_states"])[:, :N]
        d = ByteDFA(N, np.ascontiguousarray(t).reshape(-1), np.array(rec["accept"], np.uint8))
        strs = [bytes.fromhex(h) for h in rec["strings_hex"]]
        data = np.frombuffer(b"".join(strs), dtype=np.uint8).copy()
        off = np.zeros(len(strs) + 1, dtype=np.int64)
        np.cumsum([len(x) for x in strs], out=off[1:])
        st, fs, _, err = _scan(cuda, d, data, off, 64)
        assert err == 0
        for i in range(len(strs)):
            assert st[off[i]:off[i + 1]].tolist() == rec["positions"][i]
        assert fs.tolist() == rec["final_state"]


def test_scan_malformed_and_overlapping_offsets(cuda):
    rng = np.random.default_rng(4)
    dfa = random_dfa(8, np.arange(256), rng)
    T = 1 << 17
    data = rng.integers(0, 256, size=T, dtype=np.uint8)
    # a reversed string: bit 0
    _, _, _, err = _scan(cuda, dfa, data, np.array([0, 100, 50, T], dtype=np.int64), 64)
    assert err & 1
    # [0, T) twenty times: more tiles than total_bytes allows for, nothing is scanned (bit 3)
    _, _, _, err = _scan(cuda, dfa, data, np.tile(np.array([0, T], dtype=np.int64), 20), 64)
    assert err & 1 and err & 8
