"""K-gram walking of the ragged DFA kernel (the reference's monoid K-gram path,
src/kgram.py, cuda/monoid_batch.cu:103-125): results must equal the byte walk
and the C oracle bit for bit, for in-alphabet strings (gram fast path) and for
strings with other bytes (per-byte fallback), split strings included."""

import numpy as np
import pytest

from trex_b200.workloads import ByteDFA, random_dfa

pytestmark = pytest.mark.gpu

ACGT = np.frombuffer(b"ACGT", dtype=np.uint8)
AB = np.frombuffer(b"ab", dtype=np.uint8)
HEX16 = np.arange(0x61, 0x71, dtype=np.uint8)   # 'a'..'p': 4-bit codes


def _with_sink(d: ByteDFA) -> ByteDFA:
    """Bytes outside the alphabet go to a rejecting sink (DFA.simulate semantics)."""
    N = d.n_states + 1
    t = np.full((256, N), N - 1, dtype=np.uint8)
    old = d.tmap.reshape(256, d.n_states)
    t[d.symbols, :d.n_states] = old[d.symbols]
    acc = np.concatenate([d.accept, [0]]).astype(np.uint8)
    return ByteDFA(n_states=N, tmap=np.ascontiguousarray(t.reshape(-1)), accept=acc, start=d.start,
                   symbols=d.symbols)


def _batch(rng, alphabet, n=1500, dirty=0.3, maxlen=6000):
    lens = rng.integers(0, maxlen, size=n)
    lens[:8] = [0, 1, 2, 3, 31, 32, 33, 2049]
    off = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    data = alphabet[rng.integers(0, len(alphabet), size=int(off[-1]))]
    # some strings get stray bytes (the per-byte fallback), some stay clean (the gram path)
    for i in np.flatnonzero(rng.random(n) < dirty):
        a, b = off[i], off[i + 1]
        if b > a:
            k = int(rng.integers(1, 4))
            data[rng.integers(a, b, size=k)] = rng.integers(0, 256, size=k, dtype=np.uint8)
    return data.astype(np.uint8), off


def _run(torch, dfas, data, off, ids, kgram, seg_len=0):
    from trex_b200.engine import DFASet
    s = DFASet(dfas, kgram=kgram)
    d_data = torch.from_numpy(data if data.size else np.zeros(1, np.uint8)).cuda()
    fs, ac, _ = s.run(d_data[:data.size], torch.from_numpy(off).cuda(),
                      torch.from_numpy(ids.astype(np.int32)).cuda(), seg_len=seg_len)
    torch.cuda.synchronize()
    err = s.last_error_word()
    ks = [s.get_kgram(i) for i in range(len(dfas))]
    s.close()
    return fs.cpu().numpy(), ac.cpu().numpy(), err, ks


def test_kgram_max_by_alphabet(cuda):
    from trex_b200.engine import DFASet
    rng = np.random.default_rng(1)
    dfas = [random_dfa(16, ACGT, rng), random_dfa(8, AB, rng), random_dfa(12, HEX16, rng),
            random_dfa(16, np.arange(256), rng), random_dfa(20, AB, rng),
            _with_sink(random_dfa(9, ACGT, rng))]
    s = DFASet(dfas)
    assert [s.kgram_max(i) for i in range(len(dfas))] == [4, 8, 2, 1, 1, 4]
    assert s.get_kgram(0) == 1
    with pytest.raises(Exception):
        s.set_kgram(0, 8)   # 4 letters: 2-bit codes, at most 4 per gram
    s.set_kgram(0, 0)
    assert s.get_kgram(0) == 4
    s.close()


@pytest.mark.parametrize("alphabet,n_states,k", [(ACGT, 16, 4), (ACGT, 16, 2), (ACGT, 8, 4),
                                                 (AB, 16, 8), (AB, 8, 4), (AB, 5, 2),
                                                 (HEX16, 16, 2), (HEX16, 7, 2)])
@pytest.mark.parametrize("sink", [False, True])
def test_kgram_matches_oracle(cuda, oracle, alphabet, n_states, k, sink):
    rng = np.random.default_rng(n_states * 100 + k + (7 if sink else 0))
    d = random_dfa(n_states - 1 if sink else n_states, alphabet, rng)
    if sink:
        d = _with_sink(d)
    data, off = _batch(rng, alphabet)
    ids = np.zeros(len(off) - 1, np.int32)
    fs, ac, err, ks = _run(cuda, [d], data, off, ids, [k], seg_len=256)
    assert err == 0 and ks == [k]
    rfs, rac = oracle.dfa_walk([d.tmap], [d.n_states], [d.start], [d.accept], data, off)
    assert np.array_equal(fs, rfs), np.flatnonzero(fs != rfs)[:8]
    assert np.array_equal(ac, rac)


def test_kgram_mixed_set_default_segments(cuda, oracle):
    # gram and byte automata in one ragged launch, default segment length
    rng = np.random.default_rng(5)
    dfas = [random_dfa(16, ACGT, rng), random_dfa(16, np.arange(256), rng), random_dfa(8, AB, rng),
            _with_sink(random_dfa(11, HEX16, rng))]
    alpha = np.concatenate([ACGT, AB, HEX16])
    data, off = _batch(rng, alpha, n=3000, dirty=0.2, maxlen=9000)
    ids = (np.arange(len(off) - 1) % 4).astype(np.int32)
    fs0, ac0, err0, _ = _run(cuda, dfas, data, off, ids, None)
    fs, ac, err, ks = _run(cuda, dfas, data, off, ids, 0)
    assert ks == [4, 1, 8, 2]
    assert err == 0 and err0 == 0
    rfs, rac = oracle.dfa_walk([x.tmap for x in dfas], [x.n_states for x in dfas],
                               [x.start for x in dfas], [x.accept for x in dfas], data, off, ids)
    assert np.array_equal(fs0, rfs) and np.array_equal(fs, rfs) and np.array_equal(ac, rac)


@pytest.mark.parametrize("k", [1, 2])
def test_split_string_rewalk_marks_repeat(cuda, oracle, k):
    """A 5-state automaton with a sink over two letters, cut into 256-byte items:
    many items guess their entry wrong, some fix-ups never meet the chain, and the
    fix-up list overflows, so one item can be marked for a re-walk twice, with the
    chain's assumed entry and with a walked one. The walked entry must win whatever
    the order of the marks; the order changes from run to run, so the case runs
    several times."""
    rng = np.random.default_rng(5 * 100 + 2 + 7)
    d = _with_sink(random_dfa(4, AB, rng))
    data, off = _batch(rng, AB)
    ids = np.zeros(len(off) - 1, np.int32)
    rfs, rac = oracle.dfa_walk([d.tmap], [d.n_states], [d.start], [d.accept], data, off)
    for _ in range(6):
        fs, ac, err, _ = _run(cuda, [d], data, off, ids, [k], seg_len=256)
        assert err == 0
        assert np.array_equal(fs, rfs), np.flatnonzero(fs != rfs)[:8]
        assert np.array_equal(ac, rac)
