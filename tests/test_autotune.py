"""Autotuner: cache keys and file round trip on the CPU; on the GPU, a tuned
batch and scan give the oracle's results and a second call is served from the
cache."""

import json

import numpy as np
import pytest

from trex_b200.autotune import SCAN_CANDIDATES, SEG_CANDIDATES, Autotuner, _pow2_ceil


def test_pow2_ceil():
    assert [_pow2_ceil(x) for x in (0, 1, 2, 3, 4, 5, 1000, 2048, 2049)] == [1, 1, 2, 4, 4, 8, 1024, 2048, 4096]


def test_sample_is_evenly_spaced_and_bounded():
    off = np.arange(0, 1001 * 100, 100, dtype=np.int64)   # 1000 strings of 100 bytes
    idx = Autotuner._sample(off, 10_000)
    assert len(idx) <= 101 and idx[0] == 0 and np.all(np.diff(idx) == idx[1] - idx[0])
    assert len(Autotuner._sample(off, 10 ** 9)) == 1000


def test_cache_file_round_trip(tmp_path):
    p = tmp_path / "tune.json"
    t = Autotuner(cache_path=str(p))
    t.cache["dfa:N<=16:k<=4:len<2048"] = 4
    t._save()
    assert json.loads(p.read_text())["dfa:N<=16:k<=4:len<2048"] == 4
    assert Autotuner(cache_path=str(p)).cache == t.cache


@pytest.mark.gpu
def test_tuned_batch_matches_oracle_and_caches(cuda, oracle, tmp_path):
    from trex_b200.engine import DFASet
    from trex_b200.workloads import random_dfa
    rng = np.random.default_rng(3)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    dfas = [random_dfa(16, acgt, rng), random_dfa(8, np.frombuffer(b"ab", np.uint8), rng),
            random_dfa(12, np.arange(256), rng)]
    n = 6000
    lens = rng.integers(0, 5000, size=n)
    off = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=off[1:])
    ids = (np.arange(n) % 3).astype(np.int32)
    data = rng.integers(0, 256, size=int(off[-1]), dtype=np.uint8)
    for i in range(n):   # strings of the small-alphabet automata use their letters
        a, b = off[i], off[i + 1]
        if ids[i] == 0:
            data[a:b] = acgt[data[a:b] & 3]
        elif ids[i] == 1:
            data[a:b] = np.frombuffer(b"ab", np.uint8)[data[a:b] & 1]
    d_data, d_off, d_ids = (cuda.from_numpy(x).cuda() for x in (data, off, ids))
    s = DFASet(dfas)
    t = Autotuner(cache_path=str(tmp_path / "t.json"), warmup=1, reps=2)
    rep = t.tune_batch(s, d_data, d_off, d_ids)
    assert rep.seg_len in SEG_CANDIDATES
    assert rep.kgram[2] == 1 and rep.kgram[0] in (1, 2, 4) and rep.kgram[1] in (1, 2, 4, 8)
    assert [s.get_kgram(i) for i in range(3)] == rep.kgram
    assert any(x["what"] == "seg_len" for x in rep.sweep)
    fs, ac, _ = s.run(d_data, d_off, d_ids, seg_len=rep.seg_len)
    rfs, rac = oracle.dfa_walk([x.tmap for x in dfas], [x.n_states for x in dfas], [0, 0, 0],
                               [x.accept for x in dfas], data, off, ids)
    assert np.array_equal(fs.cpu().numpy(), rfs) and np.array_equal(ac.cpu().numpy(), rac)
    rep2 = Autotuner(cache_path=str(tmp_path / "t.json")).tune_batch(s, d_data, d_off, d_ids)
    assert rep2.sweep == [] and rep2.kgram == rep.kgram and rep2.seg_len == rep.seg_len
    s.close()


@pytest.mark.gpu
def test_tuned_scan_matches_oracle(cuda, oracle, tmp_path):
    from trex_b200.engine import DFASet
    from trex_b200.workloads import random_dfa
    rng = np.random.default_rng(4)
    d = random_dfa(16, np.arange(256), rng)
    off = np.array([0, 300_000, 300_000, 1_000_000], np.int64)
    data = rng.integers(0, 256, size=int(off[-1]), dtype=np.uint8)
    s = DFASet([d])
    d_data, d_off = cuda.from_numpy(data).cuda(), cuda.from_numpy(off).cuda()
    tile, sweep = Autotuner(cache_path=str(tmp_path / "s.json"), warmup=1, reps=2).tune_scan(s, 0, d_data, d_off)
    assert tile in SCAN_CANDIDATES and len(sweep) == len(SCAN_CANDIDATES)
    st, fs, ac, _ = s.scan(d_data, d_off, 0, tile_len=tile)
    assert np.array_equal(st.cpu().numpy()[:data.size], oracle.dfa_positions(d.tmap, 16, 0, data, off))
    s.close()
