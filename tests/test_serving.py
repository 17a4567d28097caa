"""Serving loop: admission and packing on the CPU; on the GPU, every request's
result in a continuous mix equals its result served alone and the oracle's."""

import collections
import threading
import time

import numpy as np
import pytest

from trex_b200.serving import Request, pack_batch, take_batch
from trex_b200.workloads import random_bool_nfa, random_dfa, random_prob_nfa


def _req(i, kind, eng, n):
    return Request(i, kind, eng, bytes([i % 251]) * n)


def test_take_batch_respects_capacities():
    q = collections.deque(_req(i, "dfa", 0, n) for i, n in enumerate([10, 20, 30, 40, 5]))
    b = take_batch(q, max_requests=10, max_bytes=60)
    assert [r.rid for r in b] == [0, 1, 2]          # 10 + 20 + 30; 40 would exceed 60
    assert [r.rid for r in q] == [3, 4]              # FIFO: the head waits, nothing skips it
    b = take_batch(q, max_requests=1, max_bytes=1000)
    assert [r.rid for r in b] == [3]
    assert take_batch(collections.deque(), 4, 100) == []


def test_pack_batch_orders_and_offsets():
    batch = [_req(0, "nfa", 1, 3), _req(1, "dfa", 2, 4), _req(2, "pnfa", 0, 2), _req(3, "nfa", 0, 0),
             _req(4, "dfa", 0, 5), _req(5, "nfa", 1, 1)]
    order, blob, doff, ids, roff, groups = pack_batch(batch)
    assert [r.rid for r in order] == [1, 4, 3, 0, 5, 2]
    assert list(doff) == [0, 4, 9] and list(ids) == [2, 0]
    assert list(roff) == [9, 9, 12, 13, 15]
    assert groups == [("nfa", 0, 0, 1), ("nfa", 1, 1, 2), ("pnfa", 0, 3, 1)]
    assert blob == b"".join(r.data for r in order)


@pytest.mark.gpu
def test_mix_equals_alone_and_oracle(cuda, oracle):
    torch = cuda
    from trex_b200.engine import NFA, PNFA, DFASet
    from trex_b200.serving import Server
    rng = np.random.default_rng(8)
    dfas = [random_dfa(n, np.arange(256), rng) for n in (16, 8, 12, 16)]
    nfas = [random_bool_nfa(rng, 64, 20, 0.05) for _ in range(3)]
    pnfas = [random_prob_nfa(rng, 64, 20) for _ in range(2)]
    srv = Server(dfas, nfas, pnfas, hbm_budget=64 << 20, max_batch_requests=512)
    reqs = []
    lock = threading.Lock()

    def client(seed):
        r = np.random.default_rng(seed)
        for _ in range(300):
            kind = ("dfa", "nfa", "pnfa")[int(r.integers(0, 3))]
            eng = int(r.integers(0, {"dfa": 4, "nfa": 3, "pnfa": 2}[kind]))
            n = int(r.integers(0, 3000)) if r.random() < 0.9 else 0
            hi = 256 if kind == "dfa" else 22   # a few bytes outside the NFAs' 20 symbols
            data = r.integers(0, hi, size=n, dtype=np.uint8).tobytes()
            q = srv.submit(kind, eng, data)
            with lock:
                reqs.append(q)
            if r.random() < 0.1:
                time.sleep(0.001)

    threads = [threading.Thread(target=client, args=(s,)) for s in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    srv.wait(reqs)
    st = srv.stats()
    assert st["requests"] == len(reqs) and st["batches"] >= 2
    # alone: each request as a batch of one through the plain engines; and the oracle
    dset = DFASet(dfas)
    nfa_h = [NFA(*x, unknown_rejects=True) for x in nfas]
    pnfa_h = [PNFA(*x) for x in pnfas]
    for q in reqs:
        d = np.frombuffer(q.data, dtype=np.uint8)
        off = np.array([0, len(d)], dtype=np.int64)
        dd = torch.from_numpy(d.copy() if d.size else np.zeros(1, np.uint8)).cuda()
        do = torch.from_numpy(off).cuda()
        if q.kind == "dfa":
            _, ac, _ = dset.run(dd, do, torch.tensor([q.engine], dtype=torch.int32, device="cuda"))
            fs_o, ac_o = oracle.dfa_walk([x.tmap for x in dfas], [x.n_states for x in dfas],
                                         [x.start for x in dfas], [x.accept for x in dfas], d, off,
                                         np.array([q.engine], np.int32))
            assert q.result == (bool(ac.item()), int(fs_o[0])) and bool(ac_o[0]) == q.result[0]
        elif q.kind == "nfa":
            fm, ac = nfa_h[q.engine].run(dd, do)
            T, s0, a0 = nfas[q.engine]
            fm_o, ac_o = oracle.nfa_bool(T, s0, a0, d, off, unknown_rejects=True)
            alone = (bool(ac.item()), int(fm.item()) & 0xFFFFFFFFFFFFFFFF)
            assert q.result == alone == (bool(ac_o[0]), int(fm_o[0]))
        else:
            ll, ac = pnfa_h[q.engine].run(dd, do, "bf16")
            assert q.result == (float(ll.item()), bool(ac.item()))
    srv.close()


@pytest.mark.gpu
def test_server_from_file(cuda, oracle, tmp_path):
    from trex_b200 import automata_io
    from trex_b200.serving import Server
    rng = np.random.default_rng(8)
    dfas = [random_dfa(12, np.arange(256), rng), random_dfa(16, np.arange(256), rng)]
    nfas = [random_bool_nfa(rng, 64, 20)]
    pnfas = [random_prob_nfa(rng, 64, 20)]
    path = automata_io.save(tmp_path / "served", dfas, nfas, pnfas)
    srv = Server.from_file(path, hbm_budget=64 << 20, max_batch_requests=256)
    items = [("dfa", i % 2, rng.integers(0, 256, size=int(rng.integers(0, 3000)), dtype=np.uint8).tobytes())
             for i in range(40)]
    items += [("nfa", 0, rng.integers(0, 20, size=500, dtype=np.uint8).tobytes()) for _ in range(10)]
    reqs = srv.submit_many(items)
    res = srv.wait(reqs, timeout=120)
    srv.close()
    for (kind, eng, data), r in zip(items, res):
        d = np.frombuffer(data, np.uint8)
        off = np.array([0, len(data)], np.int64)
        if kind == "dfa":
            fs, ac = oracle.dfa_walk([dfas[eng].tmap], [dfas[eng].n_states], [0], [dfas[eng].accept], d, off)
            assert r == (bool(ac[0]), int(fs[0]))
        else:
            _, ac = oracle.nfa_bool(*nfas[0], d, off, unknown_rejects=True)
            assert r[0] == bool(ac[0])
