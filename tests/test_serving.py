"""Serving loop: admission and packing on the CPU; on the GPU, every request's
result in a continuous mix equals its result served alone and the oracle's."""

import collections
import threading
import time

import numpy as np
import pytest

from trex_b200.serving import Bulk, Request, plan_batch, take_batch
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


def _bulk(rid, kind, engines, lens, seed=0):
    rng = np.random.default_rng(seed)
    off = np.zeros(len(lens) + 1, dtype=np.int64)
    off[1:] = np.cumsum(lens)
    data = rng.integers(0, 256, size=int(off[-1]), dtype=np.uint8)
    n = len(lens)
    z = np.zeros(n)
    return Bulk(rid, kind, np.asarray(engines, dtype=np.int32), data, off, z, z.copy(), z.copy(), z.copy())


def _emulate(plan):
    """The batch bytes a plan gives the kernels: host copies, then the device scatter."""
    out = np.zeros(plan.total, dtype=np.uint8)
    for off, src in plan.copies:
        a = np.frombuffer(src, dtype=np.uint8) if isinstance(src, (bytes, bytearray)) else src
        out[off:off + len(a)] = a
    stage = np.zeros(plan.stage_bytes, dtype=np.uint8)
    for off, a in plan.stage:
        stage[off:off + len(a)] = a
    for i in range(len(plan.stage_dst)):
        a, b = int(plan.stage_off[i]), int(plan.stage_off[i + 1])
        out[int(plan.stage_dst[i]):int(plan.stage_dst[i]) + b - a] = stage[a:b]
    return out


def _strings(plan, out):
    """(kind, engine, bytes) of every output slot: DFA slots, then the others."""
    res = {}
    for k in range(plan.nd):
        res[("dfa", k)] = (int(plan.ids[k]), out[plan.doff[k]:plan.doff[k + 1]].tobytes())
    for kind, eng, first, cnt in plan.groups:
        for k in range(first, first + cnt):
            res[("rest", k)] = (kind, eng, out[plan.roff[k]:plan.roff[k + 1]].tobytes())
    return res


def test_plan_batch_orders_and_offsets():
    batch = [_req(0, "nfa", 1, 3), _req(1, "dfa", 2, 4), _req(2, "pnfa", 0, 2), _req(3, "nfa", 0, 0),
             _req(4, "dfa", 0, 5), _req(5, "nfa", 1, 1)]
    plan = plan_batch(batch)
    assert list(plan.doff) == [0, 4, 9] and list(plan.ids) == [2, 0]
    assert list(plan.roff) == [9, 9, 12, 13, 15]
    assert plan.groups == [("nfa", 0, 0, 1), ("nfa", 1, 1, 2), ("pnfa", 0, 3, 1)]
    assert [(r.rid, j) for r, j in plan.reqs] == [(1, 0), (4, 1), (0, 1), (2, 3), (3, 0), (5, 2)]
    assert len(plan.stage_dst) == 0 and plan.parts == []
    out = _emulate(plan)
    assert out.tobytes() == b"".join(r.data for r in (batch[1], batch[4], batch[3], batch[0], batch[5],
                                                      batch[2]))


def test_take_batch_splits_bulk_submissions():
    b = _bulk(10, "nfa", [0] * 6, [10, 20, 30, 0, 40, 5])
    q = collections.deque([_req(0, "dfa", 0, 15), b, _req(1, "dfa", 0, 5)])
    t = take_batch(q, max_requests=10, max_bytes=80)
    assert t[0].rid == 0 and t[1] == (b, 0, 4)          # 15 + 10 + 20 + 30 + 0 = 75; 40 more would not fit
    assert b.next == 4 and q[0] is b
    t = take_batch(q, max_requests=1, max_bytes=1000)
    assert t == [(b, 4, 5)] and b.next == 5               # the request cap
    t = take_batch(q, max_requests=10, max_bytes=1000)
    assert t[0] == (b, 5, 6) and t[1].rid == 1 and not q  # the rest of b, then the next request
    big = _bulk(20, "dfa", [0, 0], [50, 50])
    q = collections.deque([_req(2, "dfa", 0, 60), big])
    assert [e.rid for e in take_batch(q, 10, 100)] == [2] and q[0] is big and big.next == 0


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_plan_batch_with_bulk_places_every_string(seed):
    rng = np.random.default_rng(seed)
    batch = []
    for i in range(12):
        if rng.random() < 0.5:
            kind = ("dfa", "nfa", "pnfa")[int(rng.integers(0, 3))]
            batch.append(_req(i, kind, int(rng.integers(0, 3)), int(rng.integers(0, 40))))
        else:
            kind = ("dfa", "nfa", "pnfa")[int(rng.integers(0, 3))]
            n = int(rng.integers(1, 30))
            bk = _bulk(100 + i, kind, rng.integers(0, 3, size=n), rng.integers(0, 50, size=n), seed=i)
            lo = int(rng.integers(0, n))
            batch.append((bk, lo, int(rng.integers(lo + 1, n + 1))))
    plan = plan_batch(batch)
    out = _emulate(plan)
    slots = _strings(plan, out)
    # every request and every bulk string sits in its output slot, on its automaton
    seen = set()
    for r, j in plan.reqs:
        key = ("dfa", j) if r.kind == "dfa" else ("rest", j)
        got = slots[key]
        assert got == ((r.engine, r.data) if r.kind == "dfa" else (r.kind, r.engine, r.data))
        seen.add(key)
    for bk, lo, hi, js in plan.parts:
        for i, j in zip(range(lo, hi), js.tolist()):
            data = bk.data[bk.offsets[i]:bk.offsets[i + 1]].tobytes()
            key = ("dfa", j) if bk.kind == "dfa" else ("rest", j)
            got = slots[key]
            e = int(bk.engines[i])
            assert got == ((e, data) if bk.kind == "dfa" else (bk.kind, e, data))
            seen.add(key)
    assert len(seen) == len(slots) == plan.nd + plan.nr
    # groups tile the non-DFA part in (kind, engine) order
    assert sum(c for *_, c in plan.groups) == plan.nr
    keys = [(("dfa", "nfa", "pnfa").index(k), e) for k, e, _, _ in plan.groups]
    assert keys == sorted(keys) and len(set(keys)) == len(keys)


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


@pytest.mark.gpu
def test_scatter_strings_places_and_checks(cuda):
    """trex_scatter_strings against a host copy. With bad entries (a place past
    the destination, a place before it, a source size that ends inside the last
    string) those bytes are not written, the error word is set, the other
    strings still land, and nothing past dst_bytes changes."""
    torch = cuda
    from trex_b200 import _lib
    L = _lib.load()
    rng = np.random.default_rng(5)
    for n, hi, bad in ((1, 5000, False), (300, 3000, False), (4000, 200, False), (300, 3000, True),
                       (4000, 200, True)):
        lens = rng.integers(0, hi, size=n)
        lens[rng.random(n) < 0.1] = 0
        lens[:2] = np.maximum(lens[:2], 1)
        lens[-1] = max(lens[-1], 1)
        soff = np.zeros(n + 1, dtype=np.int64)
        soff[1:] = np.cumsum(lens)
        total = int(soff[-1])
        src = rng.integers(0, 256, size=total, dtype=np.uint8)
        perm = rng.permutation(n)
        doff = np.zeros(n + 1, dtype=np.int64)
        doff[1:] = np.cumsum(lens[perm])
        dst_begin = np.empty(n, dtype=np.int64)
        dst_begin[perm] = doff[:-1]
        slot = dst_begin.copy()
        src_bytes = total
        if bad:
            dst_begin[0] = total + 8              # wholly past the destination
            dst_begin[1] = -(int(lens[1]) + 3)    # wholly before it
            src_bytes = total - 1                 # the source ends inside the last string
        d_src = torch.from_numpy(src).cuda()
        d_soff = torch.from_numpy(soff).cuda()
        d_dst = torch.full((total + 64,), 7, dtype=torch.uint8, device="cuda")
        d_db = torch.from_numpy(dst_begin).cuda()
        d_err = torch.zeros(1, dtype=torch.int32, device="cuda")
        _lib.check(L.trex_scatter_strings(d_src.data_ptr(), src_bytes, d_soff.data_ptr(), n,
                                          d_dst.data_ptr(), total, d_db.data_ptr(), d_err.data_ptr(),
                                          torch.cuda.current_stream().cuda_stream), "scatter")
        got = d_dst.cpu().numpy()
        assert (got[total:] == 7).all()
        assert bool(int(d_err.item()) & 1) == bad
        for i in range(n):
            a = int(slot[i])
            if bad and i < 2:
                assert (got[a:a + lens[i]] == 7).all()
            elif bad and i == n - 1:
                assert (got[a:a + lens[i] - 1] == src[soff[i]:soff[i + 1] - 1]).all()
            else:
                assert (got[a:a + lens[i]] == src[soff[i]:soff[i + 1]]).all()


@pytest.mark.gpu
def test_bulk_submissions_match_batched_runs(cuda, oracle):
    """Bulk submissions (arrays in, arrays out) of all three kinds, mixed with
    single requests and split over several batches, give each request the result
    of the engines run directly on the same strings, and the oracle's."""
    torch = cuda
    from trex_b200.engine import NFA, PNFA, DFASet
    from trex_b200.serving import Server
    rng = np.random.default_rng(9)
    dfas = [random_dfa(n, np.arange(256), rng) for n in (16, 8, 12, 16)]
    nfas = [random_bool_nfa(rng, 64, 20, 0.05) for _ in range(3)]
    pnfas = [random_prob_nfa(rng, 64, 20) for _ in range(2)]
    srv = Server(dfas, nfas, pnfas, hbm_budget=16 << 20, max_batch_requests=256)
    n_eng = {"dfa": 4, "nfa": 3, "pnfa": 2}
    subs = []
    singles = []
    for rep in range(3):
        for kind in ("dfa", "nfa", "pnfa"):
            n = int(rng.integers(200, 900))
            lens = rng.integers(0, 4000, size=n)
            lens[rng.random(n) < 0.05] = 0
            off = np.zeros(n + 1, dtype=np.int64)
            off[1:] = np.cumsum(lens)
            hi = 256 if kind == "dfa" else 22
            data = rng.integers(0, hi, size=int(off[-1]), dtype=np.uint8)
            eng = rng.integers(0, n_eng[kind], size=n)
            subs.append((kind, eng, data, off, srv.submit_arrays(kind, eng, data, off)))
            for _ in range(20):
                d = rng.integers(0, hi, size=int(rng.integers(0, 3000)), dtype=np.uint8).tobytes()
                singles.append(srv.submit(kind, int(rng.integers(0, n_eng[kind])), d))
    res = srv.wait([b for *_, b in subs] + singles, timeout=300)
    st = srv.stats()
    assert st["requests"] == sum(len(s[1]) for s in subs) + len(singles)
    assert st["batches"] > len(subs)   # the 16 MiB budget splits the submissions
    srv.close()
    dset = DFASet(dfas)
    nfa_h = [NFA(*x, unknown_rejects=True) for x in nfas]
    pnfa_h = [PNFA(*x) for x in pnfas]
    for (kind, eng, data, off, b), (r0, r1) in zip(subs, res):
        assert b.done and b.error is None and (b.t_done > 0).all()
        dd = torch.from_numpy(data if data.size else np.zeros(1, np.uint8)).cuda()
        if kind == "dfa":
            fs, ac, _ = dset.run(dd, torch.from_numpy(off).cuda(),
                                 torch.from_numpy(eng.astype(np.int32)).cuda())
            assert (r0 == ac.cpu().numpy().astype(bool)).all() and (r1 == fs.cpu().numpy()).all()
            fs_o, ac_o = oracle.dfa_walk([x.tmap for x in dfas], [x.n_states for x in dfas],
                                         [x.start for x in dfas], [x.accept for x in dfas], data, off,
                                         eng.astype(np.int32))
            assert (r1 == fs_o).all() and (r0 == ac_o.astype(bool)).all()
            continue
        for e in range(n_eng[kind]):
            idx = np.flatnonzero(eng == e)
            sub = np.concatenate([data[off[i]:off[i + 1]] for i in idx] + [np.zeros(0, np.uint8)])
            so = np.zeros(len(idx) + 1, dtype=np.int64)
            so[1:] = np.cumsum(off[idx + 1] - off[idx])
            ds = torch.from_numpy(sub if sub.size else np.zeros(1, np.uint8)).cuda()
            if kind == "nfa":
                fm, ac = nfa_h[e].run(ds, torch.from_numpy(so).cuda())
                assert (r0[idx] == ac.cpu().numpy().astype(bool)).all()
                assert (r1[idx] == fm.cpu().numpy().view(np.uint64)).all()
                fm_o, ac_o = oracle.nfa_bool(*nfas[e], sub, so, unknown_rejects=True)
                assert (r1[idx] == np.asarray(fm_o).astype(np.uint64)).all()
            else:
                ll, ac = pnfa_h[e].run(ds, torch.from_numpy(so).cuda(), "bf16")
                assert (r0[idx] == ll.cpu().numpy()).all()
                assert (r1[idx] == ac.cpu().numpy().astype(bool)).all()
    dset.close()
    for m in nfa_h + pnfa_h:
        m.close()


@pytest.mark.gpu
def test_submit_arrays_arguments(cuda, oracle):
    """The bulk form's checks and edge cases: an empty submission is done at once;
    engine ids out of range, offsets that run backwards or past the data, and a
    request larger than a slot are refused at submit; bytes data and a scalar
    engine id are accepted and give the oracle's results."""
    from trex_b200.serving import Server
    rng = np.random.default_rng(12)
    dfas = [random_dfa(16, np.arange(256), rng) for _ in range(2)]
    nfas = [random_bool_nfa(rng, 64, 20, 0.05)]
    srv = Server(dfas, nfas, [], hbm_budget=8 << 20, max_batch_requests=64)
    try:
        b = srv.submit_arrays("dfa", [], b"", [0])
        assert b.done and b.n == 0
        (r0, r1), = srv.wait([b])
        assert len(r0) == 0 and len(r1) == 0
        data = rng.integers(0, 256, size=1000, dtype=np.uint8)
        with pytest.raises(ValueError):
            srv.submit_arrays("dfa", [0, 2], data, [0, 10, 20])          # no DFA 2
        with pytest.raises(ValueError):
            srv.submit_arrays("dfa", 0, data, [0, 30, 20])               # backwards
        with pytest.raises(ValueError):
            srv.submit_arrays("dfa", 0, data, [0, 10, 2000])             # past the data
        with pytest.raises(ValueError):
            srv.submit_arrays("pnfa", 0, data, [0, 10])                  # no probabilistic NFA
        with pytest.raises(ValueError):
            srv.submit_arrays("dfa", 0, np.zeros(srv.max_bytes + 1, np.uint8), [0, srv.max_bytes + 1])
        off = np.array([0, 0, 17, 300, 1000], dtype=np.int64)
        b = srv.submit_arrays("dfa", 1, data.tobytes(), off)             # bytes, one id for all
        c = srv.submit_arrays("nfa", 0, (data % 22).astype(np.uint8), off)
        (ac, fs), (ac2, fm) = srv.wait([b, c])
        fs_o, ac_o = oracle.dfa_walk([dfas[1].tmap], [dfas[1].n_states], [dfas[1].start], [dfas[1].accept],
                                     data, off)
        assert np.array_equal(fs, fs_o) and np.array_equal(ac, ac_o.astype(bool))
        fm_o, ac2_o = oracle.nfa_bool(*nfas[0], (data % 22).astype(np.uint8), off, unknown_rejects=True)
        assert np.array_equal(fm, np.asarray(fm_o).astype(np.uint64)) and np.array_equal(ac2, ac2_o.astype(bool))
        assert (b.latency_ms > 0).all() and (c.latency_ms > 0).all()
    finally:
        srv.close()
