"""Serving: a continuous-batching request loop over resident automata.

The reference serves nothing (it runs one static batch per call,
cuda/monoid_batch.cu:498-588); this loop is the serving layer of the B200
engine:

* tables stay in HBM: one DFA set for all byte DFAs (up to 64, one ragged
  launch carries any mix of them, a DFA id per string), a handle per Boolean
  NFA and per probabilistic NFA;
* admission by memory footprint: the HBM budget is split over the batch
  slots; a request joins the forming batch while the slot's byte and request
  capacities allow, and waits otherwise (a request larger than a slot is
  refused at submit);
* two lanes with two slots each: DFA and Boolean NFA requests (walked in
  bulk, milliseconds even for long strings) and probabilistic NFA requests
  (a sequential product chain per string, latency proportional to its
  length), so a long probabilistic request never holds back the others;
* continuous batching: while one slot's batch runs on its stream, the loop
  packs the requests that arrived meanwhile into the lane's other slot and
  launches it; a finished slot is drained (results handed to their requests)
  and reused at once;
* CUDA graphs: the DFA part of a batch (host-to-device copies, the planning
  and ragged kernels, device-to-host copies) is captured once per slot and
  size bucket (requests and bytes rounded up to powers of two, padded with
  empty strings) and replayed;
* per-request latency (submit to result) with p50/p99 and throughput.

Results: DFA requests give (accept, final_state), NFA requests
(accept, final_mask), probabilistic NFA requests (log_likelihood, accept).
A request's result does not depend on what else is in its batch.
"""

from __future__ import annotations

import collections
import threading
import time
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

KINDS = ("dfa", "nfa", "pnfa")
kAuxStreams = 4   # extra streams of a fast-lane slot


@dataclass(slots=True)
class Request:
    """One match request. The server sets result (or error) and then t_done;
    ``done`` is true from then on (Server.wait blocks until requests are done).
    A request holds no lock or event of its own: under load the process
    creates thousands of them a second, and every object the garbage
    collector tracks lengthens its full passes (which showed up as p99
    latency spikes of tens of milliseconds)."""

    rid: int
    kind: str
    engine: int
    data: bytes
    t_submit: float = 0.0
    t_done: float = 0.0
    result: object = None
    error: Optional[str] = None

    @property
    def done(self) -> bool:
        return self.t_done > 0.0 or self.error is not None

    @property
    def latency_ms(self) -> float:
        return (self.t_done - self.t_submit) * 1e3


def take_batch(queue: collections.deque, max_requests: int, max_bytes: int) -> list:
    """FIFO admission: pop requests while the batch stays within both
    capacities; the first request that does not fit stays at the head."""
    batch, nbytes = [], 0
    while queue and len(batch) < max_requests:
        r = queue[0]
        if nbytes + len(r.data) > max_bytes:
            break
        queue.popleft()
        batch.append(r)
        nbytes += len(r.data)
    return batch


def pack_batch(batch: Sequence[Request]):
    """Order a batch as [DFA requests | NFA requests by engine | PNFA requests
    by engine]. Returns (order, blob, dfa_offsets, dfa_ids, rest_offsets,
    groups) where groups lists (kind, engine, first, count) over the non-DFA
    part and both offset arrays are absolute into blob."""
    dfa = [r for r in batch if r.kind == "dfa"]
    rest = sorted((r for r in batch if r.kind != "dfa"), key=lambda r: (KINDS.index(r.kind), r.engine))
    order = dfa + rest
    lens = np.fromiter((len(r.data) for r in order), dtype=np.int64, count=len(order))
    ends = np.cumsum(lens)
    starts = ends - lens
    blob = b"".join(r.data for r in order)
    nd = len(dfa)
    dfa_off = np.empty(nd + 1, dtype=np.int64)
    dfa_off[0] = 0
    dfa_off[1:] = ends[:nd]
    dfa_ids = np.fromiter((r.engine for r in dfa), dtype=np.int32, count=nd)
    rest_off = np.empty(len(rest) + 1, dtype=np.int64)
    rest_off[0] = ends[nd - 1] if nd else 0
    rest_off[1:] = ends[nd:]
    groups = []
    i = 0
    while i < len(rest):
        j = i
        while j < len(rest) and rest[j].kind == rest[i].kind and rest[j].engine == rest[i].engine:
            j += 1
        groups.append((rest[i].kind, rest[i].engine, i, j - i))
        i = j
    return order, blob, dfa_off, dfa_ids, rest_off, groups


def _bucket(x: int, lo: int) -> int:
    b = lo
    while b < x:
        b <<= 1
    return b


class _Slot:
    """Device and pinned host buffers of one in-flight batch."""

    def __init__(self, torch, dev, lane: str, max_requests: int, max_bytes: int, dfa_scratch: int):
        self.lane = lane
        u8, i32, i64, f64 = torch.uint8, torch.int32, torch.int64, torch.float64
        R, B = max_requests, max_bytes
        self.stream = torch.cuda.Stream(device=dev)
        self.d_data = torch.zeros(B + 16, dtype=u8, device=dev)
        self.d_doff = torch.zeros(R + 1, dtype=i64, device=dev)
        self.d_ids = torch.zeros(max(R, 1), dtype=i32, device=dev)
        self.d_roff = torch.zeros(R + 1, dtype=i64, device=dev)
        self.d_fs = torch.zeros(max(R, 1), dtype=u8, device=dev)
        self.d_ac = torch.zeros(max(R, 1), dtype=u8, device=dev)
        self.d_ac2 = torch.zeros(max(R, 1), dtype=u8, device=dev)
        self.d_mask = torch.zeros(max(R, 1), dtype=i64, device=dev)
        self.d_ll = torch.zeros(max(R, 1), dtype=f64, device=dev)
        self.d_scratch = torch.zeros(max(dfa_scratch, 16), dtype=u8, device=dev)
        pin = dict(pin_memory=True)
        self.h_data = torch.zeros(B + 16, dtype=u8, **pin)
        self.h_doff = torch.zeros(R + 1, dtype=i64, **pin)
        self.h_ids = torch.zeros(max(R, 1), dtype=i32, **pin)
        self.h_roff = torch.zeros(R + 1, dtype=i64, **pin)
        self.h_fs = torch.zeros(max(R, 1), dtype=u8, **pin)
        self.h_ac = torch.zeros(max(R, 1), dtype=u8, **pin)
        self.h_ac2 = torch.zeros(max(R, 1), dtype=u8, **pin)
        self.h_mask = torch.zeros(max(R, 1), dtype=i64, **pin)
        self.h_ll = torch.zeros(max(R, 1), dtype=f64, **pin)
        self.event = torch.cuda.Event()
        # automaton groups of a fast-lane batch run side by side on these streams (each
        # group's kernel is sized by its strings, so a few strings take one SM); the
        # probabilistic lane runs its groups on its own stream
        n_aux = kAuxStreams if lane == "fast" else 0
        self.aux = [torch.cuda.Stream(device=dev) for _ in range(n_aux)]
        self.aux_ev = [torch.cuda.Event() for _ in range(n_aux)]
        self.ready = torch.cuda.Event()
        self.graphs = {}
        self.batch = None
        self.meta = None


class Server:
    """Continuous-batching server over resident automata (see the module docstring)."""

    def __init__(self, dfas=(), nfas=(), pnfas=(), *, hbm_budget: int = 1 << 30,
                 max_batch_requests: int = 1 << 14, pnfa_mode: str = "bf16", use_graphs: bool = True,
                 device: int = 0, pnfa_auto_threshold: int = 2048, precapture: bool = True,
                 gc_freeze: bool = True, nfa_streams: int = kAuxStreams):
        import torch
        from .engine import NFA, PNFA, DFASet
        self.torch = torch
        self.dev = torch.device("cuda", device)
        torch.cuda.set_device(self.dev)
        self.dfa_set = DFASet(list(dfas)) if len(dfas) else None
        self.nfas = [NFA(T, s, a, unknown_rejects=True) for (T, s, a) in nfas]
        self.pnfas = [PNFA(T, s, a) for (T, s, a) in pnfas]
        # "auto": the CUDA-core kernel with BF16 tables in shared memory for groups of fewer
        # than pnfa_auto_threshold strings (its per-step latency is far lower than the
        # tensor-core kernel's), BF16 tcgen05 above
        if pnfa_mode not in ("bf16", "fp16", "fp32", "bf16cc", "fp16cc", "auto"):
            raise ValueError("pnfa_mode must be bf16, fp16, fp32, bf16cc, fp16cc or auto")
        self.pnfa_mode = pnfa_mode
        self.pnfa_auto_threshold = pnfa_auto_threshold
        # Boolean NFA groups of a batch run side by side on up to this many streams.
        # The process keeps 2 x (1 + kAuxStreams) + 2 streams: CUDA maps streams onto
        # CUDA_DEVICE_MAX_CONNECTIONS hardware queues (8 by default), and two streams on
        # one queue serialise, so a serving process should raise it (to 32) before CUDA
        # starts; otherwise a fast-lane kernel can wait behind a long probabilistic one.
        self.nfa_streams = max(1, min(kAuxStreams, nfa_streams))
        self.use_graphs = use_graphs and self.dfa_set is not None
        # admission: the budget is split 3:1 between the two lanes, each with two slots;
        # besides its bytes a request holds 8+4+8 B of offsets/ids and 1+1+1+8+8 B of
        # outputs, plus the DFA scratch in the fast lane
        per_req = 40
        self.max_requests = max_batch_requests

        def slot_bytes(budget, scratch_fn):
            b = max(1 << 16, budget - per_req * max_batch_requests)
            sc = scratch_fn(b)
            while sc + b + per_req * max_batch_requests > budget and b > (1 << 16):
                b //= 2
                sc = scratch_fn(b)
            return b, sc

        self.max_bytes, scratch = slot_bytes(hbm_budget * 3 // 8,
                                             lambda b: DFASet.scratch_bytes(max_batch_requests, b, 0))
        self.max_pnfa_bytes, _ = slot_bytes(hbm_budget // 8, lambda b: 0)
        self.slots = [_Slot(torch, self.dev, "fast", max_batch_requests, self.max_bytes, scratch)
                      for _ in range(2)]
        self.slots += [_Slot(torch, self.dev, "pnfa", max_batch_requests, self.max_pnfa_bytes, 0)
                       for _ in range(2)]
        if self.dfa_set is not None:   # first run outside any graph capture (one-time setup)
            s0 = self.slots[0]
            self.dfa_set.run(s0.d_data[:1], s0.d_doff[:2], s0.d_ids[:1], final_state=s0.d_fs,
                             accept=s0.d_ac, scratch=s0.d_scratch, stream=s0.stream)
            s0.stream.synchronize()
        if self.use_graphs and precapture:
            # every size bucket's graph up front: a capture in the serving loop would stall
            # the requests behind it
            for s in self.slots:
                if s.lane != "fast":
                    continue
                nb = 64
                while True:
                    bb = 1 << 16
                    while True:
                        self._graph(s, nb, bb)
                        if bb >= self.max_bytes:
                            break
                        bb = min(bb * 2, self.max_bytes)
                    if nb >= self.max_requests:
                        break
                    nb = min(nb * 2, self.max_requests)
            torch.cuda.synchronize(self.dev)
        self._queues = {"fast": collections.deque(), "pnfa": collections.deque()}
        self._cv = threading.Condition()
        self._fin = threading.Condition()   # notified when a batch's requests are done
        self._lat = {k: [] for k in KINDS}   # latencies (ms) since reset_stats: plain floats
        self._next = 0
        self._stop = False
        self._bytes_done = 0
        self._batches = 0
        self._loop_busy = 0.0   # seconds the loop spent packing, launching and handing out results
        self._t_first = None
        self._t_last = None
        self._error: Optional[BaseException] = None
        if gc_freeze:
            # the tables, buffers and graphs built above live as long as the server: move
            # them (and everything else alive now) out of the collector's passes
            import gc
            gc.collect()
            gc.freeze()
        self._thread = threading.Thread(target=self._loop, name="trex-serve", daemon=True)
        self._thread.start()

    @classmethod
    def from_file(cls, path, **kw) -> "Server":
        """A server over the automata of a file written by trex_b200.automata_io.save."""
        from .automata_io import load
        a = load(path)
        return cls(a["dfas"], a["nfas"], a["pnfas"], **kw)

    # ---- client side ---------------------------------------------------------------------------
    def submit(self, kind: str, engine: int, data: bytes) -> Request:
        if kind not in KINDS:
            raise ValueError(f"kind must be one of {KINDS}")
        n_eng = {"dfa": len(self.dfa_set.dfas) if self.dfa_set else 0, "nfa": len(self.nfas),
                 "pnfa": len(self.pnfas)}[kind]
        if not 0 <= engine < n_eng:
            raise ValueError(f"no {kind} automaton {engine}")
        data = bytes(data)
        cap = self.max_pnfa_bytes if kind == "pnfa" else self.max_bytes
        if len(data) > cap:
            raise ValueError(f"request of {len(data)} bytes exceeds the slot capacity {cap}")
        with self._cv:
            if self._error is not None:
                raise RuntimeError("server loop failed") from self._error
            r = Request(self._next, kind, engine, data, t_submit=time.perf_counter())
            self._next += 1
            self._queues["pnfa" if kind == "pnfa" else "fast"].append(r)
            self._cv.notify()
        return r

    def submit_many(self, items, t_arrival: Optional[Sequence[float]] = None) -> list:
        """Submit (kind, engine, data) triples under one lock. ``t_arrival`` gives
        each request's arrival time (time.perf_counter clock) for open-loop load
        generators that submit in bursts; latency is measured from it."""
        reqs = []
        now = time.perf_counter()
        for i, (kind, engine, data) in enumerate(items):
            if kind not in KINDS:
                raise ValueError(f"kind must be one of {KINDS}")
            data = bytes(data)
            cap = self.max_pnfa_bytes if kind == "pnfa" else self.max_bytes
            if len(data) > cap:
                raise ValueError(f"request of {len(data)} bytes exceeds the slot capacity {cap}")
            reqs.append(Request(0, kind, engine, data,
                                t_submit=t_arrival[i] if t_arrival is not None else now))
        with self._cv:
            if self._error is not None:
                raise RuntimeError("server loop failed") from self._error
            for r in reqs:
                r.rid = self._next
                self._next += 1
                self._queues["pnfa" if r.kind == "pnfa" else "fast"].append(r)
            self._cv.notify()
        return reqs

    def wait(self, reqs: Sequence[Request], timeout: float = 60.0) -> list:
        end = time.perf_counter() + timeout
        with self._fin:
            for r in reqs:
                while not r.done:
                    left = end - time.perf_counter()
                    if left <= 0:
                        raise TimeoutError(f"request {r.rid} not served in time")
                    self._fin.wait(min(left, 0.5))
        for r in reqs:
            if r.error:
                raise RuntimeError(r.error)
        return [r.result for r in reqs]

    def stats(self) -> dict:
        """Requests, batches, bytes, throughput over the serving span and latency
        percentiles (ms), overall and per kind."""
        with self._cv:
            lat = {k: np.array(v, dtype=np.float64) for k, v in self._lat.items()}
            span = (self._t_last - self._t_first) if self._t_first and self._t_last else 0.0
            nbytes, nb, busy = self._bytes_done, self._batches, self._loop_busy

        def pct(a):
            x = a if a.size else np.zeros(1)
            return {"n": int(a.size), "p50_ms": float(np.percentile(x, 50)),
                    "p99_ms": float(np.percentile(x, 99)), "mean_ms": float(x.mean())}

        allv = np.concatenate(list(lat.values()))
        out = {"requests": int(allv.size), "batches": nb, "bytes": nbytes,
               "gchar_s": nbytes / span / 1e9 if span > 0 else 0.0,
               "loop_busy_frac": busy / span if span > 0 else 0.0, **pct(allv)}
        out["by_kind"] = {k: pct(v) for k, v in lat.items()}
        return out

    def reset_stats(self):
        with self._cv:
            self._lat = {k: [] for k in KINDS}
            self._bytes_done = 0
            self._batches = 0
            self._loop_busy = 0.0
            self._t_first = self._t_last = None

    def close(self):
        with self._cv:
            self._stop = True
            self._cv.notify()
        self._thread.join(timeout=30)
        for s in self.slots:
            s.graphs.clear()
        if self.dfa_set is not None:
            self.dfa_set.close()
        for m in self.nfas + self.pnfas:
            m.close()

    # ---- loop ----------------------------------------------------------------------------------
    def _loop(self):
        torch = self.torch
        torch.cuda.set_device(self.dev)
        try:
            while True:
                for s in self.slots:
                    if s.batch is not None and s.event.query():
                        self._finish(s)
                launches = []
                with self._cv:
                    idle = all(s.batch is None for s in self.slots)
                    empty = not any(self._queues.values())
                    if self._stop and empty and idle:
                        return
                    for lane, cap in (("fast", self.max_bytes), ("pnfa", self.max_pnfa_bytes)):
                        free = [s for s in self.slots if s.lane == lane and s.batch is None]
                        if free and self._queues[lane]:
                            launches.append((free[0], take_batch(self._queues[lane], self.max_requests, cap)))
                    if not launches and idle and not self._stop:
                        self._cv.wait(timeout=0.05)
                        continue
                for slot, batch in launches:
                    if batch:
                        self._launch(slot, batch)
                if not launches:
                    time.sleep(20e-6)
        except BaseException as e:   # hand the failure to every waiting request
            with self._cv:
                self._error = e
                pending = [r for q in self._queues.values() for r in q]
                pending += [r for s in self.slots if s.batch for r in s.batch]
                for q in self._queues.values():
                    q.clear()
            for r in pending:
                r.error = f"server loop failed: {e!r}"
            with self._fin:
                self._fin.notify_all()

    def _dfa_part(self, s: _Slot, nd: int, dfa_bytes: int):
        torch = self.torch
        if nd == 0:
            return
        if not self.use_graphs:
            with torch.cuda.stream(s.stream):   # copies and kernels in one stream order
                s.d_data[:dfa_bytes].copy_(s.h_data[:dfa_bytes], non_blocking=True)
                s.d_doff[:nd + 1].copy_(s.h_doff[:nd + 1], non_blocking=True)
                s.d_ids[:nd].copy_(s.h_ids[:nd], non_blocking=True)
                self.dfa_set.run(s.d_data[:max(dfa_bytes, 1)], s.d_doff[:nd + 1], s.d_ids[:nd],
                                 final_state=s.d_fs, accept=s.d_ac, scratch=s.d_scratch,
                                 stream=s.stream)
                s.h_fs[:nd].copy_(s.d_fs[:nd], non_blocking=True)
                s.h_ac[:nd].copy_(s.d_ac[:nd], non_blocking=True)
            return
        nb = min(_bucket(nd, 64), self.max_requests)
        bb = min(_bucket(max(dfa_bytes, 1), 1 << 16), self.max_bytes)
        # padding: empty strings on automaton 0 after the last real one
        s.h_doff[nd + 1:nb + 1] = int(s.h_doff[nd])
        s.h_ids[nd:nb] = 0
        g = self._graph(s, nb, bb)
        with torch.cuda.stream(s.stream):
            g.replay()

    def _graph(self, s: _Slot, nb: int, bb: int):
        """The captured DFA part of slot s for nb strings and bb bytes (captured once)."""
        torch = self.torch
        key = (nb, bb)
        g = s.graphs.get(key)
        if g is None:
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=s.stream):
                s.d_data[:bb].copy_(s.h_data[:bb], non_blocking=True)
                s.d_doff[:nb + 1].copy_(s.h_doff[:nb + 1], non_blocking=True)
                s.d_ids[:nb].copy_(s.h_ids[:nb], non_blocking=True)
                self.dfa_set.run(s.d_data[:bb], s.d_doff[:nb + 1], s.d_ids[:nb], final_state=s.d_fs,
                                 accept=s.d_ac, scratch=s.d_scratch,
                                 stream=torch.cuda.current_stream())
                s.h_fs[:nb].copy_(s.d_fs[:nb], non_blocking=True)
                s.h_ac[:nb].copy_(s.d_ac[:nb], non_blocking=True)
            s.graphs[key] = g
        return g

    def _launch(self, s: _Slot, batch: list):
        torch = self.torch
        t_busy = time.perf_counter()
        order, blob, doff, ids, roff, groups = pack_batch(batch)
        nd = len(doff) - 1
        total = len(blob)
        if total:
            s.h_data[:total].copy_(torch.frombuffer(bytearray(blob), dtype=torch.uint8))
        s.h_doff[:nd + 1].copy_(torch.from_numpy(doff))
        if nd:
            s.h_ids[:nd].copy_(torch.from_numpy(ids))
        nr = len(roff) - 1
        s.h_roff[:nr + 1].copy_(torch.from_numpy(roff))
        dfa_bytes = int(doff[-1])
        self._dfa_part(s, nd, dfa_bytes)
        if nr:
            # an NFA or PNFA handle keeps one work queue: its launches from the two slots
            # must not overlap, so this slot's stream waits for the other slot's batch
            for o in self.slots:
                if o is not s and o.lane == s.lane and o.batch is not None:
                    s.stream.wait_event(o.event)
            with torch.cuda.stream(s.stream):
                if total > dfa_bytes:
                    s.d_data[dfa_bytes:total].copy_(s.h_data[dfa_bytes:total], non_blocking=True)
                s.d_roff[:nr + 1].copy_(s.h_roff[:nr + 1], non_blocking=True)
                s.ready.record(s.stream)
            used = set()
            for gi, (kind, eng, first, cnt) in enumerate(groups):
                if s.aux:
                    k = gi % self.nfa_streams
                    st = s.aux[k]
                    if k not in used:
                        st.wait_event(s.ready)
                        used.add(k)
                else:
                    st = s.stream
                off = s.d_roff[first:first + cnt + 1]
                data = s.d_data[:max(total, 1)]
                if kind == "nfa":
                    self.nfas[eng].run(data, off, final_mask=s.d_mask[first:first + cnt],
                                       accept=s.d_ac2[first:first + cnt], stream=st)
                else:
                    mode = self.pnfa_mode
                    if mode == "auto":
                        mode = "bf16cc" if cnt < self.pnfa_auto_threshold else "bf16"
                    self.pnfas[eng].run(data, off, mode, loglik=s.d_ll[first:first + cnt],
                                        accept=s.d_ac2[first:first + cnt], stream=st)
            for k in used:
                s.aux_ev[k].record(s.aux[k])
                s.stream.wait_event(s.aux_ev[k])
            with torch.cuda.stream(s.stream):
                s.h_mask[:nr].copy_(s.d_mask[:nr], non_blocking=True)
                s.h_ll[:nr].copy_(s.d_ll[:nr], non_blocking=True)
                s.h_ac2[:nr].copy_(s.d_ac2[:nr], non_blocking=True)
        s.event.record(s.stream)
        s.batch = order
        s.meta = (nd, nr, total)
        with self._cv:
            if self._t_first is None:
                self._t_first = time.perf_counter()
            self._loop_busy += time.perf_counter() - t_busy

    def _finish(self, s: _Slot):
        t_busy = time.perf_counter()
        nd, nr, total = s.meta
        fs = s.h_fs[:nd].numpy() if nd else None
        ac = s.h_ac[:nd].numpy() if nd else None
        ac2 = s.h_ac2[:nr].numpy() if nr else None
        mask = s.h_mask[:nr].numpy() if nr else None
        ll = s.h_ll[:nr].numpy() if nr else None
        now = time.perf_counter()
        for i, r in enumerate(s.batch):
            if i < nd:
                r.result = (bool(ac[i]), int(fs[i]))
            elif r.kind == "nfa":
                r.result = (bool(ac2[i - nd]), int(mask[i - nd]) & 0xFFFFFFFFFFFFFFFF)
            else:
                r.result = (float(ll[i - nd]), bool(ac2[i - nd]))
        with self._cv:
            for r in s.batch:
                self._lat[r.kind].append((now - r.t_submit) * 1e3)
            self._bytes_done += total
            self._batches += 1
            self._t_last = now
            self._loop_busy += time.perf_counter() - t_busy
        with self._fin:
            for r in s.batch:
                r.t_done = now
            self._fin.notify_all()
        s.batch = None
        s.meta = None
