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
* the GPU shared between the lanes: the automaton groups of a batch run side
  by side on auxiliary streams, the fast lane's streams have priority, and
  the probabilistic lane's launches are sized to stay within ``pnfa_sms``
  SMs (its chains hold an SM for a whole string), so DFA batches find free
  SMs while long probabilistic strings run;
* two submission forms: one request at a time (``submit``, a Request each),
  or many of one kind as arrays (``submit_arrays``: engine ids, bytes and
  offsets in, result arrays out, no Python object per request; the strings of
  such a submission are staged as they came and scattered to their places in
  the batch by a device kernel, ``trex_scatter_strings``);
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

from . import _lib

KINDS = ("dfa", "nfa", "pnfa")
kAuxStreams = 8   # most extra streams of a slot (the probabilistic lane's groups run side by side)


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


@dataclass(slots=True, eq=False)
class Bulk:
    """Requests of one kind submitted together as arrays (Server.submit_arrays).

    Request i is automaton ``engines[i]`` over ``data[offsets[i]:offsets[i+1]]``.
    The results are arrays in submission order, filled in as the batches that
    took the requests finish: DFA requests (accept, final_state), NFA requests
    (accept, final_mask), probabilistic NFA requests (log_likelihood, accept).
    ``t_done[i]`` is request i's completion time; ``done`` is true once every
    request has one. A large submission is spread over several batches."""

    rid: int               # id of the first request (the others follow)
    kind: str
    engines: np.ndarray    # int32 [n]
    data: np.ndarray       # uint8
    offsets: np.ndarray    # int64 [n + 1]
    t_submit: np.ndarray   # float64 [n]
    out0: np.ndarray
    out1: np.ndarray
    t_done: np.ndarray     # float64 [n], 0 until done
    next: int = 0          # first request not yet taken into a batch
    n_done: int = 0
    error: Optional[str] = None

    @property
    def n(self) -> int:
        return len(self.engines)

    @property
    def done(self) -> bool:
        return self.n_done >= len(self.engines) or self.error is not None

    @property
    def result(self):
        return (self.out0, self.out1)

    @property
    def latency_ms(self) -> np.ndarray:
        return (self.t_done - self.t_submit) * 1e3


def take_batch(queue: collections.deque, max_requests: int, max_bytes: int) -> list:
    """FIFO admission: pop requests while the batch stays within both
    capacities; the first request that does not fit stays at the head. A bulk
    submission at the head gives the batch as many of its next requests as fit,
    as one entry (bulk, lo, hi), and stays at the head while requests remain."""
    batch, nbytes, count = [], 0, 0
    while queue and count < max_requests:
        r = queue[0]
        if isinstance(r, Bulk):
            off, lo = r.offsets, r.next
            # requests lo .. hi-1 fit while off[hi] - off[lo] <= the room left
            hi = int(np.searchsorted(off, off[lo] + (max_bytes - nbytes), side="right")) - 1
            hi = min(hi, r.n, lo + (max_requests - count))
            if hi <= lo:
                break
            batch.append((r, lo, hi))
            nbytes += int(off[hi] - off[lo])
            count += hi - lo
            if hi < r.n:
                r.next = hi
                break
            queue.popleft()
            continue
        if nbytes + len(r.data) > max_bytes:
            break
        queue.popleft()
        batch.append(r)
        nbytes += len(r.data)
        count += 1
    return batch


@dataclass(slots=True)
class BatchPlan:
    """Where every string of a batch goes. The batch is laid out as
    [DFA strings | NFA strings by engine | probabilistic NFA strings by engine]
    (one DFA launch takes any mix of DFAs; an NFA launch takes one contiguous
    run of strings). Single requests are copied by the host to their places;
    the strings of bulk submissions other than DFA ones are staged in
    submission order and scattered on the device (stage_off: their offsets in
    the stage, stage_dst: their places in the batch)."""

    total: int              # bytes of the batch
    dfa_bytes: int          # bytes of its DFA part (first)
    doff: np.ndarray        # int64 [nd + 1], DFA string offsets from 0
    ids: np.ndarray         # int32 [nd], DFA of each DFA string
    roff: np.ndarray        # int64 [nr + 1], other strings' offsets (absolute)
    groups: list            # (kind, engine, first, count) over the other strings
    copies: list            # (batch offset, bytes or uint8 array): host copies
    rest_copied: bool       # some copy lands in the non-DFA part
    stage: list             # (stage offset, uint8 array): host copies into the stage
    stage_bytes: int
    stage_off: np.ndarray   # int64 [ns + 1]
    stage_dst: np.ndarray   # int64 [ns]
    reqs: list              # (Request, index into its kind's outputs), DFA ones first
    parts: list             # (Bulk, lo, hi, indices into its kind's outputs), DFA ones first
    n_dfa_reqs: int = 0
    n_dfa_parts: int = 0
    dfa_out: bool = False   # the DFA results were handed out (before the rest)

    @property
    def nd(self) -> int:
        return len(self.ids)

    @property
    def nr(self) -> int:
        return len(self.roff) - 1


def plan_batch(batch: Sequence) -> BatchPlan:
    """Lay out a batch of Requests and bulk entries (bulk, lo, hi); see BatchPlan."""
    reqs = [e for e in batch if isinstance(e, Request)]
    parts = [e for e in batch if not isinstance(e, Request)]
    dreq = [r for r in reqs if r.kind == "dfa"]
    rreq = [r for r in reqs if r.kind != "dfa"]
    dparts = [p for p in parts if p[0].kind == "dfa"]
    rparts = [p for p in parts if p[0].kind != "dfa"]
    i64 = np.int64
    # DFA part: single requests, then bulk entries, in batch order
    dlens = [np.fromiter((len(r.data) for r in dreq), dtype=i64, count=len(dreq))]
    dids = [np.fromiter((r.engine for r in dreq), dtype=np.int32, count=len(dreq))]
    dlens += [np.diff(b.offsets[lo:hi + 1]) for b, lo, hi in dparts]
    dids += [b.engines[lo:hi] for b, lo, hi in dparts]
    dlen = np.concatenate(dlens)
    nd = len(dlen)
    doff = np.zeros(nd + 1, dtype=i64)
    np.cumsum(dlen, out=doff[1:])
    copies, out_reqs, out_parts = [], [], []
    pos = 0
    for i, r in enumerate(dreq):   # one copy each, straight into the batch buffer (no join)
        copies.append((pos, r.data))
        pos += len(r.data)
    out_reqs += [(r, i) for i, r in enumerate(dreq)]
    k = len(dreq)
    for b, lo, hi in dparts:
        a0, a1 = int(b.offsets[lo]), int(b.offsets[hi])
        copies.append((pos, b.data[a0:a1]))
        pos += a1 - a0
        out_parts.append((b, lo, hi, np.arange(k, k + hi - lo)))
        k += hi - lo
    dfa_bytes = pos
    # other strings, in batch order, then sorted (stably) by kind and engine
    kc = [np.fromiter((KINDS.index(r.kind) for r in rreq), dtype=i64, count=len(rreq))]
    eng = [np.fromiter((r.engine for r in rreq), dtype=i64, count=len(rreq))]
    rl = [np.fromiter((len(r.data) for r in rreq), dtype=i64, count=len(rreq))]
    for b, lo, hi in rparts:
        kc.append(np.full(hi - lo, KINDS.index(b.kind), dtype=i64))
        eng.append(b.engines[lo:hi].astype(i64))
        rl.append(np.diff(b.offsets[lo:hi + 1]))
    key = (np.concatenate(kc) << 32) | np.concatenate(eng)
    rlen = np.concatenate(rl)
    nr = len(rlen)
    order = np.argsort(key, kind="stable")
    inv = np.empty(nr, dtype=i64)
    inv[order] = np.arange(nr, dtype=i64)
    roff = np.empty(nr + 1, dtype=i64)
    roff[0] = dfa_bytes
    np.cumsum(rlen[order], out=roff[1:])
    roff[1:] += dfa_bytes
    start = roff[:-1][inv]            # place of each string, in batch order
    groups = []
    if nr:
        sk = key[order]
        cut = np.flatnonzero(np.diff(sk)) + 1
        firsts = np.concatenate(([0], cut))
        ends = np.concatenate((cut, [nr]))
        for f, e in zip(firsts.tolist(), ends.tolist()):
            groups.append((KINDS[int(sk[f] >> 32)], int(sk[f] & 0xFFFFFFFF), f, e - f))
    if rreq:
        copies += [(p, r.data) for p, r in zip(start[:len(rreq)].tolist(), rreq)]
        out_reqs += [(r, j) for j, r in zip(inv[:len(rreq)].tolist(), rreq)]
    stage, soff, sdst = [], [], []
    spos = 0
    k = len(rreq)
    for b, lo, hi in rparts:
        a0, a1 = int(b.offsets[lo]), int(b.offsets[hi])
        stage.append((spos, b.data[a0:a1]))
        soff.append(b.offsets[lo:hi] - a0 + spos)
        sdst.append(start[k:k + hi - lo])
        out_parts.append((b, lo, hi, inv[k:k + hi - lo]))
        spos += a1 - a0
        k += hi - lo
    stage_off = np.concatenate(soff + [np.array([spos], dtype=i64)])
    stage_dst = np.concatenate(sdst) if sdst else np.zeros(0, dtype=i64)
    total = int(roff[-1])
    return BatchPlan(total, dfa_bytes, doff, np.concatenate(dids).astype(np.int32, copy=False), roff,
                     groups, copies, bool(rreq), stage, spos, stage_off, stage_dst, out_reqs, out_parts,
                     len(dreq), len(dparts))


def _bucket(x: int, lo: int) -> int:
    b = lo
    while b < x:
        b <<= 1
    return b


class _Slot:
    """Device and pinned host buffers of one in-flight batch."""

    def __init__(self, torch, dev, lane: str, max_requests: int, max_bytes: int, dfa_scratch: int,
                 n_aux: int = 1):
        self.lane = lane
        # the fast lane's streams take priority: when an SM frees, the block scheduler
        # starts their CTAs before the probabilistic lane's
        prio = -1 if lane == "fast" else 0
        u8, i32, i64, f64 = torch.uint8, torch.int32, torch.int64, torch.float64
        R, B = max_requests, max_bytes
        self.stream = torch.cuda.Stream(device=dev, priority=prio)
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
        # staging of bulk submissions (scattered into d_data) and its string offsets / places
        self.d_stage = torch.zeros(B + 16, dtype=u8, device=dev)
        self.d_soff = torch.zeros(R + 1, dtype=i64, device=dev)
        self.d_sdst = torch.zeros(max(R, 1), dtype=i64, device=dev)
        self.d_err = torch.zeros(1, dtype=torch.int32, device=dev)
        # the multi-automaton NFA run's work counters and error word
        self.d_nscr = torch.zeros(8 * 65, dtype=torch.uint8, device=dev)
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
        self.h_stage = torch.zeros(B + 16, dtype=u8, **pin)
        self.h_soff = torch.zeros(R + 1, dtype=i64, **pin)
        self.h_sdst = torch.zeros(max(R, 1), dtype=i64, **pin)
        self.h_err = torch.zeros(1, dtype=torch.int32, **pin)
        self.h_nerr = torch.zeros(1, dtype=torch.int32, **pin)
        self.h_data_np = self.h_data.numpy()
        self.h_data_mv = memoryview(self.h_data_np)
        self.h_stage_np = self.h_stage.numpy()
        self.event = torch.cuda.Event()
        # the non-DFA part of a batch runs on the first of these streams, beside the DFA
        # part; the probabilistic groups of a batch run side by side on all of them
        self.aux = [torch.cuda.Stream(device=dev, priority=prio) for _ in range(n_aux)]
        self.aux_ev = [torch.cuda.Event() for _ in range(n_aux)]
        self.ready = torch.cuda.Event()
        self.rest_done = torch.cuda.Event()   # the non-DFA part's results are on the host
        self.dfa_done = torch.cuda.Event()    # the DFA part's results are on the host
        self.graphs = {}
        self.batch = None   # the BatchPlan in flight


class Server:
    """Continuous-batching server over resident automata (see the module docstring)."""

    def __init__(self, dfas=(), nfas=(), pnfas=(), *, hbm_budget: int = 1 << 30,
                 max_batch_requests: int = 1 << 14, pnfa_mode: str = "bf16", use_graphs: bool = True,
                 device: int = 0, pnfa_auto_threshold: int = 2048, precapture: bool = True,
                 gc_freeze: bool = True, pnfa_streams: int = kAuxStreams, pnfa_sms: int = 96):
        import torch
        from .engine import NFA, PNFA, DFASet
        self.torch = torch
        self.dev = torch.device("cuda", device)
        torch.cuda.set_device(self.dev)
        self.dfa_set = DFASet(list(dfas)) if len(dfas) else None
        if len(nfas) > 64:
            raise ValueError("a server holds at most 64 Boolean NFAs (one multi-automaton launch a batch)")
        self.nfas = [NFA(T, s, a, unknown_rejects=True) for (T, s, a) in nfas]
        self.pnfas = [PNFA(T, s, a) for (T, s, a) in pnfas]
        # A probabilistic chain holds its SM for the whole string (milliseconds for long
        # ones), and the ragged DFA kernel needs whole SMs: the probabilistic lane's
        # launches (up to pnfa_streams at a time) together stay within pnfa_sms SMs, so the
        # fast lane always finds free ones (0: no limit)
        self.pnfa_sms = pnfa_sms
        if pnfa_sms > 0:
            for m in self.pnfas:
                m.set_sm_limit(max(1, pnfa_sms // max(1, min(kAuxStreams, pnfa_streams))))
        # "auto": the CUDA-core kernel with BF16 tables in shared memory for groups of fewer
        # than pnfa_auto_threshold strings (its per-step latency is far lower than the
        # tensor-core kernel's), BF16 tcgen05 above
        if pnfa_mode not in ("bf16", "fp16", "fp32", "bf16cc", "fp16cc", "auto"):
            raise ValueError("pnfa_mode must be bf16, fp16, fp32, bf16cc, fp16cc or auto")
        self.pnfa_mode = pnfa_mode
        self.pnfa_auto_threshold = pnfa_auto_threshold
        # The probabilistic groups of a batch run side by side on up to this many streams.
        # The process keeps 2 x (1 + 1) + 2 x (1 + pnfa_streams) + 2 streams: CUDA maps
        # streams onto CUDA_DEVICE_MAX_CONNECTIONS hardware queues (8 by default), and two
        # streams on one queue serialise, so a serving process should raise it (to 32)
        # before CUDA starts; otherwise a fast-lane kernel can wait behind a long
        # probabilistic one.
        self.pnfa_streams = max(1, min(kAuxStreams, pnfa_streams))
        self.use_graphs = use_graphs and self.dfa_set is not None
        # admission: the budget is split 3:1 between the two lanes, each with two slots;
        # a slot holds its bytes twice (the batch and the staging of bulk submissions);
        # besides its bytes a request holds 8+4+8+16 B of offsets/ids/staging places and
        # 1+1+1+8+8 B of outputs, plus the DFA scratch in the fast lane
        per_req = 56
        self.max_requests = max_batch_requests

        def slot_bytes(budget, scratch_fn):
            b = max(1 << 16, (budget - per_req * max_batch_requests) // 2)
            sc = scratch_fn(b)
            while sc + 2 * b + per_req * max_batch_requests > budget and b > (1 << 16):
                b //= 2
                sc = scratch_fn(b)
            return b, sc

        self.max_bytes, scratch = slot_bytes(hbm_budget * 3 // 8,
                                             lambda b: DFASet.scratch_bytes(max_batch_requests, b, 0))
        self.max_pnfa_bytes, _ = slot_bytes(hbm_budget // 8, lambda b: 0)
        self.slots = [_Slot(torch, self.dev, "fast", max_batch_requests, self.max_bytes, scratch)
                      for _ in range(2)]
        self.slots += [_Slot(torch, self.dev, "pnfa", max_batch_requests, self.max_pnfa_bytes, 0,
                             n_aux=self.pnfa_streams)
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
        self._lat_bulk = {k: [] for k in KINDS}   # and arrays of them (bulk submissions)
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

    def submit_arrays(self, kind: str, engines, data, offsets, t_arrival=None) -> Bulk:
        """Submit many requests of one kind as arrays, without a Python object per
        request: request i is automaton ``engines[i]`` (or ``engines`` for all)
        over ``data[offsets[i]:offsets[i+1]]`` (offsets nondecreasing, int64).
        ``data`` (bytes or a uint8 array) and ``offsets`` are read in place until
        the requests are done. ``t_arrival``: arrival time of each request (or
        one for all; time.perf_counter clock), latency is measured from it.
        Returns a Bulk whose result arrays fill in as its batches finish."""
        if kind not in KINDS:
            raise ValueError(f"kind must be one of {KINDS}")
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        if off.ndim != 1 or len(off) < 1:
            raise ValueError("offsets must be a 1-D array of n + 1 entries")
        n = len(off) - 1
        buf = np.frombuffer(data, dtype=np.uint8) if not isinstance(data, np.ndarray) \
            else np.ascontiguousarray(data).reshape(-1).view(np.uint8)
        lens = np.diff(off)
        if n and (off[0] < 0 or off[-1] > len(buf) or (lens < 0).any()):
            raise ValueError("offsets must be nondecreasing and within data")
        cap = self.max_pnfa_bytes if kind == "pnfa" else self.max_bytes
        if n and int(lens.max()) > cap:
            raise ValueError(f"a request of {int(lens.max())} bytes exceeds the slot capacity {cap}")
        n_eng = {"dfa": len(self.dfa_set.dfas) if self.dfa_set else 0, "nfa": len(self.nfas),
                 "pnfa": len(self.pnfas)}[kind]
        eng = np.ascontiguousarray(np.broadcast_to(np.asarray(engines, dtype=np.int64), (n,)))
        if n and (eng.min() < 0 or eng.max() >= n_eng):
            raise ValueError(f"engine ids must lie in [0, {n_eng}) for {kind}")
        now = time.perf_counter()
        t = np.ascontiguousarray(np.broadcast_to(
            np.asarray(now if t_arrival is None else t_arrival, dtype=np.float64), (n,)))
        out0 = np.zeros(n, dtype=np.float64 if kind == "pnfa" else bool)
        out1 = np.zeros(n, dtype={"dfa": np.uint8, "nfa": np.uint64, "pnfa": bool}[kind])
        b = Bulk(0, kind, eng.astype(np.int32), buf, off, t, out0, out1, np.zeros(n))
        with self._cv:
            if self._error is not None:
                raise RuntimeError("server loop failed") from self._error
            b.rid = self._next
            self._next += n
            if n:
                self._queues["pnfa" if kind == "pnfa" else "fast"].append(b)
                self._cv.notify()
        return b

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
            lat = {k: np.concatenate([np.array(v, dtype=np.float64)] + self._lat_bulk[k])
                   for k, v in self._lat.items()}
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
            self._lat_bulk = {k: [] for k in KINDS}
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
                    if s.batch is None:
                        continue
                    if not s.batch.dfa_out and s.batch.nd and s.dfa_done.query():
                        self._hand_out(s, dfa=True)   # DFA results before the batch's NFA strings end
                    if s.event.query():
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
                pending += [r for s in self.slots if s.batch for r, _ in s.batch.reqs]
                pending += [b for s in self.slots if s.batch for b, _, _, _ in s.batch.parts]
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
        from .engine import nfa_run_multi
        t_busy = time.perf_counter()
        plan = plan_batch(batch)
        nd, nr, total = plan.nd, plan.nr, plan.total
        h, hv = s.h_data_np, s.h_data_mv
        for off, src in plan.copies:
            if isinstance(src, bytes):
                hv[off:off + len(src)] = src
            else:
                h[off:off + len(src)] = src
        s.h_doff[:nd + 1].copy_(torch.from_numpy(plan.doff))
        if nd:
            s.h_ids[:nd].copy_(torch.from_numpy(plan.ids))
        s.h_roff[:nr + 1].copy_(torch.from_numpy(plan.roff))
        ns = len(plan.stage_dst)
        if ns:
            for off, a in plan.stage:
                s.h_stage_np[off:off + len(a)] = a
            s.h_soff[:ns + 1].copy_(torch.from_numpy(plan.stage_off))
            s.h_sdst[:ns].copy_(torch.from_numpy(plan.stage_dst))
        if nr:
            # the non-DFA part runs on the slot's first auxiliary stream, beside the DFA part
            st = s.aux[0]
            if s.lane == "pnfa":
                # a probabilistic NFA handle keeps one work queue: its launches from the two
                # slots must not overlap, so this batch waits for the other slot's
                for o in self.slots:
                    if o is not s and o.lane == s.lane and o.batch is not None:
                        st.wait_event(o.event)
            data = s.d_data[:max(total, 1)]
            with torch.cuda.stream(st):
                if plan.rest_copied:
                    s.d_data[plan.dfa_bytes:total].copy_(s.h_data[plan.dfa_bytes:total], non_blocking=True)
                s.d_roff[:nr + 1].copy_(s.h_roff[:nr + 1], non_blocking=True)
                if ns:
                    sb = plan.stage_bytes
                    s.d_stage[:sb].copy_(s.h_stage[:sb], non_blocking=True)
                    s.d_soff[:ns + 1].copy_(s.h_soff[:ns + 1], non_blocking=True)
                    s.d_sdst[:ns].copy_(s.h_sdst[:ns], non_blocking=True)
                    s.d_err.zero_()
                    _lib.check(_lib.load().trex_scatter_strings(
                        s.d_stage.data_ptr(), sb, s.d_soff.data_ptr(), ns, s.d_data.data_ptr(), total,
                        s.d_sdst.data_ptr(), s.d_err.data_ptr(), st.cuda_stream),
                        "trex_scatter_strings")
                    s.h_err.copy_(s.d_err, non_blocking=True)
                # Boolean NFA groups (first in the non-DFA part): one launch, side by side
                nfa_groups = [g for g in plan.groups if g[0] == "nfa"]
                if nfa_groups:
                    n_nfa = nfa_groups[-1][2] + nfa_groups[-1][3]
                    gf = [g[2] for g in nfa_groups] + [n_nfa]
                    nfa_run_multi([self.nfas[g[1]] for g in nfa_groups], gf, data, s.d_roff[:n_nfa + 1],
                                  final_mask=s.d_mask, accept=s.d_ac2, scratch=s.d_nscr, stream=st)
                    s.h_nerr.copy_(s.d_nscr[8 * len(nfa_groups):8 * len(nfa_groups) + 4].view(torch.int32),
                                   non_blocking=True)
                s.ready.record(st)
            # probabilistic NFA groups: one launch per automaton, side by side on the aux streams
            used = set()
            for gi, (kind, eng, first, cnt) in enumerate(g for g in plan.groups if g[0] == "pnfa"):
                k = gi % self.pnfa_streams
                ps = s.aux[k]
                if k not in used:
                    if k:
                        ps.wait_event(s.ready)
                    used.add(k)
                mode = self.pnfa_mode
                if mode == "auto":
                    mode = "bf16cc" if cnt < self.pnfa_auto_threshold else "bf16"
                self.pnfas[eng].run(data, s.d_roff[first:first + cnt + 1], mode,
                                    loglik=s.d_ll[first:first + cnt], accept=s.d_ac2[first:first + cnt],
                                    stream=ps)
            for k in used:
                if k:
                    s.aux_ev[k].record(s.aux[k])
                    st.wait_event(s.aux_ev[k])
            with torch.cuda.stream(st):
                s.h_mask[:nr].copy_(s.d_mask[:nr], non_blocking=True)
                s.h_ll[:nr].copy_(s.d_ll[:nr], non_blocking=True)
                s.h_ac2[:nr].copy_(s.d_ac2[:nr], non_blocking=True)
                s.rest_done.record(st)
        self._dfa_part(s, nd, plan.dfa_bytes)
        s.dfa_done.record(s.stream)
        if nr:
            s.stream.wait_event(s.rest_done)
        s.event.record(s.stream)
        s.batch = plan
        with self._cv:
            if self._t_first is None:
                self._t_first = time.perf_counter()
            self._loop_busy += time.perf_counter() - t_busy

    def _hand_out(self, s: _Slot, dfa: bool):
        """Results of the DFA (or the other) requests of slot s's batch to their requests."""
        t_busy = time.perf_counter()
        plan = s.batch
        nd, nr = plan.nd, plan.nr
        reqs = plan.reqs[:plan.n_dfa_reqs] if dfa else plan.reqs[plan.n_dfa_reqs:]
        parts = plan.parts[:plan.n_dfa_parts] if dfa else plan.parts[plan.n_dfa_parts:]
        err = None
        if dfa:
            fs = s.h_fs[:nd].numpy() if nd else None
            ac = s.h_ac[:nd].numpy() if nd else None
        else:
            ac2 = s.h_ac2[:nr].numpy() if nr else None
            mask = s.h_mask[:nr].numpy().view(np.uint64) if nr else None
            ll = s.h_ll[:nr].numpy() if nr else None
            if len(plan.stage_dst) and int(s.h_err[0]) != 0:
                err = f"staged strings out of range (scatter error word {int(s.h_err[0])})"
            if any(g[0] == "nfa" for g in plan.groups) and int(s.h_nerr[0]) != 0:
                err = f"malformed NFA offsets (error word {int(s.h_nerr[0])})"
        now = time.perf_counter()
        if reqs:   # plain Python values for the single requests (list indexing is cheap)
            if dfa:
                acl, fsl = ac.tolist(), fs.tolist()
                for r, j in reqs:
                    r.result = (acl[j] != 0, fsl[j])
            else:
                acl, ml, lll = ac2.tolist(), mask.tolist(), ll.tolist()
                for r, j in reqs:
                    r.result = (acl[j] != 0, ml[j]) if r.kind == "nfa" else (lll[j], acl[j] != 0)
            if err:
                for r, _ in reqs:
                    r.error = err
        for b, lo, hi, j in parts:
            if b.kind == "dfa":
                b.out0[lo:hi] = ac[j] != 0
                b.out1[lo:hi] = fs[j]
            elif b.kind == "nfa":
                b.out0[lo:hi] = ac2[j] != 0
                b.out1[lo:hi] = mask[j]
            else:
                b.out0[lo:hi] = ll[j]
                b.out1[lo:hi] = ac2[j] != 0
            b.t_done[lo:hi] = now
            if err:
                b.error = err
        with self._cv:
            for r, _ in reqs:
                self._lat[r.kind].append((now - r.t_submit) * 1e3)
            for b, lo, hi, _ in parts:
                self._lat_bulk[b.kind].append((now - b.t_submit[lo:hi]) * 1e3)
            self._loop_busy += time.perf_counter() - t_busy
        with self._fin:
            for r, _ in reqs:
                r.t_done = now
            for b, lo, hi, _ in parts:
                b.n_done += hi - lo
            self._fin.notify_all()
        if dfa:
            plan.dfa_out = True

    def _finish(self, s: _Slot):
        plan = s.batch
        if not plan.dfa_out:
            self._hand_out(s, dfa=True)
        self._hand_out(s, dfa=False)
        now = time.perf_counter()
        with self._cv:
            self._bytes_done += plan.total
            self._batches += 1
            self._t_last = now
        s.batch = None
