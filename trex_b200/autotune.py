"""Autotuner: K-gram width, tile shape (work-item length) and scan block size.

The reference picks its K-gram width from a table budget alone (``auto_k``,
src/kgram.py:29-66) and fixes tile sizes in its kernels. Here the choice is
measured on the GPU on a sample of the caller's own batch:

* K-gram width, per automaton: every width the automaton allows
  (``DFASet.kgram_max``: 1, 2, 4, 8) is timed on the automaton's own strings;
* tile shape of the ragged kernel (bytes per work item, ``seg_len``), per batch:
  a sweep over 512 .. 8192 bytes with the chosen widths;
* scan block size (bytes per scan tile, ``tile_len``) of the per-position
  scan, per automaton and string length, measured on the whole batch (up to
  ``scan_bytes``): the scan's parallelism comes from the tiles of all strings
  together, so a sample of fewer strings would favour smaller tiles.

Each candidate is timed with CUDA events around the library call (median of
``reps`` runs after ``warmup`` runs), on the stream the call runs on. Choices
are cached in a JSON file keyed by automaton size and shape of the input, so a
second batch of the same kind is not measured again:

    dfa:N<=8|16|256:k<=K:len<L       -> K-gram width
    seg:d<D:n<S:len<L:k<K            -> bytes per work item
    scan:N<=8|16:n<S:len<L           -> scan tile length (0: the library default)

(``len<L``: median string length rounded up to a power of two; ``n<S``:
number of strings, likewise.) The cache path is ``cache_path``, else the
environment variable ``TREX_TUNE_CACHE``, else no file (in-memory only).
"""

from __future__ import annotations

import json
import os
import statistics
from dataclasses import dataclass, field
from pathlib import Path
from typing import Optional

import numpy as np

SEG_CANDIDATES = (512, 1024, 2048, 4096, 8192)
SCAN_CANDIDATES = (0, 1024, 4096, 16384, 65536)   # 0: the library's default for the batch


def _pow2_ceil(x: float) -> int:
    x = max(1, int(np.ceil(x)))
    return 1 << (x - 1).bit_length()


def _n_class(n_states: int) -> int:
    return 8 if n_states <= 8 else 16 if n_states <= 16 else 256


@dataclass
class TuneReport:
    """What a tuning call chose and what it measured (milliseconds per run)."""

    kgram: list = field(default_factory=list)       # per automaton
    kgram_max: list = field(default_factory=list)   # per automaton: the largest K it allows
    seg_len: int = 0
    sweep: list = field(default_factory=list)       # [{"what": ..., "value": ..., "ms": ...}]
    cached: bool = False

    def as_dict(self) -> dict:
        return {"kgram": self.kgram, "kgram_max": self.kgram_max, "seg_len": self.seg_len,
                "sweep": self.sweep, "cached": self.cached}


class Autotuner:
    def __init__(self, cache_path: Optional[str] = None, warmup: int = 2, reps: int = 5,
                 sample_bytes: int = 256 << 20, scan_bytes: int = 4 << 30, seg_bytes: int = 8 << 30):
        p = cache_path or os.environ.get("TREX_TUNE_CACHE")
        self.path = Path(p) if p else None
        self.warmup, self.reps, self.sample_bytes = warmup, reps, sample_bytes
        # the work-item length is timed on the whole batch up to seg_bytes: the planning and
        # chaining kernels are latency-bound, so a sample understates their share
        self.seg_bytes = seg_bytes
        self.scan_bytes = scan_bytes
        self.cache: dict = {}
        if self.path is not None and self.path.exists():
            try:
                self.cache = json.loads(self.path.read_text())
            except (OSError, ValueError):
                self.cache = {}

    # ---- helpers -------------------------------------------------------------------------------
    def _save(self):
        if self.path is None:
            return
        self.path.parent.mkdir(parents=True, exist_ok=True)
        tmp = self.path.with_suffix(".tmp")
        tmp.write_text(json.dumps(self.cache, indent=1, sort_keys=True))
        tmp.replace(self.path)

    def _time(self, fn) -> float:
        import torch
        for _ in range(self.warmup):
            fn()
        ts = []
        for _ in range(self.reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return statistics.median(ts)

    @staticmethod
    def _sample(offsets: np.ndarray, limit_bytes: int, rows: Optional[np.ndarray] = None):
        """Strings (indices) whose bytes add up to about limit_bytes: an evenly spaced subset."""
        idx = np.arange(len(offsets) - 1) if rows is None else np.asarray(rows)
        if idx.size == 0:
            return idx
        lens = offsets[idx + 1] - offsets[idx]
        tot = int(lens.sum())
        if tot <= limit_bytes:
            return idx
        step = max(1, int(np.ceil(tot / limit_bytes)))
        return idx[::step]

    @staticmethod
    def _gather(data_dev, offsets: np.ndarray, idx: np.ndarray):
        """A compact batch (device bytes, device offsets) of the strings idx."""
        import torch
        lens = offsets[idx + 1] - offsets[idx]
        off = np.zeros(len(idx) + 1, dtype=np.int64)
        np.cumsum(lens, out=off[1:])
        starts = torch.from_numpy(offsets[idx].astype(np.int64)).to(data_dev.device)
        lens_t = torch.from_numpy(lens.astype(np.int64)).to(data_dev.device)
        total = int(off[-1])
        if total == 0:
            return data_dev[:0], torch.from_numpy(off).to(data_dev.device)
        # position of every output byte in the source: start of its string + rank inside it
        owner = torch.repeat_interleave(torch.arange(len(idx), device=data_dev.device), lens_t)
        first = torch.from_numpy(off[:-1]).to(data_dev.device)
        pos = starts[owner] + (torch.arange(total, device=data_dev.device) - first[owner])
        return data_dev[pos], torch.from_numpy(off).to(data_dev.device)

    # ---- ragged DFA batches --------------------------------------------------------------------
    def tune_batch(self, dfa_set, data, offsets, dfa_id=None, apply: bool = True) -> TuneReport:
        """Chooses the K-gram width of every automaton of dfa_set and the work-item
        length for a batch like (data, offsets, dfa_id): device tensors (offsets and
        dfa_id may also be numpy arrays). With apply, the widths are set on dfa_set;
        the caller passes report.seg_len to DFASet.run."""
        import torch
        off = offsets.cpu().numpy() if hasattr(offsets, "cpu") else np.asarray(offsets, np.int64)
        ids = (dfa_id.cpu().numpy() if hasattr(dfa_id, "cpu") else np.asarray(dfa_id)) \
            if dfa_id is not None else np.zeros(len(off) - 1, np.int32)
        dev = data.device
        n_dfas = len(dfa_set.dfas)
        lens = np.diff(off)
        rep = TuneReport()
        all_cached = True
        # K-gram width per automaton, on its own strings
        for d in range(n_dfas):
            kmax = dfa_set.kgram_max(d)
            rep.kgram_max.append(kmax)
            rows = np.flatnonzero(ids == d)
            med = _pow2_ceil(np.median(lens[rows])) if rows.size else 1
            N = dfa_set.dfas[d].n_states
            key = f"dfa:N<={_n_class(N)}:k<={kmax}:len<{med}"
            if kmax == 1 or rows.size == 0:
                k = 1
            elif key in self.cache:
                k = int(self.cache[key])
            else:
                all_cached = False
                sub = self._sample(off, self.sample_bytes, rows)
                sdata, soff = self._gather(data, off, sub)
                sub_ids = torch.full((len(sub),), d, dtype=torch.int32, device=dev)
                best = None
                for kk in (1, 2, 4, 8):
                    if kk > kmax:
                        break
                    dfa_set.set_kgram(d, kk)
                    ms = self._time(lambda: dfa_set.run(sdata, soff, sub_ids))
                    rep.sweep.append({"what": f"kgram[{d}]", "value": kk, "ms": ms,
                                      "bytes": int(soff[-1].item())})
                    if best is None or ms < best[1]:
                        best = (kk, ms)
                k = best[0]
                self.cache[key] = k
            rep.kgram.append(k)
            if apply:
                dfa_set.set_kgram(d, k)
            elif kmax > 1:
                dfa_set.set_kgram(d, 1)
        # work-item length for the whole batch, with the chosen widths
        med = _pow2_ceil(np.median(lens)) if lens.size else 1
        key = f"seg:d<{_pow2_ceil(n_dfas)}:n<{_pow2_ceil(len(lens))}:len<{med}:k<{max(rep.kgram or [1])}"
        if key in self.cache:
            rep.seg_len = int(self.cache[key])
        else:
            all_cached = False
            if int(off[-1]) <= self.seg_bytes:
                sdata = data
                soff = offsets if hasattr(offsets, "cpu") else torch.from_numpy(off).to(dev)
                sids = (dfa_id if hasattr(dfa_id, "cpu") else torch.from_numpy(ids.astype(np.int32)).to(dev)) \
                    if dfa_id is not None else torch.zeros(len(off) - 1, dtype=torch.int32, device=dev)
            else:
                sub = self._sample(off, self.sample_bytes)
                sdata, soff = self._gather(data, off, sub)
                sids = torch.from_numpy(ids[sub].astype(np.int32)).to(dev)
            if not apply:
                for d, k in enumerate(rep.kgram):
                    dfa_set.set_kgram(d, k)
            best = None
            for seg in SEG_CANDIDATES:
                ms = self._time(lambda: dfa_set.run(sdata, soff, sids, seg_len=seg))
                rep.sweep.append({"what": "seg_len", "value": seg, "ms": ms,
                                  "bytes": int(soff[-1].item())})
                if best is None or ms < best[1]:
                    best = (seg, ms)
            if not apply:
                for d in range(n_dfas):
                    dfa_set.set_kgram(d, 1)
            rep.seg_len = best[0]
            self.cache[key] = rep.seg_len
        rep.cached = all_cached
        self._save()
        return rep

    # ---- per-position scan ---------------------------------------------------------------------
    def tune_scan(self, dfa_set, dfa_index: int, data, offsets) -> tuple[int, list]:
        """Scan tile length for automaton dfa_index on strings like (data, offsets)."""
        off = offsets.cpu().numpy() if hasattr(offsets, "cpu") else np.asarray(offsets, np.int64)
        lens = np.diff(off)
        N = dfa_set.dfas[dfa_index].n_states
        med = _pow2_ceil(np.median(lens)) if lens.size else 1
        key = f"scan:N<={_n_class(N)}:n<{_pow2_ceil(len(lens))}:len<{med}"
        if key in self.cache:
            return int(self.cache[key]), []
        import torch
        if int(off[-1] - off[0]) <= self.scan_bytes and off[0] == 0:
            sub, sdata, soff = np.arange(len(lens)), data[:int(off[-1])], \
                torch.from_numpy(off.astype(np.int64)).to(data.device)
        else:
            sub = self._sample(off, self.scan_bytes)
            sdata, soff = self._gather(data, off, sub)
        states = torch.empty(max(sdata.numel(), 1), dtype=torch.uint8, device=sdata.device)
        sweep, best = [], None
        for tile in SCAN_CANDIDATES:
            from .engine import DFASet
            scratch = torch.empty(DFASet.scan_scratch_bytes(len(sub), sdata.numel(), tile),
                                  dtype=torch.uint8, device=sdata.device)
            ms = self._time(lambda: dfa_set.scan(sdata, soff, dfa_index, states=states,
                                                 scratch=scratch, tile_len=tile))
            sweep.append({"what": "scan_tile", "value": tile, "ms": ms, "bytes": int(sdata.numel())})
            if best is None or ms < best[1]:
                best = (tile, ms)
        self.cache[key] = best[0]
        self._save()
        return best[0], sweep
