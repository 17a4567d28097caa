"""Benchmark: automaton simulation on B200 (one JSON line on stdout, rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl trex|reference]
                    [--workload ragged|plain|scan|nfa|pnfa|serve] [--strings S]
                    [--no-extras] [--extras a,b,...]

Workloads (synthetic, seeded; the reference ships no dataset):
  ragged (default, the headline case): 16 random DFAs (5 x 8, 5 x 12, 6 x 16
      states) over all 256 byte values, 1M strings with log-normal lengths
      (median 2048, sigma 1.18, clipped to [16, 65536], ~4.1 GB), 10% of the
      strings over the 4-byte sub-alphabet "ACGT", string i on DFA i mod 16.
      One step = one ragged launch over the whole batch.
  plain: one random 16-state DFA over the bytes "ACGT", 4096 x 1024 bytes.
  scan: one random 16-state DFA over 256 bytes, 8 strings x 256 MiB; one step
      writes the state of every position (2 bytes moved per character).
  nfa: random 64-state Boolean NFA over 20 symbols (bytes 0..19), per-symbol
      edge density 0.05, 256K strings x 4096 symbols; bit-parallel kernel, or
      --nfa-method tc (0/1 BF16 tensor cores) / tc8 (0/1 int8 tensor cores).
  serve: the serving mix (64 resident automata, Poisson arrivals at
      --serve-rates) through trex_b200.serving.Server; reports throughput
      and p50/p99 latency per rate and the plain per-request launch.
  pnfa: probabilistic 64-state NFA over 20 symbols (rows Dirichlet(0.5) x 0.9,
      ~30% kept), 64K strings x 2048 symbols, tcgen05 kernel with BF16 (or
      --pnfa-mode fp16 / fp32) operands; also reports the log-likelihood error
      against the FP64 oracle.

Every workload's results are checked against the C oracle (oracle/oracle.c)
on the same bytes, outside the timed region: the line carries
"mismatches_vs_oracle" (all strings of the batch; every position for the
scan) and the run exits non-zero on any mismatch.

The default run (ragged headline, one GPU) also measures the other
configurations and the plain per-pattern form in the same process and adds
them under "configs": cfg1_plain, plain_per_pattern (the ragged batch as 16
per-automaton launches, device buffers and through the reference's
prefix_engine_* ABI with host buffers), cfg3a_scan, cfg3b_nfa (bit-parallel and
tensor-core forms), cfg4_pnfa (with the one-string chain latency per
position), dfa_n32_64 (the ragged batch shape, 250K strings, on 32- and
64-state automata), kgram_sweep (K = 1, 2, 4 on 4 GB of ACGT strings, where
gram tables apply), ref_shapes (the NFA kernels on the shape the reference
publishes its NFA numbers for: sigma 2, 262144 x 2048, with those numbers
beside them), cfg5_served (a Poisson sweep up to saturation, with the limiter
named). --no-extras skips them.

Multi-GPU: one process per GPU (torchrun); every rank runs its own seeded
batch (weak scaling, no data-path collective); times are the max over ranks
(an NCCL all-reduce of one float).

--impl reference times the reference's CPU algorithm for the path (the C
oracle, oracle/oracle.c: DFA.simulate over the byte map / the per-position
walk) with OpenMP on the host cores, on a bounded sample of the same workload.
"""

from __future__ import annotations

import os

# Many streams (the serving workload keeps 12): more hardware queues than the default 8, so
# that independent streams do not serialise. Must be set before CUDA starts.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

import argparse  # noqa: E402
import json  # noqa: E402
import re  # noqa: E402
import statistics  # noqa: E402
import subprocess  # noqa: E402
import sys  # noqa: E402
import threading  # noqa: E402
import time  # noqa: E402
from pathlib import Path  # noqa: E402

import numpy as np  # noqa: E402

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

from trex_b200.sharding import max_over_ranks, rank_seed  # noqa: E402

METRIC = "Gchar/s vs HBM roofline, plain vs batched/served; served p50/p99 ms (1 B200)"
SUB_ALPHABET = b"ACGT"
EXTRAS = ("cfg1_plain", "plain_per_pattern", "cfg3a_scan", "cfg3b_nfa", "cfg4_pnfa", "dfa_n32_64",
          "kgram_sweep", "ref_shapes", "frontend", "cfg5_served")


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["trex", "reference"], default="trex")
    ap.add_argument("--workload", choices=["ragged", "plain", "scan", "nfa", "pnfa", "serve"],
                    default="ragged")
    ap.add_argument("--serve-rates", type=str, default="2000,8000,32000,128000,256000,512000",
                    help="offered request rates (requests/s) of the serve workload, swept upwards "
                         "until the served rate falls below 90%% of the offered one")
    ap.add_argument("--serve-seconds", type=float, default=2.0)
    ap.add_argument("--serve-bulk-rates", type=str, default="256000,1000000,2000000,4000000,8000000,16000000",
                    help="offered request rates of the bulk-submission sweep of the serve workload")
    ap.add_argument("--serve-bulk-seconds", type=float, default=1.0)
    ap.add_argument("--serve-bulk-tick-ms", type=float, default=1.0,
                    help="period of the bulk client: it submits what arrived since its last tick")
    ap.add_argument("--serve-no-graphs", action="store_true",
                    help="launch the DFA batches directly instead of replaying CUDA graphs")
    ap.add_argument("--serve-plain", type=int, default=2000,
                    help="requests timed one by one for the plain per-request baseline")
    ap.add_argument("--pnfa-mode", choices=["bf16", "fp16", "fp32"], default="bf16",
                    help="operand type of the probabilistic NFA workload")
    ap.add_argument("--nfa-method", choices=["bitpar", "tc", "tc8"], default="bitpar",
                    help="nfa workload: bit-parallel kernel, or the Boolean NFA on the tensor cores "
                         "with 0/1 BF16 (tc) or int8 (tc8) operands")
    ap.add_argument("--nfa-sigma", type=int, default=None,
                    help="nfa / pnfa workloads: alphabet size (default 20)")
    ap.add_argument("--nfa-len", type=int, default=None,
                    help="nfa / pnfa workloads: symbols a string (default 4096 / 2048)")
    ap.add_argument("--strings", type=int, default=None, help="override the number of strings")
    ap.add_argument("--seg-len", type=int, default=0, help="bytes per work item / scan tile (0 = default)")
    ap.add_argument("--kgram", type=int, default=None,
                    help="K-gram width of every automaton of a DFA workload (0 = the largest each "
                         "allows; overrides the tuned choice)")
    ap.add_argument("--no-tune", dest="tuned", action="store_false",
                    help="DFA workloads: skip the autotuner (by default it picks the K-gram width "
                         "per automaton and the bytes per work item / scan tile on a sample of the "
                         "batch before the warm-up, outside the timed region, and the line reports "
                         "its sweep)")
    ap.set_defaults(tuned=True)
    ap.add_argument("--dfa-sizes", type=str, default=None,
                    help="comma list of DFA state counts replacing the default 5x8,5x12,6x16")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="CPU budget of the reference arm's samples")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-verify", action="store_true",
                    help="skip the oracle check of the results (profiling runs only)")
    ap.add_argument("--no-extras", action="store_true",
                    help="default run: skip the other configurations")
    ap.add_argument("--extras", type=str, default=",".join(EXTRAS),
                    help="configurations measured after the headline (comma list of "
                         + ", ".join(EXTRAS) + ")")
    return ap.parse_args(argv)


# ---------------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------------

def lognormal_offsets(n: int, seed: int):
    from trex_b200.workloads import lognormal_lengths
    rng = np.random.default_rng(seed + 1)
    lens = lognormal_lengths(n, rng)
    is_sub = np.zeros(n, dtype=bool)
    is_sub[rng.choice(n, size=int(round(0.10 * n)), replace=False)] = True
    return lens, is_sub


def offsets_of(lens):
    off = np.zeros(len(lens) + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    return off


def device_bytes(torch, lens, is_sub, seed, device):
    """Uniform random bytes; strings flagged is_sub are re-drawn over ACGT."""
    total = int(lens.sum())
    g = torch.Generator(device=device)
    g.manual_seed(seed + 2)
    data = torch.randint(0, 256, (max(total, 1),), dtype=torch.uint8, device=device, generator=g)
    if is_sub is not None and is_sub.any():
        acgt = torch.tensor(list(SUB_ALPHABET), dtype=torch.uint8, device=device)
        flag = torch.repeat_interleave(torch.from_numpy(is_sub).to(device),
                                       torch.from_numpy(lens).to(device))
        codes = acgt[(data[:total] & 3).long()]
        data[:total] = torch.where(flag, codes, data[:total])
        del flag, codes
    return data[:total]


def host_bytes(lens, is_sub, seed):
    rng = np.random.default_rng(seed + 3)
    total = int(lens.sum())
    data = rng.integers(0, 256, size=total, dtype=np.uint8)
    if is_sub is not None and is_sub.any():
        off = offsets_of(lens)
        acgt = np.frombuffer(SUB_ALPHABET, dtype=np.uint8)
        for i in np.flatnonzero(is_sub):
            a, b = off[i], off[i + 1]
            data[a:b] = acgt[data[a:b] & 3]
    return data


def host_copy(torch, t):
    """A pinned host copy of a device tensor, as numpy."""
    h = torch.empty(t.numel(), dtype=t.dtype, pin_memory=True)
    h.copy_(t)
    return h.numpy()


class DFAWorkload:
    """ragged / plain / scan: byte DFAs over CSR strings."""

    dtype = ref_dtype = "u8"

    def __init__(self, args):
        from trex_b200.workloads import ACGT, random_dfa
        self.kind = args.workload
        self.args = args
        self.host_data = None
        rng = np.random.default_rng(args.seed)
        if self.kind == "plain":
            self.n = args.strings or 4096
            self.dfas = [random_dfa(16, ACGT, rng)]
            self.lens = np.full(self.n, 1024, dtype=np.int64)
            self.is_sub = np.ones(self.n, dtype=bool)
            self.ids = np.zeros(self.n, dtype=np.int32)
            self.workload = f"plain DFA: N=16 random DFA over bytes ACGT, {self.n} strings x 1024 bytes"
        elif self.kind == "scan":
            self.n = args.strings or 8
            self.dfas = [random_dfa(16, np.arange(256), rng)]
            self.lens = np.full(self.n, 1 << 28, dtype=np.int64)
            self.is_sub = None
            self.ids = np.zeros(self.n, dtype=np.int32)
            self.workload = (f"long-string scan: N=16 random DFA over 256 bytes, {self.n} strings x "
                             "256 MiB, state of every position written")
        else:
            self.n = args.strings or 1_000_000
            sizes = (8,) * 5 + (12,) * 5 + (16,) * 6
            if args.dfa_sizes:
                base = [int(x) for x in args.dfa_sizes.split(",")]
                sizes = [base[i % len(base)] for i in range(16)]
            self.dfas = [random_dfa(n, np.arange(256), rng) for n in sizes]
            self.lens, self.is_sub = None, None
            self.ids = (np.arange(self.n) % 16).astype(np.int32)
            shape = ", ".join(f"{sizes.count(v)}x{v}" for v in sorted(set(sizes)))
            self.workload = (f"ragged DFA batch: 16 random DFAs ({shape} states) over 256 byte "
                             f"symbols; {self.n} strings, log-normal lengths median 2048 sigma 1.18 "
                             "clipped [16, 65536]; 10% of strings over 'ACGT'; string i on DFA i mod 16")

    def lengths(self, seed):
        if self.lens is None:
            return lognormal_offsets(self.n, seed)
        return self.lens, self.is_sub

    # ---- GPU side
    def setup(self, torch, dev, seed):
        from trex_b200.engine import DFASet
        self.torch = torch
        lens, is_sub = self.lengths(seed)
        self.off = offsets_of(lens)
        self.total = int(self.off[-1])
        self.data = device_bytes(torch, lens, is_sub, seed, dev)
        self.d_off = torch.from_numpy(self.off).to(dev)
        self.d_ids = torch.from_numpy(self.ids).to(dev)
        self.set = DFASet(self.dfas, kgram=self.args.kgram)
        self.tune_info = None
        if self.args.tuned:   # measured on a sample of this batch, before the warm-up
            from trex_b200.autotune import Autotuner
            tuner = Autotuner()
            if self.kind == "scan":
                tile, sweep = tuner.tune_scan(self.set, 0, self.data, self.d_off)
                self.args.seg_len = tile
                self.tune_info = {"scan_tile": tile, "sweep": sweep}
            else:
                rep = tuner.tune_batch(self.set, self.data, self.d_off, self.d_ids)
                self.args.seg_len = rep.seg_len
                self.tune_info = rep.as_dict()
                if self.args.kgram is not None:   # an explicit width wins over the tuned one
                    for i in range(len(self.dfas)):
                        if self.args.kgram != 0 or self.set.kgram_max(i) > 1:
                            self.set.set_kgram(i, self.args.kgram)
        self.kgram_used = [self.set.get_kgram(i) for i in range(len(self.dfas))]
        n = self.n
        if self.kind == "scan":
            self.scratch = torch.empty(DFASet.scan_scratch_bytes(n, self.total, self.args.seg_len),
                                       dtype=torch.uint8, device=dev)
            self.states = torch.empty(self.total, dtype=torch.uint8, device=dev)
        else:
            self.scratch = torch.empty(DFASet.scratch_bytes(n, self.total, self.args.seg_len),
                                       dtype=torch.uint8, device=dev)
        self.fs = torch.empty(n, dtype=torch.uint8, device=dev)
        self.ac = torch.empty(n, dtype=torch.uint8, device=dev)

    def step(self, stream):
        if self.kind == "scan":
            self.set.scan(self.data, self.d_off, 0, states=self.states, final_state=self.fs,
                          accept=self.ac, scratch=self.scratch, tile_len=self.args.seg_len,
                          stream=stream)
        else:
            self.set.run(self.data, self.d_off, self.d_ids, final_state=self.fs, accept=self.ac,
                         scratch=self.scratch, seg_len=self.args.seg_len, stream=stream)

    def error_word(self):
        if self.kind == "scan":
            return self.set.scan_error_word(self.scratch, self.n, self.total, self.args.seg_len)
        return self.set.last_error_word(self.scratch)

    @property
    def chars(self):
        return self.total

    @property
    def kernel(self):
        return "dfa_scan_kernel" if self.kind == "scan" else "dfa_ragged_kernel"

    @property
    def alg_bytes(self):
        # 1 B/char in (+1 B/char out for the scan) + 16 B per string
        # (64-bit offset, automaton id, state, accept)
        per_char = 2 if self.kind == "scan" else 1
        return per_char * self.total + 16 * self.n

    @property
    def launches_per_step(self):
        # scan: tile bases, empty strings, scan; ragged: count, class prefix, queue scan, fill,
        # walk, and chaining (records, fix-ups, re-walks)
        return 3 if self.kind == "scan" else 8

    def config(self):
        return {"workload": self.workload, "n_strings": self.n, "total_bytes_per_gpu": self.total,
                "seg_len": self.args.seg_len or (8192 if self.kind == "scan" else 2048),
                "kgram": getattr(self, "kgram_used", None),
                "l2": "inputs larger than L2 (126 MB), no flush" if self.total > 126e6 else
                      "inputs smaller than L2: L2 flushed by a 256 MB write between steps"}

    # ---- end to end (host buffers through the C ABI host entry point)
    def e2e(self, torch, steps, dist, dev):
        if self.kind == "scan":
            return None
        h_data = torch.empty(self.total, dtype=torch.uint8, pin_memory=True)
        h_data.copy_(self.data)
        h_off = torch.from_numpy(self.off).pin_memory()
        h_ids = torch.from_numpy(self.ids).pin_memory()
        h_fs = torch.empty(self.n, dtype=torch.uint8).pin_memory()
        h_ac = torch.empty(self.n, dtype=torch.uint8).pin_memory()
        hd, ho, hi, hf, ha = (h_data.numpy(), h_off.numpy(), h_ids.numpy(), h_fs.numpy(),
                              h_ac.numpy())
        self.set.run_host(hd, ho, hi, self.args.seg_len, hf, ha)   # warm the staging buffers
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(steps):
            self.set.run_host(hd, ho, hi, self.args.seg_len, hf, ha)
        dt = time.perf_counter() - t0
        dt = max_over_ranks(dt, dist, dev)
        if not (np.array_equal(hf, self.fs.cpu().numpy()) and np.array_equal(ha, self.ac.cpu().numpy())):
            raise RuntimeError("host-buffer run disagrees with the device run")
        self.host_data = hd
        return dt, int(self.total + self.off.nbytes + self.ids.nbytes), int(2 * self.n + 4)

    # ---- the oracle on the same bytes, every string (every position for the scan)
    def verify(self, orc):
        torch = self.torch
        if self.host_data is None:
            self.host_data = host_copy(torch, self.data)
        d = self.dfas
        fs = self.fs.cpu().numpy()
        ac = self.ac.cpu().numpy()
        t0 = time.perf_counter()
        if self.kind == "scan":
            ref = orc.dfa_positions(d[0].tmap, d[0].n_states, d[0].start, self.host_data, self.off)
            dt = time.perf_counter() - t0
            got = host_copy(torch, self.states)
            last = self.off[1:] - 1
            rfs = ref[last]
            mism = {"states": int(np.count_nonzero(got != ref)),
                    "final_state": int(np.count_nonzero(fs != rfs)),
                    "accept": int(np.count_nonzero(ac != d[0].accept[rfs])),
                    "strings": self.n, "positions": int(self.total)}
        else:
            rfs, rac = orc.dfa_walk([x.tmap for x in d], [x.n_states for x in d],
                                    [x.start for x in d], [x.accept for x in d], self.host_data,
                                    self.off, self.ids)
            dt = time.perf_counter() - t0
            mism = {"final_state": int(np.count_nonzero(fs != rfs)),
                    "accept": int(np.count_nonzero(ac != rac)), "strings": self.n,
                    "bytes": int(self.total)}
        return mism, dt, self.total

    # ---- CPU (oracle) sample, reference arm
    def cpu_run(self, orc, data, k):
        d = self.dfas
        if self.kind == "scan":
            orc.dfa_positions(d[0].tmap, d[0].n_states, d[0].start, data, self.off_cpu[:k + 1])
        else:
            orc.dfa_walk([x.tmap for x in d], [x.n_states for x in d], [x.start for x in d],
                         [x.accept for x in d], data, self.off_cpu[:k + 1], self.ids[:k])

    def cpu_sample(self, seed, seconds, threads):
        """(k strings, their bytes, host data) sized to ~seconds of oracle work."""
        from oracle import oracle as orc
        lens, is_sub = self.lengths(seed)
        if self.kind == "scan":
            # per-position walk on a prefix of each string
            per = max(1 << 16, int(seconds * 4e8 / max(1, len(lens))))
            lens = np.minimum(lens, per)
        self.off_cpu = offsets_of(lens)
        rate_guess = 3e8 * threads
        k0 = max(1, int(np.searchsorted(self.off_cpu, 0.05 * rate_guess, side="right")) - 1)
        k0 = min(k0, len(lens))
        data0 = host_bytes(lens[:k0], None if is_sub is None else is_sub[:k0], seed)
        t0 = time.perf_counter()
        self.cpu_run(orc, data0, k0)
        rate = self.off_cpu[k0] / max(time.perf_counter() - t0, 1e-6)
        k = max(1, min(len(lens), int(np.searchsorted(self.off_cpu, seconds * rate, side="right")) - 1))
        data = host_bytes(lens[:k], None if is_sub is None else is_sub[:k], seed)
        return k, int(self.off_cpu[k]), data

    def close(self):
        self.set.close()


class NFAWorkload:
    """Boolean NFA, 64 states, 20 symbols (bit-parallel kernel)."""

    kind = "nfa"
    kernel = "nfa_bitpar_kernel"
    launches_per_step = 1
    dtype = ref_dtype = "u64"

    def __init__(self, args):
        from trex_b200.workloads import random_bool_nfa
        self.args = args
        self.host_data = None
        rng = np.random.default_rng(args.seed)
        self.sigma = getattr(args, "nfa_sigma", None) or 20
        self.T, self.start, self.acc = random_bool_nfa(rng, n_states=64, sigma=self.sigma, density=0.05)
        self.n = args.strings or 262144
        self.L = getattr(args, "nfa_len", None) or 4096
        self.off = np.arange(self.n + 1, dtype=np.int64) * self.L
        self.workload = (f"Boolean NFA: random 64-state NFA over {self.sigma} symbols (bytes 0..{self.sigma - 1}), "
                         f"edge density 0.05, {self.n} strings x {self.L} symbols")

    def setup(self, torch, dev, seed):
        from trex_b200.engine import NFA
        self.torch = torch
        self.total = self.n * self.L
        self.off = np.arange(self.n + 1, dtype=np.int64) * self.L
        g = torch.Generator(device=dev)
        g.manual_seed(seed + 2)
        self.data = torch.randint(0, self.sigma, (self.total,), dtype=torch.uint8, device=dev, generator=g)
        self.d_off = torch.from_numpy(self.off).to(dev)
        self.nfa = NFA(self.T, self.start, self.acc, unknown_rejects=True)
        self.fm = torch.empty(self.n, dtype=torch.int64, device=dev)
        self.ac = torch.empty(self.n, dtype=torch.uint8, device=dev)
        self.set = self.nfa

    def step(self, stream):
        self.nfa.run(self.data, self.d_off, final_mask=self.fm, accept=self.ac, stream=stream)

    def error_word(self):
        return self.nfa.error_word()

    @property
    def chars(self):
        return self.total

    @property
    def alg_bytes(self):
        return self.total + 17 * self.n

    def config(self):
        return {"workload": self.workload, "n_strings": self.n, "total_bytes_per_gpu": self.total,
                "useful_ops_per_char": 2 * 64 * 64, "kernel_bound": "integer ALU / shared-memory lookups",
                "l2": "inputs larger than L2 (126 MB), no flush"}

    def e2e(self, torch, steps, dist, dev):
        import ctypes
        from trex_b200 import _lib
        L = _lib.load()
        Tf = np.ascontiguousarray(self.T.astype(np.float32))
        st = np.ascontiguousarray(self.start.astype(np.float32))
        ac = np.ascontiguousarray(self.acc.astype(np.float32))
        f32 = ctypes.c_float
        _lib.check(L.nfa_tc_engine_init(_lib.ptr(Tf, f32), _lib.ptr(ac, f32), _lib.ptr(st, f32), 64,
                                        20, self.n, self.L), "nfa_tc_engine_init")
        h_data = torch.empty(self.total, dtype=torch.uint8, pin_memory=True)
        h_data.copy_(self.data)
        h_off = torch.from_numpy(self.off.astype(np.int32)).pin_memory()
        h_res = torch.empty(self.n, dtype=torch.int32).pin_memory()
        hd, ho, hr = h_data.numpy(), h_off.numpy(), h_res.numpy()
        km, tm = ctypes.c_float(), ctypes.c_float()
        args = (_lib.ptr(hd, ctypes.c_uint8), _lib.ptr(ho, ctypes.c_int), _lib.ptr(hr, ctypes.c_int),
                self.n, self.total, ctypes.byref(km), ctypes.byref(tm))
        _lib.check(L.nfa_tc_engine_dispatch(*args), "nfa_tc_engine_dispatch")
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(steps):
            _lib.check(L.nfa_tc_engine_dispatch(*args), "nfa_tc_engine_dispatch")
        dt = time.perf_counter() - t0
        dt = max_over_ranks(dt, dist, dev)
        L.nfa_tc_engine_destroy()
        if not np.array_equal(hr.astype(np.uint8), self.ac.cpu().numpy()):
            raise RuntimeError("host-buffer run disagrees with the device run")
        self.host_data = hd
        return dt, int(self.total + ho.nbytes), int(hr.nbytes)

    def verify(self, orc):
        if self.host_data is None:
            self.host_data = host_copy(self.torch, self.data)
        t0 = time.perf_counter()
        rfm, rac = orc.nfa_bool(self.T, self.start, self.acc, self.host_data, self.off,
                                unknown_rejects=True)
        dt = time.perf_counter() - t0
        fm = self.fm.cpu().numpy().view(np.uint64)
        ac = self.ac.cpu().numpy()
        return ({"final_mask": int(np.count_nonzero(fm != rfm)),
                 "accept": int(np.count_nonzero(ac != rac)), "strings": self.n,
                 "bytes": int(self.total)}, dt, self.total)

    def cpu_run(self, orc, data, k):
        orc.nfa_bool(self.T, self.start, self.acc, data, self.off[:k + 1], unknown_rejects=True)

    def cpu_sample(self, seed, seconds, threads):
        rng = np.random.default_rng(seed + 3)
        k0 = max(1, min(self.n, threads * 4))
        data0 = rng.integers(0, 20, size=k0 * self.L, dtype=np.uint8)
        from oracle import oracle as orc
        t0 = time.perf_counter()
        self.cpu_run(orc, data0, k0)
        rate = k0 * self.L / max(time.perf_counter() - t0, 1e-6)
        k = max(1, min(self.n, int(seconds * rate / self.L)))
        data = rng.integers(0, 20, size=k * self.L, dtype=np.uint8)
        return k, k * self.L, data

    def close(self):
        self.nfa.close()


class PNFAWorkload:
    """Probabilistic NFA, 64 states, 20 symbols (tcgen05 kernel, or the FP32 kernel)."""

    kind = "pnfa"
    launches_per_step = 1
    bound = "tensor"
    ref_dtype = "f64"
    verify_strings = 1024

    def __init__(self, args):
        from trex_b200.workloads import random_prob_nfa
        self.args = args
        self.mode = args.pnfa_mode
        rng = np.random.default_rng(args.seed)
        self.sigma = getattr(args, "nfa_sigma", None) or 20
        self.T, self.start, self.acc = random_prob_nfa(rng, 64, self.sigma)
        self.n = args.strings or 65536
        self.L = getattr(args, "nfa_len", None) or 2048
        self.off = np.arange(self.n + 1, dtype=np.int64) * self.L
        # alphabets of at most four symbols run one string a TMEM lane
        self.kernel = ("pnfa_plain_kernel" if self.mode == "fp32" else
                       "pnfa_lane_kernel" if self.sigma <= 4 else "pnfa_tc_kernel")
        self.dtype = {"bf16": "bf16", "fp16": "f16", "fp32": "f32"}[self.mode]
        self.workload = (f"probabilistic NFA: 64 states, {self.sigma} symbols (bytes 0..{self.sigma - 1}), rows of T[c] "
                         "Dirichlet(0.5) x 0.9 with ~30% kept, start e0, accept all states; "
                         f"{self.n} strings x {self.L} symbols; {self.mode} operands"
                         + ("" if self.mode == "fp32" else ", FP32 accumulation (tcgen05)"))

    def setup(self, torch, dev, seed):
        from trex_b200.engine import PNFA
        self.torch = torch
        self.total = self.n * self.L
        g = torch.Generator(device=dev)
        g.manual_seed(seed + 4)
        self.data = torch.randint(0, self.sigma, (self.total,), dtype=torch.uint8, device=dev, generator=g)
        self.d_off = torch.from_numpy(self.off).to(dev)
        self.pnfa = PNFA(self.T, self.start, self.acc)
        self.ll = torch.empty(self.n, dtype=torch.float64, device=dev)
        self.ac = torch.empty(self.n, dtype=torch.uint8, device=dev)
        self.set = self.pnfa

    def step(self, stream):
        self.pnfa.run(self.data, self.d_off, self.mode, loglik=self.ll, accept=self.ac, stream=stream)

    def error_word(self):
        return self.pnfa.error_word()

    @property
    def chars(self):
        return self.total

    @property
    def alg_bytes(self):
        return self.total + 17 * self.n

    @property
    def alg_flops(self):
        return 2.0 * 64 * 64 * self.total

    def config(self):
        return {"workload": self.workload, "n_strings": self.n, "total_bytes_per_gpu": self.total,
                "useful_flops_per_char": 2 * 64 * 64, "mode": self.mode,
                "l2": "inputs (134 MB) larger than L2 (126 MB), no flush"}

    def verify(self, orc):
        """Log-likelihoods of the first verify_strings strings against the FP64 oracle:
        the largest relative error (the tolerance of the tests: 1e-4 relative for
        strings of this length) and the accept flags that differ."""
        k = min(self.n, self.verify_strings)
        data = self.data[:k * self.L].cpu().numpy()
        t0 = time.perf_counter()
        ref = orc.pnfa_fp64(self.T, self.start, self.acc, data, self.off[:k + 1])
        dt = time.perf_counter() - t0
        got = self.ll[:k].cpu().numpy()
        rel = float(np.max(np.abs(got - ref) / np.maximum(1.0, np.abs(ref))))
        ac = self.ac[:k].cpu().numpy().astype(bool)
        return ({"loglik_max_rel_err_vs_fp64": rel, "loglik_tolerance": 1e-4,
                 "loglik_over_tolerance": int(np.count_nonzero(
                     np.abs(got - ref) > 1e-4 * np.maximum(1.0, np.abs(ref)))),
                 "accept_flags_differ": int(np.count_nonzero(ac != (ref > np.log(0.5)))),
                 "strings": k},
                dt, k * self.L)

    def e2e(self, torch, steps, dist, dev):
        # the public API with host buffers: pinned H2D of the step's bytes and offsets,
        # the run, D2H of the log-likelihoods, every step
        h_data = torch.empty(self.total, dtype=torch.uint8, pin_memory=True)
        h_data.copy_(self.data)
        h_off = torch.from_numpy(self.off).pin_memory()
        h_ll = torch.empty(self.n, dtype=torch.float64).pin_memory()
        d_data = torch.empty_like(self.data)
        d_off = torch.empty_like(self.d_off)
        d_ll = torch.empty_like(self.ll)

        def one():
            d_data.copy_(h_data, non_blocking=True)
            d_off.copy_(h_off, non_blocking=True)
            self.pnfa.run(d_data, d_off, self.mode, loglik=d_ll)
            h_ll.copy_(d_ll, non_blocking=True)
            torch.cuda.current_stream().synchronize()

        one()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(steps):
            one()
        dt = time.perf_counter() - t0
        dt = max_over_ranks(dt, dist, dev)
        if not np.array_equal(h_ll.numpy(), self.ll.cpu().numpy()):
            raise RuntimeError("host-buffer run disagrees with the device run")
        return dt, int(self.total + self.off.nbytes), int(h_ll.numpy().nbytes)

    def cpu_run(self, orc, data, k):
        orc.pnfa_fp64(self.T, self.start, self.acc, data, self.off[:k + 1])

    def cpu_sample(self, seed, seconds, threads):
        rng = np.random.default_rng(seed + 5)
        from oracle import oracle as orc
        k0 = max(1, min(self.n, threads * 2))
        data0 = rng.integers(0, 20, size=k0 * self.L, dtype=np.uint8)
        t0 = time.perf_counter()
        self.cpu_run(orc, data0, k0)
        rate = k0 * self.L / max(time.perf_counter() - t0, 1e-6)
        k = max(1, min(self.n, int(seconds * rate / self.L)))
        data = rng.integers(0, 20, size=k * self.L, dtype=np.uint8)
        return k, k * self.L, data

    def close(self):
        self.pnfa.close()


class NFATcWorkload(PNFAWorkload):
    """The Boolean NFA workload (64 states, 20 symbols, 4096 symbols a string) on the
    tensor cores: 0/1 operands (BF16, or int8 with int32 sums), each product
    thresholded to {0, 1} every step."""

    kind = "nfa"
    ref_dtype = "u64"

    def __init__(self, args):
        from trex_b200.workloads import random_bool_nfa
        self.args = args
        self.mode = "bool8" if args.nfa_method == "tc8" else "bool"
        rng = np.random.default_rng(args.seed)
        self.sigma = getattr(args, "nfa_sigma", None) or 20
        T, start, acc = random_bool_nfa(rng, n_states=64, sigma=self.sigma, density=0.05)
        self.T, self.start, self.acc = (x.astype(np.float32) for x in (T, start, acc))
        self.n = args.strings or 262144
        self.L = getattr(args, "nfa_len", None) or 4096
        self.off = np.arange(self.n + 1, dtype=np.int64) * self.L
        self.kernel = "pnfa_lane_kernel" if self.sigma <= 4 else "pnfa_tc_kernel"
        self.dtype = "s8" if self.mode == "bool8" else "bf16"
        ops = ("0/1 int8 operands, int32 sums (tcgen05 kind::i8)" if self.mode == "bool8"
               else "0/1 BF16 operands, FP32 sums (tcgen05 kind::f16)")
        self.workload = (f"Boolean NFA: random 64-state NFA over {self.sigma} symbols (bytes "
                         f"0..{self.sigma - 1}), edge density 0.05, {self.n} strings x {self.L} symbols; "
                         f"tensor cores, {ops} thresholded every step")

    def config(self):
        return {"workload": self.workload, "n_strings": self.n, "total_bytes_per_gpu": self.total,
                "useful_ops_per_char": 2 * 64 * 64, "mode": self.mode,
                "selection_waste": "2x (each MMA computes both symbols of a pair; half is discarded)",
                "l2": "inputs larger than L2 (126 MB), no flush"}

    def verify(self, orc):
        """Accept flags of every string against the bit-parallel oracle."""
        data = host_copy(self.torch, self.data)
        t0 = time.perf_counter()
        _, ref = orc.nfa_bool(self.T != 0, self.start, self.acc, data, self.off,
                              unknown_rejects=False)
        dt = time.perf_counter() - t0
        got = self.ac.cpu().numpy().astype(bool)
        return ({"accept": int(np.count_nonzero(got != ref.astype(bool))), "strings": self.n,
                 "bytes": int(self.total)}, dt, self.total)

    def cpu_run(self, orc, data, k):
        orc.nfa_bool(self.T != 0, self.start, self.acc, data, self.off[:k + 1], unknown_rejects=False)


# ---------------------------------------------------------------------------------
# serving mix
# ---------------------------------------------------------------------------------

def serving_mix(seed: int):
    """64 resident automata: 32 DFAs (16 states, 256 bytes), 24 Boolean NFAs and
    8 probabilistic NFAs (64 states, 20 symbols)."""
    from trex_b200.workloads import random_bool_nfa, random_dfa, random_prob_nfa
    rng = np.random.default_rng(seed)
    dfas = [random_dfa(16, np.arange(256), rng) for _ in range(32)]
    nfas = [random_bool_nfa(rng, 64, 20, 0.05) for _ in range(24)]
    pnfas = [random_prob_nfa(rng, 64, 20) for _ in range(8)]
    return dfas, nfas, pnfas


def serving_requests(seed: int, n: int):
    """Request pool: automaton uniform over the 64, lengths log-normal (median
    2 KiB, sigma 1.0, clipped to [16, 1 MiB]), bytes uniform over the automaton's
    alphabet."""
    rng = np.random.default_rng(seed + 11)
    which = rng.integers(0, 64, size=n)
    lens = np.clip(np.round(np.exp(rng.normal(np.log(2048), 1.0, size=n))), 16, 1 << 20).astype(np.int64)
    pool = []
    for w, L in zip(which.tolist(), lens.tolist()):
        if w < 32:
            pool.append(("dfa", w, rng.integers(0, 256, size=L, dtype=np.uint8).tobytes()))
        elif w < 56:
            pool.append(("nfa", w - 32, rng.integers(0, 20, size=L, dtype=np.uint8).tobytes()))
        else:
            pool.append(("pnfa", w - 56, rng.integers(0, 20, size=L, dtype=np.uint8).tobytes()))
    return pool


def poisson_run(srv, pool, rate: float, duration: float, seed: int):
    """Open-loop Poisson load: request k arrives at the k-th point of a Poisson
    process of `rate` requests/s over `duration` s. The client submits every
    request whose arrival time has passed in one call (its latency is counted
    from its arrival time), then sleeps briefly. Waits for all; returns the
    server stats, plus how far the client fell behind the arrival schedule."""
    rng = np.random.default_rng(seed + 17)
    n = max(1, int(rate * duration))
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n))
    arrivals = arrivals[arrivals <= duration]
    srv.reset_stats()
    reqs = []
    lag = 0.0
    t0 = time.perf_counter()
    k = 0
    while k < len(arrivals):
        now = time.perf_counter() - t0
        j = int(np.searchsorted(arrivals, now, side="right"))
        if j > k:
            lag = max(lag, now - arrivals[k])
            items = [pool[i % len(pool)] for i in range(k, j)]
            reqs += srv.submit_many(items, t_arrival=(t0 + arrivals[k:j]).tolist())
            k = j
        else:
            time.sleep(min(5e-4, max(0.0, arrivals[k] - now)))
    srv.wait(reqs, timeout=300)
    st = srv.stats()
    st["offered_req_s"] = rate
    st["offered_gchar_s"] = rate * float(np.mean([len(p[2]) for p in pool])) / 1e9
    st["client_max_lag_ms"] = lag * 1e3
    return st


def bulk_pool(pool):
    """The request pool as arrays per kind (the pool's order within each kind):
    kinds of the pool in order, and per kind (engines, data, offsets)."""
    kinds = np.array([("dfa", "nfa", "pnfa").index(p[0]) for p in pool], dtype=np.int64)
    per = {}
    for ki, kind in enumerate(("dfa", "nfa", "pnfa")):
        sel = [p for p in pool if p[0] == kind]
        off = np.zeros(len(sel) + 1, dtype=np.int64)
        off[1:] = np.cumsum([len(p[2]) for p in sel])
        data = np.frombuffer(b"".join(p[2] for p in sel), dtype=np.uint8)
        per[kind] = (np.array([p[1] for p in sel], dtype=np.int32), data, off)
    return kinds, per


def poisson_bulk_run(srv, bpool, rate: float, duration: float, seed: int, tick: float = 1e-3):
    """Open-loop Poisson load through the bulk form: the same arrival process and
    request sequence as poisson_run, but the client wakes every `tick` seconds
    and submits the requests that arrived since as one array submission per kind
    (Server.submit_arrays; latency from each request's own arrival time, so the
    wait for the tick counts)."""
    kinds, per = bpool
    P = len(kinds)
    prefix = {ki: np.concatenate(([0], np.cumsum(kinds == ki))) for ki in range(3)}

    def n_before(ki, k):   # requests of kind ki among the first k of the cyclic sequence
        return (k // P) * int(prefix[ki][-1]) + int(prefix[ki][k % P])

    rng = np.random.default_rng(seed + 17)
    n = max(1, int(rate * duration))
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n))
    arrivals = arrivals[arrivals <= duration]
    srv.reset_stats()
    subs = []
    lag = 0.0
    t0 = time.perf_counter()
    k = 0
    while k < len(arrivals):
        now = time.perf_counter() - t0
        j = int(np.searchsorted(arrivals, now, side="right"))
        if j > k:
            lag = max(lag, now - arrivals[k])
            km = kinds[np.arange(k, j) % P]
            for ki, kind in enumerate(("dfa", "nfa", "pnfa")):
                eng, data, off = per[kind]
                m = len(eng)
                a, b = n_before(ki, k), n_before(ki, j)
                if b == a:
                    continue
                t = t0 + arrivals[k:j][km == ki]
                done = 0
                while a < b:   # split where the kind's cyclic sequence wraps
                    lo = a % m
                    hi = min(m, lo + (b - a))
                    subs.append(srv.submit_arrays(kind, eng[lo:hi], data, off[lo:hi + 1],
                                                  t_arrival=t[done:done + hi - lo]))
                    done += hi - lo
                    a += hi - lo
            k = j
        if k < len(arrivals):
            wake = max(now + tick, arrivals[k])
            time.sleep(max(0.0, wake - (time.perf_counter() - t0)))
    srv.wait(subs, timeout=600)
    st = srv.stats()
    st["offered_req_s"] = rate
    st["offered_gchar_s"] = rate * float(sum(int(per[kd][2][-1]) for kd in per)) / P / 1e9
    st["client_max_lag_ms"] = lag * 1e3
    st["submissions"] = len(subs)
    return st


def plain_run(engines, pool, n_req: int):
    """Baseline: each request alone (host-to-device copy, one launch, device-to-
    host copy, synchronise), one after another."""
    import torch
    dset, nfas, pnfas = engines
    lat = []
    nbytes = 0
    t0 = time.perf_counter()
    for kind, eng, data in pool[:n_req]:
        ts = time.perf_counter()
        d = torch.frombuffer(bytearray(data), dtype=torch.uint8).cuda(non_blocking=True)
        off = torch.tensor([0, len(data)], dtype=torch.int64).cuda(non_blocking=True)
        if kind == "dfa":
            _, ac, _ = dset.run(d, off, torch.tensor([eng], dtype=torch.int32).cuda())
            ac.cpu()
        elif kind == "nfa":
            _, ac = nfas[eng].run(d, off)
            ac.cpu()
        else:
            ll, _ = pnfas[eng].run(d, off, "fp32")
            ll.cpu()
        lat.append((time.perf_counter() - ts) * 1e3)
        nbytes += len(data)
    span = time.perf_counter() - t0
    lat = np.array(lat)
    return {"requests": n_req, "gchar_s": nbytes / span / 1e9,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99))}


def serve_measure(args) -> dict:
    """Poisson sweep over the serving mix, upwards until the served rate falls
    below 90% of the offered one; the plain per-request launch beside it."""
    import torch
    from trex_b200.engine import NFA, PNFA, DFASet
    from trex_b200.serving import Server
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    dfas, nfas, pnfas = serving_mix(args.seed)
    pool = serving_requests(args.seed, 20000)
    srv = Server(dfas, nfas, pnfas, hbm_budget=2 << 30, max_batch_requests=1 << 14, pnfa_mode="auto",
                 use_graphs=not args.serve_no_graphs)
    # warm-up (graphs captured per size bucket, first launches)
    poisson_run(srv, pool, 20000, 0.5, args.seed)
    clocks = ClockSampler(gpu_index_for(0))
    clocks.start()
    runs = _serve_sweep(lambda r, k: poisson_run(srv, pool, r, args.serve_seconds, args.seed + k),
                        [float(r) for r in args.serve_rates.split(",")])
    bpool = bulk_pool(pool)
    poisson_bulk_run(srv, bpool, 200000, 0.3, args.seed)   # warm-up of the bulk path
    bulk_runs = _serve_sweep(lambda r, k: poisson_bulk_run(srv, bpool, r, args.serve_bulk_seconds,
                                                           args.seed + k, args.serve_bulk_tick_ms * 1e-3),
                             [float(r) for r in args.serve_bulk_rates.split(",")])
    clock_info = clocks.stop()
    srv.close()
    engines = (DFASet(dfas), [NFA(*x, unknown_rejects=True) for x in nfas], [PNFA(*x) for x in pnfas])
    plain_run(engines, pool, 200)   # warm
    plain = plain_run(engines, pool, args.serve_plain)
    engines[0].close()
    for m in engines[1] + engines[2]:
        m.close()
    top, limiter = _serve_limiter(runs, "the Python request loop")
    btop, blimiter = _serve_limiter(bulk_runs, "the request loop")
    keys = ("offered_req_s", "offered_gchar_s", "gchar_s", "p50_ms", "p99_ms", "requests", "batches",
            "by_kind", "client_max_lag_ms", "loop_busy_frac", "gpu_busy_frac")
    return {
        "workload": "serving mix: 64 resident automata (32 DFA16 over 256 bytes, 24 Boolean NFA64 and "
                    "8 probabilistic NFA64 over 20 symbols), lengths log-normal median 2 KiB sigma 1.0 "
                    "clipped [16 B, 1 MiB], automaton uniform, Poisson arrivals at each offered rate",
        "parallelism": "1 GPU, continuous batching (2 lanes x 2 slots, "
                       + ("direct launches)" if args.serve_no_graphs else "CUDA graphs for DFA batches)"),
        "hbm_budget_bytes": 2 << 30,
        "pnfa_mode": "auto (BF16 tables on CUDA cores below 2048 strings a group, tcgen05 above)",
        "value": top["gchar_s"], "unit": "Gchar/s",
        "sustained_req_s": top["offered_req_s"], "p50_ms_at_sustained": top["p50_ms"],
        "p99_ms_at_sustained": top["p99_ms"], "limiter": limiter,
        "sweep": [{k: r.get(k) for k in keys} for r in runs],
        "bulk": {
            "form": "Server.submit_arrays: every tick_ms the client submits the requests that "
                    "arrived since its last tick as one array submission per kind (latency from each "
                    "request's arrival); same arrival process, request sequence and server",
            "tick_ms": args.serve_bulk_tick_ms,
            "value": btop["gchar_s"], "unit": "Gchar/s",
            "sustained_req_s": btop["offered_req_s"], "p50_ms_at_sustained": btop["p50_ms"],
            "p99_ms_at_sustained": btop["p99_ms"], "limiter": blimiter,
            "sweep": [{k: r.get(k) for k in keys + ("submissions",)} for r in bulk_runs],
        },
        "plain_per_request": plain, "clocks": clock_info,
    }


def _serve_sweep(run, rates):
    """run(rate, k) for each offered rate, upwards, until the served rate falls
    below 90% of the offered one; each run carries the device's busy share."""
    runs = []
    for k, r in enumerate(rates):
        util = UtilSampler(gpu_index_for(0))
        util.start()
        runs.append(run(r, k))
        runs[-1]["gpu_busy_frac"] = util.stop()
        if runs[-1]["gchar_s"] < 0.9 * runs[-1]["offered_gchar_s"]:
            break
    return runs


def _serve_limiter(runs, loop_name):
    """The highest sustained run, and what limited the next rate: the device (busy
    most of the span) or the host (the request loop busy, the client behind)."""
    sustained = [r for r in runs if r["gchar_s"] >= 0.9 * r["offered_gchar_s"]]
    top = max(sustained, key=lambda r: r["offered_req_s"]) if sustained else runs[0]
    last = runs[-1]
    gpu_busy = last.get("gpu_busy_frac") or 0.0
    loop_busy = last.get("loop_busy_frac") or 0.0
    lag_ms = last.get("client_max_lag_ms") or 0.0
    shares = "request loop busy {:.0%}, device busy {:.0%} of the span, client behind the arrivals by up " \
             "to {:.0f} ms".format(loop_busy, gpu_busy, lag_ms)
    if sustained and last is top:
        return top, "not reached (served >= 90% of offered at the highest rate tried)"
    if loop_busy >= gpu_busy or loop_busy >= 0.8:
        return top, "host: " + loop_name + " (" + shares + ")"
    return top, "GPU (" + shares + ")"


def serve_arm(args):
    r = serve_measure(args)
    line = {
        "metric": METRIC, "value": r["value"], "unit": "Gchar/s", "n_gpus": 1,
        "steps": len(r["sweep"]), "warmup": 1, "ms_per_step": args.serve_seconds * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded request pool, Poisson arrivals)",
        "config": {k: r[k] for k in ("workload", "parallelism", "hbm_budget_bytes", "pnfa_mode")},
        "served": r, "clocks": r["clocks"],
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------------

class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: str):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", self.gpu], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, ValueError):
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, pw, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
                pw.append(float(f[3]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "power_w_max": max(pw) if pw else None,
                "samples": len(sm), "reasons": sorted(reasons)}


class UtilSampler(ClockSampler):
    """Mean of nvidia-smi's utilization.gpu (the share of each sample period in
    which a kernel ran) while it runs, as a fraction."""
    QUERY = "utilization.gpu"

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        v = []
        for ln in self.lines:
            try:
                v.append(float(ln.split(",")[0]))
            except ValueError:
                continue
        return float(np.mean(v)) / 100.0 if v else None


def gpu_index_for(local_rank: int) -> str:
    cvd = os.environ.get("CUDA_VISIBLE_DEVICES")
    if cvd:
        parts = [p.strip() for p in cvd.split(",") if p.strip()]
        if local_rank < len(parts):
            return parts[local_rank]
    return str(local_rank)


def measured_peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def measured_tensor_peak():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d.get("bf16_tflops_sustained", d["bf16_tflops"])), "measured"
    return 1400.0, "fallback"


def committed_traffic(kernel: str, workload: str):
    """DRAM bytes per launch recorded from an ncu capture in profiles/."""
    for f in sorted((REPO / "profiles").glob("*.md")):
        txt = f.read_text()
        m = re.search(rf"traffic_per_launch\[{re.escape(kernel)}\|{re.escape(workload)}\]:\s*([0-9.eE+]+)", txt)
        if m:
            return float(m.group(1))
    return None


# ---------------------------------------------------------------------------------
# measurement
# ---------------------------------------------------------------------------------

def make_workload(args):
    if args.workload == "nfa":
        return NFATcWorkload(args) if args.nfa_method in ("tc", "tc8") else NFAWorkload(args)
    if args.workload == "pnfa":
        return PNFAWorkload(args)
    return DFAWorkload(args)


def sub_args(args, **kw):
    """A copy of the command line for one sub-configuration (defaults for it)."""
    d = dict(vars(args))
    d.update({"strings": None, "seg_len": 0, "kgram": None, "dfa_sizes": None, "nfa_sigma": None,
              "nfa_len": None})
    d.update(kw)
    return argparse.Namespace(**d)


def measure(wl, args, torch, dev, *, steps, warmup, rank=0, world=1, local_rank=0, dist=None,
            e2e_steps=3, verify=True, roof_tag=None):
    """Set up, warm, time `steps` steps between synchronisations on the device
    (CUDA events on the launching stream, max over ranks), the main kernel's
    own time (library events), the end-to-end host-buffer form, and the oracle
    check on the same bytes. Returns a dict (the line's fields)."""
    from trex_b200.engine import profile_begin, profile_end
    seed = rank_seed(args.seed, rank)
    wl.setup(torch, dev, seed)
    stream = torch.cuda.current_stream(dev)
    flush = None
    if wl.chars < 126e6:
        flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    warm = max(3, warmup)
    for _ in range(warm):
        wl.step(stream)
    torch.cuda.synchronize()
    if wl.error_word() != 0:
        raise RuntimeError("device reported malformed input or a look-back timeout")
    clocks = ClockSampler(gpu_index_for(local_rank))
    clocks.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    profile_begin(steps)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        if flush is not None:
            flush.fill_(1)
        wl.step(stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    kern_ms = profile_end(steps)
    clock_info = clocks.stop()
    if wl.error_word() != 0:
        raise RuntimeError("device reported an error during the timed steps")
    ms = ev0.elapsed_time(ev1)
    ms = max_over_ranks(ms, dist, dev)
    ms_per_step = ms / steps
    chars_all = wl.chars * world
    value = chars_all / (ms_per_step * 1e-3) / 1e9

    kmean = sum(kern_ms) / max(1, len(kern_ms))
    traffic = committed_traffic(wl.kernel, roof_tag or args.workload)
    if getattr(wl, "bound", "hbm") == "tensor":
        peak, peak_kind = measured_tensor_peak()
        achieved = wl.alg_flops / (kmean * 1e-3) / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak, "traffic": traffic, "kernel": wl.kernel,
                "kernel_ms_mean": kmean, "algorithmic_flops_per_launch": wl.alg_flops,
                "peak_source": f"MEASURED_PEAKS.json bf16_tflops_sustained ({peak_kind}); "
                               "useful flops 2*64*64 per symbol (the pair layout issues 2x)"}
    else:
        peak, peak_kind = measured_peaks()
        achieved = wl.alg_bytes / (kmean * 1e-3) / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "kernel": wl.kernel,
                "kernel_ms_mean": kmean, "algorithmic_bytes_per_launch": wl.alg_bytes,
                "step_frac": wl.alg_bytes / (ms_per_step * 1e-3) / 1e9 / peak,
                "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({peak_kind})"}

    e2e = None
    if e2e_steps > 0:
        res = wl.e2e(torch, e2e_steps, dist, dev)
        if res is not None:
            dt, h2d, d2h = res
            e2e = {"value": chars_all * e2e_steps / dt / 1e9, "unit": "Gchar/s",
                   "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}
    out = {"value": value, "unit": "Gchar/s", "ms_per_step": ms_per_step, "steps": steps,
           "warmup": warm, "roofline": roof, "e2e": e2e, "clocks": clock_info,
           "gpu_launches": wl.launches_per_step * steps,
           "config": {**wl.config(), "parallelism": f"dp{world} (independent shards, no collective)"}}
    if getattr(wl, "tune_info", None) is not None:
        out["autotune"] = wl.tune_info
    if verify:
        from oracle import oracle as orc
        orc.build()
        mism, secs, nbytes = wl.verify(orc)
        out["mismatches_vs_oracle"] = mism
        out["oracle"] = {"seconds": secs, "gchar_s": nbytes / max(secs, 1e-9) / 1e9,
                         "threads": orc.threads(), "bytes": int(nbytes)}
    return out


def failed_checks(m: dict) -> bool:
    mm = m.get("mismatches_vs_oracle") or {}
    bad = any(v for k, v in mm.items() if k in ("final_state", "accept", "states", "final_mask"))
    return bad or mm.get("loglik_over_tolerance", 0) > 0


def base_line(args, wl, value, ms_per_step, steps, warmup, world):
    return {
        "metric": METRIC, "value": value, "unit": "Gchar/s", "n_gpus": world, "steps": steps,
        "warmup": warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": wl.dtype,
        "data": "synthetic (seeded, generated on the device)",
    }


def reference_arm(args, rank):
    if rank != 0:
        return
    from oracle import oracle as orc
    orc.build()
    threads = orc.threads()
    wl = make_workload(args)
    n_runs = max(1, args.steps + args.warmup)
    per_step = max(0.02, min(2.0, max(args.cpu_seconds, 30.0) / n_runs))
    k, chars, data = wl.cpu_sample(args.seed, per_step, threads)
    times = []
    for step in range(n_runs):
        t0 = time.perf_counter()
        wl.cpu_run(orc, data, k)
        dt = time.perf_counter() - t0
        if step >= args.warmup:
            times.append(dt)
    tot = sum(times)
    value = chars * len(times) / tot / 1e9
    sample = (f"first {k} strings ({chars} bytes) of the workload per step, C oracle "
              f"(restatement of the reference's walk) with OpenMP over {threads} threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Gchar/s",
        "n_gpus": args.gpus, "steps": len(times), "warmup": args.warmup,
        "ms_per_step": tot / len(times) * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": wl.ref_dtype,
        "data": "synthetic (seeded, same generator as the trex arm)",
        "config": {"workload": wl.workload, "n_strings": wl.n, "parallelism": "cpu"},
        "cpu_baseline": {"value": value, "unit": "Gchar/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "Gchar/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gpu_launches": 0,
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------
# extra configurations (default run, one GPU)
# ---------------------------------------------------------------------------------

def plain_per_pattern(args, torch, dev, wl):
    """The ragged batch as one launch per automaton (the plain form): each
    automaton's strings gathered once (outside the timed region), then
    (device) 16 single-automaton sets run back to back on device buffers, and
    (host) 16 reference-style singleton engines, prefix_engine_init + one
    prefix_engine_dispatch per automaton, from pinned host buffers with int32
    offsets. Results are checked against the batched run of the same strings."""
    import ctypes
    from trex_b200 import _lib
    from trex_b200.engine import DFASet
    L = _lib.load()
    hd = wl.host_data if wl.host_data is not None else host_copy(torch, wl.data)
    off, ids = wl.off, wl.ids
    fs_b, ac_b = wl.fs.cpu().numpy(), wl.ac.cpu().numpy()
    lens = np.diff(off)
    pats = []
    for d in range(len(wl.dfas)):
        idx = np.flatnonzero(ids == d)
        starts, ends = off[idx], off[idx + 1]
        blob = np.concatenate([hd[a:b] for a, b in zip(starts.tolist(), ends.tolist())])
        h = torch.from_numpy(blob).pin_memory()
        o = offsets_of(lens[idx])
        pats.append({"idx": idx, "h": h, "off": o, "off32": torch.from_numpy(o.astype(np.int32)).pin_memory(),
                     "d": h.to(dev), "d_off": torch.from_numpy(o).to(dev),
                     "set": DFASet([wl.dfas[d]]),
                     "fs": torch.empty(len(idx), dtype=torch.uint8, device=dev),
                     "ac": torch.empty(len(idx), dtype=torch.uint8, device=dev)})
    for p in pats:
        p["scratch"] = torch.empty(DFASet.scratch_bytes(len(p["idx"]), int(p["off"][-1]), args.seg_len),
                                   dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def dev_step():
        for p in pats:
            p["set"].run(p["d"], p["d_off"], None, final_state=p["fs"], accept=p["ac"],
                         scratch=p["scratch"], seg_len=args.seg_len, stream=stream)

    for _ in range(3):
        dev_step()
    torch.cuda.synchronize()
    steps = 20
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        dev_step()
    ev1.record(stream)
    torch.cuda.synchronize()
    dev_ms = ev0.elapsed_time(ev1) / steps
    mism = 0
    for p in pats:
        mism += int(np.count_nonzero(p["fs"].cpu().numpy() != fs_b[p["idx"]]))
        mism += int(np.count_nonzero(p["ac"].cpu().numpy() != ac_b[p["idx"]]))

    # through the reference ABI (one resident automaton per library): init + dispatch each
    u8 = ctypes.c_uint8
    res = [np.zeros(len(p["idx"]), dtype=np.int32) for p in pats]

    def host_step():
        disp_ms = 0.0
        for d, p in enumerate(pats):
            D = wl.dfas[d]
            tm = np.ascontiguousarray(D.tmap)
            ac = np.ascontiguousarray(D.accept)
            _lib.check(L.prefix_engine_init(_lib.ptr(tm, u8), _lib.ptr(ac, u8), int(D.start), D.n_states, 1,
                                            int(p["off"][-1]), len(p["idx"])), "prefix_engine_init")
            km, tm_ = ctypes.c_float(), ctypes.c_float()
            hdp, hop = p["h"].numpy(), p["off32"].numpy()
            _lib.check(L.prefix_engine_dispatch(_lib.ptr(hdp, u8), _lib.ptr(hop, ctypes.c_int),
                                                _lib.ptr(res[d], ctypes.c_int), len(p["idx"]),
                                                int(p["off"][-1]), ctypes.byref(km), ctypes.byref(tm_)),
                       "prefix_engine_dispatch")
            disp_ms += tm_.value
        L.prefix_engine_destroy()
        return disp_ms

    host_step()
    hsteps = 2
    t0 = time.perf_counter()
    disp = [host_step() for _ in range(hsteps)]
    host_s = (time.perf_counter() - t0) / hsteps
    for d, p in enumerate(pats):
        mism += int(np.count_nonzero(res[d].astype(np.uint8) != ac_b[p["idx"]]))
    for p in pats:
        p["set"].close()
    chars = int(wl.total)
    return {"workload": "the ragged batch (same strings and automata) as 16 per-automaton launches",
            "value": chars / (dev_ms * 1e-3) / 1e9, "unit": "Gchar/s", "ms_per_step": dev_ms,
            "steps": steps, "launches_per_step": 16 * 8,
            "e2e_reference_abi": {"value": chars / host_s / 1e9, "unit": "Gchar/s",
                                  "ms_per_step": host_s * 1e3,
                                  "dispatch_only_value": chars / (np.mean(disp) * 1e-3) / 1e9,
                                  "form": "per automaton: prefix_engine_init (table upload, buffer "
                                          "allocation) + prefix_engine_dispatch (pinned H2D, run, D2H of "
                                          "int results)"},
            "mismatches_vs_batched": mism}


def pnfa_latency(args, torch, dev):
    """One string through the probabilistic NFA chain (64 states, 20 symbols):
    the step latency per position of the tensor-core and CUDA-core kernels."""
    from trex_b200.engine import PNFA
    from trex_b200.workloads import random_prob_nfa
    rng = np.random.default_rng(args.seed)
    T, s, a = random_prob_nfa(rng, 64, 20)
    L = 1 << 16
    data = torch.randint(0, 20, (L,), dtype=torch.uint8, device=dev,
                         generator=torch.Generator(device=dev).manual_seed(args.seed + 9))
    off = torch.tensor([0, L], dtype=torch.int64, device=dev)
    m = PNFA(T, s, a)
    out = {}
    clocks = ClockSampler(gpu_index_for(0))
    clocks.start()
    for mode in ("bf16", "bf16cc", "fp32"):
        for _ in range(2):
            m.run(data, off, mode)
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        reps = 3
        for _ in range(reps):
            m.run(data, off, mode)
        ev1.record()
        torch.cuda.synchronize()
        ns = ev0.elapsed_time(ev1) / reps * 1e6 / L
        out[mode] = {"ns_per_position": ns}
    ci = clocks.stop()
    mhz = ci.get("sm_mhz") or 1965.0
    for v in out.values():
        v["cycles_per_position"] = v["ns_per_position"] * mhz / 1e3
    m.close()
    return {"workload": f"one string of {L} symbols, 64-state probabilistic NFA over 20 symbols",
            "by_mode": out, "sm_mhz": mhz,
            "reference": "82.7 cycles/position: wgmma RS chain, 1 string per warpgroup, H200 "
                         "(cuda/probe_wgmma_layout.cu)"}


def kgram_sweep(args, torch, dev):
    """K-gram widths where grams apply: one 16-state automaton over the bytes
    ACGT, 4M strings x 1024 bytes (4 GB), each width timed like the headline
    (K = 8 needs two letters). The headline batch's automata distinguish all
    256 bytes, so no gram table applies to them (kgram_max 1 each)."""
    out = {}
    for k in (1, 2, 4):
        wl = DFAWorkload(sub_args(args, workload="plain", strings=4 << 20, kgram=k, tuned=False))
        m = measure(wl, wl.args, torch, dev, steps=20, warmup=3, e2e_steps=0, verify=(k == 4),
                    roof_tag="kgram")
        out[f"k{k}"] = {"value": m["value"], "kernel_ms": m["roofline"]["kernel_ms_mean"],
                        "frac": m["roofline"]["frac"], "kgram": m["config"]["kgram"]}
        if "mismatches_vs_oracle" in m:
            out[f"k{k}"]["mismatches_vs_oracle"] = m["mismatches_vs_oracle"]
        wl.close()
        del wl
        torch.cuda.empty_cache()
    return {"workload": "one random 16-state DFA over bytes ACGT, 4M strings x 1024 bytes (4 GB), "
                        "K-gram width forced per run", "by_k": out}


def run_extras(args, torch, dev, main_wl, names):
    extras = {}
    if "plain_per_pattern" in names and isinstance(main_wl, DFAWorkload) and main_wl.kind == "ragged":
        try:
            extras["plain_per_pattern"] = plain_per_pattern(args, torch, dev, main_wl)
        except Exception as e:   # keep the headline; record what failed
            extras["plain_per_pattern"] = {"error": repr(e)[:400]}
    main_wl.close()
    for k in ("data", "d_off", "d_ids", "scratch", "fs", "ac", "states", "host_data"):
        if hasattr(main_wl, k):
            setattr(main_wl, k, None)
    torch.cuda.empty_cache()
    subs = [("cfg1_plain", lambda: DFAWorkload(sub_args(args, workload="plain")), 200, "plain"),
            ("cfg3a_scan", lambda: DFAWorkload(sub_args(args, workload="scan")), 20, "scan"),
            ("cfg3b_nfa", lambda: NFAWorkload(sub_args(args, workload="nfa")), 10, "nfa"),
            ("cfg3b_nfa_tensor_bf16", lambda: NFATcWorkload(sub_args(args, workload="nfa", nfa_method="tc")),
             2, "nfa_tc"),
            ("cfg3b_nfa_tensor_int8", lambda: NFATcWorkload(sub_args(args, workload="nfa", nfa_method="tc8")),
             2, "nfa_tc8"),
            ("cfg4_pnfa", lambda: PNFAWorkload(sub_args(args, workload="pnfa", pnfa_mode="bf16")), 5, "pnfa"),
            ("dfa_n32_64", lambda: DFAWorkload(sub_args(args, workload="ragged", dfa_sizes="32,64",
                                                        strings=250_000)), 5, "ragged_n32_64")]
    for name, make, steps, tag in subs:
        if name.split("_tensor")[0] not in names:
            continue
        try:
            wl = make()
            extras[name] = measure(wl, wl.args, torch, dev, steps=steps, warmup=3,
                                   e2e_steps=0 if "tensor" in name else 2, roof_tag=tag)
            wl.close()
            del wl
        except Exception as e:
            extras[name] = {"error": repr(e)[:400]}
        torch.cuda.empty_cache()
    if "ref_shapes" in names:
        extras["ref_shapes"] = ref_shapes(args, torch, dev)
    if "cfg4_pnfa" in names:
        try:
            extras["cfg4_pnfa_latency"] = pnfa_latency(args, torch, dev)
        except Exception as e:
            extras["cfg4_pnfa_latency"] = {"error": repr(e)[:400]}
    if "kgram_sweep" in names:
        try:
            extras["kgram_sweep"] = kgram_sweep(args, torch, dev)
        except Exception as e:
            extras["kgram_sweep"] = {"error": repr(e)[:400]}
    if "frontend" in names:
        try:
            extras["frontend"] = frontend_measure(args)
        except Exception as e:
            extras["frontend"] = {"error": repr(e)[:400]}
    if "cfg5_served" in names:
        try:
            extras["cfg5_served"] = serve_measure(args)
        except Exception as e:
            extras["cfg5_served"] = {"error": repr(e)[:400]}
    return extras


FRONTEND_PATTERNS = ("[a-z]+@[a-z]+\\.[a-z]+", "(if|else|while|for|return)", "((ab|cd)(ef|gh))+",
                     "\\d+\\.\\d*", "(a|b)*abb")


def frontend_measure(args) -> dict:
    """The regex front end through the drop-in OptimizedEngine (README form,
    config "auto"): engine setup per pattern (regex -> minimal DFA -> byte table ->
    resident set on the device), the host preparation of a list of Python strings
    (one byte buffer plus offsets: the character -> index map is folded into the
    byte table, so no per-character mapping runs), and match_batch end to end,
    per million characters; results checked against the CPU engine (config
    "baseline") on every string."""
    from trex_b200._batching import pack_strings
    from trex_b200.optimized_engine import OptimizedEngine
    rng = np.random.default_rng(args.seed + 29)
    alphabet = np.frombuffer(b"abcdefghijklmnopqrstuvwxyz0123456789.@ ", dtype=np.uint8)
    n, L = 1000, 1000   # 1 Mchar a batch
    strings = [alphabet[rng.integers(0, len(alphabet), size=int(x))].tobytes().decode("latin-1")
               for x in rng.integers(L // 2, 3 * L // 2, size=n)]
    # twenty strings each pattern accepts, so both outcomes are checked
    for k in rng.integers(20, 200, size=20).tolist():
        strings += ["abc" * k + "@" + "def" * k + ".com", "while", "abefcdgh" * k,
                    "1" * k + "." + "2" * k, "ab" * k + "abb"]
    mchar = sum(len(x) for x in strings) / 1e6
    prep = []
    for _ in range(5):
        t0 = time.perf_counter()
        pack_strings(strings, offset_dtype=np.int64)
        prep.append((time.perf_counter() - t0) * 1e3)
    out = {"workload": "5 regexes; 1000 random Python str of 500-1500 characters plus 100 that the "
                       "patterns accept (1.05 Mchar) a batch",
           "host_prep_ms_per_mchar": float(np.median(prep)) / mchar,
           "reference_host_prep_ms_per_mchar": 88.0,
           "patterns": []}
    mism = 0
    for p in FRONTEND_PATTERNS:
        t0 = time.perf_counter()
        eng = OptimizedEngine(p, config="auto")
        setup_ms = (time.perf_counter() - t0) * 1e3
        eng.match_batch(strings)   # warm
        ts = []
        for _ in range(5):
            t0 = time.perf_counter()
            res = eng.match_batch(strings)
            ts.append((time.perf_counter() - t0) * 1e3)
        cpu = OptimizedEngine(p, config="baseline")
        want = cpu.match_batch(strings)
        mism += sum(a != b for a, b in zip(res, want))
        info = eng.config_info
        out["patterns"].append({"pattern": p, "backend": info.get("scan_backend"),
                                "dfa_states": info.get("dfa_states"),
                                "setup_ms": setup_ms, "match_ms_per_mchar": float(np.median(ts)) / mchar,
                                "accepted": int(sum(res))})
        eng.close()
    out["mismatches_vs_cpu_engine"] = int(mism)
    return out


def ref_shapes(args, torch, dev):
    """The NFA kernels on the shape the reference publishes its NFA numbers for: 64 states,
    sigma 2, 262144 strings x 2048 symbols (README.md:12-15, H200), each checked against the
    oracle like the default configurations."""
    R = 262144
    kw = dict(nfa_sigma=2, nfa_len=2048, strings=R)
    runs = [("nfa_bitpar", lambda: NFAWorkload(sub_args(args, workload="nfa", **kw)), 10,
             {"value": 185.0, "kernel": "bit-parallel V4", "source": "README.md:12"}),
            ("nfa_tensor_int8", lambda: NFATcWorkload(sub_args(args, workload="nfa", nfa_method="tc8", **kw)), 2,
             {"value": 12.5, "kernel": "tensor-core V3 (FP16 WMMA, 0/1 operands)", "source": "README.md:14"}),
            ("pnfa_fp16", lambda: PNFAWorkload(sub_args(args, workload="pnfa", pnfa_mode="fp16", **kw)), 3,
             {"value": 10.9, "kernel": "probabilistic V5 (FP16 WMMA)", "source": "README.md:15"}),
            ("pnfa_bf16", lambda: PNFAWorkload(sub_args(args, workload="pnfa", pnfa_mode="bf16", **kw)), 3,
             {"value": 10.9, "kernel": "probabilistic V5 (FP16 WMMA)", "source": "README.md:15"})]
    out = {}
    for name, make, steps, pub in runs:
        try:
            wl = make()
            m = measure(wl, wl.args, torch, dev, steps=steps, warmup=3, e2e_steps=0, roof_tag="ref_" + name)
            m["reference_published"] = dict(pub, unit="Gchar/s", hardware="H200")
            out[name] = m
            wl.close()
            del wl
        except Exception as e:
            out[name] = {"error": repr(e)[:400]}
        torch.cuda.empty_cache()
    return {"shape": f"64-state NFAs over 2 symbols, {R} strings x 2048 symbols", "by_kernel": out}


def trex_arm(args, rank, world, local_rank):
    import torch
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import torch.distributed as dist
    wl = make_workload(args)
    verify = not args.no_verify and rank == 0 and world == 1
    m = measure(wl, args, torch, dev, steps=args.steps, warmup=args.warmup, rank=rank, world=world,
                local_rank=local_rank, dist=dist, e2e_steps=args.e2e_steps, verify=verify)
    failed = failed_checks(m)
    if rank == 0:
        line = base_line(args, wl, m["value"], m["ms_per_step"], args.steps, m["warmup"], world)
        for k in ("config", "roofline", "autotune", "mismatches_vs_oracle", "e2e"):
            if k in m:
                line[k] = m[k]
        cpu = None
        if verify and not args.no_cpu_baseline:
            o = m["oracle"]
            cpu = {"value": o["gchar_s"], "unit": "Gchar/s", "cores": o["threads"], "kind": "port",
                   "sample": (f"the oracle check of this run: {o['bytes']} bytes of the batch (every "
                              f"string checked where the workload is a DFA, NFA or scan batch), the "
                              f"same bytes as the GPU run, OpenMP over {o['threads']} threads")}
        line["cpu_baseline"] = cpu
        line["gpu_launches"] = m["gpu_launches"]
        line["clocks"] = m["clocks"]
        if world == 1 and not args.no_extras:
            names = set(x.strip() for x in args.extras.split(",") if x.strip())
            line["configs"] = run_extras(args, torch, dev, wl, names)
            for v in line["configs"].values():
                failed |= isinstance(v, dict) and (failed_checks(v) or bool(v.get("mismatches_vs_batched")))
            for v in line["configs"].get("ref_shapes", {}).get("by_kernel", {}).values():
                failed |= isinstance(v, dict) and failed_checks(v)
        else:
            wl.close()
        print(json.dumps(line), flush=True)
    else:
        wl.close()
    if failed:
        raise SystemExit("results differ from the oracle (see mismatches_vs_oracle)")


def main():
    args = parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank)
        return
    if args.workload == "serve":
        if rank == 0:
            serve_arm(args)
        return
    if args.workload != "ragged":
        args.no_extras = True
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        try:
            trex_arm(args, rank, world, local_rank)
        finally:
            dist.destroy_process_group()
    else:
        trex_arm(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
