"""Benchmark: ragged DFA batch on B200 (one JSON line on stdout, rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl trex|reference]
                    [--workload ragged|plain] [--strings S]

Workload (default, the benchmark's headline case): 16 random DFAs (5 x 8,
5 x 12, 6 x 16 states) over all 256 byte values, 1M strings with log-normal
lengths (median 2048, sigma 1.18, clipped to [16, 65536], ~4.1 GB), 10% of
the strings over the 4-byte sub-alphabet "ACGT", string i on DFA i mod 16.
Inputs are generated on the device from a seed (synthetic; the reference
ships no dataset). One step = one ragged launch over the whole batch.

Multi-GPU: one process per GPU (torchrun); every rank runs its own seeded
batch (weak scaling, no data-path collective); timings are the max over
ranks (NCCL all-reduce of one float).

--impl reference times the reference's CPU algorithm (the C oracle,
oracle/oracle.c, a restatement of DFA.simulate over the byte map) on the
host cores over a bounded sample of the same workload.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "Gchar/s vs HBM roofline, plain vs batched/served; served p50/p99 ms (1 B200)"
SUB_ALPHABET = b"ACGT"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["trex", "reference"], default="trex")
    ap.add_argument("--workload", choices=["ragged", "plain"], default="ragged")
    ap.add_argument("--strings", type=int, default=None, help="override the number of strings")
    ap.add_argument("--seg-len", type=int, default=0)
    ap.add_argument("--dfa-sizes", type=str, default=None,
                    help="comma list of DFA state counts replacing the default 5x8,5x12,6x16")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="CPU budget of the cpu_baseline sample (trex arm) / of the whole run (reference arm)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


# ---------------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------------

def workload_spec(kind: str, n_override=None):
    if kind == "plain":
        n = n_override or 4096
        return dict(workload="plain DFA: N=16 random DFA over bytes ACGT, 4096 strings x 1024 bytes",
                    n_strings=n, kind=kind)
    n = n_override or 1_000_000
    return dict(workload=("ragged DFA batch: 16 random DFAs (5x8, 5x12, 6x16 states) over 256 byte "
                          "symbols; 1M strings, log-normal lengths median 2048 sigma 1.18 clipped "
                          "[16, 65536]; 10% of strings over 'ACGT'; string i on DFA i mod 16"),
                n_strings=n, kind=kind)


def make_automata(kind: str, seed: int, sizes_override=None):
    from trex_b200.workloads import ACGT, random_dfa
    rng = np.random.default_rng(seed)
    if kind == "plain":
        return [random_dfa(16, ACGT, rng)]
    sizes = (8,) * 5 + (12,) * 5 + (16,) * 6
    if sizes_override:
        base = [int(x) for x in sizes_override.split(",")]
        sizes = [base[i % len(base)] for i in range(16)]
    return [random_dfa(n, np.arange(256), rng) for n in sizes]


def make_lengths(kind: str, n: int, seed: int):
    from trex_b200.workloads import lognormal_lengths
    rng = np.random.default_rng(seed + 1)
    if kind == "plain":
        lens = np.full(n, 1024, dtype=np.int64)
        is_sub = np.ones(n, dtype=bool)
    else:
        lens = lognormal_lengths(n, rng)
        is_sub = np.zeros(n, dtype=bool)
        is_sub[rng.choice(n, size=int(round(0.10 * n)), replace=False)] = True
    off = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    n_dfas = 1 if kind == "plain" else 16
    ids = (np.arange(n) % n_dfas).astype(np.int32)
    return lens, off, ids, is_sub


def make_device_bytes(torch, lens, is_sub, seed, device):
    """Uniform random bytes; strings flagged is_sub are re-drawn over ACGT."""
    total = int(lens.sum())
    g = torch.Generator(device=device)
    g.manual_seed(seed + 2)
    data = torch.randint(0, 256, (max(total, 1),), dtype=torch.uint8, device=device, generator=g)
    if is_sub.any():
        acgt = torch.tensor(list(SUB_ALPHABET), dtype=torch.uint8, device=device)
        flag = torch.repeat_interleave(torch.from_numpy(is_sub).to(device),
                                       torch.from_numpy(lens).to(device))
        codes = acgt[(data[:total] & 3).long()]
        data[:total] = torch.where(flag, codes, data[:total])
        del flag, codes
    return data[:total]


def make_host_bytes(lens, is_sub, seed):
    rng = np.random.default_rng(seed + 3)
    total = int(lens.sum())
    data = rng.integers(0, 256, size=total, dtype=np.uint8)
    if is_sub.any():
        off = np.zeros(len(lens) + 1, dtype=np.int64)
        np.cumsum(lens, out=off[1:])
        acgt = np.frombuffer(SUB_ALPHABET, dtype=np.uint8)
        for i in np.flatnonzero(is_sub):
            a, b = off[i], off[i + 1]
            data[a:b] = acgt[data[a:b] & 3]
    return data


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


def gpu_index_for(local_rank: int) -> str:
    cvd = os.environ.get("CUDA_VISIBLE_DEVICES")
    if cvd:
        parts = [p.strip() for p in cvd.split(",") if p.strip()]
        if local_rank < len(parts):
            return parts[local_rank]
    return str(local_rank)


# ---------------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------------

def measured_peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def committed_traffic(kernel: str, workload: str):
    """DRAM bytes per launch recorded from an ncu capture in profiles/."""
    for f in sorted((REPO / "profiles").glob("*.md")):
        txt = f.read_text()
        m = re.search(rf"traffic_per_launch\[{re.escape(kernel)}\|{re.escape(workload)}\]:\s*([0-9.eE+]+)", txt)
        if m:
            return float(m.group(1))
    return None


def cpu_sample(off, seconds_budget, rate_guess_bps):
    """Number of leading strings whose bytes take about `seconds_budget` at
    `rate_guess_bps`."""
    target = seconds_budget * rate_guess_bps
    k = int(np.searchsorted(off, target, side="right")) - 1
    return max(1, min(k, len(off) - 1))


def run_cpu_baseline(dfas, data_host, off, ids, budget_s):
    from oracle import oracle as orc
    orc.build()
    threads = orc.threads()
    # calibrate on ~0.05 s of work, then run the bounded sample
    k0 = cpu_sample(off, 0.05, 3e8 * threads)
    t0 = time.perf_counter()
    orc.dfa_walk([d.tmap for d in dfas], [d.n_states for d in dfas], [d.start for d in dfas],
                 [d.accept for d in dfas], data_host[:off[k0]], off[:k0 + 1], ids[:k0])
    rate = off[k0] / max(time.perf_counter() - t0, 1e-6)
    k = cpu_sample(off, budget_s, rate)
    t0 = time.perf_counter()
    orc.dfa_walk([d.tmap for d in dfas], [d.n_states for d in dfas], [d.start for d in dfas],
                 [d.accept for d in dfas], data_host[:off[k]], off[:k + 1], ids[:k])
    dt = time.perf_counter() - t0
    chars = int(off[k])
    return {"value": chars / dt / 1e9, "unit": "Gchar/s", "cores": threads, "kind": "port",
            "sample": f"first {k} strings ({chars} bytes) of the same workload, OpenMP over {threads} threads"}


# ---------------------------------------------------------------------------------
# arms
# ---------------------------------------------------------------------------------

def reference_arm(args, rank):
    if rank != 0:
        return
    spec = workload_spec(args.workload, args.strings)
    dfas = make_automata(args.workload, args.seed, args.dfa_sizes)
    lens, off, ids, is_sub = make_lengths(args.workload, spec["n_strings"], args.seed)
    from oracle import oracle as orc
    orc.build()
    threads = orc.threads()
    # per-step sample sized so warmup + steps fit the CPU budget
    n_runs = max(1, args.steps + args.warmup)
    # host bytes for a generous prefix only
    calib_k = cpu_sample(off, 0.02, 3e8 * threads)
    sample_data = make_host_bytes(lens[:calib_k], is_sub[:calib_k], args.seed)
    t0 = time.perf_counter()
    orc.dfa_walk([d.tmap for d in dfas], [d.n_states for d in dfas], [0] * len(dfas),
                 [d.accept for d in dfas], sample_data, off[:calib_k + 1], ids[:calib_k])
    rate = off[calib_k] / max(time.perf_counter() - t0, 1e-6)
    per_step_s = max(0.05, min(2.0, (max(args.cpu_seconds, 30.0)) / n_runs))
    k = cpu_sample(off, per_step_s, rate)
    data = make_host_bytes(lens[:k], is_sub[:k], args.seed)
    times = []
    for step in range(n_runs):
        t0 = time.perf_counter()
        orc.dfa_walk([d.tmap for d in dfas], [d.n_states for d in dfas], [0] * len(dfas),
                     [d.accept for d in dfas], data, off[:k + 1], ids[:k])
        dt = time.perf_counter() - t0
        if step >= args.warmup:
            times.append(dt)
    chars = int(off[k])
    tot = sum(times)
    value = chars * len(times) / tot / 1e9
    sample = (f"first {k} strings ({chars} bytes) of the workload per step, C oracle "
              f"(restatement of DFA.simulate over the byte map) with OpenMP over {threads} threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Gchar/s",
        "n_gpus": args.gpus, "steps": len(times), "warmup": args.warmup,
        "ms_per_step": tot / len(times) * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded, same generator as the trex arm)",
        "config": {**{k_: v for k_, v in spec.items() if k_ != "kind"}, "parallelism": "cpu"},
        "cpu_baseline": {"value": value, "unit": "Gchar/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "Gchar/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gpu_launches": 0,
    }
    print(json.dumps(line), flush=True)


def trex_arm(args, rank, world, local_rank):
    import torch
    from trex_b200.engine import DFASet, profile_begin, profile_end
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import torch.distributed as dist
    spec = workload_spec(args.workload, args.strings)
    seed = args.seed + 7919 * rank
    dfas = make_automata(args.workload, args.seed, args.dfa_sizes)
    lens, off, ids, is_sub = make_lengths(args.workload, spec["n_strings"], seed)
    data = make_device_bytes(torch, lens, is_sub, seed, dev)
    d_off = torch.from_numpy(off).to(dev)
    d_ids = torch.from_numpy(ids).to(dev)
    n = spec["n_strings"]
    total = int(off[-1])
    s = DFASet(dfas)
    scratch = torch.empty(DFASet.scratch_bytes(n, total, args.seg_len), dtype=torch.uint8, device=dev)
    fs = torch.empty(n, dtype=torch.uint8, device=dev)
    ac = torch.empty(n, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        s.run(data, d_off, d_ids, final_state=fs, accept=ac, scratch=scratch, seg_len=args.seg_len,
              stream=stream)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    if s.last_error_word(scratch) != 0:
        raise RuntimeError("device reported malformed input")
    clocks = ClockSampler(gpu_index_for(local_rank))
    clocks.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    profile_begin(args.steps)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    kern_ms = profile_end(args.steps)
    clock_info = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    t_max = ms
    if dist:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max = float(t.item())
    ms_per_step = t_max / args.steps
    chars_all = total * world
    value = chars_all / (ms_per_step * 1e-3) / 1e9

    # roofline of the dominant kernel (dfa_ragged_kernel)
    peak, peak_kind = measured_peaks()
    alg_bytes = total + 16 * n
    kmean = sum(kern_ms) / max(1, len(kern_ms))
    achieved = alg_bytes / (kmean * 1e-3) / 1e9
    traffic = committed_traffic("dfa_ragged_kernel", args.workload)

    # end to end through the host-buffer C ABI entry point (pinned buffers)
    e2e = None
    if rank == 0 or world > 1:
        h_data = torch.empty(total, dtype=torch.uint8, pin_memory=True)
        h_data.copy_(data)
        h_off = torch.from_numpy(off).pin_memory()
        h_ids = torch.from_numpy(ids).pin_memory()
        h_fs = torch.empty(n, dtype=torch.uint8).pin_memory()
        h_ac = torch.empty(n, dtype=torch.uint8).pin_memory()
        hd, ho, hi, hf, ha = (h_data.numpy(), h_off.numpy(), h_ids.numpy(), h_fs.numpy(), h_ac.numpy())
        s.run_host(hd, ho, hi, args.seg_len, hf, ha)  # warm the staging buffers
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            s.run_host(hd, ho, hi, args.seg_len, hf, ha)
        dt = time.perf_counter() - t0
        if dist:
            t = torch.tensor([dt], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            dt = float(t.item())
        if not (np.array_equal(hf, fs.cpu().numpy()) and np.array_equal(ha, ac.cpu().numpy())):
            raise RuntimeError("host-buffer run disagrees with the device run")
        e2e = {"value": chars_all * args.e2e_steps / dt / 1e9, "unit": "Gchar/s",
               "h2d_bytes_per_step": int(total + off.nbytes + ids.nbytes),
               "d2h_bytes_per_step": int(2 * n + 4)}
        cpu_data = hd
    else:
        cpu_data = None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = run_cpu_baseline(dfas, cpu_data, off, ids, args.cpu_seconds)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Gchar/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic (seeded, generated on the device)",
            "config": {**{k: v for k, v in spec.items() if k != "kind"},
                       "total_bytes_per_gpu": total, "seg_len": args.seg_len or 8192,
                       "l2": "inputs (>= 4 GB) larger than L2, no flush",
                       "parallelism": f"dp{world} (independent shards, no collective)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": "dfa_ragged_kernel", "kernel_ms_mean": kmean,
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({peak_kind})"},
            "e2e": e2e,
            "cpu_baseline": cpu,
            "gpu_launches": 4 * args.steps,
            "clocks": clock_info,
        }
        print(json.dumps(line), flush=True)
    s.close()


def main():
    args = parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank)
        return
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
