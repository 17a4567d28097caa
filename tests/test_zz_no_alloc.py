"""The allocation-free batch entry point (trex_dfa_batch_run_static).

It serves callers that cannot allocate device memory during a run (a foreign
allocator owns the GPU memory, a real-time loop must stay out of the driver's
allocator): its scratch is a static 8 MiB device array instead of a
cudaMalloc'd buffer.

The test makes the static calls first, on a fresh automaton set that has never
run an allocating batch, and checks that the device's free memory is the same
before and after them (the set's own scratch is never made). It calls the
entry point through the C ABI twice in a row, on two different batches and on
two streams, and checks each result against the allocating entry point
trex_dfa_batch_run on the same batch (bit-exact: final states and accept flags
are integers). The second call also shows that what the first call left in the
shared array does not leak into the next result. Overlapping offsets must
raise the capacity bit in trex_dfa_batch_static_error with no output written,
and a batch above the 8 MiB limit must be refused.

This file is named to be collected last, so a run that stops at the first
failure has run every other test before it.
"""

import ctypes

import numpy as np
import pytest

from trex_b200.workloads import random_dfa, ragged_batch

pytestmark = pytest.mark.gpu


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _batch(torch, rng, n, median, hi, n_dfas):
    data, off, ids, _ = ragged_batch(n, rng, median=median, hi=hi, n_dfas=n_dfas)
    return (torch.from_numpy(data).cuda(), torch.from_numpy(off).cuda(),
            torch.from_numpy(ids).cuda(), len(off) - 1, data.size)


def _static_error(L, s):
    v = ctypes.c_int32(-1)
    assert L.trex_dfa_batch_static_error(s.handle, ctypes.byref(v)) == 0
    return v.value


def test_static_scratch_matches_allocating_entry_point(cuda):
    torch = cuda
    from trex_b200 import _lib
    from trex_b200.engine import DFASet
    L = _lib.load()
    rng = np.random.default_rng(2024)
    dfas = [random_dfa(n, np.arange(256), rng) for n in (8, 12, 16, 5)]
    s = DFASet(dfas)
    side = torch.cuda.Stream()
    streams = [ctypes.c_void_p(torch.cuda.current_stream().cuda_stream),
               ctypes.c_void_p(side.cuda_stream)]
    batches = [_batch(torch, rng, 3000, 600, 9000, len(dfas)),    # split strings included
               _batch(torch, rng, 1700, 300, 4000, len(dfas))]
    cases = [(seg_len, b) for seg_len in (256, 0) for b in batches]
    outs = []
    for seg_len, (data, off, ids, n, total) in cases:
        outs.append((torch.full((n,), 255, dtype=torch.uint8, device="cuda"),
                     torch.full((n,), 255, dtype=torch.uint8, device="cuda"),
                     torch.full((n,), -1, dtype=torch.int32, device="cuda")))

    def run_static(k, stream):
        seg_len, (data, off, ids, n, total) = cases[k]
        fs, ac, ac32 = outs[k]
        rc = L.trex_dfa_batch_run_static(s.handle, _p(data), _p(off), _p(ids), n, total,
                                         _p(fs), _p(ac), _p(ac32), seg_len, stream)
        assert rc == 0, _lib.last_error()

    # set-up call (looks up the static array on this device), then the measured calls
    run_static(0, streams[0])
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for k in range(len(cases)):
        run_static(k, streams[k % 2])
        torch.cuda.synchronize()   # calls on different streams must not overlap
        assert _static_error(L, s) == 0
    assert torch.cuda.mem_get_info()[0] == free0, "the static entry point allocated device memory"

    # the same batches through the allocating entry point
    stream = streams[0]
    for k, (seg_len, (data, off, ids, n, total)) in enumerate(cases):
        ref_fs = torch.empty(n, dtype=torch.uint8, device="cuda")
        ref_ac = torch.empty(n, dtype=torch.uint8, device="cuda")
        rc = L.trex_dfa_batch_run(s.handle, _p(data), _p(off), _p(ids), n, total, _p(ref_fs),
                                  _p(ref_ac), None, None, 0, seg_len, stream)
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        fs, ac, ac32 = outs[k]
        assert torch.equal(fs, ref_fs)
        assert torch.equal(ac, ref_ac)
        assert torch.equal(ac32, ref_ac.to(torch.int32))

    # overlapping offsets: the whole batch is skipped and the capacity bit (4) is raised
    data, off, ids, n, total = batches[1]
    bad = off.clone()
    bad[0::2] = 0             # strings 0, 2, 4, ... span the whole buffer (far more work items
    bad[1::2] = total         # than the scratch holds); 1, 3, 5, ... end before they start
    fs = torch.full((n,), 255, dtype=torch.uint8, device="cuda")
    rc = L.trex_dfa_batch_run_static(s.handle, _p(data), _p(bad), _p(ids), n, total, _p(fs), None,
                                     None, 256, stream)
    assert rc == 0, _lib.last_error()
    torch.cuda.synchronize()
    assert _static_error(L, s) & 4
    assert bool((fs == 255).all()), "a refused batch wrote outputs"
    # and the next good call clears the word
    run_static(1, stream)
    torch.cuda.synchronize()
    assert _static_error(L, s) == 0

    # beyond the static limit: refused, nothing launched
    big_n = 1_000_000
    assert L.trex_dfa_batch_scratch_bytes(big_n, 1 << 30, 0) > 8 << 20
    rc = L.trex_dfa_batch_run_static(s.handle, _p(batches[0][0]), _p(batches[0][1]), None, big_n,
                                     1 << 30, None, None, None, 0, stream)
    assert rc == -4
    s.close()
