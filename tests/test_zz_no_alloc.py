"""The allocation-free batch entry point (trex_dfa_batch_run_static).

It serves callers that cannot allocate device memory during a run (a foreign
allocator owns the GPU memory, a real-time loop must stay out of the driver's
allocator): its scratch is a static 8 MiB
device array instead of a cudaMalloc'd buffer. This test calls it through the
C ABI twice in a row, on two different batches, and checks each result
against the allocating entry point trex_dfa_batch_run on the same batch
(bit-exact: final states and accept flags are integers). The second call
also shows that what the first call left in the shared array does not leak
into the next result. A batch above the 8 MiB limit must be refused.

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


def test_static_scratch_matches_allocating_entry_point(cuda):
    torch = cuda
    from trex_b200 import _lib
    from trex_b200.engine import DFASet
    L = _lib.load()
    rng = np.random.default_rng(2024)
    dfas = [random_dfa(n, np.arange(256), rng) for n in (8, 12, 16, 5)]
    s = DFASet(dfas)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    batches = [_batch(torch, rng, 3000, 600, 9000, len(dfas)),    # split strings included
               _batch(torch, rng, 1700, 300, 4000, len(dfas))]
    for seg_len in (256, 0):
        for data, off, ids, n, total in batches:
            ref_fs = torch.empty(n, dtype=torch.uint8, device="cuda")
            ref_ac = torch.empty(n, dtype=torch.uint8, device="cuda")
            rc = L.trex_dfa_batch_run(s.handle, _p(data), _p(off), _p(ids), n, total, _p(ref_fs),
                                      _p(ref_ac), None, None, 0, seg_len, stream)
            assert rc == 0, _lib.last_error()
            fs = torch.full((n,), 255, dtype=torch.uint8, device="cuda")
            ac = torch.full((n,), 255, dtype=torch.uint8, device="cuda")
            ac32 = torch.full((n,), -1, dtype=torch.int32, device="cuda")
            rc = L.trex_dfa_batch_run_static(s.handle, _p(data), _p(off), _p(ids), n, total,
                                             _p(fs), _p(ac), _p(ac32), seg_len, stream)
            assert rc == 0, _lib.last_error()
            torch.cuda.synchronize()
            assert torch.equal(fs, ref_fs)
            assert torch.equal(ac, ref_ac)
            assert torch.equal(ac32, ref_ac.to(torch.int32))
    # beyond the static limit: refused, nothing launched
    big_n = 1_000_000
    assert L.trex_dfa_batch_scratch_bytes(big_n, 1 << 30, 0) > 8 << 20
    rc = L.trex_dfa_batch_run_static(s.handle, _p(batches[0][0]), _p(batches[0][1]), None, big_n,
                                     1 << 30, None, None, None, 0, stream)
    assert rc == -4
    s.close()
