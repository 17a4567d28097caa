"""Bounded device waits that run out (failure detection without a GPU fault).

The per-position scan's decoupled look-back polls the status word of the
previous chunk (the reference spins on it without a limit,
cuda/monoid_scan.cu:187-193), and the tensor-core NFA kernel hands work between
its warp roles through mbarriers. Every such wait here has a limit; when it
runs out the kernel sets the timeout bit (4) of the run's error word, stops,
frees what it holds and returns. These tests shrink the limits with
trex_set_wait_limits so that waits must give up, check that the launch
returns with the bit set and that the context stays usable, then restore the
defaults and check that the next run is correct. Nothing here faults or hangs
the GPU: the limits only make the kernels give up sooner.
"""

import numpy as np
import pytest

from trex_b200.workloads import random_dfa, random_prob_nfa

pytestmark = pytest.mark.gpu


def _limits(scan_polls, mbar_cycles):
    from trex_b200 import _lib
    _lib.check(_lib.load().trex_set_wait_limits(scan_polls, mbar_cycles), "trex_set_wait_limits")


def test_scan_lookback_gives_up_then_recovers(cuda, oracle):
    torch = cuda
    from trex_b200.engine import DFASet
    rng = np.random.default_rng(77)
    dfa = random_dfa(16, np.arange(256), rng)
    total = 64 << 20   # 65536 tiles of 1 KiB: 2048 chunks, all in flight at once
    data = rng.integers(0, 256, size=total, dtype=np.uint8)
    off = np.array([0, total], dtype=np.int64)
    d, o = torch.from_numpy(data).cuda(), torch.from_numpy(off).cuda()
    s = DFASet([dfa])
    try:
        timed_out = False
        _limits(1, 0)   # one poll per look-back step
        for _ in range(3):   # a step gives up only when its predecessor is not ready yet
            st, fs, ac, sc = s.scan(d, o, 0, tile_len=1024)
            torch.cuda.synchronize()   # the launch returned
            if s.scan_error_word(sc, 1, total, 1024) & 4:
                timed_out = True
                break
        assert timed_out, "no look-back step gave up with a one-poll limit"
    finally:
        _limits(0, 0)
    st, fs, ac, sc = s.scan(d, o, 0, tile_len=1024)
    torch.cuda.synchronize()
    assert s.scan_error_word(sc, 1, total, 1024) == 0
    ref = oracle.dfa_positions(dfa.tmap, 16, 0, data, off)
    assert np.array_equal(st.cpu().numpy(), ref)
    assert int(fs.cpu()[0]) == int(ref[-1])
    s.close()


@pytest.mark.parametrize("mode", ["bf16", "bool8"])
def test_tensor_nfa_handoff_gives_up_then_recovers(cuda, oracle, mode):
    torch = cuda
    from trex_b200.engine import PNFA
    rng = np.random.default_rng(78)
    T, start, acc = random_prob_nfa(rng, 64, 20)
    n, L = 4000, 96
    data = rng.integers(0, 20, size=n * L, dtype=np.uint8)
    off = np.arange(n + 1, dtype=np.int64) * L
    d, o = torch.from_numpy(data).cuda(), torch.from_numpy(off).cuda()
    m = PNFA(T, start, acc)
    try:
        _limits(0, 1)   # every hand-off that is not ready at its first poll gives up
        m.run(d, o, mode)
        torch.cuda.synchronize()   # the launch returned; the TMEM was freed
        assert m.error_word() & 4
    finally:
        _limits(0, 0)
    ll, ac = m.run(d, o, mode)
    torch.cuda.synchronize()
    assert m.error_word() == 0
    if mode == "bool8":
        _, ref = oracle.nfa_bool(T != 0, start, acc, data, off, unknown_rejects=False)
        assert np.array_equal(ac.cpu().numpy().astype(bool), ref.astype(bool))
    else:
        ref = oracle.pnfa_fp64(T, start, acc, data, off)
        got = ll.cpu().numpy()
        k = np.diff(off)
        assert np.all(np.abs(got - ref) <= np.maximum(1e-4 * np.abs(ref), 2.0 ** -8 * (k + 1)))
    m.close()
