"""The reference's ctypes bridge behaviour against this library.

The reference's Python bridge (src/gpu_bridge_prefix_compose.py:24-164) opens
``build/libprefix_compose.so``, declares prefix_engine_device_check / init /
dispatch / destroy with 32-bit ints and raw pointers, calls device_check, then
init(tmap, accept, start, N, K=32, max_total_chars, max_batch), then dispatch
with int32 CSR offsets and int32 results, and destroy. This test does the same
through the symlink that the build makes with the reference's library name,
with declarations of the same types, and checks every result against the
automaton's own walk. It exercises the drop-in claim without importing the
reference (which is not present where the GPU tests run).
"""

import ctypes
import random
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REPO = Path(__file__).resolve().parent.parent


def _declare(lib):
    u8p, ip, fp = ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float)
    lib.prefix_engine_device_check.restype = ctypes.c_int
    lib.prefix_engine_device_check.argtypes = []
    lib.prefix_engine_init.restype = ctypes.c_int
    lib.prefix_engine_init.argtypes = [u8p, u8p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int]
    lib.prefix_engine_destroy.restype = None
    lib.prefix_engine_destroy.argtypes = []
    lib.prefix_engine_dispatch.restype = ctypes.c_int
    lib.prefix_engine_dispatch.argtypes = [u8p, ip, ip, ctypes.c_int, ctypes.c_int, fp, fp]
    return u8p, ip


def _dispatch(lib, strings, u8p, ip):
    B = len(strings)
    off = np.zeros(B + 1, dtype=np.int32)
    for i, s in enumerate(strings):
        off[i + 1] = off[i] + len(s)
    raw = np.frombuffer("".join(strings).encode("latin-1"), dtype=np.uint8).copy() if off[-1] else \
        np.zeros(1, dtype=np.uint8)
    res = np.zeros(B, dtype=np.int32)
    km, tm = ctypes.c_float(0), ctypes.c_float(0)
    rc = lib.prefix_engine_dispatch(raw.ctypes.data_as(u8p), off.ctypes.data_as(ip), res.ctypes.data_as(ip),
                                    B, int(off[-1]), ctypes.byref(km), ctypes.byref(tm))
    assert rc == 0
    assert tm.value >= km.value >= 0.0
    return [bool(r) for r in res]


@pytest.mark.parametrize("pattern", ["(a|b)*abb", "(a|b)*a(a|b)", "a(b|c)*d"])
def test_reference_bridge_call_sequence(cuda, pattern):
    from trex_b200.build import build
    from trex_b200.regex_to_dfa import compile_regex
    from trex_b200.simulation import DFAMatrices, precompute_tmap
    build()
    path = REPO / "build" / "libprefix_compose.so"
    assert path.exists()
    lib = ctypes.CDLL(str(path))
    u8p, ip = _declare(lib)
    assert lib.prefix_engine_device_check() == 0
    dfa = compile_regex(pattern)
    dm = DFAMatrices(dfa)
    tmap = np.ascontiguousarray(precompute_tmap(dm))
    accept = np.zeros(dm.n_states, dtype=np.uint8)
    for s in dfa.accept_states:
        accept[s] = 1
    assert lib.prefix_engine_init(tmap.ctypes.data_as(u8p), accept.ctypes.data_as(u8p), dfa.start,
                                  dm.n_states, 32, 1 << 22, 1 << 18) == 0
    rng = random.Random(len(pattern))
    # symbols of the automaton only: outside its alphabet the byte map is the identity
    # while DFA.simulate rejects (both are the reference's semantics)
    alphabet = sorted(dfa.alphabet)
    fixed = [s for s in ("", "abb", "aabb", "ab", "abd", "bbbabb", "acbd") if set(s) <= set(alphabet)]
    for n in (300, 17):   # two dispatches on one engine, as the bridge does
        strings = ["".join(rng.choice(alphabet) for _ in range(rng.randint(0, 300))) for _ in range(n)]
        strings += fixed
        got = _dispatch(lib, strings, u8p, ip)
        assert got == [dfa.simulate(s) for s in strings]
    lib.prefix_engine_destroy()
