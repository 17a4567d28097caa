"""Family (c) on the GPU: bit-parallel Boolean NFA vs the C oracle (pinned to
the reference's simulate_nfa by tests/test_oracle_golden.py), the reference
C ABI nfa_tc_engine_* and the NFA bridge."""

import ctypes

import numpy as np
import pytest

from trex_b200.workloads import random_bool_nfa

pytestmark = pytest.mark.gpu


def _run(torch, T, start, acc, data, off, unknown_rejects):
    from trex_b200.engine import NFA
    nfa = NFA(T, start, acc, unknown_rejects=unknown_rejects)
    d = torch.from_numpy(np.ascontiguousarray(data if data.size else np.zeros(1, np.uint8))).cuda()
    fm, ac = nfa.run(d[:data.size], torch.from_numpy(off.astype(np.int64)).cuda())
    torch.cuda.synchronize()
    err = nfa.error_word()
    nfa.close()
    return fm.cpu().numpy().view(np.uint64), ac.cpu().numpy(), err


@pytest.mark.parametrize("N,sigma,density", [(64, 20, 0.05), (64, 2, 0.04), (33, 5, 0.1),
                                             (10, 3, 0.2), (64, 40, 0.05), (64, 70, 0.03),
                                             (64, 200, 0.02), (1, 1, 1.0)])
@pytest.mark.parametrize("unknown_rejects", [True, False])
def test_nfa_matches_oracle(cuda, oracle, N, sigma, density, unknown_rejects):
    rng = np.random.default_rng(N * 1000 + sigma)
    T, start, acc = random_bool_nfa(rng, n_states=N, sigma=sigma, density=density)
    lens = rng.integers(0, 600, size=400)
    lens[:5] = [0, 1, 2, 15, 16]
    off = np.zeros(len(lens) + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    hi = min(256, sigma + 2)   # a few bytes outside the alphabet
    data = rng.integers(0, hi, size=int(off[-1]), dtype=np.uint8)
    fm, ac, err = _run(cuda, T, start, acc, data, off, unknown_rejects)
    rfm, rac = oracle.nfa_bool(T, start, acc, data, off, unknown_rejects=unknown_rejects)
    assert err == 0
    assert np.array_equal(fm, rfm)
    assert np.array_equal(ac, rac)


def test_nfa_golden(cuda, golden):
    for rec in golden["nfa"]:
        N, sigma = rec["n_states"], rec["sigma"]
        T = np.stack([np.unpackbits(np.frombuffer(bytes.fromhex(h), dtype=np.uint8))[:N * N]
                      .reshape(N, N) for h in rec["T_dst_src_hex"]])
        strs = [bytes.fromhex(h) for h in rec["strings_hex"]]
        data = np.frombuffer(b"".join(strs), dtype=np.uint8).copy()
        off = np.zeros(len(strs) + 1, dtype=np.int64)
        np.cumsum([len(s) for s in strs], out=off[1:])
        fm, ac, err = _run(cuda, T, rec["start"], rec["accept"], data, off, True)
        assert err == 0
        assert [bool(a) for a in ac] == rec["nfa_accept"]
        assert [format(int(m), "x") for m in fm] == rec["final_mask_hex"]


def test_reference_abi_three_a(cuda):
    # reference cuda/nfa_tc_evolution.cu:1056-1137 (">= 3 a's", a = 0, b = 1)
    from trex_b200 import _lib
    L = _lib.load()
    N = 64
    T = np.zeros((2, N, N), dtype=np.float32)
    for i in range(3):
        T[0, i, i] = 1
        T[0, i + 1, i] = 1
    T[0, 3, 3] = 1
    for i in range(4):
        T[1, i, i] = 1
    for s in range(4, N):
        T[0, s, s] = T[1, s, s] = 1
    start = np.zeros(N, np.float32); start[0] = 1
    acc = np.zeros(N, np.float32); acc[3] = 1
    f32 = ctypes.c_float
    assert L.nfa_tc_engine_init(_lib.ptr(T, f32), _lib.ptr(acc, f32), _lib.ptr(start, f32),
                                N, 2, 64, 256) == 0
    chars = np.array([0, 0, 0, 0, 0, 0, 1, 1, 0, 1, 0, 0, 0, 1, 1, 0, 0, 0, 0, 1, 0, 1, 0, 0, 1,
                      0, 0], dtype=np.uint8)
    off = np.array([0, 0, 1, 3, 6, 7, 10, 14, 18, 22, 27], dtype=np.int32)
    res = np.zeros(10, dtype=np.int32)
    km, tm = ctypes.c_float(), ctypes.c_float()
    rc = L.nfa_tc_engine_dispatch(_lib.ptr(chars, ctypes.c_uint8), _lib.ptr(off, ctypes.c_int),
                                  _lib.ptr(res, ctypes.c_int), 10, 27, ctypes.byref(km),
                                  ctypes.byref(tm))
    L.nfa_tc_engine_destroy()
    assert rc == 0
    assert res.tolist() == [0, 0, 0, 1, 0, 0, 1, 1, 0, 1]


def test_nfa_bridge_regexes(cuda):
    from trex_b200.gpu_bridge_nfa import NFAGPUSimulator
    from trex_b200.nfa_matrices import compile_nfa_matrices, simulate_nfa
    rng = np.random.default_rng(3)
    sim = NFAGPUSimulator()
    for pat in ["(a|b)*abb", "(ab)*", "a(b|c)*d", "(b*ab*ab*)*b*", "[a-c]*abc", "x?y+z*"]:
        nm = compile_nfa_matrices(pat)
        eng = sim.create_engine(nm)
        alpha = sorted(nm.alphabet) + ["q"]
        strs = ["".join(rng.choice(alpha, size=rng.integers(0, 30))) for _ in range(300)] + [""]
        assert eng.simulate_batch(strs) == [simulate_nfa(nm, s) for s in strs], pat
        eng.destroy()


def test_nfa_run_multi_matches_oracle(cuda, oracle):
    """trex_nfa_run_multi over automata of four table layouts (sigma 2, 20, 100 in
    shared memory, 255 in global memory), an empty group and a group of one string:
    every string's mask and accept flag equals its automaton's oracle result; a
    string that ends past the data is flagged in the error word and the rest still
    run."""
    torch = cuda
    from trex_b200.engine import NFA, nfa_run_multi
    rng = np.random.default_rng(77)
    sigmas = [20, 2, 100, 255, 20, 2, 20]
    counts = [300, 50, 80, 40, 0, 1, 700]
    autos = [random_bool_nfa(rng, n_states=64, sigma=s, density=0.05) for s in sigmas]
    nfas = [NFA(*a, unknown_rejects=True) for a in autos]
    lens = [rng.integers(0, 900, size=c) for c in counts]
    datas = [[rng.integers(0, min(256, s + 2), size=int(L), dtype=np.uint8) for L in ls]
             for s, ls in zip(sigmas, lens)]
    flat = [x for ds in datas for x in ds]
    off = np.zeros(len(flat) + 1, dtype=np.int64)
    off[1:] = np.cumsum([len(x) for x in flat])
    data = np.concatenate(flat)
    gf = np.concatenate(([0], np.cumsum(counts)))
    d = torch.from_numpy(data).cuda()
    for bad in (False, True):
        o = off.copy()
        if bad:   # the last string ends past the data
            o[-1] += 5
        n = len(flat)
        fm = torch.zeros(n, dtype=torch.int64, device="cuda")
        ac = torch.full((n,), 7, dtype=torch.uint8, device="cuda")
        scr = torch.zeros(8 * (len(nfas) + 1), dtype=torch.uint8, device="cuda")
        nfa_run_multi(nfas, gf, d, torch.from_numpy(o).cuda(), final_mask=fm, accept=ac, scratch=scr)
        fm = fm.cpu().numpy().view(np.uint64)
        ac = ac.cpu().numpy()
        err = int(scr[8 * len(nfas):8 * len(nfas) + 4].view(torch.int32).item())
        assert bool(err & 1) == bad
        for g, (a, ds) in enumerate(zip(autos, datas)):
            if not ds:
                continue
            so = np.zeros(len(ds) + 1, dtype=np.int64)
            so[1:] = np.cumsum([len(x) for x in ds])
            rfm, rac = oracle.nfa_bool(*a, np.concatenate(ds), so, unknown_rejects=True)
            sel = np.arange(gf[g], gf[g + 1])
            if bad and g == len(autos) - 1:
                assert ac[n - 1] == 7   # the malformed string gets no result
                sel, rfm, rac = sel[:-1], rfm[:-1], rac[:-1]
            assert np.array_equal(fm[sel], rfm) and np.array_equal(ac[sel], rac)
    for m in nfas:
        m.close()
