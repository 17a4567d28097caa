"""Family (d) on the GPU: probabilistic NFA log-likelihoods vs the FP64 oracle.

The oracle (oracle/oracle.c oracle_pnfa_fp64) restates s' = T[c] s of the
reference's nfa_prob_v5_tc_kernel (cuda/nfa_tc_evolution.cu:506-559) in FP64
with exact power-of-two scaling. Parity for the log-likelihood is unpinned by
the reference (it has no CPU path and reports only dot > 0.5).

Tolerances. The 16-bit forms round T and the state to the operand type once
per step, so a string of k symbols can be off by about k unit roundoffs in
log-likelihood when k is small; over long strings the errors average out and
the relative error is what is bounded:
  any string:            |LL - LL_fp64| <= max(rtol * |LL_fp64|, u * (k + 1))
  strings of 2048 symbols (the benchmark shape): |LL - LL_fp64| <= 1e-4 * |LL_fp64|
with rtol = 1e-5 / 1e-4 / 1e-4 and u = 1e-7 / 2^-8 / 2^-11 for fp32 / bf16 /
fp16 (u is twice the operand type's unit roundoff).
"""

import numpy as np
import pytest

from trex_b200.workloads import random_prob_nfa

pytestmark = pytest.mark.gpu

RTOL = {"fp32": 1e-5, "bf16": 1e-4, "fp16": 1e-4, "bf16cc": 1e-4, "fp16cc": 1e-4}
U = {"fp32": 1e-7, "bf16": 2.0 ** -8, "fp16": 2.0 ** -11, "bf16cc": 2.0 ** -8, "fp16cc": 2.0 ** -11}


def _run(torch, T, start, acc, data, off, mode):
    from trex_b200.engine import PNFA
    m = PNFA(T, start, acc)
    d = torch.from_numpy(np.ascontiguousarray(data if data.size else np.zeros(16, np.uint8))).cuda()
    ll, ac = m.run(d, torch.from_numpy(off.astype(np.int64)).cuda(), mode)
    torch.cuda.synchronize()
    err = m.error_word()
    m.close()
    return ll.cpu().numpy(), ac.cpu().numpy(), err


def _symbols(data, off, sigma):
    valid = np.concatenate([[0], np.cumsum(data < sigma)])
    return valid[off[1:]] - valid[off[:-1]]


def _check(ll, ac, ref, mode, k, rtol=None):
    both_inf = np.isneginf(ll) & np.isneginf(ref)
    d = np.abs(ll - ref)
    d[both_inf] = 0.0
    assert np.all(np.isfinite(d)), f"{mode}: non-finite result where the oracle has {ref[~np.isfinite(d)][:4]}"
    if rtol is not None:   # long strings: the relative bound alone
        tol = np.maximum(rtol * np.abs(ref), 1e-12)
    else:
        tol = np.maximum(RTOL[mode] * np.abs(ref), U[mode] * (k + 1))
    worst = np.argmax(d / tol)
    assert np.all(d <= tol), (f"{mode}: |dLL| {d[worst]:.3g} > tol {tol[worst]:.3g} at LL {ref[worst]:.4g} "
                              f"({k[worst]} symbols)")
    # accept flag = dot > 0.5 = LL > log 0.5, where the margin exceeds the tolerance
    clear = np.abs(ref - np.log(0.5)) > 4 * tol
    assert np.array_equal(ac[clear].astype(bool), (ref > np.log(0.5))[clear])


@pytest.mark.parametrize("mode", ["fp32", "bf16", "fp16", "bf16cc", "fp16cc"])
def test_pnfa_ragged_matches_fp64(cuda, oracle, mode):
    rng = np.random.default_rng(7)
    T, start, acc = random_prob_nfa(rng, 64, 20)
    lens = rng.integers(0, 700, size=3000)
    lens[:6] = [0, 1, 2, 15, 16, 17]
    off = np.zeros(len(lens) + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    data = rng.integers(0, 20, size=int(off[-1]), dtype=np.uint8)
    ll, ac, err = _run(cuda, T, start, acc, data, off, mode)
    ref = oracle.pnfa_fp64(T, start, acc, data, off)
    assert err == 0
    _check(ll, ac, ref, mode, _symbols(data, off, 20))


@pytest.mark.parametrize("mode", ["fp32", "bf16", "fp16", "bf16cc", "fp16cc"])
def test_pnfa_small_automaton_skips_unknown_bytes(cuda, oracle, mode):
    # 5 states, 7 symbols (odd: the last symbol pair is half empty), bytes >= 7 skipped
    rng = np.random.default_rng(11)
    T, start, acc = random_prob_nfa(rng, 5, 7, keep=0.6)
    start = rng.random(5)
    acc = (rng.random(5) < 0.5).astype(np.float64)
    acc[0] = 1.0
    lens = rng.integers(0, 300, size=900)
    off = np.zeros(len(lens) + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    data = rng.integers(0, 10, size=int(off[-1]), dtype=np.uint8)
    data[off[7]:off[8]] = 200   # a string with no valid symbol: the start vector's likelihood
    ll, ac, err = _run(cuda, T, start, acc, data, off, mode)
    ref = oracle.pnfa_fp64(T, start, acc, data, off)
    assert err == 0
    _check(ll, ac, ref, mode, _symbols(data, off, 7))


@pytest.mark.parametrize("mode", ["bf16", "fp16"])
def test_pnfa_many_strings_multiple_waves(cuda, oracle, mode):
    # more strings than slots: slots take new strings at block boundaries
    rng = np.random.default_rng(5)
    T, start, acc = random_prob_nfa(rng, 64, 20)
    n = 160_000
    lens = rng.integers(1, 40, size=n)
    off = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    data = rng.integers(0, 20, size=int(off[-1]), dtype=np.uint8)
    ll, ac, err = _run(cuda, T, start, acc, data, off, mode)
    ref = oracle.pnfa_fp64(T, start, acc, data, off)
    assert err == 0
    _check(ll, ac, ref, mode, _symbols(data, off, 20))


def test_pnfa_long_uniform_strings_error(cuda, oracle):
    # the benchmark shape (length 2048), on a subset of strings
    rng = np.random.default_rng(3)
    T, start, acc = random_prob_nfa(rng, 64, 20)
    n, L = 4096, 2048
    off = np.arange(n + 1, dtype=np.int64) * L
    data = rng.integers(0, 20, size=n * L, dtype=np.uint8)
    ref = oracle.pnfa_fp64(T, start, acc, data, off)
    for mode in ("bf16", "fp16", "fp32", "bf16cc", "fp16cc"):
        ll, ac, err = _run(cuda, T, start, acc, data, off, mode)
        assert err == 0
        _check(ll, ac, ref, mode, _symbols(data, off, 20), rtol=RTOL[mode])


def test_pnfa_reference_stochastic_matrices(cuda, oracle):
    # the reference test's construction (nfa_tc_evolution.cu:1320-1345): sigma = 2,
    # T[dst][src] positive and normalised over dst for every src; start e0, accept ~1/4
    rng = np.random.default_rng(77)
    T = rng.integers(1, 101, size=(2, 64, 64)).astype(np.float64)
    T /= T.sum(axis=1, keepdims=True)
    start = np.zeros(64)
    start[0] = 1.0
    acc = (rng.integers(0, 4, size=64) == 0).astype(np.float64)
    lens = rng.integers(1, 300, size=500)
    off = np.zeros(len(lens) + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    data = rng.integers(0, 2, size=int(off[-1]), dtype=np.uint8)
    ref = oracle.pnfa_fp64(T, start, acc, data, off)
    for mode in ("fp32", "bf16", "fp16", "bf16cc", "fp16cc"):
        ll, ac, err = _run(cuda, T, start, acc, data, off, mode)
        assert err == 0
        _check(ll, ac, ref, mode, _symbols(data, off, 2))


def test_pnfa_malformed_offsets_flagged(cuda):
    rng = np.random.default_rng(1)
    T, start, acc = random_prob_nfa(rng, 64, 20)
    off = np.array([0, 10, 5, 20], dtype=np.int64)   # string 1 ends before it starts
    data = rng.integers(0, 20, size=20, dtype=np.uint8)
    for mode in ("fp32", "bf16"):
        _, _, err = _run(cuda, T, start, acc, data, off, mode)
        assert err & 1


@pytest.mark.parametrize("mode", ["bool", "bool8"])
@pytest.mark.parametrize("density", [0.02, 0.05, 0.12])
def test_bool_mode_matches_boolean_nfa_oracle(cuda, oracle, density, mode):
    # Boolean NFA on the tensor cores (0/1 BF16 operands with FP32 sums, or 0/1 int8
    # operands with int32 sums): thresholded products, bit-exact accept flags against
    # the bit-parallel oracle with bytes >= sigma skipped
    from trex_b200.workloads import random_bool_nfa
    rng = np.random.default_rng(int(density * 1000))
    T, start, acc = random_bool_nfa(rng, 64, 20, density=density)
    T = T.astype(np.float32) * rng.uniform(0.1, 3.0, size=T.shape).astype(np.float32)  # any nonzero = edge
    lens = rng.integers(0, 400, size=4000)
    lens[:4] = [0, 1, 2, 3]
    off = np.zeros(len(lens) + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    data = rng.integers(0, 23, size=int(off[-1]), dtype=np.uint8)   # 20..22 skipped
    ll, ac, err = _run(cuda, T, start.astype(np.float32), acc.astype(np.float32), data, off, mode)
    rfm, ref = oracle.nfa_bool(T != 0, start, acc, data, off, unknown_rejects=False)
    assert err == 0
    assert np.array_equal(ac.astype(bool), ref.astype(bool)), np.flatnonzero(ac.astype(bool) != ref.astype(bool))[:8]
    # loglik = log(number of active accepting states): exact for the Boolean forms
    accmask = np.uint64(sum(1 << int(i) for i in np.flatnonzero(acc)))
    n_act = np.array([bin(int(m)).count("1") for m in (rfm & accmask)], dtype=np.float64)
    want = np.where(n_act > 0, np.log(np.maximum(n_act, 1)), -np.inf)
    assert np.array_equal(np.isfinite(ll), np.isfinite(want))
    fin = np.isfinite(want)
    assert np.allclose(ll[fin], want[fin], rtol=0, atol=1e-6)


@pytest.mark.parametrize("mode", ["bool", "bool8"])
def test_bool_mode_small_nfa_both_outcomes(cuda, oracle, mode):
    # 9 states, 5 symbols: strings both accepted and rejected
    rng = np.random.default_rng(9)
    T = (rng.random((5, 9, 9)) < 0.25).astype(np.float32)
    start = np.zeros(9, np.float32)
    start[0] = 1
    acc = np.zeros(9, np.float32)
    acc[[3, 7]] = 1
    lens = rng.integers(0, 60, size=3000)
    off = np.zeros(len(lens) + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    data = rng.integers(0, 5, size=int(off[-1]), dtype=np.uint8)
    _, ac, err = _run(cuda, T, start, acc, data, off, mode)
    _, ref = oracle.nfa_bool(T != 0, start, acc, data, off, unknown_rejects=False)
    assert err == 0
    assert 0 < ref.sum() < len(ref)
    assert np.array_equal(ac.astype(bool), ref.astype(bool))


@pytest.mark.parametrize("sigma", [1, 2, 3, 4])
@pytest.mark.parametrize("mode", ["bf16", "fp16"])
def test_pnfa_lane_kernel_small_alphabet(cuda, oracle, sigma, mode):
    # alphabets of at most four symbols run one string a TMEM lane (no sorting by symbol):
    # ragged and empty strings, bytes >= sigma skipped, more strings than the launch has
    # lanes (148 x 512 for two symbols; fewer tiles for three and four), so lanes take
    # several strings one after another
    rng = np.random.default_rng(20 + sigma)
    T, start, acc = random_prob_nfa(rng, 64, sigma)
    n = 100_000
    lens = rng.integers(0, 20, size=n)
    lens[:6] = [0, 1, 2, 3, 64, 0]
    off = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    data = rng.integers(0, sigma + 2, size=int(off[-1]), dtype=np.uint8)
    ll, ac, err = _run(cuda, T, start, acc, data, off, mode)
    ref = oracle.pnfa_fp64(T, start, acc, data, off)
    assert err == 0
    _check(ll, ac, ref, mode, _symbols(data, off, sigma))


@pytest.mark.parametrize("mode", ["bf16", "fp16"])
def test_pnfa_lane_kernel_long_and_few(cuda, oracle, mode):
    # the lane kernel on long strings (the reference's shape, 2048 symbols, sigma 2) and on a
    # batch of three strings (one CTA, most lanes idle from the start)
    rng = np.random.default_rng(31)
    T, start, acc = random_prob_nfa(rng, 64, 2)
    for n, L in ((1024, 2048), (3, 500)):
        off = np.arange(n + 1, dtype=np.int64) * L
        data = rng.integers(0, 2, size=n * L, dtype=np.uint8)
        ll, ac, err = _run(cuda, T, start, acc, data, off, mode)
        ref = oracle.pnfa_fp64(T, start, acc, data, off)
        assert err == 0
        _check(ll, ac, ref, mode, _symbols(data, off, 2), rtol=RTOL[mode] if L == 2048 else None)


@pytest.mark.parametrize("sigma", [1, 2, 3, 4])
@pytest.mark.parametrize("mode", ["bool", "bool8"])
def test_bool_lane_kernel_small_alphabet(cuda, oracle, sigma, mode):
    # Boolean NFA with one to four symbols on the lane kernel: bit-exact accept flags and
    # log(number of active accepting states) against the bit-parallel oracle
    from trex_b200.workloads import random_bool_nfa
    rng = np.random.default_rng(40 + sigma)
    T, start, acc = random_bool_nfa(rng, 64, sigma, density=0.05)
    T = T.astype(np.float32)
    n = 90_000
    lens = rng.integers(0, 24, size=n)
    lens[:4] = [0, 1, 2, 3]
    off = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    data = rng.integers(0, sigma + 1, size=int(off[-1]), dtype=np.uint8)   # byte sigma skipped
    ll, ac, err = _run(cuda, T, start.astype(np.float32), acc.astype(np.float32), data, off, mode)
    rfm, ref = oracle.nfa_bool(T != 0, start, acc, data, off, unknown_rejects=False)
    assert err == 0
    assert np.array_equal(ac.astype(bool), ref.astype(bool)), np.flatnonzero(ac.astype(bool) != ref.astype(bool))[:8]
    accmask = np.uint64(sum(1 << int(i) for i in np.flatnonzero(acc)))
    n_act = np.array([bin(int(m)).count("1") for m in (rfm & accmask)], dtype=np.float64)
    want = np.where(n_act > 0, np.log(np.maximum(n_act, 1)), -np.inf)
    assert np.array_equal(np.isfinite(ll), np.isfinite(want))
    fin = np.isfinite(want)
    assert np.allclose(ll[fin], want[fin], rtol=0, atol=1e-6)


@pytest.mark.parametrize("sigma,mode", [(20, "bf16"), (20, "bf16cc"), (20, "fp32"), (20, "bool8"),
                                        (2, "bf16"), (2, "bool")])
def test_sm_limit_keeps_results(cuda, sigma, mode):
    """A handle sized for one or a few SMs (serving beside other work) gives the
    same results as one sized for the whole GPU: the kernels take strings from a
    work queue, so only the number of CTAs changes."""
    torch = cuda
    from trex_b200.engine import PNFA
    rng = np.random.default_rng(41)
    T, start, acc = random_prob_nfa(rng, 64, sigma)
    n = 700
    lens = rng.integers(0, 600, size=n)
    off = np.zeros(n + 1, dtype=np.int64)
    off[1:] = np.cumsum(lens)
    data = rng.integers(0, sigma, size=int(off[-1]), dtype=np.uint8)
    d, o = torch.from_numpy(data).cuda(), torch.from_numpy(off).cuda()
    m = PNFA(T, start, acc)
    ll0, ac0 = (x.cpu().numpy() for x in m.run(d, o, mode))
    for lim in (1, 3):
        m.set_sm_limit(lim)
        ll, ac = (x.cpu().numpy() for x in m.run(d, o, mode))
        assert m.error_word() == 0
        assert np.array_equal(ll, ll0) and np.array_equal(ac, ac0)
    m.set_sm_limit(0)
    m.close()
