// Family (a): ragged batch DFA simulation over raw bytes, many resident DFAs,
// one persistent launch.
//
// Semantics (reference src/simulation.py:274-297 precompute_tmap and
// cuda/prefix_compose.cu:217-258 prefix_fused_kernel): every string walks
//     s = tmap[byte * N + s]
// from the DFA's start state; outputs are the final state and accept[s].
//
// Design
//  * Planning (3 small kernels): every string is cut into work items of at
//    most seg_len bytes; items are bucketed by DFA so one CTA serves one DFA
//    at a time. Item k of a string covers bytes [k*seg_len, (k+1)*seg_len).
//  * Main kernel: one persistent 1024-thread CTA per SM. The CTA expands the
//    current DFA's 4 KiB byte map into a per-lane replicated table in shared
//    memory so that the 32 lanes of a warp always hit 32 different banks:
//      N <= 8 : byte address = c<<8 | (s>>2)<<7 | lane<<2 | (s&3)   (64 KiB)
//               the stored byte IS the next address minus c<<8, so one step
//               is PRMT (merge state byte with input byte c) + LDS.U8;
//      N <= 16: byte address = c<<9 | (s>>2)<<7 | lane<<2 | (s&3)   (128 KiB)
//               the stored byte is (s&3) | (s>>2)<<6 and one step is
//               PRMT + LOP3 + IADD3 + LDS.U8;
//      N <= 256: the plain 256*N table (bank conflicts, no string splitting).
//  * Each thread walks one item. The first item of a string starts from the
//    DFA start state. Later items compute the item's state map: all N start
//    states walk together until they coincide (random DFAs synchronise within
//    a few dozen bytes), then a single chain finishes the item. A per-string
//    counter lets the last item to finish compose the maps in order
//    (no spin-waits).
//  * Input is streamed with 16-byte non-coherent loads (L2 256-byte
//    prefetch), one load ahead of the dependent chain.
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "trex_internal.cuh"

namespace trex {

struct DfaDesc {
    int32_t n_states;
    int32_t start;
    int64_t tmap_off;
    int64_t accept_off;
};

struct WorkItem {
    uint32_t str;
    uint32_t seg;
};

// Error bits reported through the device error word.
enum : uint32_t {
    kErrBadOffsets = 1u,
    kErrBadDfaId = 2u,
};

constexpr int kRaggedThreads = 1024;
constexpr int kPlanThreads = 256;
constexpr int kDefaultSegLen = 8192;

// ---- scratch layout -----------------------------------------------------------
struct ScratchLayout {
    size_t q_count, q_base, q_head, q_cursor, q_bytes, err, items, maps, done, total;
    int64_t max_items;
};

static ScratchLayout scratch_layout(int64_t n_strings, int64_t total_bytes, int32_t seg_len) {
    ScratchLayout L{};
    if (seg_len <= 0) seg_len = kDefaultSegLen;
    L.max_items = n_strings + total_bytes / seg_len + 1;
    size_t o = 0;
    auto take = [&](size_t bytes) { size_t at = o; o = (o + bytes + 255) & ~size_t(255); return at; };
    L.q_count = take(kMaxDfasPerSet * 4);
    L.q_base = take(kMaxDfasPerSet * 4);
    L.q_head = take(kMaxDfasPerSet * 4);
    L.q_cursor = take(kMaxDfasPerSet * 4);
    L.q_bytes = take(kMaxDfasPerSet * 8);
    L.err = take(4);
    L.items = take((size_t)L.max_items * sizeof(WorkItem));
    L.maps = take((size_t)L.max_items * sizeof(uint64_t));
    L.done = take((size_t)std::max<int64_t>(n_strings, 1) * 4);
    L.total = o;
    return L;
}

// ---- planning kernels -------------------------------------------------------------
__device__ __forceinline__ uint32_t n_items_of(int64_t len, int n_states, int32_t seg_len) {
    if (len <= 0 || n_states > kSmallDfaStates) return 1;
    return (uint32_t)((len + seg_len - 1) / seg_len);
}

// Returns the DFA index of string i, or -1 (and raises an error bit) when the
// string is malformed; malformed strings get no work items.
__device__ __forceinline__ int checked_dfa(const int64_t *offsets, const int32_t *dfa_id,
                                           int64_t i, int n_dfas, int64_t total_bytes,
                                           uint32_t *err, int64_t *len_out) {
    int64_t a = offsets[i], b = offsets[i + 1];
    int d = dfa_id ? dfa_id[i] : 0;
    if (a < 0 || b < a || b > total_bytes) {
        atomicOr(err, kErrBadOffsets);
        return -1;
    }
    if (d < 0 || d >= n_dfas) {
        atomicOr(err, kErrBadDfaId);
        return -1;
    }
    *len_out = b - a;
    return d;
}

__global__ void plan_count_kernel(const int64_t *offsets, const int32_t *dfa_id, int64_t n,
                                  int64_t total_bytes, const DfaDesc *desc, int n_dfas,
                                  int32_t seg_len, uint32_t *q_count,
                                  unsigned long long *q_bytes, uint32_t *err) {
    __shared__ uint32_t cnt[kMaxDfasPerSet];
    __shared__ unsigned long long byt[kMaxDfasPerSet];
    for (int t = threadIdx.x; t < n_dfas; t += blockDim.x) { cnt[t] = 0; byt[t] = 0; }
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        int64_t len;
        int d = checked_dfa(offsets, dfa_id, i, n_dfas, total_bytes, err, &len);
        if (d < 0) continue;
        atomicAdd(&cnt[d], n_items_of(len, desc[d].n_states, seg_len));
        atomicAdd(&byt[d], (unsigned long long)len + 64ull);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < n_dfas; t += blockDim.x) {
        if (cnt[t]) atomicAdd(&q_count[t], cnt[t]);
        if (byt[t]) atomicAdd(&q_bytes[t], byt[t]);
    }
}

__global__ void plan_scan_kernel(const uint32_t *q_count, uint32_t *q_base, uint32_t *q_cursor,
                                 int n_dfas) {
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (int d = 0; d < n_dfas; ++d) {
            q_base[d] = run;
            q_cursor[d] = run;
            run += q_count[d];
        }
    }
}

__global__ void plan_fill_kernel(const int64_t *offsets, const int32_t *dfa_id, int64_t n,
                                 int64_t total_bytes, const DfaDesc *desc, int n_dfas,
                                 int32_t seg_len, uint32_t *q_cursor, WorkItem *items,
                                 uint32_t *done, uint32_t *err) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        done[i] = 0;
        int64_t len;
        int d = checked_dfa(offsets, dfa_id, i, n_dfas, total_bytes, err, &len);
        if (d < 0) continue;
        uint32_t k = n_items_of(len, desc[d].n_states, seg_len);
        uint32_t pos = atomicAdd(&q_cursor[d], k);
        for (uint32_t j = 0; j < k; ++j) items[pos + j] = WorkItem{(uint32_t)i, j};
    }
}

// ---- replicated-table walkers ------------------------------------------------------
// LAYOUT 8: N <= 8, LAYOUT 16: N <= 16, LAYOUT 0: plain table (N <= 256).
template <int LAYOUT> struct Walker;

template <> struct Walker<8> {
    static constexpr int kChains = 8;
    uint32_t lane;
    __device__ uint32_t enc(uint32_t s) const { return (s & 3u) | (lane << 2) | ((s >> 2) << 7); }
    __device__ static uint32_t dec(uint32_t e) { return (e & 3u) | ((e >> 7) << 2); }
    template <int I>
    __device__ __forceinline__ uint32_t step(const uint8_t *tbl, uint32_t e, uint32_t x) const {
        uint32_t a = __byte_perm(e, x, 0x1100 | ((4 + I) << 4));
        return tbl[a];
    }
};

template <> struct Walker<16> {
    static constexpr int kChains = 16;
    uint32_t lane;
    __device__ uint32_t enc(uint32_t s) const { return (s & 3u) | ((s >> 2) << 6); }
    __device__ static uint32_t dec(uint32_t e) { return (e & 3u) | ((e >> 6) << 2); }
    template <int I>
    __device__ __forceinline__ uint32_t step(const uint8_t *tbl, uint32_t e, uint32_t x) const {
        uint32_t t = __byte_perm(e, x, 0x1100 | ((4 + I) << 4));
        uint32_t a = t + (t & 0xFFC0u) + (lane << 2);
        return tbl[a];
    }
};

template <> struct Walker<0> {
    static constexpr int kChains = 0;
    uint32_t n;
    __device__ uint32_t enc(uint32_t s) const { return s; }
    __device__ static uint32_t dec(uint32_t e) { return e; }
    template <int I>
    __device__ __forceinline__ uint32_t step(const uint8_t *tbl, uint32_t e, uint32_t x) const {
        uint32_t c = (x >> (8 * I)) & 0xFFu;
        return tbl[c * n + e];
    }
};

template <class W>
__device__ __forceinline__ uint32_t step_word(const W &w, const uint8_t *tbl, uint32_t e,
                                              uint32_t x) {
    e = w.template step<0>(tbl, e, x);
    e = w.template step<1>(tbl, e, x);
    e = w.template step<2>(tbl, e, x);
    e = w.template step<3>(tbl, e, x);
    return e;
}

template <class W>
__device__ __forceinline__ uint32_t step16(const W &w, const uint8_t *tbl, uint32_t e, uint4 v) {
    e = step_word(w, tbl, e, v.x);
    e = step_word(w, tbl, e, v.y);
    e = step_word(w, tbl, e, v.z);
    e = step_word(w, tbl, e, v.w);
    return e;
}

// Walks bytes [p, end) from encoded state e.
template <class W>
__device__ uint32_t walk_chain(const W &w, const uint8_t *tbl, const uint8_t *__restrict__ data,
                               int64_t p, int64_t end, uint32_t e) {
    while (p < end && (p & 15)) {
        e = w.template step<0>(tbl, e, (uint32_t)__ldg(data + p));
        ++p;
    }
    if (end - p >= 32) {
        uint4 a = ld_stream16(data + p);
        uint4 b = ld_stream16(data + p + 16);
        p += 32;
        while (end - p >= 32) {
            uint4 na = ld_stream16(data + p);
            uint4 nb = ld_stream16(data + p + 16);
            e = step16(w, tbl, e, a);
            e = step16(w, tbl, e, b);
            a = na;
            b = nb;
            p += 32;
        }
        e = step16(w, tbl, e, a);
        e = step16(w, tbl, e, b);
    }
    if (end - p >= 16) {
        uint4 a = ld_stream16(data + p);
        e = step16(w, tbl, e, a);
        p += 16;
    }
    while (p < end) {
        e = w.template step<0>(tbl, e, (uint32_t)__ldg(data + p));
        ++p;
    }
    return e;
}

// State map of bytes [p, end) for states 0..n-1 packed as nibbles.
template <class W>
__device__ uint64_t walk_map(const W &w, const uint8_t *tbl, const uint8_t *__restrict__ data,
                             int64_t p, int64_t end, int n) {
    constexpr int C = W::kChains;
    uint32_t e[C];
#pragma unroll
    for (int j = 0; j < C; ++j) e[j] = w.enc(j < n ? (uint32_t)j : 0u);
    bool same = false;
    while (p < end) {
        int64_t stop = p + 8 < end ? p + 8 : end;
        for (; p < stop; ++p) {
            uint32_t c = __ldg(data + p);
#pragma unroll
            for (int j = 0; j < C; ++j) e[j] = w.template step<0>(tbl, e[j], c);
        }
        same = true;
#pragma unroll
        for (int j = 1; j < C; ++j) same &= (e[j] == e[0]);
        if (same) break;
    }
    uint64_t m = 0;
    if (same) {
        uint32_t e0 = walk_chain(w, tbl, data, p, end, e[0]);
        uint64_t s = W::dec(e0);
        m = s * 0x1111111111111111ull;
    } else {
#pragma unroll
        for (int j = 0; j < C; ++j) m |= (uint64_t)W::dec(e[j]) << (4 * j);
    }
    return m;
}

struct RaggedParams {
    const uint8_t *data;
    const int64_t *offsets;
    int64_t n_strings;
    const uint8_t *tmaps;
    const uint8_t *accepts;
    const DfaDesc *desc;
    int n_dfas;
    const WorkItem *items;
    const uint32_t *q_base;
    const uint32_t *q_count;
    uint32_t *q_head;
    const unsigned long long *q_bytes;
    uint64_t *maps;
    uint32_t *done;
    int32_t seg_len;
    uint8_t *final_state;
    uint8_t *accept;
    int32_t *accept_i32;
};

__device__ __forceinline__ void write_result(const RaggedParams &P, uint32_t str, uint32_t s,
                                             int64_t accept_off) {
    uint8_t a = P.accepts[accept_off + s];
    if (P.final_state) P.final_state[str] = (uint8_t)s;
    if (P.accept) P.accept[str] = a;
    if (P.accept_i32) P.accept_i32[str] = a ? 1 : 0;
}

template <class W>
__device__ void process_item(const RaggedParams &P, const W &w, const uint8_t *tbl, WorkItem it,
                             uint32_t item_idx, const DfaDesc &D) {
    int64_t s0 = P.offsets[it.str], s1 = P.offsets[it.str + 1];
    uint32_t nseg = n_items_of(s1 - s0, D.n_states, P.seg_len);
    int64_t b0 = (nseg == 1) ? s0 : s0 + (int64_t)it.seg * P.seg_len;
    int64_t b1 = (nseg == 1) ? s1 : min(s1, b0 + (int64_t)P.seg_len);
    uint64_t map;
    if (it.seg == 0) {
        uint32_t e = walk_chain(w, tbl, P.data, b0, b1, w.enc((uint32_t)D.start));
        uint32_t fs = W::dec(e);
        if (nseg == 1) {
            write_result(P, it.str, fs, D.accept_off);
            return;
        }
        map = (uint64_t)fs * 0x1111111111111111ull;
    } else {
        if constexpr (W::kChains > 0) map = walk_map(w, tbl, P.data, b0, b1, D.n_states);
        else map = 0;  // unreachable: large automata are never split
    }
    P.maps[item_idx] = map;
    __threadfence();
    uint32_t prev = atomicAdd(&P.done[it.str], 1u);
    if (prev == nseg - 1) {
        __threadfence();
        uint32_t base = item_idx - it.seg;
        uint32_t s = (uint32_t)D.start;
        for (uint32_t k = 0; k < nseg; ++k) {
            uint64_t m = ld_relaxed_u64(P.maps + base + k);
            s = (uint32_t)(m >> (4 * s)) & 15u;
        }
        write_result(P, it.str, s, D.accept_off);
    }
}

// Fills the shared-memory table of DFA d for the layout its size selects.
__device__ void build_table(const RaggedParams &P, const DfaDesc &D, uint8_t *tbl) {
    const uint8_t *src = P.tmaps + D.tmap_off;
    const int N = D.n_states;
    uint32_t *w32 = reinterpret_cast<uint32_t *>(tbl);
    if (N <= 8) {
        for (int w = threadIdx.x; w < kRepTableBytes8 / 4; w += blockDim.x) {
            uint32_t c = w >> 6, q = (w >> 5) & 1u, ln = w & 31u, word = 0;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                uint32_t s = q * 4 + b;
                uint32_t t = s < (uint32_t)N ? src[c * N + s] : s;
                word |= ((t & 3u) | (ln << 2) | ((t >> 2) << 7)) << (8 * b);
            }
            w32[w] = word;
        }
    } else if (N <= 16) {
        for (int w = threadIdx.x; w < kRepTableBytes16 / 4; w += blockDim.x) {
            uint32_t c = w >> 7, q = (w >> 5) & 3u, word = 0;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                uint32_t s = q * 4 + b;
                uint32_t t = s < (uint32_t)N ? src[c * N + s] : s;
                word |= ((t & 3u) | ((t >> 2) << 6)) << (8 * b);
            }
            w32[w] = word;
        }
    } else {
        for (int i = threadIdx.x; i < 256 * N; i += blockDim.x) tbl[i] = src[i];
    }
}

__global__ void __launch_bounds__(kRaggedThreads, 1) dfa_ragged_kernel(RaggedParams P) {
    extern __shared__ __align__(1024) uint8_t tbl[];
    __shared__ int s_dfa;
    if (threadIdx.x == 0) {
        // Home DFA: CTAs are spread over DFAs in proportion to their bytes.
        unsigned long long tot = 0;
        for (int d = 0; d < P.n_dfas; ++d) tot += P.q_bytes[d];
        int home = -1;
        if (tot) {
            unsigned long long pos =
                (unsigned long long)((double)tot * ((double)blockIdx.x + 0.5) / gridDim.x);
            unsigned long long run = 0;
            for (int d = 0; d < P.n_dfas; ++d) {
                run += P.q_bytes[d];
                if (P.q_count[d] && pos < run) { home = d; break; }
            }
            if (home < 0)
                for (int d = P.n_dfas - 1; d >= 0; --d)
                    if (P.q_count[d]) { home = d; break; }
        }
        s_dfa = home;
    }
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31u;
    for (int round = 0; round <= P.n_dfas; ++round) {
        const int d = s_dfa;
        if (d < 0) break;
        const DfaDesc D = P.desc[d];
        build_table(P, D, tbl);
        __syncthreads();
        const uint32_t base = P.q_base[d], count = P.q_count[d];
        while (true) {
            uint32_t idx = atomicAdd(&P.q_head[d], 1u);
            if (idx >= count) break;
            WorkItem it = P.items[base + idx];
            if (D.n_states <= 8) {
                Walker<8> w{lane};
                process_item(P, w, tbl, it, base + idx, D);
            } else if (D.n_states <= 16) {
                Walker<16> w{lane};
                process_item(P, w, tbl, it, base + idx, D);
            } else {
                Walker<0> w{(uint32_t)D.n_states};
                process_item(P, w, tbl, it, base + idx, D);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int best = -1;
            uint32_t best_rem = 0;
            for (int e = 0; e < P.n_dfas; ++e) {
                uint32_t h = *(volatile uint32_t *)&P.q_head[e];
                uint32_t c = P.q_count[e];
                uint32_t rem = h < c ? c - h : 0;
                if (rem > best_rem) { best_rem = rem; best = e; }
            }
            s_dfa = best;
        }
        __syncthreads();
    }
}

// ---- host side --------------------------------------------------------------------------

}  // namespace trex

struct trex_dfa_set {
    int n_dfas = 0;
    int max_states = 0;
    std::vector<int32_t> n_states, starts;
    std::vector<int64_t> tmap_off, accept_off;
    std::vector<uint8_t> h_accepts;      // host copy for empty-batch answers
    uint8_t *d_tmaps = nullptr;
    uint8_t *d_accepts = nullptr;
    trex::DfaDesc *d_desc = nullptr;
    void *own_scratch = nullptr;
    size_t own_scratch_bytes = 0;
    int n_sms = 0;
    size_t smem_bytes = 0;
    // Device staging for trex_dfa_batch_host (grown on demand).
    uint8_t *st_data = nullptr;
    int64_t *st_off = nullptr;
    int32_t *st_ids = nullptr;
    uint8_t *st_out = nullptr;     // final_state[n] | accept[n]
    int32_t *st_out32 = nullptr;
    int64_t st_data_cap = 0, st_n_cap = 0;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
};

namespace trex {

int dfa_set_run(trex_dfa_set *set, const uint8_t *data, const int64_t *offsets,
                const int32_t *dfa_id, int64_t n, int64_t total_bytes, uint8_t *final_state,
                uint8_t *accept, int32_t *accept_i32, void *scratch, int64_t scratch_bytes,
                int32_t seg_len, cudaStream_t stream, uint32_t **err_word_out) {
    if (!set) return TREX_ERR_NOT_INIT;
    if (n < 0 || total_bytes < 0 || (n > 0 && !offsets) || (total_bytes > 0 && !data))
        return TREX_ERR_ARG;
    if (n >= (int64_t)0x7fffffff) return TREX_ERR_CAPACITY;
    if (seg_len <= 0) seg_len = kDefaultSegLen;
    if (seg_len < 64) seg_len = 64;
    if (n == 0) return TREX_OK;
    ScratchLayout L = scratch_layout(n, total_bytes, seg_len);
    if (L.max_items >= (int64_t)0xffffffffLL) return TREX_ERR_CAPACITY;
    uint8_t *sc = static_cast<uint8_t *>(scratch);
    if (!sc) {
        if (set->own_scratch_bytes < L.total) {
            if (set->own_scratch) cudaFree(set->own_scratch);
            set->own_scratch = nullptr;
            set->own_scratch_bytes = 0;
            if (cudaMalloc(&set->own_scratch, L.total) != cudaSuccess) {
                cudaGetLastError();
                set_last_error_msg("trex_dfa_batch_run: scratch allocation failed");
                return TREX_ERR_OOM;
            }
            set->own_scratch_bytes = L.total;
        }
        sc = static_cast<uint8_t *>(set->own_scratch);
    } else if ((size_t)scratch_bytes < L.total) {
        return TREX_ERR_ARG;
    }
    uint32_t *q_count = reinterpret_cast<uint32_t *>(sc + L.q_count);
    uint32_t *q_base = reinterpret_cast<uint32_t *>(sc + L.q_base);
    uint32_t *q_head = reinterpret_cast<uint32_t *>(sc + L.q_head);
    uint32_t *q_cursor = reinterpret_cast<uint32_t *>(sc + L.q_cursor);
    auto *q_bytes = reinterpret_cast<unsigned long long *>(sc + L.q_bytes);
    uint32_t *err = reinterpret_cast<uint32_t *>(sc + L.err);
    WorkItem *items = reinterpret_cast<WorkItem *>(sc + L.items);
    uint64_t *maps = reinterpret_cast<uint64_t *>(sc + L.maps);
    uint32_t *done = reinterpret_cast<uint32_t *>(sc + L.done);

    // Counters, bases, heads, cursors, byte counts and the error word are
    // contiguous at the front of the scratch buffer.
    TREX_CUDA(cudaMemsetAsync(sc, 0, L.items, stream));
    int plan_grid = (int)std::min<int64_t>((n + kPlanThreads - 1) / kPlanThreads,
                                           (int64_t)set->n_sms * 8);
    plan_count_kernel<<<plan_grid, kPlanThreads, 0, stream>>>(
        offsets, dfa_id, n, total_bytes, set->d_desc, set->n_dfas, seg_len, q_count, q_bytes, err);
    TREX_CHECK_LAUNCH();
    plan_scan_kernel<<<1, 32, 0, stream>>>(q_count, q_base, q_cursor, set->n_dfas);
    TREX_CHECK_LAUNCH();
    plan_fill_kernel<<<plan_grid, kPlanThreads, 0, stream>>>(
        offsets, dfa_id, n, total_bytes, set->d_desc, set->n_dfas, seg_len, q_cursor, items, done,
        err);
    TREX_CHECK_LAUNCH();

    RaggedParams P;
    P.data = data;
    P.offsets = offsets;
    P.n_strings = n;
    P.tmaps = set->d_tmaps;
    P.accepts = set->d_accepts;
    P.desc = set->d_desc;
    P.n_dfas = set->n_dfas;
    P.items = items;
    P.q_base = q_base;
    P.q_count = q_count;
    P.q_head = q_head;
    P.q_bytes = q_bytes;
    P.maps = maps;
    P.done = done;
    P.seg_len = seg_len;
    P.final_state = final_state;
    P.accept = accept;
    P.accept_i32 = accept_i32;
    profile_kernel_begin(stream);
    dfa_ragged_kernel<<<set->n_sms, kRaggedThreads, set->smem_bytes, stream>>>(P);
    TREX_CHECK_LAUNCH();
    profile_kernel_end(stream);
    if (err_word_out) *err_word_out = err;
    return TREX_OK;
}

}  // namespace trex

extern "C" {

int trex_dfa_set_create(int n_dfas, const int32_t *n_states, const int32_t *starts,
                        const uint8_t *tmaps, const uint8_t *accepts, trex_dfa_set **out) {
    if (!out) return TREX_ERR_ARG;
    *out = nullptr;
    if (n_dfas <= 0 || n_dfas > trex::kMaxDfasPerSet || !n_states || !starts || !tmaps || !accepts)
        return TREX_ERR_ARG;
    trex_dfa_set *set = new (std::nothrow) trex_dfa_set();
    if (!set) return TREX_ERR_OOM;
    set->n_dfas = n_dfas;
    int64_t tsum = 0, asum = 0;
    std::vector<trex::DfaDesc> desc(n_dfas);
    for (int d = 0; d < n_dfas; ++d) {
        int N = n_states[d];
        if (N < 1 || N > trex::kMaxPlainStates || starts[d] < 0 || starts[d] >= N) {
            delete set;
            return TREX_ERR_ARG;
        }
        desc[d] = trex::DfaDesc{N, starts[d], tsum, asum};
        set->n_states.push_back(N);
        set->starts.push_back(starts[d]);
        set->tmap_off.push_back(tsum);
        set->accept_off.push_back(asum);
        set->max_states = std::max(set->max_states, N);
        tsum += 256LL * N;
        asum += N;
    }
    // Every next state must be a valid state: the kernels index tables with it.
    for (int d = 0; d < n_dfas; ++d) {
        const uint8_t *t = tmaps + set->tmap_off[d];
        for (int64_t i = 0; i < 256LL * set->n_states[d]; ++i)
            if (t[i] >= set->n_states[d]) {
                delete set;
                trex::set_last_error_msg("trex_dfa_set_create: next state out of range");
                return TREX_ERR_ARG;
            }
    }
    set->h_accepts.assign(accepts, accepts + asum);
    set->n_sms = trex::sm_count();
    if (set->n_sms <= 0) {
        delete set;
        trex::set_last_error_msg("trex_dfa_set_create: no CUDA device");
        return TREX_ERR_SHAPE;
    }
    set->smem_bytes = 0;
    for (int d = 0; d < n_dfas; ++d) {
        int N = set->n_states[d];
        size_t need = N <= 8 ? trex::kRepTableBytes8
                    : N <= 16 ? trex::kRepTableBytes16 : (size_t)256 * N;
        set->smem_bytes = std::max(set->smem_bytes, need);
    }
    auto fail = [&](cudaError_t e, const char *what) {
        trex::set_last_error(what, e);
        cudaFree(set->d_tmaps);
        cudaFree(set->d_accepts);
        cudaFree(set->d_desc);
        delete set;
        return e == cudaErrorMemoryAllocation ? TREX_ERR_OOM : TREX_ERR_CUDA;
    };
    cudaError_t e;
    if ((e = cudaMalloc(&set->d_tmaps, tsum)) != cudaSuccess) return fail(e, "cudaMalloc tmaps");
    if ((e = cudaMalloc(&set->d_accepts, asum)) != cudaSuccess) return fail(e, "cudaMalloc accepts");
    if ((e = cudaMalloc(&set->d_desc, sizeof(trex::DfaDesc) * n_dfas)) != cudaSuccess)
        return fail(e, "cudaMalloc desc");
    if ((e = cudaMemcpy(set->d_tmaps, tmaps, tsum, cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(e, "copy tmaps");
    if ((e = cudaMemcpy(set->d_accepts, accepts, asum, cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(e, "copy accepts");
    if ((e = cudaMemcpy(set->d_desc, desc.data(), sizeof(trex::DfaDesc) * n_dfas,
                        cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(e, "copy desc");
    // The attribute is per kernel, so it is always raised to the largest
    // table any set can need (128 KiB).
    if ((e = cudaFuncSetAttribute(trex::dfa_ragged_kernel,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  trex::kRepTableBytes16)) != cudaSuccess)
        return fail(e, "cudaFuncSetAttribute");
    *out = set;
    return TREX_OK;
}

void trex_dfa_set_destroy(trex_dfa_set *set) {
    if (!set) return;
    cudaFree(set->d_tmaps);
    cudaFree(set->d_accepts);
    cudaFree(set->d_desc);
    if (set->own_scratch) cudaFree(set->own_scratch);
    cudaFree(set->st_data);
    cudaFree(set->st_off);
    cudaFree(set->st_ids);
    cudaFree(set->st_out);
    cudaFree(set->st_out32);
    for (auto &e : set->ev)
        if (e) cudaEventDestroy(e);
    delete set;
}

int trex_dfa_batch_host(trex_dfa_set *set, const uint8_t *h_data, const int64_t *h_offsets,
                        const int32_t *h_dfa_id, int64_t n, int64_t total_bytes,
                        uint8_t *h_final_state, uint8_t *h_accept, int32_t *h_accept_i32,
                        int32_t seg_len, float *kernel_ms, float *total_ms) {
    if (!set) return TREX_ERR_NOT_INIT;
    if (n < 0 || total_bytes < 0 || (n > 0 && !h_offsets) || (total_bytes > 0 && !h_data))
        return TREX_ERR_ARG;
    if (kernel_ms) *kernel_ms = 0.f;
    if (total_ms) *total_ms = 0.f;
    if (n == 0) return TREX_OK;
    if (h_offsets[0] < 0 || h_offsets[n] > total_bytes) return TREX_ERR_ARG;
    // Grow staging buffers.
    if (set->st_data_cap < total_bytes) {
        cudaFree(set->st_data);
        set->st_data = nullptr;
        set->st_data_cap = 0;
        TREX_CUDA(cudaMalloc(&set->st_data, std::max<int64_t>(total_bytes, 16)));
        set->st_data_cap = total_bytes;
    }
    if (set->st_n_cap < n) {
        cudaFree(set->st_off);
        cudaFree(set->st_ids);
        cudaFree(set->st_out);
        cudaFree(set->st_out32);
        set->st_off = nullptr;
        set->st_ids = nullptr;
        set->st_out = nullptr;
        set->st_out32 = nullptr;
        set->st_n_cap = 0;
        TREX_CUDA(cudaMalloc(&set->st_off, (n + 1) * 8));
        TREX_CUDA(cudaMalloc(&set->st_ids, n * 4));
        TREX_CUDA(cudaMalloc(&set->st_out, n * 2));
        TREX_CUDA(cudaMalloc(&set->st_out32, n * 4));
        set->st_n_cap = n;
    }
    for (auto &e : set->ev)
        if (!e) TREX_CUDA(cudaEventCreate(&e));
    cudaStream_t st = 0;
    TREX_CUDA(cudaEventRecord(set->ev[0], st));
    if (total_bytes)
        TREX_CUDA(cudaMemcpyAsync(set->st_data, h_data, total_bytes, cudaMemcpyHostToDevice, st));
    TREX_CUDA(cudaMemcpyAsync(set->st_off, h_offsets, (n + 1) * 8, cudaMemcpyHostToDevice, st));
    if (h_dfa_id) TREX_CUDA(cudaMemcpyAsync(set->st_ids, h_dfa_id, n * 4, cudaMemcpyHostToDevice, st));
    TREX_CUDA(cudaEventRecord(set->ev[1], st));
    uint32_t *err = nullptr;
    int rc = trex::dfa_set_run(set, set->st_data, set->st_off, h_dfa_id ? set->st_ids : nullptr, n,
                               total_bytes, h_final_state ? set->st_out : nullptr,
                               h_accept ? set->st_out + n : nullptr,
                               h_accept_i32 ? set->st_out32 : nullptr, nullptr, 0, seg_len, st,
                               &err);
    if (rc) return rc;
    TREX_CUDA(cudaEventRecord(set->ev[2], st));
    if (h_final_state)
        TREX_CUDA(cudaMemcpyAsync(h_final_state, set->st_out, n, cudaMemcpyDeviceToHost, st));
    if (h_accept)
        TREX_CUDA(cudaMemcpyAsync(h_accept, set->st_out + n, n, cudaMemcpyDeviceToHost, st));
    if (h_accept_i32)
        TREX_CUDA(cudaMemcpyAsync(h_accept_i32, set->st_out32, n * 4, cudaMemcpyDeviceToHost, st));
    uint32_t h_err = 0;
    TREX_CUDA(cudaMemcpyAsync(&h_err, err, 4, cudaMemcpyDeviceToHost, st));
    TREX_CUDA(cudaEventRecord(set->ev[3], st));
    TREX_CUDA(cudaEventSynchronize(set->ev[3]));
    if (kernel_ms) TREX_CUDA(cudaEventElapsedTime(kernel_ms, set->ev[1], set->ev[2]));
    if (total_ms) TREX_CUDA(cudaEventElapsedTime(total_ms, set->ev[0], set->ev[3]));
    if (h_err) {
        trex::set_last_error_msg("trex_dfa_batch_host: malformed offsets or automaton id");
        return TREX_ERR_ARG;
    }
    return TREX_OK;
}

int trex_dfa_batch_error(trex_dfa_set *set, void *scratch, int32_t *err_out) {
    // Error word of the last trex_dfa_batch_run that used `scratch` (NULL =
    // the set's own scratch); synchronises with the device.
    if (!set || !err_out) return TREX_ERR_ARG;
    uint8_t *sc = static_cast<uint8_t *>(scratch ? scratch : set->own_scratch);
    if (!sc) { *err_out = 0; return TREX_OK; }
    trex::ScratchLayout L = trex::scratch_layout(0, 0, 0);
    uint32_t v = 0;
    TREX_CUDA(cudaMemcpy(&v, sc + L.err, 4, cudaMemcpyDeviceToHost));
    *err_out = (int32_t)v;
    return TREX_OK;
}

int64_t trex_dfa_batch_scratch_bytes(int64_t n_strings, int64_t total_bytes, int32_t seg_len) {
    if (n_strings < 0 || total_bytes < 0) return -1;
    return (int64_t)trex::scratch_layout(n_strings, total_bytes, seg_len).total;
}

int trex_dfa_batch_run(trex_dfa_set *set, const uint8_t *data, const int64_t *offsets,
                       const int32_t *dfa_id, int64_t n_strings, int64_t total_bytes,
                       uint8_t *final_state, uint8_t *accept, int32_t *accept_i32, void *scratch,
                       int64_t scratch_bytes, int32_t seg_len, void *stream) {
    return trex::dfa_set_run(set, data, offsets, dfa_id, n_strings, total_bytes, final_state,
                             accept, accept_i32, scratch, scratch_bytes, seg_len,
                             static_cast<cudaStream_t>(stream), nullptr);
}

}  // extern "C"
