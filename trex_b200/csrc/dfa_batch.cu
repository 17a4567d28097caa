// Family (a): ragged batch DFA simulation over raw bytes, many resident DFAs,
// one persistent launch.
//
// Semantics (reference src/simulation.py:274-297 precompute_tmap and
// cuda/prefix_compose.cu:217-258 prefix_fused_kernel): every string walks
//     s = tmap[byte * N + s]
// from its DFA's start state; outputs are the final state and accept[s].
//
// Design
//  * Planning kernels cut every string into work items of at most seg_len
//    bytes, the cuts on 32-byte aligned addresses, queue them by DFA (one CTA
//    serves one DFA at a time) and, inside a DFA, by the bytes they walk in
//    64 length classes, longest first. Queue slots are reserved per tile of
//    strings with one global atomic per (DFA, class).
//  * Speculative entry states: an item other than the first of its string
//    does not know its entry state. It starts warm_bytes(N) earlier, inside
//    the previous item, from state 0; for a synchronising DFA (random DFAs
//    merge two chains with probability ~1/N per byte) the chain has then
//    reached the true entry state. The item records that guess next to its
//    end state; three small kernels chain each string's records (a thread per
//    string), walk each item whose guess was wrong from its true entry state
//    until it meets the recorded chain at a checkpoint (a thread per item), and
//    walk again, with a whole warp, the items whose chains never meet. Results
//    are exact for every DFA; only non-synchronising DFAs pay for re-walks.
//  * Main kernel: one persistent 1024-thread CTA per SM. The CTA expands the
//    current DFA's byte map (or its K-gram tables) into a per-lane replicated
//    shared-memory table (dfa_walk.cuh) so table lookups never conflict on
//    banks. For automata of 9-256 states a warp walks 64 items of a queue
//    together, two per lane as two independent chains (the items' records sit
//    in shared memory, so the walk keeps its registers); for automata of at
//    most 8 states 32 items, one per lane. Items of a batch have lengths within
//    128 bytes of each other; one 32-byte window per chain per step, the next
//    window loaded ahead; only a batch's first and last windows and warm-up
//    capture windows apply bytes under per-lane masks. No spin-waits anywhere.
#include <algorithm>
#include <cstring>
#include <mutex>

#include <cuda.h>
#include <new>
#include <vector>

#include "dfa_walk.cuh"

namespace trex {

// 16-byte aligned: a record is stored and loaded as two 128-bit accesses
struct alignas(16) WorkItem {
    int64_t p0;          // first byte walked (warm-up bytes included)
    int64_t end;         // one past the last byte of the item
    uint32_t str;
    uint32_t segn;       // item index (low 16 bits) | items of the string (high 16 bits)
    uint32_t map_base;   // first result slot of the string (strings with > 1 item)
    uint32_t entry;      // start state (bits 0-7) | warm-up bytes (bits 8-15)
};
constexpr int64_t kMaxItemsPerString = 65535;
constexpr int64_t kMaxWalkBytes = (int64_t)1 << 36;   // one item: a 32-bit count of windows
// Warm-up bytes of an item after the first of its string: 4 N rounded up to
// whole 32-byte windows (multiples of 32 keep aligned cuts aligned), at most
// seven windows (the record keeps the warm-up length in 8 bits). Two chains of
// a random N-state automaton merge with probability ~1/N per byte, so the
// warm-up chain has missed the true entry state with probability
// (1 - 1/N)^W: 1.4% for N = 8 (W = 32), 0.4% for N = 12 and 1.6% for N = 16
// (W = 64), 1.8% for N = 32 (W = 128), 2.9% for N = 64 (W = 224). When it has,
// the item's checkpoints (its chain's state 1, 2, 4 and 8 windows into its own
// bytes) let compose_fix_kernel walk from the true entry state only until the
// two chains meet (about N bytes).
constexpr int kSplitDfaStates = 64;   // strings of larger automata are not cut
__host__ __device__ __forceinline__ int64_t warm_bytes(int n_states, int64_t seg) {
    int64_t w = ((4 * (int64_t)n_states + 31) / 32) * 32;
    w = w < 32 ? 32 : w > 224 ? 224 : w;
    return w < seg ? w : seg;
}

// Error bits reported through the device error word.
enum : uint32_t {
    kErrBadOffsets = 1u,
    kErrBadDfaId = 2u,
    kErrCapacity = 4u,   // offsets overlap: more work items than the scratch holds
};

constexpr int kRaggedThreads = 1024;
constexpr int kPlanThreads = 1024;
constexpr int kMaxPlanCtas = 148;   // planning CTAs (one per SM on a B200)
// byte maps of a set up to this size are copied into the fix-up kernel's shared memory
// (two CTAs an SM); larger sets read them from global memory
constexpr int64_t kFixSmemBytes = 96 * 1024;
constexpr int kDefaultSegLen = 2048;
constexpr int kLenClasses = 64;

// ---- scratch layout -----------------------------------------------------------
struct ScratchLayout {
    size_t q_base, q_count, q_head, q_serve, q_bytes, err, n_items, n_fix, n_rw, items, maps, split_list, fix_list,
        rw_list, cta_bins, bin_base, bin_end, cta_maps, cta_splits, total;
    int64_t max_items, fix_cap;
};

// Bytes per work item: at least 64, a multiple of 32 (item cuts fall on window
// boundaries).
static int32_t effective_seg_len(int32_t seg_len) {
    if (seg_len <= 0) seg_len = kDefaultSegLen;
    seg_len = seg_len < 64 ? 64 : seg_len;
    return (int32_t)std::min<int64_t>(((int64_t)seg_len + 31) & ~(int64_t)31, 1 << 30);
}

static ScratchLayout scratch_layout(int64_t n_strings, int64_t total_bytes, int32_t seg_len) {
    ScratchLayout L{};
    seg_len = effective_seg_len(seg_len);
    L.max_items = n_strings + total_bytes / seg_len + 1;
    size_t o = 0;
    auto take = [&](size_t bytes) { size_t at = o; o = (o + bytes + 255) & ~size_t(255); return at; };
    // the front (up to items) is cleared before every run
    L.q_base = take(kMaxDfasPerSet * 4);
    L.q_count = take(kMaxDfasPerSet * 4);
    L.q_head = take(kMaxDfasPerSet * 4);
    L.q_serve = take(kMaxDfasPerSet * 4);
    L.q_bytes = take(kMaxDfasPerSet * 8);
    L.err = take(4);
    L.n_items = take(8);
    L.n_fix = take(4);
    L.n_rw = take(4);
    L.items = take((size_t)L.max_items * sizeof(WorkItem));
    L.maps = take((size_t)L.max_items * sizeof(uint64_t));
    // every string cut into several items: string, first map slot, items | automaton << 16 |
    // (states - 1) << 24, offset of its accept table
    L.split_list = take((size_t)std::max<int64_t>(n_strings, 1) * 16);
    // chaining the records: fix-up tasks (string, item << 8 | entry state), about 1% of the
    // items of split strings for the random automata of the benchmarks; a string whose task
    // finds the list full is walked again instead. Then the strings to walk again.
    L.fix_cap = std::max<int64_t>(1024, L.max_items / 8);
    L.fix_list = take((size_t)L.fix_cap * 8);
    L.rw_list = take((size_t)std::max<int64_t>(n_strings, 1) * 4);
    // planning: items per (planning CTA, DFA x length class), then those CTAs' first
    // queue positions; each class's end; map slots per planning CTA, then its first slot
    L.cta_bins = take((size_t)kMaxPlanCtas * kMaxDfasPerSet * kLenClasses * 4);
    L.bin_base = take(kMaxDfasPerSet * kLenClasses * 4);
    L.bin_end = take(kMaxDfasPerSet * kLenClasses * 4);
    L.cta_maps = take((kMaxPlanCtas + 1) * 4);
    L.cta_splits = take((kMaxPlanCtas + 1) * 4);
    L.total = o;
    return L;
}

// ---- planning kernels -------------------------------------------------------------
// Items of one string, which starts at byte s0 of the batch (base_mis: the
// address of the batch's first byte mod 32). The cuts fall on 32-byte aligned
// addresses: the first item is seg bytes plus up to 31 up to the next aligned
// address, the others seg bytes (a multiple of 32), the last the rest; so an
// item after the first starts its warm-up, its own bytes and (but the last) its
// end on window boundaries. seg grows for strings that would need more than
// kMaxItemsPerString items; strings of automata with more than kSplitDfaStates
// states are never cut.
struct ItemGeom {
    uint32_t k;
    int64_t seg, first;
};
__device__ __forceinline__ ItemGeom item_geom(int64_t len, int64_t s0, int n_states, int32_t seg_len,
                                              uint32_t base_mis) {
    if (len <= 0 || n_states > kSplitDfaStates) return ItemGeom{1, len, len};
    int64_t seg = seg_len;
    // more than kMaxItemsPerString pieces (ceil(len / seg) > K exactly when len > K seg):
    // longer pieces
    if (len > kMaxItemsPerString * seg)
        seg = (((len + kMaxItemsPerString - 1) / kMaxItemsPerString) + 31) & ~(int64_t)31;
    const int64_t pad = (int64_t)((32u - ((base_mis + (uint32_t)s0) & 31u)) & 31u);
    const int64_t first = seg + pad;
    if (len <= first) return ItemGeom{1, seg, len};
    // a 64-bit division is a long software routine on the GPU: 32 bits when they suffice
    // (seg < 2^31 always)
    const int64_t rest = len - first + seg - 1;
    const int64_t q = rest < ((int64_t)1 << 32) ? (int64_t)((uint32_t)rest / (uint32_t)seg) : rest / seg;
    return ItemGeom{(uint32_t)(1 + q), seg, first};
}
// Bytes [b0, b1) of item j of a string (s0, len).
__device__ __forceinline__ void item_range(const ItemGeom &g, int64_t s0, int64_t len, uint32_t j,
                                           int64_t *b0, int64_t *b1) {
    *b0 = j == 0 ? s0 : s0 + g.first + (int64_t)(j - 1) * g.seg;
    *b1 = (j + 1 == g.k) ? s0 + len : (j == 0 ? s0 + g.first : *b0 + g.seg);
}

// Queue order of an item by the bytes it walks (warm-up included), longest
// first: below 4 KiB one class per 128 bytes (class 32 + (4095 - len) / 128),
// above one class per power of two (4-8 KiB: 31, 8-16 KiB: 30, ...). Items of
// one class differ by at most 128 bytes, so a warp's batch of consecutive
// items spans nearly the same number of windows.
__device__ __forceinline__ int len_class(int64_t len) {
    if (len < 4096) return 32 + (int)((4095 - len) >> 7);
    const int c = 31 - ((63 - __clzll(len)) - 12);
    return c < 0 ? 0 : c;
}

// Classes of the items of a string cut into k pieces of seg bytes: the first
// piece (no warm-up), the k - 2 middle pieces and the last piece (both with
// warm-up). A string of one piece has only the last class.
struct ItemClasses {
    int first, mid, last;
};
__device__ __forceinline__ ItemClasses item_classes(int64_t len, const ItemGeom &g, int n_states) {
    const int64_t warm = warm_bytes(n_states, g.seg);
    if (g.k == 1) return ItemClasses{0, 0, len_class(len)};
    return ItemClasses{len_class(g.first), len_class(g.seg + warm),
                       len_class(len - g.first - (int64_t)(g.k - 2) * g.seg + warm)};
}

// Returns the DFA index of string i, or -1 (and raises an error bit) when the
// string is malformed; malformed strings get no work items. Multi-pattern runs
// (multi_n > 0) walk every one of multi_n strings with every automaton: string
// i is then string i mod multi_n of the batch on automaton i / multi_n.
__device__ __forceinline__ int checked_dfa(const int64_t *offsets, const int32_t *dfa_id,
                                           int64_t i, int n_dfas, int64_t total_bytes,
                                           uint32_t *err, int64_t *len_out,
                                           int64_t *start_out = nullptr, int64_t multi_n = 0) {
    const int64_t ii = multi_n > 0 ? i % multi_n : i;
    int64_t a = offsets[ii], b = offsets[ii + 1];
    int d = multi_n > 0 ? (int)(i / multi_n) : dfa_id ? dfa_id[i] : 0;
    if (a < 0 || b < a || b > total_bytes) {
        atomicOr(err, kErrBadOffsets);
        return -1;
    }
    if (d < 0 || d >= n_dfas) {
        atomicOr(err, kErrBadDfaId);
        return -1;
    }
    if (b - a > kMaxWalkBytes) {   // longer strings are refused (flagged, no result)
        atomicOr(err, kErrCapacity);
        return -1;
    }
    *len_out = b - a;
    if (start_out) *start_out = a;
    return d;
}

// A string's offsets and automaton as loaded (the planning kernels load the
// next tile's while they work on the current one); checked by checked_loaded.
struct StringIn {
    int64_t a, b;
    int32_t d;
    bool any;   // i < n
};
__device__ __forceinline__ StringIn load_string(const int64_t *offsets, const int32_t *dfa_id, int64_t i,
                                                int64_t n, int64_t multi_n) {
    StringIn r{0, 0, 0, false};
    if (i < n) {
        const int64_t ii = multi_n > 0 ? i % multi_n : i;
        r.a = offsets[ii];
        r.b = offsets[ii + 1];
        r.d = multi_n > 0 ? (int)(i / multi_n) : dfa_id ? dfa_id[i] : 0;
        r.any = true;
    }
    return r;
}
// checked_dfa on loaded values: -1 for no string or a malformed one (error bit raised).
__device__ __forceinline__ int checked_loaded(const StringIn &s, int n_dfas, int64_t total_bytes,
                                              uint32_t *err, int64_t *len_out, int64_t *start_out) {
    if (!s.any) return -1;
    if (s.a < 0 || s.b < s.a || s.b > total_bytes) {
        atomicOr(err, kErrBadOffsets);
        return -1;
    }
    if (s.d < 0 || s.d >= n_dfas) {
        atomicOr(err, kErrBadDfaId);
        return -1;
    }
    if (s.b - s.a > kMaxWalkBytes) {
        atomicOr(err, kErrCapacity);
        return -1;
    }
    *len_out = s.b - s.a;
    *start_out = s.a;
    return s.d;
}

// Warp-aggregated shared-memory counting: lanes with pred set add 1 to
// cnt[key]; one atomic per distinct key of the warp (all lanes call it).
__device__ __forceinline__ void warp_count(uint32_t *cnt, bool pred, int key) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t grp = __match_any_sync(0xffffffffu, pred ? key : -1);
    if (pred && (uint32_t)(__ffs(grp) - 1) == lane) atomicAdd(&cnt[key], (uint32_t)__popc(grp));
}
// Same, returning each lane's rank: the counter's old value plus the number
// of lanes of the same key below this one.
__device__ __forceinline__ uint32_t warp_rank(uint32_t *cnt, bool pred, int key) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t grp = __match_any_sync(0xffffffffu, pred ? key : -1);
    const int leader = __ffs(grp) - 1;
    uint32_t b = 0;
    if (pred && (uint32_t)leader == lane) b = atomicAdd(&cnt[key], (uint32_t)__popc(grp));
    b = __shfl_sync(0xffffffffu, b, leader);
    return b + (uint32_t)__popc(grp & ((1u << lane) - 1u));
}

// The planning kernels run with the same grid of at most kMaxPlanCtas CTAs of
// kPlanThreads threads, and CTA c takes the tiles of kPlanThreads consecutive
// strings t = c, c + G, c + 2G, ... in both: so the fill meets exactly the
// items the count saw, and each CTA writes its items into a range of every
// queue class reserved for it alone (no global atomics on the hot counters).

// Counts the items of every (DFA, length class) and the map slots of this CTA's
// strings into its row of cta_bins / cta_maps, and the items of the batch.
__global__ void __launch_bounds__(kPlanThreads)
plan_count_kernel(const int64_t *offsets, const int32_t *dfa_id, int64_t n, int64_t total_bytes,
                  const DfaDesc *desc, int n_dfas, int32_t seg_len, uint32_t base_mis, int64_t multi_n,
                  uint32_t *cta_bins, uint32_t *cta_maps, uint32_t *cta_splits, unsigned long long *n_items,
                  uint32_t *err) {
    __shared__ uint32_t cnt[kMaxDfasPerSet * kLenClasses];
    __shared__ unsigned long long items;
    __shared__ uint32_t maps, splits;
    const uint32_t lane = threadIdx.x & 31u;
    const int n_bins = n_dfas * kLenClasses;
    for (int t = threadIdx.x; t < n_bins; t += blockDim.x) cnt[t] = 0;
    if (threadIdx.x == 0) { items = 0; maps = 0; splits = 0; }
    __syncthreads();
    StringIn cur = load_string(offsets, dfa_id, (int64_t)blockIdx.x * kPlanThreads + threadIdx.x, n, multi_n);
    for (int64_t tile = blockIdx.x; tile * kPlanThreads < n; tile += gridDim.x) {
        const StringIn nxt =
            load_string(offsets, dfa_id, (tile + gridDim.x) * kPlanThreads + threadIdx.x, n, multi_n);
        int64_t len = 0, s0 = 0;
        const int d = checked_loaded(cur, n_dfas, total_bytes, err, &len, &s0);
        cur = nxt;
        uint32_t k = 0;
        ItemClasses ic{0, 0, 0};
        if (d >= 0) {
            const ItemGeom g = item_geom(len, s0, desc[d].n_states, seg_len, base_mis);
            k = g.k;
            ic = item_classes(len, g, desc[d].n_states);
        }
        const int kb = d * kLenClasses;
        warp_count(cnt, d >= 0 && k > 1, kb + ic.first);
        warp_count(cnt, d >= 0, kb + ic.last);
        if (d >= 0 && k > 2) atomicAdd(&cnt[kb + ic.mid], k - 2);
        const uint32_t ksum = __reduce_add_sync(0xffffffffu, k);
        const uint32_t msum = __reduce_add_sync(0xffffffffu, k > 1 ? k : 0u);
        if (lane == 0 && ksum) atomicAdd(&items, (unsigned long long)ksum);
        const uint32_t ssum = __popc(__ballot_sync(0xffffffffu, k > 1));
        if (lane == 0 && msum) atomicAdd(&maps, msum);
        if (lane == 0 && ssum) atomicAdd(&splits, ssum);
    }
    __syncthreads();
    uint32_t *row = cta_bins + (size_t)blockIdx.x * n_bins;
    for (int t = threadIdx.x; t < n_bins; t += blockDim.x) row[t] = cnt[t];
    if (threadIdx.x == 0) {
        cta_maps[blockIdx.x] = maps;
        cta_splits[blockIdx.x] = splits;
        if (items) atomicAdd(n_items, items);
    }
}

// A length class's typical walked bytes (its middle; only weighs the CTAs' first
// automaton): classes 32-63 hold 128-byte ranges below 4 KiB, 0-31 powers of two.
__device__ __forceinline__ unsigned long long class_bytes(int c) {
    if (c >= 32) return (unsigned long long)(4032 - 128 * (c - 32));
    const int e = min(12 + 31 - c, 40);
    return 3ull << (e - 1);
}

// Per class, the exclusive prefix of the G planning CTAs' counts, written over
// cta_bins, and the class's total into bin_end. Eight threads share a class:
// thread r of a class sums rows r * G / 8 .. (r + 1) * G / 8 (all loads in
// flight), the eight partial sums are scanned by shuffles.
constexpr int kPrefixParts = 8;
constexpr int kPrefixRows = (kMaxPlanCtas + kPrefixParts - 1) / kPrefixParts;
constexpr int kPrefixThreads = 256;
__global__ void __launch_bounds__(kPrefixThreads)
plan_prefix_kernel(uint32_t *cta_bins, uint32_t *bin_end, int G, int n_bins) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int b = t / kPrefixParts, r = t % kPrefixParts;
    const bool on = b < n_bins;
    const int c0 = r * G / kPrefixParts, c1 = (r + 1) * G / kPrefixParts;
    uint32_t v[kPrefixRows], part = 0;
#pragma unroll
    for (int u = 0; u < kPrefixRows; ++u) {
        v[u] = on && c0 + u < c1 ? cta_bins[(size_t)(c0 + u) * n_bins + b] : 0u;
        part += v[u];
    }
    uint32_t incl = part;
#pragma unroll
    for (int o = 1; o < kPrefixParts; o <<= 1) {
        const uint32_t x = __shfl_up_sync(0xffffffffu, incl, o, kPrefixParts);
        if (r >= o) incl += x;
    }
    uint32_t run = incl - part;
#pragma unroll
    for (int u = 0; u < kPrefixRows; ++u)
        if (on && c0 + u < c1) {
            cta_bins[(size_t)(c0 + u) * n_bins + b] = run;
            run += v[u];
        }
    if (on && r == kPrefixParts - 1) bin_end[b] = incl;
}

// One CTA of kPlanThreads threads. Turns the class totals into positions: class
// b of CTA c starts at bin_base[b] + cta_bins[c][b] (cta_bins holds the prefix
// over the CTAs after plan_prefix_kernel); classes follow each other by DFA and, inside a
// DFA, by class (each DFA's queue is one range, longest items first). bin_end
// gets each class's end and cta_maps each CTA's first map slot (cta_maps[G]:
// the total). Offsets that overlap (each string in range, but their lengths
// summing past total_bytes) would need more items than the scratch was sized
// for: then the error bit is set and every queue is left empty, so neither the
// fill kernel nor the ragged kernel writes an item.
__global__ void __launch_bounds__(kPlanThreads)
plan_scan_kernel(uint32_t *cta_bins, uint32_t *bin_base, uint32_t *bin_end, uint32_t *cta_maps,
                 uint32_t *cta_splits, int G,
                 int n_dfas, uint32_t *q_base, uint32_t *q_count, unsigned long long *q_bytes,
                 const unsigned long long *n_items, int64_t max_items, uint32_t *err) {
    constexpr int kPer = kMaxDfasPerSet * kLenClasses / kPlanThreads;   // classes a thread (pass 2)
    __shared__ uint32_t s_tot[kMaxDfasPerSet * kLenClasses];
    __shared__ uint32_t s_warp[kPlanThreads / 32];
    const int n_bins = n_dfas * kLenClasses;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (*n_items > (unsigned long long)max_items) {
        if (threadIdx.x == 0) {
            atomicOr(err, kErrCapacity);
            cta_splits[G] = 0;
        }
        if ((int)threadIdx.x < n_dfas) q_base[threadIdx.x] = q_count[threadIdx.x] = 0;
        return;
    }
    // the class totals (plan_prefix_kernel left them in bin_end)
    for (int b = threadIdx.x; b < n_bins; b += kPlanThreads) s_tot[b] = bin_end[b];
    __syncthreads();
    // pass 2: exclusive scan of the class totals in class order (thread t: classes kPer t ..)
    uint32_t tot[kPer], mine = 0;
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
        const int b = kPer * (int)threadIdx.x + j;
        tot[j] = b < n_bins ? s_tot[b] : 0u;
        mine += tot[j];
    }
    uint32_t incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += v;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = s_warp[lane];
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= (uint32_t)o) wi += v;
        }
        s_warp[lane] = wi - w;
    }
    __syncthreads();
    uint32_t base = s_warp[warp] + incl - mine;
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
        const int b = kPer * (int)threadIdx.x + j;
        if (b < n_bins) {
            bin_base[b] = base;
            bin_end[b] = base + tot[j];
            if (b % kLenClasses == 0) q_base[b / kLenClasses] = base;
            if (b % kLenClasses == kLenClasses - 1) q_count[b / kLenClasses] = base + tot[j];
            if (tot[j]) atomicAdd(&q_bytes[b / kLenClasses], tot[j] * class_bytes(b % kLenClasses));
        }
        base += tot[j];
    }
    __syncthreads();
    if ((int)threadIdx.x < n_dfas) q_count[threadIdx.x] -= q_base[threadIdx.x];
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (int c = 0; c < G; ++c) {
            const uint32_t v = cta_maps[c];
            cta_maps[c] = run;
            run += v;
        }
        cta_maps[G] = run;
        run = 0;
        for (int c = 0; c < G; ++c) {
            const uint32_t v = cta_splits[c];
            cta_splits[c] = run;
            run += v;
        }
        cta_splits[G] = run;
    }
}

// Writes the work items. CTA c takes the same tiles as in plan_count_kernel and
// hands out positions from its own ranges (shared-memory counters starting at
// its bases). A position outside the CTA's range of a class, or a range not
// filled exactly at the end (offsets rewritten while the plan ran), raises the
// capacity bit: the ragged kernel then trusts no item.
__global__ void __launch_bounds__(kPlanThreads)
plan_fill_kernel(const int64_t *offsets, const int32_t *dfa_id, int64_t n, int64_t total_bytes,
                 const DfaDesc *desc, int n_dfas, int32_t seg_len, uint32_t base_mis,
                 int64_t multi_n, const uint32_t *cta_bins, const uint32_t *bin_base,
                 const uint32_t *bin_end, const uint32_t *cta_maps, const uint32_t *cta_splits, WorkItem *items,
                 int64_t max_items, uint4 *split_list, uint32_t *err) {
    __shared__ uint32_t s_pos[kMaxDfasPerSet * kLenClasses];
    __shared__ uint32_t s_end[kMaxDfasPerSet * kLenClasses];
    __shared__ uint32_t s_map, s_map_end, s_split, s_split_end;
    const int n_bins = n_dfas * kLenClasses;
    const int G = gridDim.x, c = blockIdx.x;
    if (*(volatile uint32_t *)err & kErrCapacity) return;   // set by plan_scan_kernel: no items
    for (int t = threadIdx.x; t < n_bins; t += blockDim.x) {
        s_pos[t] = bin_base[t] + cta_bins[(size_t)c * n_bins + t];
        s_end[t] = c + 1 < G ? bin_base[t] + cta_bins[(size_t)(c + 1) * n_bins + t] : bin_end[t];
    }
    if (threadIdx.x == 0) {
        s_map = cta_maps[c];
        s_map_end = cta_maps[c + 1];
        s_split = cta_splits[c];
        s_split_end = cta_splits[c + 1];
    }
    __syncthreads();
    bool bad = false;
    StringIn cur = load_string(offsets, dfa_id, (int64_t)blockIdx.x * kPlanThreads + threadIdx.x, n, multi_n);
    for (int64_t tile = blockIdx.x; tile * kPlanThreads < n; tile += gridDim.x) {
        const int64_t i = tile * kPlanThreads + threadIdx.x;
        const StringIn nxt =
            load_string(offsets, dfa_id, (tile + gridDim.x) * kPlanThreads + threadIdx.x, n, multi_n);
        int64_t len = 0, s0 = 0;
        const int d = checked_loaded(cur, n_dfas, total_bytes, err, &len, &s0);
        cur = nxt;
        uint32_t k = 0, p_first = 0, p_mid = 0, p_last = 0, mb = 0;
        ItemClasses ic{0, 0, 0};
        ItemGeom g{0, 0, 0};
        if (d >= 0) {
            g = item_geom(len, s0, desc[d].n_states, seg_len, base_mis);
            k = g.k;
            ic = item_classes(len, g, desc[d].n_states);
            ic.first += d * kLenClasses;
            ic.mid += d * kLenClasses;
            ic.last += d * kLenClasses;
            if (k > 2) p_mid = atomicAdd(&s_pos[ic.mid], k - 2);
        }
        p_first = warp_rank(s_pos, d >= 0 && k > 1, ic.first);
        p_last = warp_rank(s_pos, d >= 0, ic.last);
        {   // map slots of split strings: a warp prefix sum, one shared atomic a warp
            const uint32_t lane = threadIdx.x & 31u;
            const uint32_t want = (d >= 0 && k > 1) ? k : 0u;
            uint32_t incl = want;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= (uint32_t)o) incl += v;
            }
            uint32_t wb = 0;
            if (lane == 31 && incl) wb = atomicAdd(&s_map, incl);
            wb = __shfl_sync(0xffffffffu, wb, 31);
            mb = wb + incl - want;
        }
        uint32_t sp = 0;   // this string's place in the list of split strings
        {
            const uint32_t lane = threadIdx.x & 31u;
            const uint32_t sb = __ballot_sync(0xffffffffu, d >= 0 && k > 1);
            uint32_t base = 0;
            if (lane == 0 && sb) base = atomicAdd(&s_split, (uint32_t)__popc(sb));
            sp = __shfl_sync(0xffffffffu, base, 0) + (uint32_t)__popc(sb & ((1u << lane) - 1u));
        }
        uint32_t warm = 0, start = 0;
        if (d >= 0) {
            warm = (uint32_t)warm_bytes(desc[d].n_states, g.seg);
            // every position must lie in this CTA's ranges (true when the offsets did not
            // change since the count): else no item of this string is written
            const bool in = (k <= 1 || (uint64_t)p_first < s_end[ic.first]) &&
                            (k <= 2 || (uint64_t)p_mid + (k - 2) <= s_end[ic.mid]) &&
                            p_last < s_end[ic.last] &&
                            (k <= 1 || ((uint64_t)mb + k <= s_map_end && (int64_t)mb + k <= max_items &&
                                        sp < s_split_end));
            if (!in) {
                bad = true;
                k = 0;
            }
            if (k > 1)
                split_list[sp] = make_uint4((uint32_t)i, mb,
                                            k | ((uint32_t)d << 16) | ((uint32_t)(desc[d].n_states - 1) << 24),
                                            (uint32_t)desc[d].accept_off);
            start = (uint32_t)desc[d].start;
        } else {
            k = 0;
        }
        // Items 0..3 of a string are written by its lane; the rest of long strings by the
        // warp together, 32 at a time (a string of many pieces would otherwise keep its
        // lane busy while the others idle): item t of the warp's rest belongs to the lane
        // whose inclusive prefix sum of rest counts first exceeds t.
        auto item_at = [&](const ItemGeom &go, int64_t so, int64_t lo_, uint32_t j, uint32_t pf, uint32_t pm,
                           uint32_t pl, uint32_t mbo, uint32_t wo, uint32_t sto, uint32_t stro) {
            const uint32_t pos = (j + 1 == go.k) ? pl : j == 0 ? pf : pm + (j - 1);
            if ((int64_t)pos >= max_items) {
                bad = true;
                return;
            }
            int64_t b0, b1;
            item_range(go, so, lo_, j, &b0, &b1);
            items[pos] = (j == 0) ? WorkItem{b0, b1, stro, j | (go.k << 16), mbo, sto}
                                  : WorkItem{b0 - wo, b1, stro, j | (go.k << 16), mbo, wo << 8};
        };
        constexpr uint32_t kOwn = 4;
#pragma unroll
        for (uint32_t j = 0; j < kOwn; ++j)
            if (j < k) item_at(g, s0, len, j, p_first, p_mid, p_last, mb, warm, start, (uint32_t)i);
        {
            const uint32_t FULL = 0xffffffffu, lane = threadIdx.x & 31u;
            const uint32_t kx = k > kOwn ? k - kOwn : 0u;
            if (__any_sync(FULL, kx != 0)) {
                uint32_t incl = kx;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t v = __shfl_up_sync(FULL, incl, o);
                    if (lane >= (uint32_t)o) incl += v;
                }
                const uint32_t total = __shfl_sync(FULL, incl, 31);
                for (uint32_t t0 = 0; t0 < total; t0 += 32) {
                    const uint32_t t = t0 + lane;
                    uint32_t o = 0;   // lanes whose inclusive count is <= t
#pragma unroll
                    for (uint32_t step = 16; step >= 1; step >>= 1)
                        if (__shfl_sync(FULL, incl, o + step - 1) <= t) o += step;
                    const uint32_t ko = __shfl_sync(FULL, k, o), io = __shfl_sync(FULL, incl, o);
                    const int64_t so = __shfl_sync(FULL, s0, o), lo_ = __shfl_sync(FULL, len, o);
                    const ItemGeom go{ko, __shfl_sync(FULL, g.seg, o), __shfl_sync(FULL, g.first, o)};
                    const uint32_t pf = __shfl_sync(FULL, p_first, o), pm = __shfl_sync(FULL, p_mid, o);
                    const uint32_t pl = __shfl_sync(FULL, p_last, o), mbo = __shfl_sync(FULL, mb, o);
                    const uint32_t wo = __shfl_sync(FULL, warm, o), sto = __shfl_sync(FULL, start, o);
                    const uint32_t stro = __shfl_sync(FULL, (uint32_t)i, o);
                    if (t >= total) continue;
                    const uint32_t j = kOwn + t - (io - (ko - kOwn));   // the item's index in its string
                    item_at(go, so, lo_, j, pf, pm, pl, mbo, wo, sto, stro);
                }
            }
        }
    }
    __syncthreads();
    // every range of this CTA must have been filled exactly
    for (int t = threadIdx.x; t < n_bins; t += blockDim.x) bad |= s_pos[t] != s_end[t];
    if (threadIdx.x == 0) bad |= s_map != s_map_end || s_split != s_split_end;
    if (bad) atomicOr(err, kErrCapacity);
}

// ---- main kernel -------------------------------------------------------------------------
struct RaggedParams {
    const uint8_t *data;
    int64_t total_bytes;
    const int64_t *offsets;
    const uint8_t *tmaps;
    const uint8_t *accepts;
    const DfaDesc *desc;
    int n_dfas;
    int32_t seg_len;
    const WorkItem *items;
    const uint32_t *q_base;
    const uint32_t *q_count;
    uint32_t *q_head;
    uint32_t *q_serve;           // CTAs walking each queue
    const unsigned long long *q_bytes;
    uint32_t *err;
    uint64_t *maps;
    const uint4 *split_list;     // every split string: string, first map slot, items | automaton << 16
                                 // | (states - 1) << 24, offset of its accept table
    const uint32_t *n_split;     // their number
    uint2 *fix_list;             // fix-up tasks: split string, item << 8 | entry state
    uint32_t fix_cap;
    uint32_t fix_tm_bytes;   // byte maps copied to shared memory by the fix-up kernel (0: read globally)
    uint32_t *n_fix;
    uint32_t *rw_list;           // split strings to walk again
    uint32_t *n_rw;
    const int32_t *dfa_id;
    int64_t n;
    int64_t max_items;
    uint32_t base_mis;
    int64_t multi_n;
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

// Record of one item of a split string, for the compose kernels, which chain the
// items of the string after the walk: bits 0-7 the guessed entry state (the
// state after the warm-up; the start state for the first item), 8-15 the end
// state, 16-47 the checkpoints (four states, see capture_cp).
__device__ __forceinline__ void publish_item(const RaggedParams &P, uint32_t segn, uint32_t mb,
                                             uint32_t guess, uint32_t fin, uint32_t cps) {
    P.maps[mb + (segn & 0xffffu)] = (uint64_t)(guess | (fin << 8)) | ((uint64_t)cps << 16);
}

// One item of a batch, as a lane holds it (segn == 0: no item).
__device__ __forceinline__ WorkItem load_item(const RaggedParams &P, uint32_t base, uint32_t idx,
                                              uint32_t count) {
    if (idx < count) return P.items[base + idx];
    return WorkItem{0, 0, 0, 0, 0, 0};
}

// Window walk with a byte mask (bit j: byte j of the window belongs to the
// item) and a capture: when cpos > 0, cap_e takes the state after byte
// cpos - 1 (the end of the warm-up).
template <class W>
__device__ __forceinline__ uint32_t walk_masked(const W &w, uint32_t e, uint4 a, uint4 b, uint32_t m,
                                                uint32_t cpos, uint32_t &cap_e) {
    const uint32_t x[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        uint32_t n;
#define TREX_MSTEP(J)                                       \
        n = w.template step<J>(e, x[k]);                    \
        e = (m >> (4 * k + J)) & 1u ? n : e;                \
        cap_e = (4u * k + J + 1u == cpos) ? e : cap_e;
        TREX_MSTEP(0) TREX_MSTEP(1) TREX_MSTEP(2) TREX_MSTEP(3)
#undef TREX_MSTEP
    }
    return e;
}

// ---- window walkers ------------------------------------------------------------------------
// A mode advances a state over one 32-byte window: fast() when all 32 bytes
// belong to the item, masked() with a byte mask and the warm-up capture.
template <class W>
struct ByteMode {
    static constexpr bool kWideLetters = false;
    W w;
    __device__ __forceinline__ bool valid(uint4, uint4) const { return true; }
    __device__ __forceinline__ uint32_t fast(uint32_t e, uint4 a, uint4 b) const {
        e = step16(w, e, a);
        return step16(w, e, b);
    }
    // half a window (16 bytes) of two independent chains, interleaved byte by byte
    __device__ __forceinline__ void fast2_half(uint32_t &e0, uint4 a0, uint32_t &e1, uint4 a1) const {
        const uint32_t x0[4] = {a0.x, a0.y, a0.z, a0.w};
        const uint32_t x1[4] = {a1.x, a1.y, a1.z, a1.w};
        uint32_t s0 = e0, s1 = e1;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            s0 = w.template step<0>(s0, x0[k]); s1 = w.template step<0>(s1, x1[k]);
            s0 = w.template step<1>(s0, x0[k]); s1 = w.template step<1>(s1, x1[k]);
            s0 = w.template step<2>(s0, x0[k]); s1 = w.template step<2>(s1, x1[k]);
            s0 = w.template step<3>(s0, x0[k]); s1 = w.template step<3>(s1, x1[k]);
        }
        e0 = s0;
        e1 = s1;
    }
    __device__ __forceinline__ uint32_t masked(uint32_t e, uint4 a, uint4 b, uint32_t m, uint32_t cpos,
                                               uint32_t &cap_e) const {
        return walk_masked(w, e, a, b, m, cpos, cap_e);
    }
    // two chains over one window each, byte j applied where bit j of the chain's mask is set
    __device__ __forceinline__ void masked2(uint32_t &e0, uint4 a0, uint4 b0, uint32_t m0, uint32_t &e1,
                                            uint4 a1, uint4 b1, uint32_t m1) const {
        const uint32_t x0[8] = {a0.x, a0.y, a0.z, a0.w, b0.x, b0.y, b0.z, b0.w};
        const uint32_t x1[8] = {a1.x, a1.y, a1.z, a1.w, b1.x, b1.y, b1.z, b1.w};
        uint32_t s0 = e0, s1 = e1;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
#define TREX_MSTEP2(J)                                                  \
            {                                                           \
                const uint32_t n0 = w.template step<J>(s0, x0[k]);      \
                const uint32_t n1 = w.template step<J>(s1, x1[k]);      \
                s0 = (m0 >> (4 * k + J)) & 1u ? n0 : s0;                \
                s1 = (m1 >> (4 * k + J)) & 1u ? n1 : s1;                \
            }
            TREX_MSTEP2(0) TREX_MSTEP2(1) TREX_MSTEP2(2) TREX_MSTEP2(3)
#undef TREX_MSTEP2
        }
        e0 = s0;
        e1 = s1;
    }
};

// Offset of the per-code fallback table (after the largest main table).
constexpr uint32_t kFallbackOff = kRepTableBytes16;
constexpr uint32_t kFallbackBytes = 17 * 512;

// K-gram walking for an automaton whose bytes fall into at most 2^BITS
// distinguished bytes ("letters", one code each) plus one shared column for
// every other byte. A window whose 32 bytes are all letters is walked K bytes
// per lookup: the codes of K consecutive bytes (first byte most significant)
// form an 8-bit gram index into a table of K-step transitions in the same
// layout as the byte table. Other windows are walked byte by byte through a
// table of 2^BITS + 1 columns (the letters' codes, then the shared column).
// Codes come from one shift and mask; a byte is a letter exactly when the
// letter of its code equals it, which every window is checked for.
template <class W, int BITS, int K>
struct GramMode {
    W w;
    uint32_t sh;
    uint32_t alpha[4];
    static constexpr bool kWideLetters = BITS == 4;
    static constexpr uint32_t kMask = BITS == 1 ? 0x01010101u : BITS == 2 ? 0x03030303u : 0x0F0F0F0Fu;
    static constexpr uint32_t kOther = (1u << BITS) * 0x01010101u;   // the shared column, 4 bytes
    __device__ __forceinline__ uint32_t codes(uint32_t x) const { return (x >> sh) & kMask; }
    // the letter of each byte's code, in byte order
    __device__ __forceinline__ uint32_t letters(uint32_t y) const {
        if (BITS == 1) {
            const uint32_t a0 = alpha[0] & 0xFFu, a1 = (alpha[0] >> 8) & 0xFFu;
            return a0 * 0x01010101u ^ y * (a0 ^ a1);
        } else if (BITS == 2) {
            const uint32_t v = y | (y >> 12);   // selectors of bytes 0, 2, 1, 3 in nibbles 0-3
            return __byte_perm(__byte_perm(alpha[0], 0, v), 0, 0x3120);
        } else {
            const uint32_t v = y | (y >> 12);
            const uint32_t v7 = v & 0x7777u;
            const uint32_t lo = __byte_perm(alpha[0], alpha[1], v7);
            const uint32_t hi = __byte_perm(alpha[2], alpha[3], v7);
            const uint32_t sel = __byte_perm(((y >> 3) & 0x01010101u) * 0xFFu, 0, 0x3120);
            return __byte_perm((lo & ~sel) | (hi & sel), 0, 0x3120);
        }
    }
    __device__ __forceinline__ bool word_ok(uint32_t x) const { return letters(codes(x)) == x; }
    __device__ __forceinline__ bool valid(uint4 a, uint4 b) const {
        return word_ok(a.x) & word_ok(a.y) & word_ok(a.z) & word_ok(a.w) & word_ok(b.x) &
               word_ok(b.y) & word_ok(b.z) & word_ok(b.w);
    }
    __device__ __forceinline__ uint32_t grams_word(uint32_t e, uint32_t x) const {
        const uint32_t y = codes(x);
        if (BITS == 4) {   // K = 2: grams c0c1, c2c3 in bytes 1 and 3
            const uint32_t p = y * 0x1001u;
            e = w.template step<1>(e, p);
            return w.template step<3>(e, p);
        } else if (K == 2) {
            const uint32_t p = y * (BITS == 2 ? 0x401u : 0x201u);
            e = w.template step<1>(e, p);
            return w.template step<3>(e, p);
        } else {           // K = 4: one gram in byte 3
            const uint32_t p = y * (BITS == 2 ? 0x40100401u : 0x08040201u);
            return w.template step<3>(e, p);
        }
    }
    __device__ __forceinline__ uint32_t fast(uint32_t e, uint4 a, uint4 b) const {
        if (K == 8) {      // BITS = 1: the codes of two words make one gram
            const uint32_t x[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
            for (int k = 0; k < 8; k += 2) {
                const uint32_t h0 = ((codes(x[k]) * 0x08040201u) >> 20) & 0xF0u;
                const uint32_t h1 = (codes(x[k + 1]) * 0x08040201u) >> 24;
                e = w.template step<0>(e, h0 | h1);
            }
            return e;
        }
        e = grams_word(e, a.x); e = grams_word(e, a.y); e = grams_word(e, a.z); e = grams_word(e, a.w);
        e = grams_word(e, b.x); e = grams_word(e, b.y); e = grams_word(e, b.z);
        return grams_word(e, b.w);
    }
    // half a window (16 bytes) of two independent chains
    __device__ __forceinline__ void fast2_half(uint32_t &e0, uint4 a0, uint32_t &e1, uint4 a1) const {
        const uint32_t x0[4] = {a0.x, a0.y, a0.z, a0.w};
        const uint32_t x1[4] = {a1.x, a1.y, a1.z, a1.w};
        uint32_t s0 = e0, s1 = e1;
        if (K == 8) {
#pragma unroll
            for (int k = 0; k < 4; k += 2) {
                const uint32_t g0 = (((codes(x0[k]) * 0x08040201u) >> 20) & 0xF0u) |
                                    ((codes(x0[k + 1]) * 0x08040201u) >> 24);
                const uint32_t g1 = (((codes(x1[k]) * 0x08040201u) >> 20) & 0xF0u) |
                                    ((codes(x1[k + 1]) * 0x08040201u) >> 24);
                s0 = w.template step<0>(s0, g0);
                s1 = w.template step<0>(s1, g1);
            }
        } else {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                s0 = grams_word(s0, x0[k]);
                s1 = grams_word(s1, x1[k]);
            }
        }
        e0 = s0;
        e1 = s1;
    }
    // the fallback column of each byte: its code for a letter, else the shared column
    __device__ __forceinline__ uint32_t columns(uint32_t x) const {
        const uint32_t y = codes(x);
        const uint32_t d = x ^ letters(y);
        const uint32_t nz = (((d & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | d) & 0x80808080u;   // 0x80: byte differs
        const uint32_t ne = (nz >> 7) * 0xFFu;
        return (y & ~ne) | (kOther & ne);
    }
    __device__ __forceinline__ uint32_t masked(uint32_t e, uint4 a, uint4 b, uint32_t m, uint32_t cpos,
                                               uint32_t &cap_e) const {
        const uint32_t x[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint32_t col = columns(x[k]);
            uint32_t n;
#define TREX_GSTEP(J)                                               \
            n = w.template step_off<J>(kFallbackOff, e, col);       \
            e = (m >> (4 * k + J)) & 1u ? n : e;                    \
            cap_e = (4u * k + J + 1u == cpos) ? e : cap_e;
            TREX_GSTEP(0) TREX_GSTEP(1) TREX_GSTEP(2) TREX_GSTEP(3)
#undef TREX_GSTEP
        }
        return e;
    }
    // two chains through the per-code table, byte j where bit j of the chain's mask is set
    __device__ __forceinline__ void masked2(uint32_t &e0, uint4 a0, uint4 b0, uint32_t m0, uint32_t &e1,
                                            uint4 a1, uint4 b1, uint32_t m1) const {
        const uint32_t x0[8] = {a0.x, a0.y, a0.z, a0.w, b0.x, b0.y, b0.z, b0.w};
        const uint32_t x1[8] = {a1.x, a1.y, a1.z, a1.w, b1.x, b1.y, b1.z, b1.w};
        uint32_t s0 = e0, s1 = e1;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint32_t col0 = columns(x0[k]), col1 = columns(x1[k]);
#define TREX_GSTEP2(J)                                                          \
            {                                                                   \
                const uint32_t n0 = w.template step_off<J>(kFallbackOff, s0, col0); \
                const uint32_t n1 = w.template step_off<J>(kFallbackOff, s1, col1); \
                s0 = (m0 >> (4 * k + J)) & 1u ? n0 : s0;                        \
                s1 = (m1 >> (4 * k + J)) & 1u ? n1 : s1;                        \
            }
            TREX_GSTEP2(0) TREX_GSTEP2(1) TREX_GSTEP2(2) TREX_GSTEP2(3)
#undef TREX_GSTEP2
        }
        e0 = s0;
        e1 = s1;
    }
};

// Tables of a K-gram automaton: the gram table (256 columns) at 0 and the
// fallback table at kFallbackOff.
__device__ inline void build_gram_tables(const DfaDesc &D, const uint8_t *__restrict__ src) {
    const int N = D.n_states, bits = D.kbits, K = D.kgram;
    const uint32_t mask = (1u << bits) - 1u, ncode = 1u << bits;
    const uint8_t *rep = D.krep;
    build_layout(N, 256, 0, [&](uint32_t g, uint32_t s) {
        uint32_t t = s;
        for (int i = K - 1; i >= 0; --i) t = src[rep[(g >> (bits * i)) & mask] * N + t];
        return t;
    });
    build_layout(N, (int)ncode + 1, kFallbackOff,
                 [&](uint32_t c, uint32_t s) { return (uint32_t)src[rep[c] * N + s]; });
}

// Shared memory after the tables: the two work items every thread walks (16
// 32-bit words a thread).
constexpr uint32_t kLaneItemsOff = kFallbackOff + kFallbackBytes;
// Then one 32-bit word a thread and chain: the checkpoints of the chain's item.
constexpr uint32_t kCpOff = kLaneItemsOff + kRaggedThreads * 2 * (uint32_t)sizeof(WorkItem);
constexpr uint32_t kRaggedSmemBytes = kCpOff + kRaggedThreads * 2 * 4;

// Checkpoints of an item after the first of its string: its chain's state at
// the start of windows cw + 1, cw + 2, cw + 4 and cw + 8 (32, 64, 128 and 256
// bytes into the item's own bytes, which start on a window boundary), one byte
// each (encoded) of the thread's word for the chain. Called at the start of
// window `it`; any other window stores nothing.
__device__ __forceinline__ void capture_cp(int chain, uint32_t it, uint32_t cw, uint32_t e) {
    const uint32_t d = it - cw;
    if (d - 1u < 8u && (d & (d - 1u)) == 0u)
        g_dfa_tbl[kCpOff + (chain * kRaggedThreads + threadIdx.x) * 4 + (__ffs(d) - 1)] = (uint8_t)e;
}
// The four checkpoints of a finished item, decoded, packed one byte each; a
// checkpoint at or past the item's last window is its end state.
template <class W>
__device__ __forceinline__ uint32_t checkpoints(int chain, uint32_t cw, uint32_t nw, uint32_t fin) {
    const uint32_t raw =
        *reinterpret_cast<volatile uint32_t *>(g_dfa_tbl + kCpOff + (chain * kRaggedThreads + threadIdx.x) * 4);
    uint32_t cps = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint32_t v = cw + (1u << k) < nw ? W::dec((raw >> (8 * k)) & 0xffu) : fin;
        cps |= v << (8 * k);
    }
    return cps;
}

// A lane's item as the walk sees it: windows [wp, wp + 32 nw), the item's
// bytes from byte lo of the first window to byte he - 1 of the last; the
// warm-up ends at byte cpos of window cw (cw = ~0u: no warm-up).
struct ItemView {
    const uint8_t *wp;
    uint32_t lo, nw, he, cw, cpos;
};
__device__ __forceinline__ bool item_live(const WorkItem &w) { return w.segn != 0 && w.end > w.p0; }
__device__ __forceinline__ ItemView item_view(const RaggedParams &P, const WorkItem &w) {
    ItemView v;
    const bool live = item_live(w);
    const uint32_t warm = (w.entry >> 8) & 0xffu;
    const int64_t nbytes = w.end - w.p0;
    const uint8_t *q0 = P.data + (live ? w.p0 : 0);
    v.wp = reinterpret_cast<const uint8_t *>((uintptr_t)q0 & ~(uintptr_t)31);
    v.lo = (uint32_t)(q0 - v.wp);
    v.nw = live ? (uint32_t)((v.lo + nbytes + 31) >> 5) : 0u;
    v.he = live ? (uint32_t)(v.lo + nbytes - 32 * (int64_t)(v.nw - 1)) : 0u;
    const uint32_t cb = v.lo + warm;
    v.cw = warm ? (cb >> 5) : 0xffffffffu;
    v.cpos = cb & 31u;
    return v;
}
// A thread's item slot in shared memory: the record's eight 32-bit words,
// word k at slot[k * kRaggedThreads], so the lanes of a warp read and write
// consecutive words (no bank conflicts).
__device__ __forceinline__ void write_slot(uint32_t *slot, const WorkItem &w) {
    slot[0] = (uint32_t)w.p0;
    slot[kRaggedThreads] = (uint32_t)((uint64_t)w.p0 >> 32);
    slot[2 * kRaggedThreads] = (uint32_t)w.end;
    slot[3 * kRaggedThreads] = (uint32_t)((uint64_t)w.end >> 32);
    slot[4 * kRaggedThreads] = w.str;
    slot[5 * kRaggedThreads] = w.segn;
    slot[6 * kRaggedThreads] = w.map_base;
    slot[7 * kRaggedThreads] = w.entry;
}
// Read again at every use (volatile: the compiler keeps none of the fields in
// registers across the unmasked walk).
__device__ __forceinline__ WorkItem read_slot(const uint32_t *slot) {
    const volatile uint32_t *v = slot;
    WorkItem w;
    w.p0 = (int64_t)(((uint64_t)v[kRaggedThreads] << 32) | v[0]);
    w.end = (int64_t)(((uint64_t)v[3 * kRaggedThreads] << 32) | v[2 * kRaggedThreads]);
    w.str = v[4 * kRaggedThreads];
    w.segn = v[5 * kRaggedThreads];
    w.map_base = v[6 * kRaggedThreads];
    w.entry = v[7 * kRaggedThreads];
    return w;
}

// One window of one chain with per-lane masks: window `it` of the slot's item
// is (a, b); the next window is loaded into (a, b). A lane whose item ended
// before this window keeps its state.
template <class M>
__device__ __forceinline__ void masked_window(const RaggedParams &P, const M &md, const DfaDesc &D,
                                              const uint32_t *slot, int chain, uint32_t it, uint32_t &e,
                                              uint32_t &cap_e, uint4 &a, uint4 &b) {
    const uint32_t FULL = 0xffffffffu;
    const WorkItem w = read_slot(slot);
    const ItemView v = item_view(P, w);
    const uint4 ca = a, cb = b;
    if (it + 1 < v.nw) load_window(v.wp + 32 * (size_t)(it + 1), P.data, P.data + P.total_bytes, a, b);
    const uint32_t mlo = it == 0 ? v.lo : 0u;
    const uint32_t mhi = it + 1 < v.nw ? 32u : (it + 1 == v.nw ? v.he : 0u);
    const uint32_t m = bit_range((int)mlo, (int)mhi);
    const bool cap = it == v.cw;
    if (cap && v.cpos == 0) cap_e = e;   // the warm-up ended with the previous window
    capture_cp(chain, it, v.cw, e);
    const bool special = (it < v.nw && (m != FULL || !md.valid(ca, cb))) || (cap && v.cpos != 0);
    const uint32_t e_in = e;
    if (!__any_sync(FULL, special)) e = md.fast(e, ca, cb);
    else e = md.masked(e, ca, cb, m, cap ? v.cpos : 0u, cap_e);
    e = it < v.nw ? e : e_in;
}

// After a batch: the final state of the slot's item (or the split item's
// record).
template <class W>
__device__ __forceinline__ void finish_item(const RaggedParams &P, const DfaDesc &D, const uint32_t *slot,
                                            int chain, uint32_t e, uint32_t cap_e) {
    const WorkItem w = read_slot(slot);
    if (!item_live(w)) return;
    const uint32_t fin = W::dec(e);
    if ((w.segn >> 16) == 1) {
        write_result(P, w.str, fin, D.accept_off);
    } else if ((w.entry >> 8) & 0xffu) {
        const ItemView v = item_view(P, w);
        publish_item(P, w.segn, w.map_base, W::dec(cap_e), fin, checkpoints<W>(chain, v.cw, v.nw, fin));
    } else {
        publish_item(P, w.segn, w.map_base, w.entry & 0xffu, fin, 0u);
    }
}

// Queue d's first item and item count, read again at each batch (volatile:
// no register holds them across the walk).
__device__ __forceinline__ uint32_t q_base_of(const RaggedParams &P, int d) {
    return *(const volatile uint32_t *)&P.q_base[d];
}
__device__ __forceinline__ uint32_t q_count_of(const RaggedParams &P, int d) {
    return *(const volatile uint32_t *)&P.q_count[d];
}

// Both chains of a batch over the windows [it, end) that every lane walks
// whole (the next windows as well); CAPTURE: some warm-up ends in this range.
template <bool CAPTURE, class M>
__device__ __forceinline__ void whole_windows(const M &md, uint32_t &it, uint32_t end,
                                              const uint8_t *wp0, const uint8_t *wp1, uint32_t cw0,
                                              uint32_t cw1, uint32_t &e0, uint32_t &e1, uint32_t &cap0,
                                              uint32_t &cap1, uint4 &a0, uint4 &c0, uint4 &a1,
                                              uint4 &c1) {
    const uint32_t FULL = 0xffffffffu;
    for (; it < end; ++it) {
        if (CAPTURE) {
            cap0 = it == cw0 ? e0 : cap0;
            cap1 = it == cw1 ? e1 : cap1;
            capture_cp(0, it, cw0, e0);
            capture_cp(1, it, cw1, e1);
        }
        if (__all_sync(FULL, md.valid(a0, c0) && md.valid(a1, c1))) {
            // the next windows are loaded once the first halves are walked, so
            // that their registers are free
            md.fast2_half(e0, a0, e1, a1);
            const uint4 y0 = c0, y1 = c1;
            ld_stream32(wp0 + 32 * (size_t)(it + 1), a0, c0);
            ld_stream32(wp1 + 32 * (size_t)(it + 1), a1, c1);
            md.fast2_half(e0, y0, e1, y1);
        } else {
            const uint4 x0 = a0, y0 = c0, x1 = a1, y1 = c1;
            ld_stream32(wp0 + 32 * (size_t)(it + 1), a0, c0);
            ld_stream32(wp1 + 32 * (size_t)(it + 1), a1, c1);
            uint32_t unused = 0;
            if (__all_sync(FULL, md.valid(x0, y0))) e0 = md.fast(e0, x0, y0);
            else e0 = md.masked(e0, x0, y0, FULL, 0u, unused);
            if (__all_sync(FULL, md.valid(x1, y1))) e1 = md.fast(e1, x1, y1);
            else e1 = md.masked(e1, x1, y1, FULL, 0u, unused);
        }
    }
}

// Drains queue d with this warp, 32 items (one a lane, one chain a thread) at
// a time; automata of at most 8 states take this path (their two-instruction
// step gains nothing from a second chain on ragged batches, measured). The
// items of a queue are ordered by walked length (warm-up included), longest
// first, in 128-byte classes, so the items of a batch span nearly the same number of
// 32-byte windows: the lanes start and finish together, and every window
// between a batch's first and last is walked without masks. The records of the
// next batch are claimed and loaded while the current one is walked; the next
// window of every lane is loaded while the current one is walked.
template <class M>
__device__ void drain_queue_one(const RaggedParams &P, const M &md, const DfaDesc &D, int d) {
    const uint32_t base = P.q_base[d], count = P.q_count[d];
    uint32_t *const head = &P.q_head[d];
    using W = decltype(md.w);
    const W &w = md.w;
    const uint32_t FULL = 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31u;
    const uint8_t *const lo_ok = P.data, *const hi_ok = P.data + P.total_bytes;
    uint32_t b0 = 0;
    if (lane == 0) b0 = atomicAdd(head, 32u);
    b0 = __shfl_sync(FULL, b0, 0);
    if (b0 >= count) return;
    WorkItem cur = load_item(P, base, b0 + lane, count);
    while (true) {
        uint32_t b1 = 0;
        if (lane == 0) b1 = atomicAdd(head, 32u);
        b1 = __shfl_sync(FULL, b1, 0);
        const WorkItem nxt = load_item(P, base, b1 + lane, count);

        // ---- this lane's item: windows [wp, wp + 32 nw), bytes [lo, lo + nbytes) of them
        const uint32_t warm = (cur.entry >> 8) & 0xffu, entry = cur.entry & 0xffu;
        const int64_t nbytes = cur.end - cur.p0;   // walked bytes, warm-up included
        bool live = cur.segn != 0;
        if (live && nbytes <= 0) {   // empty string: its final state is the start state
            write_result(P, cur.str, entry, D.accept_off);
            live = false;
        }
        const uint8_t *q0 = P.data + (live ? cur.p0 : 0);
        const uint8_t *wp = reinterpret_cast<const uint8_t *>((uintptr_t)q0 & ~(uintptr_t)31);
        const uint32_t lo = (uint32_t)(q0 - wp);
        const uint32_t nw = live ? (uint32_t)((lo + nbytes + 31) >> 5) : 0u;
        const uint32_t he = live ? (uint32_t)(lo + nbytes - 32 * (int64_t)(nw - 1)) : 0u;   // 1..32
        const uint32_t cb = lo + warm;   // the item's own bytes start here (relative to wp)
        const uint32_t cw = warm ? (cb >> 5) : 0xffffffffu, cpos = cb & 31u;
        uint32_t e = w.enc(live ? entry : 0u);
        uint32_t cap_e = e;
        const uint32_t maxw = __reduce_max_sync(FULL, nw);
        uint4 a = make_uint4(0, 0, 0, 0), b = a;
        if (nw) load_window(wp, lo_ok, hi_ok, a, b);
        for (uint32_t it = 0; it < maxw; ++it) {
            const uint4 ca = a, cbv = b;
            if (it + 1 < nw) load_window(wp + 32 * (size_t)(it + 1), lo_ok, hi_ok, a, b);
            const uint32_t mlo = it == 0 ? lo : 0u;
            const uint32_t mhi = it + 1 < nw ? 32u : (it + 1 == nw ? he : 0u);
            const uint32_t m = bit_range((int)mlo, (int)mhi);
            const bool cap = it == cw;
            if (cap && cpos == 0) cap_e = e;   // the warm-up ended with the previous window
            capture_cp(0, it, cw, e);
            const bool special =
                (it < nw && (m != FULL || !md.valid(ca, cbv))) || (cap && cpos != 0);
            if (!__any_sync(FULL, special)) e = md.fast(e, ca, cbv);
            else e = md.masked(e, ca, cbv, m, cap ? cpos : 0u, cap_e);
            if (it + 1 == nw) {   // this lane's item ends in this window
                const uint32_t fin = W::dec(e);
                if ((cur.segn >> 16) == 1)
                    write_result(P, cur.str, fin, D.accept_off);
                else if (warm)
                    publish_item(P, cur.segn, cur.map_base, W::dec(cap_e), fin,
                                 checkpoints<W>(0, cw, nw, fin));
                else
                    publish_item(P, cur.segn, cur.map_base, entry, fin, 0u);
            }
        }
        if (b1 >= count) break;
        cur = nxt;
    }
}

// Bits of the bytes of window `it` that belong to the item (0 past its end).
__device__ __forceinline__ uint32_t window_mask(uint32_t it, const ItemView &v) {
    const uint32_t mlo = it == 0 ? v.lo : 0u;
    const uint32_t mhi = it + 1 < v.nw ? 32u : (it + 1 == v.nw ? v.he : 0u);
    return bit_range((int)mlo, (int)mhi);
}

// Windows [it, end) of both chains with per-lane masks (a batch's first and
// last windows): the two chains are walked together, byte by byte, each byte
// applied where it belongs to the lane's item; a warm-up that ends at a window
// boundary is captured before the window. A window where a warm-up ends inside
// (cuts off the 32-byte grid) goes through the one-chain masked step.
template <class M>
__device__ __forceinline__ void edge_windows(const RaggedParams &P, const M &md, const DfaDesc &D,
                                             const uint32_t *slot0, const uint32_t *slot1, uint32_t &it,
                                             uint32_t end, uint32_t &e0, uint32_t &cap0, uint4 &a0,
                                             uint4 &c0, uint32_t &e1, uint32_t &cap1, uint4 &a1,
                                             uint4 &c1) {
    const uint32_t FULL = 0xffffffffu;
    for (; it < end; ++it) {
        const ItemView v0 = item_view(P, read_slot(slot0)), v1 = item_view(P, read_slot(slot1));
        if (__any_sync(FULL, (it == v0.cw && v0.cpos != 0) || (it == v1.cw && v1.cpos != 0))) {
            masked_window(P, md, D, slot0, 0, it, e0, cap0, a0, c0);
            masked_window(P, md, D, slot1, 1, it, e1, cap1, a1, c1);
            continue;
        }
        cap0 = it == v0.cw ? e0 : cap0;
        cap1 = it == v1.cw ? e1 : cap1;
        capture_cp(0, it, v0.cw, e0);
        capture_cp(1, it, v1.cw, e1);
        const uint32_t m0 = window_mask(it, v0), m1 = window_mask(it, v1);
        const uint4 x0 = a0, y0 = c0, x1 = a1, y1 = c1;
        if (it + 1 < v0.nw) load_window(v0.wp + 32 * (size_t)(it + 1), P.data, P.data + P.total_bytes, a0, c0);
        if (it + 1 < v1.nw) load_window(v1.wp + 32 * (size_t)(it + 1), P.data, P.data + P.total_bytes, a1, c1);
        if (__all_sync(FULL, (m0 & m1) == FULL && md.valid(x0, y0) && md.valid(x1, y1))) {
            md.fast2_half(e0, x0, e1, x1);
            md.fast2_half(e0, y0, e1, y1);
        } else {
            md.masked2(e0, x0, y0, m0, e1, x1, y1, m1);
        }
    }
}

// Drains queue d with this warp, 64 items at a time: lane l walks items l and
// 32 + l of the batch as two independent chains, so every thread keeps two
// table lookups in flight (with one chain a thread, the walk is bound by the
// latency of its dependent lookups, not by the table's bandwidth). The items
// of a queue are ordered by walked length (warm-up included), longest first,
// in 128-byte classes, so the 64 items of a batch span nearly the same number
// of 32-byte windows. The windows every lane of both chains walks whole (from
// the latest first whole window to the earliest last whole window of the
// batch) go through an unmasked loop whose loads need no bounds checks; the
// batch's first and last windows go through the masked step. Results are
// written after the batch. The next batch's records are prefetched into L2
// while the current one is walked.
template <class M>
__device__ void drain_queue(const RaggedParams &P, const M &md, const DfaDesc &D, int d) {
    using W = decltype(md.w);
    const W &w = md.w;
    const uint32_t FULL = 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31u;
    // per warp: the next batch, then the batch's fl, cwmax and the windows of
    // each chain (below)
    __shared__ uint32_t s_warp[kRaggedThreads / 32][5];
    volatile uint32_t *const wv = s_warp[threadIdx.x >> 5];
    uint32_t *const slot0 = reinterpret_cast<uint32_t *>(g_dfa_tbl + kLaneItemsOff) + threadIdx.x;
    uint32_t *const slot1 = slot0 + 8 * kRaggedThreads;
    uint32_t b0 = 0;
    if (lane == 0) b0 = atomicAdd(&P.q_head[d], 64u);
    b0 = __shfl_sync(FULL, b0, 0);
    {
        const uint32_t base = q_base_of(P, d), count = q_count_of(P, d);
        if (b0 >= count) return;
        write_slot(slot0, load_item(P, base, b0 + lane, count));
        write_slot(slot1, load_item(P, base, b0 + 32 + lane, count));
    }
    while (true) {
        {
            uint32_t b1 = 0;
            if (lane == 0) b1 = atomicAdd(&P.q_head[d], 64u);
            b1 = __shfl_sync(FULL, b1, 0);
            const uint32_t base = q_base_of(P, d), count = q_count_of(P, d);
            if (b1 + lane < count) prefetch_l2(P.items + base + b1 + lane);
            if (b1 + 32 + lane < count) prefetch_l2(P.items + base + b1 + 32 + lane);
            __syncwarp();
            if (lane == 0) wv[0] = b1;
        }

        // ---- both chains: entry state, first window, whole-window range [ff, fl)
        uint32_t e0, e1, ff;
        uint4 a0 = make_uint4(0, 0, 0, 0), c0 = a0, a1 = a0, c1 = a0;
        {
            const WorkItem w0 = read_slot(slot0), w1 = read_slot(slot1);
            // empty strings: the final state is the start state
            if (w0.segn != 0 && w0.end <= w0.p0) write_result(P, w0.str, w0.entry & 0xffu, D.accept_off);
            if (w1.segn != 0 && w1.end <= w1.p0) write_result(P, w1.str, w1.entry & 0xffu, D.accept_off);
            const ItemView v0 = item_view(P, w0), v1 = item_view(P, w1);
            e0 = w.enc(item_live(w0) ? (w0.entry & 0xffu) : 0u);
            e1 = w.enc(item_live(w1) ? (w1.entry & 0xffu) : 0u);
            if (v0.nw) load_window(v0.wp, P.data, P.data + P.total_bytes, a0, c0);
            if (v1.nw) load_window(v1.wp, P.data, P.data + P.total_bytes, a1, c1);
            // window j of an item is whole when j >= (lo != 0) and j < nw - (he != 32); a
            // warm-up that ends inside a window needs the masked step there
            uint32_t f0 = v0.lo != 0 ? 1u : 0u, f1 = v1.lo != 0 ? 1u : 0u;
            if (v0.cw != 0xffffffffu && v0.cpos != 0) f0 = max(f0, v0.cw + 1u);
            if (v1.cw != 0xffffffffu && v1.cpos != 0) f1 = max(f1, v1.cw + 1u);
            const uint32_t l0 = v0.nw == 0 ? 0u : v0.nw - (v0.he != 32 ? 1u : 0u);
            const uint32_t l1 = v1.nw == 0 ? 0u : v1.nw - (v1.he != 32 ? 1u : 0u);
            ff = __reduce_max_sync(FULL, max(f0, f1));
            const uint32_t fl = __reduce_min_sync(FULL, min(l0, l1));
            const uint32_t nw0 = __reduce_max_sync(FULL, v0.nw), nw1 = __reduce_max_sync(FULL, v1.nw);
            const uint32_t nwmax = max(nw0, nw1);
            // the capture phase ends after the last checkpoint (window cw + 8) of any lane
            const uint32_t cwmax = __reduce_max_sync(FULL, max(v0.cw == 0xffffffffu ? 0u : v0.cw + 9u,
                                                               v1.cw == 0xffffffffu ? 0u : v1.cw + 9u));
            if (lane == 0) {
                wv[1] = fl;
                wv[2] = cwmax;
                wv[3] = nw0;
                wv[4] = nw1;
            }
            __syncwarp();
            ff = min(ff, nwmax);
        }
        // Warp-uniform values live in shared memory and the windows' addresses are
        // derived again after the first windows, so that the masked steps have
        // the registers to themselves.
        uint32_t cap0 = e0, cap1 = e1;
        uint32_t it = 0;
        edge_windows(P, md, D, slot0, slot1, it, ff, e0, cap0, a0, c0, e1, cap1, a1, c1);
        // windows it and it + 1 are whole for every lane of both chains, inside
        // the items' bytes and so inside the batch buffer; the warm-ups end
        // before window cwmax
        if (const uint32_t fl = wv[1]; fl > 0) {
            const ItemView v0 = item_view(P, read_slot(slot0)), v1 = item_view(P, read_slot(slot1));
            whole_windows<true>(md, it, min(fl - 1u, wv[2]), v0.wp, v1.wp, v0.cw, v1.cw, e0, e1, cap0,
                                cap1, a0, c0, a1, c1);
            whole_windows<false>(md, it, fl - 1u, v0.wp, v1.wp, v0.cw, v1.cw, e0, e1, cap0, cap1, a0, c0,
                                 a1, c1);
        }
        edge_windows(P, md, D, slot0, slot1, it, max(wv[3], wv[4]), e0, cap0, a0, c0, e1, cap1, a1, c1);
        finish_item<W>(P, D, slot0, 0, e0, cap0);
        finish_item<W>(P, D, slot1, 1, e1, cap1);
        const uint32_t b1 = wv[0], base = q_base_of(P, d), count = q_count_of(P, d);
        if (b1 >= count) break;
        write_slot(slot0, load_item(P, base, b1 + lane, count));
        write_slot(slot1, load_item(P, base, b1 + 32 + lane, count));
    }
}

// One chain a thread for automata of at most 8 states (and for K-gram walks
// over 16 letters, whose letter table leaves no registers for a second chain),
// two for larger ones.
template <class M>
__device__ __forceinline__ void drain(const RaggedParams &P, const M &md, const DfaDesc &D, int d) {
    if constexpr (decltype(md.w)::kChains == 8 || M::kWideLetters) drain_queue_one(P, md, D, d);
    else drain_queue(P, md, D, d);
}

__global__ void __launch_bounds__(kRaggedThreads, 1) dfa_ragged_kernel(RaggedParams P) {
    __shared__ int s_dfa;
    // The plan is complete when no planning CTA raised the capacity bit: each
    // filled its disjoint ranges exactly (so every item slot was written once);
    // otherwise (capacity overflow, or offsets rewritten while the plan ran) no
    // item is trusted.
    const bool planned = (*(volatile uint32_t *)P.err & kErrCapacity) == 0;
    if (threadIdx.x == 0) {
        // Home DFA: CTAs are spread over DFAs in proportion to their walking
        // time, estimated as bytes x 7/8 for automata of at most 8 states (their
        // step is two instructions instead of four; measured 0.86 of the time per
        // byte on ragged batches) and bytes x 8/8 otherwise.
        auto weight = [&](int d) { return P.q_bytes[d] * (P.desc[d].n_states <= 8 ? 7ull : 8ull); };
        unsigned long long tot = 0;
        for (int d = 0; d < P.n_dfas; ++d) tot += weight(d);
        int home = -1;
        if (tot && planned) {
            unsigned long long pos =
                (unsigned long long)((double)tot * ((double)blockIdx.x + 0.5) / gridDim.x);
            unsigned long long run = 0;
            for (int d = 0; d < P.n_dfas; ++d) {
                run += weight(d);
                if (P.q_count[d] && pos < run) { home = d; break; }
            }
            if (home < 0)
                for (int d = P.n_dfas - 1; d >= 0; --d)
                    if (P.q_count[d]) { home = d; break; }
        }
        if (home >= 0) atomicAdd(&P.q_serve[home], 1u);
        s_dfa = home;
    }
    __syncthreads();
    if (s_dfa < 0) return;
    const uint32_t lane = threadIdx.x & 31u;
    for (int round = 0; round <= P.n_dfas; ++round) {
        const int d = s_dfa;
        if (d < 0) break;
        const DfaDesc D = P.desc[d];
        const bool gram = D.kgram > 1 && D.n_states <= kSmallDfaStates;
        if (gram) build_gram_tables(D, P.tmaps + D.tmap_off);
        else build_table(P.tmaps + D.tmap_off, D.n_states);
        __syncthreads();
        if (gram) {
            const uint32_t sh = (uint32_t)D.kshift;
            const uint32_t *al = D.kalpha;
#define TREX_GRAM(WT, B, KK)                                                                                 drain(P, GramMode<WT, B, KK>{WT{lane}, sh, {al[0], al[1], al[2], al[3]}}, D, d)
#define TREX_GRAMS(WT)                                                                                       switch (D.kbits * 16 + D.kgram) {                                                                    case 16 + 2: TREX_GRAM(WT, 1, 2); break;                                                          case 16 + 4: TREX_GRAM(WT, 1, 4); break;                                                          case 16 + 8: TREX_GRAM(WT, 1, 8); break;                                                          case 32 + 2: TREX_GRAM(WT, 2, 2); break;                                                          case 32 + 4: TREX_GRAM(WT, 2, 4); break;                                                          default: TREX_GRAM(WT, 4, 2); break;                                                          }
            if (D.n_states <= 8) { TREX_GRAMS(Walker<8>) }
            else { TREX_GRAMS(Walker<16>) }
#undef TREX_GRAMS
#undef TREX_GRAM
        } else if (D.n_states <= 8) {
            drain(P, ByteMode<Walker<8>>{Walker<8>{lane}}, D, d);
        } else if (D.n_states <= 16) {
            drain(P, ByteMode<Walker<16>>{Walker<16>{lane}}, D, d);
        } else if (D.n_states <= 32) {
            drain(P, ByteMode<Walker<32>>{Walker<32>{lane}}, D, d);
        } else if (D.n_states <= 64) {
            drain(P, ByteMode<Walker<64>>{Walker<64>{lane}}, D, d);
        } else {
            drain(P, ByteMode<Walker<0>>{Walker<0>{(uint32_t)D.n_states}}, D, d);
        }
        __syncthreads();
        // Next queue: the one whose remaining walk per CTA walking it is the largest, so
        // that the queues end together (the launch ends with its last queue). Its
        // remaining bytes are estimated as items left x the longest of them (the head:
        // queues run longest first); warp 0 scores the queues in parallel.
        if (threadIdx.x < 32) {
            if (threadIdx.x == 0) atomicSub(&P.q_serve[d], 1u);
            unsigned long long best_score = 0;
            int best = -1;
            for (int e = (int)lane; e < P.n_dfas; e += 32) {
                const uint32_t h = *(volatile uint32_t *)&P.q_head[e], c = P.q_count[e];
                if (h >= c) continue;
                const WorkItem w = P.items[P.q_base[e] + h];
                const unsigned long long len = w.end > w.p0 ? (unsigned long long)(w.end - w.p0) : 1ull;
                const uint32_t serve = *(volatile uint32_t *)&P.q_serve[e];
                const unsigned long long score = (unsigned long long)(c - h) * len / (serve + 1ull);
                if (best < 0 || score > best_score) {
                    best_score = score;
                    best = e;
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const unsigned long long os = __shfl_xor_sync(0xffffffffu, best_score, o);
                const int ob = __shfl_xor_sync(0xffffffffu, best, o);
                if (ob >= 0 && (best < 0 || os > best_score || (os == best_score && ob < best))) {
                    best_score = os;
                    best = ob;
                }
            }
            if (threadIdx.x == 0) {
                if (best >= 0) atomicAdd(&P.q_serve[best], 1u);
                s_dfa = best;
            }
        }
        __syncthreads();
    }
}

// Re-walks bytes [b0, b1) of one item from state s_in with the whole warp:
// lane l computes the map of all N (<= 16) states over its 1/32 of the bytes
// (16 independent chains through the byte map in shared memory), then the 32
// maps are applied in order. Returns the end state (every lane).
__device__ __forceinline__ uint32_t warp_rewalk(const uint8_t *tbl, uint32_t N, const uint8_t *data,
                                                int64_t b0, int64_t b1, uint32_t s_in) {
    const uint32_t lane = threadIdx.x & 31u;
    const int64_t c = (b1 - b0 + 31) / 32;
    const int64_t q0 = min(b1, b0 + (int64_t)lane * c), q1 = min(b1, q0 + c);
    uint32_t st[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) st[j] = (uint32_t)j;
    for (int64_t q = q0; q < q1; ++q) {
        const uint8_t *row = tbl + (uint32_t)__ldg(data + q) * N;
#pragma unroll
        for (int j = 0; j < 16; ++j)
            if ((uint32_t)j < N) st[j] = row[st[j]];
    }
    uint64_t map = 0;
#pragma unroll
    for (int j = 0; j < 16; ++j) map |= (uint64_t)st[j] << (4 * j);
    uint32_t s = s_in;
    for (int l = 0; l < 32; ++l) {
        const uint64_t ml = __shfl_sync(0xffffffffu, map, l);
        s = (uint32_t)(ml >> (4 * s)) & 15u;
    }
    return s;
}

constexpr int kComposeThreads = 256;

// Walks bytes [p, q) of the batch from state s through a byte map in global
// memory (L1-cached): one lane, aligned 32-byte windows.
// SHARED_TM: tm points into shared memory (a generic load; the read-only global load
// below is for global memory only).
template <bool SHARED_TM = false>
__device__ __forceinline__ uint32_t lane_walk(const RaggedParams &P, const uint8_t *__restrict__ tm,
                                              uint32_t N, int64_t p, int64_t q, uint32_t s) {
    const uint8_t *lo = P.data + p, *hi = P.data + q;
    const uint8_t *w = reinterpret_cast<const uint8_t *>((uintptr_t)lo & ~(uintptr_t)31);
    uint4 na = make_uint4(0u, 0u, 0u, 0u), nb = na;
    if (w < hi) load_window(w, lo, hi, na, nb);
    for (; w < hi; w += 32) {
        // the next window is loaded while this one is walked
        const uint4 a = na, b = nb;
        if (w + 32 < hi) load_window(w + 32, lo, hi, na, nb);
        const uint32_t x[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
        for (int j = 0; j < 32; ++j)
            if (w + j >= lo && w + j < hi) {
                const uint8_t *a = tm + ((x[j >> 2] >> (8 * (j & 3))) & 0xffu) * N + s;
                s = SHARED_TM ? *a : __ldg(a);
            }
    }
    return s;
}

// Item j (> 0) of a split string whose warm-up chain missed the true entry
// state s_in: walks the item from s_in until its state equals the recorded
// chain's at one of the checkpoints (after 1, 2, 4 and 8 windows of its own
// bytes); from there the two chains are one, so the item ends in the recorded
// end state. Returns the item's end state, or 0xFFFF when the chains had not
// met by the last checkpoint (the caller then walks the item whole).
template <bool SHARED_TM = false>
__device__ __forceinline__ uint32_t fix_item_body(const RaggedParams &P, const uint8_t *__restrict__ tm,
                                                  uint32_t N, int64_t b0, int64_t b1, uint32_t s_in,
                                                  uint64_t rec) {
    // the item's own bytes start on a window boundary (aligned cuts, whole-window warm-up)
    const int64_t a0 = b0 - (int64_t)((P.base_mis + (uint32_t)b0) & 31u);
    int64_t p = b0;
    uint32_t s = s_in;
    for (int k = 0; k < 4; ++k) {
        const int64_t q = min(a0 + ((int64_t)32 << k), b1);
        s = lane_walk<SHARED_TM>(P, tm, N, p, q, s);
        if (q == b1) return s;
        if (s == ((uint32_t)(rec >> (16 + 8 * k)) & 0xffu)) return (uint32_t)(rec >> 8) & 0xffu;
        p = q;
    }
    // no meeting at a checkpoint (slowly merging or non-synchronising automata): walk on to
    // the item's end, whose state is then known either way
    return lane_walk<SHARED_TM>(P, tm, N, p, b1, s);
}
// Not inlined into the fix-up kernel's loop (keeps its registers); the re-walk
// path inlines the body instead.
template <bool SHARED_TM>
__device__ __noinline__ uint32_t fix_item(const RaggedParams &P, const uint8_t *__restrict__ tm, uint32_t N,
                                          int64_t b0, int64_t b1, uint32_t s_in, uint64_t rec) {
    return fix_item_body<SHARED_TM>(P, tm, N, b0, b1, s_in, rec);
}

// Index in a device list, with one atomic per group of lanes that append together.
__device__ __forceinline__ uint32_t append_slot(uint32_t *count) {
    const uint32_t m = __activemask();
    const uint32_t lane = threadIdx.x & 31u;
    const int leader = __ffs(m) - 1;
    uint32_t base = 0;
    if ((int)lane == leader) base = atomicAdd(count, (uint32_t)__popc(m));
    base = __shfl_sync(m, base, leader);
    return base + (uint32_t)__popc(m & ((1u << lane) - 1u));
}

// Split string x must be walked again from item j with entry state e: word j << 9 | a << 8 |
// e, where a = 1 when e is only the chain's assumption (item j - 1's recorded end) and a = 0
// when e was walked (a fix-up of item j - 1 that never met the chain walked on to its end).
// The smallest word wins: the earliest item, and for one item a walked entry over an
// assumed one (two marks can name the same item with different entries: the assumed one
// is then wrong, since item j - 1's fix-up found another end). The word lives in the low
// half of item 0's record, which nothing reads once the records are chained; the first
// mark puts the string on the re-walk list.
__device__ __forceinline__ uint32_t rewalk_word(uint32_t j, uint32_t e, bool assumed) {
    return (j << 9) | (assumed ? 256u : 0u) | e;
}
__device__ __forceinline__ void mark_rewalk(const RaggedParams &P, uint32_t x, uint32_t mb, uint32_t word) {
    if (atomicMin(reinterpret_cast<uint32_t *>(P.maps + mb), word) == 0xFFFFFFFFu)
        P.rw_list[append_slot(P.n_rw)] = x;
}

// Strings cut into several items, step 1 of 3: chains each string's records.
// Item j's record is right when its guessed entry equals the end state of item
// j - 1 (item 0 starts from the start state). A record whose guess is wrong
// becomes a fix-up task (string, item, entry state) and the chain goes on as if
// the fix-up meets the recorded chain, so the entry of item j + 1 is item j's
// recorded end state; the string's final state is written on that assumption and
// corrected by the two kernels below where it fails. A warp takes 32 strings of
// the list and lays their items out back to back (a prefix sum of the item
// counts): a pass gives each lane one item, so most passes chain a dozen strings
// at once (split strings have a few items each). Lane l compares its guess with
// lane l - 1's end state (the previous item of the same string, or, for lane 0,
// the last item of the previous pass).
__global__ void __launch_bounds__(kComposeThreads) compose_chain_kernel(RaggedParams P) {
    if (*(volatile uint32_t *)P.err & kErrCapacity) return;   // the plan was refused
    const uint32_t FULL = 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    const int64_t n_split = *P.n_split;
    const int64_t nwarps = (int64_t)gridDim.x * (kComposeThreads / 32);
    for (int64_t base = ((int64_t)blockIdx.x * (kComposeThreads / 32) + wib) * 32; base < n_split;
         base += nwarps * 32) {
        const bool mine = base + lane < n_split;
        const uint4 ent = mine ? P.split_list[base + lane] : make_uint4(0u, 0u, 0u, 0u);
        uint32_t k = mine ? ent.z & 0xffffu : 0u;
        if (k != 0 && (k < 2 || (int64_t)ent.y + (int64_t)k > P.max_items)) {
            atomicOr(P.err, kErrCapacity);   // not written by this plan
            k = 0;
        }
        // inclusive prefix of the item counts: string s owns items [incl_s - k_s, incl_s)
        uint32_t incl = k;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(FULL, incl, o);
            if (lane >= (uint32_t)o) incl += v;
        }
        const uint32_t total = __shfl_sync(FULL, incl, 31);
        uint32_t carry = 0;   // end state of the previous pass's last item
        for (uint32_t t0 = 0; t0 < total; t0 += 32) {
            const uint32_t t = t0 + lane;
            // string of item t: the first s with incl_s > t (binary search over the lanes)
            uint32_t lo = 0;
#pragma unroll
            for (uint32_t step = 16; step > 0; step >>= 1) {
                const uint32_t v = __shfl_sync(FULL, incl, (int)(lo + step - 1));
                if (v <= t) lo += step;
            }
            const uint32_t sidx = min(lo, 31u);
            const uint32_t s_incl = __shfl_sync(FULL, incl, (int)sidx);
            const uint32_t s_k = __shfl_sync(FULL, k, (int)sidx);
            const uint32_t s_mb = __shfl_sync(FULL, ent.y, (int)sidx);
            const uint32_t s_z = __shfl_sync(FULL, ent.z, (int)sidx);
            const uint32_t s_str = __shfl_sync(FULL, ent.x, (int)sidx);
            const uint32_t s_acc = __shfl_sync(FULL, ent.w, (int)sidx);
            const bool live = t < total;
            const uint32_t j = t - (s_incl - s_k);
            const uint64_t rec = live ? P.maps[s_mb + j] : 0ull;
            const uint32_t end = (uint32_t)(rec >> 8) & 0xffu;
            uint32_t prev = __shfl_up_sync(FULL, end, 1);
            if (lane == 0) prev = carry;
            carry = __shfl_sync(FULL, end, 31);
            // no re-walk yet: the low word of item 0's record (read above) becomes the mark,
            // before any lane of the warp may lower it
            if (live && j == 0) *reinterpret_cast<uint32_t *>(P.maps + s_mb) = 0xFFFFFFFFu;
            __syncwarp();
            if (!live) continue;
            const uint32_t x = (uint32_t)(base + sidx);
            if (j != 0 && ((uint32_t)rec & 0xffu) != prev) {
                const uint32_t f = append_slot(P.n_fix);
                if (f < P.fix_cap) P.fix_list[f] = make_uint2(x, (j << 8) | prev);
                else mark_rewalk(P, x, s_mb, rewalk_word(j, prev, true));   // the list is full: walk again from here
            }
            if (j + 1 == s_k) {
                if (end < (s_z >> 24) + 1u) write_result(P, s_str, end, s_acc);
                else atomicOr(P.err, kErrCapacity);   // records not written by this plan
            }
        }
    }
}

// Step 2 of 3, one thread per fix-up task: walks item j from its true entry state
// until it meets the recorded chain at a checkpoint (fix_item: about one window for
// synchronising automata), else to the item's end. Met, or the same end state: the
// chained result stands. A last item: its end state is the string's final state.
// Otherwise (the chains never met: automata that do not synchronise, such as
// permutations) the next item's entry is now known and the string is marked to be
// walked again from there.
__global__ void __launch_bounds__(kComposeThreads) compose_fix_kernel(RaggedParams P) {
    extern __shared__ __align__(16) uint8_t s_fix_tm[];
    if (*(volatile uint32_t *)P.err & kErrCapacity) return;
    const uint32_t n_fix = min(*(volatile uint32_t *)P.n_fix, P.fix_cap);
    if (blockIdx.x * kComposeThreads >= n_fix) return;   // no task for this CTA
    // small sets: every byte map in shared memory, so a fix-up's dependent lookups do not
    // wait on L1 / L2 (the slowest tasks walk up to a few hundred bytes)
    const bool shared_tm = P.fix_tm_bytes != 0;
    if (shared_tm) {
        const uint4 *src = reinterpret_cast<const uint4 *>(P.tmaps);
        uint4 *dst = reinterpret_cast<uint4 *>(s_fix_tm);
        for (uint32_t i = threadIdx.x; i < P.fix_tm_bytes / 16u; i += kComposeThreads) dst[i] = src[i];
        __syncthreads();
    }
    for (uint32_t t = blockIdx.x * kComposeThreads + threadIdx.x; t < n_fix; t += gridDim.x * kComposeThreads) {
        const uint2 task = P.fix_list[t];
        const uint32_t x = task.x, j = task.y >> 8, e = task.y & 0xffu;
        const uint4 ent = P.split_list[x];
        const uint32_t mb = ent.y, k = ent.z & 0xffffu, N = (ent.z >> 24) + 1u;
        const int d = (int)((ent.z >> 16) & 0xffu);
        int64_t len = 0, s0 = 0;
        ItemGeom g{0, 0, 0};
        if (checked_dfa(P.offsets, P.dfa_id, (int64_t)ent.x, P.n_dfas, P.total_bytes, P.err, &len, &s0,
                        P.multi_n) == d)
            g = item_geom(len, s0, (int)N, P.seg_len, P.base_mis);
        if (g.k != k || j >= k) {   // offsets changed since the plan
            atomicOr(P.err, kErrCapacity);
            continue;
        }
        const uint64_t rec = P.maps[mb + j];
        int64_t b0, b1;
        item_range(g, s0, len, j, &b0, &b1);
        const uint32_t f = e >= N ? 0xFFFFu
                           : shared_tm ? fix_item<true>(P, s_fix_tm + P.desc[d].tmap_off, N, b0, b1, e, rec)
                                       : fix_item<false>(P, P.tmaps + P.desc[d].tmap_off, N, b0, b1, e, rec);
        if (f == ((uint32_t)(rec >> 8) & 0xffu)) continue;
        if (f >= N) mark_rewalk(P, x, mb, rewalk_word(j, e, true));
        else if (j + 1 == k) write_result(P, ent.x, f, ent.w);
        else mark_rewalk(P, x, mb, rewalk_word(j + 1, f, false));
    }
}

// The re-walk of a split string of an automaton of more than 16 states, by one
// lane through the byte map in global memory: item jb (its fix-up never met the
// recorded chain) is walked whole from s_entry; each later item takes its
// recorded end state when its guess is the true entry, else a fix-up, and is
// walked whole only when that does not meet either, so a lane walks about one
// item, not the rest of the string.
__device__ __noinline__ void rewalk_lane(const RaggedParams &P, const ItemGeom &g, int64_t s0, int64_t len,
                                         int d, uint32_t N, uint32_t mb, uint32_t k, uint32_t jb,
                                         uint32_t s_entry, uint32_t str, uint32_t aoff) {
    const uint8_t *tm = P.tmaps + P.desc[d].tmap_off;
    uint32_t s = s_entry;
    for (uint32_t j = jb; j < k && s < N; ++j) {
        int64_t b0, b1;
        item_range(g, s0, len, j, &b0, &b1);
        uint32_t f = 0xFFFFu;
        bool known = false;
        if (j > jb) {
            const uint64_t rec = P.maps[mb + j];
            known = ((uint32_t)rec & 0xffu) == s;
            f = known ? ((uint32_t)(rec >> 8) & 0xffu) : fix_item_body(P, tm, N, b0, b1, s, rec);
        }
        s = (known || f != 0xFFFFu) ? f : lane_walk(P, tm, N, b0, b1, s);
    }
    if (s < N) write_result(P, str, s, aoff);
    else atomicOr(P.err, kErrCapacity);   // records not written by this plan
}

// Step 3 of 3, a warp per string on the re-walk list: walks the marked item again
// whole from its entry state (each lane maps all N states over 1/32 of the item),
// then checks the following records 32 at a time, walking again every item whose
// guess differs from its predecessor's true end state. Exact for every DFA.
__global__ void __launch_bounds__(kComposeThreads) compose_rewalk_kernel(RaggedParams P) {
    __shared__ __align__(16) uint8_t s_tbl[kComposeThreads / 32][256 * kSmallDfaStates];
    if (*(volatile uint32_t *)P.err & kErrCapacity) return;
    const uint32_t FULL = 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    uint8_t *tbl = s_tbl[wib];
    int tbl_dfa = -1;
    const uint32_t n_rw = *(volatile uint32_t *)P.n_rw;
    for (uint32_t r = blockIdx.x * (kComposeThreads / 32) + wib; r < n_rw;
         r += gridDim.x * (kComposeThreads / 32)) {
        const uint32_t x = P.rw_list[r];
        const uint4 ent = P.split_list[x];
        const uint32_t mb = ent.y, k = ent.z & 0xffffu, N = (ent.z >> 24) + 1u;
        const int d = (int)((ent.z >> 16) & 0xffu);
        const uint32_t word = *reinterpret_cast<const volatile uint32_t *>(P.maps + mb);
        const uint32_t jb = word >> 9, s_entry = word & 0xffu;
        int64_t len = 0, s0 = 0;
        ItemGeom g{0, 0, 0};
        if (checked_dfa(P.offsets, P.dfa_id, (int64_t)ent.x, P.n_dfas, P.total_bytes, P.err, &len, &s0,
                        P.multi_n) == d)
            g = item_geom(len, s0, (int)N, P.seg_len, P.base_mis);
        if (g.k != k || jb >= k) {   // offsets changed since the plan
            if (lane == 0) atomicOr(P.err, kErrCapacity);
            continue;
        }
        if (N > (uint32_t)kSmallDfaStates) {   // the warp re-walk maps at most 16 states
            if (lane == 0) rewalk_lane(P, g, s0, len, d, N, mb, k, jb, s_entry, ent.x, ent.w);
            __syncwarp();
            continue;
        }
        auto rewalk = [&](uint32_t jw, uint32_t s_in) {
            if (tbl_dfa != d) {   // this warp's copy of the automaton's byte map
                __syncwarp();
                const uint8_t *tm = P.tmaps + P.desc[d].tmap_off;
                for (uint32_t t = lane; t < 256 * N; t += 32) tbl[t] = tm[t];
                __syncwarp();
                tbl_dfa = d;
            }
            int64_t b0, b1;
            item_range(g, s0, len, jw, &b0, &b1);
            return warp_rewalk(tbl, N, P.data, b0, b1, s_in);
        };
        uint32_t s = s_entry < N ? rewalk(jb, s_entry) : 0xffu;
        for (uint32_t j0 = jb + 1; j0 < k && s < N; j0 += 32) {
            const uint32_t j = j0 + lane;
            const bool in = j < k;
            const uint32_t v = in ? (uint32_t)P.maps[mb + j] : 0u;
            uint32_t gs = v & 0xffu, f = (v >> 8) & 0xffu;
            for (;;) {
                uint32_t pf = __shfl_up_sync(FULL, f, 1);
                if (lane == 0) pf = s;
                const uint32_t bad = __ballot_sync(FULL, in && gs != pf);
                if (!bad) break;
                const int b = __ffs(bad) - 1;
                const uint32_t s_in = __shfl_sync(FULL, pf, b);
                const uint32_t s_out = s_in < N ? rewalk(j0 + (uint32_t)b, s_in) : s_in;
                if (lane == (uint32_t)b) {
                    gs = s_in;
                    f = s_out;
                }
            }
            s = __shfl_sync(FULL, f, (int)min(31u, k - 1 - j0));
        }
        if (lane == 0) {
            if (s < N) write_result(P, ent.x, s, ent.w);
            else atomicOr(P.err, kErrCapacity);   // records not written by this plan
        }
    }
}

}  // namespace trex

struct trex_dfa_set {
    int n_dfas = 0;
    int max_states = 0;
    std::vector<int32_t> n_states, starts;
    std::vector<int64_t> tmap_off, accept_off;
    std::vector<uint8_t> h_accepts;      // host copy for empty-batch answers
    std::vector<uint8_t> h_tmaps;        // host copy: K-gram eligibility
    int64_t tmap_bytes = 0;              // all byte maps (bytes)
    std::vector<trex::DfaDesc> h_desc;
    uint8_t *d_tmaps = nullptr;
    uint8_t *d_accepts = nullptr;
    trex::DfaDesc *d_desc = nullptr;
    void *own_scratch = nullptr;
    size_t own_scratch_bytes = 0;
    int n_sms = 0;
    int device = -1;   // the set's tables live on this device
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

// Batch run; multi: every string against every automaton of the set (n
// strings give n * n_dfas results, automaton-major; dfa_id unused).
static int dfa_set_run_ex(trex_dfa_set *set, const uint8_t *data, const int64_t *offsets,
                          const int32_t *dfa_id, int64_t n_strings, int64_t total_bytes,
                          uint8_t *final_state, uint8_t *accept, int32_t *accept_i32, void *scratch,
                          int64_t scratch_bytes, int32_t seg_len, cudaStream_t stream,
                          uint32_t **err_word_out, bool multi) {
    if (!set) return TREX_ERR_NOT_INIT;
    if (n_strings < 0 || total_bytes < 0 || (n_strings > 0 && !offsets) || (total_bytes > 0 && !data))
        return TREX_ERR_ARG;
    {   // the kernels read the set's tables: they must run on the set's device
        int dev = -1;
        TREX_CUDA(cudaGetDevice(&dev));
        if (dev != set->device) {
            set_last_error_msg("trex_dfa_batch: the current device is not the device the set was created on");
            return TREX_ERR_ARG;
        }
    }
    const int64_t multi_n = multi ? n_strings : 0;
    const int64_t n = multi ? n_strings * set->n_dfas : n_strings;   // strings walked
    if (n >= (int64_t)0x7fffffff) return TREX_ERR_CAPACITY;
    seg_len = effective_seg_len(seg_len);
    if (n == 0) return TREX_OK;
    // bytes walked: every byte once per automaton in a multi-pattern run
    const int64_t walked = multi ? total_bytes * set->n_dfas : total_bytes;
    ScratchLayout L = scratch_layout(n, walked, seg_len);
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
    } else if ((size_t)scratch_bytes < L.total || ((uintptr_t)scratch & 15u) != 0) {
        return TREX_ERR_ARG;   // too small, or not 16-byte aligned (records are 128-bit accesses)
    }
    uint32_t *q_count = reinterpret_cast<uint32_t *>(sc + L.q_count);
    uint32_t *q_base = reinterpret_cast<uint32_t *>(sc + L.q_base);
    uint32_t *q_head = reinterpret_cast<uint32_t *>(sc + L.q_head);
    auto *q_bytes = reinterpret_cast<unsigned long long *>(sc + L.q_bytes);
    uint32_t *err = reinterpret_cast<uint32_t *>(sc + L.err);
    auto *n_items = reinterpret_cast<unsigned long long *>(sc + L.n_items);
    WorkItem *items = reinterpret_cast<WorkItem *>(sc + L.items);
    uint64_t *maps = reinterpret_cast<uint64_t *>(sc + L.maps);
    uint4 *split_list = reinterpret_cast<uint4 *>(sc + L.split_list);
    uint32_t *cta_bins = reinterpret_cast<uint32_t *>(sc + L.cta_bins);
    uint32_t *bin_base = reinterpret_cast<uint32_t *>(sc + L.bin_base);
    uint32_t *bin_end = reinterpret_cast<uint32_t *>(sc + L.bin_end);
    uint32_t *cta_maps = reinterpret_cast<uint32_t *>(sc + L.cta_maps);
    uint32_t *cta_splits = reinterpret_cast<uint32_t *>(sc + L.cta_splits);
    const uint32_t base_mis = (uint32_t)((uintptr_t)data & 31u);

    // Queue bases, counts and heads, byte counts, the error word and the item
    // count are contiguous at the front of the scratch buffer.
    TREX_CUDA(cudaMemsetAsync(sc, 0, L.items, stream));
    const int plan_grid = (int)std::min<int64_t>({(n + kPlanThreads - 1) / kPlanThreads,
                                                  (int64_t)set->n_sms, (int64_t)kMaxPlanCtas});
    plan_count_kernel<<<plan_grid, kPlanThreads, 0, stream>>>(
        offsets, dfa_id, n, total_bytes, set->d_desc, set->n_dfas, seg_len, base_mis, multi_n,
        cta_bins, cta_maps, cta_splits, n_items, err);
    TREX_CHECK_LAUNCH();
    {
        const int n_bins = set->n_dfas * kLenClasses;
        const int prefix_grid = (n_bins * kPrefixParts + kPrefixThreads - 1) / kPrefixThreads;
        plan_prefix_kernel<<<prefix_grid, kPrefixThreads, 0, stream>>>(cta_bins, bin_end, plan_grid, n_bins);
        TREX_CHECK_LAUNCH();
    }
    plan_scan_kernel<<<1, kPlanThreads, 0, stream>>>(cta_bins, bin_base, bin_end, cta_maps, cta_splits,
                                                     plan_grid,
                                                     set->n_dfas, q_base, q_count, q_bytes, n_items,
                                                     L.max_items, err);
    TREX_CHECK_LAUNCH();
    plan_fill_kernel<<<plan_grid, kPlanThreads, 0, stream>>>(
        offsets, dfa_id, n, total_bytes, set->d_desc, set->n_dfas, seg_len, base_mis, multi_n,
        cta_bins, bin_base, bin_end, cta_maps, cta_splits, items, L.max_items, split_list, err);
    TREX_CHECK_LAUNCH();

    RaggedParams P;
    P.data = data;
    P.total_bytes = total_bytes;
    P.offsets = offsets;
    P.tmaps = set->d_tmaps;
    P.accepts = set->d_accepts;
    P.desc = set->d_desc;
    P.n_dfas = set->n_dfas;
    P.seg_len = seg_len;
    P.items = items;
    P.q_base = q_base;
    P.q_count = q_count;
    P.q_head = q_head;
    P.q_serve = reinterpret_cast<uint32_t *>(sc + L.q_serve);
    P.q_bytes = q_bytes;
    P.err = err;
    P.maps = maps;
    P.split_list = split_list;
    P.n_split = cta_splits + plan_grid;
    P.fix_list = reinterpret_cast<uint2 *>(sc + L.fix_list);
    P.fix_cap = (uint32_t)std::min<int64_t>(L.fix_cap, 0xffffffffLL);
    P.fix_tm_bytes = set->tmap_bytes <= kFixSmemBytes ? (uint32_t)set->tmap_bytes : 0u;
    P.n_fix = reinterpret_cast<uint32_t *>(sc + L.n_fix);
    P.rw_list = reinterpret_cast<uint32_t *>(sc + L.rw_list);
    P.n_rw = reinterpret_cast<uint32_t *>(sc + L.n_rw);
    P.dfa_id = dfa_id;
    P.n = n;
    P.max_items = L.max_items;
    P.base_mis = base_mis;
    P.multi_n = multi_n;
    P.final_state = final_state;
    P.accept = accept;
    P.accept_i32 = accept_i32;
    profile_kernel_begin(stream);
    // one CTA per 64 KiB of input (and at least one per automaton the batch may
    // use), at most one per SM: a small batch (a serving batch) then needs a few
    // SMs and is not held back by other kernels running beside it; CTAs take
    // work from the queues, so fewer CTAs just do more
    const int ragged_grid = (int)std::min<int64_t>(
        set->n_sms, std::max<int64_t>({(int64_t)1, (walked + (64 << 10) - 1) >> 16,
                                       std::min<int64_t>(n, set->n_dfas)}));
    dfa_ragged_kernel<<<ragged_grid, kRaggedThreads, set->smem_bytes, stream>>>(P);
    TREX_CHECK_LAUNCH();
    profile_kernel_end(stream);
    // chaining split strings: a thread per string, then per fix-up task, then a warp per
    // string to walk again (the last two read their counts on the device)
    compose_chain_kernel<<<(int)std::min<int64_t>((n + kComposeThreads - 1) / kComposeThreads,
                                                  (int64_t)set->n_sms * 4),
                           kComposeThreads, 0, stream>>>(P);
    TREX_CHECK_LAUNCH();
    compose_fix_kernel<<<set->n_sms * 2, kComposeThreads, P.fix_tm_bytes, stream>>>(P);
    TREX_CHECK_LAUNCH();
    compose_rewalk_kernel<<<set->n_sms * 2, kComposeThreads, 0, stream>>>(P);
    TREX_CHECK_LAUNCH();
    if (err_word_out) *err_word_out = err;
    return TREX_OK;
}

int dfa_set_run(trex_dfa_set *set, const uint8_t *data, const int64_t *offsets,
                const int32_t *dfa_id, int64_t n, int64_t total_bytes, uint8_t *final_state,
                uint8_t *accept, int32_t *accept_i32, void *scratch, int64_t scratch_bytes,
                int32_t seg_len, cudaStream_t stream, uint32_t **err_word_out) {
    return dfa_set_run_ex(set, data, offsets, dfa_id, n, total_bytes, final_state, accept,
                          accept_i32, scratch, scratch_bytes, seg_len, stream, err_word_out, false);
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
    set->h_tmaps.assign(tmaps, tmaps + tsum);
    set->tmap_bytes = tsum;
    set->h_desc = desc;
    set->n_sms = trex::sm_count();
    if (set->n_sms <= 0 || cudaGetDevice(&set->device) != cudaSuccess) {
        cudaGetLastError();
        delete set;
        trex::set_last_error_msg("trex_dfa_set_create: no CUDA device");
        return TREX_ERR_SHAPE;
    }
    // table region, sized for the largest layout, and the K-gram fallback table
    set->smem_bytes = (size_t)trex::kRaggedSmemBytes;
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
    // The attribute is per kernel, so it is always raised to what any set can
    // need (the largest tables and the threads' work items).
    if ((e = cudaFuncSetAttribute(trex::dfa_ragged_kernel,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  trex::kRaggedSmemBytes)) != cudaSuccess)
        return fail(e, "cudaFuncSetAttribute");
    if ((e = cudaFuncSetAttribute(trex::compose_fix_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)trex::kFixSmemBytes)) != cudaSuccess)
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

}  // extern "C"

namespace trex {
int dfa_set_table(const trex_dfa_set *set, int index, int *n_states, int *start,
                  const uint8_t **tmap, const uint8_t **accept, int *n_sms) {
    if (!set) return TREX_ERR_NOT_INIT;
    if (index < 0 || index >= set->n_dfas) return TREX_ERR_ARG;
    *n_states = set->n_states[index];
    *start = set->starts[index];
    *tmap = set->d_tmaps + set->tmap_off[index];
    *accept = set->d_accepts + set->accept_off[index];
    *n_sms = set->n_sms;
    return TREX_OK;
}
}  // namespace trex

extern "C" {

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

int trex_dfa_batch_run_multi(trex_dfa_set *set, const uint8_t *data, const int64_t *offsets,
                             int64_t n_strings, int64_t total_bytes, uint8_t *final_state,
                             uint8_t *accept, int32_t *accept_i32, void *scratch,
                             int64_t scratch_bytes, int32_t seg_len, void *stream) {
    return trex::dfa_set_run_ex(set, data, offsets, nullptr, n_strings, total_bytes, final_state,
                                accept, accept_i32, scratch, scratch_bytes, seg_len,
                                static_cast<cudaStream_t>(stream), nullptr, true);
}

}  // extern "C"

// ---- batch with statically allocated scratch ------------------------------------------------
// For callers that cannot allocate device memory while they run -- a process
// whose memory is owned by another allocator, a real-time loop that must not
// call into the driver's allocator (cudaMalloc / cudaFree can synchronise the
// device) -- the scratch of trex_dfa_batch_run_static lives in this
// file-scope device array instead of a cudaMalloc'd buffer. Every GPU that
// loads the library holds the array until the process exits. All calls on a
// device share it, so calls whose work overlaps on the GPU race.
namespace trex {

constexpr int64_t kStaticScratchBytes = 8ll << 20;   // 8 MiB per GPU
constexpr int kMaxStaticDevices = 64;

static __device__ __align__(256) uint8_t g_static_scratch[kStaticScratchBytes];

// Device address of g_static_scratch on each device, looked up once per device
// and CUDA context (in host code the symbol name is only a stand-in, not a
// device address). The cache is keyed on the context's unique id as well as
// the device ordinal: after cudaDeviceReset the primary context, and with it
// the module that holds the array, is made again, and the address is looked up
// again.
struct StaticScratchSlot {
    unsigned long long ctx_id = 0;
    void *ptr = nullptr;
};
static StaticScratchSlot g_static_scratch_slot[kMaxStaticDevices];
static std::mutex g_static_scratch_mu;

// The driver's context calls are reached through the runtime's entry-point
// query, so the library keeps loading without libcuda (CPU-only hosts).
static int current_context_id(unsigned long long *id) {
    using GetCurrent = CUresult (*)(CUcontext *);
    using GetId = CUresult (*)(CUcontext, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    if (!get_current || !get_id) {
        void *a = nullptr, *b = nullptr;
        cudaDriverEntryPointQueryResult qa, qb;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) != cudaSuccess ||
            cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) != cudaSuccess ||
            qa != cudaDriverEntryPointSuccess || qb != cudaDriverEntryPointSuccess || !a || !b) {
            cudaGetLastError();
            return TREX_ERR_CUDA;
        }
        get_current = reinterpret_cast<GetCurrent>(a);
        get_id = reinterpret_cast<GetId>(b);
    }
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return TREX_ERR_CUDA;
    return get_id(ctx, id) == CUDA_SUCCESS ? TREX_OK : TREX_ERR_CUDA;
}

static int static_scratch_address(const trex_dfa_set *set, void **out) {
    int dev = 0;
    TREX_CUDA(cudaGetDevice(&dev));
    if (dev != set->device) {
        set_last_error_msg("trex_dfa_batch_run_static: the current device is not the device the set "
                           "was created on");
        return TREX_ERR_ARG;
    }
    if (dev < 0 || dev >= kMaxStaticDevices) {
        set_last_error_msg("trex_dfa_batch_run_static: device ordinal out of range");
        return TREX_ERR_SHAPE;
    }
    std::lock_guard<std::mutex> lock(g_static_scratch_mu);
    StaticScratchSlot &slot = g_static_scratch_slot[dev];
    unsigned long long id = 0;
    // no context current yet on this thread: the lookup below makes the primary one current
    const bool known = current_context_id(&id) == TREX_OK;
    if (!known || slot.ptr == nullptr || slot.ctx_id != id) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || !p) {
            set_last_error("trex_dfa_batch_run_static: cudaGetSymbolAddress", e);
            return TREX_ERR_CUDA;
        }
        if (current_context_id(&id) != TREX_OK) {
            set_last_error_msg("trex_dfa_batch_run_static: no current CUDA context");
            return TREX_ERR_CUDA;
        }
        slot.ptr = p;
        slot.ctx_id = id;
    }
    *out = slot.ptr;
    return TREX_OK;
}

}  // namespace trex

extern "C" int trex_dfa_batch_run_static(trex_dfa_set *set, const uint8_t *data,
                                         const int64_t *offsets, const int32_t *dfa_id,
                                         int64_t n_strings, int64_t total_bytes,
                                         uint8_t *final_state, uint8_t *accept,
                                         int32_t *accept_i32, int32_t seg_len, void *stream) {
    if (!set) return TREX_ERR_NOT_INIT;
    if (n_strings < 0 || total_bytes < 0) return TREX_ERR_ARG;
    const int64_t need = (int64_t)trex::scratch_layout(n_strings, total_bytes, seg_len).total;
    if (need > trex::kStaticScratchBytes) {
        trex::set_last_error_msg(
            "trex_dfa_batch_run_static: batch needs more than the 8 MiB static scratch; "
            "use trex_dfa_batch_run with a caller-provided scratch buffer");
        return TREX_ERR_CAPACITY;
    }
    void *scratch = nullptr;
    const int rc = trex::static_scratch_address(set, &scratch);
    if (rc) return rc;
    // dfa_set_run clears the counters at the front of the scratch before use
    // and writes every item / map slot before reading it.
    return trex::dfa_set_run(set, data, offsets, dfa_id, n_strings, total_bytes, final_state,
                             accept, accept_i32, scratch, trex::kStaticScratchBytes, seg_len,
                             static_cast<cudaStream_t>(stream), nullptr);
}

extern "C" int trex_dfa_batch_static_error(trex_dfa_set *set, int32_t *err_out) {
    // Reads the error word of the last trex_dfa_batch_run_static on the set's
    // device straight from the static array (a copy from the symbol, no
    // allocation); synchronises with the device.
    if (!set) return TREX_ERR_NOT_INIT;
    if (!err_out) return TREX_ERR_ARG;
    int dev = 0;
    TREX_CUDA(cudaGetDevice(&dev));
    if (dev != set->device) {
        trex::set_last_error_msg("trex_dfa_batch_static_error: the current device is not the device "
                                 "the set was created on");
        return TREX_ERR_ARG;
    }
    const trex::ScratchLayout L = trex::scratch_layout(0, 0, 0);
    uint32_t v = 0;
    TREX_CUDA(cudaMemcpyFromSymbol(&v, trex::g_static_scratch, sizeof(v), L.err, cudaMemcpyDeviceToHost));
    *err_out = (int32_t)v;
    return TREX_OK;
}

// ---- K-gram walking ---------------------------------------------------------------------------
namespace trex {

// The K-gram form of automaton d: its distinguished bytes are those whose
// column (next state of every state) differs from the most common column;
// they get codes (b >> sh) & (2^bits - 1) for the smallest bits in {1, 2, 4}
// and shift sh that keep them apart. Returns the largest K (2^bits)^K <= 256
// allows, or 1 when the automaton has more than 16 states or more than 16
// distinguished bytes, or no shift separates them.
static int kgram_plan(const trex_dfa_set *set, int d, DfaDesc *out) {
    const int N = set->n_states[d];
    if (N > kSmallDfaStates) return 1;
    const uint8_t *t = set->h_tmaps.data() + set->tmap_off[d];
    auto same = [&](int a, int b) { return std::memcmp(t + a * N, t + b * N, N) == 0; };
    // the most common column
    int other = 0, best = 0;
    std::vector<int> cls(256, -1);
    for (int b = 0; b < 256; ++b) {
        if (cls[b] >= 0) continue;
        int cnt = 0;
        for (int c = b; c < 256; ++c)
            if (cls[c] < 0 && same(b, c)) {
                cls[c] = b;
                ++cnt;
            }
        if (cnt > best) { best = cnt; other = b; }
    }
    std::vector<int> letters;
    for (int b = 0; b < 256; ++b)
        if (cls[b] != cls[other]) letters.push_back(b);
    const int sigma = (int)letters.size();
    if (sigma < 1 || sigma > 16) return 1;
    for (int bits : {1, 2, 4}) {
        if (sigma > (1 << bits)) continue;
        for (int sh = 0; sh + bits <= 8; ++sh) {
            const int mask = (1 << bits) - 1;
            std::vector<int> owner(1 << bits, -1);
            bool ok = true;
            for (int b : letters) {
                const int c = (b >> sh) & mask;
                if (owner[c] >= 0) { ok = false; break; }
                owner[c] = b;
            }
            if (!ok) continue;
            DfaDesc D = set->h_desc[d];
            D.kbits = bits;
            D.kshift = sh;
            uint8_t alpha[16];
            for (int c = 0; c < 16; ++c) {
                // an unused code's letter is a byte of another code: no input byte matches it
                const int code_other = (c ^ 1) & mask;
                alpha[c] = owner[c & mask] >= 0 && c <= mask ? (uint8_t)owner[c] : (uint8_t)(code_other << sh);
                if (c <= mask) D.krep[c] = owner[c] >= 0 ? (uint8_t)owner[c] : (uint8_t)other;
            }
            D.krep[1 << bits] = (uint8_t)other;
            std::memcpy(D.kalpha, alpha, 16);
            *out = D;
            return 8 / bits;
        }
    }
    return 1;
}

}  // namespace trex

extern "C" {

int trex_dfa_kgram_max(const trex_dfa_set *set, int dfa_index, int *k_max) {
    if (!set || !k_max || dfa_index < 0 || dfa_index >= set->n_dfas) return TREX_ERR_ARG;
    trex::DfaDesc D{};
    *k_max = trex::kgram_plan(set, dfa_index, &D);
    return TREX_OK;
}

int trex_dfa_set_kgram(trex_dfa_set *set, int dfa_index, int k) {
    if (!set || dfa_index < 0 || dfa_index >= set->n_dfas) return TREX_ERR_ARG;
    if (k < 0 || (k > 1 && k != 2 && k != 4 && k != 8)) return TREX_ERR_ARG;
    trex::DfaDesc D = set->h_desc[dfa_index];
    if (k != 1) {
        trex::DfaDesc P{};
        const int kmax = trex::kgram_plan(set, dfa_index, &P);
        if (k == 0) k = kmax;
        if (k > kmax) {
            trex::set_last_error_msg("trex_dfa_set_kgram: the automaton does not allow this K");
            return TREX_ERR_SHAPE;
        }
        if (k > 1) D = P;
    }
    D.kgram = k > 1 ? k : 1;
    if (D.kgram == 1) {
        D.kbits = D.kshift = 0;
    }
    TREX_CUDA(cudaMemcpy(set->d_desc + dfa_index, &D, sizeof(D), cudaMemcpyHostToDevice));
    set->h_desc[dfa_index] = D;
    return TREX_OK;
}

int trex_dfa_get_kgram(const trex_dfa_set *set, int dfa_index, int *k) {
    if (!set || !k || dfa_index < 0 || dfa_index >= set->n_dfas) return TREX_ERR_ARG;
    *k = set->h_desc[dfa_index].kgram;
    return TREX_OK;
}

}  // extern "C"
