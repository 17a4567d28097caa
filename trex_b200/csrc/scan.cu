// Family (b): per-position DFA states of long strings, one persistent launch,
// single pass with a decoupled look-back between warp chunks.
//
// Semantics (reference src/simulation.py:142-153 prefix_scan_sequential):
// out[p] is the state after byte p of its string, i.e. argmax of
// (T[p] ... T[start of string]) applied to the start vector; through the byte
// map this is out[p] = tmap[byte[p] * N + out[p - 1]] with the DFA start
// state before the first byte. Also writes the final state and accept flag of
// every string.
//
// Design (N <= 16; the per-lane replicated table of dfa_walk.cuh)
//  * Strings are cut into tiles of tile_len bytes; a warp takes 32
//    consecutive tiles (a chunk) with one atomic.
//  * Sync: every lane walks all 16 states of its tile together (16
//    independent chains) until they coincide, at the same byte offset S for
//    the whole warp. From there the tile's states no longer depend on its
//    entry state: its map is constant. A tile that starts a string begins in
//    the start state and needs no sync.
//  * Body: each lane walks bytes [tile + S, tile end) with one chain and
//    writes every state (16-byte stores of packed states).
//  * Entry states: inside the warp, the entry of tile i is the exit of tile
//    i-1 (a shuffle scan over tile maps handles the general case). Across
//    warps, chunk c publishes its composed map (AGGREGATE) as soon as its body
//    is walked and its exit state (PREFIX) once its entry is known; chunk c
//    looks back over c-1, c-2, ... composing aggregates until it meets a
//    prefix (or a constant map). Every poll is bounded; a wait that runs out
//    sets the error word and the chunk gives up.
//  * Head: with the entry state known, each lane walks bytes [tile,
//    tile + S) again from it and writes those states.
//  * Tiles whose 16 states never coincide (automata that do not
//    synchronise) keep all 16 chains over the whole tile, publish the full
//    map and are walked again from their true entry state.
#include <algorithm>
#include <cstring>

#include "dfa_walk.cuh"

namespace trex {

constexpr int kScanThreads = 1024;
constexpr int kSyncCap = 512;                 // bytes walked with 16 chains before giving up

enum : uint32_t { kStAgg = 1u, kStPrefix = 2u };
enum : uint32_t { kScanErrOffsets = 1u, kScanErrTimeout = 4u, kScanErrCapacity = 8u };

// Tile length: the requested one (>= 64), or by default the length that gives
// every resident warp one 32-tile chunk (1 KiB multiples, 1 KiB .. 64 KiB).
static int32_t scan_tile_len(int32_t tile_len, int64_t total_bytes, int n_sms) {
    if (tile_len > 0) return tile_len < 64 ? 64 : tile_len;
    const int64_t warps = (int64_t)(n_sms > 0 ? n_sms : 148) * (kScanThreads / 32);
    int64_t t = total_bytes / (warps * 32);
    t = ((t + 1023) / 1024) * 1024;
    return (int32_t)std::min<int64_t>(65536, std::max<int64_t>(1024, t));
}

struct ScanScratch {
    size_t tile_base, chunk_status, chunk_map, head, err, total;
};

static ScanScratch scan_layout(int64_t n_strings, int64_t total_bytes, int32_t tile) {
    ScanScratch L{};
    const int64_t max_tiles = n_strings + total_bytes / tile + 1;
    const int64_t chunks = max_tiles / 32 + 2;
    size_t o = 0;
    auto take = [&](size_t b) { size_t at = o; o = (o + b + 255) & ~size_t(255); return at; };
    L.tile_base = take((size_t)(n_strings + 1) * 8);
    L.chunk_status = take((size_t)chunks * 4);
    L.chunk_map = take((size_t)chunks * 8);
    L.head = take(8);
    L.err = take(4);
    L.total = o;
    return L;
}

// tile_base[i] = number of tiles of strings 0..i-1 (single block, sequential
// per thread chunk then a block scan; fine for the few long strings this path
// is for, and correct for any count). The chunk buffers hold max_tiles tiles,
// enough for well-formed offsets; overlapping offsets that need more set the
// capacity bit and leave zero tiles, so the scan kernel touches nothing.
// Sums saturate at max_tiles + 1 so that they cannot wrap.
__global__ void scan_tile_base_kernel(const int64_t *offsets, int64_t n, int64_t total_bytes,
                                      int32_t tile, int64_t max_tiles, int64_t *tile_base,
                                      uint32_t *err) {
    __shared__ int64_t part[1024];
    __shared__ bool over;
    const int64_t per = (n + blockDim.x - 1) / blockDim.x;
    const int64_t lo = threadIdx.x * per, hi = min(n, lo + per);
    int64_t sum = 0;
    for (int64_t i = lo; i < hi; ++i) {
        const int64_t a = offsets[i], b = offsets[i + 1];
        if (a < 0 || b < a || b > total_bytes) {
            atomicOr(err, kScanErrOffsets);
            continue;
        }
        sum = min(sum + (b - a + tile - 1) / tile, max_tiles + 1);
    }
    part[threadIdx.x] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t run = 0;
        for (int t = 0; t < (int)blockDim.x; ++t) {
            const int64_t v = part[t];
            part[t] = run;
            run = min(run + v, max_tiles + 1);
        }
        over = run > max_tiles;
        if (over) atomicOr(err, kScanErrCapacity);
    }
    __syncthreads();
    if (over) {
        for (int64_t i = lo; i < hi; ++i) tile_base[i] = 0;
        if (threadIdx.x == 0) tile_base[n] = 0;
        return;
    }
    int64_t run = part[threadIdx.x];
    for (int64_t i = lo; i < hi; ++i) {
        tile_base[i] = run;
        const int64_t a = offsets[i], b = offsets[i + 1];
        if (!(a < 0 || b < a || b > total_bytes)) run += (b - a + tile - 1) / tile;
    }
    if (hi == n && lo < n) tile_base[n] = run;
    if (n == 0 && threadIdx.x == 0) tile_base[0] = 0;
}

// Empty strings have no tile: their final state is the start state.
__global__ void scan_empty_kernel(const int64_t *offsets, int64_t n, int start,
                                  const uint8_t *accept, uint8_t *final_state, uint8_t *acc) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        if (offsets[i + 1] == offsets[i]) {
            if (final_state) final_state[i] = (uint8_t)start;
            if (acc) acc[i] = accept[start];
        }
}

// ---- nibble maps (16 states x 4 bits) ----------------------------------------------
__device__ __forceinline__ uint32_t map_at(uint64_t m, uint32_t s) {
    return (uint32_t)(m >> (4 * s)) & 15u;
}
// (g after f)(s) = g(f(s))
__device__ __forceinline__ uint64_t map_then(uint64_t f, uint64_t g) {
    uint64_t r = 0;
#pragma unroll
    for (int s = 0; s < 16; ++s) r |= (uint64_t)map_at(g, map_at(f, s)) << (4 * s);
    return r;
}
__device__ __forceinline__ uint64_t map_const(uint32_t s) { return (uint64_t)s * 0x1111111111111111ull; }
__device__ __forceinline__ bool map_is_const(uint64_t m) { return m == map_const((uint32_t)m & 15u); }
constexpr uint64_t kMapIdentity = 0xFEDCBA9876543210ull;

struct ScanParams {
    const uint8_t *data;
    int64_t total_bytes;
    const int64_t *offsets;
    int64_t n_strings;
    const int64_t *tile_base;
    int32_t tile;
    int n_states;
    int start;
    const uint8_t *tmap;
    const uint8_t *accept_tbl;
    uint8_t *out;
    uint8_t *final_state;
    uint8_t *accept;
    uint32_t *chunk_status;
    uint64_t *chunk_map;
    unsigned long long *head;
    uint32_t *err;
    uint32_t poll_limit;   // polls of one look-back step before giving up
};

// Decodes four encoded states packed in a word into four plain states.
template <class W> __device__ __forceinline__ uint32_t dec4(uint32_t w4);
template <> __device__ __forceinline__ uint32_t dec4<Walker<8>>(uint32_t w4) {
    return (w4 & 0x03030303u) | ((w4 >> 5) & 0x04040404u);
}
template <> __device__ __forceinline__ uint32_t dec4<Walker<16>>(uint32_t w4) {
    return (w4 & 0x03030303u) | ((w4 >> 4) & 0x0C0C0C0Cu);
}

// Walks a 16-byte vector, returns the 16 decoded states packed in a uint4.
template <class W>
__device__ __forceinline__ uint4 walk16_states(const W &w, uint32_t &e, uint4 v) {
    uint32_t o[4];
    const uint32_t x[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint32_t e0 = w.template step<0>(e, x[k]);
        const uint32_t e1 = w.template step<1>(e0, x[k]);
        const uint32_t e2 = w.template step<2>(e1, x[k]);
        const uint32_t e3 = w.template step<3>(e2, x[k]);
        e = e3;
        o[k] = dec4<W>(e0 | (e1 << 8) | (e2 << 16) | (e3 << 24));
    }
    return make_uint4(o[0], o[1], o[2], o[3]);
}

// Walks bytes [p, end) from encoded state e and writes every state to out.
template <class W>
__device__ uint32_t walk_write(const W &w, const ScanParams &P, int64_t p, int64_t end, uint32_t e) {
    const uint8_t *data = P.data;
    uint8_t *out = P.out;
    // head bytes up to 16-byte alignment of the input
    while (p < end && (((uintptr_t)(data + p)) & 15u)) {
        e = w.template step<0>(e, (uint32_t)__ldg(data + p));
        out[p] = (uint8_t)W::dec(e);
        ++p;
    }
    const bool out_aligned = (((uintptr_t)(out + p)) & 15u) == 0;
    auto emit = [&](int64_t q, uint4 st) {
        if (out_aligned) {
            st_stream16(out + q, st);
        } else {
            const uint32_t sw[4] = {st.x, st.y, st.z, st.w};
#pragma unroll
            for (int j = 0; j < 16; ++j) out[q + j] = (uint8_t)(sw[j >> 2] >> (8 * (j & 3)));
        }
    };
    // 32-byte alignment for the vector-8 loads
    if (end - p >= 16 && (((uintptr_t)(data + p)) & 31u)) {
        emit(p, walk16_states(w, e, ld_stream16(data + p)));
        p += 16;
    }
    // 64-byte blocks, the next block in flight, the L2 one 256-byte block ahead
    if (end - p >= 64) {
        // data + p is 32-byte aligned here; so is out + p when out and data share it
        const bool out32 = (((uintptr_t)(out + p)) & 31u) == 0;
        uint4 a0, a1, a2, a3;
        ld_stream32(data + p, a0, a1);
        ld_stream32(data + p + 32, a2, a3);
        while (true) {
            const bool more = end - p >= 128;
            uint4 b0 = make_uint4(0, 0, 0, 0), b1 = b0, b2 = b0, b3 = b0;
            if (more) {
                ld_stream32(data + p + 64, b0, b1);
                ld_stream32(data + p + 96, b2, b3);
                if ((((uintptr_t)(data + p)) & 255u) == 0 && end - p >= 512)
                    prefetch_l2(data + p + 256);
            }
            if (out32) {   // two 16-state words a store: half the store instructions
                const uint4 s0 = walk16_states(w, e, a0);
                const uint4 s1 = walk16_states(w, e, a1);
                st_stream32(out + p, s0, s1);
                const uint4 s2 = walk16_states(w, e, a2);
                const uint4 s3 = walk16_states(w, e, a3);
                st_stream32(out + p + 32, s2, s3);
            } else {
                emit(p, walk16_states(w, e, a0));
                emit(p + 16, walk16_states(w, e, a1));
                emit(p + 32, walk16_states(w, e, a2));
                emit(p + 48, walk16_states(w, e, a3));
            }
            p += 64;
            if (!more) break;
            a0 = b0;
            a1 = b1;
            a2 = b2;
            a3 = b3;
        }
    }
    while (end - p >= 16) {
        emit(p, walk16_states(w, e, ld_stream16(data + p)));
        p += 16;
    }
    while (p < end) {
        e = w.template step<0>(e, (uint32_t)__ldg(data + p));
        out[p] = (uint8_t)W::dec(e);
        ++p;
    }
    return e;
}

// Tile geometry: string, first byte, end, whether it starts / ends the string.
struct TileInfo {
    int64_t str, b0, b1;
    bool first, last;
};

__device__ __forceinline__ TileInfo locate_tile(const ScanParams &P, int64_t t) {
    // largest string index s with tile_base[s] <= t (strings without tiles are skipped)
    int64_t lo = 0, hi = P.n_strings;   // invariant: tile_base[lo] <= t < tile_base[hi]
    while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (P.tile_base[mid] <= t) lo = mid;
        else hi = mid;
    }
    TileInfo ti;
    ti.str = lo;
    const int64_t k = t - P.tile_base[lo];
    const int64_t s0 = P.offsets[lo], s1 = P.offsets[lo + 1];
    ti.b0 = s0 + k * P.tile;
    ti.b1 = min(s1, ti.b0 + (int64_t)P.tile);
    ti.first = (k == 0);
    ti.last = (ti.b1 == s1);
    return ti;
}

template <class W>
__device__ void scan_chunk(const ScanParams &P, const W &w, int64_t chunk, int64_t n_tiles) {
    const uint32_t FULL = 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31u;
    const int64_t t = chunk * 32 + lane;
    const bool have = t < n_tiles;
    TileInfo ti{0, 0, 0, true, false};
    if (have) ti = locate_tile(P, t);
    // ---- sync: 16 chains until they coincide (same S for the whole warp)
    uint32_t ch[16];
#pragma unroll
    for (int j = 0; j < 16; ++j)
        ch[j] = w.enc(ti.first ? (uint32_t)P.start : (j < P.n_states ? (uint32_t)j : 0u));
    int64_t S = 0;
    const int64_t len = have ? ti.b1 - ti.b0 : 0;
    bool conv = true;
#pragma unroll
    for (int j = 1; j < 16; ++j) conv &= (ch[j] == ch[0]);
    while (!__all_sync(FULL, conv || S >= len) && S < kSyncCap) {
        for (int k = 0; k < 16; ++k) {
            if (S + k < len) {
                const uint32_t c = __ldg(P.data + ti.b0 + S + k);
#pragma unroll
                for (int j = 0; j < 16; ++j) ch[j] = w.template step<0>(ch[j], c);
            }
        }
        S += 16;
        conv = true;
#pragma unroll
        for (int j = 1; j < 16; ++j) conv &= (ch[j] == ch[0]);
    }
    if (S > len) S = len;
    // ---- body (converged) or full map (not converged)
    uint64_t map = kMapIdentity;
    uint32_t e = ch[0];
    if (have) {
        if (conv) {
            e = walk_write(w, P, ti.b0 + S, ti.b1, e);
            map = map_const(W::dec(e));
        } else {
            // does not synchronise: carry all 16 chains over the tile
            for (int64_t p = ti.b0 + S; p < ti.b1; ++p) {
                const uint32_t c = __ldg(P.data + p);
#pragma unroll
                for (int j = 0; j < 16; ++j) ch[j] = w.template step<0>(ch[j], c);
            }
            map = 0;
#pragma unroll
            for (int j = 0; j < 16; ++j) map |= (uint64_t)W::dec(ch[j]) << (4 * j);
            if (ti.first) map = map_const(map_at(map, (uint32_t)P.start));
        }
    }
    // ---- chunk aggregate: composition of the 32 tile maps, published at once
    uint64_t incl = map;   // inclusive scan: maps of lanes 0..lane applied in order
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t prev = __shfl_up_sync(FULL, incl, o);
        if (lane >= (uint32_t)o) incl = map_then(prev, incl);
    }
    const uint64_t agg = __shfl_sync(FULL, incl, 31);
    if (lane == 0) {
        P.chunk_map[chunk] = agg;
        __threadfence();
        st_release_u32(P.chunk_status + chunk, kStAgg);
    }
    // ---- look-back for the chunk's entry state (lane 0)
    uint32_t entry0 = (uint32_t)P.start;
    if (lane == 0) {
        uint64_t acc = kMapIdentity;   // maps of chunks (j, chunk) applied in order
        bool found = false;
        for (int64_t j = chunk - 1; j >= 0 && !found; --j) {
            uint32_t st = 0;
            uint32_t polls = 0;
            while (((st = ld_acquire_u32(P.chunk_status + j)) & 3u) == 0u) {
                if (++polls >= P.poll_limit) break;
                __nanosleep(64);
            }
            if ((st & 3u) == 0u) {
                atomicOr(P.err, kScanErrTimeout);
                break;
            }
            if (st & kStPrefix) {
                entry0 = map_at(acc, (st >> 8) & 15u);
                found = true;
            } else {
                acc = map_then(ld_relaxed_u64(P.chunk_map + j), acc);
                if (map_is_const(acc)) {
                    entry0 = (uint32_t)acc & 15u;
                    found = true;
                }
            }
        }
    }
    entry0 = __shfl_sync(FULL, entry0, 0);
    // entry of tile `lane` = (maps of lanes 0..lane-1)(entry0)
    const uint64_t excl = __shfl_up_sync(FULL, incl, 1);
    const uint32_t entry = ti.first ? (uint32_t)P.start : (lane == 0 ? entry0 : map_at(excl, entry0));
    // ---- publish the chunk's exit state
    const uint32_t chunk_exit = map_at(agg, entry0);
    if (lane == 0) st_release_u32(P.chunk_status + chunk, kStPrefix | (chunk_exit << 8));
    // ---- head (or whole tile when the states never coincided) from the true entry
    if (have) {
        uint32_t fin;
        if (conv) {
            walk_write(w, P, ti.b0, ti.b0 + S, w.enc(entry));
            fin = W::dec(e);   // body exit (independent of the entry)
        } else {
            fin = W::dec(walk_write(w, P, ti.b0, ti.b1, w.enc(entry)));
        }
        if (ti.last) {
            if (P.final_state) P.final_state[ti.str] = (uint8_t)fin;
            if (P.accept) P.accept[ti.str] = P.accept_tbl[fin];
        }
    }
}

__global__ void __launch_bounds__(kScanThreads, 1) dfa_scan_kernel(ScanParams P) {
    __shared__ unsigned long long s_chunk[kScanThreads / 32];
    build_table(P.tmap, P.n_states);
    __syncthreads();
    const int64_t n_tiles = P.tile_base[P.n_strings];
    const int64_t n_chunks = (n_tiles + 31) / 32;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    while (true) {
        if (lane == 0) s_chunk[warp] = atomicAdd(P.head, 1ull);
        __syncwarp();
        const int64_t chunk = (int64_t)s_chunk[warp];
        __syncwarp();
        if (chunk >= n_chunks) break;
        if (P.n_states <= 8) scan_chunk(P, Walker<8>{lane}, chunk, n_tiles);
        else scan_chunk(P, Walker<16>{lane}, chunk, n_tiles);
    }
}

}  // namespace trex

// Access to the resident tables of a DFA set (defined with the set).
namespace trex {
int dfa_set_table(const trex_dfa_set *set, int index, int *n_states, int *start,
                  const uint8_t **tmap, const uint8_t **accept, int *n_sms);
}

extern "C" {

int trex_dfa_scan_run(trex_dfa_set *set, int dfa_index, const uint8_t *data,
                      const int64_t *offsets, int64_t n_strings, int64_t total_bytes,
                      uint8_t *states, uint8_t *final_state, uint8_t *accept, void *scratch,
                      int64_t scratch_bytes, int32_t tile_len, void *stream_) {
    using namespace trex;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_);
    int N = 0, start = 0, n_sms = 0;
    const uint8_t *tmap = nullptr, *acc = nullptr;
    int rc = dfa_set_table(set, dfa_index, &N, &start, &tmap, &acc, &n_sms);
    if (rc) return rc;
    if (N > kSmallDfaStates) {
        set_last_error_msg("trex_dfa_scan_run: the per-position scan needs N <= 16");
        return TREX_ERR_SHAPE;
    }
    if (n_strings < 0 || total_bytes < 0 || (n_strings > 0 && !offsets) ||
        (total_bytes > 0 && (!data || !states)))
        return TREX_ERR_ARG;
    if (n_strings == 0) return TREX_OK;
    tile_len = scan_tile_len(tile_len, total_bytes, n_sms);
    const ScanScratch L = scan_layout(n_strings, total_bytes, tile_len);
    if (!scratch || scratch_bytes < (int64_t)L.total) {
        set_last_error_msg("trex_dfa_scan_run: scratch missing or too small");
        return TREX_ERR_ARG;
    }
    uint8_t *sc = static_cast<uint8_t *>(scratch);
    const int64_t max_tiles = n_strings + total_bytes / tile_len + 1;
    const int64_t chunks = max_tiles / 32 + 2;
    TREX_CUDA(cudaMemsetAsync(sc + L.chunk_status, 0, (size_t)chunks * 4, stream));
    TREX_CUDA(cudaMemsetAsync(sc + L.head, 0, 8, stream));
    TREX_CUDA(cudaMemsetAsync(sc + L.err, 0, 4, stream));
    int64_t *tile_base = reinterpret_cast<int64_t *>(sc + L.tile_base);
    uint32_t *err = reinterpret_cast<uint32_t *>(sc + L.err);
    scan_tile_base_kernel<<<1, 1024, 0, stream>>>(offsets, n_strings, total_bytes, tile_len,
                                                  max_tiles, tile_base, err);
    TREX_CHECK_LAUNCH();
    scan_empty_kernel<<<(int)std::min<int64_t>((n_strings + 255) / 256, 4096), 256, 0, stream>>>(
        offsets, n_strings, start, acc, final_state, accept);
    TREX_CHECK_LAUNCH();
    ScanParams P;
    P.data = data;
    P.total_bytes = total_bytes;
    P.offsets = offsets;
    P.n_strings = n_strings;
    P.tile_base = tile_base;
    P.tile = tile_len;
    P.n_states = N;
    P.start = start;
    P.tmap = tmap;
    P.accept_tbl = acc;
    P.out = states;
    P.final_state = final_state;
    P.accept = accept;
    P.chunk_status = reinterpret_cast<uint32_t *>(sc + L.chunk_status);
    P.chunk_map = reinterpret_cast<uint64_t *>(sc + L.chunk_map);
    P.head = reinterpret_cast<unsigned long long *>(sc + L.head);
    P.err = err;
    P.poll_limit = scan_poll_limit();
    static bool attr_set = false;
    if (!attr_set) {
        TREX_CUDA(cudaFuncSetAttribute(dfa_scan_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kRepTableBytes16));
        attr_set = true;
    }
    profile_kernel_begin(stream);
    dfa_scan_kernel<<<n_sms, kScanThreads, kRepTableBytes16, stream>>>(P);
    TREX_CHECK_LAUNCH();
    profile_kernel_end(stream);
    return TREX_OK;
}

int trex_dfa_scan_error(void *scratch, int64_t n_strings, int64_t total_bytes, int32_t tile_len,
                        int32_t *err_out) {
    using namespace trex;
    if (!scratch || !err_out) return TREX_ERR_ARG;
    tile_len = scan_tile_len(tile_len, total_bytes, sm_count());
    const ScanScratch L = scan_layout(n_strings, total_bytes, tile_len);
    uint32_t v = 0;
    TREX_CUDA(cudaMemcpy(&v, static_cast<uint8_t *>(scratch) + L.err, 4, cudaMemcpyDeviceToHost));
    *err_out = (int32_t)v;
    return TREX_OK;
}

int64_t trex_dfa_scan_scratch_bytes(int64_t n_strings, int64_t total_bytes, int32_t tile_len) {
    if (n_strings < 0 || total_bytes < 0) return -1;
    tile_len = trex::scan_tile_len(tile_len, total_bytes, trex::sm_count());
    return (int64_t)trex::scan_layout(n_strings, total_bytes, tile_len).total;
}

}  // extern "C"
