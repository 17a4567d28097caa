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
//  * Strings are cut into tiles of tile_len bytes; a warp takes two chunks of
//    32 consecutive tiles with one atomic, lane l tiles l and 32 + l.
//  * Sync: every lane walks all 16 states of its tile together (16
//    independent chains) until they coincide, at the same byte offset S for
//    the whole warp. From there the tile's states no longer depend on its
//    entry state: its map is constant. A tile that starts a string begins in
//    the start state and needs no sync.
//  * Body: each lane walks bytes [tile + S, tile end) of its two tiles as two
//    interleaved chains (two table lookups in flight; one chain a thread is
//    bound by the latency of its dependent lookups) and writes every state
//    (16-byte stores of packed states).
//  * Entry states: inside the warp, the entry of tile i is the exit of tile
//    i-1 (a shuffle scan over tile maps handles the general case). Across
//    warps, chunk c publishes its composed map (AGGREGATE) as soon as its body
//    is walked and its exit state (PREFIX) once its entry is known; chunk c
//    looks back over c-1, c-2, ... composing aggregates until it meets a
//    prefix (or a constant map). A warp publishes both its chunks' aggregates
//    before it looks back, and its second chunk's entry is its first one's exit. Every poll is bounded; a wait that runs out
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
// every resident warp one pair of 32-tile chunks (1 KiB multiples, 1 KiB .. 64 KiB).
static int32_t scan_tile_len(int32_t tile_len, int64_t total_bytes, int n_sms) {
    if (tile_len > 0) return tile_len < 64 ? 64 : tile_len;
    const int64_t warps = (int64_t)(n_sms > 0 ? n_sms : 148) * (kScanThreads / 32);
    int64_t t = total_bytes / (warps * 64);
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
            emit(p, walk16_states(w, e, a0));
            emit(p + 16, walk16_states(w, e, a1));
            emit(p + 32, walk16_states(w, e, a2));
            emit(p + 48, walk16_states(w, e, a3));
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

// Two chains over 16-byte vectors: the bytes of va and vb are applied to xa and
// xb alternately (two table lookups in flight), returns both 16 decoded states.
template <class W>
__device__ __forceinline__ void walk16_states2(const W &w, uint32_t &xa, uint4 va, uint4 &oa, uint32_t &xb,
                                               uint4 vb, uint4 &ob) {
    const uint32_t ya[4] = {va.x, va.y, va.z, va.w}, yb[4] = {vb.x, vb.y, vb.z, vb.w};
    uint32_t ra[4], rb[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint32_t a0 = w.template step<0>(xa, ya[k]), b0 = w.template step<0>(xb, yb[k]);
        const uint32_t a1 = w.template step<1>(a0, ya[k]), b1 = w.template step<1>(b0, yb[k]);
        const uint32_t a2 = w.template step<2>(a1, ya[k]), b2 = w.template step<2>(b1, yb[k]);
        const uint32_t a3 = w.template step<3>(a2, ya[k]), b3 = w.template step<3>(b2, yb[k]);
        xa = a3;
        xb = b3;
        ra[k] = dec4<W>(a0 | (a1 << 8) | (a2 << 16) | (a3 << 24));
        rb[k] = dec4<W>(b0 | (b1 << 8) | (b2 << 16) | (b3 << 24));
    }
    oa = make_uint4(ra[0], ra[1], ra[2], ra[3]);
    ob = make_uint4(rb[0], rb[1], rb[2], rb[3]);
}

// Walks bytes [pa, ea) from xa and [pb, eb) from xb and writes every state: each
// start is first brought to a 32-byte boundary alone, then 32 bytes of each per
// step as two interleaved chains (the next 32 bytes of each in flight), then the
// rests alone.
template <class W>
__device__ void walk_write2(const W &w, const ScanParams &P, int64_t pa, int64_t ea, uint32_t &xa,
                            int64_t pb, int64_t eb, uint32_t &xb) {
    const int64_t ha = min(ea, pa + (int64_t)((32u - ((uint32_t)(uintptr_t)(P.data + pa) & 31u)) & 31u));
    const int64_t hb = min(eb, pb + (int64_t)((32u - ((uint32_t)(uintptr_t)(P.data + pb) & 31u)) & 31u));
    xa = walk_write(w, P, pa, ha, xa);
    xb = walk_write(w, P, pb, hb, xb);
    pa = ha;
    pb = hb;
    const int64_t n = min(ea - pa, eb - pb) & ~(int64_t)31;
    const bool aligned = ((((uintptr_t)(P.data + pa)) | ((uintptr_t)(P.data + pb))) & 31u) == 0 &&
                         ((((uintptr_t)(P.out + pa)) | ((uintptr_t)(P.out + pb))) & 15u) == 0;
    if (aligned && n >= 32) {
        uint4 a0, a1, b0, b1;
        ld_stream32(P.data + pa, a0, a1);
        ld_stream32(P.data + pb, b0, b1);
        for (int64_t q = 0; q < n; q += 32) {
            uint4 na0 = make_uint4(0, 0, 0, 0), na1 = na0, nb0 = na0, nb1 = na0;
            if (q + 32 < n) {
                ld_stream32(P.data + pa + q + 32, na0, na1);
                ld_stream32(P.data + pb + q + 32, nb0, nb1);
                if (((q + 32) & 255) == 0 && q + 512 < n) {
                    prefetch_l2(P.data + pa + q + 288);
                    prefetch_l2(P.data + pb + q + 288);
                }
            }
            uint4 sa, sb;
            walk16_states2(w, xa, a0, sa, xb, b0, sb);
            st_stream16(P.out + pa + q, sa);
            st_stream16(P.out + pb + q, sb);
            walk16_states2(w, xa, a1, sa, xb, b1, sb);
            st_stream16(P.out + pa + q + 16, sa);
            st_stream16(P.out + pb + q + 16, sb);
            a0 = na0;
            a1 = na1;
            b0 = nb0;
            b1 = nb1;
        }
        pa += n;
        pb += n;
    }
    xa = walk_write(w, P, pa, ea, xa);
    xb = walk_write(w, P, pb, eb, xb);
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

// A tile after its sync: the byte S (the same for the warp) from which its map
// is constant (conv), the encoded state there; for a tile whose states never
// coincided (not conv) its full map, walked with all 16 chains.
struct TileSync {
    int64_t S;
    bool conv;
    uint32_t e;
    uint64_t map;
};

// Sync of one tile a lane: every lane walks all 16 states of its tile together
// (16 independent chains) until they coincide, at the same byte S for the whole
// warp. A tile that starts a string begins in the start state and needs none.
template <class W>
__device__ TileSync tile_sync(const ScanParams &P, const W &w, const TileInfo &ti, bool have) {
    const uint32_t FULL = 0xffffffffu;
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
    TileSync r{S, conv, ch[0], kMapIdentity};
    if (have && !conv) {
        // does not synchronise: carry all 16 chains over the tile
        for (int64_t p = ti.b0 + S; p < ti.b1; ++p) {
            const uint32_t c = __ldg(P.data + p);
#pragma unroll
            for (int j = 0; j < 16; ++j) ch[j] = w.template step<0>(ch[j], c);
        }
        uint64_t map = 0;
#pragma unroll
        for (int j = 0; j < 16; ++j) map |= (uint64_t)W::dec(ch[j]) << (4 * j);
        r.map = ti.first ? map_const(map_at(map, (uint32_t)P.start)) : map;
    }
    return r;
}

// Entry state of chunk c (lane 0): composes the aggregates of chunks c-1, c-2,
// ... until one has published its exit state (PREFIX) or the composition is a
// constant map. Every poll is bounded; a wait that runs out sets the error word
// and the chunk gives up (entry: the start state).
__device__ uint32_t look_back(const ScanParams &P, int64_t chunk) {
    uint64_t acc = kMapIdentity;   // maps of chunks (j, chunk) applied in order
    for (int64_t j = chunk - 1; j >= 0; --j) {
        uint32_t st = 0, polls = 0;
        while (((st = ld_acquire_u32(P.chunk_status + j)) & 3u) == 0u) {
            if (++polls >= P.poll_limit) break;
            __nanosleep(64);
        }
        if ((st & 3u) == 0u) {
            atomicOr(P.err, kScanErrTimeout);
            break;
        }
        if (st & kStPrefix) return map_at(acc, (st >> 8) & 15u);
        acc = map_then(ld_relaxed_u64(P.chunk_map + j), acc);
        if (map_is_const(acc)) return (uint32_t)acc & 15u;
    }
    return (uint32_t)P.start;
}

// Head of a tile from its true entry state (or the whole tile when its states
// never coincided), and its string's final state and accept flag.
template <class W>
__device__ __forceinline__ void tile_head(const ScanParams &P, const W &w, const TileInfo &ti,
                                          const TileSync &ts, uint32_t e_body, uint32_t entry) {
    uint32_t fin;
    if (ts.conv) {
        walk_write(w, P, ti.b0, ti.b0 + ts.S, w.enc(entry));
        fin = W::dec(e_body);   // body exit (independent of the entry)
    } else {
        fin = W::dec(walk_write(w, P, ti.b0, ti.b1, w.enc(entry)));
    }
    if (ti.last) {
        if (P.final_state) P.final_state[ti.str] = (uint8_t)fin;
        if (P.accept) P.accept[ti.str] = P.accept_tbl[fin];
    }
}

// Dynamic shared memory of the scan kernel: the table (kRepTableBytes16), then
// each thread's sync records of its two tiles (16 bytes each), kept there across
// the body walk so that the walk has the registers.
struct SyncRec {
    int32_t S;
    uint32_t conv_e;   // bit 8: converged; bits 0-7: encoded state at S
    uint64_t map;      // full map of a tile whose states never coincided
};
constexpr uint32_t kScanSyncOff = kRepTableBytes16;
constexpr uint32_t kScanSmemBytes = kScanSyncOff + 2 * kScanThreads * (uint32_t)sizeof(SyncRec);
__device__ __forceinline__ SyncRec *sync_rec(int which) {
    return reinterpret_cast<SyncRec *>(g_dfa_tbl + kScanSyncOff) + which * kScanThreads + threadIdx.x;
}

// A pair of chunks (64 consecutive tiles) with one warp: lane l takes tiles l
// (chunk 2p) and 32 + l (chunk 2p + 1). Both tiles are synced, then both bodies
// are walked as two interleaved chains (two table lookups in flight); the
// aggregates of both chunks are published before the look-back (so every
// chunk's aggregate appears without waiting on anything: the look-back cannot
// deadlock), the second chunk's entry is the first one's exit.
template <class W>
__device__ void scan_pair(const ScanParams &P, const W &w, int64_t pair, int64_t n_tiles) {
    const uint32_t FULL = 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31u;
    const int64_t ca = 2 * pair, cb = ca + 1;
    const int64_t ta_i = ca * 32 + lane, tb_i = cb * 32 + lane;
    const bool have_a = ta_i < n_tiles, have_b = tb_i < n_tiles;
    const TileInfo none{0, 0, 0, true, false};
#pragma unroll 1
    for (int k = 0; k < 2; ++k) {   // sync of both tiles (every lane: the warp votes inside)
        const bool have = k == 0 ? have_a : have_b;
        const TileInfo ti = have ? locate_tile(P, k == 0 ? ta_i : tb_i) : none;
        const TileSync r = tile_sync(P, w, ti, have);
        *sync_rec(k) = SyncRec{(int32_t)r.S, (r.conv ? 0x100u : 0u) | (r.e & 0xffu), r.map};
    }
    // ---- bodies
    const SyncRec ra = *sync_rec(0), rb = *sync_rec(1);
    const bool body_a = have_a && (ra.conv_e & 0x100u), body_b = have_b && (rb.conv_e & 0x100u);
    uint32_t ea = ra.conv_e & 0xffu, eb = rb.conv_e & 0xffu;
    {
        const TileInfo ta = have_a ? locate_tile(P, ta_i) : none;
        const TileInfo tb = have_b ? locate_tile(P, tb_i) : none;
        if (body_a && body_b) {
            walk_write2(w, P, ta.b0 + ra.S, ta.b1, ea, tb.b0 + rb.S, tb.b1, eb);
        } else {
            if (body_a) ea = walk_write(w, P, ta.b0 + ra.S, ta.b1, ea);
            if (body_b) eb = walk_write(w, P, tb.b0 + rb.S, tb.b1, eb);
        }
    }
    const uint64_t map_a = body_a ? map_const(W::dec(ea)) : sync_rec(0)->map;
    const uint64_t map_b = body_b ? map_const(W::dec(eb)) : sync_rec(1)->map;
    // ---- chunk aggregates: compositions of the 32 tile maps, published at once
    uint64_t inc_a = map_a, inc_b = map_b;   // inclusive scans: maps of lanes 0..lane in order
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t pa = __shfl_up_sync(FULL, inc_a, o), pb = __shfl_up_sync(FULL, inc_b, o);
        if (lane >= (uint32_t)o) {
            inc_a = map_then(pa, inc_a);
            inc_b = map_then(pb, inc_b);
        }
    }
    const uint64_t agg_a = __shfl_sync(FULL, inc_a, 31), agg_b = __shfl_sync(FULL, inc_b, 31);
    if (lane == 0) {
        P.chunk_map[ca] = agg_a;
        P.chunk_map[cb] = agg_b;
        __threadfence();
        st_release_u32(P.chunk_status + ca, kStAgg);
        st_release_u32(P.chunk_status + cb, kStAgg);
    }
    // ---- look-back for the first chunk's entry state (lane 0); the second follows it
    uint32_t entry_a = 0;
    if (lane == 0) entry_a = look_back(P, ca);
    entry_a = __shfl_sync(FULL, entry_a, 0);
    const uint32_t entry_b = map_at(agg_a, entry_a);
    if (lane == 0) {
        st_release_u32(P.chunk_status + ca, kStPrefix | (entry_b << 8));
        st_release_u32(P.chunk_status + cb, kStPrefix | (map_at(agg_b, entry_b) << 8));
    }
    // ---- heads from the true entry states: tile `lane` starts in (maps of lanes 0..lane-1)(entry)
    const uint64_t exc_a = __shfl_up_sync(FULL, inc_a, 1), exc_b = __shfl_up_sync(FULL, inc_b, 1);
    if (have_a) {
        const TileInfo ta = locate_tile(P, ta_i);
        const SyncRec r = *sync_rec(0);
        const TileSync ts{r.S, (r.conv_e & 0x100u) != 0, r.conv_e & 0xffu, r.map};
        tile_head(P, w, ta, ts, ea, ta.first ? (uint32_t)P.start : (lane == 0 ? entry_a : map_at(exc_a, entry_a)));
    }
    if (have_b) {
        const TileInfo tb = locate_tile(P, tb_i);
        const SyncRec r = *sync_rec(1);
        const TileSync ts{r.S, (r.conv_e & 0x100u) != 0, r.conv_e & 0xffu, r.map};
        tile_head(P, w, tb, ts, eb, tb.first ? (uint32_t)P.start : (lane == 0 ? entry_b : map_at(exc_b, entry_b)));
    }
}

__global__ void __launch_bounds__(kScanThreads, 1) dfa_scan_kernel(ScanParams P) {
    __shared__ unsigned long long s_pair[kScanThreads / 32];
    build_table(P.tmap, P.n_states);
    __syncthreads();
    const int64_t n_tiles = P.tile_base[P.n_strings];
    const int64_t n_pairs = (n_tiles + 63) / 64;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    while (true) {
        if (lane == 0) s_pair[warp] = atomicAdd(P.head, 1ull);
        __syncwarp();
        const int64_t pair = (int64_t)s_pair[warp];
        __syncwarp();
        if (pair >= n_pairs) break;
        if (P.n_states <= 8) scan_pair(P, Walker<8>{lane}, pair, n_tiles);
        else scan_pair(P, Walker<16>{lane}, pair, n_tiles);
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
                                       kScanSmemBytes));
        attr_set = true;
    }
    profile_kernel_begin(stream);
    dfa_scan_kernel<<<n_sms, kScanThreads, kScanSmemBytes, stream>>>(P);
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
