// Byte-DFA walkers over per-lane replicated shared-memory tables, shared by
// the ragged batch kernel (family a) and the per-position scan (family b).
//
// Transition semantics (reference src/simulation.py:274-297): s' = tmap[c*N + s].
//
// Table layouts (lane = threadIdx.x & 31; every lane reads only its own
// replica, so the 32 lanes of a warp always touch 32 different banks):
//   N <= 8   byte address = c<<8 | (s>>2)<<7 | lane<<2 | (s&3)       64 KiB
//            stored byte  = (s'&3) | lane<<2 | (s'>>2)<<7, i.e. the next
//            address minus c<<8: a step is PRMT (state byte | c<<8) + LDS.U8.
//   N <= 16  byte address = c<<9 | (s>>2)<<7 | lane<<2 | (s&3)       128 KiB
//            stored byte  = (s'&3) | (s'>>2)<<6: a step is PRMT, LOP3, IADD3,
//            LDS.U8 (t = e | c<<8; addr = t + (t & 0xFFC0) + lane*4).
//   N <= 32  byte address = c<<9 | (s>>2)<<6 | (lane&15)<<2 | (s&3)  128 KiB
//            (16 replicas: lanes l and l + 16 share one, so at most two-way
//            bank conflicts); stored byte = (s'&3) | (s'>>2)<<5: a step is
//            PRMT, LOP3, IADD3, LDS.U8 (addr = t + (t & 0xFFE0) + (lane&15)*4).
//   N <= 64  byte address = c<<9 | (s>>2)<<5 | (lane&7)<<2 | (s&3)   128 KiB
//            (8 replicas, a replica for lanes l, l + 8, l + 16, l + 24);
//            stored byte = (s'&3) | (s'>>2)<<4: the same four-instruction
//            step with mask 0xFFF0.
//   N <= 256 plain tmap[c*N + s] (bank conflicts).
#pragma once

#include "trex_internal.cuh"

namespace trex {

struct DfaDesc {
    int32_t n_states;
    int32_t start;
    int64_t tmap_off;
    int64_t accept_off;
    // K-gram walking (kgram > 1): byte b has code (b >> kshift) & ((1 << kbits) - 1);
    // b is one of the automaton's distinguished bytes when it equals byte `code` of
    // kalpha; krep[c] is a byte of code c's column (the other column for unused
    // codes) and krep[1 << kbits] a byte of the column every other byte shares.
    int32_t kgram = 1, kbits = 0, kshift = 0, kpad = 0;
    uint32_t kalpha[4] = {0, 0, 0, 0};
    uint8_t krep[20] = {};
};

// Dynamic shared memory of every kernel that walks a table: the table sits
// at offset 0 (1 KiB aligned).
extern __shared__ __align__(1024) uint8_t g_dfa_tbl[];

__device__ __forceinline__ uint32_t tbl_u8(uint32_t off) { return g_dfa_tbl[off]; }

template <int LAYOUT> struct Walker;

template <> struct Walker<8> {
    static constexpr int kChains = 8;
    uint32_t lane;
    __device__ uint32_t enc(uint32_t s) const { return (s & 3u) | (lane << 2) | ((s >> 2) << 7); }
    __device__ static uint32_t dec(uint32_t e) { return (e & 3u) | ((e >> 7) << 2); }
    template <int I>
    __device__ __forceinline__ uint32_t step(uint32_t e, uint32_t x) const {
        return tbl_u8(__byte_perm(e, x, 0x1100 | ((4 + I) << 4)));
    }
    // the same layout for a second table `off` bytes into shared memory
    template <int I>
    __device__ __forceinline__ uint32_t step_off(uint32_t off, uint32_t e, uint32_t x) const {
        return tbl_u8(off + __byte_perm(e, x, 0x1100 | ((4 + I) << 4)));
    }
};

template <> struct Walker<16> {
    static constexpr int kChains = 16;
    uint32_t lane;
    __device__ uint32_t enc(uint32_t s) const { return (s & 3u) | ((s >> 2) << 6); }
    __device__ static uint32_t dec(uint32_t e) { return (e & 3u) | ((e >> 6) << 2); }
    template <int I>
    __device__ __forceinline__ uint32_t step(uint32_t e, uint32_t x) const {
        uint32_t t = __byte_perm(e, x, 0x1100 | ((4 + I) << 4));
        return tbl_u8((lane << 2) + t + (t & 0xFFC0u));
    }
    template <int I>
    __device__ __forceinline__ uint32_t step_off(uint32_t off, uint32_t e, uint32_t x) const {
        uint32_t t = __byte_perm(e, x, 0x1100 | ((4 + I) << 4));
        return tbl_u8(off + (lane << 2) + t + (t & 0xFFC0u));
    }
};

template <> struct Walker<32> {
    static constexpr int kChains = 32;
    uint32_t lane;
    __device__ uint32_t enc(uint32_t s) const { return (s & 3u) | ((s >> 2) << 5); }
    __device__ static uint32_t dec(uint32_t e) { return (e & 3u) | ((e >> 5) << 2); }
    template <int I>
    __device__ __forceinline__ uint32_t step(uint32_t e, uint32_t x) const {
        uint32_t t = __byte_perm(e, x, 0x1100 | ((4 + I) << 4));
        return tbl_u8(((lane & 15u) << 2) + t + (t & 0xFFE0u));
    }
};

template <> struct Walker<64> {
    static constexpr int kChains = 64;
    uint32_t lane;
    __device__ uint32_t enc(uint32_t s) const { return (s & 3u) | ((s >> 2) << 4); }
    __device__ static uint32_t dec(uint32_t e) { return (e & 3u) | ((e >> 4) << 2); }
    template <int I>
    __device__ __forceinline__ uint32_t step(uint32_t e, uint32_t x) const {
        uint32_t t = __byte_perm(e, x, 0x1100 | ((4 + I) << 4));
        return tbl_u8(((lane & 7u) << 2) + t + (t & 0xFFF0u));
    }
};

template <> struct Walker<0> {
    static constexpr int kChains = 0;
    uint32_t n;
    __device__ uint32_t enc(uint32_t s) const { return s; }
    __device__ static uint32_t dec(uint32_t e) { return e; }
    template <int I>
    __device__ __forceinline__ uint32_t step(uint32_t e, uint32_t x) const {
        uint32_t c = (x >> (8 * I)) & 0xFFu;
        return tbl_u8(c * n + e);
    }
};

// Shared-memory bytes a DFA of n states needs.
__host__ __device__ inline int table_bytes_for(int n) {
    return n <= 8 ? 256 * 256 : n <= 64 ? 256 * 512 : 256 * n;
}

// Fills ncols columns of a replicated table (N <= 16) at byte `off` of shared
// memory in the layout N selects; next(c, s) is the next state of state s < N
// on column c (padded states loop).
template <class F>
__device__ inline void build_layout(int N, int ncols, uint32_t off, F next) {
    uint32_t *w32 = reinterpret_cast<uint32_t *>(g_dfa_tbl + off);
    if (N <= 8) {
        for (int w = threadIdx.x; w < ncols * 64; w += blockDim.x) {
            uint32_t c = w >> 6, q = (w >> 5) & 1u, ln = w & 31u, word = 0;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                uint32_t s = q * 4 + b;
                uint32_t t = s < (uint32_t)N ? next(c, s) : s;
                word |= ((t & 3u) | (ln << 2) | ((t >> 2) << 7)) << (8 * b);
            }
            w32[w] = word;
        }
    } else {
        for (int w = threadIdx.x; w < ncols * 128; w += blockDim.x) {
            uint32_t c = w >> 7, q = (w >> 5) & 3u, word = 0;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                uint32_t s = q * 4 + b;
                uint32_t t = s < (uint32_t)N ? next(c, s) : s;
                word |= ((t & 3u) | ((t >> 2) << 6)) << (8 * b);
            }
            w32[w] = word;
        }
    }
}

// Fills the shared table for `src` (256*N byte map) in the layout N selects.
__device__ inline void build_table(const uint8_t *__restrict__ src, int N) {
    uint8_t *tbl = g_dfa_tbl;
    uint32_t *w32 = reinterpret_cast<uint32_t *>(tbl);
    if (N <= 8) {
        for (int w = threadIdx.x; w < 256 * 256 / 4; w += blockDim.x) {
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
        for (int w = threadIdx.x; w < 256 * 512 / 4; w += blockDim.x) {
            uint32_t c = w >> 7, q = (w >> 5) & 3u, word = 0;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                uint32_t s = q * 4 + b;
                uint32_t t = s < (uint32_t)N ? src[c * N + s] : s;
                word |= ((t & 3u) | ((t >> 2) << 6)) << (8 * b);
            }
            w32[w] = word;
        }
    } else if (N <= 32) {
        // word address c<<7 | (s>>2)<<4 | replica: four states s = 4 q .. 4 q + 3 a word
        for (int w = threadIdx.x; w < 256 * 512 / 4; w += blockDim.x) {
            uint32_t c = w >> 7, q = (w >> 4) & 7u, word = 0;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                uint32_t s = q * 4 + b;
                uint32_t t = s < (uint32_t)N ? src[c * N + s] : s;
                word |= ((t & 3u) | ((t >> 2) << 5)) << (8 * b);
            }
            w32[w] = word;
        }
    } else if (N <= 64) {
        // word address c<<7 | (s>>2)<<3 | replica: four states s = 4 q .. 4 q + 3 a word
        for (int w = threadIdx.x; w < 256 * 512 / 4; w += blockDim.x) {
            uint32_t c = w >> 7, q = (w >> 3) & 15u, word = 0;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                uint32_t s = q * 4 + b;
                uint32_t t = s < (uint32_t)N ? src[c * N + s] : s;
                word |= ((t & 3u) | ((t >> 2) << 4)) << (8 * b);
            }
            w32[w] = word;
        }
    } else {
        for (int i = threadIdx.x; i < 256 * N; i += blockDim.x) tbl[i] = src[i];
    }
}

template <class W>
__device__ __forceinline__ uint32_t step_word(const W &w, uint32_t e, uint32_t x) {
    e = w.template step<0>(e, x);
    e = w.template step<1>(e, x);
    e = w.template step<2>(e, x);
    e = w.template step<3>(e, x);
    return e;
}

template <class W>
__device__ __forceinline__ uint32_t step16(const W &w, uint32_t e, uint4 v) {
    e = step_word(w, e, v.x);
    e = step_word(w, e, v.y);
    e = step_word(w, e, v.z);
    e = step_word(w, e, v.w);
    return e;
}

// Same as step_word but byte j is applied only when bit j of m is set.
template <class W>
__device__ __forceinline__ uint32_t step_word_masked(const W &w, uint32_t e, uint32_t x,
                                                     uint32_t m) {
    uint32_t n;
    n = w.template step<0>(e, x); e = (m & 1u) ? n : e;
    n = w.template step<1>(e, x); e = (m & 2u) ? n : e;
    n = w.template step<2>(e, x); e = (m & 4u) ? n : e;
    n = w.template step<3>(e, x); e = (m & 8u) ? n : e;
    return e;
}

template <class W>
__device__ __forceinline__ uint32_t step16_masked(const W &w, uint32_t e, uint4 v, uint32_t m) {
    e = step_word_masked(w, e, v.x, m);
    e = step_word_masked(w, e, v.y, m >> 4);
    e = step_word_masked(w, e, v.z, m >> 8);
    e = step_word_masked(w, e, v.w, m >> 12);
    return e;
}

// Bits [lo, hi) set, 0 <= lo <= hi <= 32.
__device__ __forceinline__ uint32_t bit_range(int lo, int hi) {
    uint32_t upto_hi = hi >= 32 ? 0xffffffffu : ((1u << hi) - 1u);
    uint32_t below_lo = lo >= 32 ? 0xffffffffu : ((1u << lo) - 1u);
    return upto_hi & ~below_lo;
}

// Loads the 32-byte window at absolute address w (32-aligned). Bytes outside
// [lo, hi) of the buffer are not read (returned as 0).
__device__ __forceinline__ void load_window(const uint8_t *w, const uint8_t *lo,
                                            const uint8_t *hi, uint4 &a, uint4 &b) {
    if (w >= lo && w + 32 <= hi) {
        ld_stream32(w, a, b);   // one 32-byte load (the window is 32-byte aligned)
    } else {
        uint32_t r[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            uint32_t v = 0;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint8_t *q = w + 4 * k + j;
                if (q >= lo && q < hi) v |= (uint32_t)__ldg(q) << (8 * j);
            }
            r[k] = v;
        }
        a = make_uint4(r[0], r[1], r[2], r[3]);
        b = make_uint4(r[4], r[5], r[6], r[7]);
    }
}

}  // namespace trex
