// Family (d): probabilistic NFA (weighted automaton, HMM forward pass) with up
// to 64 states.
//
// Semantics (reference cuda/nfa_tc_evolution.cu:456-561 nfa_prob_v5_tc_kernel,
// :572-610 nfa_prob_v6_cuda_kernel): T[c] is a real 64 x 64 matrix in the
// T[dst][src] convention; the state starts at the start vector and symbol c
// maps it to s' = T[c] s; a string's result is dot(s_L, accept). The
// reference returns only dot > 0.5; this engine returns the natural
// log-likelihood log(dot) in FP64 and that flag. Bytes >= sigma are skipped
// (the reference kernels leave the state unchanged for them).
//
// Range: every step renormalises s by an exact power of two 2^-f and adds the
// integer f to the string's exponent E, so log-likelihood = log(dot) + E ln 2.
//
// Plain form (FP32, CUDA cores): a warp per string, lane l owns states l and
// l + 32, T[c] rows read through L1; f = the frexp exponent of the step's
// max |s'|, the rule of the FP64 oracle.
//
// Tensor form (tcgen05, BF16 or FP16 operands, FP32 accumulation in TMEM).
// One persistent CTA per SM holds up to 512 strings ("slots") and advances
// them all one symbol per step. A tcgen05.mma (M=128, K=16) costs about the
// same time for any N up to 256 (measured: ~120-165 cycles whether N is 16 or
// 192), so the kernel is bound by the number of MMA instructions per step:
// every pair of symbols gets one MMA chain over all of the CTA's strings that
// carry it (about 40 instructions a step), and chunks pipeline inside a step
// (the MMA of one symbol pair runs while the epilogue drains the previous
// one). Orientation: D[dst][string] = T[c][dst][:] . S[:][string]
// -- the 64 states are the MMA's M rows (TMEM lanes) and the strings its N
// columns, because strings of one step carry different symbols and only the
// N side can be regrouped cheaply. Symbols are paired (2p, 2p+1): the A
// operand of pair p is [T[2p]; T[2p+1]] (M = 128), resident in TMEM for the
// whole kernel (32 columns a pair: 64 16-bit K values per lane), so the shared
// memory traffic of an MMA is only its B columns. Each step, the strings of a
// sub-batch are grouped by pair in the B buffer (even symbol first), and one
// MMA chain (K = 64 as 4 x K16) per group of <= 64 strings writes a 64-column
// region of a TMEM ring. Rows 0-63 of the result are valid for the even-symbol
// strings, rows 64-127 for the odd ones (half the MMA work is discarded: the
// price of keeping A in TMEM and B small).
//
// Warp roles (480 threads):
//  * warps 0-7, epilogue, two sets of four taking alternate chunks (warp q of a
//    set reads TMEM lanes 32q..32q+31 with 16x256b loads, four states of four
//    columns a thread): it scales each string's states by the record's 2^-f,
//    rounds them to 16 bits, stores them in pairs in the string's row of the
//    next B buffer and records max|s_t+1| (a butterfly max); on a string's
//    last symbol it writes the accept-weighted sum instead.
//  * warp 8, MMA: per chunk waits for a free ring region, issues 4
//    tcgen05.mma (A from TMEM, B from shared memory, no swizzle) and commits
//    to the region's mbarrier.
//  * warps 9-12, planner: per step and sub-batch, sorts the slots of the step
//    by symbol pair (counting sort with shared atomics), writes the chunk list
//    and the start vector into the rows of strings that begin; for the
//    previous step it writes one record per row: the string's row in the next
//    B buffer and the scale 2^-f, f = the exponent of max|s| * R_c (R_c = max
//    row sum of |T[c]|, so max|s'| < 1; max|s| left by the epilogue), adding f
//    to the string's exponent sum; and it turns finished strings' dot
//    products and exponents into the FP64 log-likelihood.
//  * warps 13-14, loader: gives each slot its next string from a global
//    atomic queue and copies the next 16 valid symbols of every slot into a
//    shared block (strings change slots only at 16-step block boundaries).
// Hand-offs are mbarriers (one per sub-batch and step parity, so no waiter is
// ever two phases behind); the planner warps meet at a named barrier and only
// their leader waits on mbarriers. B buffers (shared memory, K-major, no
// swizzle): row r, state k at (k/8)*LBO + r*16 + (k%8)*2 with LBO = rows*16 and
// rows = 1 (mod 8), so the 32 lanes of an epilogue store hit 32 different banks
// and an MMA may start at any row.
// Every wait is bounded; one that runs out sets the error word (bit 2) and an
// abort flag that every role polls; the MMA warp drains its commits and the
// TMEM is freed before the kernel returns.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "trex_internal.cuh"

namespace trex {

constexpr int kPnStates = 64;
constexpr int kPnBlk = 16;             // steps per symbol block
constexpr int kPnEpiWarps = 8, kPnMmaWarp = 8, kPnPlanWarp0 = 9, kPnPlanWarps = 4,
              kPnLoadWarp0 = 13, kPnLoadWarps = 2;
constexpr int kPnThreads = 32 * (kPnLoadWarp0 + kPnLoadWarps);
constexpr int kPnPlanThreads = 32 * kPnPlanWarps;
constexpr int kPnMaxPSub = 512;        // slots per sub-batch
constexpr int kPnSlotsPerPlanThread = kPnMaxPSub / kPnPlanThreads;
constexpr int kPnMaxChunks = 32;
constexpr int kPnRegionCols = 64;
constexpr int kPnMaxRegions = 6;
constexpr int kPnMaxSigmaTc = 28;      // 14 pairs: 448 TMEM columns + one ring region
constexpr int kPnMiscBytes = 2048;
constexpr uint32_t kPnSmemCap = 232448;
constexpr int32_t kPnTerminate = -1;
constexpr uint32_t kPnErrOffsets = 1u, kPnErrTimeout = 4u;
// The drain of committed MMAs before the TMEM is freed always waits up to the
// default limit (an MMA still writing TMEM must not outlive the allocation);
// the hand-off waits use PnParams::wait_cycles.
constexpr long long kPnDrainCycles = kDefaultMbarCycles;

constexpr uint32_t kRecFinish = 1u << 31;
// slot flags (planner)
constexpr uint8_t kSlotActive = 1, kSlotLast = 2, kSlotFresh = 4;
// header flags (loader)
constexpr uint8_t kHdrStart = 1, kHdrEnd = 2;

struct PnHdr {
    int32_t seq;
    uint8_t count, flags;
    uint16_t pad;
};
struct PnSlot {
    int32_t seq;          // string in the slot
    int32_t pend[2];      // string whose last step (of that parity) awaits its log-likelihood
    int16_t row;          // row at the last planned step
    uint8_t c, flags, blkcnt, blkflags;
};
struct PnChunk {
    uint16_t row0;
    uint8_t ncols, split, pair, pad0, pad1, pad2;
};

struct PnLayout {
    int p_sub, rows, npairs, nregions, ring_base;
    uint32_t lbo;
    uint32_t s_off, sym_off, hdr_off, rec_off, xmax_off, fin_off, fine_off, e_off, chunk_off,
        slot_off, misc_off, total;
};

__host__ __device__ inline uint32_t pn_align16(uint32_t x) { return (x + 15u) & ~15u; }

// acols: TMEM columns of a symbol pair's A operand (32 for 16-bit operands: 64 K
// values of 2 bytes a lane; 16 for int8 operands: 4 K values a 32-bit column).
static PnLayout pn_layout(int p_sub, int sigma, int acols = 32) {
    PnLayout L{};
    L.p_sub = p_sub;
    L.npairs = (sigma + 1) / 2;
    L.ring_base = acols * L.npairs;
    L.nregions = std::min(kPnMaxRegions, (512 - L.ring_base) / kPnRegionCols);
    int rows = p_sub + 16;
    while (rows % 8 != 1) ++rows;
    L.rows = rows;
    L.lbo = (uint32_t)rows * 16u;
    const uint32_t ps = (uint32_t)p_sub, nr = (uint32_t)rows;
    uint32_t off = 0;
    L.s_off = off;                    // [step parity] B buffers, 8 * lbo bytes each
    off += 2u * 8u * L.lbo;
    L.sym_off = off;                  // [buf][16 steps][p_sub] symbols
    off += 2u * kPnBlk * ps;
    L.hdr_off = pn_align16(off);      // [buf][p_sub] headers
    off = L.hdr_off + 2u * ps * (uint32_t)sizeof(PnHdr);
    L.rec_off = pn_align16(off);      // [step & 3][rows] uint2 records
    off = L.rec_off + 4u * nr * 8u;
    L.xmax_off = pn_align16(off);     // [step parity][rows] float2: max|s| of each half
    off = L.xmax_off + 2u * nr * 8u;
    L.fin_off = off;                  // [step parity][p_sub] float2: accept-weighted halves
    off += 2u * ps * 8u;
    L.fine_off = off;                 // [step parity][p_sub] int32: final exponent sums
    off += 2u * ps * 4u;
    L.e_off = off;                    // [p_sub] int32: exponent sums
    off += ps * 4u;
    L.chunk_off = pn_align16(off);    // [step & 3][kPnMaxChunks]
    off = L.chunk_off + 4u * kPnMaxChunks * (uint32_t)sizeof(PnChunk);
    L.slot_off = pn_align16(off);     // [p_sub]
    off = L.slot_off + ps * (uint32_t)sizeof(PnSlot);
    L.misc_off = pn_align16(off);
    off = L.misc_off + kPnMiscBytes;
    L.total = pn_align16(off);
    return L;
}

// misc region (bytes, relative to misc_off)
constexpr uint32_t kMTmem = 0, kMAbort = 4, kMPlanOk = 8, kMFinal = 12,
                   kMNch = 16,        // int32 [step & 3]
                   kMBlkAct = 32,     // int32 [buf][loader warp]
                   kMBar = 64,        // mbarriers, 8 bytes each
                   kMCnt = 320,       // int32 [16 pairs][2 parities]
                   kMPinfo = 448,     // int32 [16 pairs][base, neven]
                   kMRsym = 576,      // float [32]
                   kMStart = 704,     // uint4 [8]
                   kMAcc = 832;       // float [64]
// mbarrier indices
constexpr int kBarPlan1 = 0,     // [step & 3]   layout, chunk list, records   1 arrival
              kBarPlan2 = 4,     // [step & 1]   start rows                    1 arrival
              kBarEpi = 6,       // [step & 3]   epilogue done                 8 arrivals
              kBarFull = 10,     // [region]     tcgen05.commit
              kBarEmpty = 16,    // [region]     4 arrivals (the set that drained it)
              kBarLoaded = 22,   // [buf]        2 arrivals
              kBarConsumed = 24, // [buf]        1 arrival
              kBarCount = 26;
// record of a row (one string at one step): x = destination row * 16 (or kRecFinish | slot),
// y = slot | kRecFresh
constexpr uint32_t kRecFresh = 1u << 31;

struct PnParams {
    const uint8_t *data;
    int64_t total_bytes;
    const int64_t *offsets;
    int64_t n;
    const uint32_t *tpack;     // [npairs][128][32] 16-bit pairs
    const float *rsym;         // [sigma] growth bound per symbol
    const uint4 *start_img;    // [8] start vector, 16-bit, one B row
    const float *acc;          // [64] accept weights
    float start_max;
    int boolean;               // Boolean NFA: threshold every product to {0, 1}, no rescale
    int kcols;                 // 16-byte core-matrix columns of a B row: 8 (16-bit), 4 (int8)
    long long wait_cycles;     // limit of one hand-off wait
    int resc;                  // steps between rescales (power-of-two scaling is exact, so only
                               // the range matters: 4 for BF16 with growth <= 16 a step, else 1)
    double ll_empty;
    int sigma;
    double *loglik;
    uint8_t *accept;
    int32_t *accept_i32;
    unsigned long long *queue;
    uint32_t *err;
    PnLayout L;
};

// ---- small device helpers -------------------------------------------------------------------
__device__ __forceinline__ uint32_t pn_smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void pn_tc_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void pn_tc_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void pn_fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ bool pn_mbar_test(uint32_t addr, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(done) : "r"(addr), "r"(parity) : "memory");
    return done != 0;
}
// non-suspending test: a spinning waiter sees the phase flip at once (try_wait may park the
// thread for a few thousand cycles)
__device__ __forceinline__ bool pn_mbar_poll(uint32_t addr, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(done) : "r"(addr), "r"(parity) : "memory");
    return done != 0;
}
__device__ __forceinline__ void pn_mbar_arrive(uint32_t addr) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(addr) : "memory");
}

// Waits (lane 0 of the calling warp) for the completion of the phase with the
// given parity; bounded; the result is broadcast to the warp. Spins on the
// non-suspending test: the hand-offs of this kernel are on its critical path.
__device__ __forceinline__ bool pn_wait(uint32_t addr, uint32_t parity, volatile uint32_t *abort_flag,
                                        uint32_t *err, long long limit) {
    int ok = 1;
    if ((threadIdx.x & 31) == 0) {
        const long long t0 = clock64();
        while (!pn_mbar_poll(addr, parity)) {
            if (*abort_flag) { ok = 0; break; }
            if (clock64() - t0 > limit) {
                atomicOr(err, kPnErrTimeout);
                *abort_flag = 1u;
                ok = 0;
                break;
            }
        }
    }
    ok = __shfl_sync(0xffffffffu, ok, 0);
    __syncwarp();
    return ok != 0;
}

// pn_wait with the suspending test: a thread whose phase is not complete may be parked by the
// hardware instead of spinning, which leaves the issue slots to the warps with work (the lane
// kernel, whose warps wait a large share of each step)
__device__ __forceinline__ bool pn_wait_park(uint32_t addr, uint32_t parity, volatile uint32_t *abort_flag,
                                             uint32_t *err, long long limit) {
    int ok = 1;
    if ((threadIdx.x & 31) == 0) {
        const long long t0 = clock64();
        while (!pn_mbar_test(addr, parity)) {
            if (*abort_flag) { ok = 0; break; }
            if (clock64() - t0 > limit) {
                atomicOr(err, kPnErrTimeout);
                *abort_flag = 1u;
                ok = 0;
                break;
            }
        }
    }
    ok = __shfl_sync(0xffffffffu, ok, 0);
    __syncwarp();
    return ok != 0;
}

__device__ __forceinline__ void pn_write_result(double *loglik, uint8_t *accept, int32_t *accept_i32,
                                                int64_t seq, double ll) {
    if (loglik) loglik[seq] = ll;
    const int a = ll > -0.69314718055994530942;   // dot > 0.5
    if (accept) accept[seq] = (uint8_t)a;
    if (accept_i32) accept_i32[seq] = a;
}

// exponent f with x < 2^f for a finite positive float x (x >= 2^-126); 0 for x == 0
__device__ __forceinline__ int pn_ceil_exp(float x) {
    const uint32_t e = (__float_as_uint(x) >> 23) & 0xFFu;
    if (e == 0) return 0;
    return (int)e - 126;
}
__device__ __forceinline__ float pn_pow2(int f) {   // 2^f, |f| <= 126
    return __uint_as_float((uint32_t)(127 + f) << 23);
}

template <bool FP16>
__device__ __forceinline__ uint16_t pn_to16(float v) {
    if constexpr (FP16) return __half_as_ushort(__float2half_rn(v));
    else return __bfloat16_as_ushort(__float2bfloat16_rn(v));
}

__device__ __forceinline__ void pn_tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr) : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// 16 TMEM lanes x 16 columns: thread t gets lanes base + t/4 and base + t/4 + 8 for columns
// 2(t%4), 2(t%4)+1 and 8 + 2(t%4), 9 + 2(t%4):
// r = {(l, c), (l, c+1), (l+8, c), (l+8, c+1), (l, c+8), (l, c+9), (l+8, c+8), (l+8, c+9)}.
__device__ __forceinline__ void pn_tmem_ld16x256(uint32_t taddr, uint32_t (&r)[8]) {
    asm volatile("tcgen05.ld.sync.aligned.16x256b.x2.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                   "=r"(r[7])
                 : "r"(taddr) : "memory");
}
__device__ __forceinline__ void pn_tmem_wait_ld() {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// two values rounded to the operand type, packed low/high
template <bool FP16>
__device__ __forceinline__ uint32_t pn_pack2(float lo, float hi) {
    if constexpr (FP16) {
        const __half2 h = __floats2half2_rn(lo, hi);
        return *reinterpret_cast<const uint32_t *>(&h);
    } else {
        const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
        return *reinterpret_cast<const uint32_t *>(&h);
    }
}

__device__ __forceinline__ void pn_tmem_st32(uint32_t taddr, const uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
        "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};"
        :: "r"(taddr), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]),
           "r"(r[7]), "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]),
           "r"(r[14]), "r"(r[15]), "r"(r[16]), "r"(r[17]), "r"(r[18]), "r"(r[19]), "r"(r[20]),
           "r"(r[21]), "r"(r[22]), "r"(r[23]), "r"(r[24]), "r"(r[25]), "r"(r[26]), "r"(r[27]),
           "r"(r[28]), "r"(r[29]), "r"(r[30]), "r"(r[31])
        : "memory");
}

__device__ __forceinline__ void pn_tmem_st16(uint32_t taddr, const uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
        "%14,%15,%16};"
        :: "r"(taddr), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]),
           "r"(r[7]), "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]),
           "r"(r[14]), "r"(r[15])
        : "memory");
}

// ---- shared-memory view -------------------------------------------------------------------------
struct PnShared {
    uint8_t *base;
    PnLayout L;
    __device__ uint8_t *misc() const { return base + L.misc_off; }
    __device__ volatile uint32_t *u32(uint32_t off) const {
        return reinterpret_cast<volatile uint32_t *>(misc() + off);
    }
    __device__ uint32_t bar(int i) const { return pn_smem_u32(misc() + kMBar + 8 * i); }
    __device__ uint32_t sbuf(int par) const { return L.s_off + (uint32_t)par * 8u * L.lbo; }
    __device__ uint8_t *sym(int buf) const { return base + L.sym_off + buf * kPnBlk * L.p_sub; }
    __device__ PnHdr *hdr(int buf) const {
        return reinterpret_cast<PnHdr *>(base + L.hdr_off) + buf * L.p_sub;
    }
    __device__ uint2 *rec(int s) const {
        return reinterpret_cast<uint2 *>(base + L.rec_off) + (s & 3) * L.rows;
    }
    __device__ float2 *xmax(int s) const {
        return reinterpret_cast<float2 *>(base + L.xmax_off) + (s & 1) * L.rows;
    }
    __device__ float2 *fin(int s) const {
        return reinterpret_cast<float2 *>(base + L.fin_off) + (s & 1) * L.p_sub;
    }
    __device__ int32_t *finE(int s) const {
        return reinterpret_cast<int32_t *>(base + L.fine_off) + (s & 1) * L.p_sub;
    }
    __device__ int32_t *E() const { return reinterpret_cast<int32_t *>(base + L.e_off); }
    __device__ PnChunk *chunks(int s) const {
        return reinterpret_cast<PnChunk *>(base + L.chunk_off) + (s & 3) * kPnMaxChunks;
    }
    __device__ PnSlot *slots() const { return reinterpret_cast<PnSlot *>(base + L.slot_off); }
    __device__ volatile int32_t *nch(int s) const {
        return reinterpret_cast<volatile int32_t *>(misc() + kMNch) + (s & 3);
    }
    __device__ int32_t *cnt() const { return reinterpret_cast<int32_t *>(misc() + kMCnt); }
    __device__ int32_t *pinfo() const { return reinterpret_cast<int32_t *>(misc() + kMPinfo); }
};

// phase parity of the k-th completion of a barrier that completes once every `period` steps
__device__ __forceinline__ uint32_t pn_par(int step, int period) { return (uint32_t)(step / period) & 1u; }

// ---- loader: warps 13-14 -------------------------------------------------------------------------
__device__ void pn_loader(const PnParams &P, const PnShared &S, volatile uint32_t *abort_flag) {
    const int lane = threadIdx.x & 31;
    const int lw = (threadIdx.x >> 5) - kPnLoadWarp0;
    const int ll = lw * 32 + lane;
    const int PC = S.L.p_sub;
    const uint32_t sig4 = (uint32_t)P.sigma * 0x01010101u;
    int32_t seq[8];
    int64_t pos[8], end[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) { seq[i] = -1; pos[i] = 0; end[i] = 0; }
    for (int blk = 0;; ++blk) {
        const int buf = blk & 1;
        if (blk >= 2 && !pn_wait(S.bar(kBarConsumed + buf), (uint32_t)((blk - 2) >> 1) & 1u,
                                 abort_flag, P.err, P.wait_cycles))
            break;
        uint8_t *sym = S.sym(buf);
        PnHdr *hd = S.hdr(buf);
        int nact = 0;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int j = ll + 64 * i;
            if (j >= PC) continue;
            uint8_t flags = 0;
            if (seq[i] < 0 || pos[i] >= end[i]) {
                seq[i] = -1;
                for (;;) {
                    const unsigned long long idx = atomicAdd(P.queue, 1ull);
                    if (idx >= (unsigned long long)P.n) break;
                    int64_t p0 = P.offsets[idx], p1 = P.offsets[idx + 1];
                    if (p0 < 0 || p1 < p0 || p1 > P.total_bytes) {
                        atomicOr(P.err, kPnErrOffsets);
                        continue;
                    }
                    while (p0 < p1 && P.data[p0] >= (uint8_t)P.sigma) ++p0;
                    if (p0 == p1) {
                        pn_write_result(P.loglik, P.accept, P.accept_i32, (int64_t)idx, P.ll_empty);
                        continue;
                    }
                    seq[i] = (int32_t)idx;
                    pos[i] = p0;
                    end[i] = p1;
                    flags = kHdrStart;
                    break;
                }
            }
            int count = 0;
            if (seq[i] >= 0) {
                int64_t p = pos[i];
                const int64_t e = end[i];
                bool fast = false;
                // 20-byte window of aligned words; only when it lies inside [data, data + e)
                const uintptr_t ap = reinterpret_cast<uintptr_t>(P.data + p);
                const uintptr_t aw = ap & ~(uintptr_t)3;
                if (e - p >= 20 && aw >= reinterpret_cast<uintptr_t>(P.data)) {
                    const uint32_t *wp = reinterpret_cast<const uint32_t *>(aw);
                    uint32_t w[5];
#pragma unroll
                    for (int k = 0; k < 5; ++k) w[k] = __ldg(wp + k);
                    const uint32_t sh = (uint32_t)(ap & 3) * 8u;
                    uint32_t wd[4];
#pragma unroll
                    for (int k = 0; k < 4; ++k) wd[k] = __funnelshift_r(w[k], w[k + 1], sh);
                    uint32_t bad = 0;
#pragma unroll
                    for (int k = 0; k < 4; ++k) bad |= __vcmpgeu4(wd[k], sig4);
                    if (bad == 0) {
                        fast = true;
#pragma unroll
                        for (int s = 0; s < 16; ++s)
                            sym[s * PC + j] = (uint8_t)(wd[s >> 2] >> (8 * (s & 3)));
                        count = 16;
                        p += 16;
                    }
                }
                if (!fast) {
                    while (count < 16 && p < e) {
                        const uint8_t b = P.data[p++];
                        if (b < (uint8_t)P.sigma) sym[(count++) * PC + j] = b;
                    }
                }
                while (p < e && P.data[p] >= (uint8_t)P.sigma) ++p;
                pos[i] = p;
                if (p == e) flags |= kHdrEnd;
            }
            PnHdr h;
            h.seq = seq[i];
            h.count = (uint8_t)count;
            h.flags = count > 0 ? flags : 0;
            h.pad = 0;
            hd[j] = h;
            nact += count > 0;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) nact += __shfl_xor_sync(0xffffffffu, nact, o);
        if (lane == 0) {
            reinterpret_cast<volatile int32_t *>(S.misc() + kMBlkAct)[buf * 2 + lw] = nact;
            pn_mbar_arrive(S.bar(kBarLoaded + buf));
        }
        __syncwarp();
        // both loader warps have written the block: its active count decides the end
        if (!pn_wait(S.bar(kBarLoaded + buf), (uint32_t)(blk >> 1) & 1u, abort_flag, P.err, P.wait_cycles)) break;
        const volatile int32_t *ba = reinterpret_cast<const volatile int32_t *>(S.misc() + kMBlkAct);
        if (ba[buf * 2] + ba[buf * 2 + 1] == 0) break;
    }
}

// ---- planner: warps 9-12 ---------------------------------------------------------------------------
// named barrier 1: the four planner warps only; only warp 9 waits on mbarriers
__device__ __forceinline__ void pn_plan_sync() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

// Per step s, in order:
//  stage 1 (waits for the symbol block and for the epilogue of step s-4, the last user of the
//          4-deep record and chunk rings): ranks of the slots by symbol pair, the chunk list of
//          step s, the records of step s-1 (destination rows); signals kBarPlan1[s & 3].
//  stage 2 (waits for the epilogue of step s-2): log-likelihoods of the strings that ended at
//          step s-2, the start vector into the rows of strings that begin at step s (B buffer
//          s & 1, last read by the MMA of step s-2); signals kBarPlan2[s & 1].
__device__ void pn_planner(const PnParams &P, const PnShared &S, volatile uint32_t *abort_flag) {
    const int tid = threadIdx.x - 32 * kPnPlanWarp0;   // 0..127
    const int lane = tid & 31;
    const bool leader = tid == 0;
    const PnLayout &L = S.L;
    const int PS = L.p_sub;
    const uint4 *simg = reinterpret_cast<const uint4 *>(S.misc() + kMStart);
    PnSlot *slots = S.slots();
    int32_t *cnt = S.cnt();
    int32_t *pinfo = S.pinfo();
    volatile uint32_t *plan_ok = S.u32(kMPlanOk);
    volatile uint32_t *final_flag = S.u32(kMFinal);
    for (int j = tid; j < PS; j += kPnPlanThreads) {
        PnSlot z;
        z.seq = -1; z.pend[0] = -1; z.pend[1] = -1; z.row = 0; z.c = 0; z.flags = 0;
        z.blkcnt = 0; z.blkflags = 0;
        slots[j] = z;
    }
    for (int k = tid; k < 32; k += kPnPlanThreads) cnt[k] = 0;
    pn_plan_sync();
    auto emit = [&](int s_done) {   // strings whose last step was s_done
        const float2 *fin = S.fin(s_done);
        const int32_t *finE = S.finE(s_done);
        for (int j = tid; j < PS; j += kPnPlanThreads) {
            const int32_t seq = slots[j].pend[s_done & 1];
            if (seq < 0) continue;
            const float2 f = fin[j];
            const double dot = (double)f.x + (double)f.y;
            const double ll = dot > 0.0 ? log(dot) + (double)finE[j] * 0.69314718055994530942 : -INFINITY;
            pn_write_result(P.loglik, P.accept, P.accept_i32, seq, ll);
            slots[j].pend[s_done & 1] = -1;
        }
    };
    for (int s = 0;; ++s) {
        // ---------------- stage 1 ----------------
        if (tid < 32) {
            bool ok = true;
            if (s >= 4)
                ok = pn_wait(S.bar(kBarEpi + ((s - 4) & 3)), pn_par(s - 4, 4), abort_flag, P.err, P.wait_cycles);
            if (ok && s % kPnBlk == 0) {
                const int blk = s / kPnBlk;
                if (leader && blk >= 1) pn_mbar_arrive(S.bar(kBarConsumed + ((blk - 1) & 1)));
                ok = pn_wait(S.bar(kBarLoaded + (blk & 1)), (uint32_t)(blk >> 1) & 1u, abort_flag, P.err, P.wait_cycles);
                if (ok && leader) {
                    const volatile int32_t *ba =
                        reinterpret_cast<const volatile int32_t *>(S.misc() + kMBlkAct);
                    *final_flag = (ba[(blk & 1) * 2] + ba[(blk & 1) * 2 + 1]) == 0;
                }
            }
            if (leader) *plan_ok = ok ? 1u : 0u;
        }
        pn_plan_sync();
        if (!*plan_ok) return;
        const int in = s % kPnBlk;
        const int buf = (s / kPnBlk) & 1;
        const bool terminal = in == 0 && *final_flag;
        const uint8_t *sym = S.sym(buf);
        const PnHdr *hd = S.hdr(buf);
        int rank[kPnSlotsPerPlanThread], cs[kPnSlotsPerPlanThread], nseq[kPnSlotsPerPlanThread];
#pragma unroll
        for (int k = 0; k < kPnSlotsPerPlanThread; ++k) {
            rank[k] = -1;
            cs[k] = -1;
            nseq[k] = -1;
            const int j = tid + kPnPlanThreads * k;
            if (j >= PS || terminal) continue;
            PnSlot sl = slots[j];
            if (in == 0) {
                const PnHdr h = hd[j];
                sl.blkcnt = h.count;
                sl.blkflags = h.flags;
                if (h.flags & kHdrStart) nseq[k] = h.seq;
                slots[j] = sl;
            }
            if (in < sl.blkcnt) {
                const int c = sym[in * PS + j];
                cs[k] = c;
                rank[k] = atomicAdd(&cnt[(c >> 1) * 2 + (c & 1)], 1);
            }
        }
        pn_plan_sync();
        if (tid < 32) {   // pair bases and the chunk list of step s
            int ne = 0, no = 0;
            if (lane < L.npairs) {
                ne = cnt[lane * 2];
                no = cnt[lane * 2 + 1];
                cnt[lane * 2] = 0;
                cnt[lane * 2 + 1] = 0;
            }
            const int np = ne + no;
            const int nc = (np + kPnRegionCols - 1) / kPnRegionCols;
            int incl = np, cincl = nc;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int a = __shfl_up_sync(0xffffffffu, incl, o);
                const int c = __shfl_up_sync(0xffffffffu, cincl, o);
                if (lane >= o) { incl += a; cincl += c; }
            }
            const int base = incl - np, cbase = cincl - nc;
            if (lane < L.npairs) {
                pinfo[lane * 2] = base;
                pinfo[lane * 2 + 1] = ne;
                PnChunk *ch = S.chunks(s);
                for (int k = 0; k < nc; ++k) {
                    PnChunk d;
                    d.row0 = (uint16_t)(base + k * kPnRegionCols);
                    const int cols = min(kPnRegionCols, np - k * kPnRegionCols);
                    d.ncols = (uint8_t)cols;
                    d.split = (uint8_t)min(max(ne - k * kPnRegionCols, 0), cols);
                    d.pair = (uint8_t)lane;
                    d.pad0 = d.pad1 = d.pad2 = 0;
                    ch[cbase + k] = d;
                }
            }
            const int total_chunks = __shfl_sync(0xffffffffu, cincl, 31);
            if (lane == 0) *S.nch(s) = terminal ? kPnTerminate : total_chunks;
        }
        pn_plan_sync();
        uint2 *rec = S.rec(s - 1);
#pragma unroll
        for (int k = 0; k < kPnSlotsPerPlanThread; ++k) {
            const int j = tid + kPnPlanThreads * k;
            if (j >= PS) continue;
            PnSlot sl = slots[j];
            int row1 = -1;
            if (cs[k] >= 0) {
                const int p = cs[k] >> 1;
                row1 = pinfo[p * 2] + ((cs[k] & 1) ? pinfo[p * 2 + 1] : 0) + rank[k];
            }
            if (s >= 1 && (sl.flags & kSlotActive)) {
                uint2 r;
                r.y = (uint32_t)j | ((sl.flags & kSlotFresh) ? kRecFresh : 0u);
                if (sl.flags & kSlotLast) {
                    r.x = kRecFinish | (uint32_t)j;
                    sl.pend[(s - 1) & 1] = sl.seq;
                } else {
                    // a continuing string is active at step s (blocks never leave it empty)
                    r.x = (uint32_t)max(row1, 0) * 16u;
                }
                rec[sl.row] = r;
            }
            uint8_t nf = 0;
            if (nseq[k] >= 0) sl.seq = nseq[k];
            if (row1 >= 0) {
                nf |= kSlotActive;
                if ((sl.blkflags & kHdrEnd) && in == sl.blkcnt - 1) nf |= kSlotLast;
                if (nseq[k] >= 0) nf |= kSlotFresh;
                sl.row = (int16_t)row1;
                sl.c = (uint8_t)cs[k];
            }
            sl.flags = nf;
            slots[j] = sl;
        }
        pn_plan_sync();
        if (leader) pn_mbar_arrive(S.bar(kBarPlan1 + (s & 3)));
        // ---------------- stage 2 ----------------
        if (tid < 32) {
            bool ok = true;
            if (s >= 2) ok = pn_wait(S.bar(kBarEpi + ((s - 2) & 3)), pn_par(s - 2, 4), abort_flag, P.err, P.wait_cycles);
            if (leader) *plan_ok = ok ? 1u : 0u;
        }
        pn_plan_sync();
        if (!*plan_ok) return;
        if (s >= 2) emit(s - 2);
        if (!terminal) {
            const uint32_t sb = S.sbuf(s & 1);
            for (int j = tid; j < PS; j += kPnPlanThreads) {
                const PnSlot sl = slots[j];
                if ((sl.flags & kSlotFresh) == 0) continue;
                uint8_t *dst = S.base + sb + (uint32_t)sl.row * 16u;
#pragma unroll
                for (int c = 0; c < P.kcols; ++c) *reinterpret_cast<uint4 *>(dst + c * L.lbo) = simg[c];
            }
        }
        pn_fence_async_smem();
        pn_plan_sync();
        if (leader) pn_mbar_arrive(S.bar(kBarPlan2 + (s & 1)));
        if (terminal) {   // the strings that ended at step s-1, then done
            if (s >= 1) {
                if (tid < 32) {
                    const bool ok = pn_wait(S.bar(kBarEpi + ((s - 1) & 3)), pn_par(s - 1, 4), abort_flag,
                                            P.err, P.wait_cycles);
                    if (leader) *plan_ok = ok ? 1u : 0u;
                }
                pn_plan_sync();
                if (*plan_ok) emit(s - 1);
            }
            return;
        }
    }
}

// ---- MMA issuer: warp 8 ----------------------------------------------------------------------------
// KIND: 0 = BF16, 1 = FP16 operands (kind::f16, FP32 sums), 2 = 0/1 int8 operands
// (kind::i8, unsigned, int32 sums: K = 32 an instruction, half the instructions).
template <int KIND>
__device__ void pn_mma(const PnParams &P, const PnShared &S, uint32_t tbase,
                       volatile uint32_t *abort_flag) {
    constexpr bool I8 = KIND == 2;
    constexpr int kKSteps = I8 ? 2 : 4;              // K = 64 as 2 x K32 or 4 x K16
    constexpr uint32_t kACols = I8 ? 16u : 32u;      // TMEM columns of a pair's A
    const int lane = threadIdx.x & 31;
    const PnLayout &L = S.L;
    const uint32_t fmt = KIND == 1 ? 0u : 1u;
    const uint32_t smem_base = pn_smem_u32(S.base);
    const uint32_t desc_hi = (128u >> 4) | (1u << 14);   // SBO = 128 B, descriptor version 1
    const uint32_t nr = (uint32_t)L.nregions;
    uint32_t g = 0;
    for (int t = 0;; ++t) {
        if (!pn_wait(S.bar(kBarPlan2 + (t & 1)), pn_par(t, 2), abort_flag, P.err, P.wait_cycles)) break;
        const int nch = *S.nch(t);
        if (nch == kPnTerminate) break;
        if (t >= 1 && !pn_wait(S.bar(kBarEpi + ((t - 1) & 3)), pn_par(t - 1, 4), abort_flag, P.err, P.wait_cycles)) break;
        const PnChunk *ch = S.chunks(t);
        const uint32_t sb = smem_base + S.sbuf(t & 1);
        bool aborted = false;
        for (int k = 0; k < nch; ++k) {
            const PnChunk d = ch[k];
            const uint32_t r = g % nr, u = g / nr;
            if (u > 0 && !pn_wait(S.bar(kBarEmpty + (int)r), (u - 1) & 1u, abort_flag, P.err, P.wait_cycles)) {
                aborted = true;
                break;
            }
            pn_tc_after();
            if (lane == 0) {
                const uint32_t n16 = ((uint32_t)d.ncols + 15u) & ~15u;
                // instruction descriptor: D format (bits 4-5: F32 = 1, S32 = 2), A and B
                // formats (bits 7-9, 10-12: F16 = 0 / BF16 = 1; U8 = 0), N / 8 (17-22),
                // M / 16 (24-28); both operands K-major
                const uint32_t idesc = I8 ? ((2u << 4) | ((n16 >> 3) << 17) | ((128u >> 4) << 24))
                                          : ((1u << 4) | (fmt << 7) | (fmt << 10) | ((n16 >> 3) << 17) |
                                             ((128u >> 4) << 24));
                const uint32_t td = tbase + (uint32_t)L.ring_base + r * kPnRegionCols;
                // every K step spans two 16-byte core-matrix columns of B (16 states of
                // 16 bits, or 32 states of 8 bits) and 8 TMEM columns of A
#pragma unroll
                for (int kk = 0; kk < kKSteps; ++kk) {
                    const uint32_t saddr = sb + (uint32_t)d.row0 * 16u + (uint32_t)kk * 2u * L.lbo;
                    const uint64_t desc = (uint64_t)(((saddr >> 4) & 0x3FFFu) | ((L.lbo >> 4) << 16)) |
                                          ((uint64_t)desc_hi << 32);
                    const uint32_t ta = tbase + kACols * d.pair + 8u * kk;
                    const uint32_t acc = kk > 0;
                    if constexpr (I8)
                        asm volatile(
                            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::i8 [%0], [%1], %2, %3, p;\n\t}"
                            :: "r"(td), "r"(ta), "l"(desc), "r"(idesc), "r"(acc) : "memory");
                    else
                        asm volatile(
                            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}"
                            :: "r"(td), "r"(ta), "l"(desc), "r"(idesc), "r"(acc) : "memory");
                }
                asm volatile(
                    "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                    :: "r"(S.bar(kBarFull + (int)r)) : "memory");
            }
            __syncwarp();
            ++g;
        }
        if (aborted) break;
    }
    // Drain: every committed chain must have finished before the TMEM is freed.
    for (uint32_t r = 0; r < nr && r < g; ++r) {
        const uint32_t uses = (g - r + nr - 1) / nr;   // commits made to region r
        if (lane == 0) {                               // completion of the last one
            const long long t0 = clock64();
            while (!pn_mbar_test(S.bar(kBarFull + (int)r), (uses - 1) & 1u)) {
                if (clock64() - t0 > kPnDrainCycles) { atomicOr(P.err, kPnErrTimeout); break; }
            }
        }
        __syncwarp();
    }
}

// ---- epilogue: warps 0-7 ---------------------------------------------------------------------------
// Two sets of four warps take alternate chunks. Warp q of a set reads TMEM lanes 32q..32q+31: the
// even symbol's states 32(q&1).. for q < 2, the odd symbol's for q >= 2. The A rows are permuted
// so that in each 16-lane half h the lanes j and j + 8 hold the adjacent states 2j and 2j + 1: a
// 16x256b load then gives thread t (j = t/4) the states 32(q&1) + 16h + 2j, +1 of four columns,
// which it scales, packs into one 32-bit store per pair, and reduces (max) with the seven other
// threads holding the same columns. The scale of a column, 2^-f with f the exponent of
// max|s_t| * R_c (max|s_t| left by the previous step's epilogue), is computed by one lane per
// column and shuffled to the others; warps q = 0, 2 keep the exponent sums.
template <int KIND>
__device__ void pn_epilogue(const PnParams &P, const PnShared &S, uint32_t tbase,
                            volatile uint32_t *abort_flag) {
    constexpr bool I8 = KIND == 2, FP16 = KIND == 1;
    const int lane = threadIdx.x & 31;
    const int ew = threadIdx.x >> 5;
    const int q = ew & 3;                           // TMEM lane quadrant
    const uint32_t set = (uint32_t)(ew >> 2);       // chunk parity this warp drains
    const PnLayout &L = S.L;
    const int j = lane >> 2, cp = lane & 3;
    const int sg0 = 32 * (q & 1) + 2 * j, sg1 = sg0 + 16;   // first states of the two pairs
    // byte offsets of states sg0 and sg1 in a B row: 8 states of 16 bits, or 16 of 8 bits, a
    // core-matrix column
    const uint32_t toff0 = I8 ? (uint32_t)(sg0 >> 4) * L.lbo + (uint32_t)(sg0 & 15)
                              : (uint32_t)(sg0 >> 3) * L.lbo + (uint32_t)(sg0 & 7) * 2u;
    const uint32_t toff1 = I8 ? (uint32_t)(sg1 >> 4) * L.lbo + (uint32_t)(sg1 & 15)
                              : (uint32_t)(sg1 >> 3) * L.lbo + (uint32_t)(sg1 & 7) * 2u;
    const float *accv = reinterpret_cast<const float *>(S.misc() + kMAcc);
    const float a00 = accv[sg0], a01 = accv[sg0 + 1], a10 = accv[sg1], a11 = accv[sg1 + 1];
    const float *rsym = reinterpret_cast<const float *>(S.misc() + kMRsym);
    const bool even = q < 2;
    const bool owner = (q & 1) == 0;
    const bool bmode = P.boolean != 0;
    int32_t *E = S.E();
    const uint32_t nr = (uint32_t)L.nregions;
    uint32_t g = 0;
    if (!pn_wait(S.bar(kBarPlan1), 0u, abort_flag, P.err, P.wait_cycles)) return;
    for (int t = 0;; ++t) {
        const int nch = *S.nch(t);   // plan of step t: waited for in the previous iteration
        if (nch == kPnTerminate) break;
        // records of step t come with the plan of step t+1; the maxima of step t from both sets
        if (!pn_wait(S.bar(kBarPlan1 + ((t + 1) & 3)), pn_par(t + 1, 4), abort_flag, P.err, P.wait_cycles)) break;
        if (t >= 1 && !pn_wait(S.bar(kBarEpi + ((t - 1) & 3)), pn_par(t - 1, 4), abort_flag, P.err, P.wait_cycles)) break;
        const PnChunk *ch = S.chunks(t);
        const uint2 *rec = S.rec(t);
        const float2 *xm = S.xmax(t);
        // a rescale step scales by the maxima that the step before it found
        const bool scale_step = t % P.resc == 0, max_step = (t + 1) % P.resc == 0;
        float *xn = reinterpret_cast<float *>(S.xmax(t + 1)) + (q & 1);
        float *fin = reinterpret_cast<float *>(S.fin(t)) + (q & 1);
        int32_t *finE = S.finE(t);
        uint8_t *snext = S.base + S.sbuf((t + 1) & 1);
        bool aborted = false;
        for (int k = 0; k < nch; ++k, ++g) {
            if ((g & 1u) != set) continue;
            const PnChunk d = ch[k];
            const uint32_t r = g % nr, u = g / nr;
            if (!pn_wait(S.bar(kBarFull + (int)r), u & 1u, abort_flag, P.err, P.wait_cycles)) {
                aborted = true;
                break;
            }
            pn_tc_after();
            const int c_lo = even ? 0 : d.split;
            const int c_hi = even ? d.split : d.ncols;
            const float R = rsym[2 * d.pair + (even ? 0 : 1)];
            const uint32_t tcol = tbase + ((uint32_t)(32 * q) << 16) + (uint32_t)L.ring_base +
                                  r * kPnRegionCols;
            for (int c = c_lo & ~15; c < c_hi; c += 16) {
                uint32_t v0[8], v1[8];
                pn_tmem_ld16x256(tcol + (uint32_t)c, v0);
                pn_tmem_ld16x256(tcol + (16u << 16) + (uint32_t)c, v1);
                // lane l < 16: the scale of column c + l (and the exponent sum of its string)
                float scl = 1.f;
                {
                    const int col = c + lane;
                    if (lane < 16 && col >= c_lo && col < c_hi && bmode) {
                        // Boolean forms: no scaling, the exponent sum stays 0
                        const uint2 rcl = rec[d.row0 + col];
                        if (owner && (rcl.x & kRecFinish)) finE[rcl.y & 1023u] = 0;
                    } else if (lane < 16 && col >= c_lo && col < c_hi && !scale_step) {
                        // no rescale this step: a string that begins starts its exponent sum
                        const uint2 rcl = rec[d.row0 + col];
                        const int jl = (int)(rcl.y & 1023u);
                        if (owner) {
                            const int e = (rcl.y & kRecFresh) ? 0 : E[jl];
                            if (rcl.y & kRecFresh) E[jl] = 0;
                            if (rcl.x & kRecFinish) finE[jl] = e;
                        }
                    } else if (lane < 16 && col >= c_lo && col < c_hi) {
                        const int row = d.row0 + col;
                        const uint2 rcl = rec[row];
                        const bool fresh = (rcl.y & kRecFresh) != 0;
                        const int jl = (int)(rcl.y & 1023u);
                        float m;
                        if (fresh) {
                            m = P.start_max;
                        } else {
                            const float2 x2 = xm[row];
                            m = fmaxf(x2.x, x2.y);
                        }
                        int f = pn_ceil_exp(m * R);
                        f = min(max(f, -125), 125);
                        scl = pn_pow2(-f);
                        if (owner) {
                            const int e = (fresh ? 0 : E[jl]) + f;
                            E[jl] = e;
                            if (rcl.x & kRecFinish) finE[jl] = e;
                        }
                    }
                }
                // this thread's columns: c + {2cp, 2cp+1, 2cp+8, 2cp+9}
                uint2 rc[4];
                bool valid[4];
                float sc[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int co = (i >> 1) * 8 + 2 * cp + (i & 1);
                    const int col = c + co;
                    valid[i] = col >= c_lo && col < c_hi;
                    rc[i] = rec[d.row0 + (valid[i] ? col : c_lo)];
                    sc[i] = __shfl_sync(0xffffffffu, scl, co);
                }
                pn_tmem_wait_ld();
                float x[4][4], m[4];
                bool any_fin = false;
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int ri = (i >> 1) * 4 + (i & 1);
                    if constexpr (I8) {   // int32 path counts: reachable when nonzero
                        x[i][0] = v0[ri] != 0u ? 1.f : 0.f;
                        x[i][1] = v0[ri + 2] != 0u ? 1.f : 0.f;
                        x[i][2] = v1[ri] != 0u ? 1.f : 0.f;
                        x[i][3] = v1[ri + 2] != 0u ? 1.f : 0.f;
                    } else {
                        x[i][0] = __uint_as_float(v0[ri]) * sc[i];       // state sg0
                        x[i][1] = __uint_as_float(v0[ri + 2]) * sc[i];   // sg0 + 1
                        x[i][2] = __uint_as_float(v1[ri]) * sc[i];       // sg1
                        x[i][3] = __uint_as_float(v1[ri + 2]) * sc[i];   // sg1 + 1
                    }
                    if (!I8 && bmode) {   // reachability: exact, the sums are small integers
#pragma unroll
                        for (int z = 0; z < 4; ++z) x[i][z] = x[i][z] > 0.f ? 1.f : 0.f;
                    }
                    const bool fin_i = (rc[i].x & kRecFinish) != 0;
                    const bool keep = valid[i] && !fin_i;
                    any_fin |= valid[i] && fin_i;
                    if (keep) {
                        uint8_t *dst = snext + rc[i].x;
                        if constexpr (I8) {   // two adjacent states, one byte each
                            *reinterpret_cast<uint16_t *>(dst + toff0) =
                                (uint16_t)((x[i][0] != 0.f ? 1u : 0u) | (x[i][1] != 0.f ? 0x100u : 0u));
                            *reinterpret_cast<uint16_t *>(dst + toff1) =
                                (uint16_t)((x[i][2] != 0.f ? 1u : 0u) | (x[i][3] != 0.f ? 0x100u : 0u));
                        } else {
                            *reinterpret_cast<uint32_t *>(dst + toff0) = pn_pack2<FP16>(x[i][0], x[i][1]);
                            *reinterpret_cast<uint32_t *>(dst + toff1) = pn_pack2<FP16>(x[i][2], x[i][3]);
                        }
                    }
                    m[i] = keep ? fmaxf(fmaxf(fabsf(x[i][0]), fabsf(x[i][1])),
                                        fmaxf(fabsf(x[i][2]), fabsf(x[i][3])))
                                : 0.f;
                }
                // column maxima over this warp's 32 states: the 8 threads with the same cp
                // (they set the next rescale step's scale; the Boolean forms do not scale)
                if (!bmode && max_step) {
#pragma unroll
                    for (int o = 4; o < 32; o <<= 1)
#pragma unroll
                        for (int i = 0; i < 4; ++i) m[i] = fmaxf(m[i], __shfl_xor_sync(0xffffffffu, m[i], o));
                    if (j == 0) {
#pragma unroll
                        for (int i = 0; i < 4; ++i)
                            if (valid[i] && !(rc[i].x & kRecFinish)) xn[(rc[i].x >> 4) * 2] = m[i];
                    }
                }
                if (__any_sync(0xffffffffu, any_fin)) {   // last symbols: accept-weighted sums
                    float pz[4];
#pragma unroll
                    for (int i = 0; i < 4; ++i)
                        pz[i] = x[i][0] * a00 + x[i][1] * a01 + x[i][2] * a10 + x[i][3] * a11;
#pragma unroll
                    for (int o = 4; o < 32; o <<= 1)
#pragma unroll
                        for (int i = 0; i < 4; ++i) pz[i] += __shfl_xor_sync(0xffffffffu, pz[i], o);
                    if (j == 0) {
#pragma unroll
                        for (int i = 0; i < 4; ++i)
                            if (valid[i] && (rc[i].x & kRecFinish)) fin[(rc[i].x & 1023u) * 2] = pz[i];
                    }
                }
            }
            pn_tc_before();
            __syncwarp();
            if (lane == 0) pn_mbar_arrive(S.bar(kBarEmpty + (int)r));
        }
        if (aborted) break;
        pn_fence_async_smem();
        __syncwarp();
        if (lane == 0) pn_mbar_arrive(S.bar(kBarEpi + (t & 3)));
    }
}

template <int KIND>
__global__ void __launch_bounds__(kPnThreads, 1) pnfa_tc_kernel(PnParams P) {
    extern __shared__ __align__(1024) uint8_t pn_smem[];
    PnShared S{pn_smem, P.L};
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint8_t *misc = S.misc();
    for (int i = threadIdx.x; i < kPnMiscBytes / 4; i += blockDim.x)
        reinterpret_cast<uint32_t *>(misc)[i] = 0;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 0; i < kBarCount; ++i) {
            uint32_t count = 1;
            if (i >= kBarEpi && i < kBarEpi + 4)
                count = kPnEpiWarps;
            else if (i >= kBarEmpty && i < kBarEmpty + kPnMaxRegions)
                count = 4;
            else if (i >= kBarLoaded && i < kBarLoaded + 2)
                count = kPnLoadWarps;
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(S.bar(i)), "r"(count));
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (threadIdx.x < P.sigma) reinterpret_cast<float *>(misc + kMRsym)[threadIdx.x] = P.rsym[threadIdx.x];
    if (threadIdx.x < 8) reinterpret_cast<uint4 *>(misc + kMStart)[threadIdx.x] = P.start_img[threadIdx.x];
    if (threadIdx.x < 64) reinterpret_cast<float *>(misc + kMAcc)[threadIdx.x] = P.acc[threadIdx.x];
    if (warp == kPnMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(pn_smem_u32(misc + kMTmem)), "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    pn_tc_before();
    __syncthreads();
    pn_tc_after();
    const uint32_t tbase = *reinterpret_cast<volatile uint32_t *>(misc + kMTmem);
    // A operands: pair p -> TMEM columns [32p, 32p + 32) (16-bit values, two a column) or
    // [16p, 16p + 16) (int8, four a column), lane = row of [T[2p]; T[2p+1]]
    if (warp < 4) {
        for (int p = 0; p < P.L.npairs; ++p) {
            if constexpr (KIND == 2) {
                const uint32_t *src = P.tpack + ((size_t)p * 128 + 32 * warp + lane) * 16;
                uint32_t r[16];
#pragma unroll
                for (int k = 0; k < 16; ++k) r[k] = __ldg(src + k);
                pn_tmem_st16(tbase + ((uint32_t)(32 * warp) << 16) + 16u * p, r);
            } else {
                const uint32_t *src = P.tpack + ((size_t)p * 128 + 32 * warp + lane) * 32;
                uint32_t r[32];
#pragma unroll
                for (int k = 0; k < 32; ++k) r[k] = __ldg(src + k);
                pn_tmem_st32(tbase + ((uint32_t)(32 * warp) << 16) + 32u * p, r);
            }
        }
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    }
    pn_tc_before();
    __syncthreads();
    pn_tc_after();
    volatile uint32_t *abort_flag = S.u32(kMAbort);
    if (warp < kPnEpiWarps) pn_epilogue<KIND>(P, S, tbase, abort_flag);
    else if (warp == kPnMmaWarp) pn_mma<KIND>(P, S, tbase, abort_flag);
    else if (warp < kPnLoadWarp0) pn_planner(P, S, abort_flag);
    else pn_loader(P, S, abort_flag);
    pn_tc_before();
    __syncthreads();
    pn_tc_after();
    if (warp == kPnMmaWarp)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tbase), "r"(512));
}

// ---- strings on TMEM lanes (alphabets of at most two symbols) -------------------------------
// Each of four tiles of 128 strings keeps one string on each TMEM lane: the string's state is
// row m of the tile's A operand, K = 64 * sigma, with the 64 states in the K range of the
// string's next symbol and zeros in the other range; B (shared memory) stacks the tables,
// B[n][64 c + q] = T_c[n][q]. One MMA chain (M = 128, N = 64) then gives every string the
// product with its own symbol, D[m][n] = (T_c s_m)[n], with no sorting of strings by symbol.
// The epilogue is thread-local (thread = TMEM lane = string): it reads its 64 states, finds
// their maximum and rescales by an exact power of two, rounds them to the operand type and
// writes its next A row with tcgen05.st; at the string's end it forms the log-likelihood and
// takes the next string from the queue. The MMA warp issues the tiles round robin, so the
// epilogue of one tile overlaps the products of the others. Hand-offs per tile: `full`
// (tcgen05.commit, one arrival) and `ready` (the four epilogue warps, after their A rows and a
// liveness flag are written); every wait is bounded.
constexpr int kLnTiles = 4;
constexpr int kLnEpiWarps = 4 * kLnTiles;   // tile T: warps 4T .. 4T + 3 (lane quadrants 0-3)
constexpr int kLnMmaWarp = kLnEpiWarps;
constexpr int kLnMmaWarps = 2;         // issuers: warp kLnMmaWarp + i takes tiles i, i + 2
constexpr int kLnThreads = 32 * (kLnEpiWarps + kLnMmaWarps);
constexpr int kLnMaxSigma = 4;
constexpr uint32_t kLnLbo = 1024;           // B: bytes between 16-byte K columns (64 rows x 16 B)

struct LnParams {
    const uint8_t *data;
    int64_t total_bytes;
    const int64_t *offsets;
    int64_t n;
    const uint16_t *T16;   // [sigma][64][64] row-major in the operand type (probabilistic forms)
    const float *T32;      // [sigma][64][64] (Boolean forms: a nonzero entry is an edge)
    const float *start;    // [64]
    const float *acc;      // [64] accept weights (Boolean forms: 0/1)
    int sigma;
    int tiles;             // tiles in flight: as many of kLnTiles as fit in the 512 TMEM columns
    uint32_t a_cols;       // TMEM columns of a tile's A (32 sigma, int8: 16 sigma); D follows
    uint32_t tile_cols;    // a_cols + 64, rounded up to 32
    int resc;              // steps between rescales (1 for FP16 operands)
    long long wait_cycles;
    double ll_empty;
    double *loglik;
    uint8_t *accept;
    int32_t *accept_i32;
    unsigned long long *queue;
    uint32_t *err;
};

// A string's symbols: aligned 8-byte words of the batch, the next word loaded while this one
// is used; bytes >= sigma are skipped.
struct LnSym {
    uintptr_t p, e;        // next byte, end of the string (addresses)
    uintptr_t cw;          // address of the word in `cur`
    uint64_t cur, nxt;
};
__device__ __forceinline__ uint64_t ln_word(uintptr_t w, uintptr_t lo, uintptr_t hi) {
    if (w >= lo && w + 8 <= hi) return __ldg(reinterpret_cast<const unsigned long long *>(w));
    uint64_t v = 0;
    for (int k = 0; k < 8; ++k)
        if (w + k >= lo && w + k < hi) v |= (uint64_t)__ldg(reinterpret_cast<const uint8_t *>(w + k)) << (8 * k);
    return v;
}
// next symbol < sigma of the string, or -1 at its end
__device__ __forceinline__ int ln_next(LnSym &s, int sigma, uintptr_t lo, uintptr_t hi) {
    while (s.p < s.e) {
        const uintptr_t w = s.p & ~(uintptr_t)7;
        if (w != s.cw) {
            s.cur = (s.cw != 0 && w == s.cw + 8) ? s.nxt : ln_word(w, lo, hi);
            s.cw = w;
            s.nxt = ln_word(w + 8, lo, hi);
        }
        const int b = (int)((s.cur >> (8 * (s.p & 7))) & 0xffu);
        ++s.p;
        if (b < sigma) return b;
    }
    return -1;
}
// The next string from the queue (index and byte range); seq = -1 when the queue is empty.
// Not inlined: a rare path, kept out of the epilogue's registers.
struct LnRange {
    int64_t seq, a, b;
};
__device__ __noinline__ LnRange ln_take(const LnParams &P) {
    while (true) {
        const unsigned long long idx = atomicAdd(P.queue, 1ull);
        if (idx >= (unsigned long long)P.n) return LnRange{-1, 0, 0};
        const int64_t a = P.offsets[idx], b = P.offsets[idx + 1];
        if (a < 0 || b < a || b > P.total_bytes) {
            atomicOr(P.err, kPnErrOffsets);
            continue;
        }
        return LnRange{(int64_t)idx, a, b};
    }
}
__device__ __noinline__ void ln_empty(const LnParams &P, int64_t seq) {
    pn_write_result(P.loglik, P.accept, P.accept_i32, seq, P.ll_empty);
}

// A finished string: log-likelihood from the accept-weighted sum of its last state and its
// exponent sum.
__device__ __noinline__ void ln_finish(const LnParams &P, int64_t seq, float dot, int E) {
    const double ll = dot > 0.f ? log((double)dot) + (double)E * 0.69314718055994530942 : -INFINITY;
    pn_write_result(P.loglik, P.accept, P.accept_i32, seq, ll);
}

__device__ __forceinline__ void ln_tmem_st8(uint32_t taddr, const uint32_t (&r)[8]) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};"
                 :: "r"(taddr), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]),
                    "r"(r[7])
                 : "memory");
}

__device__ __forceinline__ void ln_tmem_ld32(uint32_t taddr, uint32_t *r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
        "%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
          "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
          "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr) : "memory");
}

// KIND: 0 = BF16, 1 = FP16 operands (kind::f16, FP32 sums, rescaled by exact powers of two);
// 2 = Boolean 0/1 int8 (kind::i8, int32 sums); 3 = Boolean 0/1 BF16. The Boolean forms
// threshold every product to {0, 1} (exact).
template <int KIND>
__global__ void __launch_bounds__(kLnThreads, 1) pnfa_lane_kernel(LnParams P) {
    constexpr bool I8 = KIND == 2, BOOL = KIND >= 2, FP16 = KIND == 1;
    __shared__ __align__(1024) uint8_t s_b[64 * 64 * kLnMaxSigma * 2];
    __shared__ __align__(8) uint64_t s_bar[2 * kLnTiles];   // full[T], then ready[T]
    __shared__ uint32_t s_tmem, s_abort;
    // liveness flags of a tile's four warps per ready phase parity (a warp can write the next
    // phase's flag while another still reads this phase's)
    __shared__ uint32_t s_alive[kLnTiles][2][4];
    __shared__ float s_acc[64], s_start[64];
    __shared__ uint32_t s_start8[16];   // int8 Boolean form: the start set, four states a word
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int sig = P.sigma;
    const int K = 64 * sig;
    // B: row n = destination state, K index 64 c + q (symbol c, source state q); 16-byte K
    // columns kLnLbo bytes apart, rows 16 bytes apart inside 8-row core matrices
    if constexpr (I8) {
        for (int t = threadIdx.x; t < 64 * (K / 16); t += blockDim.x) {
            const int n = t & 63, kc = t >> 6;
            uint32_t w[4] = {0u, 0u, 0u, 0u};
            for (int j = 0; j < 16; ++j) {
                const int k = 16 * kc + j;
                if (P.T32[((size_t)(k >> 6) * 64 + n) * 64 + (k & 63)] != 0.f) w[j >> 2] |= 1u << (8 * (j & 3));
            }
            *reinterpret_cast<uint4 *>(s_b + kc * kLnLbo + (n >> 3) * 128 + (n & 7) * 16) =
                make_uint4(w[0], w[1], w[2], w[3]);
        }
    } else {
        for (int t = threadIdx.x; t < 64 * (K / 8); t += blockDim.x) {
            const int n = t & 63, kc = t >> 6;
            uint32_t w[4];
            for (int j = 0; j < 4; ++j) {
                const int k = 8 * kc + 2 * j;   // k and k + 1 belong to the same symbol
                const size_t o = ((size_t)(k >> 6) * 64 + n) * 64 + (k & 63);
                uint32_t lo16, hi16;
                if constexpr (BOOL) {
                    lo16 = P.T32[o] != 0.f ? 0x3F80u : 0u;   // BF16 1.0
                    hi16 = P.T32[o + 1] != 0.f ? 0x3F80u : 0u;
                } else {
                    lo16 = P.T16[o];
                    hi16 = P.T16[o + 1];
                }
                w[j] = lo16 | (hi16 << 16);
            }
            *reinterpret_cast<uint4 *>(s_b + kc * kLnLbo + (n >> 3) * 128 + (n & 7) * 16) =
                make_uint4(w[0], w[1], w[2], w[3]);
        }
    }
    if (threadIdx.x < 64) {
        s_acc[threadIdx.x] = P.acc[threadIdx.x];
        s_start[threadIdx.x] = P.start[threadIdx.x];
    }
    if (threadIdx.x < 16) {
        uint32_t w = 0u;
        for (int b = 0; b < 4; ++b) w |= (P.start[4 * threadIdx.x + b] != 0.f ? 1u : 0u) << (8 * b);
        s_start8[threadIdx.x] = w;
    }
    if (threadIdx.x == 0) {
        s_abort = 0u;
        for (int T = 0; T < kLnTiles; ++T) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(pn_smem_u32(&s_bar[T])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;" :: "r"(pn_smem_u32(&s_bar[kLnTiles + T])));
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == kLnMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(pn_smem_u32(&s_tmem)), "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    pn_fence_async_smem();   // B, written by these stores, is read by the tensor cores
    pn_tc_before();
    __syncthreads();
    pn_tc_after();
    const uint32_t tbase = *reinterpret_cast<volatile uint32_t *>(&s_tmem);
    volatile uint32_t *abort_flag = &s_abort;
    if (warp < kLnEpiWarps && (warp >> 2) < P.tiles) {   // fewer tiles for larger alphabets
        const int T = warp >> 2, qd = warp & 3;
        const uint32_t tA = tbase + ((uint32_t)(32 * qd) << 16) + (uint32_t)T * P.tile_cols;
        const uint32_t tD = tA + P.a_cols;
        const uint32_t bar_full = pn_smem_u32(&s_bar[T]), bar_ready = pn_smem_u32(&s_bar[kLnTiles + T]);
        const uintptr_t lo = reinterpret_cast<uintptr_t>(P.data), hi = lo + (uintptr_t)P.total_bytes;
        LnSym sy{0, 0, 0, 0, 0};
        int64_t seq = -1;
        int c = 0, E = 0, since = 0;
        // the next string with its first symbol in c (strings with no symbol get their result
        // at once); false when the queue is empty
        auto fetch = [&]() -> bool {
            while (true) {
                const LnRange r = ln_take(P);
                if (r.seq < 0) return false;
                sy.p = lo + (uintptr_t)r.a;
                sy.e = lo + (uintptr_t)r.b;
                sy.cw = 0;
                c = ln_next(sy, sig, lo, hi);
                if (c >= 0) {
                    seq = r.seq;
                    return true;
                }
                ln_empty(P, r.seq);
            }
        };
        bool live = fetch();
        // A row chunk j (states 32 j .. 32 j + 31) of this string: in the K range of symbol c, zeros
        // in the other ranges (tcgen05.st is warp-wide; each thread supplies its own row)
        auto store_chunk = [&](int j, const float (&v)[32]) {
            if constexpr (I8) {
                uint32_t r[8];
#pragma unroll
                for (int k = 0; k < 8; ++k)
                    r[k] = (v[4 * k] != 0.f ? 1u : 0u) | (v[4 * k + 1] != 0.f ? 0x100u : 0u) |
                           (v[4 * k + 2] != 0.f ? 0x10000u : 0u) | (v[4 * k + 3] != 0.f ? 0x1000000u : 0u);
                for (int h = 0; h < sig; ++h) {
                    uint32_t q[8];
#pragma unroll
                    for (int k = 0; k < 8; ++k) q[k] = h == c ? r[k] : 0u;
                    ln_tmem_st8(tA + 16u * (uint32_t)h + 8u * (uint32_t)j, q);
                }
            } else {
                uint32_t r[16];
#pragma unroll
                for (int k = 0; k < 16; ++k) r[k] = pn_pack2<FP16>(v[2 * k], v[2 * k + 1]);
                for (int h = 0; h < sig; ++h) {
                    uint32_t q[16];
#pragma unroll
                    for (int k = 0; k < 16; ++k) q[k] = h == c ? r[k] : 0u;
                    pn_tmem_st16(tA + 32u * (uint32_t)h + 16u * (uint32_t)j, q);
                }
            }
        };
        auto start_chunk = [&](int j, float (&v)[32]) {
#pragma unroll
            for (int i = 0; i < 32; ++i) {
                const float s0 = s_start[32 * j + i];
                v[i] = live ? (BOOL ? (s0 != 0.f ? 1.f : 0.f) : s0) : 0.f;
            }
        };
        auto d_value = [&](uint32_t w) -> float {
            if constexpr (I8) return w != 0u ? 1.f : 0.f;
            else if constexpr (BOOL) return __uint_as_float(w) > 0.f ? 1.f : 0.f;
            else return __uint_as_float(w);
        };
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            float v[32];
            start_chunk(j, v);
            store_chunk(j, v);
        }
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        pn_tc_before();
        const uint32_t FULL = 0xffffffffu;
        for (uint32_t ph = 0;; ph ^= 1u) {
            const uint32_t any_live = __any_sync(FULL, live) ? 1u : 0u;
            if (lane == 0) {
                *reinterpret_cast<volatile uint32_t *>(&s_alive[T][ph][qd]) = any_live;
                pn_mbar_arrive(bar_ready);
            }
            __syncwarp();
            // all four warps of the tile have arrived: their flags decide whether it goes on
            if (!pn_wait_park(bar_ready, ph, abort_flag, P.err, P.wait_cycles)) break;
            const volatile uint32_t *fl = s_alive[T][ph];
            if ((fl[0] | fl[1] | fl[2] | fl[3]) == 0u) break;
            if (!pn_wait_park(bar_full, ph, abort_flag, P.err, P.wait_cycles)) break;
            pn_tc_after();
            // D row = this string's state after its symbol; what comes next
            const int nc = live ? ln_next(sy, sig, lo, hi) : -1;
            const bool ending = live && nc < 0;
            bool resc_now = false;
            if (live && !ending) {
                c = nc;
                if (!BOOL && ++since >= P.resc) {
                    since = 0;
                    resc_now = true;
                }
            }
            bool from_d = live && !ending;
            float sc = 1.f;
            if (__any_sync(FULL, ending || resc_now)) {   // pass 1: the row's maximum, accept sum
                float m = 0.f, dot = 0.f;
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    uint32_t d[32];
                    ln_tmem_ld32(tD + 32u * (uint32_t)j, d);
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                    for (int i = 0; i < 32; ++i) {
                        const float v = d_value(d[i]);
                        m = fmaxf(m, fabsf(v));
                        dot = fmaf(s_acc[32 * j + i], v, dot);
                    }
                }
                if (ending) {   // the string's log-likelihood, then the next string
                    ln_finish(P, seq, dot, E);
                    live = fetch();
                    E = 0;
                    since = 0;
                } else if (resc_now) {   // exact power-of-two rescale
                    int f = pn_ceil_exp(m);
                    f = min(max(f, -125), 125);
                    sc = pn_pow2(-f);
                    E += f;
                }
            }
            if (!live) c = 0;
            // pass 2: the next A row, 32 states at a time
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                uint32_t d[32];
                ln_tmem_ld32(tD + 32u * (uint32_t)j, d);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if constexpr (I8) {   // 0/1 bytes straight from the int32 path counts
                    uint32_t r[8];
#pragma unroll
                    for (int k = 0; k < 8; ++k)
                        r[k] = from_d ? ((d[4 * k] != 0u ? 1u : 0u) | (d[4 * k + 1] != 0u ? 0x100u : 0u) |
                                         (d[4 * k + 2] != 0u ? 0x10000u : 0u) |
                                         (d[4 * k + 3] != 0u ? 0x1000000u : 0u))
                                      : (live ? s_start8[8 * j + k] : 0u);
                    for (int h = 0; h < sig; ++h) {
                        uint32_t q[8];
#pragma unroll
                        for (int k = 0; k < 8; ++k) q[k] = h == c ? r[k] : 0u;
                        ln_tmem_st8(tA + 16u * (uint32_t)h + 8u * (uint32_t)j, q);
                    }
                    continue;
                }
                float v[32];
                if (from_d) {
#pragma unroll
                    for (int i = 0; i < 32; ++i) v[i] = d_value(d[i]) * sc;
                } else {
                    start_chunk(j, v);
                }
                store_chunk(j, v);
            }
            asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            pn_tc_before();
        }
    } else if (warp >= kLnEpiWarps) {
        // MMA issuers: each its tiles round robin, one K chain (4 sigma K16 or 2 sigma K32 steps)
        // each (two issuing threads: one alone spends ~135 cycles an instruction)
        const uint32_t fmt = KIND == 1 ? 0u : 1u;
        const uint32_t idesc = I8 ? ((2u << 4) | ((64u >> 3) << 17) | ((128u >> 4) << 24))
                                  : ((1u << 4) | (fmt << 7) | (fmt << 10) | ((64u >> 3) << 17) |
                                     ((128u >> 4) << 24));
        const uint32_t sb = pn_smem_u32(s_b);
        const uint64_t desc0 = (uint64_t)(((sb >> 4) & 0x3FFFu) | ((kLnLbo >> 4) << 16)) |
                               ((uint64_t)((128u >> 4) | (1u << 14)) << 32);
        const int nk = I8 ? 2 * sig : 4 * sig;
        const int mw = warp - kLnMmaWarp;
        uint32_t done = 0u, phs = 0u, pend = 0u;
        for (int T = 0; T < kLnTiles; ++T)
            if (T % kLnMmaWarps != mw || T >= P.tiles) done |= 1u << T;
        bool aborted = false;
        while (done != (1u << kLnTiles) - 1u && !aborted) {
            for (int T = mw; T < kLnTiles; T += kLnMmaWarps) {
                if ((done >> T) & 1u) continue;
                if (!pn_wait_park(pn_smem_u32(&s_bar[kLnTiles + T]), (phs >> T) & 1u, abort_flag, P.err, P.wait_cycles)) {
                    aborted = true;
                    break;
                }
                pn_tc_after();
                const volatile uint32_t *fl = s_alive[T][(phs >> T) & 1u];
                phs ^= 1u << T;
                pend &= ~(1u << T);   // the epilogue has read the previous product
                if ((fl[0] | fl[1] | fl[2] | fl[3]) == 0u) {
                    done |= 1u << T;
                    continue;
                }
                if (lane == 0) {
                    // K step kk: B 2 kLnLbo bytes further (+128 in the descriptor's start field,
                    // which stays below 2^14 for shared addresses), A 8 TMEM columns further
                    const uint32_t tA = tbase + (uint32_t)T * P.tile_cols, tD = tA + P.a_cols;
                    for (int kk = 0; kk < nk; ++kk) {
                        const uint64_t desc = desc0 + (uint64_t)(128u * (uint32_t)kk);
                        const uint32_t ta = tA + 8u * (uint32_t)kk;
                        const uint32_t acc = kk > 0;
                        if constexpr (I8)
                            asm volatile(
                                "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                                "tcgen05.mma.cta_group::1.kind::i8 [%0], [%1], %2, %3, p;\n\t}"
                                :: "r"(tD), "r"(ta), "l"(desc), "r"(idesc), "r"(acc) : "memory");
                        else
                            asm volatile(
                                "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                                "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}"
                                :: "r"(tD), "r"(ta), "l"(desc), "r"(idesc), "r"(acc) : "memory");
                    }
                    asm volatile(
                        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                        :: "r"(pn_smem_u32(&s_bar[T])) : "memory");
                }
                __syncwarp();
                pend |= 1u << T;
            }
        }
        // a product committed but not read must be complete before the TMEM is freed
        for (int T = 0; T < kLnTiles; ++T) {
            if (!((pend >> T) & 1u)) continue;
            if (lane == 0) {
                const uint32_t par = ((phs >> T) & 1u) ^ 1u;   // the phase of the last commit
                const long long t0 = clock64();
                while (!pn_mbar_test(pn_smem_u32(&s_bar[T]), par)) {
                    if (clock64() - t0 > kPnDrainCycles) { atomicOr(P.err, kPnErrTimeout); break; }
                }
            }
            __syncwarp();
        }
    }
    pn_tc_before();
    __syncthreads();
    pn_tc_after();
    if (warp == kLnMmaWarp)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tbase), "r"(512));
}

// ---- plain FP32 form -------------------------------------------------------------------------
struct PnPlainParams {
    const uint8_t *data;
    int64_t total_bytes;
    const int64_t *offsets;
    int64_t n;
    const float *T;         // [sigma][64][64]
    const float *start;     // [64]
    const float *acc;       // [64]
    int sigma;
    double ll_empty;
    double *loglik;
    uint8_t *accept;
    int32_t *accept_i32;
    unsigned long long *queue;
    uint32_t *err;
};

constexpr int kPnPlainWarps = 8;

__global__ void __launch_bounds__(kPnPlainWarps * 32) pnfa_plain_kernel(PnPlainParams P) {
    __shared__ __align__(16) float sv[kPnPlainWarps][64];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    float *v = sv[w];
    for (;;) {
        unsigned long long idx = 0;
        if (lane == 0) idx = atomicAdd(P.queue, 1ull);
        idx = __shfl_sync(0xffffffffu, idx, 0);
        if (idx >= (unsigned long long)P.n) break;
        const int64_t p0 = P.offsets[idx], p1 = P.offsets[idx + 1];
        if (p0 < 0 || p1 < p0 || p1 > P.total_bytes) {
            if (lane == 0) atomicOr(P.err, kPnErrOffsets);
            continue;
        }
        float s0 = P.start[lane], s1 = P.start[lane + 32];
        int64_t E = 0;
        for (int64_t base = p0; base < p1; base += 32) {
            const int64_t pl = base + lane;
            const uint32_t mybyte = pl < p1 ? P.data[pl] : 255u;
            const int nb = (int)min((int64_t)32, p1 - base);
            for (int k = 0; k < nb; ++k) {
                const uint32_t c = __shfl_sync(0xffffffffu, mybyte, k);
                if (c >= (uint32_t)P.sigma) continue;
                v[lane] = s0;
                v[lane + 32] = s1;
                __syncwarp();
                const float4 *r0 = reinterpret_cast<const float4 *>(P.T + ((size_t)c * 64 + lane) * 64);
                const float4 *r1 = reinterpret_cast<const float4 *>(P.T + ((size_t)c * 64 + lane + 32) * 64);
                const float4 *vv = reinterpret_cast<const float4 *>(v);
                float a0 = 0.f, a1 = 0.f;
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    const float4 x = vv[q];
                    const float4 t0 = __ldg(r0 + q), t1 = __ldg(r1 + q);
                    a0 = fmaf(t0.x, x.x, a0); a0 = fmaf(t0.y, x.y, a0);
                    a0 = fmaf(t0.z, x.z, a0); a0 = fmaf(t0.w, x.w, a0);
                    a1 = fmaf(t1.x, x.x, a1); a1 = fmaf(t1.y, x.y, a1);
                    a1 = fmaf(t1.z, x.z, a1); a1 = fmaf(t1.w, x.w, a1);
                }
                __syncwarp();
                float m = fmaxf(fabsf(a0), fabsf(a1));
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
                if (m > 0.f) {
                    // frexp exponent of m: m = mant * 2^e, mant in [0.5, 1)
                    uint32_t bits = __float_as_uint(m);
                    int pre = 0;
                    if (((bits >> 23) & 0xFFu) == 0) {   // subnormal: lift by 2^64 first
                        m *= 18446744073709551616.0f;
                        bits = __float_as_uint(m);
                        pre = 64;
                    }
                    const int e = (int)((bits >> 23) & 0xFFu) - 126 - pre;
                    // scale by 2^-e in (at most) two exact steps
                    const int e1 = max(min(e, 126), -126);
                    const float sc1 = pn_pow2(-e1);
                    s0 = a0 * sc1;
                    s1 = a1 * sc1;
                    if (e != e1) {
                        const float sc2 = pn_pow2(-(e - e1));
                        s0 *= sc2;
                        s1 *= sc2;
                    }
                    E += e;
                } else {
                    s0 = 0.f;
                    s1 = 0.f;
                }
            }
        }
        float d = s0 * P.acc[lane] + s1 * P.acc[lane + 32];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
        if (lane == 0) {
            const double ll = d > 0.f ? log((double)d) + (double)E * 0.69314718055994530942 : -INFINITY;
            pn_write_result(P.loglik, P.accept, P.accept_i32, (int64_t)idx, ll);
        }
    }
}

// CUDA-core form with 16-bit tables in shared memory (modes BF16_CC / FP16_CC):
// the low-latency chain. The transition tables of all symbols (sigma x 8 KB)
// are copied into shared memory once per CTA, so a step reads no global
// memory; the state stays in FP32. Four warps advance one string: thread
// (o, h) = (gt / 2, gt % 2) of the group forms the dot product of row o of
// T[c] with states 32h .. 32h + 31 (four independent FMA chains of eight),
// the two halves meet by one shuffle and the new state goes to the other of
// two state buffers, so a step costs one named barrier of the group. Rows are
// stored with their 16-byte chunks permuted by (o & 3), so the eight lanes of
// a quarter-warp read eight different chunks (no bank conflicts), and the two
// state halves sit 144 bytes apart for the same reason. Every `resc` steps
// the group finds max|s| (warp maxima through shared memory) and the next
// step scales by the exact power of two 2^-f and adds f to the exponent sum,
// as the plain kernel does every step (power-of-two scaling is exact, so only
// the rounding of the products differs between the forms). CTA = four groups
// = four strings in flight; the per-step latency is far below the
// tensor-core kernel's (which advances many strings per step): the form for
// few strings, long ones included (serving).
template <bool FP16>
__device__ __forceinline__ float pn_h2f(uint32_t h) {
    if constexpr (FP16) return __half2float(__ushort_as_half((unsigned short)h));
    else return __uint_as_float(h << 16);
}

constexpr int kChainThreads = 128;   // one string per group of four warps
constexpr int kChainGroups = 4;      // strings per CTA
struct ChainShared {
    float s[2][72];        // the state, double-buffered; state i at i + (i >= 32 ? 4 : 0)
    float wmax[2][4];      // warp maxima of a check step (by its parity)
    float red[4];
    unsigned long long idx;
    uint32_t pad[2];
};
constexpr uint32_t kChainSharedBytes = kChainGroups * (uint32_t)sizeof(ChainShared);

__device__ __forceinline__ void pn_group_bar(int g) {
    asm volatile("bar.sync %0, %1;" :: "r"(g + 1), "r"(kChainThreads) : "memory");
}
__device__ __forceinline__ int pn_sidx(int i) { return i + (i >= 32 ? 4 : 0); }

template <bool FP16>
__global__ void __launch_bounds__(kChainThreads * kChainGroups, 1)
pnfa_chain_kernel(PnPlainParams P, const uint16_t *T16, int resc) {
    extern __shared__ __align__(16) uint8_t pn_ch_smem[];
    const uint32_t FULL = 0xffffffffu;
    const int g = threadIdx.x / kChainThreads, gt = threadIdx.x % kChainThreads;
    const int lane = threadIdx.x & 31, wg = gt >> 5;
    const int o = gt >> 1, h = gt & 1, sw = o & 3;
    uint4 *tbl = reinterpret_cast<uint4 *>(pn_ch_smem);   // [sigma][64 rows][8 chunks], chunk p at p ^ (row & 3)
    ChainShared *cs = reinterpret_cast<ChainShared *>(pn_ch_smem + (size_t)P.sigma * 8192) + g;
    {
        const uint4 *src = reinterpret_cast<const uint4 *>(T16);
        const int chunks = P.sigma * 64 * 8;
        for (int i = threadIdx.x; i < chunks; i += blockDim.x) {
            const int row = i >> 3, p = i & 7;
            tbl[(row << 3) | (p ^ (row & 3))] = src[i];
        }
        __syncthreads();
    }
    const float acc_o = gt < 64 ? P.acc[gt] : 0.f;
    const float start_o = gt < 64 ? P.start[gt] : 0.f;
    for (;;) {
        if (gt == 0) cs->idx = atomicAdd(P.queue, 1ull);
        pn_group_bar(g);
        const unsigned long long idx = cs->idx;
        if (idx >= (unsigned long long)P.n) break;
        const int64_t p0 = P.offsets[idx], p1 = P.offsets[idx + 1];
        if (p0 < 0 || p1 < p0 || p1 > P.total_bytes) {
            if (gt == 0) atomicOr(P.err, kPnErrOffsets);
            pn_group_bar(g);
            continue;
        }
        if (gt < 64) cs->s[0][pn_sidx(gt)] = start_o;
        pn_group_bar(g);
        int cur = 0;          // the buffer holding the state
        int64_t E = 0;
        bool any = false;     // some symbol was applied
        bool pend = false;    // the previous step was a check step
        uint32_t par = 0;     // parity of the step
        int chk = resc;       // steps to the next check step
        for (int64_t base = p0; base < p1; base += 32) {
            const int64_t pl = base + lane;
            const uint32_t byte = pl < p1 ? P.data[pl] : 255u;
            uint32_t m = __ballot_sync(FULL, byte < (uint32_t)P.sigma);
            while (m) {
                const int src = __ffs(m) - 1;
                m &= m - 1;
                const uint32_t c = __shfl_sync(FULL, byte, src);
                const uint4 *row = tbl + ((c * 64 + o) << 3);
                float sc = 1.f;
                if (pend) {   // the maxima of the previous step's outputs: exact power-of-two scale
                    const float4 w4 = *reinterpret_cast<const float4 *>(cs->wmax[par ^ 1u]);
                    const float mx = fmaxf(fmaxf(w4.x, w4.y), fmaxf(w4.z, w4.w));
                    const uint32_t eb = (__float_as_uint(mx) >> 23) & 0xFFu;
                    if (mx > 0.f && eb != 0) {
                        const int f = min(max((int)eb - 126, -125), 125);
                        sc = pn_pow2(-f);
                        E += f;
                    }
                    pend = false;
                }
                const float4 *sv = reinterpret_cast<const float4 *>(&cs->s[cur][h * 36]);
                float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const uint4 t = row[(4 * h + k) ^ sw];   // states 32h + 8k .. + 7 of row o
                    const float4 x0 = sv[2 * k], x1 = sv[2 * k + 1];
                    a0 = fmaf(pn_h2f<FP16>(t.x & 0xFFFFu), x0.x, a0);
                    a1 = fmaf(pn_h2f<FP16>(t.x >> 16), x0.y, a1);
                    a2 = fmaf(pn_h2f<FP16>(t.y & 0xFFFFu), x0.z, a2);
                    a3 = fmaf(pn_h2f<FP16>(t.y >> 16), x0.w, a3);
                    a0 = fmaf(pn_h2f<FP16>(t.z & 0xFFFFu), x1.x, a0);
                    a1 = fmaf(pn_h2f<FP16>(t.z >> 16), x1.y, a1);
                    a2 = fmaf(pn_h2f<FP16>(t.w & 0xFFFFu), x1.z, a2);
                    a3 = fmaf(pn_h2f<FP16>(t.w >> 16), x1.w, a3);
                }
                float sum = (a0 + a1) + (a2 + a3);
                sum += __shfl_xor_sync(FULL, sum, 1);
                sum *= sc;
                if (--chk == 0) {   // a check step: this group's max|s'|
                    float mx = fabsf(sum);
#pragma unroll
                    for (int d = 2; d < 32; d <<= 1) mx = fmaxf(mx, __shfl_xor_sync(FULL, mx, d));
                    if (lane == 0) cs->wmax[par][wg] = mx;
                    pend = true;
                    chk = resc;
                }
                if (h == 0) cs->s[cur ^ 1][pn_sidx(o)] = sum;
                cur ^= 1;
                par ^= 1u;
                any = true;
                pn_group_bar(g);
            }
        }
        if (!any) {
            if (gt == 0) pn_write_result(P.loglik, P.accept, P.accept_i32, (int64_t)idx, P.ll_empty);
        } else {
            float d = gt < 64 ? cs->s[cur][pn_sidx(gt)] * acc_o : 0.f;
#pragma unroll
            for (int k = 16; k > 0; k >>= 1) d += __shfl_xor_sync(FULL, d, k);
            if (lane == 0) cs->red[wg] = d;
            pn_group_bar(g);
            if (gt == 0) {
                const float dot = (cs->red[0] + cs->red[1]) + (cs->red[2] + cs->red[3]);
                const double ll = dot > 0.f ? log((double)dot) + (double)E * 0.69314718055994530942 : -INFINITY;
                pn_write_result(P.loglik, P.accept, P.accept_i32, (int64_t)idx, ll);
            }
        }
        pn_group_bar(g);   // the slot (idx, red) is free again
    }
}

}  // namespace trex

// ---- handle -----------------------------------------------------------------------------------
struct trex_pnfa {
    int n_states = 0, sigma = 0, npairs = 0, n_sms = 0;
    double ll_empty = 0.0, ll_empty_bool = 0.0;
    // tensor-core tables: [bf16, fp16, Boolean 0/1 in bf16, Boolean 0/1 in int8]
    float start_max16[4] = {0.f, 0.f, 0.f, 0.f};
    float *d_T32 = nullptr, *d_start32 = nullptr, *d_acc = nullptr, *d_acc_bool = nullptr;
    uint16_t *d_T16[2] = {nullptr, nullptr};   // [sigma][64][64] row-major: bf16, fp16
    uint32_t *d_tpack[4] = {nullptr, nullptr, nullptr, nullptr};
    float *d_rsym[4] = {nullptr, nullptr, nullptr, nullptr};
    uint4 *d_simg[4] = {nullptr, nullptr, nullptr, nullptr};
    uint8_t *d_misc = nullptr;   // [0,8) queue, [8,12) error word
    // steps between the rescale checks of the chain kernel per 16-bit table type: 4
    // when the tables' growth bound allows (max |T s| / max |s| <= 16 a step, so five
    // unchecked steps stay far inside FP32), else every step
    int chain_resc[2] = {1, 1};
    int tc_resc = 1;   // the tensor-core kernel's rescale period for BF16 operands (same bound)
    int sm_limit = 0;  // launches size their grids for at most this many SMs (0: all)
};

namespace trex {

static uint16_t pn_host16(float x, bool fp16) {
    if (fp16) {
        const __half h = __float2half_rn(x);
        return __half_as_ushort(h);
    }
    const __nv_bfloat16 b = __float2bfloat16_rn(x);
    return __bfloat16_as_ushort(b);
}
static float pn_host16_to_f(uint16_t v, bool fp16) {
    if (fp16) return __half2float(__ushort_as_half(v));
    return __bfloat162float(__ushort_as_bfloat16(v));
}

static void pn_free(trex_pnfa *h) {
    cudaFree(h->d_T32);
    cudaFree(h->d_T16[0]);
    cudaFree(h->d_T16[1]);
    cudaFree(h->d_start32);
    cudaFree(h->d_acc);
    cudaFree(h->d_acc_bool);
    for (int k = 0; k < 4; ++k) {
        cudaFree(h->d_tpack[k]);
        cudaFree(h->d_rsym[k]);
        cudaFree(h->d_simg[k]);
    }
    cudaFree(h->d_misc);
}

static int64_t pn_sms(const trex_pnfa *h) {
    return h->sm_limit > 0 ? std::min(h->sm_limit, h->n_sms) : h->n_sms;
}

static int pn_choose(const trex_pnfa *h, int64_t n, int *grid, int *p_sub) {
    int pmax = 0;
    for (int p = 32; p <= kPnMaxPSub; p += 32)
        if (pn_layout(p, h->sigma).total <= kPnSmemCap) pmax = p;
    if (pmax == 0) return TREX_ERR_SHAPE;
    const int64_t sms = pn_sms(h);
    if (n <= sms * 64) {
        *grid = (int)std::max<int64_t>(1, (n + 63) / 64);
        *p_sub = 64;
    } else {
        *grid = (int)sms;
        int64_t need = (n + sms - 1) / sms;
        need = (need + 31) / 32 * 32;
        *p_sub = (int)std::min<int64_t>(need, pmax);
    }
    return TREX_OK;
}

}  // namespace trex

extern "C" {

int trex_pnfa_create(int n_states, int sigma, const float *T, const float *start, const float *accept,
                     trex_pnfa **out) {
    using namespace trex;
    if (!out) return TREX_ERR_ARG;
    *out = nullptr;
    if (n_states < 1 || n_states > kPnStates || sigma < 1 || sigma > 255 || !T || !start || !accept)
        return TREX_ERR_ARG;
    trex_pnfa *h = new (std::nothrow) trex_pnfa();
    if (!h) return TREX_ERR_OOM;
    h->n_states = n_states;
    h->sigma = sigma;
    h->npairs = (sigma + 1) / 2;
    h->n_sms = sm_count();
    if (h->n_sms <= 0) {
        delete h;
        set_last_error_msg("trex_pnfa_create: no CUDA device");
        return TREX_ERR_SHAPE;
    }
    const int N = n_states;
    // padded FP32 copies (states >= n_states are zero: they never gain mass)
    std::vector<float> T32((size_t)sigma * 64 * 64, 0.f), s32(64, 0.f), a32(64, 0.f);
    for (int c = 0; c < sigma; ++c)
        for (int d = 0; d < N; ++d)
            for (int q = 0; q < N; ++q) T32[((size_t)c * 64 + d) * 64 + q] = T[((size_t)c * N + d) * N + q];
    double dot = 0.0;
    for (int i = 0; i < N; ++i) {
        s32[i] = start[i];
        a32[i] = accept[i];
        dot += (double)start[i] * (double)accept[i];
    }
    h->ll_empty = dot > 0.0 ? std::log(dot) : -INFINITY;
    // Boolean form: every nonzero entry is an edge (1), start and accept are sets
    std::vector<float> Tb(T32.size()), sb(64), ab(64);
    for (size_t i = 0; i < T32.size(); ++i) Tb[i] = T32[i] != 0.f ? 1.f : 0.f;
    int nacc = 0;
    for (int i = 0; i < 64; ++i) {
        sb[i] = s32[i] != 0.f ? 1.f : 0.f;
        ab[i] = a32[i] != 0.f ? 1.f : 0.f;
        nacc += sb[i] != 0.f && ab[i] != 0.f;
    }
    h->ll_empty_bool = nacc ? std::log((double)nacc) : -INFINITY;
    std::vector<uint32_t> tp[4];
    std::vector<float> rs[4];
    std::vector<uint4> simg[4];
    for (int k = 0; k < 3; ++k) {
        const bool fp16 = k == 1;
        const std::vector<float> &Tk = k == 2 ? Tb : T32;
        const std::vector<float> &sk = k == 2 ? sb : s32;
        tp[k].assign((size_t)h->npairs * 128 * 32, 0u);
        rs[k].assign(sigma, 0.f);
        for (int c = 0; c < sigma; ++c) {
            const int p = c >> 1, half_ = c & 1;
            double rmax = 0.0;
            for (int rr = 0; rr < 64; ++rr) {
                // A row rr holds destination state d: in each group of 16 rows, rows 0-7 are the
                // even states and rows 8-15 the odd ones, so TMEM lanes j and j+8 of a 16-lane
                // half carry the adjacent states 2j and 2j+1 (the epilogue's 16x256b loads)
                const int d = (rr & ~15) | ((rr & 7) << 1) | ((rr >> 3) & 1);
                double rsum = 0.0;
                for (int q = 0; q < 64; ++q) {
                    const uint16_t v = pn_host16(Tk[((size_t)c * 64 + d) * 64 + q], fp16);
                    rsum += std::fabs((double)pn_host16_to_f(v, fp16));
                    uint32_t &w = tp[k][((size_t)p * 128 + half_ * 64 + rr) * 32 + (q >> 1)];
                    w |= (uint32_t)v << (16 * (q & 1));
                }
                rmax = std::max(rmax, rsum);
            }
            // a little above the largest row sum: bounds max|T s| / max|s| through FP32 rounding
            rs[k][c] = (float)(rmax * (1.0 + 1.0 / 64));
        }
        simg[k].assign(8, make_uint4(0, 0, 0, 0));
        float smax = 0.f;
        for (int i = 0; i < 64; ++i) {
            const uint16_t v = pn_host16(sk[i], fp16);
            smax = std::max(smax, std::fabs(pn_host16_to_f(v, fp16)));
            uint32_t *w = reinterpret_cast<uint32_t *>(&simg[k][i >> 3]);
            w[(i & 7) >> 1] |= (uint32_t)v << (16 * (i & 1));
        }
        h->start_max16[k] = smax;
        if (k < 2) {
            float rmax = 0.f;
            for (int c = 0; c < sigma; ++c) rmax = std::max(rmax, rs[k][c]);
            h->chain_resc[k] = rmax <= 16.f ? 4 : 1;
            if (k == 0) h->tc_resc = h->chain_resc[0];
        }
    }
    {   // int8 Boolean tables: the same A rows as above with 0/1 bytes, four K values a word
        tp[3].assign((size_t)h->npairs * 128 * 16, 0u);
        for (int c = 0; c < sigma; ++c) {
            const int p = c >> 1, half_ = c & 1;
            for (int rr = 0; rr < 64; ++rr) {
                const int d = (rr & ~15) | ((rr & 7) << 1) | ((rr >> 3) & 1);
                for (int q = 0; q < 64; ++q)
                    if (Tb[((size_t)c * 64 + d) * 64 + q] != 0.f)
                        tp[3][((size_t)p * 128 + half_ * 64 + rr) * 16 + (q >> 2)] |= 1u << (8 * (q & 3));
            }
        }
        rs[3] = rs[2];
        simg[3].assign(8, make_uint4(0, 0, 0, 0));   // a B row: 16 states a 16-byte column
        uint8_t *b = reinterpret_cast<uint8_t *>(simg[3].data());
        for (int i = 0; i < 64; ++i) b[(i >> 4) * 16 + (i & 15)] = sb[i] != 0.f ? 1 : 0;
        h->start_max16[3] = 1.f;
    }
    cudaError_t e = cudaSuccess;
    auto up = [&](void **dst, const void *src, size_t bytes) {
        if (e != cudaSuccess) return;
        if ((e = cudaMalloc(dst, std::max<size_t>(bytes, 16))) != cudaSuccess) return;
        if (bytes) e = cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice);
    };
    up((void **)&h->d_T32, T32.data(), T32.size() * 4);
    for (int k = 0; k < 2; ++k) {
        std::vector<uint16_t> t16(T32.size());
        for (size_t i = 0; i < T32.size(); ++i) t16[i] = pn_host16(T32[i], k == 1);
        up((void **)&h->d_T16[k], t16.data(), t16.size() * 2);
    }
    up((void **)&h->d_start32, s32.data(), 256);
    up((void **)&h->d_acc, a32.data(), 256);
    up((void **)&h->d_acc_bool, ab.data(), 256);
    for (int k = 0; k < 4; ++k) {
        up((void **)&h->d_tpack[k], tp[k].data(), tp[k].size() * 4);
        up((void **)&h->d_rsym[k], rs[k].data(), rs[k].size() * 4);
        up((void **)&h->d_simg[k], simg[k].data(), 8 * sizeof(uint4));
    }
    if (e == cudaSuccess) e = cudaMalloc(&h->d_misc, 16);
    if (e == cudaSuccess) e = cudaMemset(h->d_misc, 0, 16);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(pnfa_tc_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kPnSmemCap);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(pnfa_tc_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kPnSmemCap);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(pnfa_chain_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kPnSmemCap);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(pnfa_chain_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kPnSmemCap);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(pnfa_tc_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kPnSmemCap);
    if (e != cudaSuccess) {
        set_last_error("trex_pnfa_create", e);
        pn_free(h);
        delete h;
        return e == cudaErrorMemoryAllocation ? TREX_ERR_OOM : TREX_ERR_CUDA;
    }
    *out = h;
    return TREX_OK;
}

void trex_pnfa_destroy(trex_pnfa *h) {
    if (!h) return;
    trex::pn_free(h);
    delete h;
}

int trex_pnfa_run(trex_pnfa *h, int mode, const uint8_t *data, const int64_t *offsets,
                  int64_t n_strings, int64_t total_bytes, double *loglik, uint8_t *accept,
                  int32_t *accept_i32, void *stream) {
    using namespace trex;
    if (!h) return TREX_ERR_NOT_INIT;
    if (n_strings < 0 || total_bytes < 0 || n_strings >= (int64_t)1 << 31) return TREX_ERR_ARG;
    if (mode < TREX_PNFA_BF16 || mode > TREX_PNFA_BOOL8) return TREX_ERR_ARG;
    if (n_strings == 0) return TREX_OK;
    if (!offsets || (total_bytes > 0 && !data)) return TREX_ERR_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned long long *queue = reinterpret_cast<unsigned long long *>(h->d_misc);
    uint32_t *err = reinterpret_cast<uint32_t *>(h->d_misc + 8);
    TREX_CUDA(cudaMemsetAsync(h->d_misc, 0, 16, st));
    if (mode == TREX_PNFA_FP32 || mode == TREX_PNFA_BF16_CC || mode == TREX_PNFA_FP16_CC) {
        PnPlainParams Q;
        Q.data = data;
        Q.total_bytes = total_bytes;
        Q.offsets = offsets;
        Q.n = n_strings;
        Q.T = h->d_T32;
        Q.start = h->d_start32;
        Q.acc = h->d_acc;
        Q.sigma = h->sigma;
        Q.ll_empty = h->ll_empty;
        Q.loglik = loglik;
        Q.accept = accept;
        Q.accept_i32 = accept_i32;
        Q.queue = queue;
        Q.err = err;
        if (mode != TREX_PNFA_FP32) {
            const size_t smem = (size_t)h->sigma * 64 * 64 * 2 + kChainSharedBytes;
            if (smem > kPnSmemCap) {
                set_last_error_msg("trex_pnfa_run: the shared-memory CUDA-core form takes at most 28 symbols");
                return TREX_ERR_SHAPE;
            }
            // one CTA an SM (the tables fill its shared memory), four strings at a time each
            const int grid = (int)std::max<int64_t>(
                1, std::min<int64_t>((n_strings + kChainGroups - 1) / kChainGroups, pn_sms(h)));
            const bool fp16 = mode == TREX_PNFA_FP16_CC;
            profile_kernel_begin(st);
            if (fp16)
                pnfa_chain_kernel<true><<<grid, kChainThreads * kChainGroups, smem, st>>>(Q, h->d_T16[1],
                                                                                          h->chain_resc[1]);
            else
                pnfa_chain_kernel<false><<<grid, kChainThreads * kChainGroups, smem, st>>>(Q, h->d_T16[0],
                                                                                           h->chain_resc[0]);
            profile_kernel_end(st);
            TREX_CHECK_LAUNCH();
            return TREX_OK;
        }
        const int64_t warps = std::min<int64_t>(n_strings, pn_sms(h) * 64);
        const int grid = (int)std::max<int64_t>(1, (warps + kPnPlainWarps - 1) / kPnPlainWarps);
        profile_kernel_begin(st);
        pnfa_plain_kernel<<<grid, kPnPlainWarps * 32, 0, st>>>(Q);
        profile_kernel_end(st);
        TREX_CHECK_LAUNCH();
        return TREX_OK;
    }
    if (h->sigma <= kLnMaxSigma) {   // strings on TMEM lanes, no sorting by symbol (sigma <= 4)
        const int k = mode == TREX_PNFA_FP16 ? 1 : mode == TREX_PNFA_BOOL8 ? 2 : mode == TREX_PNFA_BOOL ? 3 : 0;
        LnParams Q;
        Q.data = data;
        Q.total_bytes = total_bytes;
        Q.offsets = offsets;
        Q.n = n_strings;
        Q.T16 = h->d_T16[k == 1 ? 1 : 0];
        Q.T32 = h->d_T32;
        Q.start = h->d_start32;
        Q.acc = k >= 2 ? h->d_acc_bool : h->d_acc;
        Q.sigma = h->sigma;
        Q.a_cols = (uint32_t)(k == 2 ? 16 : 32) * (uint32_t)h->sigma;
        Q.tile_cols = (Q.a_cols + 64u + 31u) & ~31u;
        Q.tiles = (int)std::min<uint32_t>((uint32_t)kLnTiles, 512u / Q.tile_cols);
        Q.resc = k == 0 ? h->tc_resc : 1;
        Q.wait_cycles = mbar_wait_cycles();
        Q.ll_empty = k >= 2 ? h->ll_empty_bool : h->ll_empty;
        Q.loglik = loglik;
        Q.accept = accept;
        Q.accept_i32 = accept_i32;
        Q.queue = queue;
        Q.err = err;
        // one CTA an SM (it owns the 512 TMEM columns), 128 strings in flight a tile
        const int64_t per_cta = (int64_t)Q.tiles * 128;
        const int grid = (int)std::max<int64_t>(
            1, std::min<int64_t>((n_strings + per_cta - 1) / per_cta, pn_sms(h)));
        profile_kernel_begin(st);
        if (k == 1) pnfa_lane_kernel<1><<<grid, kLnThreads, 0, st>>>(Q);
        else if (k == 2) pnfa_lane_kernel<2><<<grid, kLnThreads, 0, st>>>(Q);
        else if (k == 3) pnfa_lane_kernel<3><<<grid, kLnThreads, 0, st>>>(Q);
        else pnfa_lane_kernel<0><<<grid, kLnThreads, 0, st>>>(Q);
        profile_kernel_end(st);
        TREX_CHECK_LAUNCH();
        return TREX_OK;
    }
    if (h->sigma > kPnMaxSigmaTc) {
        set_last_error_msg("trex_pnfa_run: the tensor-core form takes at most 28 symbols");
        return TREX_ERR_SHAPE;
    }
    int grid = 0, p_sub = 0;
    int rc = pn_choose(h, n_strings, &grid, &p_sub);
    if (rc) return rc;
    const int k = mode == TREX_PNFA_FP16 ? 1 : mode == TREX_PNFA_BOOL ? 2 : mode == TREX_PNFA_BOOL8 ? 3 : 0;
    PnParams P;
    P.data = data;
    P.total_bytes = total_bytes;
    P.offsets = offsets;
    P.n = n_strings;
    P.tpack = h->d_tpack[k];
    P.rsym = h->d_rsym[k];
    P.start_img = h->d_simg[k];
    P.acc = k >= 2 ? h->d_acc_bool : h->d_acc;
    P.start_max = h->start_max16[k];
    P.ll_empty = k >= 2 ? h->ll_empty_bool : h->ll_empty;
    P.boolean = k >= 2;
    P.kcols = k == 3 ? 4 : 8;
    P.wait_cycles = mbar_wait_cycles();
    P.resc = k == 0 ? h->tc_resc : 1;
    P.sigma = h->sigma;
    P.loglik = loglik;
    P.accept = accept;
    P.accept_i32 = accept_i32;
    P.queue = queue;
    P.err = err;
    P.L = pn_layout(p_sub, h->sigma, k == 3 ? 16 : 32);
    // one CTA per SM: it owns all 512 TMEM columns
    const uint32_t smem = std::max<uint32_t>(P.L.total, 120u * 1024u);
    profile_kernel_begin(st);
    if (k == 1) pnfa_tc_kernel<1><<<grid, kPnThreads, smem, st>>>(P);
    else if (k == 3) pnfa_tc_kernel<2><<<grid, kPnThreads, smem, st>>>(P);
    else pnfa_tc_kernel<0><<<grid, kPnThreads, smem, st>>>(P);
    profile_kernel_end(st);
    TREX_CHECK_LAUNCH();
    return TREX_OK;
}

int trex_pnfa_set_sm_limit(trex_pnfa *pnfa, int max_sms) {
    if (!pnfa || max_sms < 0) return TREX_ERR_ARG;
    pnfa->sm_limit = max_sms;
    return TREX_OK;
}

int trex_pnfa_error(trex_pnfa *h, int32_t *err_out) {
    if (!h || !err_out) return TREX_ERR_ARG;
    uint32_t v = 0;
    TREX_CUDA(cudaMemcpy(&v, h->d_misc + 8, 4, cudaMemcpyDeviceToHost));
    *err_out = (int32_t)v;
    return TREX_OK;
}

}  // extern "C"
