// Family (c): Boolean NFA with up to 64 states, bit-parallel on uint64 masks.
//
// Semantics (reference src/nfa_matrices.py:133-157 simulate_nfa and
// cuda/nfa_tc_evolution.cu:683-745 nfa_bitpar_v4_kernel): the state is the
// set of active NFA states; one symbol c maps it to
//     s' = OR over active sources j of col[c][j]      (= min(T[c] s, 1))
// where col[c][j] is the destination mask of source j (epsilon closure
// folded in). A byte >= sigma is either skipped (the C engine) or rejects
// the string (Python simulate_nfa). Outputs: the final mask and accept flag
// (s & accept_mask != 0; a rejected string has the empty mask).
//
// Design: "four Russians" tables. For every symbol c the 64 source bits are
// cut into groups of B bits and tbl[c][g][v] holds the OR of the columns of
// the set bits of v, so a step is ceil(64/B) table lookups ORed together.
// Symbol index sigma is an extra table: the identity (skip) or all zeros
// (reject), so bytes >= sigma need no branch. B is picked so all tables fit
// in shared memory: the widest of 8, 7, 6, 5, 4 bits that fits (8 lookups a
// byte for sigma <= 12, 10 for sigma <= 21, 11 for sigma <= 39); larger
// alphabets read 8-bit tables (8 lookups) from global memory through L1.
// One persistent CTA per SM, a thread per string; threads take strings from
// an atomic counter and walk them in 16-byte windows.
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "trex_internal.cuh"

namespace trex {

constexpr int kNfaThreads = 1024;
constexpr size_t kNfaSmemBudget = 220 * 1024;

__host__ __device__ constexpr int nfa_groups(int B) { return (64 + B - 1) / B; }
// Entries of symbol c are stored at v ^ swizzle(c): with dense states many
// lanes look up the same v for different symbols, and every table starts on
// the same bank; the XOR sends them to different bank pairs.
__host__ __device__ constexpr uint32_t nfa_swizzle(uint32_t c) { return (c ^ (c >> 4)) & 15u; }
__host__ __device__ constexpr int nfa_table_entries(int B) { return nfa_groups(B) << B; }

struct NfaParams {
    const uint8_t *data;
    int64_t total_bytes;
    const int64_t *offsets;
    int64_t n;
    const uint64_t *tables;   // (sigma + 1) x groups x 2^B
    int sigma;
    uint64_t start_mask, accept_mask;
    uint64_t *final_mask;
    uint8_t *accept;
    int32_t *accept_i32;
    unsigned long long *head;
    uint32_t *err;
};

template <int B>
__device__ __forceinline__ uint64_t nfa_step(const uint64_t *tbl, uint64_t s, uint32_t byte,
                                             int sigma) {
    constexpr int G = nfa_groups(B);
    constexpr uint32_t MASK = (1u << B) - 1u;
    const uint32_t sym = min(byte, (uint32_t)sigma);
    const uint64_t *t = tbl + (size_t)sym * nfa_table_entries(B);
    const uint32_t x = nfa_swizzle(sym) & MASK;
    uint64_t acc = 0;
#pragma unroll
    for (int g = 0; g < G; ++g) {
        const uint32_t v = ((uint32_t)(s >> (B * g)) & MASK) ^ x;
        acc |= t[(g << B) + v];
    }
    return acc;
}

// Threads take strings first .. first + n - 1 from the counter *head and walk them
// in 16-byte windows; results go to index i of the output arrays.
template <int B>
__device__ __forceinline__ void nfa_walk_queue(const uint64_t *tbl, int sigma, uint64_t start_mask,
                                               uint64_t accept_mask, const uint8_t *d, int64_t total_bytes,
                                               const int64_t *offsets, int64_t first, int64_t n,
                                               unsigned long long *head, uint32_t *err, uint64_t *final_mask,
                                               uint8_t *accept, int32_t *accept_i32) {
    while (true) {
        const unsigned long long k = atomicAdd(head, 1ull);
        if (k >= (unsigned long long)n) break;
        const int64_t i = first + (int64_t)k;
        const int64_t a = offsets[i], b = offsets[i + 1];
        if (a < 0 || b < a || b > total_bytes) {
            atomicOr(err, 1u);
            continue;
        }
        uint64_t s = start_mask;
        int64_t p = a;
        while (p < b && (((uintptr_t)(d + p)) & 15u)) s = nfa_step<B>(tbl, s, __ldg(d + p++), sigma);
        if (b - p >= 16) {
            uint4 v = ld_stream16(d + p);
            while (true) {
                const bool more = b - p >= 32;
                uint4 nv = make_uint4(0, 0, 0, 0);
                if (more) nv = ld_stream16(d + p + 16);
                const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int k2 = 0; k2 < 16; ++k2) s = nfa_step<B>(tbl, s, (w[k2 >> 2] >> (8 * (k2 & 3))) & 0xffu, sigma);
                p += 16;
                if (!more) break;
                v = nv;
            }
        }
        while (p < b) s = nfa_step<B>(tbl, s, __ldg(d + p++), sigma);
        const bool ok = (s & accept_mask) != 0;
        if (final_mask) final_mask[i] = s;
        if (accept) accept[i] = ok ? 1 : 0;
        if (accept_i32) accept_i32[i] = ok ? 1 : 0;
    }
}

template <int B, bool SMEM>
__global__ void __launch_bounds__(kNfaThreads, 1) nfa_bitpar_kernel(NfaParams P) {
    extern __shared__ __align__(16) uint64_t s_tbl[];
    const uint64_t *tbl = P.tables;
    if (SMEM) {
        const int words = (P.sigma + 1) * nfa_table_entries(B);
        for (int i = threadIdx.x; i < words; i += blockDim.x) s_tbl[i] = P.tables[i];
        __syncthreads();
        tbl = s_tbl;
    }
    nfa_walk_queue<B>(tbl, P.sigma, P.start_mask, P.accept_mask, P.data, P.total_bytes, P.offsets, 0, P.n,
                      P.head, P.err, P.final_mask, P.accept, P.accept_i32);
}

// Many automata in one launch (a serving batch: strings grouped by automaton). Group g
// owns CTAs cta_first[g] .. cta_first[g+1] - 1 and strings first[g] .. first[g] +
// count[g] - 1; each CTA loads its group's tables and its threads take the group's
// strings, so the groups run side by side instead of one launch after another.
constexpr int kNfaMultiMax = 64;
struct NfaMultiParams {
    const uint8_t *data;
    int64_t total_bytes;
    const int64_t *offsets;
    uint64_t *final_mask;
    uint8_t *accept;
    int32_t *accept_i32;
    unsigned long long *heads;   // one counter a group
    uint32_t *err;
    int n_groups;
    const uint64_t *tables[kNfaMultiMax];
    uint64_t start_mask[kNfaMultiMax], accept_mask[kNfaMultiMax];
    int64_t first[kNfaMultiMax], count[kNfaMultiMax];
    int32_t cta_first[kNfaMultiMax + 1];
    int32_t sigma[kNfaMultiMax];
};

template <int B, bool SMEM>
__global__ void __launch_bounds__(kNfaThreads, 1) nfa_bitpar_multi_kernel(const __grid_constant__ NfaMultiParams P) {
    extern __shared__ __align__(16) uint64_t s_tbl[];
    int g = 0;
    while (g + 1 < P.n_groups && (int)blockIdx.x >= P.cta_first[g + 1]) ++g;
    const int sigma = P.sigma[g];
    const uint64_t *tbl = P.tables[g];
    if (SMEM) {
        const int words = (sigma + 1) * nfa_table_entries(B);
        for (int i = threadIdx.x; i < words; i += blockDim.x) s_tbl[i] = tbl[i];
        __syncthreads();
        tbl = s_tbl;
    }
    nfa_walk_queue<B>(tbl, sigma, P.start_mask[g], P.accept_mask[g], P.data, P.total_bytes, P.offsets,
                      P.first[g], P.count[g], P.heads + g, P.err, P.final_mask, P.accept,
                      P.accept_i32);
}

}  // namespace trex

struct trex_nfa {
    int n_states = 0, sigma = 0, B = 6;
    bool smem = true;
    uint64_t start_mask = 0, accept_mask = 0;
    uint64_t *d_tables = nullptr;
    size_t table_words = 0;
    void *d_misc = nullptr;   // head counter + error word
    int n_sms = 0;
    std::vector<uint64_t> cols;   // host copy: sigma x 64 destination masks
    int unknown_rejects = 0;
};

namespace trex {

static void nfa_choose_layout(int sigma, int *B, bool *smem) {
    // the widest groups (fewest lookups a byte) whose tables fit in shared memory
    for (int b : {8, 7, 6, 5, 4}) {
        if ((size_t)(sigma + 1) * nfa_table_entries(b) * 8 <= kNfaSmemBudget) {
            *B = b;
            *smem = true;
            return;
        }
    }
    *B = 8;
    *smem = false;
}

static std::vector<uint64_t> nfa_build_tables(const std::vector<uint64_t> &cols, int sigma, int B,
                                              int unknown_rejects) {
    const int G = nfa_groups(B), E = nfa_table_entries(B);
    std::vector<uint64_t> t((size_t)(sigma + 1) * E, 0);
    for (int c = 0; c <= sigma; ++c) {
        uint64_t *tc = t.data() + (size_t)c * E;
        for (int g = 0; g < G; ++g) {
            for (int v = 0; v < (1 << B); ++v) {
                uint64_t acc = 0;
                for (int bit = 0; bit < B; ++bit) {
                    const int src = g * B + bit;
                    if (!((v >> bit) & 1) || src >= 64) continue;
                    if (c < sigma) acc |= cols[(size_t)c * 64 + src];
                    else if (!unknown_rejects) acc |= 1ull << src;   // identity: skip the byte
                }
                tc[(g << B) + (v ^ (int)(nfa_swizzle((uint32_t)c) & ((1u << B) - 1u)))] = acc;
            }
        }
    }
    return t;
}

int nfa_run(trex_nfa *nfa, const uint8_t *data, const int64_t *offsets, int64_t n,
            int64_t total_bytes, uint64_t *final_mask, uint8_t *accept, int32_t *accept_i32,
            cudaStream_t stream, uint32_t **err_out) {
    if (!nfa) return TREX_ERR_NOT_INIT;
    if (n < 0 || total_bytes < 0 || (n > 0 && !offsets) || (total_bytes > 0 && !data))
        return TREX_ERR_ARG;
    if (n == 0) return TREX_OK;
    unsigned long long *head = static_cast<unsigned long long *>(nfa->d_misc);
    uint32_t *err = reinterpret_cast<uint32_t *>(head + 1);
    TREX_CUDA(cudaMemsetAsync(nfa->d_misc, 0, 16, stream));
    NfaParams P;
    P.data = data;
    P.total_bytes = total_bytes;
    P.offsets = offsets;
    P.n = n;
    P.tables = nfa->d_tables;
    P.sigma = nfa->sigma;
    P.start_mask = nfa->start_mask;
    P.accept_mask = nfa->accept_mask;
    P.final_mask = final_mask;
    P.accept = accept;
    P.accept_i32 = accept_i32;
    P.head = head;
    P.err = err;
    const size_t smem = nfa->smem ? nfa->table_words * 8 : 0;
    // a thread a string: a few strings need one CTA, so that batches of several
    // automata launched on separate streams run side by side
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(nfa->n_sms, (n + 31) / 32));
    profile_kernel_begin(stream);
    switch (nfa->B) {
        case 8: nfa->smem ? nfa_bitpar_kernel<8, true><<<grid, kNfaThreads, smem, stream>>>(P)
                          : nfa_bitpar_kernel<8, false><<<grid, kNfaThreads, 0, stream>>>(P); break;
        case 7: nfa_bitpar_kernel<7, true><<<grid, kNfaThreads, smem, stream>>>(P); break;
        case 6: nfa_bitpar_kernel<6, true><<<grid, kNfaThreads, smem, stream>>>(P); break;
        case 5: nfa_bitpar_kernel<5, true><<<grid, kNfaThreads, smem, stream>>>(P); break;
        default: nfa_bitpar_kernel<4, true><<<grid, kNfaThreads, smem, stream>>>(P); break;
    }
    TREX_CHECK_LAUNCH();
    profile_kernel_end(stream);
    if (err_out) *err_out = err;
    return TREX_OK;
}

template <int B, bool SMEM>
static cudaError_t nfa_multi_launch(const NfaMultiParams &P, int grid, size_t smem, cudaStream_t st) {
    if (SMEM) {
        const cudaError_t e = cudaFuncSetAttribute(nfa_bitpar_multi_kernel<B, SMEM>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    nfa_bitpar_multi_kernel<B, SMEM><<<grid, kNfaThreads, SMEM ? smem : 0, st>>>(P);
    return cudaGetLastError();
}

int nfa_run_multi(trex_nfa *const *nfas, int n_groups, const int64_t *group_first, const uint8_t *data,
                  const int64_t *offsets, int64_t total_bytes, uint64_t *final_mask, uint8_t *accept,
                  int32_t *accept_i32, void *scratch, cudaStream_t st) {
    if (n_groups < 1 || n_groups > kNfaMultiMax || !nfas || !group_first || !scratch) return TREX_ERR_ARG;
    if (group_first[0] != 0) return TREX_ERR_ARG;
    for (int g = 0; g < n_groups; ++g)
        if (!nfas[g] || group_first[g + 1] < group_first[g]) return TREX_ERR_ARG;
    const int64_t n = group_first[n_groups];
    if (total_bytes < 0 || (n > 0 && !offsets) || (total_bytes > 0 && !data)) return TREX_ERR_ARG;
    TREX_CUDA(cudaMemsetAsync(scratch, 0, 8 * (size_t)(n_groups + 1), st));
    if (n == 0) return TREX_OK;
    unsigned long long *heads = static_cast<unsigned long long *>(scratch);
    uint32_t *err = reinterpret_cast<uint32_t *>(heads + n_groups);
    // one launch per table layout (bits a lookup; tables in shared or global memory)
    bool taken[kNfaMultiMax] = {};
    int used_heads = 0;
    for (int g0 = 0; g0 < n_groups; ++g0) {
        if (taken[g0]) continue;
        const int B = nfas[g0]->B;
        const bool sm = nfas[g0]->smem;
        NfaMultiParams P{};
        P.data = data;
        P.total_bytes = total_bytes;
        P.offsets = offsets;
        P.final_mask = final_mask;
        P.accept = accept;
        P.accept_i32 = accept_i32;
        P.heads = heads + used_heads;
        P.err = err;
        int k = 0, ctas = 0;
        size_t smem = 0;
        for (int g = g0; g < n_groups; ++g) {
            const trex_nfa *h = nfas[g];
            if (taken[g] || h->B != B || h->smem != sm) continue;
            taken[g] = true;
            const int64_t cnt = group_first[g + 1] - group_first[g];
            if (cnt == 0) continue;
            P.tables[k] = h->d_tables;
            P.start_mask[k] = h->start_mask;
            P.accept_mask[k] = h->accept_mask;
            P.sigma[k] = h->sigma;
            P.first[k] = group_first[g];
            P.count[k] = cnt;
            P.cta_first[k] = ctas;
            // a thread a string, as in a single-automaton run
            ctas += (int)std::max<int64_t>(1, std::min<int64_t>(h->n_sms, (cnt + 31) / 32));
            smem = std::max(smem, h->table_words * 8);
            ++k;
        }
        if (k == 0) continue;
        P.n_groups = k;
        P.cta_first[k] = ctas;
        used_heads += k;
        cudaError_t e;
        switch (B) {
            case 8: e = sm ? nfa_multi_launch<8, true>(P, ctas, smem, st) : nfa_multi_launch<8, false>(P, ctas, 0, st); break;
            case 7: e = nfa_multi_launch<7, true>(P, ctas, smem, st); break;
            case 6: e = nfa_multi_launch<6, true>(P, ctas, smem, st); break;
            case 5: e = nfa_multi_launch<5, true>(P, ctas, smem, st); break;
            default: e = nfa_multi_launch<4, true>(P, ctas, smem, st); break;
        }
        if (e != cudaSuccess) {
            set_last_error("trex_nfa_run_multi", e);
            return TREX_ERR_CUDA;
        }
    }
    return TREX_OK;
}

}  // namespace trex

extern "C" {

int trex_nfa_create(int n_states, int sigma, const uint64_t *cols, uint64_t start_mask,
                    uint64_t accept_mask, int unknown_rejects, trex_nfa **out) {
    using namespace trex;
    if (!out) return TREX_ERR_ARG;
    *out = nullptr;
    if (n_states < 1 || n_states > 64 || sigma < 0 || sigma > 255 || (sigma > 0 && !cols))
        return TREX_ERR_ARG;
    trex_nfa *nfa = new (std::nothrow) trex_nfa();
    if (!nfa) return TREX_ERR_OOM;
    nfa->n_states = n_states;
    nfa->sigma = sigma;
    nfa->unknown_rejects = unknown_rejects ? 1 : 0;
    const uint64_t keep = n_states == 64 ? ~0ull : ((1ull << n_states) - 1);
    nfa->start_mask = start_mask & keep;
    nfa->accept_mask = accept_mask & keep;
    nfa->cols.assign((size_t)sigma * 64, 0);
    for (int c = 0; c < sigma; ++c)
        for (int j = 0; j < n_states; ++j) nfa->cols[(size_t)c * 64 + j] = cols[(size_t)c * 64 + j] & keep;
    nfa_choose_layout(sigma, &nfa->B, &nfa->smem);
    std::vector<uint64_t> t = nfa_build_tables(nfa->cols, sigma, nfa->B, nfa->unknown_rejects);
    nfa->table_words = t.size();
    nfa->n_sms = sm_count();
    if (nfa->n_sms <= 0) {
        delete nfa;
        set_last_error_msg("trex_nfa_create: no CUDA device");
        return TREX_ERR_SHAPE;
    }
    cudaError_t e;
    if ((e = cudaMalloc(&nfa->d_tables, t.size() * 8)) != cudaSuccess ||
        (e = cudaMalloc(&nfa->d_misc, 16)) != cudaSuccess ||
        (e = cudaMemcpy(nfa->d_tables, t.data(), t.size() * 8, cudaMemcpyHostToDevice)) != cudaSuccess) {
        set_last_error("trex_nfa_create", e);
        cudaFree(nfa->d_tables);
        cudaFree(nfa->d_misc);
        delete nfa;
        return e == cudaErrorMemoryAllocation ? TREX_ERR_OOM : TREX_ERR_CUDA;
    }
    if (nfa->smem) {
        const int smem = (int)(t.size() * 8);
        switch (nfa->B) {
            case 8: e = cudaFuncSetAttribute(nfa_bitpar_kernel<8, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem); break;
            case 7: e = cudaFuncSetAttribute(nfa_bitpar_kernel<7, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem); break;
            case 6: e = cudaFuncSetAttribute(nfa_bitpar_kernel<6, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem); break;
            case 5: e = cudaFuncSetAttribute(nfa_bitpar_kernel<5, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem); break;
            default: e = cudaFuncSetAttribute(nfa_bitpar_kernel<4, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem); break;
        }
        if (e != cudaSuccess) {
            set_last_error("trex_nfa_create: cudaFuncSetAttribute", e);
            cudaFree(nfa->d_tables);
            cudaFree(nfa->d_misc);
            delete nfa;
            return TREX_ERR_CUDA;
        }
    }
    *out = nfa;
    return TREX_OK;
}

void trex_nfa_destroy(trex_nfa *nfa) {
    if (!nfa) return;
    cudaFree(nfa->d_tables);
    cudaFree(nfa->d_misc);
    delete nfa;
}

int trex_nfa_run(trex_nfa *nfa, const uint8_t *data, const int64_t *offsets, int64_t n_strings,
                 int64_t total_bytes, uint64_t *final_mask, uint8_t *accept, int32_t *accept_i32,
                 void *stream) {
    return trex::nfa_run(nfa, data, offsets, n_strings, total_bytes, final_mask, accept, accept_i32,
                         static_cast<cudaStream_t>(stream), nullptr);
}

int trex_nfa_run_multi(trex_nfa *const *nfas, int n_groups, const int64_t *group_first,
                       const uint8_t *data, const int64_t *offsets, int64_t total_bytes,
                       uint64_t *final_mask, uint8_t *accept, int32_t *accept_i32, void *scratch,
                       void *stream) {
    return trex::nfa_run_multi(nfas, n_groups, group_first, data, offsets, total_bytes, final_mask, accept,
                               accept_i32, scratch, static_cast<cudaStream_t>(stream));
}

int trex_nfa_error(trex_nfa *nfa, int32_t *err_out) {
    if (!nfa || !err_out) return TREX_ERR_ARG;
    uint32_t v = 0;
    TREX_CUDA(cudaMemcpy(&v, static_cast<uint8_t *>(nfa->d_misc) + 8, 4, cudaMemcpyDeviceToHost));
    *err_out = (int32_t)v;
    return TREX_OK;
}

}  // extern "C"

// ---- reference C ABI: nfa_tc_engine_* (cuda/nfa_tc_evolution.cu:936-1015) -----------------
namespace trex {
struct RefNfaEngine {
    trex_nfa *nfa = nullptr;
    uint8_t *d_data = nullptr;
    int64_t *d_off64 = nullptr;
    int32_t *d_off32 = nullptr;
    int32_t *d_res = nullptr;
    int64_t max_chars = 0, max_b = 0;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    bool ready = false;
    void destroy() {
        trex_nfa_destroy(nfa);
        cudaFree(d_data);
        cudaFree(d_off64);
        cudaFree(d_off32);
        cudaFree(d_res);
        for (auto &x : ev)
            if (x) cudaEventDestroy(x);
        *this = RefNfaEngine();
    }
};
static RefNfaEngine g_ref_nfa;
__global__ void nfa_widen_kernel(const int32_t *in, int64_t *out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = in[i];
}
}  // namespace trex

extern "C" {

int nfa_tc_engine_init(const float *T_matrices, const float *accept_mask, const float *start_vec,
                       int n, int sigma, int max_B, int max_L) {
    using namespace trex;
    RefNfaEngine &E = g_ref_nfa;
    E.destroy();
    if (!T_matrices || !accept_mask || !start_vec || max_B < 0 || max_L < 0) return TREX_ERR_ARG;
    if (n < 1 || n > 64 || sigma < 1 || sigma > 255) return TREX_ERR_SHAPE;
    // T[c][dst][src] > 0.5 is an edge (reference float_to_bitpar, nfa_tc_evolution.cu:632-644)
    std::vector<uint64_t> cols((size_t)sigma * 64, 0);
    for (int c = 0; c < sigma; ++c)
        for (int dst = 0; dst < n; ++dst)
            for (int src = 0; src < n; ++src)
                if (T_matrices[((size_t)c * n + dst) * n + src] > 0.5f) cols[(size_t)c * 64 + src] |= 1ull << dst;
    uint64_t sm = 0, am = 0;
    for (int i = 0; i < n; ++i) {
        if (start_vec[i] > 0.5f) sm |= 1ull << i;
        if (accept_mask[i] > 0.5f) am |= 1ull << i;
    }
    int rc = trex_nfa_create(n, sigma, cols.data(), sm, am, 0, &E.nfa);
    if (rc) return rc;
    E.max_b = max_B;
    E.max_chars = (int64_t)max_B * max_L;
    cudaError_t e;
    if ((e = cudaMalloc(&E.d_data, std::max<int64_t>(E.max_chars, 16))) != cudaSuccess ||
        (e = cudaMalloc(&E.d_off64, (max_B + 1) * 8)) != cudaSuccess ||
        (e = cudaMalloc(&E.d_off32, (max_B + 1) * 4)) != cudaSuccess ||
        (e = cudaMalloc(&E.d_res, std::max(max_B, 1) * 4)) != cudaSuccess) {
        set_last_error("nfa_tc_engine_init", e);
        E.destroy();
        return TREX_ERR_OOM;
    }
    for (auto &x : E.ev) TREX_CUDA(cudaEventCreate(&x));
    E.ready = true;
    return TREX_OK;
}

int nfa_tc_engine_dispatch(const uint8_t *raw_concat, const int *offsets, int *results, int B,
                           int total_chars, float *kernel_ms, float *total_ms) {
    using namespace trex;
    RefNfaEngine &E = g_ref_nfa;
    if (!E.ready) return TREX_ERR_NOT_INIT;
    if (B < 0 || total_chars < 0 || (B > 0 && (!offsets || !results))) return TREX_ERR_ARG;
    if (B > E.max_b || total_chars > E.max_chars) return TREX_ERR_CAPACITY;
    if (kernel_ms) *kernel_ms = 0.f;
    if (total_ms) *total_ms = 0.f;
    if (B == 0) return TREX_OK;
    cudaStream_t st = 0;
    TREX_CUDA(cudaEventRecord(E.ev[0], st));
    if (total_chars) TREX_CUDA(cudaMemcpyAsync(E.d_data, raw_concat, total_chars, cudaMemcpyHostToDevice, st));
    TREX_CUDA(cudaMemcpyAsync(E.d_off32, offsets, (size_t)(B + 1) * 4, cudaMemcpyHostToDevice, st));
    nfa_widen_kernel<<<std::min(1024, (B + 256) / 256), 256, 0, st>>>(E.d_off32, E.d_off64, B + 1);
    TREX_CHECK_LAUNCH();
    TREX_CUDA(cudaEventRecord(E.ev[1], st));
    uint32_t *err = nullptr;
    int rc = nfa_run(E.nfa, E.d_data, E.d_off64, B, total_chars, nullptr, nullptr, E.d_res, st, &err);
    if (rc) return rc;
    TREX_CUDA(cudaEventRecord(E.ev[2], st));
    TREX_CUDA(cudaMemcpyAsync(results, E.d_res, (size_t)B * 4, cudaMemcpyDeviceToHost, st));
    uint32_t h_err = 0;
    TREX_CUDA(cudaMemcpyAsync(&h_err, err, 4, cudaMemcpyDeviceToHost, st));
    TREX_CUDA(cudaEventRecord(E.ev[3], st));
    TREX_CUDA(cudaEventSynchronize(E.ev[3]));
    if (kernel_ms) TREX_CUDA(cudaEventElapsedTime(kernel_ms, E.ev[1], E.ev[2]));
    if (total_ms) TREX_CUDA(cudaEventElapsedTime(total_ms, E.ev[0], E.ev[3]));
    return h_err ? TREX_ERR_ARG : TREX_OK;
}

void nfa_tc_engine_destroy(void) { trex::g_ref_nfa.destroy(); }

}  // extern "C"
