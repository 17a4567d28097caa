// Reference-compatible singleton engines (host buffers in, host results out)
// for the DFA families: prefix_engine_*, monoid_batch_engine_*,
// monoid_engine_*, plus the 64-bit host-buffer batch entry point.
//
// Contract kept from the reference (cuda/monoid_batch.cu:378-673,
// cuda/prefix_compose.cu:263-472, cuda/monoid_scan.cu:227-515): init copies
// the tables to the device and allocates input/output buffers sized by
// max_total_chars / max_batch; dispatch copies the CSR batch in, runs, copies
// int results[B] out and reports kernel_ms (kernel events) and total_ms
// (copy + kernel + copy). Differences: capacity is checked (the reference
// overruns), CUDA failures return TREX_ERR_CUDA instead of exiting.
#include <algorithm>
#include <cstring>
#include <vector>

#include "trex_internal.cuh"

namespace trex {

int dfa_set_run(trex_dfa_set *set, const uint8_t *data, const int64_t *offsets,
                const int32_t *dfa_id, int64_t n, int64_t total_bytes, uint8_t *final_state,
                uint8_t *accept, int32_t *accept_i32, void *scratch, int64_t scratch_bytes,
                int32_t seg_len, cudaStream_t stream, uint32_t **err_word_out);

__global__ void widen_offsets_kernel(const int32_t *in, int64_t *out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = in[i];
}

int device_check() {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return -1;
    }
    int dev = 0, major = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    return major < 7 ? -2 : 0;
}

// One resident DFA plus device buffers for host-buffer dispatches.
struct HostDfaEngine {
    trex_dfa_set *set = nullptr;
    uint8_t *d_data = nullptr;
    int32_t *d_off32 = nullptr;
    int64_t *d_off64 = nullptr;
    int32_t *d_results = nullptr;
    void *d_scratch = nullptr;
    int64_t scratch_bytes = 0;
    int64_t max_chars = 0, max_batch = 0;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    bool ready = false;

    void destroy() {
        if (set) trex_dfa_set_destroy(set);
        cudaFree(d_data);
        cudaFree(d_off32);
        cudaFree(d_off64);
        cudaFree(d_results);
        cudaFree(d_scratch);
        for (auto &e : ev)
            if (e) cudaEventDestroy(e);
        *this = HostDfaEngine();
    }

    int init(int N, int start, const uint8_t *tmap, const uint8_t *accept, int64_t max_c,
             int64_t max_b) {
        destroy();
        if (max_c < 0 || max_b < 0) return TREX_ERR_ARG;
        int32_t n32 = N, s32 = start;
        int rc = trex_dfa_set_create(1, &n32, &s32, tmap, accept, &set);
        if (rc) return rc;
        max_chars = max_c;
        max_batch = max_b;
        scratch_bytes = trex_dfa_batch_scratch_bytes(max_b, max_c, 0);
        auto alloc = [&](void **p, size_t bytes) {
            return cudaMalloc(p, std::max<size_t>(bytes, 16));
        };
        cudaError_t e;
        if ((e = alloc((void **)&d_data, max_c)) != cudaSuccess ||
            (e = alloc((void **)&d_off32, (max_b + 1) * 4)) != cudaSuccess ||
            (e = alloc((void **)&d_off64, (max_b + 1) * 8)) != cudaSuccess ||
            (e = alloc((void **)&d_results, max_b * 4)) != cudaSuccess ||
            (e = alloc(&d_scratch, scratch_bytes)) != cudaSuccess) {
            set_last_error("engine init allocation", e);
            destroy();
            return TREX_ERR_OOM;
        }
        for (auto &x : ev) TREX_CUDA(cudaEventCreate(&x));
        ready = true;
        return TREX_OK;
    }

    int dispatch(const uint8_t *h_data, const int *h_off, int *h_results, int B, int total,
                 float *kernel_ms, float *total_ms) {
        if (!ready) return TREX_ERR_NOT_INIT;
        if (B < 0 || total < 0 || (B > 0 && (!h_off || !h_results))) return TREX_ERR_ARG;
        if (B > max_batch || total > max_chars) return TREX_ERR_CAPACITY;
        if (B == 0) {
            if (kernel_ms) *kernel_ms = 0.f;
            if (total_ms) *total_ms = 0.f;
            return TREX_OK;
        }
        if (h_off[0] < 0 || h_off[B] > total) return TREX_ERR_ARG;
        cudaStream_t st = 0;
        TREX_CUDA(cudaEventRecord(ev[0], st));
        if (total > 0) TREX_CUDA(cudaMemcpyAsync(d_data, h_data, total, cudaMemcpyHostToDevice, st));
        TREX_CUDA(cudaMemcpyAsync(d_off32, h_off, (size_t)(B + 1) * 4, cudaMemcpyHostToDevice, st));
        widen_offsets_kernel<<<std::min(1024, (B + 256) / 256), 256, 0, st>>>(d_off32, d_off64,
                                                                              B + 1);
        TREX_CHECK_LAUNCH();
        TREX_CUDA(cudaEventRecord(ev[1], st));
        uint32_t *err = nullptr;
        int rc = dfa_set_run(set, d_data, d_off64, nullptr, B, total, nullptr, nullptr, d_results,
                             d_scratch, scratch_bytes, 0, st, &err);
        if (rc) return rc;
        TREX_CUDA(cudaEventRecord(ev[2], st));
        TREX_CUDA(cudaMemcpyAsync(h_results, d_results, (size_t)B * 4, cudaMemcpyDeviceToHost, st));
        uint32_t h_err = 0;
        TREX_CUDA(cudaMemcpyAsync(&h_err, err, 4, cudaMemcpyDeviceToHost, st));
        TREX_CUDA(cudaEventRecord(ev[3], st));
        TREX_CUDA(cudaEventSynchronize(ev[3]));
        if (kernel_ms) TREX_CUDA(cudaEventElapsedTime(kernel_ms, ev[1], ev[2]));
        if (total_ms) TREX_CUDA(cudaEventElapsedTime(total_ms, ev[0], ev[3]));
        if (h_err) {
            set_last_error_msg("dispatch: malformed offsets");
            return TREX_ERR_ARG;
        }
        return TREX_OK;
    }
};

static HostDfaEngine g_prefix, g_monoid_batch;
static int g_monoid_batch_M = 0, g_monoid_batch_sigma_ext = 0;
static std::vector<uint8_t> g_monoid_batch_char_compose, g_monoid_batch_charmap;

// ---- monoid scan engine: uint16 element stream, M x M compose table --------------------
__global__ void monoid_walk_kernel(const uint16_t *__restrict__ compose, int M, int identity,
                                   const uint8_t *__restrict__ accept,
                                   const uint16_t *__restrict__ chars,
                                   const int64_t *__restrict__ off, int64_t B,
                                   int32_t *__restrict__ results, int use_smem) {
    extern __shared__ uint16_t sh_compose[];
    const uint16_t *tbl = compose;
    if (use_smem) {
        for (int i = threadIdx.x; i < M * M; i += blockDim.x) sh_compose[i] = compose[i];
        __syncthreads();
        tbl = sh_compose;
    }
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < B;
         i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t acc = (uint32_t)identity;
        for (int64_t k = off[i]; k < off[i + 1]; ++k)
            acc = tbl[(uint32_t)__ldg(chars + k) * (uint32_t)M + acc];
        results[i] = accept[acc] ? 1 : 0;
    }
}

__global__ void monoid_validate_kernel(const uint16_t *chars, int64_t n, int M, uint32_t *err) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        if (chars[i] >= M) atomicOr(err, 1u);
}

struct MonoidScanEngine {
    int M = 0, identity = 0;
    uint16_t *d_compose = nullptr;
    uint8_t *d_accept = nullptr;
    uint16_t *d_chars = nullptr;
    int32_t *d_off32 = nullptr;
    int64_t *d_off64 = nullptr;
    int32_t *d_results = nullptr;
    uint32_t *d_err = nullptr;
    int64_t max_chars = 0, max_batch = 0;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    bool ready = false;

    void destroy() {
        cudaFree(d_compose);
        cudaFree(d_accept);
        cudaFree(d_chars);
        cudaFree(d_off32);
        cudaFree(d_off64);
        cudaFree(d_results);
        cudaFree(d_err);
        for (auto &e : ev)
            if (e) cudaEventDestroy(e);
        *this = MonoidScanEngine();
    }
};
static MonoidScanEngine g_monoid_scan;

}  // namespace trex

using namespace trex;

extern "C" {

// ---- prefix compose ------------------------------------------------------------------------
int prefix_engine_device_check(void) { return device_check(); }

int prefix_engine_init(const uint8_t *tmap, const uint8_t *accept, int start_state, int N, int K,
                       int max_total_chars, int max_batch) {
    (void)K;
    if (!tmap || !accept) return TREX_ERR_ARG;
    return g_prefix.init(N, start_state, tmap, accept, max_total_chars, max_batch);
}

int prefix_engine_dispatch(const uint8_t *raw_concat, const int *offsets, int *results, int B,
                           int total_chars, float *kernel_ms, float *total_ms) {
    return g_prefix.dispatch(raw_concat, offsets, results, B, total_chars, kernel_ms, total_ms);
}

void prefix_engine_destroy(void) { g_prefix.destroy(); }

// ---- monoid batch ----------------------------------------------------------------------------
int monoid_batch_engine_device_check(void) { return device_check(); }

int monoid_batch_engine_init(int M, int sigma_ext, int identity, const uint8_t *char_compose,
                             const uint8_t *raw_char_map, const uint8_t *accept,
                             const uint8_t *monoid_compose, int max_total_chars, int max_batch) {
    (void)monoid_compose;
    g_monoid_batch.destroy();
    if (M < 1 || M > 255 || sigma_ext < 1 || identity < 0 || identity >= M || !char_compose ||
        !raw_char_map || !accept)
        return TREX_ERR_ARG;
    // The monoid is an automaton over its M elements: element m on byte b
    // goes to char_compose[m * sigma_ext + raw_char_map[b]].
    std::vector<uint8_t> tmap(256 * (size_t)M);
    for (int b = 0; b < 256; ++b) {
        int ci = raw_char_map[b];
        if (ci >= sigma_ext) return TREX_ERR_ARG;
        for (int m = 0; m < M; ++m) {
            uint8_t nxt = char_compose[(size_t)m * sigma_ext + ci];
            if (nxt >= M) return TREX_ERR_ARG;
            tmap[(size_t)b * M + m] = nxt;
        }
    }
    g_monoid_batch_M = M;
    g_monoid_batch_sigma_ext = sigma_ext;
    g_monoid_batch_char_compose.assign(char_compose, char_compose + (size_t)M * sigma_ext);
    g_monoid_batch_charmap.assign(raw_char_map, raw_char_map + 256);
    return g_monoid_batch.init(M, identity, tmap.data(), accept, max_total_chars, max_batch);
}

int monoid_batch_engine_set_kgram(const uint8_t *fused_compose, const uint8_t *kgram_compose,
                                  int kgram_k, int sigma_k, int sigma) {
    (void)kgram_compose;
    (void)kgram_k;
    (void)sigma_k;
    (void)sigma;
    if (!g_monoid_batch.ready) return TREX_ERR_NOT_INIT;
    if (fused_compose) {
        // The fused table must agree with char_compose o raw_char_map, which
        // is what the engine already walks.
        const int M = g_monoid_batch_M, se = g_monoid_batch_sigma_ext;
        for (int m = 0; m < M; ++m)
            for (int b = 0; b < 256; ++b)
                if (fused_compose[(size_t)m * 256 + b] !=
                    g_monoid_batch_char_compose[(size_t)m * se + g_monoid_batch_charmap[b]])
                    return TREX_ERR_ARG;
    }
    return TREX_OK;
}

void monoid_batch_engine_destroy(void) { g_monoid_batch.destroy(); }

int monoid_batch_engine_dispatch(const uint8_t *raw_concat, const int *offsets, int *results,
                                 int B, int total_chars, float *kernel_ms, float *total_ms) {
    return g_monoid_batch.dispatch(raw_concat, offsets, results, B, total_chars, kernel_ms,
                                   total_ms);
}

int monoid_batch_engine_dispatch_prefix(const uint8_t *raw_concat, const int *offsets,
                                        int *results, int B, int total_chars, float *kernel_ms,
                                        float *total_ms) {
    return g_monoid_batch.dispatch(raw_concat, offsets, results, B, total_chars, kernel_ms,
                                   total_ms);
}

// ---- monoid scan -------------------------------------------------------------------------------
int monoid_engine_device_check(void) { return device_check(); }

int monoid_engine_init(int monoid_size, int identity_idx, const uint16_t *compose_table,
                       const uint8_t *accept_table, int max_total_chars, int max_batch) {
    MonoidScanEngine &E = g_monoid_scan;
    E.destroy();
    if (monoid_size < 1 || monoid_size > 65536 || identity_idx < 0 || identity_idx >= monoid_size ||
        !compose_table || !accept_table || max_total_chars < 0 || max_batch < 0)
        return TREX_ERR_ARG;
    const size_t MM = (size_t)monoid_size * monoid_size;
    for (size_t i = 0; i < MM; ++i)
        if (compose_table[i] >= monoid_size) return TREX_ERR_ARG;
    E.M = monoid_size;
    E.identity = identity_idx;
    E.max_chars = max_total_chars;
    E.max_batch = max_batch;
    cudaError_t e;
    if ((e = cudaMalloc(&E.d_compose, MM * 2)) != cudaSuccess ||
        (e = cudaMalloc(&E.d_accept, monoid_size)) != cudaSuccess ||
        (e = cudaMalloc(&E.d_chars, std::max<size_t>((size_t)max_total_chars * 2, 16))) != cudaSuccess ||
        (e = cudaMalloc(&E.d_off32, ((size_t)max_batch + 1) * 4)) != cudaSuccess ||
        (e = cudaMalloc(&E.d_off64, ((size_t)max_batch + 1) * 8)) != cudaSuccess ||
        (e = cudaMalloc(&E.d_results, std::max<size_t>((size_t)max_batch * 4, 16))) != cudaSuccess ||
        (e = cudaMalloc(&E.d_err, 4)) != cudaSuccess) {
        set_last_error("monoid_engine_init allocation", e);
        E.destroy();
        return TREX_ERR_OOM;
    }
    TREX_CUDA(cudaMemcpy(E.d_compose, compose_table, MM * 2, cudaMemcpyHostToDevice));
    TREX_CUDA(cudaMemcpy(E.d_accept, accept_table, monoid_size, cudaMemcpyHostToDevice));
    for (auto &x : E.ev) TREX_CUDA(cudaEventCreate(&x));
    if (MM * 2 <= 200 * 1024)
        TREX_CUDA(cudaFuncSetAttribute(monoid_walk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(MM * 2)));
    E.ready = true;
    return TREX_OK;
}

void monoid_engine_destroy(void) { g_monoid_scan.destroy(); }

int monoid_engine_dispatch_batch(const uint16_t *chars, const int *offsets, int *results, int B,
                                 int total_chars, float *kernel_ms, float *total_ms) {
    MonoidScanEngine &E = g_monoid_scan;
    if (!E.ready) return TREX_ERR_NOT_INIT;
    if (B < 0 || total_chars < 0 || (B > 0 && (!offsets || !results))) return TREX_ERR_ARG;
    if (B > E.max_batch || total_chars > E.max_chars) return TREX_ERR_CAPACITY;
    if (B == 0) {
        if (kernel_ms) *kernel_ms = 0.f;
        if (total_ms) *total_ms = 0.f;
        return TREX_OK;
    }
    for (int i = 0; i < B; ++i)
        if (offsets[i] < 0 || offsets[i + 1] < offsets[i] || offsets[i + 1] > total_chars)
            return TREX_ERR_ARG;
    cudaStream_t st = 0;
    TREX_CUDA(cudaEventRecord(E.ev[0], st));
    if (total_chars)
        TREX_CUDA(cudaMemcpyAsync(E.d_chars, chars, (size_t)total_chars * 2, cudaMemcpyHostToDevice, st));
    TREX_CUDA(cudaMemcpyAsync(E.d_off32, offsets, (size_t)(B + 1) * 4, cudaMemcpyHostToDevice, st));
    TREX_CUDA(cudaMemsetAsync(E.d_err, 0, 4, st));
    widen_offsets_kernel<<<std::min(1024, (B + 256) / 256), 256, 0, st>>>(E.d_off32, E.d_off64, B + 1);
    TREX_CHECK_LAUNCH();
    if (total_chars) {
        monoid_validate_kernel<<<std::min<int64_t>(1024, (total_chars + 255) / 256), 256, 0, st>>>(
            E.d_chars, total_chars, E.M, E.d_err);
        TREX_CHECK_LAUNCH();
    }
    uint32_t h_err = 0;
    TREX_CUDA(cudaMemcpyAsync(&h_err, E.d_err, 4, cudaMemcpyDeviceToHost, st));
    TREX_CUDA(cudaStreamSynchronize(st));
    if (h_err) return TREX_ERR_ARG;   // element index >= M: refuse before walking
    TREX_CUDA(cudaEventRecord(E.ev[1], st));
    const size_t MM = (size_t)E.M * E.M;
    int use_smem = MM * 2 <= 200 * 1024;
    int grid = std::max(1, std::min((B + 127) / 128, sm_count() * 4));
    monoid_walk_kernel<<<grid, 128, use_smem ? MM * 2 : 0, st>>>(
        E.d_compose, E.M, E.identity, E.d_accept, E.d_chars, E.d_off64, B, E.d_results, use_smem);
    TREX_CHECK_LAUNCH();
    TREX_CUDA(cudaEventRecord(E.ev[2], st));
    TREX_CUDA(cudaMemcpyAsync(results, E.d_results, (size_t)B * 4, cudaMemcpyDeviceToHost, st));
    TREX_CUDA(cudaEventRecord(E.ev[3], st));
    TREX_CUDA(cudaEventSynchronize(E.ev[3]));
    if (kernel_ms) TREX_CUDA(cudaEventElapsedTime(kernel_ms, E.ev[1], E.ev[2]));
    if (total_ms) TREX_CUDA(cudaEventElapsedTime(total_ms, E.ev[0], E.ev[3]));
    return TREX_OK;
}

}  // extern "C"
