// Error strings, device queries and the library version.
#include <atomic>
#include <cstdio>
#include <cstring>
#include <vector>

#include "trex_internal.cuh"

namespace trex {

static thread_local char g_last_error[512] = "";

void set_last_error(const char *where, cudaError_t err) {
    snprintf(g_last_error, sizeof(g_last_error), "%s: %s (%d)", where,
             cudaGetErrorString(err), (int)err);
}

void set_last_error_msg(const char *msg) {
    snprintf(g_last_error, sizeof(g_last_error), "%s", msg);
}

int sm_count() {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    return n;
}

// ---- wait limits -------------------------------------------------------------------
static std::atomic<uint32_t> g_scan_polls{kDefaultScanPolls};
static std::atomic<long long> g_mbar_cycles{kDefaultMbarCycles};
uint32_t scan_poll_limit() { return g_scan_polls.load(std::memory_order_relaxed); }
long long mbar_wait_cycles() { return g_mbar_cycles.load(std::memory_order_relaxed); }

// ---- launch profiler: CUDA events around the main kernel of each run -----------
struct Profiler {
    std::vector<cudaEvent_t> start, stop;
    int used = 0;
    bool on = false;
};
static Profiler g_prof;

void profile_kernel_begin(cudaStream_t s) {
    if (!g_prof.on || g_prof.used >= (int)g_prof.start.size()) return;
    cudaEventRecord(g_prof.start[g_prof.used], s);
}

void profile_kernel_end(cudaStream_t s) {
    if (!g_prof.on || g_prof.used >= (int)g_prof.start.size()) return;
    cudaEventRecord(g_prof.stop[g_prof.used], s);
    ++g_prof.used;
}

}  // namespace trex

extern "C" int trex_profile_begin(int max_launches) {
    using trex::g_prof;
    if (max_launches < 1) return TREX_ERR_ARG;
    for (auto e : g_prof.start) cudaEventDestroy(e);
    for (auto e : g_prof.stop) cudaEventDestroy(e);
    g_prof.start.assign(max_launches, nullptr);
    g_prof.stop.assign(max_launches, nullptr);
    for (int i = 0; i < max_launches; ++i) {
        TREX_CUDA(cudaEventCreate(&g_prof.start[i]));
        TREX_CUDA(cudaEventCreate(&g_prof.stop[i]));
    }
    g_prof.used = 0;
    g_prof.on = true;
    return TREX_OK;
}

extern "C" int trex_profile_end(float *ms_out, int capacity, int *count) {
    using trex::g_prof;
    g_prof.on = false;
    int n = g_prof.used;
    if (count) *count = n;
    for (int i = 0; i < n && i < capacity && ms_out; ++i) {
        TREX_CUDA(cudaEventSynchronize(g_prof.stop[i]));
        TREX_CUDA(cudaEventElapsedTime(&ms_out[i], g_prof.start[i], g_prof.stop[i]));
    }
    g_prof.used = 0;
    return TREX_OK;
}

extern "C" int trex_set_wait_limits(int64_t scan_polls, int64_t mbar_cycles) {
    if (scan_polls < 0 || mbar_cycles < 0 || scan_polls > 0xffffffffll) return TREX_ERR_ARG;
    trex::g_scan_polls.store(scan_polls ? (uint32_t)scan_polls : trex::kDefaultScanPolls);
    trex::g_mbar_cycles.store(mbar_cycles ? (long long)mbar_cycles : trex::kDefaultMbarCycles);
    return TREX_OK;
}

extern "C" const char *trex_last_error(void) { return trex::g_last_error; }

extern "C" const char *trex_version(void) { return "trex_b200 0.1 (sm_100a)"; }
