// Serving: moves strings from a staging buffer to their places in a batch.
//
// A serving batch lays its strings out by automaton (the Boolean and probabilistic NFA
// launches take one contiguous run of strings each), while a client's bulk submission
// arrives in its own order. The server stages such a submission as it came (one host-to-
// device copy) and this kernel scatters its strings to their batch positions.
#include "trex_internal.cuh"

namespace trex {

int sm_count();

namespace {

constexpr int kScatterThreads = 256;
constexpr int kScatterLaneBytes = 32;                 // bytes a lane moves per tile
constexpr int kScatterTile = 32 * kScatterLaneBytes;  // source bytes a warp moves per tile

// A warp moves a contiguous run of 1 KiB source tiles. Byte p of a tile belongs to lane
// p mod 32, so every load and store instruction of the warp covers 32 consecutive bytes.
// A lane follows the string holding its current byte with a cursor that only moves
// forward (its bytes increase). Every byte is checked against its string's source range
// and the destination size; a byte that fails is not written and sets bit 0 of *err.
__global__ void __launch_bounds__(kScatterThreads)
scatter_strings_kernel(const uint8_t *__restrict__ src, int64_t src_bytes,
                       const int64_t *__restrict__ src_off, int64_t n,
                       uint8_t *__restrict__ dst, int64_t dst_bytes,
                       const int64_t *__restrict__ dst_begin, int64_t tiles_per_warp,
                       int32_t *__restrict__ err)
{
    const int lane = threadIdx.x & 31;
    const int64_t warp = (int64_t(blockIdx.x) * kScatterThreads + threadIdx.x) >> 5;
    int64_t total = src_off[n];
    if (total > src_bytes || total < 0) {
        if (warp == 0 && lane == 0) atomicOr(err, 1);
        total = total < 0 ? 0 : src_bytes;
    }
    const int64_t lo_byte = warp * tiles_per_warp * kScatterTile;
    if (lo_byte >= total) return;
    const int64_t hi_byte = min(total, lo_byte + tiles_per_warp * kScatterTile);
    // the string holding byte lo_byte: the last i < n with src_off[i] <= lo_byte
    int64_t a = 0, b = n;
    while (b - a > 1) {
        const int64_t m = (a + b) >> 1;
        if (src_off[m] <= lo_byte) a = m; else b = m;
    }
    int64_t cur = a;
    int64_t beg = src_off[cur], end = src_off[cur + 1], db = dst_begin[cur];
    bool bad = false;
    for (int64_t t = lo_byte; t < hi_byte; t += kScatterTile) {
        uint8_t v[kScatterLaneBytes];
#pragma unroll
        for (int k = 0; k < kScatterLaneBytes; ++k) {
            const int64_t p = t + k * 32 + lane;
            v[k] = p < hi_byte ? src[p] : 0;
        }
#pragma unroll
        for (int k = 0; k < kScatterLaneBytes; ++k) {
            const int64_t p = t + k * 32 + lane;
            if (p >= hi_byte) continue;
            while (end <= p && cur + 1 < n) {
                ++cur;
                beg = src_off[cur];
                end = src_off[cur + 1];
                db = dst_begin[cur];
            }
            const int64_t d = db + (p - beg);
            if (p >= beg && p < end && d >= 0 && d < dst_bytes) dst[d] = v[k];
            else bad = true;
        }
    }
    if (bad) atomicOr(err, 1);
}

}  // namespace
}  // namespace trex

extern "C" int trex_scatter_strings(const uint8_t *src, int64_t src_bytes, const int64_t *src_offsets,
                                    int64_t n_strings, uint8_t *dst, int64_t dst_bytes,
                                    const int64_t *dst_begin, int32_t *err, void *stream)
{
    using namespace trex;
    if (n_strings < 0 || src_bytes < 0 || dst_bytes < 0) return TREX_ERR_ARG;
    if (n_strings == 0 || src_bytes == 0) return TREX_OK;
    if (!src || !src_offsets || !dst || !dst_begin || !err) return TREX_ERR_ARG;
    const int n_sms = sm_count();
    if (n_sms <= 0) return TREX_ERR_SHAPE;
    const int64_t tiles = (src_bytes + kScatterTile - 1) / kScatterTile;
    const int64_t warps = std::min<int64_t>(tiles, int64_t(n_sms) * 32);   // 64 registers: 32 warps an SM
    const int64_t tiles_per_warp = (tiles + warps - 1) / warps;
    const int64_t warps_per_block = kScatterThreads / 32;
    const unsigned blocks = unsigned((warps + warps_per_block - 1) / warps_per_block);
    scatter_strings_kernel<<<blocks, kScatterThreads, 0, (cudaStream_t)stream>>>(
        src, src_bytes, src_offsets, n_strings, dst, dst_bytes, dst_begin, tiles_per_warp, err);
    TREX_CHECK_LAUNCH();
    return TREX_OK;
}
