// Block-wide int64 prefix scans shared by the intersection count and the
// packed projection (256-thread CTAs; one value per thread).
#pragma once
#include "tg_common.cuh"

namespace tg {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanChunk = kScanThreads * kScanItems;

__device__ __forceinline__ int64_t warp_incl_scan(int64_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
    }
    return v;
}

// Block-wide exclusive scan of one int64 per thread (blockDim = kScanThreads).
__device__ __forceinline__ int64_t block_excl_scan(int64_t v, int64_t* s_warp, int64_t& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t inc = warp_incl_scan(v);
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        int64_t w = lane < kScanThreads / 32 ? s_warp[lane] : 0;
        w = warp_incl_scan(w);
        if (lane < kScanThreads / 32) s_warp[lane] = w;
    }
    __syncthreads();
    const int64_t warp_prefix = warp == 0 ? 0 : s_warp[warp - 1];
    total = s_warp[kScanThreads / 32 - 1];
    __syncthreads();
    return warp_prefix + inc - v;
}

// Phase 2 of a chunked scan: exclusive scan of the chunk sums in place, in
// one CTA; writes the grand total to *n_total (device).  One launch.
cudaError_t launch_scan_chunk_sums(int64_t* chunk_sums, int64_t n_chunks, int64_t* n_total, cudaStream_t s);

}  // namespace tg
