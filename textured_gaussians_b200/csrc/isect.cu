// Tile intersection, prefix sum, onesweep radix sort and tile offsets for sm_100a.
//
// Semantics follow textured_gaussians/cuda/csrc/isect_tiles.cu of the
// reference:  per projected Gaussian the tile AABB [floor((x-r)/ts),
// ceil((x+r)/ts)) clamped to the grid (:60-70), keys
// cam << (32+tile_bits) | tile << 32 | sign-extended float bits of depth
// (:90-101), a stable sort on key bits [0, 32+tile_bits+cam_bits) (:262-299)
// and per-tile run offsets (:309-355).
//
// The sort is a hand-written LSD onesweep radix sort (8-bit digits): one
// read of the keys builds the digit histograms of every pass, then each pass
// is a single kernel whose CTAs take 4096-key tiles in launch order, rank the
// keys with warp match-any, publish their digit counts and resolve their
// global digit offsets by decoupled look-back over earlier tiles.  Every
// look-back wait is bounded; a wait that gives up raises a workspace error
// flag that the host turns into TG_ERR_TIMEOUT.
#include "scan.cuh"

namespace tg {

// ------------------------------------------------------------------ tile boxes
__device__ __forceinline__ void tile_box(float mx, float my, int32_t radius, int tile_size, uint32_t tw, uint32_t th,
                                         uint32_t& x0, uint32_t& y0, uint32_t& x1, uint32_t& y1) {
    const float ts = (float)tile_size;
    const float tr = __fdiv_rn((float)radius, ts);
    const float tx = __fdiv_rn(mx, ts), ty = __fdiv_rn(my, ts);
    // float -> u32 conversions saturate (negative -> 0), as in the reference
    x0 = min((uint32_t)floorf(tx - tr), tw);
    y0 = min((uint32_t)floorf(ty - tr), th);
    x1 = min((uint32_t)ceilf(tx + tr), tw);
    y1 = min((uint32_t)ceilf(ty + tr), th);
}

// Camera of element e and its tile grid; false if the camera id is out of range.
__device__ __forceinline__ bool camera_grid(const tg_isect_args& a, int64_t e, uint32_t& tw, uint32_t& th) {
    const int64_t cid = a.camera_ids ? a.camera_ids[e] : e / a.N;
    if (cid < 0 || cid >= a.n_cameras) return false;
    if (a.views) {
        tw = (uint32_t)a.views[cid].tile_width;
        th = (uint32_t)a.views[cid].tile_height;
    } else {
        tw = (uint32_t)a.tile_width;
        th = (uint32_t)a.tile_height;
    }
    return true;
}

// Phase 1: tile counts per element and per-chunk sums.
__global__ void __launch_bounds__(kScanThreads) isect_count_kernel(tg_isect_args a, int64_t* chunk_sums) {
    __shared__ int64_t s_warp[kScanThreads / 32];
    const int64_t base = (int64_t)blockIdx.x * kScanChunk;
    int64_t local = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        const int64_t e = base + (int64_t)i * kScanThreads + threadIdx.x;
        if (e >= a.n_elems) break;
        int32_t cnt = 0;
        const int32_t r = a.radii[e];
        uint32_t tw, th;
        if (r > 0 && camera_grid(a, e, tw, th)) {
            const float2 m = reinterpret_cast<const float2*>(a.means2d)[e];
            uint32_t x0, y0, x1, y1;
            tile_box(m.x, m.y, r, a.tile_size, tw, th, x0, y0, x1, y1);
            cnt = (int32_t)((y1 - y0) * (x1 - x0));
        }
        a.tiles_per_gauss[e] = cnt;
        local += cnt;
    }
    int64_t total;
    block_excl_scan(local, s_warp, total);
    if (threadIdx.x == 0) chunk_sums[blockIdx.x] = total;
}

// Phase 2: exclusive scan of the chunk sums in one CTA; writes the grand total.
__global__ void __launch_bounds__(kScanThreads) scan_chunk_sums_kernel(int64_t* chunk_sums, int64_t n_chunks,
                                                                       int64_t* n_total) {
    __shared__ int64_t s_warp[kScanThreads / 32];
    int64_t carry = 0;
    for (int64_t b = 0; b < n_chunks; b += kScanThreads) {
        const int64_t i = b + threadIdx.x;
        const int64_t v = i < n_chunks ? chunk_sums[i] : 0;
        int64_t total;
        const int64_t ex = block_excl_scan(v, s_warp, total);
        if (i < n_chunks) chunk_sums[i] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) *n_total = carry;
}

cudaError_t launch_scan_chunk_sums(int64_t* chunk_sums, int64_t n_chunks, int64_t* n_total, cudaStream_t s) {
    scan_chunk_sums_kernel<<<1, kScanThreads, 0, s>>>(chunk_sums, n_chunks, n_total);
    note_launches(1);
    return cudaGetLastError();
}

// Phase 3: inclusive prefix of tiles_per_gauss within each chunk plus the chunk offset.
__global__ void __launch_bounds__(kScanThreads) scan_apply_kernel(const int32_t* counts, int64_t n,
                                                                  const int64_t* chunk_offsets, int64_t* cum) {
    __shared__ int64_t s_warp[kScanThreads / 32];
    const int64_t base = (int64_t)blockIdx.x * kScanChunk;
    // blocked arrangement: thread t owns items [t*16, t*16+16) of the chunk
    int32_t v[kScanItems];
    int64_t local = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        const int64_t e = base + (int64_t)threadIdx.x * kScanItems + i;
        v[i] = e < n ? counts[e] : 0;
        local += v[i];
    }
    int64_t total;
    int64_t run = chunk_offsets[blockIdx.x] + block_excl_scan(local, s_warp, total);
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        const int64_t e = base + (int64_t)threadIdx.x * kScanItems + i;
        run += v[i];
        if (e < n) cum[e] = run;
    }
}

__global__ void __launch_bounds__(256) isect_emit_kernel(tg_isect_args a, int tile_n_bits) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= a.n_elems) return;
    const int32_t r = a.radii[e];
    uint32_t tw, th;
    if (r <= 0 || !camera_grid(a, e, tw, th)) return;
    const float2 m = reinterpret_cast<const float2*>(a.means2d)[e];
    uint32_t x0, y0, x1, y1;
    tile_box(m.x, m.y, r, a.tile_size, tw, th, x0, y0, x1, y1);
    const int64_t cid = a.camera_ids ? a.camera_ids[e] : e / a.N;
    const int64_t cid_enc = cid << (32 + tile_n_bits);
    const int64_t depth_enc = (int64_t)__float_as_int(a.depths[e]);  // sign-extended like the reference
    int64_t cur = e == 0 ? 0 : a.cum_tiles[e - 1];
    // capacity mode: only the first `capacity` entries exist
    const int64_t limit = a.overflow ? a.capacity : INT64_MAX;
    if (a.overflow && a.cum_tiles[e] > limit) atomicOr(a.overflow, 1u);
    for (uint32_t y = y0; y < y1; ++y)
        for (uint32_t x = x0; x < x1; ++x) {
            if (cur >= limit) return;
            const int64_t tile_id = (int64_t)y * tw + x;
            a.isect_ids[cur] = cid_enc | (tile_id << 32) | depth_enc;
            a.flatten_ids[cur] = (int32_t)e;
            ++cur;
        }
}

// Capacity mode: keys past the valid count sort after every real key.
__global__ void __launch_bounds__(256) isect_pad_kernel(int64_t* keys, int32_t* vals, const int64_t* n_dev,
                                                        int64_t capacity, int64_t pad_key) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= capacity || i < *n_dev) return;
    keys[i] = pad_key;
    vals[i] = 0;
}

// offsets[t] = lower_bound over sorted keys of (camera, tile) index t.
__global__ void __launch_bounds__(256) offset_encode_kernel(const int64_t* keys, int64_t n, int64_t n_ids,
                                                            int n_tiles, int tile_n_bits, uint64_t key_mask,
                                                            int32_t* offsets) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_ids) return;
    int64_t lo = 0, hi = n;
    const uint64_t tmask = (1ull << tile_n_bits) - 1ull;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        const uint64_t h = ((uint64_t)__ldg(keys + mid) & key_mask) >> 32;
        const int64_t id = (int64_t)(h >> tile_n_bits) * n_tiles + (int64_t)(h & tmask);
        if (id < t) lo = mid + 1; else hi = mid;
    }
    offsets[t] = (int32_t)lo;
}

// Batching form: flat tile t of view c = tile_view[t] is the key prefix
// (c << tile_bits) | (t - tile_base_c); offsets[t] = its lower bound.
__global__ void __launch_bounds__(256) offset_encode_views_kernel(const int64_t* keys, int64_t n, int64_t n_tiles,
                                                                  int C, const tg_view* views,
                                                                  const int32_t* tile_view, int tile_n_bits,
                                                                  uint64_t key_mask, int32_t* offsets) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tiles) return;
    const int c = tile_view[t];
    uint64_t target = ~0ull;  // an out-of-range view sorts after every key
    if (c >= 0 && c < C) target = ((uint64_t)c << tile_n_bits) | (uint64_t)(t - views[c].tile_base);
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        const uint64_t h = ((uint64_t)__ldg(keys + mid) & key_mask) >> 32;
        if (h < target) lo = mid + 1; else hi = mid;
    }
    offsets[t] = (int32_t)lo;
}

// ------------------------------------------------------------------ onesweep radix sort
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096 keys per CTA
constexpr int kRadix = 256;
constexpr int kMaxPasses = 8;
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagInc = 2u << 30;
constexpr uint32_t kFlagMask = 3u << 30;
constexpr uint32_t kValueMask = kFlagAgg - 1u;
constexpr uint32_t kSpinLimit = 1u << 22;  // ~0.3 s of polling with 64 ns sleeps

struct SortWorkspace {
    uint32_t* hist;          // [kMaxPasses][256] digit counts
    uint32_t* digit_offsets; // [kMaxPasses][256] exclusive scans
    uint32_t* tile_counter;  // [kMaxPasses]
    uint32_t* error;         // [1]
    uint32_t* status;        // [passes][n_tiles][256]
    size_t bytes;
};


inline SortWorkspace carve_sort_workspace(void* base, int64_t n, int passes) {
    SortWorkspace w;
    const int64_t n_tiles = (n + kSortTile - 1) / kSortTile;
    char* p = static_cast<char*>(base);
    size_t off = 0;
    w.hist = reinterpret_cast<uint32_t*>(p + off); off += align256(sizeof(uint32_t) * kMaxPasses * kRadix);
    w.digit_offsets = reinterpret_cast<uint32_t*>(p + off); off += align256(sizeof(uint32_t) * kMaxPasses * kRadix);
    w.tile_counter = reinterpret_cast<uint32_t*>(p + off); off += align256(sizeof(uint32_t) * kMaxPasses);
    w.error = reinterpret_cast<uint32_t*>(p + off); off += align256(sizeof(uint32_t));
    w.status = reinterpret_cast<uint32_t*>(p + off); off += align256(sizeof(uint32_t) * (size_t)passes * n_tiles * kRadix);
    w.bytes = off;
    return w;
}

__global__ void __launch_bounds__(kSortThreads) sort_histogram_kernel(const uint64_t* keys, int64_t n, int passes,
                                                                      int end_bit, uint32_t* hist) {
    __shared__ uint32_t s_hist[kMaxPasses * kRadix];
    for (int i = threadIdx.x; i < passes * kRadix; i += kSortThreads) s_hist[i] = 0;
    __syncthreads();
    const uint64_t mask = end_bit >= 64 ? ~0ull : ((1ull << end_bit) - 1ull);
    for (int64_t i = (int64_t)blockIdx.x * kSortThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kSortThreads) {
        const uint64_t k = keys[i] & mask;
        for (int p = 0; p < passes; ++p) atomicAdd(&s_hist[p * kRadix + ((k >> (8 * p)) & 0xffu)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * kRadix; i += kSortThreads)
        if (s_hist[i]) atomicAdd(&hist[i], s_hist[i]);
}

__global__ void __launch_bounds__(kRadix) sort_digit_offsets_kernel(const uint32_t* hist, uint32_t* offsets) {
    // one CTA per pass, one thread per digit
    __shared__ uint32_t s[kRadix];
    const int p = blockIdx.x, d = threadIdx.x;
    s[d] = hist[p * kRadix + d];
    __syncthreads();
    // Hillis-Steele inclusive scan over 256 digits
    for (int o = 1; o < kRadix; o <<= 1) {
        const uint32_t v = d >= o ? s[d - o] : 0u;
        __syncthreads();
        s[d] += v;
        __syncthreads();
    }
    offsets[p * kRadix + d] = s[d] - hist[p * kRadix + d];
}

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) { return *reinterpret_cast<const volatile uint32_t*>(p); }
__device__ __forceinline__ void st_volatile(uint32_t* p, uint32_t v) { *reinterpret_cast<volatile uint32_t*>(p) = v; }

__global__ void __launch_bounds__(kSortThreads) sort_pass_kernel(const uint64_t* __restrict__ keys_in,
                                                                 const uint32_t* __restrict__ vals_in,
                                                                 uint64_t* __restrict__ keys_out,
                                                                 uint32_t* __restrict__ vals_out, int64_t n, int shift,
                                                                 uint32_t digit_mask, const uint32_t* digit_offsets,
                                                                 uint32_t* status, uint32_t* tile_counter,
                                                                 uint32_t* error) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint64_t* s_keys = reinterpret_cast<uint64_t*>(smem_raw);
    uint32_t* s_vals = reinterpret_cast<uint32_t*>(s_keys + kSortTile);
    uint32_t* s_whist = s_vals + kSortTile;             // [warps][256]
    uint32_t* s_tile_start = s_whist + kSortWarps * kRadix;  // [256]
    uint32_t* s_gbase = s_tile_start + kRadix;          // [256]
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_scan[kSortWarps];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(tile_counter, 1u);
    for (int i = tid; i < kSortWarps * kRadix; i += kSortThreads) s_whist[i] = 0;
    __syncthreads();
    const uint32_t tile = s_tile;
    const int64_t base = (int64_t)tile * kSortTile;

    uint64_t k[kSortItems];
    uint32_t v[kSortItems];
    uint32_t dg[kSortItems];
    uint32_t rk[kSortItems];
    const int64_t wbase = base + (int64_t)warp * (kSortItems * 32);
#pragma unroll
    for (int i = 0; i < kSortItems; ++i) {
        const int64_t pos = wbase + i * 32 + lane;
        const bool ok = pos < n;
        k[i] = ok ? keys_in[pos] : 0ull;
        v[i] = ok ? vals_in[pos] : 0u;
        dg[i] = ok ? (uint32_t)((k[i] >> shift) & digit_mask) : (uint32_t)kRadix;  // kRadix marks padding
    }
    const unsigned lt = lanemask_lt();
    uint32_t* wh = s_whist + warp * kRadix;
#pragma unroll
    for (int i = 0; i < kSortItems; ++i) {
        const unsigned peers = __match_any_sync(0xffffffffu, dg[i]);
        const int leader = __ffs(peers) - 1;
        uint32_t b = 0;
        if (lane == leader && dg[i] < (uint32_t)kRadix) {
            b = wh[dg[i]];
            wh[dg[i]] = b + __popc(peers);
        }
        b = __shfl_sync(peers, b, leader);
        rk[i] = b + __popc(peers & lt);
    }
    __syncthreads();

    // per digit (thread = digit): exclusive scan over warps, tile total
    const int d = tid;
    uint32_t count = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) {
        const uint32_t c = s_whist[w * kRadix + d];
        s_whist[w * kRadix + d] = count;
        count += c;
    }
    uint32_t* st = status + (size_t)tile * kRadix;
    if (tile == 0) {
        st_volatile(st + d, kFlagInc | count);
    } else {
        st_volatile(st + d, kFlagAgg | count);
    }
    uint32_t prefix = 0;
    if (tile > 0) {
        int64_t j = (int64_t)tile - 1;
        while (j >= 0) {
            const uint32_t* src = status + (size_t)j * kRadix + d;
            uint32_t s = ld_volatile(src);
            uint32_t iter = 0;
            while ((s & kFlagMask) == 0u) {
                if (++iter > kSpinLimit) break;
                __nanosleep(64);
                s = ld_volatile(src);
            }
            if ((s & kFlagMask) == 0u) {  // gave up: record and stop waiting
                atomicExch(error, 1u);
                break;
            }
            prefix += s & kValueMask;
            if (s & kFlagInc) break;
            --j;
        }
        st_volatile(st + d, kFlagInc | (prefix + count));
    }
    s_gbase[d] = digit_offsets[d] + prefix;

    // exclusive scan of the tile's digit counts -> start of each digit in the tile
    uint32_t incl = count;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t u = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += u;
    }
    if (lane == 31) s_scan[warp] = incl;
    __syncthreads();
    uint32_t wpre = 0;
    for (int w = 0; w < warp; ++w) wpre += s_scan[w];
    s_tile_start[d] = wpre + incl - count;
    __syncthreads();

#pragma unroll
    for (int i = 0; i < kSortItems; ++i) {
        if (dg[i] < (uint32_t)kRadix) {
            const uint32_t lp = s_tile_start[dg[i]] + wh[dg[i]] + rk[i];
            s_keys[lp] = k[i];
            s_vals[lp] = v[i];
        }
    }
    __syncthreads();
    const int64_t rem = n - base;
    const int tile_n = rem < kSortTile ? (int)rem : kSortTile;
    for (int j = tid; j < tile_n; j += kSortThreads) {
        const uint64_t key = s_keys[j];
        const uint32_t dd = (uint32_t)((key >> shift) & digit_mask);
        const uint32_t pos = s_gbase[dd] + ((uint32_t)j - s_tile_start[dd]);
        keys_out[pos] = key;
        vals_out[pos] = s_vals[j];
    }
}

constexpr size_t kSortSmem = sizeof(uint64_t) * kSortTile + sizeof(uint32_t) * kSortTile +
                             sizeof(uint32_t) * (kSortWarps * kRadix + 2 * kRadix);

size_t sort_workspace_bytes(int64_t n, int end_bit) {
    const int passes = (end_bit + 7) / 8;
    return carve_sort_workspace(nullptr, n, passes).bytes;
}

// Returns TG_OK / TG_ERR_*; *result_in_alt tells where the sorted data ends.
int sort_pairs(int64_t* keys, int32_t* vals, int64_t* keys_alt, int32_t* vals_alt, int64_t n, int end_bit,
               void* workspace, size_t ws_bytes, int32_t* result_in_alt, cudaStream_t s, cudaError_t& cerr) {
    cerr = cudaSuccess;
    *result_in_alt = 0;
    if (n <= 1 || end_bit <= 0) return TG_OK;
    const int passes = (end_bit + 7) / 8;
    if (passes > kMaxPasses) return TG_ERR_INVALID_ARG;
    SortWorkspace w = carve_sort_workspace(workspace, n, passes);
    if (ws_bytes < w.bytes) return TG_ERR_WORKSPACE;
    const int64_t n_tiles = (n + kSortTile - 1) / kSortTile;
    if ((cerr = cudaMemsetAsync(workspace, 0, w.bytes, s)) != cudaSuccess) return TG_ERR_CUDA;
    const int hist_blocks = (int)std::min<int64_t>(n_tiles, (int64_t)kNumSMs * 4);
    sort_histogram_kernel<<<hist_blocks, kSortThreads, 0, s>>>(reinterpret_cast<const uint64_t*>(keys), n, passes,
                                                               end_bit, w.hist);
    sort_digit_offsets_kernel<<<passes, kRadix, 0, s>>>(w.hist, w.digit_offsets);
    note_launches(2);
    if ((cerr = cudaGetLastError()) != cudaSuccess) return TG_ERR_CUDA;
    // a per-device function attribute: set on every call (cheap, allowed during stream capture)
    if ((cerr = cudaFuncSetAttribute(sort_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)kSortSmem)) != cudaSuccess)
        return TG_ERR_CUDA;
    uint64_t* kin = reinterpret_cast<uint64_t*>(keys);
    uint32_t* vin = reinterpret_cast<uint32_t*>(vals);
    uint64_t* kout = reinterpret_cast<uint64_t*>(keys_alt);
    uint32_t* vout = reinterpret_cast<uint32_t*>(vals_alt);
    for (int p = 0; p < passes; ++p) {
        const int shift = 8 * p;
        const int bits = std::min(8, end_bit - shift);
        const uint32_t dmask = (1u << bits) - 1u;
        sort_pass_kernel<<<(unsigned)n_tiles, kSortThreads, kSortSmem, s>>>(
            kin, vin, kout, vout, n, shift, dmask, w.digit_offsets + p * kRadix,
            w.status + (size_t)p * n_tiles * kRadix, w.tile_counter + p, w.error);
        if ((cerr = cudaGetLastError()) != cudaSuccess) return TG_ERR_CUDA;
        note_launches(1);
        std::swap(kin, kout);
        std::swap(vin, vout);
    }
    *result_in_alt = passes & 1;
    return TG_OK;
}

__global__ void set_u32_kernel(uint32_t* p, uint32_t v) { *p = v; }

// Diagnostic: one pass over two tiles (8192 pairs, 8 key bits) run by a single
// CTA whose tile counter is preset to 1, so its look-back waits on tile 0,
// which never publishes.  The bounded wait gives up after kSpinLimit polls and
// raises the error flag; a partial prefix only lowers scatter positions, so
// every write stays inside the output buffers.
int sort_lookback_selftest(int64_t* keys, int32_t* vals, int64_t* keys_alt, int32_t* vals_alt, void* workspace,
                           size_t ws_bytes, cudaStream_t s, cudaError_t& cerr) {
    cerr = cudaSuccess;
    constexpr int64_t n = 2 * kSortTile;
    SortWorkspace w = carve_sort_workspace(workspace, n, 1);
    if (ws_bytes < w.bytes) return TG_ERR_WORKSPACE;
    if ((cerr = cudaMemsetAsync(workspace, 0, w.bytes, s)) != cudaSuccess) return TG_ERR_CUDA;
    set_u32_kernel<<<1, 1, 0, s>>>(w.tile_counter, 1u);  // the single CTA takes tile 1
    sort_histogram_kernel<<<2, kSortThreads, 0, s>>>(reinterpret_cast<const uint64_t*>(keys), n, 1, 8, w.hist);
    sort_digit_offsets_kernel<<<1, kRadix, 0, s>>>(w.hist, w.digit_offsets);
    if ((cerr = cudaFuncSetAttribute(sort_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)kSortSmem)) != cudaSuccess)
        return TG_ERR_CUDA;
    sort_pass_kernel<<<1, kSortThreads, kSortSmem, s>>>(
        reinterpret_cast<const uint64_t*>(keys), reinterpret_cast<const uint32_t*>(vals),
        reinterpret_cast<uint64_t*>(keys_alt), reinterpret_cast<uint32_t*>(vals_alt), n, 0, 0xffu, w.digit_offsets,
        w.status, w.tile_counter, w.error);
    note_launches(4);
    if ((cerr = cudaGetLastError()) != cudaSuccess) return TG_ERR_CUDA;
    uint32_t h = 0;
    if ((cerr = cudaStreamSynchronize(s)) != cudaSuccess) return TG_ERR_CUDA;
    if ((cerr = cudaMemcpy(&h, w.error, sizeof(h), cudaMemcpyDeviceToHost)) != cudaSuccess) return TG_ERR_CUDA;
    return h ? TG_ERR_TIMEOUT : TG_OK;
}

// error flag location inside a carved workspace (for the host to read back)
uint32_t* sort_error_flag(void* workspace, int64_t n, int end_bit) {
    return carve_sort_workspace(workspace, n, (end_bit + 7) / 8).error;
}

size_t scan_workspace_bytes(int64_t n_elems) {
    const int64_t chunks = (n_elems + kScanChunk - 1) / kScanChunk;
    return align256(sizeof(int64_t) * (size_t)std::max<int64_t>(chunks, 1));
}

cudaError_t launch_isect_count(const tg_isect_args& a, cudaStream_t s) {
    const int64_t chunks = (a.n_elems + kScanChunk - 1) / kScanChunk;
    if (a.n_elems == 0) return cudaMemsetAsync(a.n_isects, 0, sizeof(int64_t), s);
    int64_t* sums = static_cast<int64_t*>(a.scan_workspace);
    isect_count_kernel<<<(unsigned)chunks, kScanThreads, 0, s>>>(a, sums);
    scan_chunk_sums_kernel<<<1, kScanThreads, 0, s>>>(sums, chunks, a.n_isects);
    scan_apply_kernel<<<(unsigned)chunks, kScanThreads, 0, s>>>(a.tiles_per_gauss, a.n_elems, sums, a.cum_tiles);
    note_launches(3);
    return cudaGetLastError();
}

cudaError_t launch_isect_emit(const tg_isect_args& a, int tile_n_bits, int end_bit, cudaStream_t s) {
    if (a.n_elems > 0) {
        isect_emit_kernel<<<(unsigned)((a.n_elems + 255) / 256), 256, 0, s>>>(a, tile_n_bits);
        note_launches(1);
    }
    if (a.overflow && a.capacity > 0) {
        const int64_t pad = end_bit >= 63 ? INT64_MAX : (int64_t)((1ull << end_bit) - 1ull);
        isect_pad_kernel<<<(unsigned)((a.capacity + 255) / 256), 256, 0, s>>>(a.isect_ids, a.flatten_ids, a.n_isects,
                                                                              a.capacity, pad);
        note_launches(1);
    }
    return cudaGetLastError();
}

cudaError_t launch_offset_encode_views(const int64_t* keys, int64_t n, int C, int64_t n_tiles, const tg_view* views,
                                       const int32_t* tile_view, int tile_n_bits, int end_bit, int32_t* offsets,
                                       cudaStream_t s) {
    if (n_tiles == 0) return cudaSuccess;
    const uint64_t key_mask = end_bit >= 64 ? ~0ull : ((1ull << end_bit) - 1ull);
    offset_encode_views_kernel<<<(unsigned)((n_tiles + 255) / 256), 256, 0, s>>>(keys, n, n_tiles, C, views, tile_view,
                                                                                tile_n_bits, key_mask, offsets);
    note_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_offset_encode(const int64_t* keys, int64_t n, int C, int tw, int th, int tile_n_bits,
                                 int end_bit, int32_t* offsets, cudaStream_t s) {
    const int64_t n_ids = (int64_t)C * tw * th;
    if (n_ids == 0) return cudaSuccess;
    const uint64_t mask = end_bit >= 64 ? ~0ull : ((1ull << end_bit) - 1ull);
    offset_encode_kernel<<<(unsigned)((n_ids + 255) / 256), 256, 0, s>>>(keys, n, n_ids, tw * th, tile_n_bits, mask,
                                                                       offsets);
    note_launches(1);
    return cudaGetLastError();
}

}  // namespace tg
