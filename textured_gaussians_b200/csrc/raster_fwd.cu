// Textured / plain 2DGS compositor, forward, for sm_100a.
//
// One CTA per (camera, tile) work item, front-to-back over the tile's depth-sorted
// splats in batches of `batch_depth` splats (tile_size^2 by default) staged in
// shared memory (the gather of each splat's record happens once per CTA, not
// once per pixel).  8x8 and 16x16 tiles run one thread per pixel; 32x32 tiles
// run 256 threads owning PPT = 4 pixels each (rows r, r+8, r+16, r+24): the
// PPT evaluations of a splat are independent, so their texture loads are in
// flight together, and the splat's shared-memory record is read once for all.
// Each pixel samples its splat's RGBA texture with one 16-byte (FP32), 8-byte
// (BF16/FP16) or 4-byte (FP8) load per bilinear tap and reuses the four taps for
// the alpha scale and every colour channel.  A warp whose pixels are all
// saturated stops early; a CTA whose pixels are all saturated stops at the next
// batch boundary.  Per-Gaussian contribution statistics are reduced across the
// warp before one global atomic.
//
// Semantics: textured_gaussians/cuda/csrc/rasterize_to_pixels_textured_
// gaussians_2dgs_fwd.cu:73-445 and rasterize_to_pixels_2dgs_fwd.cu (plain),
// with the texture / statistics row of element e taken as e % N (dense) or
// gaussian_ids[e] (packed) instead of the reference's out-of-range e.
#include "raster_common.cuh"

namespace tg {

// Resident CTAs per SM the register allocation targets.
#ifndef TG_FWD_MIN_CTAS
#define TG_FWD_MIN_CTAS 4
#endif

// Register budget: 4 resident CTAs of 256 threads for one pixel per thread;
// one CTA for the four-pixel (32x32 tile) form.  The anisotropic_bilinear
// forward keeps this budget too (TG_FWD_MIN_CTAS_ANISO): it spills ~0.5 KB at
// 64 registers but runs 13 % faster than at 128 and 2-3.5 % faster than at 3
// CTAs (measured).
#ifndef TG_FWD_MIN_CTAS_ANISO
#define TG_FWD_MIN_CTAS_ANISO TG_FWD_MIN_CTAS
#endif
template <int PPT, class Filt>
struct FwdBounds {
    static constexpr int kMinCtas = PPT == 1 ? (Filt::kAniso ? TG_FWD_MIN_CTAS_ANISO : TG_FWD_MIN_CTAS) : 1;
};

// One work item (tile) of the forward; every early return is uniform over the CTA.
template <int D, class Tex, int PPT, class Filt = FiltBilinear>
__device__ __forceinline__ void fwd_tile(const tg_raster_fwd_args& a, const int bs, const int64_t item) {
    constexpr bool kTextured = Tex::kFormat != TG_TEX_NONE;
    extern __shared__ float4 smem4[];
    const int nt = blockDim.x;  // threads: tile_size^2 / PPT; bs = splats staged per batch
    float4* s_box = smem4;  // per-splat cull box (see cull_box)
    float4* s_xyo = s_box + bs;
    float4* s_m0 = s_xyo + bs;
    float4* s_m1 = s_m0 + bs;
    float4* s_m2 = s_m1 + bs;
    float4* s_nrm = s_m2 + bs;
    float* s_col = reinterpret_cast<float*>(s_nrm + bs);
    int* s_row = reinterpret_cast<int*>(s_col + bs * D);
    // anisotropic_bilinear: the boundary integration's per-warp area (16-byte aligned: bs is a multiple of 32)
    float4* s_aniso = Filt::kAniso ? reinterpret_cast<float4*>(s_row + bs) + (threadIdx.x >> 5) * kAnisoWarpF4
                                   : nullptr;

    const unsigned wmask = __activemask();
    const TileWork tc = tile_work(a, item);
    if (!tc.valid) return;  // uniform over the CTA
    const int tr = threadIdx.x, lane = tr & 31;
    const int ts = a.tile_size;

    int64_t pix[PPT];
    bool inside[PPT], done[PPT];
    float px[PPT], py[PPT];
#pragma unroll
    for (int q = 0; q < PPT; ++q) {
        const int local = tr + q * nt;
        const int i = tc.ty * ts + local / ts;
        const int j = tc.tx * ts + local % ts;
        pix[q] = pixel_index(tc, i, j);
        inside[q] = pix[q] >= 0;
        px[q] = (float)j + 0.5f;
        py[q] = (float)i + 0.5f;
        done[q] = !inside[q];
    }

    if (a.masks != nullptr && !a.masks[tc.t]) {
#pragma unroll
        for (int q = 0; q < PPT; ++q) {
            if (!inside[q]) continue;
            const int64_t p = pix[q];
#pragma unroll
            for (int k = 0; k < D; ++k) a.out_colors[p * D + k] = a.backgrounds ? a.backgrounds[tc.c * D + k] : 0.f;
            a.out_alphas[p] = 0.f;
            a.out_normals[p * 3] = a.out_normals[p * 3 + 1] = a.out_normals[p * 3 + 2] = 0.f;
            a.out_distort[p] = 0.f;
            a.out_median[p] = 0.f;
            a.last_ids[p] = 0;
            a.median_ids[p] = 0;
        }
        return;
    }

    // pixel-centre rectangle covered by this warp (for the warp-level cull)
    float wx0 = INFINITY, wx1 = -INFINITY, wy0 = INFINITY, wy1 = -INFINITY;
#pragma unroll
    for (int q = 0; q < PPT; ++q) {
        const int local = tr + q * nt;
        const float cx = (float)(tc.tx * ts + local % ts) + 0.5f, cy = (float)(tc.ty * ts + local / ts) + 0.5f;
        wx0 = fminf(wx0, cx); wx1 = fmaxf(wx1, cx); wy0 = fminf(wy0, cy); wy1 = fmaxf(wy1, cy);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        wx0 = fminf(wx0, __shfl_xor_sync(wmask, wx0, o)); wx1 = fmaxf(wx1, __shfl_xor_sync(wmask, wx1, o));
        wy0 = fminf(wy0, __shfl_xor_sync(wmask, wy0, o)); wy1 = fmaxf(wy1, __shfl_xor_sync(wmask, wy1, o));
    }
    const int32_t range_start = tc.range_start;
    const int32_t range_end = tc.range_end;
    const int num_batches = (range_end - range_start + bs - 1) / bs;
    const int64_t tex_stride = (int64_t)a.tex_ry * a.tex_rx;
    const int mip_clen = Filt::kMip ? ((1 << (2 * a.mip_levels)) - 1) / 3 : 0;

    float T[PPT], pix_out[PPT][D], nrm_out[PPT][3], distort[PPT], accum_vis_depth[PPT], median_depth[PPT];
    int32_t cur_idx[PPT], median_idx[PPT];
    // anisotropic_bilinear records: footprint integrals computed so far, and those up to the last contributor
    int32_t rec_n[PPT], rec_last[PPT];
    const bool records = Filt::kAniso && a.aniso_records != nullptr;
#pragma unroll
    for (int q = 0; q < PPT; ++q) {
        T[q] = 1.f;
#pragma unroll
        for (int k = 0; k < D; ++k) pix_out[q][k] = 0.f;
        nrm_out[q][0] = nrm_out[q][1] = nrm_out[q][2] = 0.f;
        distort[q] = accum_vis_depth[q] = median_depth[q] = 0.f;
        cur_idx[q] = median_idx[q] = 0;
        rec_n[q] = rec_last[q] = 0;
    }

    for (int b = 0; b < num_batches; ++b) {
        bool all_done = true;
#pragma unroll
        for (int q = 0; q < PPT; ++q) all_done &= done[q];
        if (__syncthreads_count(all_done) >= nt) break;
        const int32_t batch_start = range_start + bs * b;
        for (int slot = tr; slot < bs; slot += nt) {
            const int32_t idx = batch_start + slot;
            if (idx < range_end) {
                const int32_t g = a.flatten_ids[idx];
                const float2 xy = reinterpret_cast<const float2*>(a.means2d)[g];
                const int32_t row = a.gaussian_ids ? (int32_t)a.gaussian_ids[g] : g % a.N;
                const float scale = (Tex::kFormat == TG_TEX_FP8_E4M3) ? a.tex_scales[row] : 1.f;
                s_xyo[slot] = make_float4(xy.x, xy.y, a.opacities[g], scale);
                const float* m = a.ray_transforms + 9 * (int64_t)g;
                s_m0[slot] = make_float4(m[0], m[1], m[2], 0.f);
                s_m1[slot] = make_float4(m[3], m[4], m[5], 0.f);
                s_m2[slot] = make_float4(m[6], m[7], m[8], 0.f);
                s_box[slot] = cull_box(s_xyo[slot], s_m0[slot], s_m1[slot], s_m2[slot], kTextured, a.range_x, a.range_y,
                                       a.g_weight, !Filt::kAniso);
                const float* n = a.normals + 3 * (int64_t)g;
                s_nrm[slot] = make_float4(n[0], n[1], n[2], 0.f);
#pragma unroll
                for (int k = 0; k < D; ++k) s_col[slot * D + k] = a.colors[(int64_t)g * D + k];
                s_row[slot] = row;
            }
        }
        __syncthreads();
        const int batch_size = min(bs, range_end - batch_start);
        for (int t = 0; t < batch_size; ++t) {
            bool warp_done = true;
#pragma unroll
            for (int q = 0; q < PPT; ++q) warp_done &= done[q];
            if (__all_sync(wmask, warp_done)) break;
            const float4 box = s_box[t];
            if (box.z < wx0 || box.x > wx1 || box.w < wy0 || box.y > wy1) continue;  // no pixel of this warp can be valid
            const float4 xyo = s_xyo[t], m0 = s_m0[t], m1 = s_m1[t], m2 = s_m2[t];
            const int row = s_row[t];
            const int64_t tex_base = (int64_t)row * tex_stride;
            float csum = 0.f;
            int ccount = 0;
#pragma unroll
            for (int q = 0; q < PPT; ++q) {
                const bool act = !done[q] && in_box(box, px[q], py[q]);
                PairOf<Filt> e;
                if constexpr (Filt::kAniso) {  // every lane takes part: the warp integrates footprints together
                    eval_aniso_coop<Tex>(e, act, px[q], py[q], xyo, m0, m1, m2, a.textures, tex_base, a.tex_rx,
                                         a.tex_ry, a.range_x, a.range_y, a.g_weight, wmask,
                                         a.aniso_prefix ? reinterpret_cast<const float4*>(a.aniso_prefix) + tex_base
                                                        : nullptr,
                                         s_aniso);
                    if (!act) continue;
                    if (records && e.tex_valid) {  // every integral, in order, whether or not the pair is kept
                        if (rec_n[q] < a.aniso_record_cap)
                            reinterpret_cast<float4*>(a.aniso_records)[pix[q] * a.aniso_record_cap + rec_n[q]] =
                                e.tsum;
                        ++rec_n[q];
                    }
                } else {
                    if (!act) continue;
                    eval_pair<Tex, Filt>(e, px[q], py[q], xyo, m0, m1, m2, a.textures, tex_base, a.tex_rx, a.tex_ry,
                                         a.range_x, a.range_y, a.g_weight,
                                         MipSrc{a.tex_coarse, (int64_t)row * mip_clen, mip_clen, a.mip_levels});
                }
                if (!e.valid) continue;
                const float next_T = T[q] * (1.f - e.alpha);
                if (next_T <= 1e-4f) {
                    done[q] = true;
                    continue;
                }
                const float vis = e.alpha * T[q];
                const float* cp = s_col + t * D;
#pragma unroll
                for (int k = 0; k < D; ++k) pix_out[q][k] += (cp[k] + (kTextured ? tex_color(e, k) : 0.f)) * vis;
                const float4 nn = s_nrm[t];
                nrm_out[q][0] += nn.x * vis;
                nrm_out[q][1] += nn.y * vis;
                nrm_out[q][2] += nn.z * vis;
                const float depth = cp[D - 1];
                distort[q] += 2.f * (vis * depth * (1.f - T[q]) - vis * accum_vis_depth[q]);
                accum_vis_depth[q] += vis * depth;
                if (T[q] > 0.5f) {
                    median_depth[q] = depth;
                    median_idx[q] = batch_start + t;
                }
                cur_idx[q] = batch_start + t;
                rec_last[q] = rec_n[q];
                T[q] = next_T;
                if (e.alpha > a.contrib_threshold) {
                    csum += e.alpha;
                    ++ccount;
                }
            }
            if (__any_sync(wmask, ccount > 0)) {
                // one-instruction warp sums: the alphas (each < 1, at most PPT per lane) in 2^-24 fixed point,
                // so 32 lanes' sums fit in 32 bits; the quantisation is at the FP32 rounding level of the sum
                const unsigned s = __reduce_add_sync(wmask, __float2uint_rn(csum * 16777216.f));
                const unsigned c = __reduce_add_sync(wmask, (unsigned)ccount);
                if (lane == __ffs(wmask) - 1) {
                    atomicAdd(a.contrib_sum + row, (float)s * (1.f / 16777216.f));
                    atomicAdd(a.contrib_count + row, (float)c);
                }
            }
        }
        if (a.t_checkpoints != nullptr) {  // every pixel's transmittance at the end of this batch
            float* ck = a.t_checkpoints + ((int64_t)tc.t + range_start / bs + b) * (int64_t)(nt * PPT);
#pragma unroll
            for (int q = 0; q < PPT; ++q) ck[tr + q * nt] = T[q];
        }
    }
#pragma unroll
    for (int q = 0; q < PPT; ++q) {
        if (!inside[q]) continue;
        const int64_t p = pix[q];
        a.out_alphas[p] = 1.f - T[q];
#pragma unroll
        for (int k = 0; k < D; ++k)
            a.out_colors[p * D + k] = a.backgrounds ? pix_out[q][k] + T[q] * a.backgrounds[tc.c * D + k] : pix_out[q][k];
        a.out_normals[p * 3] = nrm_out[q][0];
        a.out_normals[p * 3 + 1] = nrm_out[q][1];
        a.out_normals[p * 3 + 2] = nrm_out[q][2];
        a.last_ids[p] = cur_idx[q];
        a.out_distort[p] = distort[q];
        a.out_median[p] = median_depth[q];
        a.median_ids[p] = median_idx[q];
        if (records) a.aniso_record_count[p] = rec_last[q];
    }
}

// CTA per work item, or (work_queue != NULL) a persistent grid whose CTAs take
// items from the queue counter until none is left.
template <int D, class Tex, int PPT, bool kPersistent, class Filt = FiltBilinear>
__global__ void __launch_bounds__(256, FwdBounds<PPT, Filt>::kMinCtas) raster_fwd_kernel(const tg_raster_fwd_args a,
                                                                                   const int bs,
                                                                                   const int64_t n_items) {
    if constexpr (!kPersistent) {
        fwd_tile<D, Tex, PPT, Filt>(a, bs, blockIdx.x);
        return;
    }
    else {
        __shared__ int64_t s_item;
        for (;;) {
            if (threadIdx.x == 0) s_item = (int64_t)atomicAdd(a.work_queue, 1u);
            __syncthreads();  // also: every thread is done with the previous item's shared memory
            const int64_t item = s_item;
            __syncthreads();  // s_item read by all before it is rewritten
            if (item >= n_items) return;
            fwd_tile<D, Tex, PPT, Filt>(a, bs, item);
        }
    }
}

size_t fwd_smem_bytes(int D, int bs) { return (size_t)bs * (6 * sizeof(float4) + D * sizeof(float) + sizeof(int)); }

// mipmapped2 / anisotropic_bilinear filters: one pixel per thread (8x8 / 16x16 tiles), one CTA per tile
template <int D, class Tex, class Filt>
cudaError_t launch_fwd_filter(const tg_raster_fwd_args& a, cudaStream_t s) {
    const int tile_px = a.tile_size * a.tile_size;
    const int bs = a.batch_depth > 0 ? a.batch_depth : tile_px;
    const size_t smem = fwd_smem_bytes(D, bs) + (Filt::kAniso ? (size_t)(tile_px / 32) * kAnisoWarpF4 * 16 : 0);
    const int64_t blocks = a.views ? a.n_tiles : (int64_t)a.C * a.tile_width * a.tile_height;
    if (blocks == 0) return cudaSuccess;
    cudaError_t err = cudaFuncSetAttribute(raster_fwd_kernel<D, Tex, 1, false, Filt>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    raster_fwd_kernel<D, Tex, 1, false, Filt><<<(unsigned)blocks, tile_px, smem, s>>>(a, bs, blocks);
    note_launches(1);
    return cudaGetLastError();
}

template <int D, class Tex>
cudaError_t launch_fwd_t(const tg_raster_fwd_args& a, cudaStream_t s) {
    if constexpr ((D == 3 || D == 4) && (Tex::kFormat == TG_TEX_F32 || Tex::kFormat == TG_TEX_BF16)) {
        if (a.mip_levels > 0) return launch_fwd_filter<D, Tex, FiltMip2>(a, s);
        if (a.filter == TG_FILTER_ANISO_BILINEAR) return launch_fwd_filter<D, Tex, FiltAniso>(a, s);
    }
    if (a.mip_levels > 0 || a.filter != TG_FILTER_BILINEAR) return cudaErrorInvalidValue;
    const int tile_px = a.tile_size * a.tile_size;
    const int bs = a.batch_depth > 0 ? a.batch_depth : tile_px;
    const size_t smem = fwd_smem_bytes(D, bs);
    const int64_t blocks = a.views ? a.n_tiles : (int64_t)a.C * a.tile_width * a.tile_height;
    if (blocks == 0) return cudaSuccess;
    const bool four = tile_px > 256;  // 32x32 tiles: four pixels per thread, 256 threads
    const bool pers = a.work_queue != nullptr;
    const void* fn = four ? (pers ? (const void*)raster_fwd_kernel<D, Tex, 4, true>
                                  : (const void*)raster_fwd_kernel<D, Tex, 4, false>)
                          : (pers ? (const void*)raster_fwd_kernel<D, Tex, 1, true>
                                  : (const void*)raster_fwd_kernel<D, Tex, 1, false>);
    const int threads = four ? tile_px / 4 : tile_px;
    cudaError_t err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    int64_t grid = blocks;
    if (pers) {
        if ((err = cudaMemsetAsync(a.work_queue, 0, sizeof(uint32_t), s)) != cudaSuccess) return err;
        if ((err = persistent_grid(fn, threads, smem, blocks, grid)) != cudaSuccess) return err;
    }
    const dim3 g((unsigned)grid), b((unsigned)threads);
    if (four && pers) raster_fwd_kernel<D, Tex, 4, true><<<g, b, smem, s>>>(a, bs, blocks);
    else if (four) raster_fwd_kernel<D, Tex, 4, false><<<g, b, smem, s>>>(a, bs, blocks);
    else if (pers) raster_fwd_kernel<D, Tex, 1, true><<<g, b, smem, s>>>(a, bs, blocks);
    else raster_fwd_kernel<D, Tex, 1, false><<<g, b, smem, s>>>(a, bs, blocks);
    note_launches(1);
    return cudaGetLastError();
}

template <class Tex>
cudaError_t launch_fwd_d(const tg_raster_fwd_args& a, cudaStream_t s) {
    switch (a.D) {
        case 1: return launch_fwd_t<1, Tex>(a, s);
        case 2: return launch_fwd_t<2, Tex>(a, s);
        case 3: return launch_fwd_t<3, Tex>(a, s);
        case 4: return launch_fwd_t<4, Tex>(a, s);
        case 5: return launch_fwd_t<5, Tex>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

// Low-precision texture forms are built for the RGB and RGB+D channel counts.
template <class Tex>
cudaError_t launch_fwd_d34(const tg_raster_fwd_args& a, cudaStream_t s) {
    switch (a.D) {
        case 3: return launch_fwd_t<3, Tex>(a, s);
        case 4: return launch_fwd_t<4, Tex>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_raster_fwd(const tg_raster_fwd_args& a, cudaStream_t s) {
    switch (a.tex_format) {
        case TG_TEX_NONE: return launch_fwd_d<TexNone>(a, s);
        case TG_TEX_F32: return launch_fwd_d<TexF32>(a, s);
        case TG_TEX_BF16: return launch_fwd_d34<TexBF16>(a, s);
        case TG_TEX_F16: return launch_fwd_d34<TexF16>(a, s);
        case TG_TEX_FP8_E4M3: return launch_fwd_d34<TexFP8>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace tg
