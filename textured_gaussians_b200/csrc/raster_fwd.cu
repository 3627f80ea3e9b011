// Textured / plain 2DGS compositor, forward, for sm_100a.
//
// One CTA per (camera, tile), one thread per pixel, front-to-back over the
// tile's depth-sorted splats in batches of blockDim splats staged in shared
// memory (the gather of each splat's record happens once per CTA, not once
// per pixel).  Each pixel samples its splat's RGBA texture with one 16-byte
// (FP32) or 8-byte (BF16/FP16) or 4-byte (FP8) load per bilinear tap and
// reuses the four taps for the alpha scale and every colour channel.  A warp
// whose pixels are all saturated stops early; a CTA whose pixels are all
// saturated stops at the next batch boundary.  Per-Gaussian contribution
// statistics are reduced across the warp before one global atomic.
//
// Semantics: textured_gaussians/cuda/csrc/rasterize_to_pixels_textured_
// gaussians_2dgs_fwd.cu:73-445 and rasterize_to_pixels_2dgs_fwd.cu (plain),
// with the texture / statistics row of element e taken as e % N (dense) or
// gaussian_ids[e] (packed) instead of the reference's out-of-range e.
#include "raster_common.cuh"

namespace tg {

template <int D, class Tex>
__global__ void __launch_bounds__(256) raster_fwd_kernel(const tg_raster_fwd_args a) {
    constexpr bool kTextured = Tex::kFormat != TG_TEX_NONE;
    extern __shared__ float4 smem4[];
    const int bs = blockDim.x;
    float4* s_xyo = smem4;
    float4* s_m0 = s_xyo + bs;
    float4* s_m1 = s_m0 + bs;
    float4* s_m2 = s_m1 + bs;
    float4* s_nrm = s_m2 + bs;
    float* s_col = reinterpret_cast<float*>(s_nrm + bs);
    int* s_row = reinterpret_cast<int*>(s_col + bs * D);

    const unsigned wmask = __activemask();  // lanes of this warp that exist (tile_size^2 may not fill it)
    const TileCoord tc = tile_of_block(a.tile_width, a.tile_height);
    const int tr = threadIdx.x, lane = tr & 31;
    const int ts = a.tile_size;
    const int i = tc.ty * ts + tr / ts;
    const int j = tc.tx * ts + tr % ts;
    const bool inside = i < a.height && j < a.width;
    const int64_t pix = ((int64_t)tc.c * a.height + i) * a.width + j;
    const int per_cam = a.tile_width * a.tile_height;

    if (a.masks != nullptr && !a.masks[(int64_t)tc.c * per_cam + tc.tile]) {
        if (inside) {
#pragma unroll
            for (int k = 0; k < D; ++k)
                a.out_colors[pix * D + k] = a.backgrounds ? a.backgrounds[tc.c * D + k] : 0.f;
            a.out_alphas[pix] = 0.f;
            a.out_normals[pix * 3] = a.out_normals[pix * 3 + 1] = a.out_normals[pix * 3 + 2] = 0.f;
            a.out_distort[pix] = 0.f;
            a.out_median[pix] = 0.f;
            a.last_ids[pix] = 0;
            a.median_ids[pix] = 0;
        }
        return;
    }

    const int64_t toff = (int64_t)tc.c * per_cam + tc.tile;
    const int32_t range_start = a.tile_offsets[toff];
    const int32_t range_end = (tc.c == a.C - 1 && tc.tile == per_cam - 1) ? (int32_t)a.n_isects : a.tile_offsets[toff + 1];
    const int num_batches = (range_end - range_start + bs - 1) / bs;

    const float px = (float)j + 0.5f, py = (float)i + 0.5f;
    const int64_t tex_stride = (int64_t)a.tex_ry * a.tex_rx;
    bool done = !inside;
    float T = 1.f;
    float pix_out[D];
#pragma unroll
    for (int k = 0; k < D; ++k) pix_out[k] = 0.f;
    float nrm_out[3] = {0.f, 0.f, 0.f};
    float distort = 0.f, accum_vis_depth = 0.f, median_depth = 0.f;
    int32_t cur_idx = 0, median_idx = 0;

    for (int b = 0; b < num_batches; ++b) {
        if (__syncthreads_count(done) >= bs) break;
        const int32_t batch_start = range_start + bs * b;
        const int32_t idx = batch_start + tr;
        if (idx < range_end) {
            const int32_t g = a.flatten_ids[idx];
            const float2 xy = reinterpret_cast<const float2*>(a.means2d)[g];
            const int32_t row = a.gaussian_ids ? (int32_t)a.gaussian_ids[g] : g % a.N;
            const float scale = (Tex::kFormat == TG_TEX_FP8_E4M3) ? a.tex_scales[row] : 1.f;
            s_xyo[tr] = make_float4(xy.x, xy.y, a.opacities[g], scale);
            const float* m = a.ray_transforms + 9 * (int64_t)g;
            s_m0[tr] = make_float4(m[0], m[1], m[2], 0.f);
            s_m1[tr] = make_float4(m[3], m[4], m[5], 0.f);
            s_m2[tr] = make_float4(m[6], m[7], m[8], 0.f);
            const float* n = a.normals + 3 * (int64_t)g;
            s_nrm[tr] = make_float4(n[0], n[1], n[2], 0.f);
#pragma unroll
            for (int k = 0; k < D; ++k) s_col[tr * D + k] = a.colors[(int64_t)g * D + k];
            s_row[tr] = row;
        }
        __syncthreads();
        const int batch_size = min(bs, range_end - batch_start);
        for (int t = 0; t < batch_size; ++t) {
            if (__all_sync(wmask, done)) break;
            bool contributes = false;
            float alpha = 0.f;
            if (!done) {
                PairEval e;
                const int row = s_row[t];
                eval_pair<Tex>(e, px, py, s_xyo[t], s_m0[t], s_m1[t], s_m2[t], a.textures, (int64_t)row * tex_stride,
                               a.tex_rx, a.tex_ry, a.range_x, a.range_y, a.g_weight);
                if (e.valid) {
                    const float next_T = T * (1.f - e.alpha);
                    if (next_T <= 1e-4f) {
                        done = true;
                    } else {
                        const float vis = e.alpha * T;
                        const float* cp = s_col + t * D;
#pragma unroll
                        for (int k = 0; k < D; ++k) pix_out[k] += (cp[k] + (kTextured ? tex_color(e, k) : 0.f)) * vis;
                        const float4 nn = s_nrm[t];
                        nrm_out[0] += nn.x * vis;
                        nrm_out[1] += nn.y * vis;
                        nrm_out[2] += nn.z * vis;
                        const float depth = cp[D - 1];
                        distort += 2.f * (vis * depth * (1.f - T) - vis * accum_vis_depth);
                        accum_vis_depth += vis * depth;
                        if (T > 0.5f) {
                            median_depth = depth;
                            median_idx = batch_start + t;
                        }
                        cur_idx = batch_start + t;
                        T = next_T;
                        alpha = e.alpha;
                        contributes = e.alpha > a.contrib_threshold;
                    }
                }
            }
            const unsigned m = __ballot_sync(wmask, contributes);
            if (m) {
                const float s = warp_sum(contributes ? alpha : 0.f, wmask);
                if (lane == __ffs(wmask) - 1) {
                    const int row = s_row[t];
                    atomicAdd(a.contrib_sum + row, s);
                    atomicAdd(a.contrib_count + row, (float)__popc(m));
                }
            }
        }
    }
    if (inside) {
        a.out_alphas[pix] = 1.f - T;
#pragma unroll
        for (int k = 0; k < D; ++k)
            a.out_colors[pix * D + k] = a.backgrounds ? pix_out[k] + T * a.backgrounds[tc.c * D + k] : pix_out[k];
        a.out_normals[pix * 3] = nrm_out[0];
        a.out_normals[pix * 3 + 1] = nrm_out[1];
        a.out_normals[pix * 3 + 2] = nrm_out[2];
        a.last_ids[pix] = cur_idx;
        a.out_distort[pix] = distort;
        a.out_median[pix] = median_depth;
        a.median_ids[pix] = median_idx;
    }
}

template <int D, class Tex>
cudaError_t launch_fwd_t(const tg_raster_fwd_args& a, cudaStream_t s) {
    const int bs = a.tile_size * a.tile_size;
    const size_t smem = (size_t)bs * (5 * sizeof(float4) + D * sizeof(float) + sizeof(int));
    const int64_t blocks = (int64_t)a.C * a.tile_width * a.tile_height;
    if (blocks == 0) return cudaSuccess;
    raster_fwd_kernel<D, Tex><<<(unsigned)blocks, bs, smem, s>>>(a);
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
