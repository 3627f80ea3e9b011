// Textured / plain 2DGS compositor, adjoint, for sm_100a.
//
// One CTA per (camera, tile) work item, one thread per pixel (four for 32x32
// tiles), back-to-front in batches of `batch_depth` staged splats over the
// splats that can still matter to the tile (batches beyond every pixel's last
// contributor are skipped).  Transmittance is recovered from the stored final
// T and last-contributor index by division, as the reference does
// (rasterize_to_pixels_textured_gaussians_2dgs_bwd.cu:160, :456-457); nothing
// per splat is stored by the forward.
//
// Reductions, B200-first:
//  * per-splat gradients (colour, normal, ray transform, means2d, opacity,
//    |means2d|) are reduced across the warp by a reduce-scatter butterfly --
//    31 shuffles leave lane k holding the warp total of value k -- instead of
//    one 5-level shuffle tree per value; lanes then add into a per-batch
//    shared-memory accumulator, and the CTA flushes each splat's values with
//    one global atomic per value (8x fewer global atomics than per-warp);
//  * per-texel gradients are RGBA float4 vector atomics, one per bilinear tap
//    (4 per pixel-splat pair instead of the reference's up to 4*(D+1) scalar
//    atomics).
//
// Adjoint forms: TG_ADJ_REFERENCE follows ..._bwd.cu:438-627; TG_ADJ_BWD2 adds
// the reference's texture-UV term (..._bwd2.cu:612-676, du/ds = (R-1)/range);
// TG_ADJ_EXACT adds the UV term with the true du/ds = (R-1)/(2 range).
#include "raster_common.cuh"

namespace tg {

// reduce-scatter: on return vals[0] of lane l holds the warp sum of value l.
__device__ __forceinline__ void warp_reduce_scatter32(float (&vals)[32], unsigned mask) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1) {
        const bool upper = (lane & s) != 0;
        const bool have = ((mask >> (lane ^ s)) & 1u) != 0;
#pragma unroll
        for (int i = 0; i < s; ++i) {
            const float send = upper ? vals[i] : vals[i + s];
            const float keep = upper ? vals[i + s] : vals[i];
            const float recv = __shfl_xor_sync(mask, send, s);
            vals[i] = keep + (have ? recv : 0.f);
        }
    }
}

template <int D>
struct GradSlots {
    static constexpr int kRgb = 0;
    static constexpr int kNrm = D;
    static constexpr int kM = D + 3;
    static constexpr int kXY = D + 12;
    static constexpr int kOpac = D + 14;
    static constexpr int kAbs = D + 15;
    static constexpr int kCount = D + 17;
};

// Resident CTAs per SM the register allocation targets.
#ifndef TG_BWD_MIN_CTAS
#define TG_BWD_MIN_CTAS 2
#endif
// Register budget: TG_BWD_MIN_CTAS resident CTAs for one pixel per thread,
// one CTA of 256 threads for the four-pixel (32x32 tile) form.  The
// anisotropic_bilinear adjoint targets 3 CTAs (80 registers allocated): with its clips
// branch-free and its cell boundary sum out of line it spills ~1 KB there but
// runs 3.9 % faster than at 128, which was already 28 % faster than the
// unconstrained 245; 64 registers lose 17 % (1M splats, 4 views, measured).
#ifndef TG_BWD_MIN_CTAS_ANISO
#define TG_BWD_MIN_CTAS_ANISO 3
#endif
template <int PPT, class Filt>
struct BwdBounds {
    static constexpr int kMinCtas = PPT == 1 ? (Filt::kAniso ? TG_BWD_MIN_CTAS_ANISO : TG_BWD_MIN_CTAS) : 1;
};

// Per-pixel state of the back-to-front sweep.
template <int D>
struct PixelAdj {
    int64_t pix;
    float px, py;
    bool inside;
    float T_final, T, v_a, v_dist, v_med, bg_dot;
    float v_c[D], buf[D];
    float v_n[3], buf_n[3];
    int32_t bin_final, median_idx;
    float acc_d_buf, acc_d, acc_w_buf, acc_w, dist_buf;
    int32_t local;     // pixel index within the tile
    int32_t ck_batch;  // forward batch whose end transmittance T was last restarted from (-1: none)
    int32_t rec;       // anisotropic_bilinear: the forward's record of the next footprint integral (counting down)
};

// The forward's transmittance checkpoints of one tile (tg_raster_fwd_args.t_checkpoints): base is the tile's
// first row, rows of `stride` pixels, forward batches of bs splats from range_start rs.  base NULL: none.
struct TileCkpt {
    const float* base;
    int64_t stride;
    int32_t rs, bs;
};

// Adds one (pixel, splat) pair's gradient contributions to the lane's per-splat
// sums `vals` (slots of GradSlots<D>), issues the pair's texel-gradient atomics,
// and advances the pixel's back-to-front state.  Follows
// rasterize_to_pixels_textured_gaussians_2dgs_bwd.cu:438-627 (+ bwd2.cu:612-676).
template <int D, class Tex, class Filt = FiltBilinear>
__device__ __forceinline__ void accumulate_pair(const tg_raster_bwd_args& a, const PairOf<Filt>& e,
                                                PixelAdj<D>& P, const float4 xyo, const float4 nn, const float* cp,
                                                int32_t idx, float* vt, float uv_scale, float (&vals)[32],
                                                const TileCkpt& ck, float* vct = nullptr, int mip_clen = 0,
                                                float4* aniso_g = nullptr) {
    // aniso_g (anisotropic_bilinear): receives the texel-gradient factor of the pair (divided by the area), which
    // the warp scatters over the footprint together
    constexpr bool kTextured = Tex::kFormat != TG_TEX_NONE;
    using GS = GradSlots<D>;
    const tg_raster_fwd_args& f = a.f;
    const float opac = xyo.z;
    if (idx == P.median_idx) vals[GS::kRgb + D - 1] += P.v_med;
    if (ck.base != nullptr) {
        // first pair of a new forward batch (back to front): T restarts from the forward's exact value at the
        // batch's end -- no splat after this one in the batch contributed to this pixel, or it would have
        // been met first
        const int32_t fb = (idx - ck.rs) / ck.bs;
        if (fb != P.ck_batch) {
            P.ck_batch = fb;
            P.T = ck.base[(int64_t)fb * ck.stride + P.local];
        }
    }
    const float ra = 1.f / (1.f - e.alpha);
    P.T *= ra;
    const float T = P.T;
    const float fac = e.alpha * T;
    float texc[D];
#pragma unroll
    for (int k = 0; k < D; ++k) {
        vals[GS::kRgb + k] += fac * P.v_c[k];
        texc[k] = kTextured ? tex_color_adj(e, k) : 0.f;
    }
    float v_alpha = 0.f;
#pragma unroll
    for (int k = 0; k < D; ++k) v_alpha += ((texc[k] + cp[k]) * T - P.buf[k] * ra) * P.v_c[k];
    vals[GS::kNrm + 0] += fac * P.v_n[0];
    vals[GS::kNrm + 1] += fac * P.v_n[1];
    vals[GS::kNrm + 2] += fac * P.v_n[2];
    v_alpha += (nn.x * T - P.buf_n[0] * ra) * P.v_n[0];
    v_alpha += (nn.y * T - P.buf_n[1] * ra) * P.v_n[1];
    v_alpha += (nn.z * T - P.buf_n[2] * ra) * P.v_n[2];
    v_alpha += P.T_final * ra * P.v_a;
    if (f.backgrounds) v_alpha += -P.T_final * ra * P.bg_dot;
    {
        const float depth = cp[D - 1];
        const float dl_dw = 2.f * (2.f * (depth * P.acc_w_buf - P.acc_d_buf) + (P.acc_d - depth * P.acc_w));
        v_alpha += (dl_dw * T - P.dist_buf * ra) * P.v_dist;
        P.acc_d_buf -= fac * depth;
        P.acc_w_buf -= fac;
        P.dist_buf += dl_dw * fac;
        vals[GS::kRgb + D - 1] += 2.f * fac * (2.f - 2.f * T - P.acc_w + fac) * P.v_dist;
    }
    // d L / d s, from the Gaussian kernel (3D branch) and, for the UV-aware adjoints, from the
    // texture lookup; both go back through s = zeta.xy / zeta.z and zeta = h_u x h_v once
    float vsx = 0.f, vsy = 0.f;
    const bool unclamped = kTextured ? (opac * e.vis * e.asf <= 0.999f) : (opac * e.vis <= 0.999f);
    float tex_a_grad = 0.f;  // d L / d (texture alpha) / w_i
    if (unclamped) {
        const float v_G = kTextured ? opac * v_alpha * e.asf : opac * v_alpha;
        const float dG = kTextured ? -f.g_weight * e.kern : -e.vis;
        if (e.g3 <= e.g2) {
            vsx = v_G * dG * e.sx;
            vsy = v_G * dG * e.sy;
        } else {
            const float vx = v_G * (dG * kFilterInvSquare * e.dx);
            const float vy = v_G * (dG * kFilterInvSquare * e.dy);
            vals[GS::kXY] += vx;
            vals[GS::kXY + 1] += vy;
            vals[GS::kAbs] += fabsf(vx);
            vals[GS::kAbs + 1] += fabsf(vy);
        }
        vals[GS::kOpac] += kTextured ? e.vis * v_alpha * e.asf : e.vis * v_alpha;
        tex_a_grad = e.vis * opac * v_alpha;
    }
    if constexpr (Filt::kAniso) {
        if (e.tex_valid && vt != nullptr) {
            const float4 g = make_float4(D > 0 ? fac * P.v_c[0] : 0.f, D > 1 ? fac * P.v_c[D > 1 ? 1 : 0] : 0.f,
                                         D > 2 ? fac * P.v_c[D > 2 ? 2 : 0] : 0.f,
                                         (D > 3 ? fac * P.v_c[D > 3 ? 3 : 0] : 0.f) + tex_a_grad);
            const float ia = e.F.iarea;
            *aniso_g = make_float4(g.x * ia, g.y * ia, g.z * ia, g.w * ia);
        }
    } else if (kTextured && e.tex_valid && vt != nullptr) {
#pragma unroll
        for (int q = 0; q < Filt::kTaps; ++q) {
            float4 gq;
            gq.x = 0 < D ? fac * e.w[q] * P.v_c[0] : 0.f;
            gq.y = 1 < D ? fac * e.w[q] * P.v_c[1 < D ? 1 : 0] : 0.f;
            gq.z = 2 < D ? fac * e.w[q] * P.v_c[2 < D ? 2 : 0] : 0.f;
            gq.w = (3 < D ? fac * e.w[q] * P.v_c[3 < D ? 3 : 0] : 0.f) + e.w[q] * tex_a_grad;
            if (gq.x != 0.f || gq.y != 0.f || gq.z != 0.f || gq.w != 0.f) {
                if constexpr (Filt::kMip) {  // pyramid coordinate: coarse levels, or level 0 = the texture
                    const int mc = e.toff[q];
                    float* dst = mc < mip_clen ? vct + 4 * (int64_t)mc : vt + 4 * (int64_t)(mc - mip_clen);
                    atomicAdd(reinterpret_cast<float4*>(dst), gq);
                } else {
                    atomicAdd(reinterpret_cast<float4*>(vt + 4 * (int64_t)e.toff[q]), gq);
                }
            }
        }
    }
    if constexpr (Filt::kUV) if (kTextured && e.tex_valid && uv_scale != 0.f) {
        const float wu = e.w[1] + e.w[3], wv = e.w[2] + e.w[3];
        const float dbu[4] = {-(1.f - wv), 1.f - wv, -wv, wv};
        const float dbv[4] = {-(1.f - wu), -wu, 1.f - wu, wu};
        const float du = uv_scale * (float)(f.tex_rx - 1) / f.range_x;
        const float dv = uv_scale * (float)(f.tex_ry - 1) / f.range_y;
        float tsx = 0.f, tsy = 0.f;
#pragma unroll
        for (int k = 0; k < D && k < 4; ++k) {
            const float vt_k = fac * P.v_c[k];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float tv = f4get(e.tx[q], k);
                tsx += vt_k * dbu[q] * tv;
                tsy += vt_k * dbv[q] * tv;
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            tsx += tex_a_grad * dbu[q] * e.tx[q].w;
            tsy += tex_a_grad * dbv[q] * e.tx[q].w;
        }
        vsx += tsx * du;
        vsy += tsy * dv;
    }
    if (vsx != 0.f || vsy != 0.f) {
        const float iz = 1.f / e.z.z;
        const float a_ = vsx * iz, b_ = vsy * iz;
        const f3 vz = mk3(a_, b_, -(a_ * e.sx + b_ * e.sy));
        const f3 vhu = cross(e.hv, vz), vhv = cross(vz, e.hu);
        vals[GS::kM + 0] -= vhu.x; vals[GS::kM + 1] -= vhu.y; vals[GS::kM + 2] -= vhu.z;
        vals[GS::kM + 3] -= vhv.x; vals[GS::kM + 4] -= vhv.y; vals[GS::kM + 5] -= vhv.z;
        vals[GS::kM + 6] += P.px * vhu.x + P.py * vhv.x;
        vals[GS::kM + 7] += P.px * vhu.y + P.py * vhv.y;
        vals[GS::kM + 8] += P.px * vhu.z + P.py * vhv.z;
    }
#pragma unroll
    for (int k = 0; k < D; ++k) P.buf[k] += (texc[k] + cp[k]) * fac;
    P.buf_n[0] += nn.x * fac;
    P.buf_n[1] += nn.y * fac;
    P.buf_n[2] += nn.z * fac;
}

// One work item (tile) of the adjoint; every early return is uniform over the CTA.
template <int D, class Tex, int PPT, class Filt = FiltBilinear>
__device__ __forceinline__ void bwd_tile(const tg_raster_bwd_args& a, const float uv_scale, const int bs,
                                         const int64_t item) {
    using GS = GradSlots<D>;
    constexpr int NV = GS::kCount;
    const tg_raster_fwd_args& f = a.f;
    extern __shared__ float4 smem4[];
    const int nt = blockDim.x;  // tile_size^2 / PPT threads; bs = splats staged per batch
    float4* s_box = smem4;  // per-splat cull box (see cull_box)
    float4* s_xyo = s_box + bs;
    float4* s_m0 = s_xyo + bs;
    float4* s_m1 = s_m0 + bs;
    float4* s_m2 = s_m1 + bs;
    float4* s_nrm = s_m2 + bs;
    float* s_col = reinterpret_cast<float*>(s_nrm + bs);
    int* s_row = reinterpret_cast<int*>(s_col + bs * D);
    int* s_g = s_row + bs;
    float* s_grad = reinterpret_cast<float*>(s_g + bs);  // [bs][NV]
    // anisotropic_bilinear: the boundary integration's per-warp area (16-byte aligned: bs is a multiple of 32)
    float4* s_aniso = Filt::kAniso ? reinterpret_cast<float4*>(s_grad + bs * NV) + (threadIdx.x >> 5) * kAnisoWarpF4
                                   : nullptr;
    __shared__ int s_max_bin;

    const unsigned wmask = __activemask();
    const TileWork tc = tile_work(f, item);
    if (!tc.valid) return;  // uniform over the CTA
    const int tr = threadIdx.x, lane = tr & 31;
    if (f.masks != nullptr && !f.masks[tc.t]) return;

    const int ts = f.tile_size;
    const int32_t range_start = tc.range_start;
    const int32_t range_end = tc.range_end;

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
    for (int k = tr; k < bs * NV; k += nt) s_grad[k] = 0.f;
    if (tr == 0) s_max_bin = -1;

    PixelAdj<D> P[PPT];
    int32_t thread_bin = -1;
#pragma unroll
    for (int q = 0; q < PPT; ++q) {
        PixelAdj<D>& p = P[q];
        const int local = tr + q * nt;
        const int i = tc.ty * ts + local / ts;
        const int j = tc.tx * ts + local % ts;
        p.pix = pixel_index(tc, i, j);
        p.inside = p.pix >= 0;
        p.local = local;
        p.ck_batch = -1;
        p.rec = -1;
        p.px = (float)j + 0.5f;
        p.py = (float)i + 0.5f;
        p.T_final = 1.f; p.v_a = p.v_dist = p.v_med = p.bg_dot = 0.f;
        p.bin_final = -1; p.median_idx = -1;
        p.acc_d_buf = p.acc_d = p.acc_w_buf = p.acc_w = p.dist_buf = 0.f;
        p.v_n[0] = p.v_n[1] = p.v_n[2] = 0.f;
        p.buf_n[0] = p.buf_n[1] = p.buf_n[2] = 0.f;
#pragma unroll
        for (int k = 0; k < D; ++k) { p.v_c[k] = 0.f; p.buf[k] = 0.f; }
        if (p.inside) {
            const int64_t px_ = p.pix;
            const float alpha_out = a.render_alphas[px_];
            p.T_final = 1.f - alpha_out;
            p.bin_final = a.last_ids[px_];
            p.median_idx = a.median_ids[px_];
            if (Filt::kAniso && f.aniso_records != nullptr) p.rec = f.aniso_record_count[px_] - 1;
#pragma unroll
            for (int k = 0; k < D; ++k) p.v_c[k] = a.v_render_colors[px_ * D + k];
            p.v_a = a.v_render_alphas[px_];
            p.v_n[0] = a.v_render_normals[px_ * 3];
            p.v_n[1] = a.v_render_normals[px_ * 3 + 1];
            p.v_n[2] = a.v_render_normals[px_ * 3 + 2];
            p.v_dist = a.v_render_distort[px_];
            p.v_med = a.v_render_median[px_];
            p.acc_d_buf = a.render_colors[px_ * D + D - 1];
            p.acc_d = p.acc_d_buf;
            p.acc_w_buf = alpha_out;
            p.acc_w = alpha_out;
            if (f.backgrounds) {
#pragma unroll
                for (int k = 0; k < D; ++k) p.bg_dot += f.backgrounds[tc.c * D + k] * p.v_c[k];
            }
        }
        p.T = p.T_final;
        thread_bin = max(thread_bin, p.bin_final);
    }
    // last contributor over the warp (uniform) and over the CTA
    const int32_t warp_bin_final = __reduce_max_sync(wmask, thread_bin);
    __syncthreads();
    if (lane == __ffs(wmask) - 1) atomicMax(&s_max_bin, warp_bin_final);
    __syncthreads();
    const int32_t block_max_bin = s_max_bin;
    const int64_t tex_stride = (int64_t)f.tex_ry * f.tex_rx;
    const int mip_clen = Filt::kMip ? ((1 << (2 * f.mip_levels)) - 1) / 3 : 0;
    const int tile_px = nt * PPT;
    const TileCkpt ck{f.t_checkpoints != nullptr
                          ? f.t_checkpoints + ((int64_t)tc.t + range_start / bs) * (int64_t)tile_px : nullptr,
                      (int64_t)tile_px, range_start, bs};

    for (int32_t batch_end = range_end - 1; batch_end >= range_start; batch_end -= bs) {
        if (batch_end - (bs - 1) > block_max_bin) continue;  // every splat here is past all last contributors
        const int32_t batch_size = min(bs, batch_end + 1 - range_start);
        __syncthreads();  // previous batch fully flushed before restaging
        for (int slot = tr; slot < bs; slot += nt) {
            const int32_t idx_load = batch_end - slot;
            if (idx_load >= range_start) {
                const int32_t g = f.flatten_ids[idx_load];
                const float2 xy = reinterpret_cast<const float2*>(f.means2d)[g];
                const int32_t row = f.gaussian_ids ? (int32_t)f.gaussian_ids[g] : g % f.N;
                const float scale = (Tex::kFormat == TG_TEX_FP8_E4M3) ? f.tex_scales[row] : 1.f;
                s_xyo[slot] = make_float4(xy.x, xy.y, f.opacities[g], scale);
                const float* m = f.ray_transforms + 9 * (int64_t)g;
                s_m0[slot] = make_float4(m[0], m[1], m[2], 0.f);
                s_m1[slot] = make_float4(m[3], m[4], m[5], 0.f);
                s_m2[slot] = make_float4(m[6], m[7], m[8], 0.f);
                s_box[slot] = cull_box(s_xyo[slot], s_m0[slot], s_m1[slot], s_m2[slot], Tex::kFormat != TG_TEX_NONE,
                                       f.range_x, f.range_y, f.g_weight, !Filt::kAniso);
                const float* n = f.normals + 3 * (int64_t)g;
                s_nrm[slot] = make_float4(n[0], n[1], n[2], 0.f);
#pragma unroll
                for (int k = 0; k < D; ++k) s_col[slot * D + k] = f.colors[(int64_t)g * D + k];
                s_row[slot] = row;
                s_g[slot] = g;
            }
        }
        __syncthreads();
        for (int t = max(0, batch_end - warp_bin_final); t < batch_size; ++t) {
            const int32_t idx = batch_end - t;
            const float4 box = s_box[t];
            if (box.z < wx0 || box.x > wx1 || box.w < wy0 || box.y > wy1) continue;  // no pixel of this warp can be valid
            const float4 xyo = s_xyo[t], m0 = s_m0[t], m1 = s_m1[t], m2 = s_m2[t];
            const int row = s_row[t];
            const int64_t tex_base = (int64_t)row * tex_stride;
            const float4 nn = s_nrm[t];
            const float* cp = s_col + t * D;
            float* vt = a.v_textures != nullptr ? a.v_textures + 4 * tex_base : nullptr;
            float* vct = Filt::kMip && a.v_tex_coarse != nullptr ? a.v_tex_coarse + 4 * (int64_t)row * mip_clen
                                                                 : nullptr;
            float vals[32];
#pragma unroll
            for (int k = 0; k < 32; ++k) vals[k] = 0.f;
            bool any = false;
#pragma unroll
            for (int q = 0; q < PPT; ++q) {
                if constexpr (Filt::kAniso) {  // every lane takes part: the warp integrates footprints together
                    const bool act = P[q].inside && idx <= P[q].bin_final && in_box(box, P[q].px, P[q].py);
                    // the forward's integral of this pair's footprint, if it has one (it keeps the first
                    // aniso_record_cap of each pixel's, in order; this walks them back to front)
                    const float4* rec = act && P[q].rec >= 0 && P[q].rec < f.aniso_record_cap
                                            ? reinterpret_cast<const float4*>(f.aniso_records) +
                                                  P[q].pix * f.aniso_record_cap + P[q].rec
                                            : nullptr;
                    PairOf<Filt> e;
                    eval_aniso_coop<Tex, true>(e, act, P[q].px, P[q].py, xyo, m0, m1, m2, f.textures, tex_base, f.tex_rx,
                                         f.tex_ry, f.range_x, f.range_y, f.g_weight, wmask,
                                         f.aniso_prefix ? reinterpret_cast<const float4*>(f.aniso_prefix) + tex_base
                                                        : nullptr,
                                         s_aniso, rec);
                    if (e.tex_valid) --P[q].rec;  // this pair's footprint was integrated (or read): one record
                    const bool use = act && e.valid;
                    float4 g4 = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (use) {
                        any = true;
                        accumulate_pair<D, Tex, Filt>(a, e, P[q], xyo, nn, cp, idx, vt, uv_scale, vals, ck, vct,
                                                      mip_clen, &g4);
                    }
                    aniso_coop_scatter<true>(e.F, g4,
                                       use && e.tex_valid && vt != nullptr &&
                                           (g4.x != 0.f || g4.y != 0.f || g4.z != 0.f || g4.w != 0.f),
                                       vt, f.tex_rx, wmask,
                                       a.v_aniso_prefix != nullptr ? a.v_aniso_prefix + 4 * tex_base : nullptr,
                                       f.tex_ry, s_aniso);
                    continue;
                }
                if (!(P[q].inside && idx <= P[q].bin_final) || !in_box(box, P[q].px, P[q].py)) continue;
                PairOf<Filt> e;
                eval_pair<Tex, Filt>(e, P[q].px, P[q].py, xyo, m0, m1, m2, f.textures, tex_base, f.tex_rx,
                                     f.tex_ry, f.range_x, f.range_y, f.g_weight,
                                     MipSrc{f.tex_coarse, (int64_t)row * mip_clen, mip_clen, f.mip_levels});
                if (!e.valid) continue;
                any = true;
                accumulate_pair<D, Tex, Filt>(a, e, P[q], xyo, nn, cp, idx, vt, uv_scale, vals, ck, vct, mip_clen);
            }
            if (!__any_sync(wmask, any)) continue;
            warp_reduce_scatter32(vals, wmask);
            if (lane < NV && vals[0] != 0.f) atomicAdd(s_grad + t * NV + lane, vals[0]);
        }
        __syncthreads();
        // flush this batch's per-splat sums: one global atomic per (splat, value)
        for (int k = tr; k < batch_size * NV; k += nt) {
            const float v = s_grad[k];
            if (v == 0.f) continue;
            s_grad[k] = 0.f;
            const int t = k / NV, slot = k - t * NV;
            const int64_t g = s_g[t];
            float* dst;
            if (slot < GS::kNrm) dst = a.v_colors + g * D + slot;
            else if (slot < GS::kM) dst = a.v_normals + g * 3 + (slot - GS::kNrm);
            else if (slot < GS::kXY) dst = a.v_ray_transforms + g * 9 + (slot - GS::kM);
            else if (slot < GS::kOpac) dst = a.v_means2d + g * 2 + (slot - GS::kXY);
            else if (slot == GS::kOpac) dst = a.v_opacities + g;
            else dst = a.v_means2d_abs ? a.v_means2d_abs + g * 2 + (slot - GS::kAbs) : nullptr;
            if (dst) atomicAdd(dst, v);
        }
    }
}

// CTA per work item, or (work_queue != NULL) a persistent grid whose CTAs take
// items from the queue counter until none is left.
template <int D, class Tex, int PPT, bool kPersistent, class Filt = FiltBilinear>
__global__ void __launch_bounds__(256, BwdBounds<PPT, Filt>::kMinCtas) raster_bwd_kernel(const tg_raster_bwd_args a,
                                                                                   const float uv_scale,
                                                                                   const int bs,
                                                                                   const int64_t n_items) {
    if constexpr (!kPersistent) {
        bwd_tile<D, Tex, PPT, Filt>(a, uv_scale, bs, blockIdx.x);
        return;
    }
    else {
        __shared__ int64_t s_item;
        for (;;) {
            if (threadIdx.x == 0) s_item = (int64_t)atomicAdd(a.f.work_queue, 1u);
            __syncthreads();  // also: every thread is done with the previous item's shared memory
            const int64_t item = s_item;
            __syncthreads();  // s_item read by all before it is rewritten
            if (item >= n_items) return;
            bwd_tile<D, Tex, PPT, Filt>(a, uv_scale, bs, item);
        }
    }
}

// v_densify[e] = (v_M[e][2], v_M[e][5]) * M[e][8], once every contribution is in.
__global__ void densify_grad_kernel(const float* __restrict__ v_M, const float* __restrict__ M, int64_t n,
                                    float* __restrict__ v_densify) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const float depth = M[9 * e + 8];
    v_densify[2 * e] = v_M[9 * e + 2] * depth;
    v_densify[2 * e + 1] = v_M[9 * e + 5] * depth;
}

size_t bwd_smem_bytes(int D, int bs) {
    return (size_t)bs * (6 * sizeof(float4) + D * sizeof(float) + 2 * sizeof(int) + (D + 17) * sizeof(float));
}

// The mipmapped2 / anisotropic_bilinear kernels exist for FP32 / BF16 storage and 3 or 4 channels only.
template <int D, class Tex, class Filt>
constexpr bool filter_instance() {
    return (D == 3 || D == 4) && (Tex::kFormat == TG_TEX_F32 || Tex::kFormat == TG_TEX_BF16);
}
template <int D, class Tex, class Filt>
const void* filter_bwd_fn() {
    if constexpr (filter_instance<D, Tex, Filt>()) return (const void*)raster_bwd_kernel<D, Tex, 1, false, Filt>;
    else return nullptr;
}
template <int D, class Tex, class Filt>
void launch_filter_bwd(dim3 g, dim3 b, size_t smem, cudaStream_t s, const tg_raster_bwd_args& a, float uv_scale, int bs,
                       int64_t blocks) {
    if constexpr (filter_instance<D, Tex, Filt>())
        raster_bwd_kernel<D, Tex, 1, false, Filt><<<g, b, smem, s>>>(a, uv_scale, bs, blocks);
}

// The bilinear adjoint instances: 32x32 tiles (four pixels per thread) or not, persistent or not.
template <int D, class Tex, class F>
const void* bilinear_bwd_fn(bool four, bool pers) {
    if constexpr (F::kUV && Tex::kFormat == TG_TEX_NONE) return nullptr;  // (never asked for)
    else
        return four ? (pers ? (const void*)raster_bwd_kernel<D, Tex, 4, true, F>
                            : (const void*)raster_bwd_kernel<D, Tex, 4, false, F>)
                    : (pers ? (const void*)raster_bwd_kernel<D, Tex, 1, true, F>
                            : (const void*)raster_bwd_kernel<D, Tex, 1, false, F>);
}
template <int D, class Tex, class F>
void launch_bilinear_bwd(bool four, bool pers, dim3 g, dim3 b, size_t smem, cudaStream_t s,
                         const tg_raster_bwd_args& a, float uv_scale, int bs, int64_t blocks) {
    if constexpr (!(F::kUV && Tex::kFormat == TG_TEX_NONE)) {
        if (four && pers) raster_bwd_kernel<D, Tex, 4, true, F><<<g, b, smem, s>>>(a, uv_scale, bs, blocks);
        else if (four) raster_bwd_kernel<D, Tex, 4, false, F><<<g, b, smem, s>>>(a, uv_scale, bs, blocks);
        else if (pers) raster_bwd_kernel<D, Tex, 1, true, F><<<g, b, smem, s>>>(a, uv_scale, bs, blocks);
        else raster_bwd_kernel<D, Tex, 1, false, F><<<g, b, smem, s>>>(a, uv_scale, bs, blocks);
    }
}

template <int D, class Tex>
cudaError_t launch_bwd_t(const tg_raster_bwd_args& a, cudaStream_t s) {
    const tg_raster_fwd_args& f = a.f;
    const int tile_px = f.tile_size * f.tile_size;
    const int bs = f.batch_depth > 0 ? f.batch_depth : tile_px;
    size_t smem = bwd_smem_bytes(D, bs);
    const int64_t blocks = f.views ? f.n_tiles : (int64_t)f.C * f.tile_width * f.tile_height;
    const float uv_scale = a.adjoint == TG_ADJ_BWD2 ? 1.f : (a.adjoint == TG_ADJ_EXACT ? 0.5f : 0.f);
    // mipmapped2 / anisotropic_bilinear: one pixel per thread, one CTA per tile
    const bool mip = f.mip_levels > 0, aniso = f.filter == TG_FILTER_ANISO_BILINEAR;
    if (aniso) smem += (size_t)(tile_px / 32) * kAnisoWarpF4 * 16;  // the boundary integration's per-warp area
    if ((mip || aniso) && !filter_instance<D, Tex, FiltMip2>()) return cudaErrorInvalidValue;
    const bool four = tile_px > 256;  // 32x32 tiles: four pixels per thread, 256 threads
    const bool pers = f.work_queue != nullptr;
    // the bwd2 / exact adjoints (uv_scale != 0) take the instances that carry the UV term
    const bool uv = Tex::kFormat != TG_TEX_NONE && uv_scale != 0.f;
    const void* fn = mip ? filter_bwd_fn<D, Tex, FiltMip2>()
                   : aniso ? filter_bwd_fn<D, Tex, FiltAniso>()
                   : uv ? bilinear_bwd_fn<D, Tex, FiltBilinearUV>(four, pers)
                        : bilinear_bwd_fn<D, Tex, FiltBilinear>(four, pers);
    const int threads = four ? tile_px / 4 : tile_px;
    cudaError_t err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    if (blocks > 0 && f.n_isects > 0) {
        int64_t grid = blocks;
        if (pers) {
            if ((err = cudaMemsetAsync(f.work_queue, 0, sizeof(uint32_t), s)) != cudaSuccess) return err;
            if ((err = persistent_grid(fn, threads, smem, blocks, grid)) != cudaSuccess) return err;
        }
        const dim3 g((unsigned)grid), b((unsigned)threads);
        if (mip) launch_filter_bwd<D, Tex, FiltMip2>(g, b, smem, s, a, uv_scale, bs, blocks);
        else if (aniso) launch_filter_bwd<D, Tex, FiltAniso>(g, b, smem, s, a, uv_scale, bs, blocks);
        else if (uv) launch_bilinear_bwd<D, Tex, FiltBilinearUV>(four, pers, g, b, smem, s, a, uv_scale, bs, blocks);
        else launch_bilinear_bwd<D, Tex, FiltBilinear>(four, pers, g, b, smem, s, a, uv_scale, bs, blocks);
        note_launches(1);
    }
    if ((err = cudaGetLastError()) != cudaSuccess) return err;
    if (a.n_elems > 0)
        densify_grad_kernel<<<(unsigned)((a.n_elems + 255) / 256), 256, 0, s>>>(a.v_ray_transforms,
                                                                               f.ray_transforms, a.n_elems,
                                                                               a.v_densify);
    if (a.n_elems > 0) note_launches(1);
    return cudaGetLastError();
}

template <class Tex>
cudaError_t launch_bwd_d(const tg_raster_bwd_args& a, cudaStream_t s) {
    switch (a.f.D) {
        case 1: return launch_bwd_t<1, Tex>(a, s);
        case 2: return launch_bwd_t<2, Tex>(a, s);
        case 3: return launch_bwd_t<3, Tex>(a, s);
        case 4: return launch_bwd_t<4, Tex>(a, s);
        case 5: return launch_bwd_t<5, Tex>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

template <class Tex>
cudaError_t launch_bwd_d34(const tg_raster_bwd_args& a, cudaStream_t s) {
    switch (a.f.D) {
        case 3: return launch_bwd_t<3, Tex>(a, s);
        case 4: return launch_bwd_t<4, Tex>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_raster_bwd(const tg_raster_bwd_args& a, cudaStream_t s) {
    switch (a.f.tex_format) {
        case TG_TEX_NONE: return launch_bwd_d<TexNone>(a, s);
        case TG_TEX_F32: return launch_bwd_d<TexF32>(a, s);
        case TG_TEX_BF16: return launch_bwd_d34<TexBF16>(a, s);
        case TG_TEX_F16: return launch_bwd_d34<TexF16>(a, s);
        case TG_TEX_FP8_E4M3: return launch_bwd_d34<TexFP8>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace tg
