// Per-(pixel, splat) evaluation shared by the compositor forward and adjoint.
//
// Both kernels call eval_pair with the same inputs, so a splat's alpha -- and
// therefore the set of splats that contributed to a pixel -- is recomputed
// bit-identically in the backward.  The arithmetic follows
// rasterize_to_pixels_textured_gaussians_2dgs_fwd.cu:283-347 (textured) and
// rasterize_to_pixels_2dgs_fwd.cu:281-310 (plain) of the reference, and the
// bilinear addressing filters/bilinear.cuh:16-64.
#pragma once
#include "tg_common.cuh"

namespace tg {

constexpr float kFilterInvSquare = 2.0f;

struct PairEval {
    f3 hu, hv, z;
    float sx, sy, dx, dy;
    float g3, g2, kern, vis, alpha, asf;
    float w[4];
    float4 tx[4];  // the four RGBA taps
    int toff[4];   // texel index of each tap inside the splat's texture
    bool valid, tex_valid;
};

// Splat data staged in shared memory: xyo = (x, y, opacity, texture scale),
// m0/m1/m2 = rows of the ray transform (w unused).
template <class Tex>
__device__ __forceinline__ void eval_pair(PairEval& e, float px, float py, const float4 xyo, const float4 m0,
                                          const float4 m1, const float4 m2, const void* textures, int64_t tex_base,
                                          int rx, int ry, float range_x, float range_y, float g_weight) {
    constexpr bool kTextured = Tex::kFormat != TG_TEX_NONE;
    e.hu = mk3(px * m2.x - m0.x, px * m2.y - m0.y, px * m2.z - m0.z);
    e.hv = mk3(py * m2.x - m1.x, py * m2.y - m1.y, py * m2.z - m1.z);
    e.z = cross(e.hu, e.hv);
    e.valid = true;
    e.tex_valid = false;
    e.asf = 1.f;
    if (e.z.z == 0.f) {
        e.valid = false;
        return;
    }
    e.sx = e.z.x / e.z.z;
    e.sy = e.z.y / e.z.z;
    if (kTextured) {
        if (!(e.sx < -range_x || e.sx > range_x || e.sy < -range_y || e.sy > range_y)) {
            float u = (e.sx + range_x) / (range_x * 2.f) * (float)(rx - 1);
            float v = (e.sy + range_y) / (range_y * 2.f) * (float)(ry - 1);
            if (u < 0.f) u = 0.f; else if (u > (float)(rx - 1)) u = (float)(rx - 1);
            if (v < 0.f) v = 0.f; else if (v > (float)(ry - 1)) v = (float)(ry - 1);
            const int ul = (int)floorf(u), vl = (int)floorf(v), uh = (int)ceilf(u), vh = (int)ceilf(v);
            const float wu = u - (float)ul, wv = v - (float)vl;
            e.w[0] = (1.f - wu) * (1.f - wv);
            e.w[1] = wu * (1.f - wv);
            e.w[2] = (1.f - wu) * wv;
            e.w[3] = wu * wv;
            e.toff[0] = vl * rx + ul;
            e.toff[1] = vl * rx + uh;
            e.toff[2] = vh * rx + ul;
            e.toff[3] = vh * rx + uh;
#pragma unroll
            for (int i = 0; i < 4; ++i) e.tx[i] = Tex::load(textures, tex_base + e.toff[i], xyo.w);
            float asf = 0.f;
#pragma unroll
            for (int i = 0; i < 4; ++i) asf += e.w[i] * e.tx[i].w;
            e.asf = asf;
            e.tex_valid = true;
        }
    }
    e.g3 = e.sx * e.sx + e.sy * e.sy;
    e.dx = xyo.x - px;
    e.dy = xyo.y - py;
    e.g2 = kFilterInvSquare * (e.dx * e.dx + e.dy * e.dy);
    const float sigma = 0.5f * fminf(e.g3, e.g2);
    e.kern = __expf(-sigma);
    if (kTextured) {
        e.vis = 0.998f - g_weight + g_weight * e.kern;
        e.alpha = fminf(0.999f, xyo.z * e.vis * e.asf);
    } else {
        e.vis = e.kern;
        e.alpha = fminf(0.999f, xyo.z * e.vis);
    }
    if (sigma < 0.f || e.alpha < 1.f / 255.f) e.valid = false;
}

// Texture contribution to colour channel k (channels >= 4 have none).
__device__ __forceinline__ float tex_color(const PairEval& e, int k) {
    if (k >= 4 || !e.tex_valid) return 0.f;
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < 4; ++i) s += e.w[i] * f4get(e.tx[i], k);
    return s;
}

// Sum over the lanes in `mask`; lanes outside it contribute zero.  The
// butterfly reads lane^o, which exists whenever the mask is a prefix of
// lanes whose count is a power of two, or the full warp.
__device__ __forceinline__ float warp_sum(float v, unsigned mask) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float u = __shfl_xor_sync(mask, v, o);
        if (((threadIdx.x & 31) ^ o) < 32 && (mask >> ((threadIdx.x & 31) ^ o)) & 1u) v += u;
    }
    return v;
}

struct TileCoord {
    int c, ty, tx, tile;
};
__device__ __forceinline__ TileCoord tile_of_block(int tile_w, int tile_h) {
    TileCoord t;
    const int per_cam = tile_w * tile_h;
    t.c = blockIdx.x / per_cam;
    t.tile = blockIdx.x - t.c * per_cam;
    t.ty = t.tile / tile_w;
    t.tx = t.tile - t.ty * tile_w;
    return t;
}

}  // namespace tg
