// Coarse mip levels of the per-Gaussian textures (for the mipmapped2 filter)
// and their adjoint, for sm_100a.
//
// Follows generate_mipmap_fwd.cu / generate_mipmap_bwd.cu of the reference:
// level t (side 2^(L-t)) of texture g sits at texel (4^(L-t) - 1) / 3 of the
// pyramid, coarsest first; a texel is ((a + b) + c + d) / 4 of its four
// children in the reference's order, and the adjoint adds a quarter of each
// parent's (complete) gradient to each child, coarsest level first.
//
// B200 form: level 0 is never copied into the pyramid (the compositor reads it
// from the texture storage), and one CTA builds levels 1..5 of a 32 x 32 block
// of its input level in one pass -- the input read once, coalesced, the
// intermediate levels kept in shared memory -- so a 32 x 32 texture's whole
// pyramid is one read of the texture and one write of its coarse levels.
// Levels above 5 (textures wider than 32) repeat the pass on level 5.  The
// adjoint mirrors it: one CTA per block loads the block's coarse gradients,
// folds them down in shared memory and adds the result into level 0 in one
// read-modify-write, so the coarse gradients are read once and never written.
#include "tg_common.cuh"

namespace tg {

__host__ __device__ __forceinline__ int64_t level_base(int L, int t) { return (((int64_t)1 << (2 * (L - t))) - 1) / 3; }

constexpr int kBlockSide = 32;   // input texels per block side
constexpr int kBlockLevels = 5;  // levels one pass builds: 32 -> 16 -> 8 -> 4 -> 2 -> 1

__device__ __forceinline__ float4 quad_mean(float4 a, float4 b, float4 c, float4 d) {
    return make_float4((a.x + b.x + c.x + d.x) * 0.25f, (a.y + b.y + c.y + d.y) * 0.25f,
                       (a.z + b.z + c.z + d.z) * 0.25f, (a.w + b.w + c.w + d.w) * 0.25f);
}

// Levels t0 + 1 .. t0 + nl of every texture from level t0 (the texture itself
// when t0 == 0).  Grid: G x (blocks per texture); block side S = min(32,
// side of level t0); 256 threads.
__global__ void __launch_bounds__(256) mip_build_kernel(const float4* __restrict__ tex, float4* __restrict__ coarse,
                                                        int L, int t0, int nl) {
    __shared__ float4 s_lvl[2][256];  // the two most recent levels (level t0+1 has at most 16 x 16 texels)
    const int64_t g = blockIdx.x;
    const int side_in = 1 << (L - t0);
    const int S = min(kBlockSide, side_in);
    const int nb = side_in / S;  // blocks per row
    const int bx = (int)(blockIdx.y % nb), by = (int)(blockIdx.y / nb);
    const int64_t clen = level_base(L, 0);
    const float4* src = t0 == 0 ? tex + g * (int64_t)side_in * side_in : coarse + g * clen + level_base(L, t0);
    float4* dst = coarse + g * clen;
    // level t0 + 1: each thread reduces a 2 x 2 of the input
    int h = S >> 1;  // output side within the block
    int buf = 0;
    for (int i = threadIdx.x; i < h * h; i += blockDim.x) {
        const int v = i / h, u = i - v * h;
        const int gx = bx * S + 2 * u, gy = by * S + 2 * v;
        const float4 a = src[(int64_t)gy * side_in + gx], b = src[(int64_t)gy * side_in + gx + 1];
        const float4 c = src[(int64_t)(gy + 1) * side_in + gx], d = src[(int64_t)(gy + 1) * side_in + gx + 1];
        const float4 m = quad_mean(a, b, c, d);
        s_lvl[buf][i] = m;
        const int side_out = side_in >> 1;
        dst[level_base(L, t0 + 1) + (int64_t)(by * h + v) * side_out + bx * h + u] = m;
    }
    for (int k = 2; k <= nl; ++k) {
        __syncthreads();
        const int hi = h;  // input side within the block
        h >>= 1;
        const int side_out = side_in >> k;
        for (int i = threadIdx.x; i < h * h; i += blockDim.x) {
            const int v = i / h, u = i - v * h;
            const float4* p = s_lvl[buf];
            const float4 m = quad_mean(p[(2 * v) * hi + 2 * u], p[(2 * v) * hi + 2 * u + 1], p[(2 * v + 1) * hi + 2 * u],
                                       p[(2 * v + 1) * hi + 2 * u + 1]);
            s_lvl[buf ^ 1][i] = m;
            dst[level_base(L, t0 + k) + (int64_t)(by * h + v) * side_out + bx * h + u] = m;
        }
        buf ^= 1;
    }
}

// Adjoint of one pass: the gradients of levels t0+1 .. t0+nl of a block
// (complete: every coarser level already folded into level t0+nl) are folded
// down to level t0, whose gradient (the texture's when t0 == 0) receives them
// in one read-modify-write.  Coarse gradients of the block are only read.
__global__ void __launch_bounds__(256) mip_fold_kernel(const float4* __restrict__ v_coarse, float4* __restrict__ v_tex,
                                                       float4* __restrict__ v_coarse_rw, int L, int t0, int nl) {
    __shared__ float4 s_g[341];  // levels t0+1 .. t0+5 of one block: 256 + 64 + 16 + 4 + 1
    const int64_t g = blockIdx.x;
    const int side_in = 1 << (L - t0);
    const int S = min(kBlockSide, side_in);
    const int nb = side_in / S;
    const int bx = (int)(blockIdx.y % nb), by = (int)(blockIdx.y / nb);
    const int64_t clen = level_base(L, 0);
    const float4* vc = v_coarse + g * clen;
    // shared layout: level t0+k of the block at offset off(k), side S >> k
    auto off = [S](int k) {
        int o = 0;
        for (int j = 1; j < k; ++j) o += (S >> j) * (S >> j);
        return o;
    };
    for (int k = 1; k <= nl; ++k) {
        const int h = S >> k, side_out = side_in >> k;
        for (int i = threadIdx.x; i < h * h; i += blockDim.x) {
            const int v = i / h, u = i - v * h;
            s_g[off(k) + i] = vc[level_base(L, t0 + k) + (int64_t)(by * h + v) * side_out + bx * h + u];
        }
    }
    // fold the coarsest levels down, one level per step (a child gets exactly one addition)
    for (int k = nl; k >= 2; --k) {
        __syncthreads();
        const int hc = S >> (k - 1);  // child side
        for (int i = threadIdx.x; i < hc * hc; i += blockDim.x) {
            const int v = i / hc, u = i - v * hc;
            const float4 p = s_g[off(k) + (v >> 1) * (hc >> 1) + (u >> 1)];
            float4& q = s_g[off(k - 1) + i];
            q.x += p.x * 0.25f;
            q.y += p.y * 0.25f;
            q.z += p.z * 0.25f;
            q.w += p.w * 0.25f;
        }
    }
    __syncthreads();
    // level t0: the texture gradient (t0 == 0) or the coarse level t0, read-modify-write
    // (all of a thread's loads are issued before its stores: S * S <= 4 * 256 texels per block)
    float4* out = t0 == 0 ? v_tex + g * (int64_t)side_in * side_in : v_coarse_rw + g * clen + level_base(L, t0);
    const int h1 = S >> 1;
    float4 q[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int i = threadIdx.x + j * 256;
        if (i < S * S) q[j] = out[(int64_t)(by * S + i / S) * side_in + bx * S + i % S];
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int i = threadIdx.x + j * 256;
        if (i >= S * S) continue;
        const int v = i / S, u = i - v * S;
        const float4 p = s_g[(v >> 1) * h1 + (u >> 1)];
        q[j].x += p.x * 0.25f;
        q[j].y += p.y * 0.25f;
        q[j].z += p.z * 0.25f;
        q[j].w += p.w * 0.25f;
        out[(int64_t)(by * S + v) * side_in + bx * S + u] = q[j];
    }
}

cudaError_t launch_generate_mipmap(const float* textures, float* coarse, int64_t G, int L, cudaStream_t s) {
    for (int t0 = 0; t0 < L; t0 += kBlockLevels) {
        const int nl = min(kBlockLevels, L - t0);
        const int64_t side_in = (int64_t)1 << (L - t0);
        const int64_t S = std::min<int64_t>(kBlockSide, side_in);
        const int64_t blocks = (side_in / S) * (side_in / S);
        if (G > 0x7fffffff || blocks > 65535) return cudaErrorInvalidValue;
        mip_build_kernel<<<dim3((unsigned)G, (unsigned)blocks), 256, 0, s>>>(
            reinterpret_cast<const float4*>(textures), reinterpret_cast<float4*>(coarse), L, t0, nl);
        note_launches(1);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_generate_mipmap_bwd(float* v_coarse, float* v_textures, int64_t G, int L, cudaStream_t s) {
    // passes from the coarsest down: pass t0 folds levels t0+1..t0+nl into level t0
    int t0 = ((L - 1) / kBlockLevels) * kBlockLevels;
    for (; t0 >= 0; t0 -= kBlockLevels) {
        const int nl = min(kBlockLevels, L - t0);
        const int64_t side_in = (int64_t)1 << (L - t0);
        const int64_t S = std::min<int64_t>(kBlockSide, side_in);
        const int64_t blocks = (side_in / S) * (side_in / S);
        if (G > 0x7fffffff || blocks > 65535) return cudaErrorInvalidValue;
        mip_fold_kernel<<<dim3((unsigned)G, (unsigned)blocks), 256, 0, s>>>(
            reinterpret_cast<const float4*>(v_coarse), reinterpret_cast<float4*>(v_textures),
            reinterpret_cast<float4*>(v_coarse), L, t0, nl);
        note_launches(1);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace tg
