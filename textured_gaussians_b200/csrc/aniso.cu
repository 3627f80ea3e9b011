// Row-prefix tables of the per-splat textures for the anisotropic_bilinear
// filter, and the adjoint that folds their gradient back into the texels,
// for sm_100a.
//
// The compositor integrates a convex footprint along its boundary (Green's
// theorem), which needs, for every texture row r, the integral of the
// row's linear interpolant from column 0 to each column u:
//   P_r[u] = sum_{k<u} (t(k,r) + t(k+1,r)) / 2,   P_r[0] = 0.
// One warp scans one row in chunks of 32 texels: the row is read once and the
// table written once, coalesced (HBM-bound: 16 B/texel written plus the
// storage format's bytes read).  The adjoint is the transposed scan: with
// S(j) = sum_{u>=j} dP[u],
//   dt(0) = S(1) / 2,   dt(j) = (S(j) + S(j+1)) / 2   (j >= 1),
// added into the texel gradients in one read-modify-write per texel.
#include "tg_common.cuh"

namespace tg {

__device__ __forceinline__ float4 add4(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }

__device__ __forceinline__ float4 shfl_up4(float4 v, int d) {
    return make_float4(__shfl_up_sync(0xffffffffu, v.x, d), __shfl_up_sync(0xffffffffu, v.y, d),
                       __shfl_up_sync(0xffffffffu, v.z, d), __shfl_up_sync(0xffffffffu, v.w, d));
}
__device__ __forceinline__ float4 shfl_down4(float4 v, int d) {
    return make_float4(__shfl_down_sync(0xffffffffu, v.x, d), __shfl_down_sync(0xffffffffu, v.y, d),
                       __shfl_down_sync(0xffffffffu, v.z, d), __shfl_down_sync(0xffffffffu, v.w, d));
}
__device__ __forceinline__ float4 shfl4(float4 v, int src) {
    return make_float4(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src),
                       __shfl_sync(0xffffffffu, v.z, src), __shfl_sync(0xffffffffu, v.w, src));
}

// Grid-stride over rows (G * ry of them), one warp each; 256 threads.
template <class Tex>
__global__ void __launch_bounds__(256) aniso_prefix_kernel(const void* __restrict__ textures,
                                                           const float* __restrict__ tex_scales, int64_t rows, int ry,
                                                           int rx, float4* __restrict__ prefix) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t r = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < rows; r += warps) {
        const float scale = Tex::kFormat == TG_TEX_FP8_E4M3 ? tex_scales[r / ry] : 1.f;
        const int64_t base = r * rx;
        float4 carry = make_float4(0.f, 0.f, 0.f, 0.f);
        if (lane == 0) prefix[base] = carry;
        for (int c = 0; c < rx - 1; c += 32) {
            const int k = c + lane;  // trapezoid k spans columns k, k + 1 and ends prefix entry k + 1
            float4 d = make_float4(0.f, 0.f, 0.f, 0.f);
            if (k < rx - 1) {
                const float4 a = Tex::load(textures, base + k, scale), b = Tex::load(textures, base + k + 1, scale);
                d = make_float4(0.5f * (a.x + b.x), 0.5f * (a.y + b.y), 0.5f * (a.z + b.z), 0.5f * (a.w + b.w));
            }
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {  // inclusive warp scan
                const float4 n = shfl_up4(d, o);
                if (lane >= o) d = add4(d, n);
            }
            d = add4(d, carry);
            if (k < rx - 1) prefix[base + k + 1] = d;
            carry = shfl4(d, 31);
        }
    }
}

// Adds the row-prefix gradient dP ([rows, rx] float4) into the texel
// gradient v_tex of the same layout; dP[.., 0] is ignored (P_r[0] is 0).
__global__ void __launch_bounds__(256) aniso_prefix_fold_kernel(const float4* __restrict__ dP, int64_t rows, int rx,
                                                                float4* __restrict__ v_tex) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t r = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < rows; r += warps) {
        const int64_t base = r * rx;
        float4 carry = make_float4(0.f, 0.f, 0.f, 0.f);  // S of the first column right of the chunk
        const int nchunks = (rx + 31) / 32;
        for (int ci = nchunks - 1; ci >= 0; --ci) {
            const int j = ci * 32 + lane;
            const float4 g = (j < rx && j > 0) ? dP[base + j] : make_float4(0.f, 0.f, 0.f, 0.f);
            float4 s = g;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {  // inclusive suffix scan within the chunk
                const float4 n = shfl_down4(s, o);
                if (lane + o < 32) s = add4(s, n);
            }
            s = add4(s, carry);  // S(j)
            const float4 s1 = make_float4(s.x - g.x, s.y - g.y, s.z - g.z, s.w - g.w);  // S(j + 1)
            if (j < rx) {
                float4 v = v_tex[base + j];
                if (j > 0) v = add4(v, make_float4(0.5f * (s.x + s1.x), 0.5f * (s.y + s1.y), 0.5f * (s.z + s1.z),
                                                   0.5f * (s.w + s1.w)));
                else v = add4(v, make_float4(0.5f * s1.x, 0.5f * s1.y, 0.5f * s1.z, 0.5f * s1.w));
                v_tex[base + j] = v;
            }
            carry = shfl4(s, 0);
        }
    }
}

static int grid_for(int64_t rows) {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t want = (rows + 7) / 8;  // 8 warps per CTA
    return (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)sms * 8));
}

cudaError_t launch_aniso_prefix(const void* textures, int tex_format, const float* tex_scales, int64_t G, int ry,
                                int rx, float* prefix, cudaStream_t s) {
    const int64_t rows = G * ry;
    if (rows == 0) return cudaSuccess;
    const int grid = grid_for(rows);
    float4* P = reinterpret_cast<float4*>(prefix);
    switch (tex_format) {
        case TG_TEX_F32: aniso_prefix_kernel<TexF32><<<grid, 256, 0, s>>>(textures, tex_scales, rows, ry, rx, P); break;
        case TG_TEX_BF16: aniso_prefix_kernel<TexBF16><<<grid, 256, 0, s>>>(textures, tex_scales, rows, ry, rx, P); break;
        case TG_TEX_F16: aniso_prefix_kernel<TexF16><<<grid, 256, 0, s>>>(textures, tex_scales, rows, ry, rx, P); break;
        case TG_TEX_FP8_E4M3: aniso_prefix_kernel<TexFP8><<<grid, 256, 0, s>>>(textures, tex_scales, rows, ry, rx, P); break;
        default: return cudaErrorInvalidValue;
    }
    note_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_aniso_prefix_fold(const float* v_prefix, int64_t G, int ry, int rx, float* v_textures,
                                     cudaStream_t s) {
    const int64_t rows = G * ry;
    if (rows == 0) return cudaSuccess;
    aniso_prefix_fold_kernel<<<grid_for(rows), 256, 0, s>>>(reinterpret_cast<const float4*>(v_prefix), rows, rx,
                                                             reinterpret_cast<float4*>(v_textures));
    note_launches(1);
    return cudaGetLastError();
}

}  // namespace tg
