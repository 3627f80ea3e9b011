// The gradient consumers after the backward: densification statistics and the
// selective Adam step, for sm_100a.
//
// Selective Adam follows textured_gaussians/cuda/csrc/adam.cu:17-45 of the
// reference (rows whose visibility flag is off are left untouched; no bias
// correction).  B200 form: one pass over float4 vectors of each visible row
// (a 32x32 RGBA texture row is 1024 float4) that also writes the updated
// parameters into a BF16 or FP16 shadow copy -- the storage the compositor
// samples -- so the low-precision textures never need a separate conversion
// pass after the step.
//
// Densification statistics follow DefaultStrategy._update_state
// (textured_gaussians/strategy/default.py:213-261): per visible (camera,
// Gaussian) entry the norm of its 2D-mean gradient scaled to [-1, 1] screen
// units (x by width/2 * C, y by height/2 * C) is added to grad2d[g], count[g]
// is incremented, and max_radii[g] keeps the largest radius / max(W, H).  The
// dense layout runs one thread per Gaussian looping over cameras (no
// atomics); the packed layout one thread per entry with atomics.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "tg_common.cuh"

namespace tg {

__device__ __forceinline__ float adam_one(float& p, float g, float& m, float& v, float lr, float b1, float b2,
                                          float eps) {
    m = b1 * m + (1.0f - b1) * g;
    v = b2 * v + (1.0f - b2) * g * g;
    p += -lr * m / (sqrtf(v) + eps);
    return p;
}

template <int kShadow>
__device__ __forceinline__ void store_shadow4(void* shadow, int64_t i4, float4 p) {
    if constexpr (kShadow == TG_TEX_BF16) {
        __nv_bfloat162* d = reinterpret_cast<__nv_bfloat162*>(shadow) + 2 * i4;
        d[0] = __floats2bfloat162_rn(p.x, p.y);
        d[1] = __floats2bfloat162_rn(p.z, p.w);
    } else if constexpr (kShadow == TG_TEX_F16) {
        __half2* d = reinterpret_cast<__half2*>(shadow) + 2 * i4;
        d[0] = __floats2half2_rn(p.x, p.y);
        d[1] = __floats2half2_rn(p.z, p.w);
    }
}

template <int kShadow>
__device__ __forceinline__ void store_shadow1(void* shadow, int64_t i, float p) {
    if constexpr (kShadow == TG_TEX_BF16) reinterpret_cast<__nv_bfloat16*>(shadow)[i] = __float2bfloat16_rn(p);
    else if constexpr (kShadow == TG_TEX_F16) reinterpret_cast<__half*>(shadow)[i] = __float2half_rn(p);
}

// Rows of M = 4*M4 floats: thread per float4, grid-stride; a row's visibility
// flag is read once per float4 (rows of textures are 1024 float4 long, so a
// warp's threads share one row and skip it together).
template <int kShadow>
__global__ void __launch_bounds__(256) selective_adam4_kernel(float4* __restrict__ param, const float4* __restrict__ grad,
                                                              float4* __restrict__ m, float4* __restrict__ v,
                                                              const uint8_t* __restrict__ vis, float lr, float b1,
                                                              float b2, float eps, int64_t N, int64_t M4,
                                                              void* __restrict__ shadow) {
    const int64_t total = N * M4;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (!vis[i / M4]) continue;
        float4 p = param[i], mm = m[i], vv = v[i];
        const float4 g = grad[i];
        adam_one(p.x, g.x, mm.x, vv.x, lr, b1, b2, eps);
        adam_one(p.y, g.y, mm.y, vv.y, lr, b1, b2, eps);
        adam_one(p.z, g.z, mm.z, vv.z, lr, b1, b2, eps);
        adam_one(p.w, g.w, mm.w, vv.w, lr, b1, b2, eps);
        param[i] = p;
        m[i] = mm;
        v[i] = vv;
        store_shadow4<kShadow>(shadow, i, p);
    }
}

template <int kShadow>
__global__ void __launch_bounds__(256) selective_adam1_kernel(float* __restrict__ param, const float* __restrict__ grad,
                                                              float* __restrict__ m, float* __restrict__ v,
                                                              const uint8_t* __restrict__ vis, float lr, float b1,
                                                              float b2, float eps, int64_t N, int64_t M,
                                                              void* __restrict__ shadow) {
    const int64_t total = N * M;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (!vis[i / M]) continue;
        float p = param[i], mm = m[i], vv = v[i];
        adam_one(p, grad[i], mm, vv, lr, b1, b2, eps);
        param[i] = p;
        m[i] = mm;
        v[i] = vv;
        store_shadow1<kShadow>(shadow, i, p);
    }
}

template <int kShadow>
cudaError_t launch_adam_t(float* param, const float* grad, float* m, float* v, const uint8_t* vis, float lr, float b1,
                          float b2, float eps, int64_t N, int64_t M, void* shadow, cudaStream_t s) {
    const bool vec = (M % 4) == 0 && ((uintptr_t)param | (uintptr_t)grad | (uintptr_t)m | (uintptr_t)v) % 16 == 0 &&
                     (kShadow == TG_TEX_NONE || (uintptr_t)shadow % 8 == 0);
    const int64_t work = vec ? N * (M / 4) : N * M;
    const unsigned grid = (unsigned)std::min<int64_t>((work + 255) / 256, (int64_t)kNumSMs * 32);
    if (vec)
        selective_adam4_kernel<kShadow><<<grid, 256, 0, s>>>(
            reinterpret_cast<float4*>(param), reinterpret_cast<const float4*>(grad), reinterpret_cast<float4*>(m),
            reinterpret_cast<float4*>(v), vis, lr, b1, b2, eps, N, M / 4, shadow);
    else
        selective_adam1_kernel<kShadow><<<grid, 256, 0, s>>>(param, grad, m, v, vis, lr, b1, b2, eps, N, M, shadow);
    note_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_selective_adam(float* param, const float* grad, float* m, float* v, const uint8_t* vis, float lr,
                                  float b1, float b2, float eps, int64_t N, int64_t M, int shadow_format, void* shadow,
                                  cudaStream_t s) {
    if (N * M == 0) return cudaSuccess;
    switch (shadow_format) {
        case TG_TEX_NONE: return launch_adam_t<TG_TEX_NONE>(param, grad, m, v, vis, lr, b1, b2, eps, N, M, nullptr, s);
        case TG_TEX_BF16: return launch_adam_t<TG_TEX_BF16>(param, grad, m, v, vis, lr, b1, b2, eps, N, M, shadow, s);
        case TG_TEX_F16: return launch_adam_t<TG_TEX_F16>(param, grad, m, v, vis, lr, b1, b2, eps, N, M, shadow, s);
        default: return cudaErrorInvalidValue;
    }
}

// ------------------------------------------------------------------ densification statistics
__device__ __forceinline__ float screen_grad_norm(const float* g2, int64_t e, float sx, float sy) {
    const float gx = g2[2 * e] * sx, gy = g2[2 * e + 1] * sy;
    return sqrtf(gx * gx + gy * gy);
}

// radius / max(W, H) as an IEEE-rounded division, as the reference's torch division computes it
__device__ __forceinline__ float radius_fraction(int32_t r, float extent) { return __fdiv_rn((float)r, extent); }

__global__ void __launch_bounds__(256) densify_stats_dense_kernel(tg_densify_stats_args a, float sx, float sy,
                                                                  float extent) {
    const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= a.N) return;
    float sum = 0.f, cnt = 0.f, rmax = -INFINITY;
    for (int c = 0; c < a.C; ++c) {
        const int64_t e = (int64_t)c * a.N + n;
        const int32_t r = a.radii[e];
        if (r <= 0) continue;
        sum += screen_grad_norm(a.grads2d, e, sx, sy);
        cnt += 1.f;
        rmax = fmaxf(rmax, radius_fraction(r, extent));
    }
    if (cnt == 0.f) return;
    a.grad2d[n] += sum;
    a.count[n] += cnt;
    if (a.max_radii) a.max_radii[n] = fmaxf(a.max_radii[n], rmax);
}

__global__ void __launch_bounds__(256) densify_stats_packed_kernel(tg_densify_stats_args a, float sx, float sy,
                                                                   float extent) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= a.n_elems) return;
    const int32_t r = a.radii[e];
    const int64_t g = a.gaussian_ids[e];
    if (r <= 0 || g < 0 || g >= a.N) return;
    atomicAdd(a.grad2d + g, screen_grad_norm(a.grads2d, e, sx, sy));
    atomicAdd(a.count + g, 1.f);
    // non-negative floats order as their bit patterns do
    if (a.max_radii) atomicMax(reinterpret_cast<int*>(a.max_radii + g), __float_as_int(radius_fraction(r, extent)));
}

cudaError_t launch_densify_stats(const tg_densify_stats_args& a, cudaStream_t s) {
    const float sx = 0.5f * (float)a.width * (float)a.C, sy = 0.5f * (float)a.height * (float)a.C;
    const float extent = (float)std::max(a.width, a.height);
    if (a.gaussian_ids) {
        if (a.n_elems == 0) return cudaSuccess;
        densify_stats_packed_kernel<<<(unsigned)((a.n_elems + 255) / 256), 256, 0, s>>>(a, sx, sy, extent);
    } else {
        if (a.N == 0) return cudaSuccess;
        densify_stats_dense_kernel<<<(unsigned)((a.N + 255) / 256), 256, 0, s>>>(a, sx, sy, extent);
    }
    note_launches(1);
    return cudaGetLastError();
}

}  // namespace tg
