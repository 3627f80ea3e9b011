// Spherical-harmonics colour evaluation (degree <= 4) and its adjoint, sm_100a.
//
// Bases and their dual-number adjoint are in sh_eval.cuh (the reference's
// convention, textured_gaussians/cuda/csrc/spherical_harmonics.cuh:17-111).
// One thread per (camera, Gaussian) element computes all three channels.
#include "sh_eval.cuh"

namespace tg {

__global__ void sh_fwd_kernel(int64_t n, int64_t rows, int degree, int K, const float* __restrict__ dirs,
                              const float* __restrict__ coeffs, const uint8_t* __restrict__ masks,
                              float* __restrict__ colors) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float r0 = 0.f, r1 = 0.f, r2 = 0.f;
    if (masks == nullptr || masks[i]) {
        float b[25];
        if (degree >= 1) {
            const float dx = dirs[3 * i], dy = dirs[3 * i + 1], dz = dirs[3 * i + 2];
            const float inv = rsqrtf(dx * dx + dy * dy + dz * dz);
            sh_bases<float>(degree, dx * inv, dy * inv, dz * inv, b);
        } else {
            b[0] = 0.2820947917738781f;
        }
        const int nb = (degree + 1) * (degree + 1);
        const float* c = coeffs + (i % rows) * K * 3;
        for (int k = 0; k < nb; ++k) {
            r0 += b[k] * c[3 * k];
            r1 += b[k] * c[3 * k + 1];
            r2 += b[k] * c[3 * k + 2];
        }
    }
    colors[3 * i] = r0;
    colors[3 * i + 1] = r1;
    colors[3 * i + 2] = r2;
}

// One thread per coefficient row, looping over the elements that share it, so
// the coefficient gradient is summed in registers (no atomics).
__global__ void sh_bwd_kernel(int64_t n, int64_t rows, int degree, int K, const float* __restrict__ dirs,
                              const float* __restrict__ coeffs, const uint8_t* __restrict__ masks,
                              const float* __restrict__ v_colors, float* __restrict__ v_coeffs,
                              float* __restrict__ v_dirs) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    const int nb = (degree + 1) * (degree + 1);
    const float* c = coeffs + r * K * 3;
    float acc[25 * 3];
#pragma unroll
    for (int k = 0; k < 75; ++k) acc[k] = 0.f;
    for (int64_t i = r; i < n; i += rows) {
        const bool on = masks == nullptr || masks[i];
        if (!on) {
            if (v_dirs) v_dirs[3 * i] = v_dirs[3 * i + 1] = v_dirs[3 * i + 2] = 0.f;
            continue;
        }
        const float g0 = v_colors[3 * i], g1 = v_colors[3 * i + 1], g2 = v_colors[3 * i + 2];
        Dual b[25];
        if (degree >= 1) {
            const float dx = dirs[3 * i], dy = dirs[3 * i + 1], dz = dirs[3 * i + 2];
            const Dual X{dx, 1.f, 0.f, 0.f}, Y{dy, 0.f, 1.f, 0.f}, Z{dz, 0.f, 0.f, 1.f};
            const Dual n2 = X * X + Y * Y + Z * Z;
            const float inv = rsqrtf(n2.v);
            const float dinv = -0.5f * inv * inv * inv;
            const Dual invd{inv, dinv * n2.d0, dinv * n2.d1, dinv * n2.d2};
            sh_bases<Dual>(degree, X * invd, Y * invd, Z * invd, b);
        } else {
            b[0] = Dual{0.2820947917738781f, 0.f, 0.f, 0.f};
        }
        float gd0 = 0.f, gd1 = 0.f, gd2 = 0.f;
#pragma unroll
        for (int k = 0; k < 25; ++k) {
            if (k < nb) {
                acc[3 * k] += b[k].v * g0;
                acc[3 * k + 1] += b[k].v * g1;
                acc[3 * k + 2] += b[k].v * g2;
                const float w = c[3 * k] * g0 + c[3 * k + 1] * g1 + c[3 * k + 2] * g2;
                gd0 += w * b[k].d0;
                gd1 += w * b[k].d1;
                gd2 += w * b[k].d2;
            }
        }
        if (v_dirs) {
            v_dirs[3 * i] = gd0;
            v_dirs[3 * i + 1] = gd1;
            v_dirs[3 * i + 2] = gd2;
        }
    }
    float* vc = v_coeffs + r * K * 3;
    for (int k = 0; k < K; ++k) {
        const bool in = k < nb;
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) vc[3 * k + ch] = in ? acc[3 * (k < 25 ? k : 0) + ch] : 0.f;
    }
}

cudaError_t launch_sh_fwd(int64_t n, int64_t rows, int degree, int K, const float* dirs, const float* coeffs,
                          const uint8_t* masks, float* colors, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    sh_fwd_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, rows, degree, K, dirs, coeffs, masks, colors);
    note_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_sh_bwd(int64_t n, int64_t rows, int degree, int K, const float* dirs, const float* coeffs,
                          const uint8_t* masks, const float* v_colors, float* v_coeffs, float* v_dirs,
                          cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    sh_bwd_kernel<<<(unsigned)((rows + 127) / 128), 128, 0, s>>>(n, rows, degree, K, dirs, coeffs, masks, v_colors,
                                                                 v_coeffs, v_dirs);
    note_launches(1);
    return cudaGetLastError();
}

}  // namespace tg
