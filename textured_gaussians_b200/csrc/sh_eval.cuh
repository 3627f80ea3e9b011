// Real spherical-harmonics bases (degree <= 4) and their use for one colour:
// evaluation and adjoint, shared by the SH kernels and the projection with
// fused SH.  Bases follow the real-SH convention of the reference
// (textured_gaussians/cuda/csrc/spherical_harmonics.cuh:17-111, which uses
// Sloan, "Efficient Spherical Harmonic Evaluation", JCGT 2013).  The adjoint
// w.r.t. the direction uses forward-mode dual numbers over the same basis code.
#pragma once
#include "tg_common.cuh"

namespace tg {

struct Dual {
    float v, d0, d1, d2;
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d0 + b.d0, a.d1 + b.d1, a.d2 + b.d2}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d0 - b.d0, a.d1 - b.d1, a.d2 - b.d2}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) {
    return {a.v * b.v, a.d0 * b.v + a.v * b.d0, a.d1 * b.v + a.v * b.d1, a.d2 * b.v + a.v * b.d2};
}
__device__ __forceinline__ Dual operator*(float s, Dual a) { return {s * a.v, s * a.d0, s * a.d1, s * a.d2}; }
__device__ __forceinline__ Dual operator+(Dual a, float s) { return {a.v + s, a.d0, a.d1, a.d2}; }

template <typename S>
__device__ __forceinline__ void sh_bases(int degree, S x, S y, S z, S* b) {
    b[0] = S{} + 0.2820947917738781f;
    if (degree < 1) return;
    b[1] = -0.48860251190292f * y;
    b[2] = 0.48860251190292f * z;
    b[3] = -0.48860251190292f * x;
    if (degree < 2) return;
    const S z2 = z * z, fC1 = x * x - y * y, fS1 = 2.f * (x * y);
    b[4] = 0.5462742152960395f * fS1;
    b[5] = -1.092548430592079f * (z * y);
    b[6] = 0.9461746957575601f * z2 + (-0.3153915652525201f);
    b[7] = -1.092548430592079f * (z * x);
    b[8] = 0.5462742152960395f * fC1;
    if (degree < 3) return;
    const S fC2 = x * fC1 - y * fS1, fS2 = x * fS1 + y * fC1;
    const S t0c = -2.285228997322329f * z2 + 0.4570457994644658f;
    b[9] = -0.5900435899266435f * fS2;
    b[10] = 1.445305721320277f * (z * fS1);
    b[11] = t0c * y;
    b[12] = z * (1.865881662950577f * z2 + (-1.119528997770346f));
    b[13] = t0c * x;
    b[14] = 1.445305721320277f * (z * fC1);
    b[15] = -0.5900435899266435f * fC2;
    if (degree < 4) return;
    const S fC3 = x * fC2 - y * fS2, fS3 = x * fS2 + y * fC2;
    const S t0d = z * (-4.683325804901025f * z2 + 2.007139630671868f);
    const S t1c = 3.31161143515146f * z2 + (-0.47308734787878f);
    b[16] = 0.6258357354491763f * fS3;
    b[17] = -1.770130769779931f * (z * fS2);
    b[18] = t1c * fS1;
    b[19] = t0d * y;
    b[20] = 1.984313483298443f * (z * b[12]) - 1.006230589874905f * b[6];
    b[21] = t0d * x;
    b[22] = t1c * fC1;
    b[23] = -1.770130769779931f * (z * fC2);
    b[24] = 0.6258357354491763f * fC3;
}

// Colour (before the +0.5 / clamp) of direction d (not normalised) under the
// coefficients c [K][3].
__device__ __forceinline__ f3 sh_color(int degree, f3 d, const float* __restrict__ c) {
    float b[25];
    if (degree >= 1) {
        const float inv = rsqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
        sh_bases<float>(degree, d.x * inv, d.y * inv, d.z * inv, b);
    } else {
        b[0] = 0.2820947917738781f;
    }
    const int nb = (degree + 1) * (degree + 1);
    float r0 = 0.f, r1 = 0.f, r2 = 0.f;
    for (int k = 0; k < nb; ++k) {
        r0 += b[k] * c[3 * k];
        r1 += b[k] * c[3 * k + 1];
        r2 += b[k] * c[3 * k + 2];
    }
    return mk3(r0, r1, r2);
}

// Adjoint of sh_color for the colour gradient g: adds d/dc into acc[3k+ch]
// (k < NB = (degree+1)^2) and returns d/dd.
template <int NB = 25>
__device__ __forceinline__ f3 sh_color_vjp(int degree, f3 d, const float* __restrict__ c, f3 g, float* acc) {
    Dual b[25];
    if (degree >= 1) {
        const Dual X{d.x, 1.f, 0.f, 0.f}, Y{d.y, 0.f, 1.f, 0.f}, Z{d.z, 0.f, 0.f, 1.f};
        const Dual n2 = X * X + Y * Y + Z * Z;
        const float inv = rsqrtf(n2.v);
        const float dinv = -0.5f * inv * inv * inv;
        const Dual invd{inv, dinv * n2.d0, dinv * n2.d1, dinv * n2.d2};
        sh_bases<Dual>(degree, X * invd, Y * invd, Z * invd, b);
    } else {
        b[0] = Dual{0.2820947917738781f, 0.f, 0.f, 0.f};
    }
    const int nb = (degree + 1) * (degree + 1);
    float gd0 = 0.f, gd1 = 0.f, gd2 = 0.f;
#pragma unroll
    for (int k = 0; k < NB; ++k) {
        if (k < nb) {
            acc[3 * k] += b[k].v * g.x;
            acc[3 * k + 1] += b[k].v * g.y;
            acc[3 * k + 2] += b[k].v * g.z;
            const float w = c[3 * k] * g.x + c[3 * k + 1] * g.y + c[3 * k + 2] * g.z;
            gd0 += w * b[k].d0;
            gd1 += w * b[k].d1;
            gd2 += w * b[k].d2;
        }
    }
    return mk3(gd0, gd1, gd2);
}

}  // namespace tg
