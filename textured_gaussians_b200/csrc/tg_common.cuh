// Shared device helpers for the B200 textured 2DGS kernels (sm_100a).
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "../../include/tg2dgs.h"

namespace tg {

constexpr int kNumSMs = 148;  // B200: 2 dies x 74 SMs

// Process-wide count of kernel launches (defined in capi.cu).
void note_launches(unsigned n);

__host__ __device__ inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

struct f3 {
    float x, y, z;
};
__device__ __forceinline__ f3 mk3(float a, float b, float c) { return f3{a, b, c}; }
__device__ __forceinline__ f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ f3 operator*(float s, f3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ f3 cross(f3 a, f3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// 3x3 matrix held as three columns.
struct m3 {
    f3 c0, c1, c2;
};
__device__ __forceinline__ f3 mul(const m3& m, f3 v) {
    return {m.c0.x * v.x + m.c1.x * v.y + m.c2.x * v.z, m.c0.y * v.x + m.c1.y * v.y + m.c2.y * v.z,
            m.c0.z * v.x + m.c1.z * v.y + m.c2.z * v.z};
}
__device__ __forceinline__ f3 mulT(const m3& m, f3 v) { return {dot(m.c0, v), dot(m.c1, v), dot(m.c2, v)}; }

// Rotation (columns) of a wxyz quaternion, normalised first.
__device__ __forceinline__ m3 quat_rot(float w, float x, float y, float z) {
    const float inv = rsqrtf(x * x + y * y + z * z + w * w);
    x *= inv; y *= inv; z *= inv; w *= inv;
    const float x2 = x * x, y2 = y * y, z2 = z * z, xy = x * y, xz = x * z, yz = y * z;
    const float wx = w * x, wy = w * y, wz = w * z;
    m3 R;
    R.c0 = mk3(1.f - 2.f * (y2 + z2), 2.f * (xy + wz), 2.f * (xz - wy));
    R.c1 = mk3(2.f * (xy - wz), 1.f - 2.f * (x2 + z2), 2.f * (yz + wx));
    R.c2 = mk3(2.f * (xz + wy), 2.f * (yz - wx), 1.f - 2.f * (x2 + y2));
    return R;
}

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// ------------------------------------------------------------- texel loads
// One RGBA texel as float4, from each storage format.  Textures are read-only
// for the whole launch, so the non-coherent path (ld.global.nc) is used.
struct TexF32 {
    using storage = float4;
    static constexpr int kFormat = TG_TEX_F32;
    __device__ __forceinline__ static float4 load(const void* base, int64_t texel, float /*scale*/) {
        return __ldg(reinterpret_cast<const float4*>(base) + texel);
    }
};
struct TexBF16 {
    static constexpr int kFormat = TG_TEX_BF16;
    __device__ __forceinline__ static float4 load(const void* base, int64_t texel, float) {
        const uint2 v = __ldg(reinterpret_cast<const uint2*>(base) + texel);
        float4 r;
        r.x = __uint_as_float(v.x << 16);
        r.y = __uint_as_float(v.x & 0xffff0000u);
        r.z = __uint_as_float(v.y << 16);
        r.w = __uint_as_float(v.y & 0xffff0000u);
        return r;
    }
};
struct TexF16 {
    static constexpr int kFormat = TG_TEX_F16;
    __device__ __forceinline__ static float4 load(const void* base, int64_t texel, float) {
        const uint2 v = __ldg(reinterpret_cast<const uint2*>(base) + texel);
        const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&v.x));
        const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&v.y));
        return make_float4(a.x, a.y, b.x, b.y);
    }
};
struct TexFP8 {
    static constexpr int kFormat = TG_TEX_FP8_E4M3;
    __device__ __forceinline__ static float4 load(const void* base, int64_t texel, float scale) {
        const uint32_t v = __ldg(reinterpret_cast<const uint32_t*>(base) + texel);
        __nv_fp8x4_e4m3 q;
        *reinterpret_cast<uint32_t*>(&q) = v;
        const float4 f = static_cast<float4>(q);
        return make_float4(f.x * scale, f.y * scale, f.z * scale, f.w * scale);
    }
};
struct TexNone {
    static constexpr int kFormat = TG_TEX_NONE;
    __device__ __forceinline__ static float4 load(const void*, int64_t, float) { return make_float4(0, 0, 0, 0); }
};

__device__ __forceinline__ float f4get(const float4& v, int k) {
    return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w));
}

}  // namespace tg
