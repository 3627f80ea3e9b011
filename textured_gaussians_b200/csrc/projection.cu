// 2DGS projection: forward (ray-splat transform, screen AABB radius, depth,
// camera-facing normal) and its adjoint, for sm_100a.
//
// Forward follows fully_fused_projection_2dgs_fwd.cu:58-238 of the reference
// (same operation order, FP32); the adjoint follows
// fully_fused_projection_2dgs_bwd.cu:44-147 and utils.cuh:660-790, with a third,
// exact form of the d(means2d)/d(ray transform) term.
//
// B200 layout choices: the forward is one thread per (camera, Gaussian), the
// adjoint one thread per Gaussian looping over cameras, so the per-Gaussian
// gradient is summed in registers and written once -- no atomics, bitwise
// deterministic -- instead of the reference's per-(camera, Gaussian) atomics.
#include "tg_common.cuh"

namespace tg {

__global__ void __launch_bounds__(256) project_fwd_kernel(tg_project_fwd_args a) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t total = (int64_t)a.C * a.N;
    if (idx >= total) return;
    const int c = (int)(idx / a.N);
    const int64_t n = idx - (int64_t)c * a.N;

    int32_t radius_out = 0;
    float2 m2d = make_float2(0.f, 0.f);
    float depth = 0.f;
    float Mo[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    f3 nrm = mk3(0, 0, 0);

    const float* vm = a.viewmats + 16 * c;
    const m3 R = {mk3(__ldg(vm + 0), __ldg(vm + 4), __ldg(vm + 8)), mk3(__ldg(vm + 1), __ldg(vm + 5), __ldg(vm + 9)),
                  mk3(__ldg(vm + 2), __ldg(vm + 6), __ldg(vm + 10))};
    const f3 t = mk3(__ldg(vm + 3), __ldg(vm + 7), __ldg(vm + 11));
    const f3 p = mk3(a.means[3 * n], a.means[3 * n + 1], a.means[3 * n + 2]);
    const f3 mc = mul(R, p) + t;
    do {
        if (mc.z < a.near_plane || mc.z > a.far_plane) break;
        const float4 q = __ldg(reinterpret_cast<const float4*>(a.quats) + n);
        const m3 Rq = quat_rot(q.x, q.y, q.z, q.w);
        const float s0 = a.scales[3 * n], s1 = a.scales[3 * n + 1];
        const f3 RS0 = s0 * mul(R, Rq.c0);
        const f3 RS1 = s1 * mul(R, Rq.c1);
        const f3 RS2 = mul(R, Rq.c2);
        const float* K = a.Ks + 9 * c;
        const float fx = __ldg(K + 0), cx = __ldg(K + 2), fy = __ldg(K + 4), cy = __ldg(K + 5);
        const f3 M0 = mk3(fx * RS0.x + cx * RS0.z, fx * RS1.x + cx * RS1.z, fx * mc.x + cx * mc.z);
        const f3 M1 = mk3(fy * RS0.y + cy * RS0.z, fy * RS1.y + cy * RS1.z, fy * mc.y + cy * mc.z);
        const f3 M2 = mk3(RS0.z, RS1.z, mc.z);
        const float distance = M2.x * M2.x + M2.y * M2.y - M2.z * M2.z;
        if (distance == 0.f) break;
        const float inv = 1.f / distance;
        const f3 f = mk3(inv, inv, -inv);
        const float mx = f.x * M0.x * M2.x + f.y * M0.y * M2.y + f.z * M0.z * M2.z;
        const float my = f.x * M1.x * M2.x + f.y * M1.y * M2.y + f.z * M1.z * M2.z;
        const float tx = f.x * M0.x * M0.x + f.y * M0.y * M0.y + f.z * M0.z * M0.z;
        const float ty = f.x * M1.x * M1.x + f.y * M1.y * M1.y + f.z * M1.z * M1.z;
        const float hx = mx * mx - tx, hy = my * my - ty;
        const float radius = ceilf(3.f * sqrtf(fmaxf(1e-4f, fmaxf(hx, hy))));
        if (radius <= a.radius_clip) break;
        if (mx + radius <= 0.f || mx - radius >= (float)a.width || my + radius <= 0.f || my - radius >= (float)a.height)
            break;
        const float mult = dot(-1.f * RS2, mc) > 0.f ? 1.f : -1.f;
        radius_out = (int32_t)radius;
        m2d = make_float2(mx, my);
        depth = mc.z;
        Mo[0] = M0.x; Mo[1] = M0.y; Mo[2] = M0.z;
        Mo[3] = M1.x; Mo[4] = M1.y; Mo[5] = M1.z;
        Mo[6] = M2.x; Mo[7] = M2.y; Mo[8] = M2.z;
        nrm = mult * RS2;
    } while (false);
    a.radii[idx] = radius_out;
    reinterpret_cast<float2*>(a.means2d)[idx] = m2d;
    a.depths[idx] = depth;
    float* mo = a.ray_transforms + 9 * idx;
#pragma unroll
    for (int k = 0; k < 9; ++k) mo[k] = Mo[k];
    a.normals[3 * idx] = nrm.x;
    a.normals[3 * idx + 1] = nrm.y;
    a.normals[3 * idx + 2] = nrm.z;
}

// d L / d q from d L / d R (G.cN = dL/d column N of R), through normalisation.
__device__ __forceinline__ float4 quat_rot_vjp(float w, float x, float y, float z, const m3& G) {
    const float inv = rsqrtf(x * x + y * y + z * z + w * w);
    x *= inv; y *= inv; z *= inv; w *= inv;
    // g(r,c) = dL/dR[r][c]
    const float g00 = G.c0.x, g10 = G.c0.y, g20 = G.c0.z;
    const float g01 = G.c1.x, g11 = G.c1.y, g21 = G.c1.z;
    const float g02 = G.c2.x, g12 = G.c2.y, g22 = G.c2.z;
    const float dw = 2.f * (x * (g21 - g12) + y * (g02 - g20) + z * (g10 - g01));
    const float dx = 2.f * (-2.f * x * (g11 + g22) + y * (g10 + g01) + z * (g20 + g02) + w * (g21 - g12));
    const float dy = 2.f * (x * (g10 + g01) - 2.f * y * (g00 + g22) + z * (g21 + g12) + w * (g02 - g20));
    const float dz = 2.f * (x * (g20 + g02) + y * (g21 + g12) - 2.f * z * (g00 + g11) + w * (g10 - g01));
    const float d = dw * w + dx * x + dy * y + dz * z;
    return make_float4((dw - d * w) * inv, (dx - d * x) * inv, (dy - d * y) * inv, (dz - d * z) * inv);
}

__global__ void __launch_bounds__(256) project_bwd_kernel(tg_project_bwd_args a) {
    const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= a.N) return;
    const f3 p = mk3(a.means[3 * n], a.means[3 * n + 1], a.means[3 * n + 2]);
    const float4 q = __ldg(reinterpret_cast<const float4*>(a.quats) + n);
    const float s0 = a.scales[3 * n], s1 = a.scales[3 * n + 1];
    const m3 Rq = quat_rot(q.x, q.y, q.z, q.w);
    f3 v_mean = mk3(0, 0, 0);
    float4 v_quat = make_float4(0, 0, 0, 0);
    float v_s0 = 0.f, v_s1 = 0.f;
    for (int c = 0; c < a.C; ++c) {
        const int64_t idx = (int64_t)c * a.N + n;
        if (a.radii[idx] <= 0) continue;
        const float* vm = a.viewmats + 16 * c;
        const m3 R = {mk3(__ldg(vm + 0), __ldg(vm + 4), __ldg(vm + 8)),
                      mk3(__ldg(vm + 1), __ldg(vm + 5), __ldg(vm + 9)),
                      mk3(__ldg(vm + 2), __ldg(vm + 6), __ldg(vm + 10))};
        const f3 t = mk3(__ldg(vm + 3), __ldg(vm + 7), __ldg(vm + 11));
        const f3 mc = mul(R, p) + t;
        const float* K = a.Ks + 9 * c;
        const float fx = __ldg(K + 0), cx = __ldg(K + 2), fy = __ldg(K + 4), cy = __ldg(K + 5);
        float G[9];
        const float* vM = a.v_ray_transforms + 9 * idx;
#pragma unroll
        for (int k = 0; k < 9; ++k) G[k] = vM[k];
        G[8] += a.v_depths[idx];
        const float gx = a.v_means2d[2 * idx], gy = a.v_means2d[2 * idx + 1];
        if (gx != 0.f || gy != 0.f) {
            const float* rt = a.ray_transforms + 9 * idx;
            float r[9];
#pragma unroll
            for (int k = 0; k < 9; ++k) r[k] = rt[k];
            const float d = r[6] * r[6] + r[7] * r[7] - r[8] * r[8];
            const float f = 1.f / d;
            if (a.mode != TG_ADJ_EXACT) {
                // reference: diagonal terms of d means2d / d M only
                G[0] += gx * (f * r[6]);
                G[1] += gx * (f * r[7]);
                G[2] += gx * (-f * r[8]);
                G[3] += gy * (f * r[6]);
                G[4] += gy * (f * r[7]);
                G[5] += gy * (-f * r[8]);
                G[6] += gx * (r[0] * (f - 2.f * f * f * r[6] * r[6])) + gy * (r[3] * (f - 2.f * f * f * r[6] * r[6]));
                G[7] += gx * (r[1] * (f - 2.f * f * f * r[7] * r[7])) + gy * (r[4] * (f - 2.f * f * f * r[7] * r[7]));
                G[8] += gx * (-r[2] * (f + 2.f * f * f * r[8] * r[8])) + gy * (-r[5] * (f + 2.f * f * f * r[8] * r[8]));
            } else {
                const float mx = (r[0] * r[6] + r[1] * r[7] - r[2] * r[8]) * f;
                const float my = (r[3] * r[6] + r[4] * r[7] - r[5] * r[8]) * f;
                const float sg[3] = {1.f, 1.f, -1.f};
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    G[i] += gx * sg[i] * r[6 + i] * f;
                    G[3 + i] += gy * sg[i] * r[6 + i] * f;
                    G[6 + i] += gx * sg[i] * (r[i] - 2.f * mx * r[6 + i]) * f +
                                gy * sg[i] * (r[3 + i] - 2.f * my * r[6 + i]) * f;
                }
            }
        }
        // dL/dWH = K^T G, WH = [RS0 RS1 mean_c]
        const f3 w0 = mk3(fx * G[0], fy * G[3], cx * G[0] + cy * G[3] + G[6]);
        const f3 w1 = mk3(fx * G[1], fy * G[4], cx * G[1] + cy * G[4] + G[7]);
        const f3 w2 = mk3(fx * G[2], fy * G[5], cx * G[2] + cy * G[5] + G[8]);
        const f3 vRS0 = mulT(R, w0), vRS1 = mulT(R, w1), vRS2 = mulT(R, w2);
        f3 vtn = mulT(R, mk3(a.v_normals[3 * idx], a.v_normals[3 * idx + 1], a.v_normals[3 * idx + 2]));
        const f3 tn = mul(R, Rq.c2);
        vtn = (dot(-1.f * tn, mc) > 0.f ? 1.f : -1.f) * vtn;
        m3 gR;
        if (a.mode == TG_ADJ_BWD2) {
            gR.c0 = mk3(vRS0.x / s0, vRS0.y / s0, vRS0.z / s0);
            gR.c1 = mk3(vRS1.x / s1, vRS1.y / s1, vRS1.z / s1);
        } else {
            gR.c0 = s0 * vRS0;
            gR.c1 = s1 * vRS1;
        }
        gR.c2 = vtn;
        const float4 dq = quat_rot_vjp(q.x, q.y, q.z, q.w, gR);
        v_quat.x += dq.x; v_quat.y += dq.y; v_quat.z += dq.z; v_quat.w += dq.w;
        v_s0 += dot(vRS0, Rq.c0);
        v_s1 += dot(vRS1, Rq.c1);
        v_mean = v_mean + vRS2;
    }
    a.v_means[3 * n] = v_mean.x;
    a.v_means[3 * n + 1] = v_mean.y;
    a.v_means[3 * n + 2] = v_mean.z;
    reinterpret_cast<float4*>(a.v_quats)[n] = v_quat;
    a.v_scales[3 * n] = v_s0;
    a.v_scales[3 * n + 1] = v_s1;
    a.v_scales[3 * n + 2] = 0.f;
}

cudaError_t launch_project_fwd(const tg_project_fwd_args& a, cudaStream_t s) {
    const int64_t total = (int64_t)a.C * a.N;
    if (total == 0) return cudaSuccess;
    project_fwd_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(a);
    note_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_project_bwd(const tg_project_bwd_args& a, cudaStream_t s) {
    if (a.N == 0) return cudaSuccess;
    project_bwd_kernel<<<(unsigned)((a.N + 255) / 256), 256, 0, s>>>(a);
    note_launches(1);
    return cudaGetLastError();
}

}  // namespace tg
