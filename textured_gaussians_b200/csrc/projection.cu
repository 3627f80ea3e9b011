// 2DGS projection: forward (ray-splat transform, screen AABB radius, depth,
// camera-facing normal) and its adjoint, for sm_100a.
//
// Forward follows fully_fused_projection_2dgs_fwd.cu:58-238 of the reference
// (same operation order, FP32); the adjoint follows
// fully_fused_projection_2dgs_bwd.cu:44-147 and utils.cuh:660-790, with a third,
// exact form of the d(means2d)/d(ray transform) term.
//
// The packed layout follows fully_fused_projection_packed_2dgs_fwd.cu:19-230
// and fully_fused_projection_packed_2dgs_bwd.cu:19-170 (entries ordered by
// camera, then Gaussian; int64 ids; int32 indptr[C+1]).
//
// B200 layout choices: the dense forward is one thread per (camera, Gaussian),
// the dense adjoint one thread per Gaussian looping over cameras, so the
// per-Gaussian gradient is summed in registers and written once -- no
// atomics, bitwise deterministic -- instead of the reference's
// per-(camera, Gaussian) atomics.  The packed forward is two passes over
// 4096-entry chunks of one camera row (count, then emit after a chunk scan),
// recomputing the projection in the second pass rather than storing a dense
// [C,N] intermediate; dense and packed share one device function, so a
// packed entry is bit-identical to the dense entry it came from.
#include "scan.cuh"

namespace tg {

// One projected (camera, Gaussian) entry.
struct Projected {
    int32_t radius;
    float2 m2d;
    float depth;
    float M[9];
    f3 nrm;
};

// Projects Gaussian n into camera c; false when it is culled (near/far plane,
// degenerate transform, radius clip or off-screen box).
__device__ __forceinline__ bool project_one(const float* __restrict__ means, const float* __restrict__ quats,
                                            const float* __restrict__ scales, const float* __restrict__ viewmats,
                                            const float* __restrict__ Ks, int32_t width, int32_t height,
                                            float near_plane, float far_plane, float radius_clip, int c, int64_t n,
                                            Projected& o) {
    const float* vm = viewmats + 16 * c;
    const m3 R = {mk3(__ldg(vm + 0), __ldg(vm + 4), __ldg(vm + 8)), mk3(__ldg(vm + 1), __ldg(vm + 5), __ldg(vm + 9)),
                  mk3(__ldg(vm + 2), __ldg(vm + 6), __ldg(vm + 10))};
    const f3 t = mk3(__ldg(vm + 3), __ldg(vm + 7), __ldg(vm + 11));
    const f3 p = mk3(means[3 * n], means[3 * n + 1], means[3 * n + 2]);
    const f3 mc = mul(R, p) + t;
    if (mc.z < near_plane || mc.z > far_plane) return false;
    const float4 q = __ldg(reinterpret_cast<const float4*>(quats) + n);
    const m3 Rq = quat_rot(q.x, q.y, q.z, q.w);
    const float s0 = scales[3 * n], s1 = scales[3 * n + 1];
    const f3 RS0 = s0 * mul(R, Rq.c0);
    const f3 RS1 = s1 * mul(R, Rq.c1);
    const f3 RS2 = mul(R, Rq.c2);
    const float* K = Ks + 9 * c;
    const float fx = __ldg(K + 0), cx = __ldg(K + 2), fy = __ldg(K + 4), cy = __ldg(K + 5);
    const f3 M0 = mk3(fx * RS0.x + cx * RS0.z, fx * RS1.x + cx * RS1.z, fx * mc.x + cx * mc.z);
    const f3 M1 = mk3(fy * RS0.y + cy * RS0.z, fy * RS1.y + cy * RS1.z, fy * mc.y + cy * mc.z);
    const f3 M2 = mk3(RS0.z, RS1.z, mc.z);
    const float distance = M2.x * M2.x + M2.y * M2.y - M2.z * M2.z;
    if (distance == 0.f) return false;
    const float inv = 1.f / distance;
    const f3 f = mk3(inv, inv, -inv);
    const float mx = f.x * M0.x * M2.x + f.y * M0.y * M2.y + f.z * M0.z * M2.z;
    const float my = f.x * M1.x * M2.x + f.y * M1.y * M2.y + f.z * M1.z * M2.z;
    const float tx = f.x * M0.x * M0.x + f.y * M0.y * M0.y + f.z * M0.z * M0.z;
    const float ty = f.x * M1.x * M1.x + f.y * M1.y * M1.y + f.z * M1.z * M1.z;
    const float hx = mx * mx - tx, hy = my * my - ty;
    const float radius = ceilf(3.f * sqrtf(fmaxf(1e-4f, fmaxf(hx, hy))));
    if (radius <= radius_clip) return false;
    if (mx + radius <= 0.f || mx - radius >= (float)width || my + radius <= 0.f || my - radius >= (float)height)
        return false;
    const float mult = dot(-1.f * RS2, mc) > 0.f ? 1.f : -1.f;
    o.radius = (int32_t)radius;
    o.m2d = make_float2(mx, my);
    o.depth = mc.z;
    o.M[0] = M0.x; o.M[1] = M0.y; o.M[2] = M0.z;
    o.M[3] = M1.x; o.M[4] = M1.y; o.M[5] = M1.z;
    o.M[6] = M2.x; o.M[7] = M2.y; o.M[8] = M2.z;
    o.nrm = mult * RS2;
    return true;
}

__device__ __forceinline__ void store_projected(const Projected& o, int64_t i, int32_t* radii, float* means2d,
                                                float* depths, float* ray_transforms, float* normals) {
    radii[i] = o.radius;
    reinterpret_cast<float2*>(means2d)[i] = o.m2d;
    depths[i] = o.depth;
    float* mo = ray_transforms + 9 * i;
#pragma unroll
    for (int k = 0; k < 9; ++k) mo[k] = o.M[k];
    normals[3 * i] = o.nrm.x;
    normals[3 * i + 1] = o.nrm.y;
    normals[3 * i + 2] = o.nrm.z;
}

__global__ void __launch_bounds__(256) project_fwd_kernel(tg_project_fwd_args a) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t total = (int64_t)a.C * a.N;
    if (idx >= total) return;
    const int c = (int)(idx / a.N);
    const int64_t n = idx - (int64_t)c * a.N;
    Projected o;
    if (!project_one(a.means, a.quats, a.scales, a.viewmats, a.Ks, a.width, a.height, a.near_plane, a.far_plane,
                     a.radius_clip, c, n, o)) {
        o.radius = 0;
        o.m2d = make_float2(0.f, 0.f);
        o.depth = 0.f;
#pragma unroll
        for (int k = 0; k < 9; ++k) o.M[k] = 0.f;
        o.nrm = mk3(0, 0, 0);
    }
    store_projected(o, idx, a.radii, a.means2d, a.depths, a.ray_transforms, a.normals);
}

// ------------------------------------------------------------------ packed forward
constexpr int kPackThreads = 256;
constexpr int kPackItems = 16;
constexpr int kPackChunk = kPackThreads * kPackItems;  // entries of one camera row per CTA

// Row of camera c: Gaussians [g0, g0 + len) (all N, or the camera's scene in
// the batching form, clamped to [0, N)) and its image size.
struct PackRow {
    int64_t g0, len;
    int32_t width, height;
};
__device__ __forceinline__ PackRow pack_row(const tg_project_packed_args& a, int c) {
    PackRow r{0, a.N, a.width, a.height};
    if (a.gauss_ranges) {
        const int64_t b = min(max(a.gauss_ranges[2 * c], (int64_t)0), (int64_t)a.N);
        const int64_t e = min(max(a.gauss_ranges[2 * c + 1], b), (int64_t)a.N);
        r.g0 = b;
        r.len = e - b;
    }
    if (a.views) {
        r.width = a.views[c].width;
        r.height = a.views[c].height;
    }
    return r;
}

// Pass 1: number of visible entries in each chunk (blockIdx.x) of camera blockIdx.y.
__global__ void __launch_bounds__(kPackThreads) project_packed_count_kernel(tg_project_packed_args a,
                                                                           int64_t* chunk_counts) {
    __shared__ int64_t s_warp[kPackThreads / 32];
    const int c = blockIdx.y;
    const PackRow row = pack_row(a, c);
    const int64_t base = (int64_t)blockIdx.x * kPackChunk;
    int64_t local = 0;
#pragma unroll 1
    for (int i = 0; i < kPackItems; ++i) {
        const int64_t k = base + (int64_t)i * kPackThreads + threadIdx.x;
        if (k >= row.len) break;
        Projected o;
        local += project_one(a.means, a.quats, a.scales, a.viewmats, a.Ks, row.width, row.height, a.near_plane,
                             a.far_plane, a.radius_clip, c, row.g0 + k, o);
    }
    int64_t total;
    block_excl_scan(local, s_warp, total);
    if (threadIdx.x == 0) chunk_counts[(int64_t)c * gridDim.x + blockIdx.x] = total;
}

// indptr[c] = first packed entry of camera c = scanned offset of its first chunk.
__global__ void packed_indptr_kernel(const int64_t* chunk_offsets, const int64_t* nnz, int C, int64_t chunks_per_row,
                                     int32_t* indptr) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c > C) return;
    const int64_t v = c == C ? *nnz : chunk_offsets[(int64_t)c * chunks_per_row];
    indptr[c] = (int32_t)v;
}

// Pass 2: recompute, rank the visible entries of each 256-entry slice with a
// warp ballot plus a CTA prefix over warps, and write them at chunk offset +
// rank, so entries keep (camera, Gaussian) order.
__global__ void __launch_bounds__(kPackThreads) project_packed_emit_kernel(tg_project_packed_args a,
                                                                          const int64_t* chunk_offsets) {
    __shared__ int32_t s_warp[kPackThreads / 32];
    const int c = blockIdx.y;
    const PackRow row = pack_row(a, c);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t base = (int64_t)blockIdx.x * kPackChunk;
    int64_t run = chunk_offsets[(int64_t)c * gridDim.x + blockIdx.x];
#pragma unroll 1
    for (int i = 0; i < kPackItems; ++i) {
        const int64_t slice = base + (int64_t)i * kPackThreads;
        if (slice >= row.len) break;  // uniform across the CTA
        const int64_t k = slice + threadIdx.x;
        const int64_t n = row.g0 + k;
        Projected o;
        const bool vis = k < row.len && project_one(a.means, a.quats, a.scales, a.viewmats, a.Ks, row.width,
                                                    row.height, a.near_plane, a.far_plane, a.radius_clip, c, n, o);
        const unsigned ballot = __ballot_sync(0xffffffffu, vis);
        if (lane == 0) s_warp[warp] = __popc(ballot);
        __syncthreads();
        int32_t before = 0, slice_total = 0;
#pragma unroll
        for (int w = 0; w < kPackThreads / 32; ++w) {
            const int32_t cnt = s_warp[w];
            before += w < warp ? cnt : 0;
            slice_total += cnt;
        }
        __syncthreads();  // s_warp is rewritten by the next slice
        if (vis) {
            const int64_t pos = run + before + __popc(ballot & lanemask_lt());
            if (pos < a.nnz_host) {
                a.camera_ids[pos] = c;
                a.gaussian_ids[pos] = n;
                store_projected(o, pos, a.radii, a.means2d, a.depths, a.ray_transforms, a.normals);
            } else if (a.overflow) {
                atomicOr(a.overflow, 1u);
            }
        }
        run += slice_total;
    }
}

// Capacity mode: the unused tail [*nnz, capacity) keeps radius 0 (it intersects
// nothing) and gets Gaussian ids spread over all N, so gathers and their
// scatter-add adjoints over the tail do not pile onto one Gaussian.
__global__ void __launch_bounds__(256) packed_tail_kernel(const int64_t* nnz, int64_t capacity, int32_t N,
                                                          int64_t* gaussian_ids) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= capacity || i < *nnz) return;
    gaussian_ids[i] = N > 0 ? i % N : 0;
}

// ------------------------------------------------------------------ adjoint
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


// Gradient of one (camera, Gaussian) entry with respect to the Gaussian's
// mean, rotation and scales, given the upstream gradients of its means2d,
// depth, normal and ray transform (rt: the forward's ray transform).
struct EntryGrad {
    f3 v_mean;
    float4 v_quat;
    float v_s0, v_s1;
};

__device__ __forceinline__ EntryGrad project_entry_vjp(const float* __restrict__ viewmats,
                                                       const float* __restrict__ Ks, int c, f3 p, float4 q,
                                                       float s0, float s1, const m3& Rq, const float* rt,
                                                       const float* vM, float v_depth, float gx, float gy, f3 v_nrm,
                                                       int mode) {
    const float* vm = viewmats + 16 * c;
    const m3 R = {mk3(__ldg(vm + 0), __ldg(vm + 4), __ldg(vm + 8)),
                  mk3(__ldg(vm + 1), __ldg(vm + 5), __ldg(vm + 9)),
                  mk3(__ldg(vm + 2), __ldg(vm + 6), __ldg(vm + 10))};
    const f3 t = mk3(__ldg(vm + 3), __ldg(vm + 7), __ldg(vm + 11));
    const f3 mc = mul(R, p) + t;
    const float* K = Ks + 9 * c;
    const float fx = __ldg(K + 0), cx = __ldg(K + 2), fy = __ldg(K + 4), cy = __ldg(K + 5);
    float G[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) G[k] = vM[k];
    G[8] += v_depth;
    if (gx != 0.f || gy != 0.f) {
        float r[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) r[k] = rt[k];
        const float d = r[6] * r[6] + r[7] * r[7] - r[8] * r[8];
        const float f = 1.f / d;
        if (mode != TG_ADJ_EXACT) {
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
    f3 vtn = mulT(R, v_nrm);
    const f3 tn = mul(R, Rq.c2);
    vtn = (dot(-1.f * tn, mc) > 0.f ? 1.f : -1.f) * vtn;
    m3 gR;
    if (mode == TG_ADJ_BWD2) {
        gR.c0 = mk3(vRS0.x / s0, vRS0.y / s0, vRS0.z / s0);
        gR.c1 = mk3(vRS1.x / s1, vRS1.y / s1, vRS1.z / s1);
    } else {
        gR.c0 = s0 * vRS0;
        gR.c1 = s1 * vRS1;
    }
    gR.c2 = vtn;
    EntryGrad out;
    out.v_quat = quat_rot_vjp(q.x, q.y, q.z, q.w, gR);
    out.v_s0 = dot(vRS0, Rq.c0);
    out.v_s1 = dot(vRS1, Rq.c1);
    out.v_mean = vRS2;
    return out;
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
        const EntryGrad g = project_entry_vjp(
            a.viewmats, a.Ks, c, p, q, s0, s1, Rq, a.ray_transforms + 9 * idx, a.v_ray_transforms + 9 * idx,
            a.v_depths[idx], a.v_means2d[2 * idx], a.v_means2d[2 * idx + 1],
            mk3(a.v_normals[3 * idx], a.v_normals[3 * idx + 1], a.v_normals[3 * idx + 2]), a.mode);
        v_quat.x += g.v_quat.x; v_quat.y += g.v_quat.y; v_quat.z += g.v_quat.z; v_quat.w += g.v_quat.w;
        v_s0 += g.v_s0;
        v_s1 += g.v_s1;
        v_mean = v_mean + g.v_mean;
    }
    a.v_means[3 * n] = v_mean.x;
    a.v_means[3 * n + 1] = v_mean.y;
    a.v_means[3 * n + 2] = v_mean.z;
    reinterpret_cast<float4*>(a.v_quats)[n] = v_quat;
    a.v_scales[3 * n] = v_s0;
    a.v_scales[3 * n + 1] = v_s1;
    a.v_scales[3 * n + 2] = 0.f;
}

// Packed adjoint: one thread per entry.  Sparse: the entry's gradient is
// written at its own row.  Dense: added into the Gaussian's row with float
// atomics (entries of one Gaussian sit C-strided apart in camera-major order,
// so there is nothing to combine inside a warp first).
__global__ void __launch_bounds__(256) project_packed_bwd_kernel(tg_project_packed_bwd_args a) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nnz) return;
    const int64_t c = a.camera_ids[i], n = a.gaussian_ids[i];
    if (c < 0 || c >= a.C || n < 0 || n >= a.N) return;
    const f3 p = mk3(a.means[3 * n], a.means[3 * n + 1], a.means[3 * n + 2]);
    const float4 q = __ldg(reinterpret_cast<const float4*>(a.quats) + n);
    const float s0 = a.scales[3 * n], s1 = a.scales[3 * n + 1];
    const m3 Rq = quat_rot(q.x, q.y, q.z, q.w);
    const EntryGrad g = project_entry_vjp(
        a.viewmats, a.Ks, (int)c, p, q, s0, s1, Rq, a.ray_transforms + 9 * i, a.v_ray_transforms + 9 * i,
        a.v_depths[i], a.v_means2d[2 * i], a.v_means2d[2 * i + 1],
        mk3(a.v_normals[3 * i], a.v_normals[3 * i + 1], a.v_normals[3 * i + 2]), a.mode);
    if (a.sparse_grad) {
        a.v_means[3 * i] = g.v_mean.x;
        a.v_means[3 * i + 1] = g.v_mean.y;
        a.v_means[3 * i + 2] = g.v_mean.z;
        reinterpret_cast<float4*>(a.v_quats)[i] = g.v_quat;
        a.v_scales[3 * i] = g.v_s0;
        a.v_scales[3 * i + 1] = g.v_s1;
        a.v_scales[3 * i + 2] = 0.f;
    } else {
        atomicAdd(a.v_means + 3 * n, g.v_mean.x);
        atomicAdd(a.v_means + 3 * n + 1, g.v_mean.y);
        atomicAdd(a.v_means + 3 * n + 2, g.v_mean.z);
        atomicAdd(reinterpret_cast<float4*>(a.v_quats) + n, g.v_quat);
        atomicAdd(a.v_scales + 3 * n, g.v_s0);
        atomicAdd(a.v_scales + 3 * n + 1, g.v_s1);
    }
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

size_t project_packed_workspace_bytes(int32_t C, int32_t N) {
    const int64_t chunks = (int64_t)std::max(C, 0) * (((int64_t)std::max(N, 0) + kPackChunk - 1) / kPackChunk);
    return align256(sizeof(int64_t) * (size_t)std::max<int64_t>(chunks, 1));
}

// Chunks per camera row: the longest row over 4096.
inline int64_t packed_chunks_per_row(const tg_project_packed_args& a) {
    const int64_t len = a.gauss_ranges ? std::min<int64_t>(a.max_range, a.N) : a.N;
    return (len + kPackChunk - 1) / kPackChunk;
}

// Count pass: chunk counts, their scan (-> *nnz), indptr.  Three launches.
cudaError_t launch_project_packed_count(const tg_project_packed_args& a, cudaStream_t s) {
    const int64_t per_row = packed_chunks_per_row(a);
    if ((int64_t)a.C * per_row == 0) {
        cudaError_t e = cudaMemsetAsync(a.nnz, 0, sizeof(int64_t), s);
        if (e == cudaSuccess) e = cudaMemsetAsync(a.indptr, 0, sizeof(int32_t) * ((size_t)a.C + 1), s);
        return e;
    }
    int64_t* chunk = static_cast<int64_t*>(a.workspace);
    project_packed_count_kernel<<<dim3((unsigned)per_row, (unsigned)a.C), kPackThreads, 0, s>>>(a, chunk);
    note_launches(1);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = launch_scan_chunk_sums(chunk, (int64_t)a.C * per_row, a.nnz, s);
    if (e != cudaSuccess) return e;
    packed_indptr_kernel<<<(unsigned)((a.C + 1 + 255) / 256), 256, 0, s>>>(chunk, a.nnz, a.C, per_row, a.indptr);
    note_launches(1);
    return cudaGetLastError();
}

// Emit pass; the chunk offsets left in the workspace by the count pass are reused.
cudaError_t launch_project_packed_emit(const tg_project_packed_args& a, cudaStream_t s) {
    const int64_t per_row = packed_chunks_per_row(a);
    if ((int64_t)a.C * per_row == 0 || a.nnz_host == 0) return cudaSuccess;
    project_packed_emit_kernel<<<dim3((unsigned)per_row, (unsigned)a.C), kPackThreads, 0, s>>>(
        a, static_cast<const int64_t*>(a.workspace));
    note_launches(1);
    if (a.overflow) {
        packed_tail_kernel<<<(unsigned)((a.nnz_host + 255) / 256), 256, 0, s>>>(a.nnz, a.nnz_host, a.N,
                                                                                a.gaussian_ids);
        note_launches(1);
    }
    return cudaGetLastError();
}

cudaError_t launch_project_packed_bwd(const tg_project_packed_bwd_args& a, cudaStream_t s) {
    if (a.nnz == 0) return cudaSuccess;
    project_packed_bwd_kernel<<<(unsigned)((a.nnz + 255) / 256), 256, 0, s>>>(a);
    note_launches(1);
    return cudaGetLastError();
}

}  // namespace tg
