// 2DGS projection: forward (ray-splat transform, screen AABB radius, depth,
// camera-facing normal) and its adjoint, for sm_100a.
//
// Forward follows fully_fused_projection_2dgs_fwd.cu:58-238 of the reference
// (same operation order, FP32), except that a near-degenerate transform (the
// splat's plane through the camera centre, where the FP32 solve cancels) is
// redone in FP64 from the FP32 parameters; the adjoint follows
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
#include "sh_eval.cuh"

namespace tg {

// One projected (camera, Gaussian) entry.
struct Projected {
    int32_t radius;
    float2 m2d;
    float depth;
    float M[9];
    f3 nrm;
};

// The projection of Gaussian n into camera c entirely in FP64 from the FP32
// parameters: taken only when the FP32 chain has cancelled (see project_one).
// The same operations as project_one; outputs rounded to FP32 at the end.
__device__ __noinline__ bool project_one_f64(const float* __restrict__ means, const float* __restrict__ quats,
                                             const float* __restrict__ scales, const float* __restrict__ viewmats,
                                             const float* __restrict__ Ks, int32_t width, int32_t height,
                                             float near_plane, float far_plane, float radius_clip, int c, int64_t n,
                                             Projected& o) {
    const float* vm = viewmats + 16 * c;
    double R[3][3], t[3], p[3], mc[3];
    for (int r = 0; r < 3; ++r) {
        for (int k = 0; k < 3; ++k) R[r][k] = (double)vm[4 * r + k];
        t[r] = (double)vm[4 * r + 3];
        p[r] = (double)means[3 * n + r];
    }
    for (int r = 0; r < 3; ++r) mc[r] = R[r][0] * p[0] + R[r][1] * p[1] + R[r][2] * p[2] + t[r];
    if (mc[2] < (double)near_plane || mc[2] > (double)far_plane) return false;
    double w = quats[4 * n], x = quats[4 * n + 1], y = quats[4 * n + 2], z = quats[4 * n + 3];
    const double inv = 1.0 / sqrt(w * w + x * x + y * y + z * z);
    w *= inv; x *= inv; y *= inv; z *= inv;
    const double q0[3] = {1.0 - 2.0 * (y * y + z * z), 2.0 * (x * y + w * z), 2.0 * (x * z - w * y)};
    const double q1[3] = {2.0 * (x * y - w * z), 1.0 - 2.0 * (x * x + z * z), 2.0 * (y * z + w * x)};
    const double q2[3] = {2.0 * (x * z + w * y), 2.0 * (y * z - w * x), 1.0 - 2.0 * (x * x + y * y)};
    const double s0 = scales[3 * n], s1 = scales[3 * n + 1];
    double RS0[3], RS1[3], RS2[3];
    for (int r = 0; r < 3; ++r) {
        RS0[r] = s0 * (R[r][0] * q0[0] + R[r][1] * q0[1] + R[r][2] * q0[2]);
        RS1[r] = s1 * (R[r][0] * q1[0] + R[r][1] * q1[1] + R[r][2] * q1[2]);
        RS2[r] = R[r][0] * q2[0] + R[r][1] * q2[1] + R[r][2] * q2[2];
    }
    const float* K = Ks + 9 * c;
    const double fx = K[0], cx = K[2], fy = K[4], cy = K[5];
    const double M0[3] = {fx * RS0[0] + cx * RS0[2], fx * RS1[0] + cx * RS1[2], fx * mc[0] + cx * mc[2]};
    const double M1[3] = {fy * RS0[1] + cy * RS0[2], fy * RS1[1] + cy * RS1[2], fy * mc[1] + cy * mc[2]};
    const double M2[3] = {RS0[2], RS1[2], mc[2]};
    const double distance = M2[0] * M2[0] + M2[1] * M2[1] - M2[2] * M2[2];
    if (distance == 0.0) return false;
    const double f = 1.0 / distance;
    const double mx = f * (M0[0] * M2[0] + M0[1] * M2[1] - M0[2] * M2[2]);
    const double my = f * (M1[0] * M2[0] + M1[1] * M2[1] - M1[2] * M2[2]);
    const double tx = f * (M0[0] * M0[0] + M0[1] * M0[1] - M0[2] * M0[2]);
    const double ty = f * (M1[0] * M1[0] + M1[1] * M1[1] - M1[2] * M1[2]);
    const double radius = ceil(3.0 * sqrt(fmax(1e-4, fmax(mx * mx - tx, my * my - ty))));
    if (!(radius > (double)radius_clip)) return false;
    if (mx + radius <= 0.0 || mx - radius >= (double)width || my + radius <= 0.0 || my - radius >= (double)height)
        return false;
    const double mult = -(RS2[0] * mc[0] + RS2[1] * mc[1] + RS2[2] * mc[2]) > 0.0 ? 1.0 : -1.0;
    o.radius = (int32_t)fmin(radius, 2147483647.0);  // saturates as the FP32 path's conversion does
    o.m2d = make_float2((float)mx, (float)my);
    o.depth = (float)mc[2];
    for (int k = 0; k < 3; ++k) {
        o.M[k] = (float)M0[k];
        o.M[3 + k] = (float)M1[k];
        o.M[6 + k] = (float)M2[k];
    }
    o.nrm = mk3((float)(mult * RS2[0]), (float)(mult * RS2[1]), (float)(mult * RS2[2]));
    return true;
}

// Below this |distance| / |M2|^2 the FP32 solve has lost 6 or more of its 24
// bits to cancellation (the splat's plane passes close to the camera centre:
// relative error of means2d ~1e-8 / ratio), and the projection is redone in
// FP64.  Ordinary splats (scale << depth) have a ratio near 1 and never
// take this path.
constexpr float kDegenerateRel = 1.0f / 64.0f;

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
    // K applied to each column as the reference's (W H)^T K^T product accumulates it
    // (fully_fused_projection_2dgs_fwd.cu:157): the fx / fy term first, then the cx / cy term fused onto
    // it -- the same rounding, so the ray transforms equal the reference's bit for bit
    const f3 M0 = mk3(__fmaf_rn(RS0.z, cx, RS0.x * fx), __fmaf_rn(RS1.z, cx, RS1.x * fx), __fmaf_rn(mc.z, cx, mc.x * fx));
    const f3 M1 = mk3(__fmaf_rn(RS0.z, cy, RS0.y * fy), __fmaf_rn(RS1.z, cy, RS1.y * fy), __fmaf_rn(mc.z, cy, mc.y * fy));
    const f3 M2 = mk3(RS0.z, RS1.z, mc.z);
    const float distance = M2.x * M2.x + M2.y * M2.y - M2.z * M2.z;
    if (fabsf(distance) < kDegenerateRel * (M2.x * M2.x + M2.y * M2.y + M2.z * M2.z))
        return project_one_f64(means, quats, scales, viewmats, Ks, width, height, near_plane, far_plane, radius_clip,
                               c, n, o);
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

// Camera centre of a world-to-camera matrix [R | t]: -R^-1 t, the translation
// of the inverse view matrix (R^-1 by cofactors, so R need not be orthonormal).
__device__ __forceinline__ f3 camera_centre(const float* __restrict__ vm) {
    const float a = vm[0], b = vm[1], c = vm[2], d = vm[4], e = vm[5], f = vm[6], g = vm[8], h = vm[9], i = vm[10];
    const float c00 = e * i - f * h, c01 = f * g - d * i, c02 = d * h - e * g;
    const float c10 = c * h - b * i, c11 = a * i - c * g, c12 = b * g - a * h;
    const float c20 = b * f - c * e, c21 = c * d - a * f, c22 = a * e - b * d;
    const float inv_det = 1.f / (a * c00 + b * c01 + c * c02);
    const float t0 = vm[3], t1 = vm[7], t2 = vm[11];
    return mk3(-(c00 * t0 + c10 * t1 + c20 * t2) * inv_det, -(c01 * t0 + c11 * t1 + c21 * t2) * inv_det,
               -(c02 * t0 + c12 * t1 + c22 * t2) * inv_det);
}

// Fused SH colour of Gaussian n seen from camera c: max(SH + 0.5, 0) for a
// visible entry, 0.5 (the value the unfused path gives a masked entry) otherwise.
__device__ __forceinline__ f3 fused_sh_color(const float* __restrict__ means, const float* __restrict__ viewmats,
                                             int degree, int K, const float* __restrict__ coeffs, int c, int64_t n,
                                             bool visible) {
    if (!visible) return mk3(0.5f, 0.5f, 0.5f);
    const f3 o = camera_centre(viewmats + 16 * c);
    const f3 d = mk3(means[3 * n] - o.x, means[3 * n + 1] - o.y, means[3 * n + 2] - o.z);
    const f3 col = sh_color(degree, d, coeffs + n * K * 3);
    return mk3(fmaxf(col.x + 0.5f, 0.f), fmaxf(col.y + 0.5f, 0.f), fmaxf(col.z + 0.5f, 0.f));
}

__device__ __forceinline__ void store3(float* dst, int64_t i, f3 v) {
    dst[3 * i] = v.x;
    dst[3 * i + 1] = v.y;
    dst[3 * i + 2] = v.z;
}

// Adjoint of fused_sh_color for a visible entry with NB = (degree+1)^2 bases:
// the clamp passes the gradient where SH + 0.5 >= 0 (as torch.clamp_min's
// backward does); coefficient gradients are added into acc[3*NB], the
// direction gradient is returned (it is the gradient of the mean, the camera
// centre being a constant).
template <int NB>
__device__ __forceinline__ f3 fused_sh_vjp(const float* __restrict__ means, const float* __restrict__ viewmats,
                                           int K, const float* __restrict__ coeffs, int c, int64_t n, f3 g,
                                           float* acc) {
    constexpr int degree = NB == 1 ? 0 : NB == 4 ? 1 : NB == 9 ? 2 : NB == 16 ? 3 : 4;
    const f3 o = camera_centre(viewmats + 16 * c);
    const f3 d = mk3(means[3 * n] - o.x, means[3 * n + 1] - o.y, means[3 * n + 2] - o.z);
    const float* crow = coeffs + n * K * 3;
    const f3 col = sh_color(degree, d, crow);
    g.x = col.x + 0.5f >= 0.f ? g.x : 0.f;
    g.y = col.y + 0.5f >= 0.f ? g.y : 0.f;
    g.z = col.z + 0.5f >= 0.f ? g.z : 0.f;
    return sh_color_vjp<NB>(degree, d, crow, g, acc);
}

__global__ void __launch_bounds__(256) project_fwd_kernel(tg_project_fwd_args a) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t total = (int64_t)a.C * a.N;
    if (idx >= total) return;
    const int c = (int)(idx / a.N);
    const int64_t n = idx - (int64_t)c * a.N;
    Projected o;
    const bool vis = project_one(a.means, a.quats, a.scales, a.viewmats, a.Ks, a.width, a.height, a.near_plane,
                                 a.far_plane, a.radius_clip, c, n, o);
    if (!vis) {
        o.radius = 0;
        o.m2d = make_float2(0.f, 0.f);
        o.depth = 0.f;
#pragma unroll
        for (int k = 0; k < 9; ++k) o.M[k] = 0.f;
        o.nrm = mk3(0, 0, 0);
    }
    store_projected(o, idx, a.radii, a.means2d, a.depths, a.ray_transforms, a.normals);
    if (a.sh_coeffs)
        store3(a.colors, idx, fused_sh_color(a.means, a.viewmats, a.sh_degree, a.sh_K, a.sh_coeffs, c, n, vis));
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
                if (a.sh_coeffs)
                    store3(a.colors, pos,
                           fused_sh_color(a.means, a.viewmats, a.sh_degree, a.sh_K, a.sh_coeffs, c, n, true));
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

// NB: SH bases of the fused SH adjoint ((degree+1)^2; 0 = no fused SH), which
// sizes the per-thread coefficient-gradient accumulator.
template <int NB>
__global__ void __launch_bounds__(256) project_bwd_kernel(tg_project_bwd_args a) {
    constexpr bool kSH = NB > 0;
    const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= a.N) return;
    float acc[kSH ? 3 * NB : 1];  // SH coefficient gradient, summed over cameras in registers
    if constexpr (kSH) {
#pragma unroll
        for (int k = 0; k < 3 * NB; ++k) acc[k] = 0.f;
    }
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
        if constexpr (kSH) {
            const f3 gc = mk3(a.v_colors[3 * idx], a.v_colors[3 * idx + 1], a.v_colors[3 * idx + 2]);
            v_mean = v_mean + fused_sh_vjp<NB>(a.means, a.viewmats, a.sh_K, a.sh_coeffs, c, n, gc, acc);
        }
    }
    if constexpr (kSH) {
        float* vc = a.v_sh_coeffs + n * a.sh_K * 3;
#pragma unroll
        for (int k = 0; k < 3 * NB; ++k) vc[k] = acc[k];
        for (int k = 3 * NB; k < 3 * a.sh_K; ++k) vc[k] = 0.f;
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
template <int NB>
__global__ void __launch_bounds__(256) project_packed_bwd_kernel(tg_project_packed_bwd_args a) {
    constexpr bool kSH = NB > 0;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nnz) return;
    const int64_t c = a.camera_ids[i], n = a.gaussian_ids[i];
    if (c < 0 || c >= a.C || n < 0 || n >= a.N) return;
    f3 v_dir = mk3(0, 0, 0);
    if constexpr (kSH) {
        float acc[3 * NB];
#pragma unroll
        for (int k = 0; k < 3 * NB; ++k) acc[k] = 0.f;
        const f3 gc = mk3(a.v_colors[3 * i], a.v_colors[3 * i + 1], a.v_colors[3 * i + 2]);
        if (gc.x != 0.f || gc.y != 0.f || gc.z != 0.f) {
            v_dir = fused_sh_vjp<NB>(a.means, a.viewmats, a.sh_K, a.sh_coeffs, (int)c, n, gc, acc);
            float* vc = a.v_sh_coeffs + n * a.sh_K * 3;
#pragma unroll
            for (int k = 0; k < 3 * NB; ++k)
                if (acc[k] != 0.f) atomicAdd(vc + k, acc[k]);
        }
    }
    const f3 p = mk3(a.means[3 * n], a.means[3 * n + 1], a.means[3 * n + 2]);
    const float4 q = __ldg(reinterpret_cast<const float4*>(a.quats) + n);
    const float s0 = a.scales[3 * n], s1 = a.scales[3 * n + 1];
    const m3 Rq = quat_rot(q.x, q.y, q.z, q.w);
    const EntryGrad g = project_entry_vjp(
        a.viewmats, a.Ks, (int)c, p, q, s0, s1, Rq, a.ray_transforms + 9 * i, a.v_ray_transforms + 9 * i,
        a.v_depths[i], a.v_means2d[2 * i], a.v_means2d[2 * i + 1],
        mk3(a.v_normals[3 * i], a.v_normals[3 * i + 1], a.v_normals[3 * i + 2]), a.mode);
    const f3 vm_total = g.v_mean + v_dir;
    if (a.sparse_grad) {
        a.v_means[3 * i] = vm_total.x;
        a.v_means[3 * i + 1] = vm_total.y;
        a.v_means[3 * i + 2] = vm_total.z;
        reinterpret_cast<float4*>(a.v_quats)[i] = g.v_quat;
        a.v_scales[3 * i] = g.v_s0;
        a.v_scales[3 * i + 1] = g.v_s1;
        a.v_scales[3 * i + 2] = 0.f;
    } else {
        atomicAdd(a.v_means + 3 * n, vm_total.x);
        atomicAdd(a.v_means + 3 * n + 1, vm_total.y);
        atomicAdd(a.v_means + 3 * n + 2, vm_total.z);
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
    const unsigned grid = (unsigned)((a.N + 255) / 256);
    switch (a.sh_coeffs ? a.sh_degree : -1) {
        case 0: project_bwd_kernel<1><<<grid, 256, 0, s>>>(a); break;
        case 1: project_bwd_kernel<4><<<grid, 256, 0, s>>>(a); break;
        case 2: project_bwd_kernel<9><<<grid, 256, 0, s>>>(a); break;
        case 3: project_bwd_kernel<16><<<grid, 256, 0, s>>>(a); break;
        case 4: project_bwd_kernel<25><<<grid, 256, 0, s>>>(a); break;
        default: project_bwd_kernel<0><<<grid, 256, 0, s>>>(a); break;
    }
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
    const unsigned grid = (unsigned)((a.nnz + 255) / 256);
    switch (a.sh_coeffs ? a.sh_degree : -1) {
        case 0: project_packed_bwd_kernel<1><<<grid, 256, 0, s>>>(a); break;
        case 1: project_packed_bwd_kernel<4><<<grid, 256, 0, s>>>(a); break;
        case 2: project_packed_bwd_kernel<9><<<grid, 256, 0, s>>>(a); break;
        case 3: project_packed_bwd_kernel<16><<<grid, 256, 0, s>>>(a); break;
        case 4: project_packed_bwd_kernel<25><<<grid, 256, 0, s>>>(a); break;
        default: project_packed_bwd_kernel<0><<<grid, 256, 0, s>>>(a); break;
    }
    note_launches(1);
    return cudaGetLastError();
}

}  // namespace tg
