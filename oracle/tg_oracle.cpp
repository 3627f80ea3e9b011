// CPU oracle for the textured 2DGS rasterization path -- TEST INFRASTRUCTURE ONLY.
//
// This file restates, in plain C++17 (OpenMP over tiles), the algorithm of the
// reference's CUDA kernels for projection, tile intersection, stable key sort,
// offset encoding, the textured / plain compositor forward and the three
// compositor adjoints.  It is compiled by oracle/build.py into
// oracle/libtg_oracle.so and is only ever loaded by tests/, by
// __graft_entry__.smoke() and by bench.py's CPU-baseline leg, always as the
// checker.  The product path (textured_gaussians_b200) never links or calls it.
//
// Every function is templated on the scalar type: T=float is the FP32 parity
// mode (IEEE arithmetic, no fused multiply-add, same operation order as the
// reference), T=double is the FP64 oracle used for error tables and finite
// differences.
//
// Pinning: projection, intersection, offsets and SH are pinned by golden
// vectors produced from the reference's own pure-torch twins
// (tests/golden/make_golden.py).  The plain-2DGS compositor forward is pinned
// against the reference's torch `accumulate_2dgs` on the contributing pairs.
// The TEXTURED compositor has no executable reference on any machine here (the
// reference ships no CPU textured rasterizer and its CUDA build needs the
// missing GLM headers), so its parity is UNPINNED: it rests on this
// restatement of textured_gaussians/cuda/csrc/rasterize_to_pixels_textured_
// gaussians_2dgs_{fwd,bwd,bwd2}.cu, line by line.
//
// Reference files followed (paths inside the reference project):
//   projection fwd   textured_gaussians/cuda/csrc/fully_fused_projection_2dgs_fwd.cu:58-238
//   projection bwd   textured_gaussians/cuda/csrc/fully_fused_projection_2dgs_bwd.cu:44-147,
//                    textured_gaussians/cuda/csrc/utils.cuh:16-65, :660-790
//   intersection     textured_gaussians/cuda/csrc/isect_tiles.cu:44-104, :152-160, :246-300
//   offsets          textured_gaussians/cuda/csrc/isect_tiles.cu:309-355
//   bilinear filter  textured_gaussians/cuda/csrc/filters/bilinear.cuh:16-64
//   compositor fwd   textured_gaussians/cuda/csrc/rasterize_to_pixels_textured_gaussians_2dgs_fwd.cu:73-445
//                    textured_gaussians/cuda/csrc/rasterize_to_pixels_2dgs_fwd.cu:281-366 (plain alpha)
//   compositor bwd   textured_gaussians/cuda/csrc/rasterize_to_pixels_textured_gaussians_2dgs_bwd.cu:77-700
//                    textured_gaussians/cuda/csrc/rasterize_to_pixels_textured_gaussians_2dgs_bwd2.cu:612-676
//                    textured_gaussians/cuda/csrc/rasterize_to_pixels_2dgs_bwd.cu:347-560 (plain)
//   spherical harm.  textured_gaussians/cuda/csrc/spherical_harmonics.cuh:17-111
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

namespace {

template <typename T> struct V3 { T x, y, z; };
template <typename T> inline V3<T> v3(T a, T b, T c) { return V3<T>{a, b, c}; }
template <typename T> inline V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <typename T> inline V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <typename T> inline V3<T> operator*(T s, V3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <typename T> inline T dot3(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T> inline V3<T> cross3(V3<T> a, V3<T> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// 3x3 matrix stored by columns, like the column-major matrices of the reference.
template <typename T> struct M3 { V3<T> c[3]; };
template <typename T> inline V3<T> mul(const M3<T>& m, V3<T> v) {
    // column combination, evaluated left to right: c0*x + c1*y + c2*z
    return {m.c[0].x * v.x + m.c[1].x * v.y + m.c[2].x * v.z,
            m.c[0].y * v.x + m.c[1].y * v.y + m.c[2].y * v.z,
            m.c[0].z * v.x + m.c[1].z * v.y + m.c[2].z * v.z};
}
template <typename T> inline V3<T> mulT(const M3<T>& m, V3<T> v) {  // m^T v
    return {dot3(m.c[0], v), dot3(m.c[1], v), dot3(m.c[2], v)};
}

// Rotation matrix (columns) of a not-necessarily-normalised wxyz quaternion.
// Reference: utils.cuh:16-39.
template <typename T> inline M3<T> quat_rot(const T* q, T* inv_norm_out = nullptr) {
    T w = q[0], x = q[1], y = q[2], z = q[3];
    T inv = T(1) / std::sqrt(x * x + y * y + z * z + w * w);
    if (inv_norm_out) *inv_norm_out = inv;
    x *= inv; y *= inv; z *= inv; w *= inv;
    T x2 = x * x, y2 = y * y, z2 = z * z, xy = x * y, xz = x * z, yz = y * z, wx = w * x, wy = w * y, wz = w * z;
    M3<T> R;
    R.c[0] = v3<T>(T(1) - T(2) * (y2 + z2), T(2) * (xy + wz), T(2) * (xz - wy));
    R.c[1] = v3<T>(T(2) * (xy - wz), T(1) - T(2) * (x2 + z2), T(2) * (yz + wx));
    R.c[2] = v3<T>(T(2) * (xz + wy), T(2) * (yz - wx), T(1) - T(2) * (x2 + y2));
    return R;
}

// d L / d q given d L / d R (gR.c[j] = dL/d(column j of R)).  Derived from the
// rotation formula above, then projected through the normalisation.
// Reference: utils.cuh:41-65.
template <typename T> inline void quat_rot_vjp(const T* q, const M3<T>& gR, T* vq) {
    T w = q[0], x = q[1], y = q[2], z = q[3];
    T inv = T(1) / std::sqrt(x * x + y * y + z * z + w * w);
    x *= inv; y *= inv; z *= inv; w *= inv;
    // g(r, c) = dL/dR[r][c] = gR.c[c] component r
    auto g = [&](int r, int c) -> T { const V3<T>& col = gR.c[c]; return r == 0 ? col.x : (r == 1 ? col.y : col.z); };
    T dw = T(2) * (x * (g(2, 1) - g(1, 2)) + y * (g(0, 2) - g(2, 0)) + z * (g(1, 0) - g(0, 1)));
    T dx = T(2) * (-T(2) * x * (g(1, 1) + g(2, 2)) + y * (g(1, 0) + g(0, 1)) + z * (g(2, 0) + g(0, 2)) +
                   w * (g(2, 1) - g(1, 2)));
    T dy = T(2) * (x * (g(1, 0) + g(0, 1)) - T(2) * y * (g(0, 0) + g(2, 2)) + z * (g(2, 1) + g(1, 2)) +
                   w * (g(0, 2) - g(2, 0)));
    T dz = T(2) * (x * (g(2, 0) + g(0, 2)) + y * (g(2, 1) + g(1, 2)) - T(2) * z * (g(0, 0) + g(1, 1)) +
                   w * (g(1, 0) - g(0, 1)));
    T d = dw * w + dx * x + dy * y + dz * z;
    vq[0] += (dw - d * w) * inv;
    vq[1] += (dx - d * x) * inv;
    vq[2] += (dy - d * y) * inv;
    vq[3] += (dz - d * z) * inv;
}

template <typename T> inline void view_rt(const T* vm, M3<T>& R, V3<T>& t) {
    R.c[0] = v3<T>(vm[0], vm[4], vm[8]);
    R.c[1] = v3<T>(vm[1], vm[5], vm[9]);
    R.c[2] = v3<T>(vm[2], vm[6], vm[10]);
    t = v3<T>(vm[3], vm[7], vm[11]);
}

// ---------------------------------------------------------------- projection
template <typename T>
void project_fwd(int C, int N, const T* means, const T* quats, const T* scales, const T* viewmats, const T* Ks,
                 int W, int H, T near_plane, T far_plane, T radius_clip, int32_t* radii, T* means2d, T* depths,
                 T* M, T* normals) {
#pragma omp parallel for schedule(static)
    for (int64_t idx = 0; idx < (int64_t)C * N; ++idx) {
        const int c = (int)(idx / N), n = (int)(idx % N);
        radii[idx] = 0;
        means2d[2 * idx] = means2d[2 * idx + 1] = 0;
        depths[idx] = 0;
        for (int k = 0; k < 9; ++k) M[9 * idx + k] = 0;
        for (int k = 0; k < 3; ++k) normals[3 * idx + k] = 0;
        M3<T> R; V3<T> t;
        view_rt(viewmats + 16 * c, R, t);
        const T* K = Ks + 9 * c;
        const V3<T> p = v3<T>(means[3 * n], means[3 * n + 1], means[3 * n + 2]);
        const V3<T> mc = mul(R, p) + t;
        if (mc.z < near_plane || mc.z > far_plane) continue;
        const M3<T> Rq = quat_rot<T>(quats + 4 * n);
        const T s0 = scales[3 * n], s1 = scales[3 * n + 1];
        const V3<T> RS0 = s0 * mul(R, Rq.c[0]);
        const V3<T> RS1 = s1 * mul(R, Rq.c[1]);
        const V3<T> RS2 = mul(R, Rq.c[2]);
        const T fx = K[0], cx = K[2], fy = K[4], cy = K[5];
        // rows of K * [RS0 RS1 mc]
        const V3<T> M0 = v3<T>(fx * RS0.x + cx * RS0.z, fx * RS1.x + cx * RS1.z, fx * mc.x + cx * mc.z);
        const V3<T> M1 = v3<T>(fy * RS0.y + cy * RS0.z, fy * RS1.y + cy * RS1.z, fy * mc.y + cy * mc.z);
        const V3<T> M2 = v3<T>(RS0.z, RS1.z, mc.z);
        const T distance = M2.x * M2.x + M2.y * M2.y - M2.z * M2.z;
        if (distance == T(0)) continue;  // reference leaves radii unwritten here; we write 0
        const T inv = T(1) / distance;
        const V3<T> f = v3<T>(inv, inv, -inv);
        const T mx = f.x * M0.x * M2.x + f.y * M0.y * M2.y + f.z * M0.z * M2.z;
        const T my = f.x * M1.x * M2.x + f.y * M1.y * M2.y + f.z * M1.z * M2.z;
        const T tx = f.x * M0.x * M0.x + f.y * M0.y * M0.y + f.z * M0.z * M0.z;
        const T ty = f.x * M1.x * M1.x + f.y * M1.y * M1.y + f.z * M1.z * M1.z;
        const T hx = mx * mx - tx, hy = my * my - ty;
        const T radius = std::ceil(T(3) * std::sqrt(std::max(T(1e-4), std::max(hx, hy))));
        if (radius <= radius_clip) continue;
        if (mx + radius <= 0 || mx - radius >= W || my + radius <= 0 || my - radius >= H) continue;
        const T mult = dot3(T(-1) * RS2, mc) > 0 ? T(1) : T(-1);
        radii[idx] = (int32_t)radius;
        means2d[2 * idx] = mx;
        means2d[2 * idx + 1] = my;
        depths[idx] = mc.z;
        T* m = M + 9 * idx;
        m[0] = M0.x; m[1] = M0.y; m[2] = M0.z;
        m[3] = M1.x; m[4] = M1.y; m[5] = M1.z;
        m[6] = M2.x; m[7] = M2.y; m[8] = M2.z;
        normals[3 * idx] = mult * RS2.x;
        normals[3 * idx + 1] = mult * RS2.y;
        normals[3 * idx + 2] = mult * RS2.z;
    }
}

// mode: 0 = reference adjoint (bwd), 1 = reference norm_rot_grad adjoint (bwd2),
//       2 = exact derivative of the forward (full d means2d / d M).
template <typename T>
void project_bwd(int C, int N, const T* means, const T* quats, const T* scales, const T* viewmats, const T* Ks,
                 const int32_t* radii, const T* M, const T* v_means2d, const T* v_depths, const T* v_normals,
                 const T* v_M, int mode, T* v_means, T* v_quats, T* v_scales) {
    // serial accumulation keeps the oracle deterministic
    for (int64_t idx = 0; idx < (int64_t)C * N; ++idx) {
        if (radii[idx] <= 0) continue;
        const int c = (int)(idx / N), n = (int)(idx % N);
        M3<T> R; V3<T> t;
        view_rt(viewmats + 16 * c, R, t);
        const T* K = Ks + 9 * c;
        const T fx = K[0], cx = K[2], fy = K[4], cy = K[5];
        const V3<T> p = v3<T>(means[3 * n], means[3 * n + 1], means[3 * n + 2]);
        const V3<T> mc = mul(R, p) + t;
        const T* q = quats + 4 * n;
        const T s0 = scales[3 * n], s1 = scales[3 * n + 1];
        // G[i][j] = dL / d M[i][j]  (row-major ray transform)
        T G[3][3];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) G[i][j] = v_M[9 * idx + 3 * i + j];
        G[2][2] += v_depths[idx];
        const T* rt = M + 9 * idx;
        const T gx = v_means2d[2 * idx], gy = v_means2d[2 * idx + 1];
        if (gx != 0 || gy != 0) {
            const T d = rt[6] * rt[6] + rt[7] * rt[7] - rt[8] * rt[8];
            const T f = 1 / d;
            if (mode != 2) {
                // reference: only the diagonal terms of d means2d / d M (utils.cuh:675-701)
                G[0][0] += gx * (f * rt[6]);
                G[0][1] += gx * (f * rt[7]);
                G[0][2] += gx * (-f * rt[8]);
                G[1][0] += gy * (f * rt[6]);
                G[1][1] += gy * (f * rt[7]);
                G[1][2] += gy * (-f * rt[8]);
                G[2][0] += gx * (rt[0] * (f - 2 * f * f * rt[6] * rt[6])) + gy * (rt[3] * (f - 2 * f * f * rt[6] * rt[6]));
                G[2][1] += gx * (rt[1] * (f - 2 * f * f * rt[7] * rt[7])) + gy * (rt[4] * (f - 2 * f * f * rt[7] * rt[7]));
                G[2][2] += gx * (-rt[2] * (f + 2 * f * f * rt[8] * rt[8])) + gy * (-rt[5] * (f + 2 * f * f * rt[8] * rt[8]));
            } else {
                // exact: mx = sum_i a_i M0_i M2_i / d, my = sum_i a_i M1_i M2_i / d, a = (1,1,-1)
                const T a[3] = {1, 1, -1};
                T mx = 0, my = 0;
                for (int i = 0; i < 3; ++i) { mx += a[i] * rt[i] * rt[6 + i]; my += a[i] * rt[3 + i] * rt[6 + i]; }
                mx *= f; my *= f;
                for (int i = 0; i < 3; ++i) {
                    G[0][i] += gx * a[i] * rt[6 + i] * f;
                    G[1][i] += gy * a[i] * rt[6 + i] * f;
                    G[2][i] += gx * a[i] * (rt[i] - 2 * mx * rt[6 + i]) * f + gy * a[i] * (rt[3 + i] - 2 * my * rt[6 + i]) * f;
                }
            }
        }
        // dL/dWH = K^T G  (WH columns: RS0, RS1, mean_c)
        V3<T> vWH[3];
        for (int j = 0; j < 3; ++j) vWH[j] = v3<T>(fx * G[0][j], fy * G[1][j], cx * G[0][j] + cy * G[1][j] + G[2][j]);
        V3<T> vRS[3];
        for (int j = 0; j < 3; ++j) vRS[j] = mulT(R, vWH[j]);
        const M3<T> Rq = quat_rot<T>(q);
        V3<T> vtn = mulT(R, v3<T>(v_normals[3 * idx], v_normals[3 * idx + 1], v_normals[3 * idx + 2]));
        const V3<T> tn = mul(R, Rq.c[2]);
        const T mult = dot3(T(-1) * tn, mc) > 0 ? T(1) : T(-1);
        vtn = mult * vtn;
        M3<T> gRq;
        if (mode == 1) {
            gRq.c[0] = v3<T>(vRS[0].x / s0, vRS[0].y / s0, vRS[0].z / s0);
            gRq.c[1] = v3<T>(vRS[1].x / s1, vRS[1].y / s1, vRS[1].z / s1);
        } else {
            gRq.c[0] = s0 * vRS[0];
            gRq.c[1] = s1 * vRS[1];
        }
        gRq.c[2] = vtn;
        quat_rot_vjp<T>(q, gRq, v_quats + 4 * n);
        v_scales[3 * n] += dot3(vRS[0], Rq.c[0]);
        v_scales[3 * n + 1] += dot3(vRS[1], Rq.c[1]);
        v_means[3 * n] += vRS[2].x;
        v_means[3 * n + 1] += vRS[2].y;
        v_means[3 * n + 2] += vRS[2].z;
    }
}

// ------------------------------------------------------------ intersection
inline uint32_t sat_u32(double v) {  // float -> uint32 with the GPU's saturating conversion
    if (!(v > 0)) return 0u;
    if (v >= 4294967295.0) return 4294967295u;
    return (uint32_t)v;
}

template <typename T>
inline void tile_box(T mx, T my, int32_t radius, uint32_t tile_size, uint32_t tw, uint32_t th, uint32_t& x0,
                     uint32_t& y0, uint32_t& x1, uint32_t& y1) {
    const float r = (float)radius;
    const float ts = (float)tile_size;
    // the reference computes in float (OpType of float); keep that for T=float
    const T tr = (T)r / (T)ts, tx = mx / (T)ts, ty = my / (T)ts;
    x0 = std::min(sat_u32((double)std::floor(tx - tr)), tw);
    y0 = std::min(sat_u32((double)std::floor(ty - tr)), th);
    x1 = std::min(sat_u32((double)std::ceil(tx + tr)), tw);
    y1 = std::min(sat_u32((double)std::ceil(ty + tr)), th);
}

template <typename T>
void isect_count(int64_t n_elems, const T* means2d, const int32_t* radii, uint32_t tile_size, uint32_t tw,
                 uint32_t th, int32_t* tiles_per_gauss) {
    for (int64_t i = 0; i < n_elems; ++i) {
        if (radii[i] <= 0) { tiles_per_gauss[i] = 0; continue; }
        uint32_t x0, y0, x1, y1;
        tile_box<T>(means2d[2 * i], means2d[2 * i + 1], radii[i], tile_size, tw, th, x0, y0, x1, y1);
        tiles_per_gauss[i] = (int32_t)((y1 - y0) * (x1 - x0));
    }
}

// camera_ids may be null (dense layout: camera = i / N).
template <typename T>
void isect_emit(int64_t n_elems, int64_t N, const int64_t* camera_ids, const T* means2d, const int32_t* radii,
                const float* depths, const int64_t* cum_tiles, uint32_t tile_size, uint32_t tw, uint32_t th,
                uint32_t tile_n_bits, int64_t* isect_ids, int32_t* flatten_ids) {
    for (int64_t i = 0; i < n_elems; ++i) {
        if (radii[i] <= 0) continue;
        uint32_t x0, y0, x1, y1;
        tile_box<T>(means2d[2 * i], means2d[2 * i + 1], radii[i], tile_size, tw, th, x0, y0, x1, y1);
        const int64_t cid = camera_ids ? camera_ids[i] : i / N;
        const int64_t cid_enc = cid << (32 + tile_n_bits);
        int32_t dbits;
        std::memcpy(&dbits, depths + i, 4);
        const int64_t depth_enc = (int64_t)dbits;  // sign-extended like the reference
        int64_t cur = i == 0 ? 0 : cum_tiles[i - 1];
        for (uint32_t y = y0; y < y1; ++y)
            for (uint32_t x = x0; x < x1; ++x) {
                const int64_t tile_id = (int64_t)y * tw + x;
                isect_ids[cur] = cid_enc | (tile_id << 32) | depth_enc;
                flatten_ids[cur] = (int32_t)i;
                ++cur;
            }
    }
}

// Stable ascending sort of (key, value) pairs on key bits [0, end_bit), as the
// reference's cub::DeviceRadixSort::SortPairs (isect_tiles.cu:246-300) does.
void sort_pairs(int64_t n, int64_t* keys, int32_t* vals, int end_bit) {
    const uint64_t mask = end_bit >= 64 ? ~0ull : ((1ull << end_bit) - 1ull);
    std::vector<int64_t> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) {
        return ((uint64_t)keys[a] & mask) < ((uint64_t)keys[b] & mask);
    });
    std::vector<int64_t> k2(n);
    std::vector<int32_t> v2(n);
    for (int64_t i = 0; i < n; ++i) { k2[i] = keys[order[i]]; v2[i] = vals[order[i]]; }
    std::memcpy(keys, k2.data(), n * 8);
    std::memcpy(vals, v2.data(), n * 4);
}

// offsets[t] = first sorted isect whose (camera, tile) index is >= t; the
// result the reference's boundary-filling kernel produces (isect_tiles.cu:309-355).
void offset_encode(int64_t n, const int64_t* keys, int C, int n_tiles, int tile_n_bits, int32_t* offsets) {
    const int64_t total = (int64_t)C * n_tiles;
    int64_t j = 0;
    for (int64_t t = 0; t < total; ++t) {
        while (j < n) {
            const int64_t hi = keys[j] >> 32;
            const int64_t id = (hi >> tile_n_bits) * n_tiles + (hi & ((1ll << tile_n_bits) - 1));
            if (id >= t) break;
            ++j;
        }
        offsets[t] = (int32_t)j;
    }
}

// ------------------------------------------------------------ compositor
template <typename T>
inline int bilinear_taps(T sx, T sy, int rx, int ry, T range_x, T range_y, int (&uc)[4], int (&vc)[4], T (&w)[4]) {
    if (sx < -range_x || sx > range_x || sy < -range_y || sy > range_y) return -1;
    T u = (sx + range_x) / (range_x * 2) * (rx - 1);
    T v = (sy + range_y) / (range_y * 2) * (ry - 1);
    if (u < 0) u = 0; else if (u > rx - 1) u = (T)(rx - 1);
    if (v < 0) v = 0; else if (v > ry - 1) v = (T)(ry - 1);
    const int ul = (int)std::floor(u), vl = (int)std::floor(v), uh = (int)std::ceil(u), vh = (int)std::ceil(v);
    uc[0] = ul; uc[1] = uh; uc[2] = ul; uc[3] = uh;
    vc[0] = vl; vc[1] = vl; vc[2] = vh; vc[3] = vh;
    const T wu = u - (T)ul, wv = v - (T)vl;
    w[0] = (T(1) - wu) * (T(1) - wv);
    w[1] = wu * (T(1) - wv);
    w[2] = (T(1) - wu) * wv;
    w[3] = wu * wv;
    return 1;
}

template <typename T> struct RasterIn {
    int C, N, D, W, H, tile_size, tile_w, tile_h;
    int64_t n_isects;
    const T* means2d;      // [E,2]  (E = C*N dense or nnz packed)
    const T* M;            // [E,9]
    const T* colors;       // [E,D]
    const T* opacities;    // [E]
    const T* normals;      // [E,3]
    const T* textures;     // [G,ry,rx,4] or null for the plain compositor
    int tex_ry, tex_rx;
    T range_x, range_y;
    const T* backgrounds;  // [C,D] or null
    const uint8_t* masks;  // [C,tile_h,tile_w] or null
    const int32_t* offsets;
    const int32_t* flatten_ids;
    const int64_t* gaussian_ids;  // packed: [nnz] texture row of each element, else null (row = e % N)
    T contrib_threshold, g_weight;
    int mip_L;  // 0: bilinear on [G,ry,rx,4]; L > 0: mipmapped2 on the full pyramid [G,(4^(L+1)-1)/3,4]
    int aniso;  // 1: anisotropic_bilinear on [G,ry,rx,4]
};

template <typename T> inline int64_t tex_row(const RasterIn<T>& a, int64_t e) {
    return a.gaussian_ids ? a.gaussian_ids[e] : e % a.N;
}

// texels per splat row of the texture array
template <typename T> inline int64_t tex_texels(const RasterIn<T>& a) {
    return a.mip_L > 0 ? ((int64_t(1) << (2 * (a.mip_L + 1))) - 1) / 3 : (int64_t)a.tex_ry * a.tex_rx;
}

// mipmapped2 taps, restating filters/mip2.cuh:27-105 (pyramid coordinate of level t of a 2^L texture:
// (4^(L-t) - 1) / 3, coarsest first); a level beyond the coarsest is treated as invalid.
template <typename T>
inline int mip2_taps(T sx, T sy, T dxx, T dxy, T dyx, T dyy, int R, int L, T xr, T yr, int64_t (&mc)[8], T (&w)[8]) {
    const T fr = T(R - 1);
    const T ax = dxx / (xr * 2) * fr, ay = dxy / (xr * 2) * fr;
    const T bx = dyx / (yr * 2) * fr, by = dyy / (yr * 2) * fr;
    const T duv = std::max(std::sqrt(ax * ax + ay * ay), std::sqrt(bx * bx + by * by));
    T t = std::log2(duv);
    if (t < 0) t = 0;
    else if (t > 31) t = 31;
    const T u = (sx + xr) / (xr * 2) * fr, v = (sy + yr) / (yr * 2) * fr;
    // a NaN level converts to level 0 (the GPU's float -> int conversion); its weights stay NaN
    const int tl = t == t ? (int)std::floor(t) : 0, th = t == t ? (int)std::ceil(t) : 0;
    if (th > L) return -1;
    const T sl = T(1u << tl), sh = T(1u << th);
    const T us = (u + T(0.5)) / sl - T(0.5), ug = (u + T(0.5)) / sh - T(0.5);
    const T vs = (v + T(0.5)) / sl - T(0.5), vg = (v + T(0.5)) / sh - T(0.5);
    const int uls = (int)std::floor(us), ulg = (int)std::floor(ug), vls = (int)std::floor(vs), vlg = (int)std::floor(vg);
    const int uhs = (int)std::ceil(us), uhg = (int)std::ceil(ug), vhs = (int)std::ceil(vs), vhg = (int)std::ceil(vg);
    if (uls < 0 || ulg < 0 || vls < 0 || vlg < 0 || uhs > ((R - 1) >> tl) || uhg > ((R - 1) >> th) ||
        vhs > ((R - 1) >> tl) || vhg > ((R - 1) >> th))
        return -1;
    const int64_t rl = R >> tl, rh = R >> th;
    const int64_t bl = ((int64_t(1) << (2 * (L - tl))) - 1) / 3, bh = ((int64_t(1) << (2 * (L - th))) - 1) / 3;
    mc[0] = bl + vls * rl + uls; mc[1] = bl + vls * rl + uhs; mc[2] = bl + vhs * rl + uls; mc[3] = bl + vhs * rl + uhs;
    mc[4] = bh + vlg * rh + ulg; mc[5] = bh + vlg * rh + uhg; mc[6] = bh + vhg * rh + ulg; mc[7] = bh + vhg * rh + uhg;
    const T wus = us - T(uls), wvs = vs - T(vls), wug = ug - T(ulg), wvg = vg - T(vlg), wt = t - T(tl);
    w[0] = (1 - wus) * (1 - wvs) * (1 - wt); w[1] = wus * (1 - wvs) * (1 - wt);
    w[2] = (1 - wus) * wvs * (1 - wt);       w[3] = wus * wvs * (1 - wt);
    w[4] = (1 - wug) * (1 - wvg) * wt;       w[5] = wug * (1 - wvg) * wt;
    w[6] = (1 - wug) * wvg * wt;             w[7] = wug * wvg * wt;
    return 1;
}

template <typename T> struct SplatEval {
    bool valid;
    int valid_tex;
    int uc[4], vc[4];  // bilinear texel coordinates
    int nt;            // taps: 4 bilinear, 8 mipmapped2, 4 per footprint cell for anisotropic_bilinear
    int64_t ti[8];     // texel index of each tap within the splat's row (fixed-size filters)
    T w[8];
    bool dyn = false;  // anisotropic_bilinear: taps in ati / aw
    std::vector<int64_t> ati;
    std::vector<T> aw;
    T area;  // anisotropic_bilinear: footprint area in texels
    T asf, g3, g2, kern, vis, alpha;
    V3<T> hu, hv, zeta;
    T sx, sy, dx, dy;
    int64_t tap(int t) const { return dyn ? ati[t] : ti[t]; }
    T wt(int t) const { return dyn ? aw[t] : w[t]; }
};

// ---------------------------------------------------------------- anisotropic_bilinear
// Restates filters/anisotropic_bilinear.cuh:15-235: the pixel's footprint quad
// in texel coordinates, clipped (Sutherland-Hodgman) against every texel cell
// [u, u+1] x [v, v+1] it overlaps; the moments of each clipped polygon weight
// the cell's four texels (the exact integral of the bilinear interpolant), and
// the sum is divided by the quad's area.
template <typename T> struct V2 { T x, y; };
template <typename T> inline V2<T> v2sub(V2<T> a, V2<T> b) { return {a.x - b.x, a.y - b.y}; }
template <typename T> inline T v2cross(V2<T> a, V2<T> b) { return a.x * b.y - a.y * b.x; }
template <typename T> inline T v2dot(V2<T> a, V2<T> b) { return a.x * b.x + a.y * b.y; }

// float -> int as the GPU converts: NaN -> 0, saturating at the int range
template <typename T> inline int sat_int(T x) {
    if (x != x) return 0;
    if (x >= T(2147483647.0)) return 2147483647;
    if (x <= T(-2147483648.0)) return -2147483647 - 1;
    return (int)x;
}

template <typename T> struct AnisoFoot {
    V2<T> s[4], n[4];
    T nmax[4];
    int minu, maxu, minv, maxv;
};

template <typename T> inline void aniso_edge_normal(V2<T> s0, V2<T> e, V2<T> c, V2<T>& n) {
    if (e.x == 0 && e.y == 0) n = v2sub(s0, c);
    else n = {e.y, -e.x};
    const T l = std::sqrt(n.x * n.x + n.y * n.y);
    if (l == 0) return;  // left as is (the reference ignores this status)
    n.x /= l;
    n.y /= l;
}

// Orientation, texel bounds, edge normals; returns the area (precompute, :193-245).
template <typename T> inline T aniso_setup(AnisoFoot<T>& F, int rx, int ry) {
    V2<T> e01 = v2sub(F.s[1], F.s[0]), e12 = v2sub(F.s[2], F.s[1]), e23 = v2sub(F.s[3], F.s[2]),
          e30 = v2sub(F.s[0], F.s[3]);
    T area = T(0.5) * (v2cross(e01, e12) + v2cross(e23, e30));
    if (area < 0) {
        area *= -1;
        std::swap(F.s[1], F.s[3]);
        e01 = v2sub(F.s[1], F.s[0]); e12 = v2sub(F.s[2], F.s[1]);
        e23 = v2sub(F.s[3], F.s[2]); e30 = v2sub(F.s[0], F.s[3]);
    }
    const V2<T>* s = F.s;
    F.minu = std::max(0, sat_int(std::floor(std::min(std::min(s[0].x, s[1].x), std::min(s[2].x, s[3].x)))));
    F.maxu = std::min(rx - 1, sat_int(std::ceil(std::max(std::max(s[0].x, s[1].x), std::max(s[2].x, s[3].x)))));
    F.minv = std::max(0, sat_int(std::floor(std::min(std::min(s[0].y, s[1].y), std::min(s[2].y, s[3].y)))));
    F.maxv = std::min(ry - 1, sat_int(std::ceil(std::max(std::max(s[0].y, s[1].y), std::max(s[2].y, s[3].y)))));
    const V2<T> c = {(((s[0].x + s[1].x) + s[2].x) + s[3].x) / T(4), (((s[0].y + s[1].y) + s[2].y) + s[3].y) / T(4)};
    aniso_edge_normal(s[0], e01, c, F.n[0]);
    aniso_edge_normal(s[1], e12, c, F.n[1]);
    aniso_edge_normal(s[2], e23, c, F.n[2]);
    aniso_edge_normal(s[3], e30, c, F.n[3]);
    for (int i = 0; i < 4; ++i)
        F.nmax[i] = std::max(std::abs(F.n[i].x * T(0.5) + F.n[i].y * T(0.5)),
                             std::abs(F.n[i].x * T(0.5) + F.n[i].y * T(-0.5)));
    return area;
}

// Moments (A, Sx, Sy, Sxy) of the quad clipped to cell (u, v), in cell-local
// coordinates (clip_and_compute_moments, :58-190); false if fewer than 3
// vertices remain.  A clip that would overflow 8 vertices (only a
// self-intersecting quad can) also returns false.
template <typename T> inline bool aniso_cell(const AnisoFoot<T>& F, int u, int v, T& A, T& Sx, T& Sy, T& Sxy) {
    const V2<T> sc = {T(u) + T(0.5), T(v) + T(0.5)};
    if (v2dot(v2sub(F.s[0], sc), F.n[0]) >= F.nmax[0] && v2dot(v2sub(F.s[1], sc), F.n[1]) >= F.nmax[1] &&
        v2dot(v2sub(F.s[2], sc), F.n[2]) >= F.nmax[2] && v2dot(v2sub(F.s[3], sc), F.n[3]) >= F.nmax[3]) {
        A = T(1); Sx = T(0.5); Sy = T(0.5); Sxy = T(0.25);
        return true;
    }
    V2<T> p[8], q[8];
    int n = 4;
    for (int i = 0; i < 4; ++i) p[i] = {F.s[i].x - T(u), F.s[i].y - T(v)};
    // one half-plane: axis 0 = x, 1 = y; keep coordinate >= 0 (hi = false) or <= 1 (hi = true)
    auto clip = [&](const V2<T>* in, V2<T>* out, int axis, bool hi) -> int {
        int m = 0;
        for (int i = 0; i < n; ++i) {
            const V2<T> a = in[i], b = in[(i + 1) % n];
            const T ac = axis ? a.y : a.x, bc = axis ? b.y : b.x;
            const bool ain = hi ? ac <= T(1) : ac >= T(0), bin = hi ? bc <= T(1) : bc >= T(0);
            if (ain) {
                if (m == 8) return -1;
                out[m++] = a;
            }
            if (ain != bin) {
                if (m == 8) return -1;
                const T t = hi ? (ac - T(1)) / (ac - bc) : ac / (ac - bc);
                out[m++] = axis ? V2<T>{a.x + t * (b.x - a.x), hi ? T(1) : T(0)}
                                : V2<T>{hi ? T(1) : T(0), a.y + t * (b.y - a.y)};
            }
        }
        return m;
    };
    if ((n = clip(p, q, 0, false)) < 3) return false;
    if ((n = clip(q, p, 0, true)) < 3) return false;
    if ((n = clip(p, q, 1, false)) < 3) return false;
    if ((n = clip(q, p, 1, true)) < 3) return false;
    A = Sx = Sy = Sxy = T(0);
    for (int i = 0; i < n; ++i) {
        const V2<T> a = p[i], b = p[(i + 1) % n];
        const T c = v2cross(a, b);
        A += c;
        Sx += c * (a.x + b.x);
        Sy += c * (a.y + b.y);
        Sxy += c * (T(2) * a.x * a.y + a.x * b.y + b.x * a.y + T(2) * b.x * b.y);
    }
    A *= T(0.5);
    Sx *= T(1) / T(6);
    Sy *= T(1) / T(6);
    Sxy *= T(1) / T(24);
    return true;
}

// Per (pixel, splat) evaluation shared by forward and backward, as the
// reference recomputes it (fwd.cu:283-347, bwd.cu:338-397).
template <typename T>
inline void eval_splat(const RasterIn<T>& a, int64_t g, T px, T py, SplatEval<T>& e) {
    const T* m = a.M + 9 * g;
    const V3<T> M0 = v3<T>(m[0], m[1], m[2]), M1 = v3<T>(m[3], m[4], m[5]), M2 = v3<T>(m[6], m[7], m[8]);
    e.hu = px * M2 - M0;
    e.hv = py * M2 - M1;
    e.zeta = cross3(e.hu, e.hv);
    e.valid = true;
    e.valid_tex = -1;
    e.nt = 4;
    if (e.zeta.z == T(0)) { e.valid = false; return; }
    e.sx = e.zeta.x / e.zeta.z;
    e.sy = e.zeta.y / e.zeta.z;
    const T opac = a.opacities[g];
    if (a.textures && a.aniso) {
        // anisotropic_bilinear (aniso_bilinear fwd.cu:296-340): s at the pixel's four corners
        const V3<T> dxw = cross3(e.hu, M2), dyw = cross3(e.hv, M2);
        const V3<T> hx = T(0.5) * dxw, hy = T(0.5) * dyw;
        const V3<T> cr[4] = {(e.zeta - hx) - hy, (e.zeta + hx) - hy, (e.zeta + hx) + hy, (e.zeta - hx) + hy};
        if (cr[0].z == T(0) || cr[1].z == T(0) || cr[2].z == T(0) || cr[3].z == T(0)) {
            e.valid = false;
            e.g3 = e.g2 = T(0);
            return;
        }
        AnisoFoot<T> F;
        for (int i = 0; i < 4; ++i)
            F.s[i] = {(cr[i].x / cr[i].z + a.range_x) / (a.range_x * 2) * T(a.tex_rx - 1),
                      (cr[i].y / cr[i].z + a.range_y) / (a.range_y * 2) * T(a.tex_ry - 1)};
        e.area = aniso_setup(F, a.tex_rx, a.tex_ry);
        e.dyn = true;
        e.nt = 0;
        e.valid_tex = (e.area == T(0) || F.minu == F.maxu || F.minv == F.maxv) ? 0 : 1;
        if (e.valid_tex > 0) {
            const T ia = T(1) / e.area;
            for (int v = F.minv; v < F.maxv; ++v)
                for (int u = F.minu; u < F.maxu; ++u) {
                    T A, Sx, Sy, Sxy;
                    if (!aniso_cell(F, u, v, A, Sx, Sy, Sxy)) continue;
                    const int64_t t00 = (int64_t)v * a.tex_rx + u;
                    const int64_t tq[4] = {t00, t00 + 1, t00 + a.tex_rx, t00 + a.tex_rx + 1};
                    const T wq[4] = {((A - Sx) - Sy) + Sxy, Sx - Sxy, Sy - Sxy, Sxy};
                    for (int q = 0; q < 4; ++q) {
                        e.ati.push_back(tq[q]);
                        e.aw.push_back(wq[q] * ia);
                    }
                }
            e.nt = (int)e.ati.size();
        }
    } else if (a.textures && a.mip_L > 0) {
        // mipmapped2 (mip2 fwd.cu:293-347): s at the pixel's edge midpoints gives the footprint
        const V3<T> hw = T(0.5) * M2;
        const V3<T> cx0 = cross3(e.hu - hw, e.hv), cx1 = cross3(e.hu + hw, e.hv);
        const V3<T> cy0 = cross3(e.hu, e.hv - hw), cy1 = cross3(e.hu, e.hv + hw);
        if (cx0.z == T(0) || cx1.z == T(0) || cy0.z == T(0) || cy1.z == T(0)) {
            e.valid = false;
            e.g3 = e.g2 = T(0);
            return;
        }
        e.nt = 8;
        e.valid_tex = mip2_taps<T>(e.sx, e.sy, cx1.x / cx1.z - cx0.x / cx0.z, cx1.y / cx1.z - cx0.y / cx0.z,
                                   cy1.x / cy1.z - cy0.x / cy0.z, cy1.y / cy1.z - cy0.y / cy0.z, a.tex_rx, a.mip_L,
                                   a.range_x, a.range_y, e.ti, e.w);
    } else if (a.textures) {
        T w4[4];
        e.valid_tex = bilinear_taps<T>(e.sx, e.sy, a.tex_rx, a.tex_ry, a.range_x, a.range_y, e.uc, e.vc, w4);
        for (int i = 0; i < 4; ++i) {
            e.w[i] = w4[i];
            e.ti[i] = (int64_t)e.vc[i] * a.tex_rx + e.uc[i];
        }
    }
    if (a.textures) {
        if (e.valid_tex > 0) {
            const T* tex = a.textures + tex_row(a, g) * tex_texels(a) * 4;
            e.asf = 0;
            for (int i = 0; i < e.nt; ++i) e.asf += e.wt(i) * tex[e.tap(i) * 4 + 3];
        } else {
            e.asf = a.aniso ? T(0) : T(1);  // anisotropic_bilinear zeroes alpha without a texture sample
        }
    } else {
        e.asf = 1;
    }
    e.g3 = e.sx * e.sx + e.sy * e.sy;
    e.dx = a.means2d[2 * g] - px;
    e.dy = a.means2d[2 * g + 1] - py;
    e.g2 = T(2) * (e.dx * e.dx + e.dy * e.dy);
    const T sigma = T(0.5) * std::min(e.g3, e.g2);
    e.kern = std::exp(-sigma);
    if (a.textures) {
        e.vis = T(0.998) - a.g_weight + a.g_weight * e.kern;
        e.alpha = std::min(T(0.999), opac * e.vis * e.asf);
    } else {
        e.vis = e.kern;
        e.alpha = std::min(T(0.999), opac * e.vis);
    }
    if (sigma < T(0) || e.alpha < T(1) / T(255)) e.valid = false;
    // anisotropic_bilinear tests the untextured alpha first (aniso_bilinear fwd.cu:358-366); the adjoint follows
    // the forward's tests, so the pairs it revisits are the ones the forward composited
    if (a.textures && a.aniso && opac * e.vis < T(1) / T(255)) e.valid = false;
}

template <typename T> inline T tex_channel(const RasterIn<T>& a, int64_t g, const SplatEval<T>& e, int k) {
    // texture channel k for colour channel k; channels >= 4 have no texture term
    if (k >= 4 || e.valid_tex <= 0) return T(0);
    const T* tex = a.textures + tex_row(a, g) * tex_texels(a) * 4;
    T s = 0;
    for (int i = 0; i < e.nt; ++i) s += e.wt(i) * tex[e.tap(i) * 4 + k];
    return s;
}

template <typename T> struct RasterOut {
    T* colors;      // [C,H,W,D]
    T* alphas;      // [C,H,W]
    T* normals;     // [C,H,W,3]
    T* distort;     // [C,H,W]
    T* median;      // [C,H,W]
    int32_t* last_ids;
    int32_t* median_ids;
    T* contrib_sum;    // [N or G]
    T* contrib_count;  // [N or G]
};

template <typename T> inline void tile_range(const RasterIn<T>& a, int c, int tile, int64_t& s, int64_t& e) {
    const int T_ = a.tile_w * a.tile_h;
    s = a.offsets[(int64_t)c * T_ + tile];
    e = (c == a.C - 1 && tile == T_ - 1) ? a.n_isects : a.offsets[(int64_t)c * T_ + tile + 1];
}

template <typename T>
void raster_fwd(const RasterIn<T>& a, const RasterOut<T>& o, int32_t* pair_count /* optional, [C,H,W] */,
                uint64_t* branch_sig /* optional, [C,H,W] */) {
    const int T_ = a.tile_w * a.tile_h;
    const int D = a.D;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t ct = 0; ct < (int64_t)a.C * T_; ++ct) {
        const int c = (int)(ct / T_), tile = (int)(ct % T_);
        const int ty = tile / a.tile_w, tx = tile % a.tile_w;
        int64_t rs, re;
        tile_range(a, c, tile, rs, re);
        std::vector<T> pix(D);
        for (int dy = 0; dy < a.tile_size; ++dy)
            for (int dx = 0; dx < a.tile_size; ++dx) {
                const int i = ty * a.tile_size + dy, j = tx * a.tile_size + dx;
                if (i >= a.H || j >= a.W) continue;
                const int64_t pid = ((int64_t)c * a.H + i) * a.W + j;
                if (a.masks && !a.masks[ct]) {
                    for (int k = 0; k < D; ++k) o.colors[pid * D + k] = a.backgrounds ? a.backgrounds[c * D + k] : T(0);
                    o.alphas[pid] = 0;
                    for (int k = 0; k < 3; ++k) o.normals[pid * 3 + k] = 0;
                    o.distort[pid] = 0; o.median[pid] = 0; o.last_ids[pid] = 0; o.median_ids[pid] = 0;
                    if (pair_count) pair_count[pid] = 0;
                    if (branch_sig) branch_sig[pid] = 0;
                    continue;
                }
                const T px = (T)j + T(0.5), py = (T)i + T(0.5);
                T Tr = 1, distort = 0, accum = 0, med = 0;
                int64_t cur = 0, med_idx = 0;
                int32_t pairs = 0;
                uint64_t sig = 1469598103934665603ull;  // FNV-1a over every discrete decision
                auto mix = [&](uint64_t v) { sig = (sig ^ v) * 1099511628211ull; };
                T nrm[3] = {0, 0, 0};
                std::fill(pix.begin(), pix.end(), T(0));
                for (int64_t idx = rs; idx < re; ++idx) {
                    const int64_t g = a.flatten_ids[idx];
                    SplatEval<T> e;
                    eval_splat(a, g, px, py, e);
                    if (branch_sig) {
                        mix((uint64_t)g);
                        mix(e.valid ? 1 : 0);
                        if (e.zeta.z != T(0)) {
                            mix(e.g3 <= e.g2 ? 3 : 4);
                            mix((uint64_t)(e.valid_tex + 2));
                            if (e.valid_tex > 0)
                                for (int q = 0; q < e.nt; ++q) mix((uint64_t)e.tap(q));
                            const T op = a.opacities[g];
                            mix(a.textures ? (op * e.vis * e.asf <= T(0.999) ? 5 : 6) : (op * e.vis <= T(0.999) ? 5 : 6));
                        }
                    }
                    if (!e.valid) continue;
                    const T next_T = Tr * (T(1) - e.alpha);
                    if (next_T <= T(1e-4)) break;
                    const T vis = e.alpha * Tr;
                    const T* cp = a.colors + g * D;
                    for (int k = 0; k < D; ++k) pix[k] += (cp[k] + tex_channel(a, g, e, k)) * vis;
                    for (int k = 0; k < 3; ++k) nrm[k] += a.normals[3 * g + k] * vis;
                    const T depth = cp[D - 1];
                    distort += T(2) * (vis * depth * (T(1) - Tr) - vis * accum);
                    accum += vis * depth;
                    if (Tr > T(0.5)) { med = depth; med_idx = idx; }
                    cur = idx;
                    Tr = next_T;
                    ++pairs;
                    if (e.alpha > a.contrib_threshold) {
                        const int64_t row = tex_row(a, g);
#pragma omp atomic
                        o.contrib_sum[row] += e.alpha;
#pragma omp atomic
                        o.contrib_count[row] += T(1);
                    }
                }
                o.alphas[pid] = T(1) - Tr;
                for (int k = 0; k < D; ++k) o.colors[pid * D + k] = a.backgrounds ? pix[k] + Tr * a.backgrounds[c * D + k] : pix[k];
                for (int k = 0; k < 3; ++k) o.normals[pid * 3 + k] = nrm[k];
                o.last_ids[pid] = (int32_t)cur;
                o.distort[pid] = distort;
                o.median[pid] = med;
                o.median_ids[pid] = (int32_t)med_idx;
                if (pair_count) pair_count[pid] = pairs;
                if (branch_sig) branch_sig[pid] = sig ^ (uint64_t)(T(0.5) < Tr);
            }
    }
}

template <typename T> struct RasterGradIn {
    const T* colors;   // forward outputs [C,H,W,D]
    const T* alphas;   // [C,H,W]
    const int32_t* last_ids;
    const int32_t* median_ids;
    const T* v_colors;   // [C,H,W,D]
    const T* v_alphas;   // [C,H,W]
    const T* v_normals;  // [C,H,W,3]
    const T* v_distort;  // [C,H,W]
    const T* v_median;   // [C,H,W]
};

template <typename T> struct RasterGradOut {
    T* v_means2d;      // [E,2]
    T* v_means2d_abs;  // [E,2] or null
    T* v_M;            // [E,9]
    T* v_colors;       // [E,D]
    T* v_opacities;    // [E]
    T* v_normals;      // [E,3]
    T* v_textures;     // [G,ry,rx,4] or null
    T* v_densify;      // [E,2]
};

template <typename T> inline void atomic_add(T* p, T v) {
#pragma omp atomic
    *p += v;
}

// mode: 0 = reference "bilinear" adjoint, 1 = reference "bilinear_bwd2"
//       adjoint, 2 = exact derivative of the forward; plus kRecomputeT (16):
//       the transmittance in front of each splat is the front-to-back product
//       recomputed per pixel, instead of the reference's back-to-front division
//       of the final transmittance by (1 - alpha)
//       (rasterize_to_pixels_textured_gaussians_2dgs_bwd.cu:160, :456-457).
constexpr int kRecomputeT = 16;
template <typename T>
void raster_bwd(const RasterIn<T>& a, const RasterGradIn<T>& gi, const RasterGradOut<T>& go, int mode, int64_t E) {
    const bool recompute = (mode & kRecomputeT) != 0;
    mode &= ~kRecomputeT;
    const int T_ = a.tile_w * a.tile_h;
    const int D = a.D;
    std::vector<uint8_t> touched(E, 0);
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t ct = 0; ct < (int64_t)a.C * T_; ++ct) {
        const int c = (int)(ct / T_), tile = (int)(ct % T_);
        if (a.masks && !a.masks[ct]) continue;
        const int ty = tile / a.tile_w, tx = tile % a.tile_w;
        int64_t rs, re;
        tile_range(a, c, tile, rs, re);
        std::vector<T> buf(D), vrgb(D), texc(D), t_before;
        for (int dy = 0; dy < a.tile_size; ++dy)
            for (int dx = 0; dx < a.tile_size; ++dx) {
                const int i = ty * a.tile_size + dy, j = tx * a.tile_size + dx;
                if (i >= a.H || j >= a.W) continue;
                const int64_t pid = ((int64_t)c * a.H + i) * a.W + j;
                const T px = (T)j + T(0.5), py = (T)i + T(0.5);
                const T T_final = T(1) - gi.alphas[pid];
                T Tr = T_final;
                std::fill(buf.begin(), buf.end(), T(0));
                T bufn[3] = {0, 0, 0};
                const int64_t bin_final = gi.last_ids[pid];
                const int64_t med_idx = gi.median_ids[pid];
                const T* vc = gi.v_colors + pid * D;
                const T va = gi.v_alphas[pid];
                const T* vn = gi.v_normals + pid * 3;
                const T vdist = gi.v_distort[pid];
                T acc_d_buf = gi.colors[pid * D + D - 1], acc_d = acc_d_buf;
                T acc_w_buf = gi.alphas[pid], acc_w = acc_w_buf;
                T dist_buf = 0;
                const T vmed = gi.v_median[pid];
                if (recompute) {  // T in front of every splat of the pixel's list, front to back
                    const int64_t last = std::min<int64_t>(bin_final, re - 1);
                    t_before.assign(std::max<int64_t>(last - rs + 1, 0), T(1));
                    T tf = T(1);
                    for (int64_t idx = rs; idx <= last; ++idx) {
                        t_before[idx - rs] = tf;
                        SplatEval<T> e;
                        eval_splat(a, a.flatten_ids[idx], px, py, e);
                        if (e.valid) tf *= T(1) - e.alpha;
                    }
                }
                for (int64_t idx = std::min<int64_t>(bin_final, re - 1); idx >= rs; --idx) {
                    const int64_t g = a.flatten_ids[idx];
                    SplatEval<T> e;
                    eval_splat(a, g, px, py, e);
                    if (!e.valid) continue;
                    const T opac = a.opacities[g];
                    const T* cp = a.colors + g * D;
                    std::fill(vrgb.begin(), vrgb.end(), T(0));
                    if (idx == med_idx) vrgb[D - 1] += vmed;
                    const T ra = T(1) / (T(1) - e.alpha);
                    Tr = recompute ? t_before[idx - rs] : Tr * ra;
                    const T fac = e.alpha * Tr;
                    const bool tex_on = a.textures && e.valid_tex > 0;
                    T* vtex = tex_on ? go.v_textures + tex_row(a, g) * tex_texels(a) * 4 : nullptr;
                    const T* tex = tex_on ? a.textures + tex_row(a, g) * tex_texels(a) * 4 : nullptr;
                    for (int k = 0; k < D; ++k) {
                        vrgb[k] += fac * vc[k];
                        texc[k] = 0;
                        if (tex_on && k < 4)
                            for (int t = 0; t < e.nt; ++t) {
                                const int64_t o = e.tap(t) * 4 + k;
                                atomic_add(vtex + o, fac * e.wt(t) * vc[k]);
                                texc[k] += e.wt(t) * tex[o];
                            }
                        // anisotropic_bilinear's adjoint uses the texture colour without the division by the
                        // footprint area (aniso_bilinear bwd.cu:499-522 with filters/anisotropic_bilinear.cuh:372-389)
                        if (a.aniso) texc[k] *= e.area;
                    }
                    T v_alpha = 0;
                    for (int k = 0; k < D; ++k) v_alpha += ((texc[k] + cp[k]) * Tr - buf[k] * ra) * vc[k];
                    T vnl[3];
                    for (int k = 0; k < 3; ++k) vnl[k] = fac * vn[k];
                    for (int k = 0; k < 3; ++k) v_alpha += (a.normals[3 * g + k] * Tr - bufn[k] * ra) * vn[k];
                    v_alpha += T_final * ra * va;
                    if (a.backgrounds) {
                        T accb = 0;
                        for (int k = 0; k < D; ++k) accb += a.backgrounds[c * D + k] * vc[k];
                        v_alpha += -T_final * ra * accb;
                    }
                    {
                        const T depth = cp[D - 1];
                        const T dl_dw = T(2) * (T(2) * (depth * acc_w_buf - acc_d_buf) + (acc_d - depth * acc_w));
                        v_alpha += (dl_dw * Tr - dist_buf * ra) * vdist;
                        acc_d_buf -= fac * depth;
                        acc_w_buf -= fac;
                        dist_buf += dl_dw * fac;
                        vrgb[D - 1] += T(2) * fac * (T(2) - T(2) * Tr - acc_w + fac) * vdist;
                    }
                    V3<T> vM0 = v3<T>(0, 0, 0), vM1 = v3<T>(0, 0, 0), vM2 = v3<T>(0, 0, 0);
                    T vx = 0, vy = 0, v_op = 0;
                    const bool unclamped = a.textures ? (opac * e.vis * e.asf <= T(0.999)) : (opac * e.vis <= T(0.999));
                    auto back_s = [&](T vsx, T vsy) {
                        const T a_ = vsx / e.zeta.z, b_ = vsy / e.zeta.z;
                        const V3<T> vz = v3<T>(a_, b_, -(a_ * e.sx + b_ * e.sy));
                        const V3<T> vhu = cross3(e.hv, vz);
                        const V3<T> vhv = cross3(vz, e.hu);
                        vM0 = vM0 - vhu;
                        vM1 = vM1 - vhv;
                        vM2 = vM2 + (px * vhu + py * vhv);
                    };
                    if (unclamped) {
                        const T vG = a.textures ? opac * v_alpha * e.asf : opac * v_alpha;
                        const T dGk = a.textures ? -a.g_weight * e.kern : -e.vis;  // dG/dsigma
                        if (e.g3 <= e.g2) {
                            back_s(vG * dGk * e.sx, vG * dGk * e.sy);
                        } else {
                            const T ddx = dGk * T(2) * e.dx, ddy = dGk * T(2) * e.dy;
                            vx = vG * ddx;
                            vy = vG * ddy;
                        }
                        v_op = a.textures ? e.vis * v_alpha * e.asf : e.vis * v_alpha;
                        if (tex_on)
                            for (int t = 0; t < e.nt; ++t) atomic_add(vtex + e.tap(t) * 4 + 3, e.wt(t) * e.vis * opac * v_alpha);
                    }
                    if (mode >= 1 && tex_on && a.mip_L == 0 && !a.aniso) {
                        const T wu = e.w[1] + e.w[3], wv = e.w[2] + e.w[3];
                        const T dbu[4] = {-(T(1) - wv), T(1) - wv, -wv, wv};
                        const T dbv[4] = {-(T(1) - wu), -wu, T(1) - wu, wu};
                        const T scale = mode == 1 ? T(1) : T(0.5);
                        const T du = scale * T(a.tex_rx - 1) / a.range_x;
                        const T dv = scale * T(a.tex_ry - 1) / a.range_y;
                        T tsx = 0, tsy = 0;
                        for (int k = 0; k < D && k < 4; ++k) {
                            const T vt = fac * vc[k];
                            for (int t = 0; t < 4; ++t) {
                                const T tv = tex[((int64_t)e.vc[t] * a.tex_rx + e.uc[t]) * 4 + k];
                                tsx += vt * dbu[t] * tv * du;
                                tsy += vt * dbv[t] * tv * dv;
                            }
                        }
                        if (unclamped) {
                            const T vasf = e.vis * opac * v_alpha;
                            for (int t = 0; t < 4; ++t) {
                                const T tv = tex[((int64_t)e.vc[t] * a.tex_rx + e.uc[t]) * 4 + 3];
                                tsx += vasf * dbu[t] * tv * du;
                                tsy += vasf * dbv[t] * tv * dv;
                            }
                        }
                        back_s(tsx, tsy);
                    }
                    for (int k = 0; k < D; ++k) buf[k] += (texc[k] + cp[k]) * fac;
                    for (int k = 0; k < 3; ++k) bufn[k] += a.normals[3 * g + k] * fac;
                    for (int k = 0; k < D; ++k) atomic_add(go.v_colors + g * D + k, vrgb[k]);
                    for (int k = 0; k < 3; ++k) atomic_add(go.v_normals + g * 3 + k, vnl[k]);
                    const T vm[9] = {vM0.x, vM0.y, vM0.z, vM1.x, vM1.y, vM1.z, vM2.x, vM2.y, vM2.z};
                    for (int k = 0; k < 9; ++k) atomic_add(go.v_M + g * 9 + k, vm[k]);
                    atomic_add(go.v_means2d + g * 2, vx);
                    atomic_add(go.v_means2d + g * 2 + 1, vy);
                    if (go.v_means2d_abs) {
                        atomic_add(go.v_means2d_abs + g * 2, std::abs(vx));
                        atomic_add(go.v_means2d_abs + g * 2 + 1, std::abs(vy));
                    }
                    atomic_add(go.v_opacities + g, v_op);
                    touched[g] = 1;
                }
            }
    }
    // densification gradient, taken after every contribution is in (the
    // reference reads it while other warps still accumulate: bwd.cu:692-699)
    for (int64_t g = 0; g < E; ++g) {
        if (!touched[g]) continue;
        go.v_densify[2 * g] = go.v_M[9 * g + 2] * a.M[9 * g + 8];
        go.v_densify[2 * g + 1] = go.v_M[9 * g + 5] * a.M[9 * g + 8];
    }
}

// ------------------------------------------------------------ spherical harmonics
// Forward-mode dual numbers give d(basis)/d(dir) without hand-derived formulas.
template <typename T> struct Dual {
    T v, d[3];
};
template <typename T> inline Dual<T> dc(T c) { return Dual<T>{c, {0, 0, 0}}; }
template <typename T> inline Dual<T> operator+(Dual<T> a, Dual<T> b) { return {a.v + b.v, {a.d[0] + b.d[0], a.d[1] + b.d[1], a.d[2] + b.d[2]}}; }
template <typename T> inline Dual<T> operator-(Dual<T> a, Dual<T> b) { return {a.v - b.v, {a.d[0] - b.d[0], a.d[1] - b.d[1], a.d[2] - b.d[2]}}; }
template <typename T> inline Dual<T> operator*(Dual<T> a, Dual<T> b) {
    return {a.v * b.v, {a.d[0] * b.v + a.v * b.d[0], a.d[1] * b.v + a.v * b.d[1], a.d[2] * b.v + a.v * b.d[2]}};
}
template <typename T> inline Dual<T> operator*(T s, Dual<T> a) { return {s * a.v, {s * a.d[0], s * a.d[1], s * a.d[2]}}; }
template <typename T> inline Dual<T> operator+(Dual<T> a, T s) { return {a.v + s, {a.d[0], a.d[1], a.d[2]}}; }

// Real SH bases up to degree 4 at a unit direction (x,y,z), in the sign and
// ordering convention of the reference (Sloan, "Efficient Spherical Harmonic
// Evaluation", JCGT 2013; spherical_harmonics.cuh:17-111).
template <typename S, typename T> inline void sh_bases(int degree, S x, S y, S z, S* b) {
    b[0] = S{} + T(0.2820947917738781);
    if (degree < 1) return;
    b[1] = T(-0.48860251190292) * y;
    b[2] = T(0.48860251190292) * z;
    b[3] = T(-0.48860251190292) * x;
    if (degree < 2) return;
    const S z2 = z * z, fC1 = x * x - y * y, fS1 = T(2) * (x * y);
    b[4] = T(0.5462742152960395) * fS1;
    b[5] = T(-1.092548430592079) * (z * y);
    b[6] = T(0.9461746957575601) * z2 + T(-0.3153915652525201);
    b[7] = T(-1.092548430592079) * (z * x);
    b[8] = T(0.5462742152960395) * fC1;
    if (degree < 3) return;
    const S fC2 = x * fC1 - y * fS1, fS2 = x * fS1 + y * fC1;
    const S t0c = T(-2.285228997322329) * z2 + T(0.4570457994644658);
    b[9] = T(-0.5900435899266435) * fS2;
    b[10] = T(1.445305721320277) * (z * fS1);
    b[11] = t0c * y;
    b[12] = z * (T(1.865881662950577) * z2 + T(-1.119528997770346));
    b[13] = t0c * x;
    b[14] = T(1.445305721320277) * (z * fC1);
    b[15] = T(-0.5900435899266435) * fC2;
    if (degree < 4) return;
    const S fC3 = x * fC2 - y * fS2, fS3 = x * fS2 + y * fC2;
    const S t0d = z * (T(-4.683325804901025) * z2 + T(2.007139630671868));
    const S t1c = T(3.31161143515146) * z2 + T(-0.47308734787878);
    b[16] = T(0.6258357354491763) * fS3;
    b[17] = T(-1.770130769779931) * (z * fS2);
    b[18] = t1c * fS1;
    b[19] = t0d * y;
    b[20] = T(1.984313483298443) * (z * b[12]) - T(1.006230589874905) * b[6];
    b[21] = t0d * x;
    b[22] = t1c * fC1;
    b[23] = T(-1.770130769779931) * (z * fC2);
    b[24] = T(0.6258357354491763) * fC3;
}

template <typename T>
void sh_fwd(int64_t n, int degree, int K, const T* dirs, const T* coeffs, const uint8_t* masks, T* colors) {
    const int nb = (degree + 1) * (degree + 1);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        for (int c = 0; c < 3; ++c) colors[3 * i + c] = 0;
        if (masks && !masks[i]) continue;
        T b[25];
        const T* d = dirs + 3 * i;
        if (degree >= 1) {
            const T inv = T(1) / std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            sh_bases<T, T>(degree, d[0] * inv, d[1] * inv, d[2] * inv, b);
        } else {
            b[0] = T(0.2820947917738781);
        }
        for (int c = 0; c < 3; ++c) {
            T acc = 0;
            for (int k = 0; k < nb; ++k) acc += b[k] * coeffs[(i * K + k) * 3 + c];
            colors[3 * i + c] = acc;
        }
    }
}

template <typename T>
void sh_bwd(int64_t n, int degree, int K, const T* dirs, const T* coeffs, const uint8_t* masks, const T* v_colors,
            T* v_coeffs, T* v_dirs) {
    const int nb = (degree + 1) * (degree + 1);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        if (masks && !masks[i]) continue;
        const T* d = dirs + 3 * i;
        Dual<T> dx{d[0], {1, 0, 0}}, dy{d[1], {0, 1, 0}}, dz{d[2], {0, 0, 1}};
        Dual<T> b[25];
        if (degree >= 1) {
            const Dual<T> n2 = dx * dx + dy * dy + dz * dz;
            const T inv = T(1) / std::sqrt(n2.v);
            // d(1/sqrt(n2)) = -0.5 n2^{-3/2} d(n2)
            const T dinv = T(-0.5) * inv * inv * inv;
            const Dual<T> invd{inv, {dinv * n2.d[0], dinv * n2.d[1], dinv * n2.d[2]}};
            sh_bases<Dual<T>, T>(degree, dx * invd, dy * invd, dz * invd, b);
        } else {
            b[0] = dc<T>(T(0.2820947917738781));
        }
        T gd[3] = {0, 0, 0};
        for (int k = 0; k < nb; ++k)
            for (int c = 0; c < 3; ++c) {
                const T vcol = v_colors[3 * i + c];
                v_coeffs[(i * K + k) * 3 + c] += b[k].v * vcol;
                const T w = coeffs[(i * K + k) * 3 + c] * vcol;
                gd[0] += w * b[k].d[0]; gd[1] += w * b[k].d[1]; gd[2] += w * b[k].d[2];
            }
        if (v_dirs)
            for (int j = 0; j < 3; ++j) v_dirs[3 * i + j] += gd[j];
    }
}

}  // namespace

// ============================================================ C ABI (ctypes)
#define TGO_EXPORT extern "C" __attribute__((visibility("default")))

#define TGO_DEF_PROJ(SUF, T)                                                                                         \
    TGO_EXPORT void tgo_project_fwd_##SUF(int C, int N, const T* means, const T* quats, const T* scales,              \
                                          const T* viewmats, const T* Ks, int W, int H, double near_plane,            \
                                          double far_plane, double radius_clip, int32_t* radii, T* means2d,           \
                                          T* depths, T* M, T* normals) {                                              \
        project_fwd<T>(C, N, means, quats, scales, viewmats, Ks, W, H, (T)near_plane, (T)far_plane, (T)radius_clip,  \
                       radii, means2d, depths, M, normals);                                                          \
    }                                                                                                                \
    TGO_EXPORT void tgo_project_bwd_##SUF(int C, int N, const T* means, const T* quats, const T* scales,              \
                                          const T* viewmats, const T* Ks, const int32_t* radii, const T* M,           \
                                          const T* v_means2d, const T* v_depths, const T* v_normals, const T* v_M,    \
                                          int mode, T* v_means, T* v_quats, T* v_scales) {                            \
        project_bwd<T>(C, N, means, quats, scales, viewmats, Ks, radii, M, v_means2d, v_depths, v_normals, v_M,      \
                       mode, v_means, v_quats, v_scales);                                                             \
    }                                                                                                                \
    TGO_EXPORT void tgo_isect_count_##SUF(int64_t n, const T* means2d, const int32_t* radii, int tile_size, int tw,   \
                                          int th, int32_t* tiles_per_gauss) {                                         \
        isect_count<T>(n, means2d, radii, tile_size, tw, th, tiles_per_gauss);                                       \
    }                                                                                                                \
    TGO_EXPORT void tgo_isect_emit_##SUF(int64_t n, int64_t N, const int64_t* camera_ids, const T* means2d,          \
                                         const int32_t* radii, const float* depths, const int64_t* cum, int tile_size, \
                                         int tw, int th, int tile_n_bits, int64_t* isect_ids, int32_t* flatten_ids) { \
        isect_emit<T>(n, N, camera_ids, means2d, radii, depths, cum, tile_size, tw, th, tile_n_bits, isect_ids,     \
                      flatten_ids);                                                                                  \
    }                                                                                                                \
    TGO_EXPORT void tgo_sh_fwd_##SUF(int64_t n, int degree, int K, const T* dirs, const T* coeffs,                   \
                                     const uint8_t* masks, T* colors) {                                               \
        sh_fwd<T>(n, degree, K, dirs, coeffs, masks, colors);                                                        \
    }                                                                                                                \
    TGO_EXPORT void tgo_sh_bwd_##SUF(int64_t n, int degree, int K, const T* dirs, const T* coeffs,                   \
                                     const uint8_t* masks, const T* v_colors, T* v_coeffs, T* v_dirs) {                \
        sh_bwd<T>(n, degree, K, dirs, coeffs, masks, v_colors, v_coeffs, v_dirs);                                    \
    }                                                                                                                \
    TGO_EXPORT void tgo_raster_fwd_##SUF(                                                                            \
        int C, int N, int D, int W, int H, int tile_size, int tile_w, int tile_h, int64_t n_isects, const T* means2d, \
        const T* M, const T* colors, const T* opacities, const T* normals, const T* textures, int tex_ry, int tex_rx, \
        int mip_L, int aniso, double range_x, double range_y, const T* backgrounds, const uint8_t* masks,             \
        const int32_t* offsets,                                                                                      \
        const int32_t* flatten_ids, const int64_t* gaussian_ids, double contrib_threshold, double g_weight,           \
        T* out_colors, T* out_alphas, T* out_normals, T* out_distort, T* out_median, int32_t* last_ids,              \
        int32_t* median_ids, T* contrib_sum, T* contrib_count, int32_t* pair_count, uint64_t* branch_sig) {          \
        RasterIn<T> a{C, N, D, W, H, tile_size, tile_w, tile_h, n_isects, means2d, M, colors, opacities, normals,    \
                      textures, tex_ry, tex_rx, (T)range_x, (T)range_y, backgrounds, masks, offsets, flatten_ids,     \
                      gaussian_ids, (T)contrib_threshold, (T)g_weight, mip_L, aniso};                                \
        RasterOut<T> o{out_colors, out_alphas, out_normals, out_distort, out_median, last_ids, median_ids,            \
                       contrib_sum, contrib_count};                                                                   \
        raster_fwd<T>(a, o, pair_count, branch_sig);                                                                             \
    }                                                                                                                \
    TGO_EXPORT void tgo_raster_bwd_##SUF(                                                                            \
        int C, int N, int D, int W, int H, int tile_size, int tile_w, int tile_h, int64_t n_isects, int64_t E,       \
        const T* means2d, const T* M, const T* colors, const T* opacities, const T* normals, const T* textures,       \
        int tex_ry, int tex_rx, int mip_L, int aniso, double range_x, double range_y, const T* backgrounds,          \
        const uint8_t* masks,                                                                                        \
        const int32_t* offsets, const int32_t* flatten_ids, const int64_t* gaussian_ids, double g_weight,             \
        const T* f_colors, const T* f_alphas, const int32_t* last_ids, const int32_t* median_ids, const T* v_colors,  \
        const T* v_alphas, const T* v_normals, const T* v_distort, const T* v_median, int mode, T* g_means2d,         \
        T* g_means2d_abs, T* g_M, T* g_colors, T* g_opacities, T* g_normals, T* g_textures, T* g_densify) {           \
        RasterIn<T> a{C, N, D, W, H, tile_size, tile_w, tile_h, n_isects, means2d, M, colors, opacities, normals,    \
                      textures, tex_ry, tex_rx, (T)range_x, (T)range_y, backgrounds, masks, offsets, flatten_ids,     \
                      gaussian_ids, T(0), (T)g_weight, mip_L, aniso};                                                \
        RasterGradIn<T> gi{f_colors, f_alphas, last_ids, median_ids, v_colors, v_alphas, v_normals, v_distort,       \
                           v_median};                                                                                \
        RasterGradOut<T> go{g_means2d, g_means2d_abs, g_M, g_colors, g_opacities, g_normals, g_textures, g_densify}; \
        raster_bwd<T>(a, gi, go, mode, E);                                                                           \
    }

TGO_DEF_PROJ(f32, float)
TGO_DEF_PROJ(f64, double)

// anisotropic_bilinear on one footprint: corners [4,2] in texel coordinates, texture [ry,rx,4];
// out = the filtered RGBA (zero when the footprint has no texture sample); returns the footprint area.
TGO_EXPORT double tgo_aniso_sample(const double* corners, int rx, int ry, const double* tex, double* out) {
    AnisoFoot<double> F;
    for (int i = 0; i < 4; ++i) F.s[i] = {corners[2 * i], corners[2 * i + 1]};
    const double area = aniso_setup(F, rx, ry);
    for (int k = 0; k < 4; ++k) out[k] = 0;
    if (area == 0 || F.minu == F.maxu || F.minv == F.maxv) return area;
    for (int v = F.minv; v < F.maxv; ++v)
        for (int u = F.minu; u < F.maxu; ++u) {
            double A, Sx, Sy, Sxy;
            if (!aniso_cell(F, u, v, A, Sx, Sy, Sxy)) continue;
            const double w[4] = {((A - Sx) - Sy) + Sxy, Sx - Sxy, Sy - Sxy, Sxy};
            const int64_t t00 = (int64_t)v * rx + u;
            const int64_t tq[4] = {t00, t00 + 1, t00 + rx, t00 + rx + 1};
            for (int q = 0; q < 4; ++q)
                for (int k = 0; k < 4; ++k) out[k] += w[q] * tex[tq[q] * 4 + k] / area;
        }
    return area;
}

TGO_EXPORT void tgo_sort_pairs(int64_t n, int64_t* keys, int32_t* vals, int end_bit) { sort_pairs(n, keys, vals, end_bit); }

TGO_EXPORT void tgo_offset_encode(int64_t n, const int64_t* keys, int C, int n_tiles, int tile_n_bits,
                                  int32_t* offsets) {
    offset_encode(n, keys, C, n_tiles, tile_n_bits, offsets);
}
