// Per-(pixel, splat) evaluation shared by the compositor forward and adjoint.
//
// Both kernels call eval_pair with the same inputs, so a splat's alpha -- and
// therefore the set of splats that contributed to a pixel -- is recomputed
// bit-identically in the backward.  The arithmetic follows
// rasterize_to_pixels_textured_gaussians_2dgs_fwd.cu:283-347 (textured) and
// rasterize_to_pixels_2dgs_fwd.cu:281-310 (plain) of the reference, the
// bilinear addressing filters/bilinear.cuh:16-64, for the mipmapped2 filter
// rasterize_to_pixels_mip2_textured_gaussians_2dgs_fwd.cu:293-347, and for the
// anisotropic_bilinear filter
// rasterize_to_pixels_aniso_bilinear_textured_gaussians_2dgs_fwd.cu:296-391.
#pragma once
#include "tg_common.cuh"

namespace tg {

constexpr float kFilterInvSquare = 2.0f;

// Texture filters: bilinear (4 taps in the splat's texture), mipmapped2
// (8 taps: bilinear in the two pyramid levels around the pixel footprint's
// level, filters/mip2.cuh:27-105 of the reference) and anisotropic_bilinear
// (the bilinear interpolant integrated over the pixel's footprint quad,
// filters/anisotropic_bilinear.cuh:15-400: a variable number of texel cells).
// kUV: the adjoint carries the texture lookup's dependence on the UV point (the bwd2 and exact adjoints); a
// compile-time property so that the reference adjoint does not keep the taps live for it.
struct FiltBilinear {
    static constexpr int kTaps = 4;
    static constexpr bool kMip = false;
    static constexpr bool kAniso = false;
    static constexpr bool kUV = false;
};
struct FiltBilinearUV : FiltBilinear {
    static constexpr bool kUV = true;
};
struct FiltMip2 {
    static constexpr int kTaps = 8;
    static constexpr bool kMip = true;
    static constexpr bool kAniso = false;
    static constexpr bool kUV = false;
};
struct FiltAniso {
    static constexpr int kTaps = 1;  // unused: the footprint replaces the tap list
    static constexpr bool kMip = false;
    static constexpr bool kAniso = true;
    static constexpr bool kUV = false;
};

template <int NT>
struct PairEvalT {
    f3 hu, hv, z;
    float sx, sy, dx, dy;
    float g3, g2, kern, vis, alpha, asf;
    float w[NT];
    float4 tx[NT];  // the RGBA taps
    float4 trgba;   // the filtered texture: sum over taps of w * tap (asf = its alpha)
    int toff[NT];   // bilinear: texel index in the splat's texture; mip: pyramid coordinate (see MipSrc)
    bool valid, tex_valid;
};
using PairEval = PairEvalT<4>;

// The anisotropic_bilinear footprint of one (pixel, splat) pair: the pixel's
// corners mapped to texel coordinates (counter-clockwise), their edges, the
// reference's edge normals and fast-path margins, the texel-cell range and
// 1 / area; tsum is the texture integral before the division by the area.
struct AnisoFoot {
    float2 s[4], n[4];
    float2 r[4];  // 1 / x and 1 / y of edge i, s[i+1] - s[i] (the cell clip divisors; unused where a component is 0)
    float nmax[4];
    int minu, maxu, minv, maxv;
    float iarea;
    bool convex;  // the four corner rays meet the splat plane on one side (same sign of z) and no two
                  // adjacent corners coincide: the boundary sum applies, else the polygon clipping
};
struct PairEvalAniso : PairEvalT<1> {
    AnisoFoot F;
    float4 tsum;
    float a0;   // opacity x Gaussian weight: the alpha before the texture term
    bool need;  // the footprint has texel cells to integrate
};
template <class Filt> struct PairOfT { using type = PairEvalT<Filt::kTaps>; };
template <> struct PairOfT<FiltAniso> { using type = PairEvalAniso; };
template <class Filt> using PairOf = typename PairOfT<Filt>::type;

__device__ __forceinline__ float cross2(float2 a, float2 b) { return a.x * b.y - a.y * b.x; }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// Orientation (counter-clockwise) and texel-cell range of the footprint quad;
// returns its area (precompute, filters/anisotropic_bilinear.cuh:193-245).
// Clears F.convex for a quad with a zero-length edge.  What only the
// cell-by-cell integration needs (edge reciprocals, normals, margins) is
// aniso_cells_setup's.
__device__ __forceinline__ float aniso_setup(AnisoFoot& F, int rx, int ry) {
    float area = 0.5f * (cross2(sub2(F.s[1], F.s[0]), sub2(F.s[2], F.s[1])) +
                         cross2(sub2(F.s[3], F.s[2]), sub2(F.s[0], F.s[3])));
    if (area < 0.f) {
        area = -area;
        const float2 t = F.s[1];
        F.s[1] = F.s[3];
        F.s[3] = t;
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float2 e = sub2(F.s[(i + 1) & 3], F.s[i]);
        // a zero-length edge (collapsed corner) has no half-plane: the polygon clipping handles that quad
        if (e.x == 0.f && e.y == 0.f) F.convex = false;
    }
    // float -> int conversions saturate (NaN -> 0), so the cell range stays within the texture
    F.minu = max(0, (int)floorf(fminf(fminf(F.s[0].x, F.s[1].x), fminf(F.s[2].x, F.s[3].x))));
    F.maxu = min(rx - 1, (int)ceilf(fmaxf(fmaxf(F.s[0].x, F.s[1].x), fmaxf(F.s[2].x, F.s[3].x))));
    F.minv = max(0, (int)floorf(fminf(fminf(F.s[0].y, F.s[1].y), fminf(F.s[2].y, F.s[3].y))));
    F.maxv = min(ry - 1, (int)ceilf(fmaxf(fmaxf(F.s[0].y, F.s[1].y), fmaxf(F.s[2].y, F.s[3].y))));
    return area;
}

// Edge reciprocals, normals and margins of the (oriented) footprint quad, for the cell-by-cell integration
// (filters/anisotropic_bilinear.cuh:193-245).
__device__ __forceinline__ void aniso_cells_setup(AnisoFoot& F) {
    float2 e[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        e[i] = sub2(F.s[(i + 1) & 3], F.s[i]);
        F.r[i] = make_float2(__frcp_rn(e[i].x), __frcp_rn(e[i].y));
    }
    const float cx = (((F.s[0].x + F.s[1].x) + F.s[2].x) + F.s[3].x) * 0.25f;
    const float cy = (((F.s[0].y + F.s[1].y) + F.s[2].y) + F.s[3].y) * 0.25f;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        float2 n = (e[i].x == 0.f && e[i].y == 0.f) ? make_float2(F.s[i].x - cx, F.s[i].y - cy)
                                                    : make_float2(e[i].y, -e[i].x);
        const float l = sqrtf(n.x * n.x + n.y * n.y);
        if (l != 0.f) n = make_float2(n.x / l, n.y / l);
        F.n[i] = n;
        F.nmax[i] = fmaxf(fabsf(n.x * 0.5f + n.y * 0.5f), fabsf(n.x * 0.5f - n.y * 0.5f));
    }
}

// Green's-theorem terms of one directed boundary segment a -> b (cell-local
// coordinates), as (A, Sx, Sy, Sxy) before their 1/2, 1/6, 1/6, 1/24 factors.
__device__ __forceinline__ void seg_moments(float2 a, float2 b, float4& m) {
    const float c = a.x * b.y - a.y * b.x;
    m.x += c;
    m.y += c * (a.x + b.x);
    m.z += c * (a.y + b.y);
    m.w += c * (2.f * a.x * a.y + a.x * b.y + b.x * a.y + 2.f * b.x * b.y);
}

// Restricts [t0, t1] to the t with p + t q >= 0 (rq = 1 / q), without
// branches; false only when q = 0 and p < 0 (no t qualifies).  The interval
// only shrinks, so the callers test t0 < t1 once, after all their clips: the
// same segments as stopping at the first empty interval (measured 8 % faster
// for anisotropic_bilinear than the early-exit chain).
__device__ __forceinline__ bool clip_t(float p, float q, float rq, float& t0, float& t1) {
    const float t = -p * rq;
    t0 = q > 0.f ? fmaxf(t0, t) : t0;
    t1 = q < 0.f ? fminf(t1, t) : t1;
    return q != 0.f || p >= 0.f;
}

// Sutherland-Hodgman clip of the polygon p[0..n) to one side of the unit
// cell (axis 0: x, 1: y; hi: keep <= 1, else >= 0) into q; returns the new
// vertex count, or -1 if it would exceed 8 (only a self-intersecting quad can).
__device__ __forceinline__ int sh_clip(const float2* p, int n, float2* q, int axis, bool hi) {
    int m = 0;
    for (int i = 0; i < n; ++i) {
        const float2 a = p[i], b = p[i + 1 == n ? 0 : i + 1];
        const float ac = axis ? a.y : a.x, bc = axis ? b.y : b.x;
        const bool ain = hi ? ac <= 1.f : ac >= 0.f, bin = hi ? bc <= 1.f : bc >= 0.f;
        if (ain) {
            if (m == 8) return -1;
            q[m++] = a;
        }
        if (ain != bin) {
            if (m == 8) return -1;
            const float t = hi ? (ac - 1.f) / (ac - bc) : ac / (ac - bc);
            q[m++] = axis ? make_float2(a.x + t * (b.x - a.x), hi ? 1.f : 0.f)
                          : make_float2(hi ? 1.f : 0.f, a.y + t * (b.y - a.y));
        }
    }
    return m;
}

// The reference's polygon clipping, kept for footprints whose corner rays meet
// the splat plane on both sides (the quad then is not convex): clip against
// x >= 0, x <= 1, y >= 0, y <= 1, then sum the polygon's edge terms.
static __device__ __noinline__ float4 aniso_cell_polygon(const AnisoFoot F, int u, int v) {
    float2 p[8], q[8];
#pragma unroll
    for (int i = 0; i < 4; ++i) p[i] = make_float2(F.s[i].x - (float)u, F.s[i].y - (float)v);
    int n = 4;
    const float4 none = make_float4(0.f, 0.f, 0.f, 0.f);
    if ((n = sh_clip(p, n, q, 0, false)) < 3) return none;
    if ((n = sh_clip(q, n, p, 0, true)) < 3) return none;
    if ((n = sh_clip(p, n, q, 1, false)) < 3) return none;
    if ((n = sh_clip(q, n, p, 1, true)) < 3) return none;
    float4 m = none;
    for (int i = 0; i < n; ++i) seg_moments(p[i], p[i + 1 == n ? 0 : i + 1], m);
    return make_float4(m.x * 0.5f, m.y * (1.f / 6.f), m.z * (1.f / 6.f), m.w * (1.f / 24.f));
}

// The piecewise boundary sum of a convex quad (corners s, counter-clockwise;
// rc: reciprocals of its edges' components) over cell [u, u+1] x [v, v+1].
__device__ __forceinline__ float4 cell_edges_sum(const float2 (&s)[4], const float2 (&rc)[4], int u, int v) {
    float2 e[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) e[i] = sub2(s[(i + 1) & 3], s[i]);
    const float fu = (float)u, fv = (float)v;
    float4 m = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int i = 0; i < 4; ++i) {  // quad edges inside the cell
        const float2 a = make_float2(s[i].x - fu, s[i].y - fv), d = e[i], rd = rc[i];
        float t0 = 0.f, t1 = 1.f;
        const bool k0 = clip_t(a.x, d.x, rd.x, t0, t1), k1 = clip_t(1.f - a.x, -d.x, -rd.x, t0, t1);
        const bool k2 = clip_t(a.y, d.y, rd.y, t0, t1), k3 = clip_t(1.f - a.y, -d.y, -rd.y, t0, t1);
        if (k0 & k1 & k2 & k3 & (t0 < t1))
            seg_moments(make_float2(a.x + t0 * d.x, a.y + t0 * d.y), make_float2(a.x + t1 * d.x, a.y + t1 * d.y), m);
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {  // cell edges inside the quad, counter-clockwise
        const float2 a = make_float2((j == 1 || j == 2) ? 1.f : 0.f, j >= 2 ? 1.f : 0.f);
        const float2 d = make_float2(j == 0 ? 1.f : (j == 2 ? -1.f : 0.f), j == 1 ? 1.f : (j == 3 ? -1.f : 0.f));
        float t0 = 0.f, t1 = 1.f;
        bool keep = true;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float2 r = make_float2(a.x + fu - s[i].x, a.y + fv - s[i].y);
            const float p = cross2(e[i], r), q = cross2(e[i], d);
            // q is -e.y, e.x, e.y, -e.x for the cell edges j = 0..3: its reciprocal is the footprint's
            const float rq = j == 0 ? -rc[i].y : (j == 1 ? rc[i].x : (j == 2 ? rc[i].y : -rc[i].x));
            // parallel to quad edge i (q = 0): kept if inside it, or on it running the other way (a quad
            // with a zero-length edge, for which this would drop every cell edge, takes the polygon clipping)
            const bool par = p > 0.f || (p == 0.f && e[i].x * d.x + e[i].y * d.y < 0.f);
            const bool k = clip_t(p, q, rq, t0, t1);
            keep = keep & (q == 0.f ? par : k);
        }
        if (keep && t0 < t1)
            seg_moments(make_float2(a.x + t0 * d.x, a.y + t0 * d.y), make_float2(a.x + t1 * d.x, a.y + t1 * d.y), m);
    }
    return make_float4(m.x * 0.5f, m.y * (1.f / 6.f), m.z * (1.f / 6.f), m.w * (1.f / 24.f));
}

// The same sum as one out-of-line copy.  The adjoint integrates every
// footprint twice (its integral, then its texel gradients); with the sum
// inlined at both places its hot code outgrew the instruction cache.
static __device__ __noinline__ float4 cell_edges_sum_shared(float2 s0, float2 s1, float2 s2, float2 s3, float2 r0,
                                                            float2 r1, float2 r2, float2 r3, int u, int v) {
    const float2 s[4] = {s0, s1, s2, s3}, rc[4] = {r0, r1, r2, r3};
    return cell_edges_sum(s, rc, u, v);
}

// Moments (A, Sx, Sy, Sxy) of the footprint quad clipped to texel cell
// [u, u+1] x [v, v+1], in cell-local coordinates (the reference's
// clip_and_compute_moments, filters/anisotropic_bilinear.cuh:58-190).  The
// reference clips the quad polygon Sutherland-Hodgman style into local arrays;
// for a convex quad (every footprint whose corner rays meet the splat plane on
// one side) the clipped polygon's boundary is summed piecewise here instead --
// the quad's edges clipped to the cell plus the cell's edges clipped to the
// quad -- the same polygon's moments without dynamically indexed storage.  A
// cell edge lying on a quad edge of the same direction is left to the quad
// edge (counted once); of opposite direction, both count and cancel.
// kShared: take the boundary sum from its out-of-line copy.
template <bool kShared = false>
__device__ __forceinline__ float4 aniso_cell(const AnisoFoot& F, int u, int v) {
    const float2 c = make_float2((float)u + 0.5f, (float)v + 0.5f);
    bool inside = true, outside = false;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float d = sub2(F.s[i], c).x * F.n[i].x + sub2(F.s[i], c).y * F.n[i].y;  // c's depth inside edge i
        const float2 e = sub2(F.s[(i + 1) & 3], F.s[i]);
        inside = inside && d >= F.nmax[i];
        // the whole cell beyond a (non-degenerate) edge of a convex quad: nothing to integrate
        outside = outside || (d < -F.nmax[i] && (e.x != 0.f || e.y != 0.f));
    }
    if (inside) return make_float4(1.f, 0.5f, 0.5f, 0.25f);  // the reference's fast path: the whole cell
    if (!F.convex) return aniso_cell_polygon(F, u, v);
    if (outside) return make_float4(0.f, 0.f, 0.f, 0.f);
    if constexpr (kShared)
        return cell_edges_sum_shared(F.s[0], F.s[1], F.s[2], F.s[3], F.r[0], F.r[1], F.r[2], F.r[3], u, v);
    else
        return cell_edges_sum(F.s, F.r, u, v);
}

// ---------------------------------------------------------------- anisotropic_bilinear by boundary integral
// The footprint integral of the bilinear interpolant f over P = quad ∩ [0, rx-1] x [0, ry-1] (the cells the
// reference visits, clamped to the texture) is turned into a line integral by Green's theorem:
//   ∫∫_P f dA = ∮_∂P F dy,   F(x, y) = ∫_{x0}^{x} f(s, y) ds   (∂P counter-clockwise, x0 = the first cell column),
// and F is read from per-row prefix integrals of the texture (the rows' trapezoid sums,
// P_r[u] = Σ_{k<u} (t(k,r) + t(k+1,r)) / 2, built once per call by tg_aniso_prefix):
//   F = (1 - y') (P_v[u] - P_v[x0] + a (x' - x'²/2) + b x'²/2) + y' (P_{v+1}[u] - P_{v+1}[x0] + c (x' - x'²/2) + d x'²/2)
// in cell (u, v) with texels a, b, c, d = t(u,v), t(u+1,v), t(u,v+1), t(u+1,v+1) and x' = x - u, y' = y - v.
// Along a straight piece inside one cell F is a cubic in the line parameter, so two-point Gauss-Legendre is
// exact.  The boundary is the quad's four edges clipped to the texture box plus the box's right edge
// x = rx - 1 where the quad reaches past it (on the left edge x = x0 = 0 F vanishes; the top and bottom
// edges have dy = 0).  Work per footprint is proportional to its perimeter in cells, not its area.  Only
// convex footprints take this route; the others keep the reference's per-cell polygon clipping.

// Weights of one piece a -> b of the boundary inside cell (u, v): the piece's integral is
//   wa a + wb b + wc c + wd d + wp0 (P_v[u] - P_v[x0]) + wp1 (P_{v+1}[u] - P_{v+1}[x0]).
struct PieceW {
    float wa, wb, wc, wd, wp0, wp1;
};
__device__ __forceinline__ PieceW piece_weights(float2 a, float2 b, int u, int v) {
    constexpr float kG = 0.21132486540518713f;  // (1 - 1/sqrt(3)) / 2: the Gauss points are kG and 1 - kG
    const float dx = b.x - a.x, dy = b.y - a.y;
    PieceW w{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const float tq = q == 0 ? kG : 1.f - kG;
        const float x = (a.x - (float)u) + tq * dx, y = (a.y - (float)v) + tq * dy;
        const float x2 = 0.5f * x * x, x1 = x - x2;
        w.wa += (1.f - y) * x1;
        w.wb += (1.f - y) * x2;
        w.wc += y * x1;
        w.wd += y * x2;
        w.wp0 += 1.f - y;
        w.wp1 += y;
    }
    const float h = 0.5f * dy;  // the two Gauss weights (1/2 each) times the piece's dy
    w.wa *= h; w.wb *= h; w.wc *= h; w.wd *= h; w.wp0 *= h; w.wp1 *= h;
    return w;
}

// Walks the segment a -> b through the texel cells it crosses (cells clamped to [0, rx-2] x [0, ry-2]) and
// calls visit(piece start, piece end, u, v) for each piece with dy != 0.
template <class Visit>
__device__ __forceinline__ void walk_cells(float2 a, float2 b, int rx, int ry, Visit&& visit) {
    const float dx = b.x - a.x, dy = b.y - a.y;
    if (dy == 0.f) return;  // nothing to integrate along a horizontal piece
    // starting cell: the one the segment enters from a (ties at a grid line go the way it heads)
    int ix = dx >= 0.f ? (int)floorf(a.x) : (int)ceilf(a.x) - 1;
    int iy = dy >= 0.f ? (int)floorf(a.y) : (int)ceilf(a.y) - 1;
    const int sx = dx > 0.f ? 1 : (dx < 0.f ? -1 : 0), sy = dy > 0.f ? 1 : -1;
    const float rdx = dx != 0.f ? 1.f / dx : 0.f, rdy = 1.f / dy;
    float t = 0.f;
    float2 p = a;
    const int limit = 2 * (rx + ry) + 8;  // cells a clipped segment can cross, with margin
    for (int it = 0; it < limit; ++it) {
        const float tx = sx == 0 ? INFINITY : ((float)(sx > 0 ? ix + 1 : ix) - a.x) * rdx;
        const float ty = ((float)(sy > 0 ? iy + 1 : iy) - a.y) * rdy;
        const float tn = fminf(fminf(tx, ty), 1.f);
        const float2 q = tn >= 1.f ? b : make_float2(a.x + tn * dx, a.y + tn * dy);
        if (tn > t) visit(p, q, min(max(ix, 0), rx - 2), min(max(iy, 0), ry - 2));
        if (tn >= 1.f) break;
        if (tx <= tn) ix += sx;
        if (ty <= tn) iy += sy;
        t = tn;
        p = q;
    }
}

// Clips the boundary of a convex footprint F to the texture box [0, rx-1] x [0, ry-1]: segments 0..3 are the
// quad's edges inside the box, segment 4 the box's right edge inside the quad; sk[i]: segment i is kept.
__device__ __forceinline__ void foot_segments(const AnisoFoot& F, int rx, int ry, float2 (&sa)[5], float2 (&sb)[5],
                                              bool (&sk)[5]) {
    const float X1 = (float)(rx - 1), Y1 = (float)(ry - 1);
#pragma unroll
    for (int i = 0; i < 4; ++i) {  // the quad's edges inside the box
        const float2 a = F.s[i], d = sub2(F.s[(i + 1) & 3], F.s[i]);
        const float2 r = make_float2(1.f / d.x, 1.f / d.y);  // unused where a component is 0 (see clip_t)
        float t0 = 0.f, t1 = 1.f;
        const bool k0 = clip_t(a.x, d.x, r.x, t0, t1), k1 = clip_t(X1 - a.x, -d.x, -r.x, t0, t1);
        const bool k2 = clip_t(a.y, d.y, r.y, t0, t1), k3 = clip_t(Y1 - a.y, -d.y, -r.y, t0, t1);
        sk[i] = k0 & k1 & k2 & k3 & (t0 < t1);
        sa[i] = make_float2(a.x + t0 * d.x, a.y + t0 * d.y);
        sb[i] = make_float2(a.x + t1 * d.x, a.y + t1 * d.y);
    }
    // the box's right edge x = X1 inside the quad, upward (counter-clockwise for the box): the segment
    // (X1, 0) -> (X1, Y1) clipped against the quad's four half-planes cross(e_i, p - s_i) >= 0
    float t0 = 0.f, t1 = 1.f;
    bool keep = true;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float2 e = sub2(F.s[(i + 1) & 3], F.s[i]);
        // cross(e, (X1, t Y1) - s_i) = cross(e, (X1, 0) - s_i) + t Y1 e.x
        const float p = e.x * (0.f - F.s[i].y) - e.y * (X1 - F.s[i].x), q = e.x * Y1;
        const bool k = clip_t(p, q, q != 0.f ? 1.f / q : 0.f, t0, t1);
        // a quad edge on the line x = X1: the box edge is kept if the quad lies beyond it, or on it running
        // downward (the two cancel); running upward the quad edge itself is the boundary, counted once
        keep = keep & (q == 0.f ? (p > 0.f || (p == 0.f && e.y < 0.f)) : k);
    }
    sk[4] = keep && t0 < t1;
    sa[4] = make_float2(X1, t0 * Y1);
    sb[4] = make_float2(X1, t1 * Y1);
}

// The integral of F dy along one boundary segment a -> b, F measured from column x0 (see above), from the
// splat's texture and its row-prefix table P ([ry, rx] float4 rows).  (Keeping the texels of the cell being
// walked in registers, to read only the two a step to the next cell does not share, measured 1.8x slower:
// the loads hit L1, the branches do not pay.)
template <class Tex>
__device__ __forceinline__ float4 segment_sum(float2 a, float2 b, int x0, const void* textures, int64_t tex_base,
                                              const float4* P, int rx, int ry, float scale) {
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    walk_cells(a, b, rx, ry, [&](float2 pa, float2 pb, int u, int v) {
        const PieceW w = piece_weights(pa, pb, u, v);
        const int64_t t00 = tex_base + (int64_t)v * rx + u;
        const float4 ta = Tex::load(textures, t00, scale), tb = Tex::load(textures, t00 + 1, scale);
        const float4 tc = Tex::load(textures, t00 + rx, scale), td = Tex::load(textures, t00 + rx + 1, scale);
        // P(u) - P(x0): exactly 0 in the column x0 itself (the same entry read twice)
        const float4 a0 = __ldg(P + (int64_t)v * rx + u), b0 = __ldg(P + (int64_t)v * rx + x0);
        const float4 a1 = __ldg(P + (int64_t)(v + 1) * rx + u), b1 = __ldg(P + (int64_t)(v + 1) * rx + x0);
        const float4 p0 = make_float4(a0.x - b0.x, a0.y - b0.y, a0.z - b0.z, a0.w - b0.w);
        const float4 p1 = make_float4(a1.x - b1.x, a1.y - b1.y, a1.z - b1.z, a1.w - b1.w);
        acc.x += w.wa * ta.x + w.wb * tb.x + w.wc * tc.x + w.wd * td.x + w.wp0 * p0.x + w.wp1 * p1.x;
        acc.y += w.wa * ta.y + w.wb * tb.y + w.wc * tc.y + w.wd * td.y + w.wp0 * p0.y + w.wp1 * p1.y;
        acc.z += w.wa * ta.z + w.wb * tb.z + w.wc * tc.z + w.wd * td.z + w.wp0 * p0.z + w.wp1 * p1.z;
        acc.w += w.wa * ta.w + w.wb * tb.w + w.wc * tc.w + w.wd * td.w + w.wp0 * p0.w + w.wp1 * p1.w;
    });
    return acc;
}

// The same as one out-of-line copy, for the adjoint (which also has the scatter's walk: both inlined
// outgrow the instruction cache).
template <class Tex>
static __device__ __noinline__ float4 segment_sum_shared(float2 a, float2 b, int x0, const void* textures,
                                                         int64_t tex_base, const float4* P, int rx, int ry,
                                                         float scale) {
    return segment_sum<Tex>(a, b, x0, textures, tex_base, P, rx, ry, scale);
}

// Adjoint of segment_sum for the gradient g (already divided by the area): texel gradients into vt (the
// splat's [ry, rx] float4 rows) and row-prefix gradients into vP, which tg_rasterize_bwd folds back into the
// texels afterwards.  The x0 terms are left out: over the closed boundary they integrate a function of y
// alone, which gives zero, so the footprint's gradient is the same without them (and the column x0 would
// take an atomic from every piece).  Six atomics per piece, without branches: keeping the weights of the
// cell being walked in registers and carrying the texels it shares with the next one (about three atomics
// per piece) measured 28 % slower.
static __device__ __noinline__ void segment_scatter(float2 a, float2 b, float4 g, float* vt, float* vP, int rx,
                                                    int ry) {
    float4* T4 = reinterpret_cast<float4*>(vt);
    float4* P4 = reinterpret_cast<float4*>(vP);
    walk_cells(a, b, rx, ry, [&](float2 pa, float2 pb, int u, int v) {
        const PieceW w = piece_weights(pa, pb, u, v);
        const int64_t t00 = (int64_t)v * rx + u;
        atomicAdd(T4 + t00, make_float4(g.x * w.wa, g.y * w.wa, g.z * w.wa, g.w * w.wa));
        atomicAdd(T4 + t00 + 1, make_float4(g.x * w.wb, g.y * w.wb, g.z * w.wb, g.w * w.wb));
        atomicAdd(T4 + t00 + rx, make_float4(g.x * w.wc, g.y * w.wc, g.z * w.wc, g.w * w.wc));
        atomicAdd(T4 + t00 + rx + 1, make_float4(g.x * w.wd, g.y * w.wd, g.z * w.wd, g.w * w.wd));
        atomicAdd(P4 + t00, make_float4(g.x * w.wp0, g.y * w.wp0, g.z * w.wp0, g.w * w.wp0));
        atomicAdd(P4 + t00 + rx, make_float4(g.x * w.wp1, g.y * w.wp1, g.z * w.wp1, g.w * w.wp1));
    });
}

// Per-warp shared memory of the boundary integration: a list of the warp's clipped boundary segments (up to
// kAnisoSegs at a time: a warp pass has 19 on average, at most 5 for each of its 32 footprints), each
// segment's owner lane (and x0), and one float4 per lane.  Small on purpose: the compositor's shared memory
// comes out of the L1 that the boundary walk reads the texture through.
constexpr int kAnisoSegs = 64;
constexpr int kAnisoWarpF4 = kAnisoSegs + 32 + kAnisoSegs / 4;  // segments, per-lane slots, owners (int)
struct AnisoWarp {
    float4* seg;  // [kAnisoSegs] (a.x, a.y, b.x, b.y)
    float4* lane; // [32]
    int* own;     // [kAnisoSegs] owner lane | x0 << 5
};
__device__ __forceinline__ AnisoWarp aniso_warp(float4* base) {
    return AnisoWarp{base, base + kAnisoSegs, reinterpret_cast<int*>(base + kAnisoSegs + 32)};
}

// The kept boundary segments of a lane's footprint (want: a convex footprint with cells to integrate) and
// their position in the warp's list (lane order): the segments base .. base + n - 1 of total.
struct SegList {
    float2 sa[5], sb[5];
    bool sk[5];
    int base, total;
};
__device__ __forceinline__ void aniso_segments(const AnisoFoot& F, bool want, int rx, int ry, unsigned mask,
                                               SegList& L) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int i = 0; i < 5; ++i) L.sk[i] = false;
    if (want) foot_segments(F, rx, ry, L.sa, L.sb, L.sk);
    int n = 0;
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        L.sk[i] = L.sk[i] && want;
        n += L.sk[i];
    }
    int incl = n;  // inclusive warp scan of the counts
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(mask, incl, o);
        if (lane >= o) incl += t;
    }
    L.base = incl - n;
    L.total = __shfl_sync(mask, incl, 31);
}

// Writes the segments r0 .. r0 + kAnisoSegs - 1 of the warp's list (those of this lane among them) to the
// warp's shared memory.  The segments are then spread over the warp's lanes: a warp typically has a handful
// of footprints of four segments each, so integrating each footprint on its own lane leaves most lanes idle
// behind the longest boundary.  (Cutting the segments further into chunks of a few cells, to fill all 32
// lanes, measured slower: 5-27 %.)
__device__ __forceinline__ void aniso_put(const SegList& L, int r0, const AnisoWarp& W, int tag) {
    int j = L.base - r0;
#pragma unroll
    for (int i = 0; i < 5; ++i)
        if (L.sk[i]) {
            if (j >= 0 && j < kAnisoSegs) {
                W.seg[j] = make_float4(L.sa[i].x, L.sa[i].y, L.sb[i].x, L.sb[i].y);
                W.own[j] = tag;
            }
            ++j;
        }
}

// Every lane's footprint integral (before the division by the area) for the lanes with want set, the warp's
// boundary segments spread over its lanes and summed per owner in shared memory.  Called by the full warp.
template <class Tex, bool kShared>
__device__ __forceinline__ float4 aniso_boundary_sum(const AnisoFoot& F, bool want, const void* textures,
                                                     int64_t tex_base, const float4* P, int rx, int ry, float scale,
                                                     const AnisoWarp& W, unsigned mask) {
    const int lane = threadIdx.x & 31;
    want = want && F.maxu > F.minu && F.maxv > F.minv;  // no cell (also: rx or ry below 2): nothing to walk
    if (!__any_sync(mask, want)) return make_float4(0.f, 0.f, 0.f, 0.f);  // (the adjoint reading records)
    SegList L;
    aniso_segments(F, want, rx, ry, mask, L);
    W.lane[lane] = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int r0 = 0; r0 < L.total; r0 += kAnisoSegs) {
        aniso_put(L, r0, W, lane | (F.minu << 5));
        __syncwarp(mask);
        const int n = min(kAnisoSegs, L.total - r0);
        for (int t = lane; t < n; t += 32) {
            const float4 sg = W.seg[t];
            const int ow = W.own[t];
            const float2 a = make_float2(sg.x, sg.y), b = make_float2(sg.z, sg.w);
            float4 r;
            if constexpr (kShared) r = segment_sum_shared<Tex>(a, b, ow >> 5, textures, tex_base, P, rx, ry, scale);
            else r = segment_sum<Tex>(a, b, ow >> 5, textures, tex_base, P, rx, ry, scale);
            float* dst = reinterpret_cast<float*>(W.lane + (ow & 31));
            atomicAdd(dst, r.x);
            atomicAdd(dst + 1, r.y);
            atomicAdd(dst + 2, r.z);
            atomicAdd(dst + 3, r.w);
        }
        __syncwarp(mask);  // the list is read before the next round rewrites it
    }
    const float4 r = W.lane[lane];
    __syncwarp(mask);  // read before the next call reuses the slots
    return r;
}

// Adjoint of aniso_boundary_sum: the gradient g of every lane with want set (already divided by the area)
// scattered along its footprint's boundary, the segments spread over the warp.  Called by the full warp.
__device__ __forceinline__ void aniso_boundary_scatter(const AnisoFoot& F, float4 g, bool want, float* vt, float* vP,
                                                       int rx, int ry, const AnisoWarp& W, unsigned mask) {
    const int lane = threadIdx.x & 31;
    want = want && F.maxu > F.minu && F.maxv > F.minv;
    if (!__any_sync(mask, want)) return;
    SegList L;
    aniso_segments(F, want, rx, ry, mask, L);
    W.lane[lane] = g;
    for (int r0 = 0; r0 < L.total; r0 += kAnisoSegs) {
        aniso_put(L, r0, W, lane);
        __syncwarp(mask);
        const int n = min(kAnisoSegs, L.total - r0);
        for (int t = lane; t < n; t += 32) {
            const float4 sg = W.seg[t];
            segment_scatter(make_float2(sg.x, sg.y), make_float2(sg.z, sg.w), W.lane[W.own[t] & 31], vt, vP, rx,
                            ry);
        }
        __syncwarp(mask);  // the list is read before the next round rewrites it
    }
}

// Bilinear weights of a cell's four texels (u,v), (u+1,v), (u,v+1), (u+1,v+1) from its moments.
__device__ __forceinline__ float4 cell_weights(float4 mo) {
    return make_float4(((mo.x - mo.y) - mo.z) + mo.w, mo.y - mo.w, mo.z - mo.w, mo.w);
}


// Coarse pyramid levels of the mip filter for one splat.  Pyramid coordinate
// mc addresses the reference's per-splat pyramid [coarse levels | level 0]:
// mc < clen lies in `coarse` (levels 1..L, FP32), mc >= clen is texel mc - clen
// of the splat's full-resolution texture (the texture storage itself, so level
// 0 is never copied).
struct MipSrc {
    const float* coarse;
    int64_t cbase;  // first coarse texel of the splat
    int clen;       // coarse texels per splat: (4^L - 1) / 3
    int L;          // log2 of the texture side
};

// First pyramid coordinate of level t (side 2^(L-t)): (4^(L-t) - 1) / 3.
__device__ __forceinline__ int mip_level_base(int L, int t) { return ((1 << ((L - t) * 2)) - 1) / 3; }

// Trilinear taps of the mipmapped2 filter (filters/mip2.cuh:27-105): level
// t = log2 of the largest texture-space footprint edge, clamped to [0, 31],
// bilinear taps in levels floor(t) and ceil(t) with corner-aligned coordinates
// (u + 0.5) / 2^level - 0.5; false when a tap falls outside its level (also
// for a level beyond the coarsest, where the reference's index is undefined).
__device__ __forceinline__ bool mip2_taps(float sx, float sy, float dxx, float dxy, float dyx, float dyy, int R, int L,
                                          float range_x, float range_y, int (&mc)[8], float (&w)[8]) {
    const float fr = (float)(R - 1);
    const float ax = dxx / (range_x * 2.f) * fr, ay = dxy / (range_x * 2.f) * fr;  // both with range_x, as the reference
    const float bx = dyx / (range_y * 2.f) * fr, by = dyy / (range_y * 2.f) * fr;
    const float duv = fmaxf(sqrtf(ax * ax + ay * ay), sqrtf(bx * bx + by * by));
    float t = log2f(duv);
    if (t < 0.f) t = 0.f;
    else if (t > 31.f) t = 31.f;
    const float u = (sx + range_x) / (range_x * 2.f) * fr;
    const float v = (sy + range_y) / (range_y * 2.f) * fr;
    const int tl = (int)floorf(t), th = (int)ceilf(t);
    if (th > L) return false;
    const float il = 1.f / (float)(1u << tl), ih = 1.f / (float)(1u << th);  // exact powers of two
    const float us = (u + 0.5f) * il - 0.5f, ug = (u + 0.5f) * ih - 0.5f;
    const float vs = (v + 0.5f) * il - 0.5f, vg = (v + 0.5f) * ih - 0.5f;
    const int uls = (int)floorf(us), ulg = (int)floorf(ug), vls = (int)floorf(vs), vlg = (int)floorf(vg);
    const int uhs = (int)ceilf(us), uhg = (int)ceilf(ug), vhs = (int)ceilf(vs), vhg = (int)ceilf(vg);
    if (uls < 0 || ulg < 0 || vls < 0 || vlg < 0 || uhs > ((R - 1) >> tl) || uhg > ((R - 1) >> th) ||
        vhs > ((R - 1) >> tl) || vhg > ((R - 1) >> th))
        return false;
    const int rl = R >> tl, rh = R >> th;
    const int bl = mip_level_base(L, tl), bh = mip_level_base(L, th);
    mc[0] = bl + vls * rl + uls;
    mc[1] = bl + vls * rl + uhs;
    mc[2] = bl + vhs * rl + uls;
    mc[3] = bl + vhs * rl + uhs;
    mc[4] = bh + vlg * rh + ulg;
    mc[5] = bh + vlg * rh + uhg;
    mc[6] = bh + vhg * rh + ulg;
    mc[7] = bh + vhg * rh + uhg;
    const float wus = us - (float)uls, wvs = vs - (float)vls, wug = ug - (float)ulg, wvg = vg - (float)vlg;
    const float wt = t - (float)tl;
    w[0] = (1.f - wus) * (1.f - wvs) * (1.f - wt);
    w[1] = wus * (1.f - wvs) * (1.f - wt);
    w[2] = (1.f - wus) * wvs * (1.f - wt);
    w[3] = wus * wvs * (1.f - wt);
    w[4] = (1.f - wug) * (1.f - wvg) * wt;
    w[5] = wug * (1.f - wvg) * wt;
    w[6] = (1.f - wug) * wvg * wt;
    w[7] = wug * wvg * wt;
    return true;
}

// sum over taps of w[i] * tap[i], per channel, accumulated in tap order
template <int NT>
__device__ __forceinline__ float4 filter_taps(const float (&w)[NT], const float4 (&tx)[NT]) {
    float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int i = 0; i < NT; ++i) {
        s.x += w[i] * tx[i].x;
        s.y += w[i] * tx[i].y;
        s.z += w[i] * tx[i].z;
        s.w += w[i] * tx[i].w;
    }
    return s;
}

// Splat data staged in shared memory: xyo = (x, y, opacity, texture scale),
// m0/m1/m2 = rows of the ray transform (w unused).
template <class Tex, class Filt = FiltBilinear>
__device__ __forceinline__ void eval_pair(PairOf<Filt>& e, float px, float py, const float4 xyo,
                                          const float4 m0, const float4 m1, const float4 m2, const void* textures,
                                          int64_t tex_base, int rx, int ry, float range_x, float range_y,
                                          float g_weight, const MipSrc mip = MipSrc{nullptr, 0, 0, 0}) {
    constexpr bool kTextured = Tex::kFormat != TG_TEX_NONE;
    e.hu = mk3(px * m2.x - m0.x, px * m2.y - m0.y, px * m2.z - m0.z);
    e.hv = mk3(py * m2.x - m1.x, py * m2.y - m1.y, py * m2.z - m1.z);
    e.z = cross(e.hu, e.hv);
    e.valid = true;
    e.tex_valid = false;
    e.asf = 1.f;
    if (e.z.z == 0.f) {
        e.valid = false;
        return;
    }
    const float iz = 1.f / e.z.z;
    e.sx = e.z.x * iz;
    e.sy = e.z.y * iz;
    if constexpr (Filt::kAniso) {
        // s at the pixel's four corners (fwd.cu:296-320): the texture-space footprint quad
        const f3 m2v = mk3(m2.x, m2.y, m2.z);
        const f3 hx = 0.5f * cross(e.hu, m2v), hy = 0.5f * cross(e.hv, m2v);
        const f3 c0 = (e.z - hx) - hy, c1 = (e.z + hx) - hy, c2 = (e.z + hx) + hy, c3 = (e.z - hx) + hy;
        if (c0.z == 0.f || c1.z == 0.f || c2.z == 0.f || c3.z == 0.f) {
            e.valid = false;
            return;
        }
        e.g3 = e.sx * e.sx + e.sy * e.sy;
        e.dx = xyo.x - px;
        e.dy = xyo.y - py;
        e.g2 = kFilterInvSquare * (e.dx * e.dx + e.dy * e.dy);
        const float sigma = 0.5f * fminf(e.g3, e.g2);
        e.kern = __expf(-sigma);
        e.vis = 0.998f - g_weight + g_weight * e.kern;
        e.asf = 0.f;
        // the untextured alpha is tested before the footprint is sampled (fwd.cu:358-366)
        const float a0 = xyo.z * e.vis;
        if (sigma < 0.f || a0 < 1.f / 255.f) {
            e.valid = false;
            return;
        }
        const float ku = (float)(rx - 1) / (range_x * 2.f), kv = (float)(ry - 1) / (range_y * 2.f);
        e.F.s[0] = make_float2((c0.x / c0.z + range_x) * ku, (c0.y / c0.z + range_y) * kv);
        e.F.s[1] = make_float2((c1.x / c1.z + range_x) * ku, (c1.y / c1.z + range_y) * kv);
        e.F.s[2] = make_float2((c2.x / c2.z + range_x) * ku, (c2.y / c2.z + range_y) * kv);
        e.F.s[3] = make_float2((c3.x / c3.z + range_x) * ku, (c3.y / c3.z + range_y) * kv);
        e.F.convex = (c0.z > 0.f) == (c1.z > 0.f) && (c0.z > 0.f) == (c2.z > 0.f) && (c0.z > 0.f) == (c3.z > 0.f);
        const float area = aniso_setup(e.F, rx, ry);
        e.a0 = a0;
        // no texture sample: the reference zeroes alpha (fwd.cu:384-387)
        e.need = !(area == 0.f || e.F.minu == e.F.maxu || e.F.minv == e.F.maxv);
        if (e.need) e.F.iarea = 1.f / area;
        return;  // the footprint is integrated by the warp together (eval_aniso_coop)
    } else if constexpr (Filt::kMip) {
        // s at the pixel's left/right and top/bottom edge midpoints: the texture-space footprint
        // cross(hu +- hw, hv) = z +- cross(hw, hv) and cross(hu, hv +- hw) = z +- cross(hu, hw): two cross
        // products instead of four (the reference forms the four directly; rounding differs at the ulp level)
        const f3 hw = mk3(0.5f * m2.x, 0.5f * m2.y, 0.5f * m2.z);
        const f3 ax = cross(hw, e.hv), ay = cross(e.hu, hw);
        const f3 cx0 = e.z - ax, cx1 = e.z + ax;
        const f3 cy0 = e.z - ay, cy1 = e.z + ay;
        if (cx0.z == 0.f || cx1.z == 0.f || cy0.z == 0.f || cy1.z == 0.f) {
            e.valid = false;
            return;
        }
        const float dxx = cx1.x / cx1.z - cx0.x / cx0.z, dxy = cx1.y / cx1.z - cx0.y / cx0.z;
        const float dyx = cy1.x / cy1.z - cy0.x / cy0.z, dyy = cy1.y / cy1.z - cy0.y / cy0.z;
        if (mip2_taps(e.sx, e.sy, dxx, dxy, dyx, dyy, rx, mip.L, range_x, range_y, e.toff, e.w)) {
            // an integer level (e.g. t clamped to 0 under magnification): the second level's taps are the first's
            // texels again (weight 0), so they are not fetched twice
            const bool one_level = e.toff[4] == e.toff[0];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int mc = e.toff[i];
                if (i >= 4 && one_level) {
                    e.tx[i] = e.tx[i - 4];
                    continue;
                }
                e.tx[i] = mc < mip.clen ? __ldg(reinterpret_cast<const float4*>(mip.coarse) + mip.cbase + mc)
                                        : Tex::load(textures, tex_base + (mc - mip.clen), xyo.w);
            }
            e.trgba = filter_taps<8>(e.w, e.tx);
            e.asf = e.trgba.w;
            e.tex_valid = true;
        }
    } else if (kTextured) {
        if (!(e.sx < -range_x || e.sx > range_x || e.sy < -range_y || e.sy > range_y)) {
            // u = (s + range) / (2 range) * (R - 1), clamped to [0, R-1]
            const float ku = (float)(rx - 1) / (range_x * 2.f), kv = (float)(ry - 1) / (range_y * 2.f);
            const float u = fminf(fmaxf((e.sx + range_x) * ku, 0.f), (float)(rx - 1));
            const float v = fminf(fmaxf((e.sy + range_y) * kv, 0.f), (float)(ry - 1));
            // u >= 0, so truncation is floor; ceil is floor + 1 exactly when u has a fractional part
            const int ul = (int)u, vl = (int)v;
            const float wu = u - (float)ul, wv = v - (float)vl;
            const int uh = ul + (wu > 0.f), vh = vl + (wv > 0.f);
            e.w[0] = (1.f - wu) * (1.f - wv);
            e.w[1] = wu * (1.f - wv);
            e.w[2] = (1.f - wu) * wv;
            e.w[3] = wu * wv;
            e.toff[0] = vl * rx + ul;
            e.toff[1] = vl * rx + uh;
            e.toff[2] = vh * rx + ul;
            e.toff[3] = vh * rx + uh;
#pragma unroll
            for (int i = 0; i < 4; ++i) e.tx[i] = Tex::load(textures, tex_base + e.toff[i], xyo.w);
            e.trgba = filter_taps<4>(e.w, e.tx);
            e.asf = e.trgba.w;
            e.tex_valid = true;
        }
    }
    e.g3 = e.sx * e.sx + e.sy * e.sy;
    e.dx = xyo.x - px;
    e.dy = xyo.y - py;
    e.g2 = kFilterInvSquare * (e.dx * e.dx + e.dy * e.dy);
    const float sigma = 0.5f * fminf(e.g3, e.g2);
    e.kern = __expf(-sigma);
    if (kTextured) {
        e.vis = 0.998f - g_weight + g_weight * e.kern;
        e.alpha = fminf(0.999f, xyo.z * e.vis * e.asf);
    } else {
        e.vis = e.kern;
        e.alpha = fminf(0.999f, xyo.z * e.vis);
    }
    if (sigma < 0.f || e.alpha < 1.f / 255.f) e.valid = false;
}

// ---------------------------------------------------------------- anisotropic_bilinear, warp-cooperative
// A pair's footprint can span anything from one texel cell to the whole
// texture, so a lane per pixel integrating its own footprint leaves most lanes
// idle behind the largest one (measured: 4.5 of 32 lanes active per
// instruction).  Instead the warp integrates the footprints of its lanes one
// after another, each footprint's cells spread over all 32 lanes (the
// footprint is broadcast from its lane) and the partial sums reduced.

__device__ __forceinline__ AnisoFoot shfl_foot(const AnisoFoot& F, int src, unsigned mask) {
    AnisoFoot G;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        G.s[i] = make_float2(__shfl_sync(mask, F.s[i].x, src), __shfl_sync(mask, F.s[i].y, src));
        G.r[i] = make_float2(__shfl_sync(mask, F.r[i].x, src), __shfl_sync(mask, F.r[i].y, src));
        G.n[i] = make_float2(__shfl_sync(mask, F.n[i].x, src), __shfl_sync(mask, F.n[i].y, src));
        G.nmax[i] = __shfl_sync(mask, F.nmax[i], src);
    }
    G.minu = __shfl_sync(mask, F.minu, src);
    G.maxu = __shfl_sync(mask, F.maxu, src);
    G.minv = __shfl_sync(mask, F.minv, src);
    G.maxv = __shfl_sync(mask, F.maxv, src);
    G.iarea = __shfl_sync(mask, F.iarea, src);
    G.convex = __shfl_sync(mask, (int)F.convex, src) != 0;
    return G;
}

__device__ __forceinline__ float4 warp_allsum4(float4 v, unsigned mask) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(mask, v.x, o);
        v.y += __shfl_xor_sync(mask, v.y, o);
        v.z += __shfl_xor_sync(mask, v.z, o);
        v.w += __shfl_xor_sync(mask, v.w, o);
    }
    return v;
}

// Cell i of the footprint's bounding cell range, row-major.
__device__ __forceinline__ void foot_cell(const AnisoFoot& F, int i, int& u, int& v) {
    const int wu = F.maxu - F.minu;
    const int r = i / wu;
    v = F.minv + r;
    u = F.minu + (i - r * wu);
}

// Every lane calls this with its own footprint and whether it needs one
// integrated; returns the lane's own integral (not yet divided by the area).
// The warp must be full (mask = all 32 lanes).
template <class Tex, bool kShared = false>
__device__ __forceinline__ float4 aniso_coop_sum(const AnisoFoot& Fown, bool need, const void* textures,
                                                 int64_t tex_base, int rx, float scale, unsigned mask,
                                                 const float4* P = nullptr, int ry = 0, float4* s_warp = nullptr) {
    const int lane = threadIdx.x & 31;
    float4 mine = make_float4(0.f, 0.f, 0.f, 0.f);
    // with the row-prefix table, convex footprints are integrated along their boundaries (P is the same for
    // the whole warp); the others cell by cell
    if (P != nullptr) {
        mine = aniso_boundary_sum<Tex, kShared>(Fown, need && Fown.convex, textures, tex_base, P, rx, ry, scale,
                                                aniso_warp(s_warp), mask);
        need = need && !Fown.convex;
    }
    unsigned pending = __ballot_sync(mask, need);
    while (pending) {
        const int L = __ffs(pending) - 1;
        pending &= pending - 1;
        const AnisoFoot F = shfl_foot(Fown, L, mask);
        // a footprint wholly outside the texture has an empty (possibly inverted) cell range: no cells
        const int n = (F.maxu > F.minu && F.maxv > F.minv) ? (F.maxu - F.minu) * (F.maxv - F.minv) : 0;
        float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int i = lane; i < n; i += 32) {
            int u, v;
            foot_cell(F, i, u, v);
            const float4 mo = aniso_cell<kShared>(F, u, v);
            if (mo.x == 0.f && mo.y == 0.f && mo.z == 0.f && mo.w == 0.f) continue;
            const float4 w = cell_weights(mo);
            const int64_t t00 = tex_base + (int64_t)v * rx + u;
            const float4 a = Tex::load(textures, t00, scale), b = Tex::load(textures, t00 + 1, scale);
            const float4 c = Tex::load(textures, t00 + rx, scale), d = Tex::load(textures, t00 + rx + 1, scale);
            acc.x += a.x * w.x + b.x * w.y + c.x * w.z + d.x * w.w;
            acc.y += a.y * w.x + b.y * w.y + c.y * w.z + d.y * w.w;
            acc.z += a.z * w.x + b.z * w.y + c.z * w.z + d.z * w.w;
            acc.w += a.w * w.x + b.w * w.y + c.w * w.z + d.w * w.w;
        }
        acc = warp_allsum4(acc, mask);
        if (lane == L) mine = acc;
    }
    return mine;
}

// Texel-gradient scatter of every lane's footprint (gown: the lane's gradient
// already divided by the area; need: it has one), cells spread over the warp.
template <bool kShared = false>
__device__ __forceinline__ void aniso_coop_scatter(const AnisoFoot& Fown, float4 gown, bool need, float* vt, int rx,
                                                   unsigned mask, float* vP = nullptr, int ry = 0,
                                                   float4* s_warp = nullptr) {
    const int lane = threadIdx.x & 31;
    if (vP != nullptr) {  // uniform over the warp
        aniso_boundary_scatter(Fown, gown, need && Fown.convex, vt, vP, rx, ry, aniso_warp(s_warp), mask);
        need = need && !Fown.convex;
    }
    unsigned pending = __ballot_sync(mask, need);
    while (pending) {
        const int L = __ffs(pending) - 1;
        pending &= pending - 1;
        const AnisoFoot F = shfl_foot(Fown, L, mask);
        const float4 g = make_float4(__shfl_sync(mask, gown.x, L), __shfl_sync(mask, gown.y, L),
                                     __shfl_sync(mask, gown.z, L), __shfl_sync(mask, gown.w, L));
        // a footprint wholly outside the texture has an empty (possibly inverted) cell range: no cells
        const int n = (F.maxu > F.minu && F.maxv > F.minv) ? (F.maxu - F.minu) * (F.maxv - F.minv) : 0;
        for (int i = lane; i < n; i += 32) {
            int u, v;
            foot_cell(F, i, u, v);
            const float4 mo = aniso_cell<kShared>(F, u, v);
            if (mo.x == 0.f && mo.y == 0.f && mo.z == 0.f && mo.w == 0.f) continue;
            const float4 w = cell_weights(mo);
            float4* t00 = reinterpret_cast<float4*>(vt + 4 * ((int64_t)v * rx + u));
            atomicAdd(t00, make_float4(g.x * w.x, g.y * w.x, g.z * w.x, g.w * w.x));
            atomicAdd(t00 + 1, make_float4(g.x * w.y, g.y * w.y, g.z * w.y, g.w * w.y));
            atomicAdd(t00 + rx, make_float4(g.x * w.z, g.y * w.z, g.z * w.z, g.w * w.z));
            atomicAdd(t00 + rx + 1, make_float4(g.x * w.w, g.y * w.w, g.z * w.w, g.w * w.w));
        }
    }
}

// The anisotropic_bilinear pair evaluation for a whole (full) warp working on
// one splat: every lane calls it, act = the lane has a pair to evaluate; the
// footprints that need integrating are integrated by the warp together.
template <class Tex, bool kShared = false>
__device__ __forceinline__ void eval_aniso_coop(PairEvalAniso& e, bool act, float px, float py, const float4 xyo,
                                                const float4 m0, const float4 m1, const float4 m2,
                                                const void* textures, int64_t tex_base, int rx, int ry, float range_x,
                                                float range_y, float g_weight, unsigned mask,
                                                const float4* P = nullptr, float4* s_warp = nullptr,
                                                const float4* rec = nullptr) {
    e.valid = false;
    e.need = false;
    e.tex_valid = false;
    if (act)
        eval_pair<Tex, FiltAniso>(e, px, py, xyo, m0, m1, m2, textures, tex_base, rx, ry, range_x, range_y, g_weight);
    const bool need = act && e.valid && e.need;
    const bool have = need && rec != nullptr;  // rec: the forward's record of this footprint's integral
    if (need && (P == nullptr || !e.F.convex)) aniso_cells_setup(e.F);  // integrated (or scattered) cell by cell
    float4 ts = aniso_coop_sum<Tex, kShared>(e.F, need && !have, textures, tex_base, rx, xyo.w, mask, P, ry, s_warp);
    if (have) ts = *rec;
    if (!(act && e.valid)) return;
    e.asf = 0.f;
    if (need) {
        e.tsum = ts;
        e.tex_valid = true;
        e.asf = ts.w * e.F.iarea;
    }
    e.alpha = fminf(0.999f, e.a0 * e.asf);
    if (e.alpha < 1.f / 255.f) e.valid = false;
}

// Pixel-space box outside of which a (pixel, splat) pair is provably invalid
// (alpha < 1/255), so skipping it leaves every output unchanged.
//
// A pair is valid only if opac * vis * asf >= 1/255 with
// vis = 0.998 - g_weight + g_weight exp(-sigma), sigma = min(|s|^2, 2|d|^2) / 2.
// Outside the texture square |s_x| <= range_x, |s_y| <= range_y the texture
// alpha scale asf is exactly 1, so validity there needs sigma <= sigma1 with
// exp(-sigma1) = (1/(255 opac) - 0.998 + g_weight) / g_weight: either the UV
// point lies in the disk |s|^2 <= 2 sigma1 (inside the square of half-side
// sqrt(2 sigma1)) or the pixel lies within sqrt(sigma1) of the projected
// centre.  Inside the texture square anything is possible.  The UV squares map
// to pixel space through the splat's homography pixel(s) = (M0.(s,1),
// M1.(s,1)) / M2.(s,1); when M2.(s,1) has one sign at all four corners the
// image is a bounded convex quadrilateral, whose corners' box bounds it.
// Otherwise (or if no bound on sigma exists) the box is unbounded.  The
// anisotropic_bilinear filter tests opac * vis >= 1/255 before any texture
// term, so for it (tex_square = false) the texture square drops out.  The box is
// widened by a margin that covers FP32 rounding of the pair evaluation.
__device__ __forceinline__ float4 cull_box(const float4 xyo, const float4 m0, const float4 m1, const float4 m2,
                                           bool textured, float range_x, float range_y, float g_weight,
                                           bool tex_square = true) {
    const float4 all = make_float4(-INFINITY, -INFINITY, INFINITY, INFINITY);
    const float opac = xyo.z;
    float K;  // lower bound on exp(-sigma) for a valid pair outside the texture square
    if (textured) {
        if (!(g_weight > 0.f)) return all;
        K = (1.f / (255.f * opac) - 0.998f + g_weight) / g_weight;
    } else {
        K = 1.f / (255.f * opac);
    }
    K *= 0.999f;  // rounding slack: never cull a pair the evaluation could still accept
    if (!(K > 0.f)) return all;
    const float sig1 = K >= 1.f ? 0.f : -logf(K) * 1.001f + 1e-3f;
    const float rs = sqrtf(2.f * sig1);   // half-side of the UV square around the Gaussian disk
    const float rd = sqrtf(sig1);         // radius of the 2D-filter disk, pixels
    const float hx = textured && tex_square ? fmaxf(rs, range_x) : rs;
    const float hy = textured && tex_square ? fmaxf(rs, range_y) : rs;
    float x0 = xyo.x - rd, x1 = xyo.x + rd, y0 = xyo.y - rd, y1 = xyo.y + rd;
    int pos = 0, neg = 0;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const float u = (c & 1) ? hx : -hx, v = (c & 2) ? hy : -hy;
        const float X = m0.x * u + m0.y * v + m0.z;
        const float Y = m1.x * u + m1.y * v + m1.z;
        const float Z = m2.x * u + m2.y * v + m2.z;
        pos += Z > 0.f;
        neg += Z < 0.f;
        const float iz = 1.f / Z;
        const float px = X * iz, py = Y * iz;
        x0 = fminf(x0, px); x1 = fmaxf(x1, px);
        y0 = fminf(y0, py); y1 = fmaxf(y1, py);
    }
    if (!(pos == 4 || neg == 4)) return all;
    const float margin = 1.f + 1e-3f * ((x1 - x0) + (y1 - y0));
    const float4 box = make_float4(x0 - margin, y0 - margin, x1 + margin, y1 + margin);
    if (!(box.x == box.x && box.y == box.y && box.z == box.z && box.w == box.w) ||
        !(fabsf(box.x) < 1e30f && fabsf(box.y) < 1e30f && fabsf(box.z) < 1e30f && fabsf(box.w) < 1e30f))
        return all;
    return box;
}

__device__ __forceinline__ bool in_box(const float4 b, float px, float py) {
    return px >= b.x && px <= b.z && py >= b.y && py <= b.w;
}

// Texture contribution to colour channel k (channels >= 4 have none).
template <int NT>
__device__ __forceinline__ float tex_color(const PairEvalT<NT>& e, int k) {
    return (k >= 4 || !e.tex_valid) ? 0.f : f4get(e.trgba, k);
}
__device__ __forceinline__ float tex_color(const PairEvalAniso& e, int k) {
    return (k >= 4 || !e.tex_valid) ? 0.f : f4get(e.tsum, k) * e.F.iarea;
}

// The texture colour the adjoint uses: the forward's, except that the
// anisotropic_bilinear adjoint of the reference omits the division by the
// footprint area (bwd.cu:499-522 with filters/anisotropic_bilinear.cuh:372-389).
template <int NT>
__device__ __forceinline__ float tex_color_adj(const PairEvalT<NT>& e, int k) { return tex_color(e, k); }
__device__ __forceinline__ float tex_color_adj(const PairEvalAniso& e, int k) {
    return (k >= 4 || !e.tex_valid) ? 0.f : f4get(e.tsum, k);
}

// Sum over the lanes in `mask`; lanes outside it contribute zero.  The
// butterfly reads lane^o, which exists whenever the mask is a prefix of
// lanes whose count is a power of two, or the full warp.
__device__ __forceinline__ float warp_sum(float v, unsigned mask) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float u = __shfl_xor_sync(mask, v, o);
        if (((threadIdx.x & 31) ^ o) < 32 && (mask >> ((threadIdx.x & 31) ^ o)) & 1u) v += u;
    }
    return v;
}

// The tile a CTA works on and the image it belongs to.  Work item `item`
// (blockIdx.x) maps to flat tile tile_order[item] (or item); the flat tile
// maps to (view, tile x, tile y) through the view table in the batching form,
// or through the one tile grid otherwise.  valid is false for an item whose
// tile or view index is out of range (the CTA then does nothing).
struct TileWork {
    int c, tx, ty;
    int64_t t;
    int width, height;
    int64_t pix_base;   // first flat pixel of the view
    int64_t pix_limit;  // pixels of all views: every pixel index is checked against it
    int32_t range_start, range_end;
    bool valid;
};

__device__ __forceinline__ TileWork tile_work(const tg_raster_fwd_args& a, int64_t item) {
    TileWork w;
    const int64_t per_cam = (int64_t)a.tile_width * a.tile_height;
    const int64_t n_tiles = a.views ? a.n_tiles : (int64_t)a.C * per_cam;
    w.t = a.tile_order ? (int64_t)a.tile_order[item] : item;
    w.valid = w.t >= 0 && w.t < n_tiles;
    if (!w.valid) return w;
    if (a.views) {
        w.c = a.tile_view[w.t];
        w.valid = w.c >= 0 && w.c < a.C;
        if (!w.valid) return w;
        const tg_view v = a.views[w.c];
        const int64_t local = w.t - v.tile_base;
        w.valid = v.tile_width > 0 && local >= 0 && local < (int64_t)v.tile_width * v.tile_height;
        if (!w.valid) return w;
        w.ty = (int)(local / v.tile_width);
        w.tx = (int)(local - (int64_t)w.ty * v.tile_width);
        w.width = v.width;
        w.height = v.height;
        w.pix_base = v.pix_base;
        w.pix_limit = a.n_pixels;
    } else {
        w.c = (int)(w.t / per_cam);
        const int64_t local = w.t - (int64_t)w.c * per_cam;
        w.ty = (int)(local / a.tile_width);
        w.tx = (int)(local - (int64_t)w.ty * a.tile_width);
        w.width = a.width;
        w.height = a.height;
        w.pix_base = (int64_t)w.c * a.height * a.width;
        w.pix_limit = (int64_t)a.C * a.height * a.width;
    }
    // capacity mode: the valid intersections are the first *n_isects_dev of the n_isects entries
    const int64_t n_valid = a.n_isects_dev ? min(max(*a.n_isects_dev, (int64_t)0), a.n_isects) : a.n_isects;
    w.range_start = min(a.tile_offsets[w.t], (int32_t)n_valid);
    w.range_end = w.t == n_tiles - 1 ? (int32_t)n_valid : min(a.tile_offsets[w.t + 1], (int32_t)n_valid);
    return w;
}

// Flat index of pixel (i, j) of the work item's view, or -1 outside the view
// or the flat outputs.
__device__ __forceinline__ int64_t pixel_index(const TileWork& w, int i, int j) {
    if (i >= w.height || j >= w.width) return -1;
    const int64_t p = w.pix_base + (int64_t)i * w.width + j;
    return (p >= 0 && p < w.pix_limit) ? p : -1;
}

// Grid of a persistent launch: every CTA that fits on the device at once, at
// most one per work item.
inline cudaError_t persistent_grid(const void* fn, int threads, size_t smem, int64_t n_items, int64_t& grid) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem);
    if (e != cudaSuccess) return e;
    grid = std::min<int64_t>(n_items, (int64_t)std::max(sms, 1) * std::max(per_sm, 1));
    return cudaSuccess;
}

}  // namespace tg
