"""CPU check of the compositor's boundary integration of the anisotropic_bilinear
filter (Green's theorem over row-prefix tables) against the oracle's polygon
clipping (the reference's clip_and_compute_moments,
filters/anisotropic_bilinear.cuh:58-190, summed cell by cell).

For a convex footprint quad the CUDA kernels (foot_segments, walk_cells,
piece_weights, segment_sum and segment_scatter in
textured_gaussians_b200/csrc/raster_common.cuh; the prefix table and its fold
in textured_gaussians_b200/csrc/aniso.cu) integrate the bilinear interpolant f
over the quad clipped to the texel grid [0, rx-1] x [0, ry-1] as the closed
line integral of F dy, F(x, y) = integral of f(s, y) ds from column x0 (the
footprint's first cell column) to x, read from the rows' prefix integrals:
the quad's edges clipped to the grid plus the grid's right edge inside the
quad, walked cell by cell, each piece integrated by two-point Gauss-Legendre
(exact: F is cubic along a piece).  The adjoint leaves out the x0 terms (they
integrate a function of y alone around a closed curve) and accumulates
prefix-table gradients that a transposed scan folds back into the texels.

This test restates those steps in FP64 and checks (1) the filtered value
against the oracle on quads built to hit the special cases -- edges on grid
lines (both windings), an edge lying on the grid's right edge (with the quad
inside and outside it), axis-parallel edges, corners on grid vertices, quads
reaching past the grid, slivers, footprints within one cell, and random convex
quads -- and (2) that the adjoint with the fold is the exact transpose of the
forward (random texture perturbations).
"""
import math

import numpy as np
import pytest

from oracle import oracle as O

KG = (1.0 - 1.0 / math.sqrt(3.0)) / 2.0  # the two-point Gauss-Legendre nodes on [0, 1]: KG and 1 - KG


def _clip(p, q, t0, t1):
    if q > 0:
        t0 = max(t0, -p / q)
    elif q < 0:
        t1 = min(t1, -p / q)
    return (q != 0 or p >= 0), t0, t1


def _oriented(s):
    s = [tuple(map(float, p)) for p in s]
    area = 0.5 * sum(s[i][0] * s[(i + 1) % 4][1] - s[(i + 1) % 4][0] * s[i][1] for i in range(4))
    if area < 0:
        area = -area
        s[1], s[3] = s[3], s[1]
    return s, area


def _segments(s, rx, ry):
    """foot_segments: the quad's edges clipped to the grid, then the grid's right edge clipped to the quad."""
    X1, Y1 = rx - 1.0, ry - 1.0
    out = []
    for i in range(4):
        a, b = s[i], s[(i + 1) % 4]
        d = (b[0] - a[0], b[1] - a[1])
        t0, t1, ok = 0.0, 1.0, True
        for p, q in ((a[0], d[0]), (X1 - a[0], -d[0]), (a[1], d[1]), (Y1 - a[1], -d[1])):
            k, t0, t1 = _clip(p, q, t0, t1)
            ok = ok and k
        if ok and t0 < t1:
            out.append(((a[0] + t0 * d[0], a[1] + t0 * d[1]), (a[0] + t1 * d[0], a[1] + t1 * d[1])))
    t0, t1, keep = 0.0, 1.0, True
    for i in range(4):
        e = (s[(i + 1) % 4][0] - s[i][0], s[(i + 1) % 4][1] - s[i][1])
        p = e[0] * (0.0 - s[i][1]) - e[1] * (X1 - s[i][0])
        q = e[0] * Y1
        k, t0, t1 = _clip(p, q, t0, t1)
        keep = keep and ((p > 0 or (p == 0 and e[1] < 0)) if q == 0 else k)
    if keep and t0 < t1:
        out.append(((X1, t0 * Y1), (X1, t1 * Y1)))
    return out


def _walk(a, b, rx, ry):
    """walk_cells: the pieces of a -> b in the cells it crosses (cells clamped to the grid), dy != 0 only."""
    dx, dy = b[0] - a[0], b[1] - a[1]
    if dy == 0:
        return []
    ix = math.floor(a[0]) if dx >= 0 else math.ceil(a[0]) - 1
    iy = math.floor(a[1]) if dy >= 0 else math.ceil(a[1]) - 1
    sx = 1 if dx > 0 else (-1 if dx < 0 else 0)
    sy = 1 if dy > 0 else -1
    t, p, out = 0.0, a, []
    for _ in range(2 * (rx + ry) + 8):
        tx = math.inf if sx == 0 else ((ix + 1 if sx > 0 else ix) - a[0]) / dx
        ty = ((iy + 1 if sy > 0 else iy) - a[1]) / dy
        tn = min(tx, ty, 1.0)
        q = b if tn >= 1 else (a[0] + tn * dx, a[1] + tn * dy)
        if tn > t:
            out.append((p, q, min(max(ix, 0), rx - 2), min(max(iy, 0), ry - 2)))
        if tn >= 1:
            return out
        if tx <= tn:
            ix += sx
        if ty <= tn:
            iy += sy
        t, p = tn, q
    raise AssertionError("walk did not end")


def _weights(a, b, u, v):
    """piece_weights: (texel a, b, c, d, prefix row v, prefix row v+1) weights of one piece."""
    dx, dy = b[0] - a[0], b[1] - a[1]
    w = np.zeros(6)
    for tq in (KG, 1.0 - KG):
        x, y = a[0] - u + tq * dx, a[1] - v + tq * dy
        x2 = 0.5 * x * x
        x1 = x - x2
        w += [(1 - y) * x1, (1 - y) * x2, y * x1, y * x2, 1 - y, y]
    return w * 0.5 * dy


def _prefix(tex):
    P = np.zeros_like(tex)
    P[:, 1:] = np.cumsum(0.5 * (tex[:, :-1] + tex[:, 1:]), axis=1)
    return P


def _cell_range(s, rx, ry):
    xs, ys = [p[0] for p in s], [p[1] for p in s]
    minu, maxu = max(0, math.floor(min(xs))), min(rx - 1, math.ceil(max(xs)))
    minv, maxv = max(0, math.floor(min(ys))), min(ry - 1, math.ceil(max(ys)))
    return minu, maxu, minv, maxv


def boundary_integral(corners, tex):
    """The kernels' integral (before the division by the area) and the quad's area."""
    ry, rx = tex.shape[:2]
    s, area = _oriented(corners)
    minu, maxu, minv, maxv = _cell_range(s, rx, ry)
    acc = np.zeros(tex.shape[2])
    if not (maxu > minu and maxv > minv):
        return acc, area
    P, x0 = _prefix(tex), minu
    for a, b in _segments(s, rx, ry):
        for pa, pb, u, v in _walk(a, b, rx, ry):
            w = _weights(pa, pb, u, v)
            p0 = P[v, u] - P[v, x0] if u != x0 else 0.0
            p1 = P[v + 1, u] - P[v + 1, x0] if u != x0 else 0.0
            acc += (w[0] * tex[v, u] + w[1] * tex[v, u + 1] + w[2] * tex[v + 1, u] + w[3] * tex[v + 1, u + 1]
                    + w[4] * p0 + w[5] * p1)
    return acc, area


def boundary_adjoint(corners, g, shape):
    """segment_scatter (each piece's six weights, no x0 terms) plus the prefix fold."""
    ry, rx = shape[:2]
    s, _ = _oriented(corners)
    minu, maxu, minv, maxv = _cell_range(s, rx, ry)
    vt, vP = np.zeros(shape), np.zeros(shape)
    if not (maxu > minu and maxv > minv):
        return vt
    for a, b in _segments(s, rx, ry):
        for pa, pb, u, v in _walk(a, b, rx, ry):
            w = _weights(pa, pb, u, v)
            vt[v, u] += g * w[0]
            vt[v, u + 1] += g * w[1]
            vt[v + 1, u] += g * w[2]
            vt[v + 1, u + 1] += g * w[3]
            vP[v, u] += g * w[4]
            vP[v + 1, u] += g * w[5]
    # the fold (aniso_prefix_fold_kernel): dt(0) = S(1) / 2, dt(j) = (S(j) + S(j+1)) / 2, S(j) = sum_{u>=j} dP[u]
    for r in range(ry):
        dP = vP[r].copy()
        dP[0] = 0.0
        S = np.zeros((rx + 1,) + shape[2:])
        S[:rx] = np.cumsum(dP[::-1], axis=0)[::-1]
        for j in range(rx):
            vt[r, j] += 0.5 * S[j + 1] + (0.5 * S[j] if j > 0 else 0.0)
    return vt


def _has_zero_edge(s):
    return any(tuple(s[i]) == tuple(s[(i + 1) % 4]) for i in range(4))


def _check(corners, tex):
    corners = np.asarray(corners, float)
    got, area = boundary_integral(corners, tex)
    ref, area_o = O.aniso_sample(corners, tex)
    assert area == pytest.approx(area_o, rel=1e-12, abs=1e-12)
    if area == 0:
        return
    scale = max(1.0, float(np.abs(ref).max()))
    assert np.abs(got / area - ref).max() <= 1e-10 * scale, (corners.tolist(), got / area, ref)


SPECIAL = [
    [(1, 1), (3, 1), (3, 3), (1, 3)],                 # edges on grid lines
    [(1, 3), (3, 3), (3, 1), (1, 1)],                 # the same, clockwise
    [(5, 2), (7, 2), (7, 4), (5, 4)],                 # right edge on the grid's right edge x = rx - 1 (rx = 8)
    [(7, 2), (9, 2), (9, 4), (7, 4)],                 # left edge on it, the quad outside the grid
    [(6.5, 2.0), (7.0, 2.5), (7.0, 3.0), (6.0, 2.5)],  # a corner and an edge on it
    [(-2, -1), (9.5, -1), (9.5, 8.5), (-2, 8.5)],     # the whole grid inside the quad
    [(0.2, 0.3), (0.7, 0.3), (0.7, 0.9), (0.2, 0.9)],  # within one cell
    [(0.5, 0.5), (6.5, 6.4), (6.6, 6.5), (0.6, 0.6)],  # a diagonal sliver
    [(2, 0), (4, 2), (2, 4), (0, 2)],                 # corners on grid vertices, edges at 45 degrees
    [(-1.5, 3.2), (2.5, 1.1), (3.7, 6.6), (0.1, 9.3)],  # reaching past two sides
    [(3.3, 2.0), (5.1, 2.0), (5.1, 2.0 + 1e-9), (3.3, 2.0 + 1e-9)],  # nearly flat
]


@pytest.mark.parametrize("k", range(len(SPECIAL)))
def test_boundary_integral_matches_oracle_on_special_quads(k):
    rng = np.random.default_rng(100 + k)
    _check(SPECIAL[k], rng.normal(size=(8, 8, 4)))


def test_boundary_integral_matches_oracle_on_random_convex_quads():
    rng = np.random.default_rng(7)
    n = 0
    for _ in range(400):
        ry, rx = int(rng.choice([2, 3, 8, 32])), int(rng.choice([2, 5, 8, 32]))
        tex = rng.normal(size=(ry, rx, 4))
        c = np.array([rng.uniform(-0.3 * rx, 1.3 * rx), rng.uniform(-0.3 * ry, 1.3 * ry)])
        sc = 10 ** rng.uniform(-1.5, 1.3)
        ang, an = rng.uniform(0, 2 * np.pi), rng.uniform(0.05, 1)
        A = np.array([[np.cos(ang), -np.sin(ang)], [np.sin(ang), np.cos(ang)]]) @ np.diag([sc, sc * an])
        sq = np.array([[-1, -1], [1, -1], [1, 1], [-1, 1]], float)
        if rng.uniform() < 0.5:
            sq = sq[::-1]
        H = np.eye(3)
        H[2, :2] = rng.uniform(-0.3, 0.3, 2)  # a projective image of a square (w > 0: convex)
        pts = np.c_[sq, np.ones(4)] @ H.T
        s = (pts[:, :2] / pts[:, 2:]) @ A.T + c
        if rng.uniform() < 0.25:
            s = np.round(s * 2) / 2  # corners and edges on grid lines
        if _has_zero_edge(s):
            continue  # the kernels take the polygon clipping for these
        _check(s, tex)
        n += 1
    assert n > 350


def test_adjoint_with_fold_is_the_transpose_of_the_integral():
    rng = np.random.default_rng(11)
    n = 0
    for k in range(120):
        ry, rx = int(rng.choice([2, 4, 8])), int(rng.choice([2, 5, 8]))
        tex = rng.normal(size=(ry, rx, 4))
        s = SPECIAL[k % len(SPECIAL)] if k < len(SPECIAL) else \
            [(rng.uniform(-1, rx), rng.uniform(-1, ry)) for _ in range(4)]
        s, _ = _oriented(s)
        # keep convex quads only (random corners may cross): every turn the same way
        e = [np.subtract(s[(i + 1) % 4], s[i]) for i in range(4)]
        if any(e[i][0] * e[(i + 1) % 4][1] - e[i][1] * e[(i + 1) % 4][0] <= 0 for i in range(4)):
            continue
        g = rng.normal(size=4)
        vt = boundary_adjoint(s, g, tex.shape)
        d = rng.normal(size=tex.shape)
        i0, _ = boundary_integral(s, tex)
        i1, _ = boundary_integral(s, tex + d)
        lhs = float(g @ (i1 - i0))  # the integral is linear in the texture
        rhs = float((vt * d).sum())
        assert abs(lhs - rhs) <= 1e-10 * max(1.0, abs(lhs)), (k, lhs, rhs)
        n += 1
    assert n >= 30, n
