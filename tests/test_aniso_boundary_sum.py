"""CPU check of the compositor's convex-footprint formulation of the
anisotropic_bilinear filter against the oracle's polygon clipping.

For a convex footprint quad the CUDA kernels (aniso_cell / cell_edges_sum /
clip_t in textured_gaussians_b200/csrc/raster_common.cuh) do not clip the quad
polygon to each texel cell (the reference's clip_and_compute_moments,
filters/anisotropic_bilinear.cuh:58-190); they sum the clipped polygon's
boundary piecewise -- the quad's edges clipped to the cell plus the cell's
edges clipped to the quad, each a parametric clip against four half-planes
done without branches and one interval test at the end -- with the
reference's whole-cell fast path and a skip for cells wholly outside.  This
test restates that formulation in FP64 and compares the filtered value with
the oracle on quads built to hit its special cases: quad edges lying on cell
edges (both directions), edges parallel to an axis (zero clip divisor), a
collapsed corner (a zero-length edge), quads reaching outside the texel grid,
and random convex quads in both windings.  A quad with a zero-length edge (a
collapsed corner) takes the polygon clipping: that edge's half-plane has
divisor and offset 0, on which the boundary sum's on-edge rule would drop
every cell edge of the cells it touches.
"""
import math
import zlib

import numpy as np
import pytest

from oracle import oracle as O


def _cross(a, b):
    return a[0] * b[1] - a[1] * b[0]


def _setup(s, rx, ry):
    """Orientation, cell range, normals and margins (aniso_setup)."""
    s = [np.array(p, float) for p in s]
    area = 0.5 * (_cross(s[1] - s[0], s[2] - s[1]) + _cross(s[3] - s[2], s[0] - s[3]))
    if area < 0:
        area = -area
        s[1], s[3] = s[3], s[1]
    e = [s[(i + 1) % 4] - s[i] for i in range(4)]
    xs, ys = [p[0] for p in s], [p[1] for p in s]
    minu, maxu = max(0, math.floor(min(xs))), min(rx - 1, math.ceil(max(xs)))
    minv, maxv = max(0, math.floor(min(ys))), min(ry - 1, math.ceil(max(ys)))
    cen = sum(s) / 4
    n, nmax = [], []
    for i in range(4):
        v = (s[i] - cen) if (e[i] == 0).all() else np.array([e[i][1], -e[i][0]])
        ln = math.hypot(*v)
        v = v / ln if ln else v
        n.append(v)
        nmax.append(max(abs(0.5 * v[0] + 0.5 * v[1]), abs(0.5 * v[0] - 0.5 * v[1])))
    return s, e, n, nmax, (minu, maxu, minv, maxv), area


def _clip(p, q, t0, t1):
    """clip_t: narrow [t0, t1] to p + t q >= 0 without branching on the interval; False only when q = 0, p < 0."""
    if q > 0:
        t0 = max(t0, -p / q)
    elif q < 0:
        t1 = min(t1, -p / q)
    return (q != 0 or p >= 0), t0, t1


def _seg(a, b, m):
    c = a[0] * b[1] - a[1] * b[0]
    m[0] += c
    m[1] += c * (a[0] + b[0])
    m[2] += c * (a[1] + b[1])
    m[3] += c * (2 * a[0] * a[1] + a[0] * b[1] + b[0] * a[1] + 2 * b[0] * b[1])


def _cell(s, e, n, nmax, u, v, convex=True):
    """Moments (A, Sx, Sy, Sxy) of the quad clipped to cell (u, v), cell-local (aniso_cell): the whole-cell fast
    path, then the polygon clipping for a quad that is not convex, else the outside skip and the boundary sum."""
    c = np.array([u + 0.5, v + 0.5])
    d = [(s[i] - c) @ n[i] for i in range(4)]
    if all(d[i] >= nmax[i] for i in range(4)):
        return np.array([1.0, 0.5, 0.5, 0.25])
    if not convex:
        return _cell_polygon(s, u, v)
    if any(d[i] < -nmax[i] and (e[i] != 0).any() for i in range(4)):
        return np.zeros(4)
    m = np.zeros(4)
    for i in range(4):  # quad edges inside the cell
        a, dd = s[i] - (u, v), e[i]
        t0, t1, keep = 0.0, 1.0, True
        for p, q in ((a[0], dd[0]), (1 - a[0], -dd[0]), (a[1], dd[1]), (1 - a[1], -dd[1])):
            k, t0, t1 = _clip(p, q, t0, t1)
            keep &= k
        if keep and t0 < t1:
            _seg(a + t0 * dd, a + t1 * dd, m)
    for j in range(4):  # cell edges inside the quad, counter-clockwise
        a = np.array([1.0 if j in (1, 2) else 0.0, 1.0 if j >= 2 else 0.0])
        dd = np.array([[1.0, 0.0], [0.0, 1.0], [-1.0, 0.0], [0.0, -1.0]][j])
        t0, t1, keep = 0.0, 1.0, True
        for i in range(4):
            r = a + (u, v) - s[i]
            p, q = _cross(e[i], r), _cross(e[i], dd)
            par = p > 0 or (p == 0 and e[i] @ dd < 0)  # on the quad edge: kept only running the other way
            k, t0, t1 = _clip(p, q, t0, t1)
            keep &= par if q == 0 else k
        if keep and t0 < t1:
            _seg(a + t0 * dd, a + t1 * dd, m)
    return m * np.array([0.5, 1 / 6, 1 / 6, 1 / 24])


def _sh_clip(p, axis, hi):
    """One Sutherland-Hodgman pass against x or y >= 0 (hi: <= 1); None past 8 vertices (sh_clip)."""
    out = []
    for i in range(len(p)):
        a, b = p[i], p[(i + 1) % len(p)]
        ac, bc = a[axis], b[axis]
        ain, bin_ = (ac <= 1, bc <= 1) if hi else (ac >= 0, bc >= 0)
        if ain:
            out.append(a)
        if ain != bin_:
            t = (ac - 1) / (ac - bc) if hi else ac / (ac - bc)
            edge = 1.0 if hi else 0.0
            out.append(np.array([a[0] + t * (b[0] - a[0]), edge]) if axis else np.array([edge, a[1] + t * (b[1] - a[1])]))
        if len(out) > 8:
            return None
    return out


def _cell_polygon(s, u, v):
    """The polygon clipping the kernels keep for the other quads (aniso_cell_polygon)."""
    p = [si - (u, v) for si in s]
    for axis, hi in ((0, False), (0, True), (1, False), (1, True)):
        p = _sh_clip(p, axis, hi)
        if p is None or len(p) < 3:
            return np.zeros(4)
    m = np.zeros(4)
    for i in range(len(p)):
        _seg(p[i], p[(i + 1) % len(p)], m)
    return m * np.array([0.5, 1 / 6, 1 / 6, 1 / 24])


def boundary_sum_filter(corners, tex, convex=None):
    """The kernels' anisotropic_bilinear value of one quad over tex [ry, rx, 4]: the boundary sum for a quad
    without a zero-length edge, the polygon clipping otherwise (the quads here have corners on one side of
    the splat plane)."""
    ry, rx = tex.shape[:2]
    s, e, n, nmax, (minu, maxu, minv, maxv), area = _setup(corners, rx, ry)
    if convex is None:  # the kernels also clear it when the corner rays straddle the splat plane
        convex = all((ei != 0).any() for ei in e)
    convex = convex and all((ei != 0).any() for ei in e)
    acc = np.zeros(4)
    for v in range(minv, maxv):
        for u in range(minu, maxu):
            mo = _cell(s, e, n, nmax, u, v, convex)
            w = np.array([mo[0] - mo[1] - mo[2] + mo[3], mo[1] - mo[3], mo[2] - mo[3], mo[3]])
            acc += w[0] * tex[v, u] + w[1] * tex[v, u + 1] + w[2] * tex[v + 1, u] + w[3] * tex[v + 1, u + 1]
    return acc / area if area > 0 else acc, area


ADVERSARIAL = {
    # edges on the grid lines v = 3 and v = 6, counter-clockwise and clockwise
    "edges_on_grid_ccw": [(2.3, 3.0), (5.7, 3.0), (5.7, 6.0), (2.3, 6.0)],
    "edges_on_grid_cw": [(2.3, 6.0), (5.7, 6.0), (5.7, 3.0), (2.3, 3.0)],
    # every edge on a grid line: whole cells only
    "integer_rectangle": [(2.0, 3.0), (6.0, 3.0), (6.0, 5.0), (2.0, 5.0)],
    # axis-parallel but off the grid (zero clip divisors, nonzero offsets)
    "axis_parallel": [(1.25, 2.75), (4.5, 2.75), (4.5, 5.125), (1.25, 5.125)],
    # a collapsed corner: a triangle with a zero-length edge
    "collapsed_corner": [(1.5, 1.5), (5.5, 2.5), (5.5, 2.5), (2.5, 5.5)],
    # a thin sliver along a diagonal
    "sliver": [(1.1, 1.0), (6.9, 6.8), (7.0, 7.0), (1.0, 1.2)],
    # reaching outside the texel grid on two sides
    "outside_grid": [(-1.5, 2.2), (3.3, -0.7), (5.4, 3.9), (0.6, 6.1)],
    # a corner exactly on a grid vertex with a diagonal edge through grid vertices
    "grid_vertices": [(2.0, 2.0), (5.0, 2.0), (5.0, 5.0), (3.5, 6.5)],
}


@pytest.mark.parametrize("name", sorted(ADVERSARIAL))
def test_adversarial_quads_match_polygon_clipping(name):
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    tex = rng.uniform(-1, 1, size=(9, 9, 4))
    q = np.array(ADVERSARIAL[name], float)
    ref, ref_area = O.aniso_sample(q, tex)
    out, area = boundary_sum_filter(q, tex)
    assert abs(area - ref_area) <= 1e-12 * max(1.0, ref_area)
    np.testing.assert_allclose(out, ref, rtol=0, atol=1e-12)


@pytest.mark.parametrize("seed", range(12))
def test_random_convex_quads_match_polygon_clipping(seed):
    rng = np.random.default_rng(100 + seed)
    R = 12
    tex = rng.uniform(-1, 1, size=(R, R, 4))
    for _ in range(6):
        # a convex quad: four points at increasing angles around a centre, possibly reaching past the grid
        c = rng.uniform(-1, R, size=2)
        ang = np.sort(rng.uniform(0, 2 * np.pi, size=4))
        rad = rng.uniform(0.3, 4.0, size=4)
        q = c + np.stack([rad * np.cos(ang), rad * np.sin(ang)], 1)
        if not all(_cross(q[(i + 1) % 4] - q[i], q[(i + 2) % 4] - q[(i + 1) % 4]) > 0 for i in range(4)):
            continue  # not strictly convex
        if seed % 2:
            q = q[::-1].copy()
        ref, ref_area = O.aniso_sample(q, tex)
        out, area = boundary_sum_filter(q, tex)
        assert abs(area - ref_area) <= 1e-12 * max(1.0, ref_area)
        np.testing.assert_allclose(out, ref, rtol=0, atol=1e-11)


def test_collapsed_corner_needs_the_polygon_clipping():
    """The boundary sum on its own loses the cell edges of a quad with a zero-length edge (hence the routing)."""
    tex = np.random.default_rng(3).uniform(-1, 1, size=(9, 9, 4))
    q = np.array(ADVERSARIAL["collapsed_corner"], float)
    ref, _ = O.aniso_sample(q, tex)
    s, e, n, nmax, (minu, maxu, minv, maxv), area = _setup(q, 9, 9)
    acc = np.zeros(4)
    for v in range(minv, maxv):
        for u in range(minu, maxu):
            mo = _cell(s, e, n, nmax, u, v)
            w = np.array([mo[0] - mo[1] - mo[2] + mo[3], mo[1] - mo[3], mo[2] - mo[3], mo[3]])
            acc += w[0] * tex[v, u] + w[1] * tex[v, u + 1] + w[2] * tex[v + 1, u] + w[3] * tex[v + 1, u + 1]
    assert np.abs(acc / area - ref).max() > 1e-3
    np.testing.assert_allclose(boundary_sum_filter(q, tex)[0], ref, rtol=0, atol=1e-12)


@pytest.mark.parametrize("quad", [[(1.0, 1.0), (6.0, 4.0), (6.0, 1.5), (1.5, 4.5)],
                                  [(2.2, 1.3), (6.7, 6.1), (1.4, 6.6), (6.9, 2.0)]])
def test_self_intersecting_quads_take_the_polygon_clipping(quad):
    """Corner rays on both sides of the splat plane give a self-intersecting quad; the kernels then use the
    reference's polygon clipping (after the whole-cell fast path), which the oracle restates too."""
    tex = np.random.default_rng(9).uniform(-1, 1, size=(9, 9, 4))
    q = np.array(quad, float)
    ref, ref_area = O.aniso_sample(q, tex)
    out, area = boundary_sum_filter(q, tex, convex=False)
    assert abs(area - ref_area) <= 1e-12 * max(1.0, ref_area)
    np.testing.assert_allclose(out, ref, rtol=0, atol=1e-12)
