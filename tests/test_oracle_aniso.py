"""CPU checks of the oracle's anisotropic_bilinear footprint filter against
closed forms: the filter integrates the texture's bilinear interpolant over
the footprint quad and divides by the quad's area, so a constant texture gives
the constant and a texture that is linear in (u, v) gives its value at the
quad's centroid (both exact while the quad lies inside the texel grid), in
either winding; partial coverage is checked against a dense midpoint-rule
integral."""
import numpy as np
import pytest

from oracle import oracle as O


def _quad(rng, R, scale):
    c = rng.uniform(2.5, R - 3.5, size=2)
    th = rng.uniform(0, np.pi)
    rot = np.array([[np.cos(th), -np.sin(th)], [np.sin(th), np.cos(th)]])
    a, b = rng.uniform(0.2, scale, size=2)
    pts = np.array([[-a, -b], [a, -b], [a, b], [-a, b]]) * rng.uniform(0.7, 1.3, size=(4, 2))
    return c + pts @ rot.T


def _centroid(q):
    x, y = q[:, 0], q[:, 1]
    xn, yn = np.roll(x, -1), np.roll(y, -1)
    cr = x * yn - xn * y
    A = cr.sum() / 2
    return np.array([((x + xn) * cr).sum(), ((y + yn) * cr).sum()]) / (6 * A), abs(A)


@pytest.mark.parametrize("seed", range(8))
def test_constant_and_linear_textures_exact(seed):
    rng = np.random.default_rng(seed)
    R = 16
    q = _quad(rng, R, 2.0)
    if seed % 2:
        q = q[::-1].copy()  # clockwise: the filter reorients
    const = np.broadcast_to(rng.uniform(size=4), (R, R, 4)).copy()
    out, area = O.aniso_sample(q, const)
    cen, A = _centroid(q)
    assert abs(area - A) < 1e-12 * A
    np.testing.assert_allclose(out, const[0, 0], rtol=0, atol=1e-12)
    coef = rng.normal(size=(3, 4))
    vv, uu = np.meshgrid(np.arange(R), np.arange(R), indexing="ij")
    lin = coef[0] + uu[..., None] * coef[1] + vv[..., None] * coef[2]
    out, _ = O.aniso_sample(q, lin)
    np.testing.assert_allclose(out, coef[0] + cen[0] * coef[1] + cen[1] * coef[2], rtol=0, atol=1e-11)


def test_partial_coverage_matches_dense_integral():
    rng = np.random.default_rng(5)
    R = 8
    tex = rng.uniform(size=(R, R, 4))
    q = np.array([[-1.2, 2.1], [2.3, 1.4], [3.1, 4.2], [0.4, 5.6]])  # crosses the u = 0 edge of the grid
    out, area = O.aniso_sample(q, tex)
    n = 1500
    lo, hi = q.min(0), q.max(0)
    xs = lo[0] + (np.arange(n) + 0.5) * (hi[0] - lo[0]) / n
    ys = lo[1] + (np.arange(n) + 0.5) * (hi[1] - lo[1]) / n
    X, Y = np.meshgrid(xs, ys)
    inside = np.ones_like(X, bool)
    for i in range(4):
        e = q[(i + 1) % 4] - q[i]
        inside &= e[0] * (Y - q[i][1]) - e[1] * (X - q[i][0]) >= 0
    inside &= (X >= 0) & (X <= R - 1) & (Y >= 0) & (Y <= R - 1)
    x, y = X[inside], Y[inside]
    x0, y0 = np.minimum(np.floor(x).astype(int), R - 2), np.minimum(np.floor(y).astype(int), R - 2)
    fx, fy = (x - x0)[:, None], (y - y0)[:, None]
    val = (tex[y0, x0] * (1 - fx) * (1 - fy) + tex[y0, x0 + 1] * fx * (1 - fy) + tex[y0 + 1, x0] * (1 - fx) * fy
           + tex[y0 + 1, x0 + 1] * fx * fy)
    ref = val.sum(0) * (hi - lo).prod() / n ** 2 / area
    np.testing.assert_allclose(out, ref, rtol=0, atol=2e-3)


def test_degenerate_footprints_give_no_sample():
    tex = np.ones((8, 8, 4))
    out, area = O.aniso_sample(np.array([[1.0, 1.0], [2.0, 2.0], [3.0, 3.0], [4.0, 4.0]]), tex)  # zero area
    assert area == 0 and not out.any()
    out, _ = O.aniso_sample(np.array([[-3.0, 1.0], [-1.0, 1.0], [-1.0, 3.0], [-3.0, 3.0]]), tex)  # left of the grid
    assert not out.any()  # minu == maxu == 0: no cell to integrate
