"""CPU check of the compositor's per-splat cull box against the oracle.

Both compositor kernels skip a (pixel, splat) pair when the pixel lies outside
a pixel-space box computed once per splat (cull_box in
textured_gaussians_b200/csrc/raster_common.cuh): outside it the pair is
provably invalid (alpha < 1/255), so skipping must leave every output
unchanged.  The reference evaluates every pair of a tile instead
(rasterize_to_pixels_textured_gaussians_2dgs_fwd.cu:293-354).  This test
restates the box in FP64 and renders single random splats with the FP32
oracle over every tile of a small image; every pixel the oracle lights must
lie inside the box -- untextured, bilinear, mipmapped2 and
anisotropic_bilinear (whose box drops the texture square), with textures
whose alpha exceeds 1, opacities near the 1/255 cut, several g_weight values
and oblique splats.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O

W = H = 64
TILE = 16


def cull_box(xy, opac, M, textured, range_x, range_y, g_weight, tex_square=True):
    """(x0, y0, x1, y1) outside of which the pair is invalid, or None when unbounded (cull_box)."""
    if textured:
        if not g_weight > 0:
            return None
        K = (1 / (255 * opac) - 0.998 + g_weight) / g_weight
    else:
        K = 1 / (255 * opac)
    K *= 0.999
    if not K > 0:
        return None
    sig1 = 0.0 if K >= 1 else -math.log(K) * 1.001 + 1e-3
    rs, rd = math.sqrt(2 * sig1), math.sqrt(sig1)
    hx = max(rs, range_x) if textured and tex_square else rs
    hy = max(rs, range_y) if textured and tex_square else rs
    x0, x1, y0, y1 = xy[0] - rd, xy[0] + rd, xy[1] - rd, xy[1] + rd
    zs = []
    for c in range(4):
        u, v = (hx if c & 1 else -hx), (hy if c & 2 else -hy)
        X, Y, Z = (M[r, 0] * u + M[r, 1] * v + M[r, 2] for r in range(3))
        zs.append(Z)
        if Z == 0:
            return None
        x0, x1 = min(x0, X / Z), max(x1, X / Z)
        y0, y1 = min(y0, Y / Z), max(y1, Y / Z)
    if not (all(z > 0 for z in zs) or all(z < 0 for z in zs)):
        return None
    m = 1 + 1e-3 * ((x1 - x0) + (y1 - y0))
    box = (x0 - m, y0 - m, x1 + m, y1 + m)
    if not all(math.isfinite(b) and abs(b) < 1e30 for b in box):
        return None
    return box


def random_splat(rng):
    z = rng.uniform(1.0, 4.0)
    means = np.array([[rng.uniform(-0.6, 0.6) * z, rng.uniform(-0.6, 0.6) * z, z]])
    quats = rng.normal(size=(1, 4))
    quats /= np.linalg.norm(quats)
    s = np.exp(rng.normal(-2.3, 0.9, size=2))
    scales = np.array([[s[0], s[1], s[1]]])
    K = np.array([[[50.0, 0, W / 2], [0, 50.0, H / 2], [0, 0, 1]]])
    return O.project_fwd(means, quats, scales, np.eye(4)[None], K, W, H)


def render_alpha(m2d, M, nrm, opac, textures, g_weight, mip_levels=0, aniso=False):
    tw, th = W // TILE, H // TILE
    offsets = np.arange(tw * th, dtype=np.int32).reshape(1, th, tw)  # the one splat listed in every tile
    flatten = np.zeros(tw * th, np.int32)
    o = O.raster_fwd(m2d, M, np.full((1, 1, 3), 0.5), np.array([[opac]]), nrm, textures, offsets, flatten, W, H,
                     TILE, g_weight=g_weight, mip_levels=mip_levels, aniso=aniso, dtype=np.float32)
    return o.alphas[0, :, :, 0]


@pytest.mark.parametrize("form", ["plain", "bilinear", "mipmapped2", "anisotropic_bilinear"])
def test_no_lit_pixel_outside_the_cull_box(form):
    rng = np.random.default_rng({"plain": 1, "bilinear": 2, "mipmapped2": 3, "anisotropic_bilinear": 4}[form])
    ys, xs = np.mgrid[0:H, 0:W]
    px, py = xs + 0.5, ys + 0.5
    lit_total = culled_total = 0
    for it in range(40):
        radii, m2d, _, M, nrm = random_splat(rng)
        if radii[0, 0] <= 0:
            continue
        opac = float(rng.choice([1.0 / 254, 0.02, 0.3, 0.95]))
        g_weight = float(rng.choice([1.0, 0.6, 0.15]))
        textured = form != "plain"
        tex = tex_arg = None
        mip = 0
        if textured:
            tex = rng.uniform(0, 1, size=(1, 8, 8, 4))
            tex[..., 3] *= rng.choice([1.0, 3.0])  # texture alpha above 1 inside the texture square
            tex_arg = O.generate_mipmap(tex) if form == "mipmapped2" else tex
            mip = 3 if form == "mipmapped2" else 0
        alpha = render_alpha(m2d, M, nrm, opac, tex_arg, g_weight, mip, form == "anisotropic_bilinear")
        box = cull_box(m2d[0, 0].astype(float), opac, M[0, 0].astype(float), textured, 3.0, 3.0, g_weight,
                       tex_square=form != "anisotropic_bilinear")
        lit = alpha > 0
        lit_total += int(lit.sum())
        if box is None:
            continue
        inside = (px >= box[0]) & (px <= box[2]) & (py >= box[1]) & (py <= box[3])
        assert not (lit & ~inside).any(), (form, it, box, np.argwhere(lit & ~inside)[:5])
        culled_total += int((~inside).sum())
    # the check is not vacuous: splats light pixels and their boxes exclude most of the image
    assert lit_total > 0
    assert culled_total > 0.5 * 40 * W * H * 0.5
