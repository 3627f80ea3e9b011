"""CPU check of how the oracle's three bilinear compositor adjoints relate.

The reference's "bilinear" adjoint drops the texture lookup's dependence on
the ray transform
(rasterize_to_pixels_textured_gaussians_2dgs_bwd.cu:552-609); its
"bilinear_bwd2" adjoint adds that term with du/ds = (R-1)/range, twice the
(R-1)/(2 range) of the forward's addressing (..._bwd2.cu:627-628 against
filters/bilinear.cuh:25-26); the exact adjoint adds it with the true factor,
and is itself pinned by finite differences (tests/test_adjoint_fd.py). So, in
FP64 on the adjoint-check workload (2,000 Gaussians, 16x16 textures, one
128x128 camera), the three differ only in the ray-transform gradient (and the
densification gradient formed from it), and there bwd2 - reference = 2 (exact
- reference) -- away from texel-aligned UV coordinates, where bwd2's term
collapses to 0 (u_low == u_high, filters/bilinear.cuh:44-47), which random
inputs do not hit.
"""
import numpy as np
import pytest

from oracle import oracle as O
from textured_gaussians_b200 import scenes

F64 = np.float64


@pytest.fixture(scope="module")
def adjoints():
    s = scenes.adjoint(seed=2)
    radii, m2d, dep, M, nrm = O.project_fwd(s.means, s.quats, s.scales, s.viewmats, s.Ks, s.width, s.height, 0.01,
                                            s.far_plane, dtype=F64)
    tw, th = -(-s.width // 16), -(-s.height // 16)
    _, ids, fl = O.isect_tiles(m2d, radii, dep, 16, tw, th, 1)
    off = O.isect_offset_encode(ids, 1, tw, th)
    colors, opac, tex = s.colors[:, 0][None].astype(F64), s.opacities[None].astype(F64), s.textures.astype(F64)
    w = np.random.default_rng(7).normal(size=(1, s.height, s.width, 3))
    fo = O.raster_fwd(m2d, M, colors, opac, nrm, tex, off, fl, s.width, s.height, 16, dtype=F64)
    z = np.zeros_like
    return {mode: O.raster_bwd(m2d, M, colors, opac, nrm, tex, off, fl, s.width, s.height, 16, fo, w,
                               z(fo.alphas), z(fo.normals), z(fo.distort), z(fo.median), mode=mode, dtype=F64)
            for mode in (0, 1, 2)}


@pytest.mark.parametrize("name", ["v_M", "v_densify"])  # v_densify is formed from v_M (..._bwd.cu:692-699)
def test_bwd2_adds_twice_the_exact_uv_term(adjoints, name):
    ref, bwd2, exact = (getattr(adjoints[m], name).ravel() for m in (0, 1, 2))
    d_exact, d_bwd2 = exact - ref, bwd2 - ref
    assert np.linalg.norm(d_exact) > 1e-3 * np.linalg.norm(exact)  # the term is not negligible here
    np.testing.assert_allclose(d_bwd2, 2 * d_exact, rtol=0, atol=1e-12 * np.linalg.norm(d_bwd2))


@pytest.mark.parametrize("name", ["v_means2d", "v_opacities", "v_colors", "v_textures", "v_normals"])
def test_other_gradients_agree_across_adjoints(adjoints, name):
    a0 = getattr(adjoints[0], name)
    scale = max(np.abs(a0).max(), 1e-300)
    for mode in (1, 2):
        np.testing.assert_allclose(getattr(adjoints[mode], name), a0, rtol=0, atol=1e-12 * scale)
