"""FP64 finite differences against the oracle's mipmapped2 and
anisotropic_bilinear texture-colour adjoints.

The rendered colour is linear in the textures' RGB channels: a texture's
colour enters as (c + filtered RGB) * alpha * T, and alpha and T depend on its
alpha channel only (rasterize_to_pixels_{mip2,aniso_bilinear}_textured_
gaussians_2dgs_fwd.cu).  So along any direction that moves RGB alone, a central
difference of L = sum(w * colors) is the directional derivative up to
rounding, and the adjoint's texture gradient (the reference's, which both
filters share with the kernels: rasterize_to_pixels_*_bwd.cu) must reproduce
it -- for mipmapped2 after the pyramid adjoint folds the coarse levels back
into the texture (generate_mipmap_bwd.cu).  The alpha channel is checked by
small steps on one splat at a time where the per-pixel branch signature does
not change: exact for mipmapped2; for anisotropic_bilinear exact once the
textures' colour is zeroed, and not otherwise -- the reference's colour term
in d(alpha) lacks the footprint's 1/area, which the oracle reproduces.
Workload: the adjoint-check scene (2,000 Gaussians, 16x16 textures, one
128x128 camera).
"""
import numpy as np
import pytest

from oracle import oracle as O
from textured_gaussians_b200 import scenes

F64 = np.float64
TILE = 16


@pytest.fixture(scope="module")
def scene():
    s = scenes.adjoint(seed=2)
    radii, m2d, dep, M, nrm = O.project_fwd(s.means, s.quats, s.scales, s.viewmats, s.Ks, s.width, s.height, 0.01,
                                            s.far_plane, dtype=F64)
    tw, th = -(-s.width // TILE), -(-s.height // TILE)
    _, ids, fl = O.isect_tiles(m2d, radii, dep, TILE, tw, th, 1)
    off = O.isect_offset_encode(ids, 1, tw, th)
    colors = s.colors[:, 0][None].astype(F64)
    opac = s.opacities[None].astype(F64)
    w = np.random.default_rng(7).normal(size=(1, s.height, s.width, 3))
    return dict(s=s, m2d=m2d, M=M, nrm=nrm, off=off, fl=fl, colors=colors, opac=opac, w=w)


def _tex_in(tex, filt):
    return O.generate_mipmap(tex) if filt == "mipmapped2" else tex


def _forward(g, tex, filt):
    s = g["s"]
    L = int(np.log2(tex.shape[1])) if filt == "mipmapped2" else 0
    fo = O.raster_fwd(g["m2d"], g["M"], g["colors"], g["opac"], g["nrm"], _tex_in(tex, filt), g["off"], g["fl"],
                      s.width, s.height, TILE, mip_levels=L, aniso=filt == "anisotropic_bilinear", dtype=F64)
    return fo, L


def _texture_gradient(g, tex, filt):
    s = g["s"]
    fo, L = _forward(g, tex, filt)
    z = lambda a: np.zeros_like(a)  # noqa: E731
    bo = O.raster_bwd(g["m2d"], g["M"], g["colors"], g["opac"], g["nrm"], _tex_in(tex, filt), g["off"], g["fl"],
                      s.width, s.height, TILE, fo, g["w"], z(fo.alphas), z(fo.normals), z(fo.distort), z(fo.median),
                      mip_levels=L, aniso=filt == "anisotropic_bilinear", dtype=F64)
    v = bo.v_textures
    return O.generate_mipmap_bwd(v, L) if filt == "mipmapped2" else v


def _loss(g, tex, filt):
    return float((_forward(g, tex, filt)[0].colors * g["w"]).sum())


@pytest.mark.parametrize("filt", ["mipmapped2", "anisotropic_bilinear"])
def test_texture_colour_adjoint_matches_finite_differences(scene, filt):
    tex = scene["s"].textures.astype(F64)
    grad = _texture_gradient(scene, tex, filt)
    assert grad.shape == tex.shape
    rng = np.random.default_rng(11)
    for _ in range(3):
        d = rng.normal(size=tex.shape)
        d[..., 3] = 0.0  # RGB only: the alpha channel moves alpha and T
        h = 0.05
        fd = (_loss(scene, tex + h * d, filt) - _loss(scene, tex - h * d, filt)) / (2 * h)
        an = float((grad * d).sum())
        assert abs(fd) > 1e-3
        assert abs(fd - an) <= 1e-9 * abs(fd), (filt, fd, an)


@pytest.mark.parametrize("filt", ["mipmapped2", "anisotropic_bilinear"])
def test_texture_gradient_is_zero_off_the_contributing_splats(scene, filt):
    tex = scene["s"].textures.astype(F64)
    grad = _texture_gradient(scene, tex, filt)
    contributing = np.zeros(tex.shape[0], bool)
    contributing[np.unique(scene["fl"] % tex.shape[0])] = True
    assert not grad[~contributing].any()
    assert np.abs(grad[contributing][..., :3]).sum() > 0


def _alpha_channel_fd(g, tex, filt, n=30, seed=5, h=1e-5):
    """(fd, adjoint) pairs along random directions over one contributing splat's alpha channel, kept only when
    the per-pixel branch signature is the same at both ends (alpha and T are not smooth across its changes)."""
    grad = _texture_gradient(g, tex, filt)
    rng = np.random.default_rng(seed)
    contributing = np.unique(g["fl"] % tex.shape[0])
    out = []
    for _ in range(n):
        d = np.zeros_like(tex)
        d[int(rng.choice(contributing)), :, :, 3] = rng.normal(size=tex.shape[1:3])
        fp, _ = _forward(g, tex + h * d, filt)
        fm, _ = _forward(g, tex - h * d, filt)
        if fp.branch_sig.tobytes() != fm.branch_sig.tobytes():
            continue
        fd = float(((fp.colors - fm.colors) * g["w"]).sum()) / (2 * h)
        if abs(fd) > 1e-8:
            out.append((fd, float((grad * d).sum())))
    r = np.array(out)
    assert len(r) >= 10
    cos = float(r[:, 0] @ r[:, 1] / np.linalg.norm(r[:, 0]) / np.linalg.norm(r[:, 1]))
    return r, cos


def test_mipmapped2_alpha_channel_adjoint_matches_finite_differences(scene):
    r, cos = _alpha_channel_fd(scene, scene["s"].textures.astype(F64), "mipmapped2")
    assert cos > 0.99999
    assert np.median(np.abs(r[:, 0] - r[:, 1]) / np.abs(r[:, 0])) < 1e-6


def test_anisotropic_alpha_channel_adjoint_deviates_only_through_the_reference_colour_term(scene):
    """The reference's anisotropic_bilinear adjoint takes the texture colour entering d(alpha) and the
    back-to-front colour buffer without the footprint's 1/area (filters/anisotropic_bilinear.cuh:372-389, used
    at ..._aniso_bilinear_..._bwd.cu:499-536), and the oracle reproduces it: with the textures' colour zeroed
    that term vanishes and the alpha-channel adjoint is exact; with colour it is not."""
    tex = scene["s"].textures.astype(F64)
    no_colour = tex.copy()
    no_colour[..., :3] = 0.0
    r, cos = _alpha_channel_fd(scene, no_colour, "anisotropic_bilinear")
    assert cos > 0.99999
    assert np.median(np.abs(r[:, 0] - r[:, 1]) / np.abs(r[:, 0])) < 1e-6
    _, cos_colour = _alpha_channel_fd(scene, tex, "anisotropic_bilinear")
    assert cos_colour < 0.99
