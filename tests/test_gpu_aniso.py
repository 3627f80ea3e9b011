"""GPU parity of the anisotropic_bilinear filter: the compositor integrating
each pixel's texture-space footprint quad, forward and reference adjoint,
against the CPU oracle (the reference's Sutherland-Hodgman clipping restated),
with both integrations the compositor has: "cells" (cell by cell, each clipped
polygon's boundary summed piecewise) and "boundary" (a convex footprint along
its boundary over the textures' row-prefix tables, Green's theorem).

Tolerances: the oracle evaluated in FP64 on the same FP32 inputs; 1e-5
absolute per forward output with a 1e-3 fraction of branch flips (cell ranges
are floor / ceil of footprint corners, the fast path a >= test), gradients to
1e-4 relative L2 per tensor plus the elementwise flip budget.  Contribution
counts per Gaussian: at most 1 % of the Gaussians (at least one) off, by at
most 2 (pairs at the 1/255 alpha cut).
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from textured_gaussians_b200 import _backend as B
from textured_gaussians_b200.cuda import _wrapper as W
from tests._util import assert_close, rel_l2, to_np
from textured_gaussians_b200 import rasterization_textured_gaussians, scenes
from textured_gaussians_b200.cuda import (
    fully_fused_projection_2dgs,
    isect_offset_encode,
    isect_tiles,
    make_texture_storage,
    rasterize_to_pixels_textured_gaussians,
)

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
F64 = np.float64


@pytest.fixture(autouse=True, params=["boundary", "cells"])
def integration(request, monkeypatch):
    monkeypatch.setattr(W, "ANISO_INTEGRATION", request.param)
    return request.param

SCENES = {"tiny": lambda: scenes.tiny(), "tiny32": lambda: scenes.tiny(R=32),
          "tiny3cam": lambda: scenes.tiny(seed=7, n_cams=3), "small": lambda: scenes.small(),
          "adjoint": lambda: scenes.adjoint()}


def T(x, dtype=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(x)).to(DEV, dtype)


def _inputs(s, tile, fmt="fp32"):
    radii, means2d, depths, M, normals = fully_fused_projection_2dgs(
        T(s.means), T(s.quats), T(s.scales), T(s.viewmats), T(s.Ks), s.width, s.height, 0.3, s.near_plane,
        s.far_plane, 0.0)
    C, N = radii.shape
    tw, th = -(-s.width // tile), -(-s.height // tile)
    _, ids, fl = isect_tiles(means2d, radii, depths, tile, tw, th)
    off = isect_offset_encode(ids, C, tw, th)
    rng = np.random.default_rng(1)
    colors = rng.uniform(0, 1, size=(C, N, 3)).astype(np.float32)
    opac = np.tile(s.opacities[None], (C, 1))
    tex = T(s.textures)
    store, _ = make_texture_storage(tex, fmt)
    return dict(means2d=means2d, M=M, normals=normals, fl=fl, off=off, colors=colors, opac=opac, tex=tex,
                store=store, deq=store.float().cpu().numpy(), C=C, N=N, tile=tile)


def _oracle_fwd(s, d, bg):
    return O.raster_fwd(to_np(d["means2d"]), to_np(d["M"]), d["colors"], d["opac"], to_np(d["normals"]), d["deq"],
                        d["off"].cpu().numpy(), d["fl"].cpu().numpy(), s.width, s.height, d["tile"],
                        backgrounds=bg, aniso=True, dtype=F64)


@pytest.mark.parametrize("name,tile,fmt", [("tiny", 16, "fp32"), ("tiny", 8, "fp32"), ("tiny32", 16, "fp32"),
                                           ("tiny3cam", 16, "fp32"), ("small", 16, "fp32"), ("small", 8, "bf16"),
                                           ("adjoint", 16, "fp32")])
def test_aniso_forward(name, tile, fmt):
    s = SCENES[name]()
    d = _inputs(s, tile, fmt)
    bg = np.full((d["C"], 3), 0.25, np.float32)
    g = rasterize_to_pixels_textured_gaussians(
        d["means2d"], d["M"], T(d["colors"]), T(d["opac"]), d["tex"], 3.0, 3.0, d["normals"],
        torch.zeros_like(d["means2d"]), s.width, s.height, tile, d["off"], d["fl"], backgrounds=T(bg),
        filtering="anisotropic_bilinear", texture_storage=None if fmt == "fp32" else d["store"])
    o = _oracle_fwd(s, d, bg)
    rc, ra, rn, rd, rm, cs, cc = (to_np(x) for x in g)
    frac = 1e-3
    assert_close(rc, o.colors, 1e-5, 1e-5, frac, "colors")
    assert_close(ra, o.alphas, 1e-5, 0, frac, "alphas")
    assert_close(rn, o.normals, 1e-5, 1e-5, frac, "normals")
    assert_close(rd, o.distort, 1e-5, 1e-4, frac, "distort")
    assert_close(rm, o.median, 1e-5, 1e-5, frac, "median")
    # a pair at the 1/255 alpha cut flips on a rounding-level change of the filtered alpha: count flips, not drift
    nflip = int((cc != o.contrib_count).sum())
    assert nflip <= max(1, 0.01 * cc.size) and np.abs(cc - o.contrib_count).max() <= 2, nflip
    assert rel_l2(rc, o.colors) < 1e-4
    b = rasterize_to_pixels_textured_gaussians(
        d["means2d"], d["M"], T(d["colors"]), T(d["opac"]), d["tex"], 3.0, 3.0, d["normals"],
        torch.zeros_like(d["means2d"]), s.width, s.height, tile, d["off"], d["fl"], backgrounds=T(bg))
    assert float((b[0] - g[0]).abs().max()) > 1e-2  # not the bilinear filter


@pytest.mark.parametrize("name,tile", [("tiny", 16), ("tiny32", 16), ("tiny3cam", 8), ("small", 16), ("adjoint", 16)])
def test_aniso_backward(name, tile):
    s = SCENES[name]()
    d = _inputs(s, tile)
    C, H, W = d["C"], s.height, s.width
    rng = np.random.default_rng(3)
    up = dict(c=rng.normal(size=(C, H, W, 3)), a=rng.normal(size=(C, H, W, 1)), n=rng.normal(size=(C, H, W, 3)),
              d=rng.normal(size=(C, H, W, 1)) * 0.1, m=rng.normal(size=(C, H, W, 1)))
    up = {k: v.astype(np.float32) for k, v in up.items()}
    bg = np.full((C, 3), 0.5, np.float32)
    m2d = d["means2d"].detach().clone().requires_grad_()
    M = d["M"].detach().clone().requires_grad_()
    cols = T(d["colors"]).requires_grad_()
    opac = T(d["opac"]).requires_grad_()
    nrm = d["normals"].detach().clone().requires_grad_()
    dens = torch.zeros_like(d["means2d"]).requires_grad_()
    tex = d["tex"].detach().clone().requires_grad_()
    out = rasterize_to_pixels_textured_gaussians(m2d, M, cols, opac, tex, 3.0, 3.0, nrm, dens, W, H, tile, d["off"],
                                                 d["fl"], backgrounds=T(bg), absgrad=True,
                                                 filtering="anisotropic_bilinear")
    loss = ((out[0] * T(up["c"])).sum() + (out[1] * T(up["a"])).sum() + (out[2] * T(up["n"])).sum()
            + (out[3] * T(up["d"])).sum() + (out[4] * T(up["m"])).sum())
    loss.backward()
    fo = _oracle_fwd(s, d, bg)
    o = O.raster_bwd(to_np(d["means2d"]), to_np(d["M"]), d["colors"], d["opac"], to_np(d["normals"]), d["deq"],
                     d["off"].cpu().numpy(), d["fl"].cpu().numpy(), W, H, tile, fo, up["c"], up["a"], up["n"],
                     up["d"], up["m"], backgrounds=bg, mode=0, aniso=True, dtype=F64)
    pairs = [("means2d", m2d.grad, o.v_means2d), ("M", M.grad, o.v_M), ("colors", cols.grad, o.v_colors),
             ("opac", opac.grad, o.v_opacities), ("normals", nrm.grad, o.v_normals),
             ("textures", tex.grad, o.v_textures), ("densify", dens.grad, o.v_densify),
             ("absgrad", m2d.absgrad, o.v_means2d_abs)]
    for k, got, ref in pairs:
        got = to_np(got)
        assert rel_l2(got, ref) < 1e-4, (k, rel_l2(got, ref))
        assert_close(got, ref, 1e-5 * max(np.abs(ref).max(), 1), 1e-3, 1e-3, k)


@pytest.mark.parametrize("tile", [8, 16])
def test_aniso_packed_and_dense_agree_end_to_end(tile):
    s = scenes.tiny(seed=7, n_cams=3, R=16)
    res = {}
    for packed in (False, True):
        L = [T(x).requires_grad_() for x in (s.means, s.quats, s.scales, s.opacities, s.colors, s.textures)]
        out = rasterization_textured_gaussians(*L, T(s.viewmats), T(s.Ks), s.width, s.height, sh_degree=0,
                                               far_plane=s.far_plane, packed=packed, tile_size=tile,
                                               filtering="anisotropic_bilinear")
        rng = np.random.default_rng(2)
        (out[0] * T(rng.normal(size=tuple(out[0].shape)))).sum().backward()
        res[packed] = (to_np(out[0]), [to_np(x.grad) for x in L])
    (ia, ga), (ib, gb) = res[False], res[True]
    assert_close(ib, ia, 1e-5, 1e-5, 1e-4, "image")
    for name, x, y in zip(("means", "quats", "scales", "opacities", "colors", "textures"), gb, ga):
        assert rel_l2(x, y) < 1e-4, (name, rel_l2(x, y))


def test_aniso_rejects_what_it_does_not_support():
    s = scenes.tiny()
    d = _inputs(s, 32)
    args = (d["means2d"], d["M"], T(d["colors"]), T(d["opac"]), d["tex"], 3.0, 3.0, d["normals"],
            torch.zeros_like(d["means2d"]), s.width, s.height, 32, d["off"], d["fl"])
    with pytest.raises(RuntimeError, match="tile 8 or 16"):
        rasterize_to_pixels_textured_gaussians(*args, filtering="anisotropic_bilinear")
    d = _inputs(s, 16)
    store, scales = make_texture_storage(d["tex"], "fp8")
    args = (d["means2d"], d["M"], T(d["colors"]), T(d["opac"]), d["tex"], 3.0, 3.0, d["normals"],
            torch.zeros_like(d["means2d"]), s.width, s.height, 16, d["off"], d["fl"])
    with pytest.raises(RuntimeError, match="FP32 and BF16"):
        rasterize_to_pixels_textured_gaussians(*args, filtering="anisotropic_bilinear", texture_storage=store,
                                               texture_scales=scales)


@pytest.mark.parametrize("fmt", ["fp32", "bf16", "fp16", "fp8"])
@pytest.mark.parametrize("ry,rx", [(32, 32), (3, 70), (5, 1), (1, 2)])
def test_aniso_prefix_table_matches_the_rows_trapezoid_sums(fmt, ry, rx, integration):
    if integration != "boundary":
        pytest.skip("one run is enough")
    rng = np.random.default_rng(ry * 100 + rx)
    tex = T(rng.uniform(-1, 2, size=(37, ry, rx, 4)).astype(np.float32))
    store, scales = make_texture_storage(tex, fmt)
    st = torch.cuda.current_stream().cuda_stream
    P = W._aniso_prefix(store, scales, st)
    deq = store.float() if scales is None else store.float() * scales[:, None, None, None]
    t = deq.double().cpu().numpy()
    ref = np.zeros_like(t)
    ref[:, :, 1:] = np.cumsum(0.5 * (t[:, :, :-1] + t[:, :, 1:]), axis=2)
    got = P.cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-5 * max(1.0, np.abs(ref).max()), np.abs(got - ref).max()
    assert np.all(got[:, :, 0] == 0)


def test_aniso_boundary_and_cells_agree_on_a_large_scene(integration):
    """Both integrations on one 1600x1200 view of a 150,000-splat mixture scene (32x32 textures)."""
    if integration != "boundary":
        pytest.skip("one run is enough")
    s = scenes.mixture1m(N=150_000, n_cams=1)
    outs = {}
    for mode in ("cells", "boundary"):
        W.ANISO_INTEGRATION = mode
        d = _inputs(s, 8)
        tex = d["tex"].detach().clone().requires_grad_()
        out = rasterize_to_pixels_textured_gaussians(
            d["means2d"], d["M"], T(d["colors"]), T(d["opac"]), tex, 3.0, 3.0, d["normals"],
            torch.zeros_like(d["means2d"]), s.width, s.height, 8, d["off"], d["fl"], filtering="anisotropic_bilinear")
        (out[0].sum() + out[1].sum()).backward()
        outs[mode] = (to_np(out[0]), to_np(out[1]), to_np(tex.grad))
    for i, name in enumerate(("colors", "alphas")):
        assert_close(outs["boundary"][i], outs["cells"][i], 1e-5, 1e-5, 1e-3, name)
    assert rel_l2(outs["boundary"][2], outs["cells"][2]) < 1e-4


@pytest.mark.parametrize("name", ["small", "adjoint"])
def test_aniso_adjoint_from_forward_records_matches_integrating_again(name, integration, monkeypatch):
    """The adjoint reading the forward's footprint integrals (all of them, or only each pixel's first two: the
    rest integrated again) against the adjoint integrating every footprint again."""
    if integration != "boundary":
        pytest.skip("records exist with the boundary integration only")
    s = SCENES[name]()
    d = _inputs(s, 8)
    C, H, Wd = d["C"], s.height, s.width
    rng = np.random.default_rng(5)
    up_c = T(rng.normal(size=(C, H, Wd, 3)).astype(np.float32))
    up_a = T(rng.normal(size=(C, H, Wd, 1)).astype(np.float32))
    grads = {}
    for cap in (0, 2, 32):
        monkeypatch.setattr(W, "ANISO_RECORDS", cap)
        leaves = [d["means2d"].detach().clone().requires_grad_(), d["M"].detach().clone().requires_grad_(),
                  T(d["colors"]).requires_grad_(), T(d["opac"]).requires_grad_(), d["tex"].detach().clone().requires_grad_()]
        out = rasterize_to_pixels_textured_gaussians(
            leaves[0], leaves[1], leaves[2], leaves[3], leaves[4], 3.0, 3.0, d["normals"],
            torch.zeros_like(d["means2d"]), Wd, H, 8, d["off"], d["fl"], filtering="anisotropic_bilinear")
        ((out[0] * up_c).sum() + (out[1] * up_a).sum()).backward()
        grads[cap] = [to_np(x.grad) for x in leaves]
    for cap in (2, 32):
        for k, (got, ref) in enumerate(zip(grads[cap], grads[0])):
            assert np.abs(ref).max() > 0
            assert rel_l2(got, ref) < 1e-6, (cap, k, rel_l2(got, ref))


def test_aniso_transmittance_checkpoints_match_division(integration):
    """The adjoint restarting its transmittance from the forward's checkpoints (with the boundary form's
    records and prefix fold, or cell by cell) against recovering it by division alone."""
    s = SCENES["small"]()
    d = _inputs(s, 8)
    rng = np.random.default_rng(9)
    up = T(rng.normal(size=(d["C"], s.height, s.width, 3)).astype(np.float32))
    grads = {}
    for mode in ("divide", "checkpoint"):
        leaves = [d["means2d"].detach().clone().requires_grad_(), d["M"].detach().clone().requires_grad_(),
                  T(d["opac"]).requires_grad_(), d["tex"].detach().clone().requires_grad_()]
        out = rasterize_to_pixels_textured_gaussians(
            leaves[0], leaves[1], T(d["colors"]), leaves[2], leaves[3], 3.0, 3.0, d["normals"],
            torch.zeros_like(d["means2d"]), s.width, s.height, 8, d["off"], d["fl"], filtering="anisotropic_bilinear",
            transmittance=mode)
        (out[0] * up).sum().backward()
        grads[mode] = [to_np(x.grad) for x in leaves]
    for k, (a, b) in enumerate(zip(grads["checkpoint"], grads["divide"])):
        assert np.abs(b).max() > 0
        assert rel_l2(a, b) < 1e-4, (k, rel_l2(a, b))
