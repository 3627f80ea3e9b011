"""The CUDA path against the reference's OWN CUDA path: golden vectors made by
running the unmodified reference (its Python package and its kernels, built
from its sources) on one B200, one camera per call (tests/golden/
make_ref_golden.py).

Stage tests feed this library the reference's own intermediate tensors
(projected splats, SH colours, intersection lists), so each stage is compared
on identical inputs:

  * projection (radii, means2d, depths, ray transforms, normals) from the
    same scene: bit-exact; SH colours 1e-5;
  * intersections, sorted keys, flatten ids and tile offsets computed from the
    reference's projected splats: bit-exact;
  * compositor forward (colours, alphas, normals, distortion, median) for
    bilinear, bilinear_bwd2, mipmapped2, anisotropic_bilinear and the plain
    2DGS form: 1e-5 absolute with a 1e-3 fraction of branch flips (the 1/255
    alpha cut, the 1e-4 stop, tap choices flip on a 1-ulp difference between
    two --use_fast_math builds); contribution sums 1e-4 relative;
  * compositor adjoint: every gradient within 1e-4 relative L2 per tensor
    (texture gradients on the stored rows, and every row's norm); for the
    sampled large workloads (views8 and the benchmark scene's camera 0 with
    bilinear, bilinear_bwd2, mipmapped2 and anisotropic_bilinear), where pixels hold up to ~190
    contributors and both builds recover transmittance by division, 1e-3;
  * the renderer end to end (rasterization_textured_gaussians, the
    reference's public entry point) on the small workloads: images 1e-5 with
    the flip budget, leaf gradients 1e-4 relative L2 (1e-3 for mipmapped2 and
    anisotropic_bilinear, whose level / cell choices follow projected
    footprints that the two projections round differently).
"""
import numpy as np
import pytest
import torch

import bench
from oracle import oracle as O
from oracle import pipeline as P
from tests import _refgold as RG
from tests._util import assert_close, rel_l2, to_np
from textured_gaussians_b200 import rasterization_textured_gaussians, scenes
from textured_gaussians_b200.cuda import (
    fully_fused_projection_2dgs,
    isect_offset_encode,
    isect_tiles,
    rasterize_to_pixels_2dgs,
    rasterize_to_pixels_textured_gaussians,
    spherical_harmonics,
)

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
FLIPS = 1e-3

SMALL = {"small": ("bilinear", "bilinear_bwd2"), "adjoint": ("bilinear", "bilinear_bwd2", "mipmapped2"),
         "adjoint_aniso": ("anisotropic_bilinear",)}
GRAD_TOL = {"bilinear": 1e-4, "bilinear_bwd2": 1e-4, "mipmapped2": 1e-4, "anisotropic_bilinear": 1e-4}
E2E_GRAD_TOL = {"bilinear": 1e-4, "bilinear_bwd2": 1e-4, "mipmapped2": 1e-3, "anisotropic_bilinear": 1e-3}


def T(x, dtype=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(x)).to(DEV, dtype)


_CACHE = {}


def fixture(case):
    if case not in _CACHE:
        g = RG.load(case)
        _CACHE[case] = (g, RG.scene(case, g))
    return _CACHE[case]


def check_grad(name, got, ref, tol):
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    assert np.abs(ref).max() > 0, f"{name}: reference gradient is all zero"
    r = rel_l2(got, ref)
    assert r < tol, f"{name}: relative L2 {r:.3g} >= {tol}"


def check_texture_grad(g, prefix, v_tex, tol):
    rows, vals, norms, ours = RG.texture_rows_check(g, prefix, v_tex)
    check_grad(f"{prefix} texture rows", ours, vals, tol)
    mine = np.linalg.norm(v_tex.reshape(v_tex.shape[0], -1).astype(np.float64), axis=1)
    check_grad(f"{prefix} texture row norms", mine, norms, tol)


@pytest.mark.parametrize("case", list(SMALL))
def test_projection_and_sh_match_reference(case):
    g, s = fixture(case)
    radii, means2d, depths, M, normals = fully_fused_projection_2dgs(
        T(s.means), T(s.quats), T(s.scales), T(s.viewmats), T(s.Ks), s.width, s.height, 0.3, s.near_plane,
        s.far_plane, 0.0)
    radii = radii.cpu().numpy()
    ref_r = g["stage__radii"]
    # the projection follows the reference's arithmetic and its fused multiply-adds operation by operation:
    # every output of every visible entry equals the reference's bit for bit (culled entries are zero here
    # and left unwritten by the reference)
    np.testing.assert_array_equal(radii, ref_r)
    vis = ref_r > 0
    assert vis.sum() > 0
    for name, got in (("means2d", means2d), ("depths", depths), ("M", M), ("normals", normals)):
        np.testing.assert_array_equal(to_np(got)[vis], g[f"stage__{name}"][vis], err_msg=name)
    cam = torch.linalg.inv(T(s.viewmats))[:, :3, 3]
    dirs = T(s.means)[None] - cam[:, None]
    sh = spherical_harmonics(s.sh_degree, dirs, T(s.colors)[None], masks=T(ref_r, torch.int32) > 0)
    colors = torch.clamp_min(sh + 0.5, 0.0)
    assert_close(to_np(colors)[vis], g["stage__colors"][vis], 1e-5, 1e-6, name="sh colours")


@pytest.mark.parametrize("case", list(SMALL))
def test_projection_adjoint_matches_reference(case):
    """The projection's adjoint alone (reference mode, no norm_rot_grad): seeded upstream gradients on the
    visible entries' means2d, depths, ray transforms and normals; gradients of means, quats and scales
    within 1e-4 relative L2 of the reference's, or no farther from the FP64 oracle's than 1.5 times the
    reference's own distance from it."""
    g, s = fixture(case)
    leaves = [T(x).requires_grad_(True) for x in (s.means, s.quats, s.scales)]
    pr = fully_fused_projection_2dgs(*leaves, T(s.viewmats), T(s.Ks), s.width, s.height, 0.3, s.near_plane,
                                     s.far_plane, 0.0)
    C, N = pr[0].shape
    ups = RG.proj_upstream(g["projvjp_seed"], C, N)
    vis = (pr[0] > 0).float()
    sum((o * T(u) * vis.view(vis.shape + (1,) * (o.dim() - 2))).sum() for o, u in zip(pr[1:], ups)).backward()
    # FP64 oracle: the reference-mode adjoint on the oracle's own FP64 projection
    radii, _, _, M64, _ = O.project_fwd(s.means, s.quats, s.scales, s.viewmats, s.Ks, s.width, s.height,
                                        s.near_plane, s.far_plane, dtype=np.float64)
    m = (radii > 0).astype(np.float64)
    ex = O.project_bwd(s.means, s.quats, s.scales, s.viewmats, s.Ks, radii, M64, ups[0] * m[..., None],
                       ups[1] * m, ups[3] * m[..., None], ups[2] * m[..., None, None], mode=0, dtype=np.float64)
    problems, report = [], []
    for name, leaf, exact in zip(("means", "quats", "scales"), leaves, ex):
        got, ref = to_np(leaf.grad), g[f"projvjp__v_{name}"]
        r, e_ours, e_ref = rel_l2(got, ref), rel_l2(got, exact), rel_l2(ref, exact)
        report.append(f"v_{name}: rel L2 {r:.2e} (to FP64: ours {e_ours:.2e}, reference {e_ref:.2e})")
        if not (r < 1e-4 or e_ours <= max(1e-4, 1.5 * e_ref)):
            problems.append(name)
    print(f"projection adjoint [{case}]: " + "; ".join(report))
    assert not problems, (problems, report)


@pytest.mark.parametrize("case", list(SMALL))
def test_intersections_bit_exact_on_reference_projection(case):
    g, s = fixture(case)
    tw, th = -(-s.width // s.tile_size), -(-s.height // s.tile_size)
    tpg, ids, fl = isect_tiles(T(g["stage__means2d"]), T(g["stage__radii"], torch.int32), T(g["stage__depths"]),
                               s.tile_size, tw, th)
    off = isect_offset_encode(ids, 1, tw, th)
    assert g["stage__isect_ids"].size > 1000
    np.testing.assert_array_equal(tpg.cpu().numpy(), g["stage__tpg"])
    np.testing.assert_array_equal(ids.cpu().numpy(), g["stage__isect_ids"])
    np.testing.assert_array_equal(fl.cpu().numpy(), g["stage__flatten_ids"])
    np.testing.assert_array_equal(off.cpu().numpy(), g["stage__offsets"])


def _stage_inputs(g, s):
    leaves = dict(means2d=T(g["stage__means2d"]), M=T(g["stage__M"]), colors=T(g["stage__colors"]),
                  opacities=T(s.opacities[None]), normals=T(g["stage__normals"]))
    for v in leaves.values():
        v.requires_grad_(True)
    return leaves


def _compare_outputs(g, prefix, out, flips=FLIPS):
    names = ("colors", "alphas", "normals", "distort", "median")
    for i, name in enumerate(names):
        assert_close(to_np(out[i]), g[f"{prefix}__out{i}"], 1e-5, 1e-5, flips, f"{prefix} {name}")
    ref_cnt = g[f"{prefix}__out6"]
    cnt = to_np(out[6])
    off = np.abs(cnt - ref_cnt) > 0
    assert off.sum() <= max(1, 0.01 * off.size) and np.abs(cnt - ref_cnt).max() <= 2, f"{prefix} contrib counts"
    assert rel_l2(to_np(out[5]), g[f"{prefix}__out5"]) < 1e-4, f"{prefix} contrib sums"


@pytest.mark.parametrize("case,filtering", [(c, f) for c, fs in SMALL.items() for f in fs])
def test_compositor_matches_reference(case, filtering):
    g, s = fixture(case)
    leaves = _stage_inputs(g, s)
    tex = T(s.textures).requires_grad_(True)
    densify = torch.zeros_like(leaves["means2d"], requires_grad=True)
    bg = T(s.backgrounds) if s.backgrounds is not None else None
    out = rasterize_to_pixels_textured_gaussians(
        leaves["means2d"], leaves["M"], leaves["colors"], leaves["opacities"], tex, 3.0, 3.0, leaves["normals"],
        densify, s.width, s.height, s.tile_size, T(g["stage__offsets"], torch.int32),
        T(g["stage__flatten_ids"], torch.int32), backgrounds=bg, filtering=filtering)
    prefix = f"comp_{filtering}"
    _compare_outputs(g, prefix, out)
    ups = RG.upstream(g["up_seed"], s)
    sum((o * T(u)).sum() for o, u in zip(out[:5], ups)).backward()
    tol = GRAD_TOL[filtering]
    for k, v in leaves.items():
        check_grad(f"{prefix} v_{k}", to_np(v.grad), g[f"{prefix}__v_{k}"], tol)
    check_texture_grad(g, prefix, to_np(tex.grad), tol)


@pytest.mark.parametrize("case", ["small", "adjoint"])
def test_plain_compositor_matches_reference(case):
    g, s = fixture(case)
    leaves = _stage_inputs(g, s)
    densify = torch.zeros_like(leaves["means2d"], requires_grad=True)
    bg = T(s.backgrounds) if s.backgrounds is not None else None
    out = rasterize_to_pixels_2dgs(leaves["means2d"], leaves["M"], leaves["colors"], leaves["opacities"],
                                   leaves["normals"], densify, s.width, s.height, s.tile_size,
                                   T(g["stage__offsets"], torch.int32), T(g["stage__flatten_ids"], torch.int32),
                                   backgrounds=bg)
    _compare_outputs(g, "plain", out)
    ups = RG.upstream(g["up_seed"], s)
    sum((o * T(u)).sum() for o, u in zip(out[:5], ups)).backward()
    for k, v in leaves.items():
        check_grad(f"plain v_{k}", to_np(v.grad), g[f"plain__v_{k}"], 1e-4)


@pytest.mark.parametrize("case,filtering", [(c, f) for c, fs in SMALL.items() for f in fs])
def test_renderer_end_to_end_matches_reference(case, filtering):
    """Both renderers end to end from the same scene.  Unlike the stage tests, the two pipelines project
    the splats themselves, so the compositor inputs already differ in the last bits; the images are held
    to 1e-5 with a 2e-3 fraction of elements allowed up to 1e-3 (pixels where that difference moves a
    discrete choice or accumulates over many contributors).  A leaf gradient passes when it is within
    the tolerance of the reference's, or -- for the bilinear adjoints, which the FP64 oracle pipeline
    restates end to end -- when it is no farther from the FP64 result than 1.5 times the reference's
    own distance from it (the reference's FP32 gradients of means, quats and scales sit up to ~1e-3
    from FP64 on these scenes: they go through the ray-transform adjoint, which divides by the
    ray-plane cross product's z)."""
    g, s = fixture(case)
    leaves = [T(x).requires_grad_(True) for x in (s.means, s.quats, s.scales, s.opacities, s.colors, s.textures)]
    bg = T(s.backgrounds) if s.backgrounds is not None else None
    out = rasterization_textured_gaussians(*leaves, T(s.viewmats), T(s.Ks), s.width, s.height,
                                           near_plane=s.near_plane, far_plane=s.far_plane, sh_degree=s.sh_degree,
                                           tile_size=s.tile_size, backgrounds=bg, filtering=filtering)
    outs = [out[0], out[1], out[2], out[4], out[5]]
    pre = f"e2e_{filtering}"
    problems, report = [], []
    for i, (o, name) in enumerate(zip(outs, ("colors", "alphas", "normals", "distort", "median"))):
        a, b = to_np(o).astype(np.float64), g[f"{pre}__out{i}"].astype(np.float64)
        err = np.abs(a - b)
        frac = float((err > 1e-5 + 1e-5 * np.abs(b)).mean())
        report.append(f"{name}: max {err.max():.2e}, frac>1e-5 {frac:.2e}")
        if frac > 2e-3 or err.max() > 1e-3:
            problems.append(name)
    ups = RG.upstream(g["up_seed"], s)
    sum((o * T(u)).sum() for o, u in zip(outs, ups)).backward()
    tol = E2E_GRAD_TOL[filtering]
    exact = None
    if filtering in ("bilinear", "bilinear_bwd2"):
        _, _, _, cache = P.render(s.means, s.quats, s.scales, s.opacities, s.colors, s.textures, s.viewmats, s.Ks,
                                  s.width, s.height, sh_degree=s.sh_degree, tile_size=s.tile_size,
                                  far_plane=s.far_plane, backgrounds=s.backgrounds, dtype=np.float64)
        exact = P.render_backward(cache, s.means, s.quats, s.scales, s.opacities, s.colors, s.textures, s.viewmats,
                                  s.Ks, s.width, s.height, *ups, sh_degree=s.sh_degree, tile_size=s.tile_size,
                                  backgrounds=s.backgrounds, raster_mode=0 if filtering == "bilinear" else 1)
    for name, leaf in zip(("means", "quats", "scales", "opacities", "colors"), leaves[:5]):
        got, ref = to_np(leaf.grad), g[f"{pre}__v_{name}"]
        r = rel_l2(got, ref)
        msg = f"v_{name}: rel L2 {r:.2e}"
        ok = r < tol
        if exact is not None:
            e_ours, e_ref = rel_l2(got, exact[name]), rel_l2(ref, exact[name])
            msg += f" (to FP64: ours {e_ours:.2e}, reference {e_ref:.2e})"
            ok = ok or e_ours <= max(tol, 1.5 * e_ref)
        report.append(msg)
        if not ok:
            problems.append(f"v_{name}")
    rows, vals, norms, ours = RG.texture_rows_check(g, pre, to_np(leaves[5].grad))
    r = rel_l2(ours, vals)
    report.append(f"v_textures (rows): rel L2 {r:.2e}")
    if not r < tol:
        problems.append("v_textures")
    print(f"{pre} [{case}]: " + "; ".join(report))
    assert not problems, f"{pre} [{case}] outside tolerance: {problems} ({'; '.join(report)})"


# ---------------------------------------------------------------- sampled large workloads
def _sampled_textures(case, g, N):
    if case == "views8":
        gen = torch.Generator(device=DEV)
        gen.manual_seed(1)
        full = torch.rand((N, 50, 50, 4), generator=gen, device=DEV)
    else:
        full = bench.gpu_textures(N, 32, torch.device(DEV))
    tex = full[T(g["rows"], torch.int64)].contiguous()
    del full
    torch.cuda.empty_cache()
    assert RG.digest(tex.cpu().numpy()) == str(g["tex_sha256_rows"]), f"{case}: regenerated textures differ"
    return tex


def _sampled_scene(case):
    if case == "views8":
        s = scenes.views8(with_textures=False)
        return s, s.opacities, 16
    sc = bench.make_scene(0, 1, 1_000_000, 4)
    s = scenes.Scene(sc["means"], sc["quats"], sc["scales"], sc["opacities"], sc["colors"], None, sc["viewmats"][:1],
                     sc["Ks"][:1], sc["width"], sc["height"], 0, far_plane=100.0, tile_size=8)
    return s, s.opacities, 8


@pytest.mark.parametrize("case", ["views8", "mix1m", "mix1m_bwd2", "mix1m_mip", "mix1m_aniso"])
def test_compositor_matches_reference_on_sampled_tiles(case):
    """mix1m_bwd2 / _mip / _aniso: the bilinear_bwd2 adjoint, and the mipmapped2 and anisotropic_bilinear
    filters (the latter by boundary integration, forward records and prefix fold) on the benchmark scene's
    camera 0 against the reference's own kernels."""
    g = RG.load(case)
    filtering = {"mix1m_bwd2": "bilinear_bwd2", "mix1m_mip": "mipmapped2",
                 "mix1m_aniso": "anisotropic_bilinear"}.get(case, "bilinear")
    pre = f"comp_{filtering}"
    s, opac, tile = _sampled_scene(case)
    N = s.means.shape[0]
    rows = g["rows"]
    tex = _sampled_textures(case, g, N).requires_grad_(True)
    W, H = s.width, s.height
    tw, th = -(-W // tile), -(-H // tile)
    offsets, fl = RG.sampled_layout(g, th, tw)
    leaves = dict(means2d=T(g["stage__means2d"][None]), M=T(g["stage__M"][None]), colors=T(g["stage__colors"][None]),
                  opacities=T(opac[rows][None]), normals=T(g["stage__normals"][None]))
    for v in leaves.values():
        v.requires_grad_(True)
    densify = torch.zeros_like(leaves["means2d"], requires_grad=True)
    out = rasterize_to_pixels_textured_gaussians(
        leaves["means2d"], leaves["M"], leaves["colors"], leaves["opacities"], tex, 3.0, 3.0, leaves["normals"],
        densify, W, H, tile, T(offsets, torch.int32), T(fl, torch.int32), filtering=filtering)
    sel = RG.pixel_mask(g, tile, th, tw, H, W)
    assert sel.sum() >= 2000
    problems, report = [], []
    for i, name in enumerate(("colors", "alphas", "normals", "distort", "median")):
        a, b = to_np(out[i])[sel].astype(np.float64), g[f"{pre}__out{i}"].astype(np.float64)
        err = np.abs(a - b)
        frac = float((err > 1e-5 + 1e-5 * np.abs(b)).mean())
        report.append(f"{name}: max {err.max():.2e}, frac>1e-5 {frac:.2e}")
        if frac > FLIPS:
            problems.append(name)
    selt = T(sel.astype(np.float32)[..., None])
    ups = RG.upstream(g["up_seed"], s)
    sum((o * T(u) * selt).sum() for o, u in zip(out[:5], ups)).backward()
    grads = [(k, to_np(v.grad)[0], g[f"{pre}__v_{k}"]) for k, v in leaves.items()]
    rows_k, vals, norms, ours = RG.texture_rows_check(g, pre, to_np(tex.grad))
    grads.append(("texture rows", ours, vals))
    mine = np.linalg.norm(to_np(tex.grad).reshape(rows.size, -1).astype(np.float64), axis=1)
    grads.append(("texture row norms", mine, norms))
    for k, got, ref in grads:
        r = rel_l2(got, ref)
        report.append(f"v_{k}: rel L2 {r:.2e}")
        if not r < 1e-3:
            problems.append(f"v_{k}")
    print(f"{case}: " + "; ".join(report))
    assert not problems, f"{case} outside tolerance: {problems} ({'; '.join(report)})"
