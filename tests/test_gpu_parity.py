"""GPU parity: every stage of the CUDA path against the CPU oracle on the same
seeded inputs.

The arbiter for floating-point outputs is the oracle evaluated in FP64 on the
very same FP32 inputs: the ray-splat cross product cancels badly at some
pixels, where an IEEE-FP32 evaluation without fused multiply-add is itself
~1e-5 off while the GPU's FP32 result stays within ~1e-6 of the FP64 value.

Tolerances (stated per test):
  * integer / index outputs (tiles per Gaussian, isect ids, flatten ids,
    offsets, sort permutations): bit-exact, given identical projected inputs;
  * FP32 forward outputs: 1e-5 absolute (plus 1e-5 relative for values far
    from 1, e.g. pixel coordinates), allowing a small stated fraction of
    branch flips where the GPU's --use_fast_math arithmetic and the IEEE
    oracle land on different sides of a discrete test;
  * gradients: 1e-4 relative in L2 norm per tensor, plus an elementwise check
    with a flip budget.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from oracle import pipeline as P
from tests._util import assert_close, cosine, rel_l2, to_np
from textured_gaussians_b200 import scenes
from textured_gaussians_b200.cuda import (
    fully_fused_projection_2dgs,
    isect_offset_encode,
    isect_tiles,
    make_texture_storage,
    rasterize_to_pixels_2dgs,
    rasterize_to_pixels_textured_gaussians,
    sort_pairs,
    spherical_harmonics,
)

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
F64 = np.float64  # oracle precision for every floating-point comparison


def T(x, dtype=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(x)).to(DEV, dtype)


def project_gpu(s):
    return fully_fused_projection_2dgs(T(s.means), T(s.quats), T(s.scales), T(s.viewmats), T(s.Ks), s.width,
                                       s.height, 0.3, s.near_plane, s.far_plane, 0.0)


SCENES = {"tiny": lambda: scenes.tiny(), "tiny3cam": lambda: scenes.tiny(seed=7, n_cams=3),
          "small": lambda: scenes.small(), "adjoint": lambda: scenes.adjoint()}


@pytest.mark.parametrize("name", list(SCENES))
def test_projection_forward(name):
    s = SCENES[name]()
    radii, means2d, depths, M, normals = (to_np(x) if x.dtype != torch.int32 else x.cpu().numpy()
                                          for x in project_gpu(s))
    o_radii, o_m2d, o_d, o_M, o_n = O.project_fwd(s.means, s.quats, s.scales, s.viewmats, s.Ks, s.width, s.height,
                                                  s.near_plane, s.far_plane, dtype=F64)
    # radius is a ceil(): count boundary flips, require them to be rare and off by one
    diff = radii != o_radii
    assert diff.sum() <= max(2, 5e-3 * diff.size), f"{diff.sum()} radius flips"
    if diff.any():
        assert np.abs(radii[diff] - o_radii[diff]).max() <= 1 or ((radii[diff] == 0) | (o_radii[diff] == 0)).all()
    vis = (radii > 0) & (o_radii > 0)
    assert vis.sum() > 0
    assert_close(means2d[vis], o_m2d[vis], 1e-5, 1e-5, name="means2d")
    assert_close(depths[vis], o_d[vis], 1e-5, 1e-6, name="depths")
    assert_close(M[vis], o_M[vis], 1e-5, 1e-5, name="ray_transforms")
    assert_close(normals[vis], o_n[vis], 1e-5, 0, name="normals")
    # culled entries are zero-filled
    assert (means2d[radii == 0] == 0).all() and (M[radii == 0] == 0).all()


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_projection_backward(mode):
    s = scenes.small(N=3000)
    rng = np.random.default_rng(11)
    radii, means2d, depths, M, normals = project_gpu(s)
    C, N = radii.shape
    vm2d = rng.normal(size=(C, N, 2)).astype(np.float32)
    vd = rng.normal(size=(C, N)).astype(np.float32)
    vn = rng.normal(size=(C, N, 3)).astype(np.float32)
    vM = rng.normal(size=(C, N, 3, 3)).astype(np.float32)
    means = T(s.means).requires_grad_()
    quats = T(s.quats).requires_grad_()
    scales = T(s.scales).requires_grad_()
    out = fully_fused_projection_2dgs(means, quats, scales, T(s.viewmats), T(s.Ks), s.width, s.height, 0.3,
                                      s.near_plane, s.far_plane, 0.0, norm_rot_grad=(mode == 1),
                                      adjoint="exact" if mode == 2 else "reference")
    loss = (out[1] * T(vm2d)).sum() + (out[2] * T(vd)).sum() + (out[3] * T(vM)).sum() + (out[4] * T(vn)).sum()
    loss.backward()
    o = O.project_bwd(s.means, s.quats, s.scales, s.viewmats, s.Ks, radii.cpu().numpy(), to_np(M), vm2d, vd, vn, vM,
                      mode=mode, dtype=F64)
    for got, ref, nm in zip((means.grad, quats.grad, scales.grad), o, ("means", "quats", "scales")):
        got = to_np(got)
        assert rel_l2(got, ref) < 1e-4, (nm, rel_l2(got, ref))
        assert_close(got, ref, 1e-4, 1e-3, max_bad_frac=1e-3, name=nm)


def _isect_both(s):
    radii, means2d, depths, _, _ = project_gpu(s)
    ts = s.tile_size
    tw, th = -(-s.width // ts), -(-s.height // ts)
    C = radii.shape[0]
    g = isect_tiles(means2d, radii, depths, ts, tw, th)
    o = O.isect_tiles(to_np(means2d), radii.cpu().numpy(), to_np(depths), ts, tw, th, C)
    return g, o, (C, tw, th)


@pytest.mark.parametrize("name", list(SCENES))
def test_isect_and_offsets_bit_exact(name):
    (g_tpg, g_ids, g_fl), (o_tpg, o_ids, o_fl), (C, tw, th) = _isect_both(SCENES[name]())
    assert g_tpg.dtype == torch.int32 and g_ids.dtype == torch.int64 and g_fl.dtype == torch.int32
    np.testing.assert_array_equal(g_tpg.cpu().numpy(), o_tpg)
    np.testing.assert_array_equal(g_ids.cpu().numpy(), o_ids)
    np.testing.assert_array_equal(g_fl.cpu().numpy(), o_fl)
    g_off = isect_offset_encode(g_ids, C, tw, th)
    np.testing.assert_array_equal(g_off.cpu().numpy(), O.isect_offset_encode(o_ids, C, tw, th))


def test_isect_unsorted_emission_order():
    s = scenes.tiny(seed=3)
    radii, means2d, depths, _, _ = project_gpu(s)
    tw, th = -(-s.width // 16), -(-s.height // 16)
    _, ids, fl = isect_tiles(means2d, radii, depths, 16, tw, th, sort=False)
    _, o_ids, o_fl = O.isect_tiles(to_np(means2d), radii.cpu().numpy(), to_np(depths), 16, tw, th, 1, sort=False)
    np.testing.assert_array_equal(ids.cpu().numpy(), o_ids)
    np.testing.assert_array_equal(fl.cpu().numpy(), o_fl)


@pytest.mark.parametrize("n,end_bit,distinct", [(2, 40, 2), (4095, 40, 7), (4097, 44, 1 << 20), (100_000, 48, 13),
                                                (1_000_003, 48, 1 << 30), (3_000_000, 56, 257), (123_457, 64, 1000)])
def test_sort_pairs_bit_exact(n, end_bit, distinct):
    rng = np.random.default_rng(n)
    keys = rng.integers(0, distinct, size=n, dtype=np.int64) * np.int64(2654435761) + rng.integers(0, 3, size=n)
    keys = keys & np.int64((1 << 62) - 1)
    if end_bit < 64:
        keys |= np.int64(1) << np.int64(62)  # bits above end_bit must not affect the order
    vals = np.arange(n, dtype=np.int32)
    gk, gv = sort_pairs(torch.from_numpy(keys).to(DEV), torch.from_numpy(vals).to(DEV), end_bit)
    ok, ov = O.sort_pairs(keys, vals, end_bit)
    np.testing.assert_array_equal(gk.cpu().numpy(), ok)
    np.testing.assert_array_equal(gv.cpu().numpy(), ov)


def test_offsets_with_empty_tiles_and_cameras():
    C, tw, th = 3, 5, 4
    tb = (tw * th).bit_length()
    rng = np.random.default_rng(5)
    cam = np.array([0, 0, 2, 2, 2], np.int64)
    tile = np.array([3, 3, 0, 7, 19], np.int64)
    ids = (cam << (32 + tb)) | (tile << 32) | rng.integers(0, 1 << 30, size=5)
    off = isect_offset_encode(torch.from_numpy(ids).to(DEV), C, tw, th).cpu().numpy()
    np.testing.assert_array_equal(off, O.isect_offset_encode(ids, C, tw, th))
    empty = isect_offset_encode(torch.zeros(0, dtype=torch.int64, device=DEV), C, tw, th)
    assert (empty == 0).all()


def _raster_inputs(s, tex_fmt="fp32"):
    radii, means2d, depths, M, normals = project_gpu(s)
    C, N = radii.shape
    ts = s.tile_size
    tw, th = -(-s.width // ts), -(-s.height // ts)
    _, ids, fl = isect_tiles(means2d, radii, depths, ts, tw, th)
    off = isect_offset_encode(ids, C, tw, th)
    rng = np.random.default_rng(1)
    colors = rng.uniform(0, 1, size=(C, N, 3)).astype(np.float32)
    opac = np.tile(s.opacities[None], (C, 1))
    tex = T(s.textures)
    store, scales = make_texture_storage(tex, tex_fmt)
    if tex_fmt == "fp8":
        deq = (store.float() * scales[:, None, None, None]).cpu().numpy()
    else:
        deq = store.float().cpu().numpy()
    return dict(radii=radii, means2d=means2d, depths=depths, M=M, normals=normals, ids=ids, fl=fl, off=off,
                colors=colors, opac=opac, tex=tex, store=store, scales=scales, deq=deq, C=C, N=N)


def _oracle_fwd(s, d, textured, bg=None, g_weight=1.0):
    return O.raster_fwd(to_np(d["means2d"]), to_np(d["M"]), d["colors"], d["opac"], to_np(d["normals"]),
                        d["deq"] if textured else None, d["off"].cpu().numpy(), d["fl"].cpu().numpy(), s.width,
                        s.height, s.tile_size, backgrounds=bg, g_weight=g_weight, dtype=F64)


def _compare_fwd(g, o, frac):
    rc, ra, rn, rd, rm, cs, cc = (to_np(x) for x in g)
    assert_close(rc, o.colors, 1e-5, 1e-5, frac, "colors")
    assert_close(ra, o.alphas, 1e-5, 0, frac, "alphas")
    assert_close(rn, o.normals, 1e-5, 1e-5, frac, "normals")
    assert_close(rd, o.distort, 1e-5, 1e-4, frac, "distort")
    assert_close(rm, o.median, 1e-5, 1e-5, frac, "median")
    assert_close(cs, o.contrib_sum, 1e-4, 1e-5, frac, "contrib_sum")
    assert_close(cc, o.contrib_count, 0, 0, frac, "contrib_count")


@pytest.mark.parametrize("name,fmt", [("tiny", "fp32"), ("small", "fp32"), ("adjoint", "fp32"), ("tiny3cam", "fp32"),
                                      ("small", "bf16"), ("small", "fp16"), ("small", "fp8")])
def test_textured_forward(name, fmt):
    s = SCENES[name]()
    d = _raster_inputs(s, fmt)
    C = d["C"]
    bg = np.ones((C, 3), np.float32) * 0.25
    g = rasterize_to_pixels_textured_gaussians(
        d["means2d"], d["M"], T(d["colors"]), T(d["opac"]), d["tex"], 3.0, 3.0, d["normals"],
        torch.zeros_like(d["means2d"]), s.width, s.height, s.tile_size, d["off"], d["fl"], backgrounds=T(bg),
        texture_storage=None if fmt == "fp32" else d["store"], texture_scales=d["scales"])
    o = _oracle_fwd(s, d, True, bg)
    _compare_fwd(g, o, 1e-4)
    assert rel_l2(to_np(g[0]), o.colors) < 1e-5


@pytest.mark.parametrize("name", ["tiny", "small", "tiny3cam"])
def test_plain_forward(name):
    s = SCENES[name]()
    d = _raster_inputs(s)
    g = rasterize_to_pixels_2dgs(d["means2d"], d["M"], T(d["colors"]), T(d["opac"]), d["normals"],
                                 torch.zeros_like(d["means2d"]), s.width, s.height, s.tile_size, d["off"], d["fl"])
    o = _oracle_fwd(s, d, False)
    _compare_fwd(g, o, 1e-4)


def _grads_gpu(s, d, textured, filtering, bg=None, absgrad=False, seed=3, depth=0, persistent=False):
    rng = np.random.default_rng(seed)
    C, H, W = d["C"], s.height, s.width
    up = dict(c=rng.normal(size=(C, H, W, 3)), a=rng.normal(size=(C, H, W, 1)), n=rng.normal(size=(C, H, W, 3)),
              d=rng.normal(size=(C, H, W, 1)) * 0.1, m=rng.normal(size=(C, H, W, 1)))
    up = {k: v.astype(np.float32) for k, v in up.items()}
    m2d = d["means2d"].detach().clone().requires_grad_()
    M = d["M"].detach().clone().requires_grad_()
    cols = T(d["colors"]).requires_grad_()
    opac = T(d["opac"]).requires_grad_()
    nrm = d["normals"].detach().clone().requires_grad_()
    dens = torch.zeros_like(d["means2d"]).requires_grad_()
    tex = d["tex"].detach().clone().requires_grad_()
    if textured:
        out = rasterize_to_pixels_textured_gaussians(
            m2d, M, cols, opac, tex, 3.0, 3.0, nrm, dens, W, H, s.tile_size, d["off"], d["fl"],
            backgrounds=None if bg is None else T(bg), absgrad=absgrad, filtering=filtering, batch_depth=depth,
            persistent=persistent)
    else:
        out = rasterize_to_pixels_2dgs(m2d, M, cols, opac, nrm, dens, W, H, s.tile_size, d["off"], d["fl"],
                                       backgrounds=None if bg is None else T(bg), absgrad=absgrad, batch_depth=depth,
                                       persistent=persistent)
    loss = ((out[0] * T(up["c"])).sum() + (out[1] * T(up["a"])).sum() + (out[2] * T(up["n"])).sum()
            + (out[3] * T(up["d"])).sum() + (out[4] * T(up["m"])).sum())
    loss.backward()
    grads = dict(means2d=m2d.grad, M=M.grad, colors=cols.grad, opac=opac.grad, normals=nrm.grad, densify=dens.grad,
                 textures=tex.grad if textured else None, absgrad=getattr(m2d, "absgrad", None))
    return grads, up, out


@pytest.mark.parametrize("name,filtering,mode", [("tiny", "bilinear", 0), ("small", "bilinear", 0),
                                                 ("small", "bilinear_bwd2", 1), ("small", "bilinear_exact", 2),
                                                 ("tiny3cam", "bilinear", 0), ("adjoint", "bilinear_exact", 2)])
def test_textured_backward(name, filtering, mode):
    s = SCENES[name]()
    d = _raster_inputs(s)
    bg = np.full((d["C"], 3), 0.5, np.float32)
    g, up, out = _grads_gpu(s, d, True, filtering, bg=bg, absgrad=True)
    fo = _oracle_fwd(s, d, True, bg)
    o = O.raster_bwd(to_np(d["means2d"]), to_np(d["M"]), d["colors"], d["opac"], to_np(d["normals"]), d["deq"],
                     d["off"].cpu().numpy(), d["fl"].cpu().numpy(), s.width, s.height, s.tile_size, fo, up["c"],
                     up["a"], up["n"], up["d"], up["m"], backgrounds=bg, mode=mode, dtype=F64)
    pairs = [("means2d", o.v_means2d), ("M", o.v_M), ("colors", o.v_colors), ("opac", o.v_opacities),
             ("normals", o.v_normals), ("textures", o.v_textures), ("densify", o.v_densify),
             ("absgrad", o.v_means2d_abs)]
    for k, ref in pairs:
        got = to_np(g[k])
        assert rel_l2(got, ref) < 1e-4, (k, rel_l2(got, ref))
        assert_close(got, ref, 1e-5 * max(np.abs(ref).max(), 1), 1e-3, 1e-3, k)


@pytest.mark.parametrize("name", ["tiny", "small"])
def test_plain_backward(name):
    s = SCENES[name]()
    d = _raster_inputs(s)
    g, up, _ = _grads_gpu(s, d, False, None)
    fo = _oracle_fwd(s, d, False)
    o = O.raster_bwd(to_np(d["means2d"]), to_np(d["M"]), d["colors"], d["opac"], to_np(d["normals"]), None,
                     d["off"].cpu().numpy(), d["fl"].cpu().numpy(), s.width, s.height, s.tile_size, fo, up["c"],
                     up["a"], up["n"], up["d"], up["m"], mode=0, dtype=F64)
    for k, ref in [("means2d", o.v_means2d), ("M", o.v_M), ("colors", o.v_colors), ("opac", o.v_opacities),
                   ("normals", o.v_normals), ("densify", o.v_densify)]:
        assert rel_l2(to_np(g[k]), ref) < 1e-4, (k, rel_l2(to_np(g[k]), ref))


@pytest.mark.parametrize("degree", [0, 1, 2, 3, 4])
def test_spherical_harmonics(degree):
    rng = np.random.default_rng(degree)
    n, K = 5000, 25
    dirs = rng.normal(size=(n, 3)).astype(np.float32)
    coeffs = rng.normal(size=(n, K, 3)).astype(np.float32)
    masks = rng.uniform(size=n) > 0.2
    dt, ct = T(dirs).requires_grad_(), T(coeffs).requires_grad_()
    out = spherical_harmonics(degree, dt, ct, T(masks, torch.bool))
    vc = rng.normal(size=(n, 3)).astype(np.float32)
    (out * T(vc)).sum().backward()
    ref = O.sh_fwd(degree, dirs, coeffs, masks, dtype=F64)
    assert_close(to_np(out), ref, 1e-5, 1e-5, 0, "sh")
    v_coeffs, v_dirs = O.sh_bwd(degree, dirs, coeffs, vc, masks, dtype=F64)
    assert_close(to_np(ct.grad), v_coeffs, 1e-5, 1e-5, 0, "v_coeffs")
    assert_close(to_np(dt.grad), v_dirs, 1e-4, 1e-4, 0, "v_dirs")


def test_end_to_end_small_matches_oracle_pipeline():
    from textured_gaussians_b200 import rasterization_textured_gaussians

    s = scenes.small()
    means = T(s.means).requires_grad_()
    quats = T(s.quats).requires_grad_()
    scales_ = T(s.scales).requires_grad_()
    opac = T(s.opacities).requires_grad_()
    cols = T(s.colors).requires_grad_()
    tex = T(s.textures).requires_grad_()
    out = rasterization_textured_gaussians(means, quats, scales_, opac, cols, tex, T(s.viewmats), T(s.Ks), s.width,
                                           s.height, sh_degree=0, far_plane=s.far_plane,
                                           backgrounds=T(s.backgrounds))
    rng = np.random.default_rng(0)
    vc = rng.normal(size=tuple(out[0].shape)).astype(np.float32)
    (out[0] * T(vc)).sum().backward()
    meta = out[-1]
    proj = tuple(to_np(meta[k]) if k != "radii" else meta[k].cpu().numpy()
                 for k in ("radii", "means2d", "depths", "ray_transforms", "normals"))
    rc, ra, rn, cache = P.render(s.means, s.quats, s.scales, s.opacities, s.colors, s.textures, s.viewmats, s.Ks,
                                 s.width, s.height, sh_degree=0, far_plane=s.far_plane, backgrounds=s.backgrounds,
                                 proj_override=proj, dtype=F64)
    np.testing.assert_array_equal(meta["isect_ids"].cpu().numpy(), cache.isect_ids)
    np.testing.assert_array_equal(meta["flatten_ids"].cpu().numpy(), cache.flatten_ids)
    assert_close(to_np(out[0]), rc, 1e-5, 1e-5, 1e-4, "colors")
    assert_close(to_np(out[1]), ra, 1e-5, 0, 1e-4, "alphas")
    assert_close(to_np(out[2]), rn, 1e-5, 1e-5, 1e-4, "normals (world)")
    g = P.render_backward(cache, s.means, s.quats, s.scales, s.opacities, s.colors, s.textures, s.viewmats, s.Ks,
                          s.width, s.height, vc, sh_degree=0, backgrounds=s.backgrounds)
    for nm, t in [("means", means), ("quats", quats), ("scales", scales_), ("opacities", opac), ("colors", cols),
                  ("textures", tex)]:
        assert rel_l2(to_np(t.grad), g[nm]) < 1e-4, (nm, rel_l2(to_np(t.grad), g[nm]))
        assert cosine(to_np(t.grad), g[nm]) > 0.99999


def test_sort_bounded_wait_gives_up_with_a_status_and_the_context_survives():
    """Failure detection without a fault: a look-back wait that nothing will
    satisfy gives up after its poll limit, the call returns TG_ERR_TIMEOUT,
    and the next sort on the same context is correct (and reports OK)."""
    from textured_gaussians_b200 import _backend as B

    L = B.lib()
    n = 8192
    keys = torch.randint(0, 1 << 40, (n,), dtype=torch.int64, device=DEV)
    vals = torch.arange(n, dtype=torch.int32, device=DEV)
    ka, va = torch.empty_like(keys), torch.empty_like(vals)
    wsb = L.tg_sort_workspace_bytes(n, 8)
    ws = torch.empty((wsb,), dtype=torch.uint8, device=DEV)
    st = torch.cuda.current_stream().cuda_stream
    rc = L.tg_sort_lookback_selftest(B.ptr(keys), B.ptr(vals), B.ptr(ka), B.ptr(va), B.ptr(ws), wsb, st)
    assert rc == -5, (rc, L.tg_last_error())
    k2, v2 = sort_pairs(keys.clone(), vals.clone(), 40, check=True)
    ref = torch.sort(keys, stable=True)
    assert torch.equal(k2, ref.values) and torch.equal(v2.long(), ref.indices)


@pytest.mark.parametrize("tile,textured", [(32, True), (32, False), (8, True)])
def test_other_tile_sizes_match_oracle(tile, textured):
    """32x32 tiles (four pixels per thread) and 8x8 tiles against the FP64 oracle run with the same tile size."""
    s = scenes.small()
    s.tile_size = tile
    d = _raster_inputs(s)
    g, up, out = _grads_gpu(s, d, textured, "bilinear_exact" if textured else None)
    fo = _oracle_fwd(s, d, textured)
    _compare_fwd(out, fo, 1e-4)
    o = O.raster_bwd(to_np(d["means2d"]), to_np(d["M"]), d["colors"], d["opac"], to_np(d["normals"]),
                     d["deq"] if textured else None, d["off"].cpu().numpy(), d["fl"].cpu().numpy(), s.width,
                     s.height, tile, fo, up["c"], up["a"], up["n"], up["d"], up["m"], mode=2 if textured else 0,
                     dtype=F64)
    pairs = [("means2d", o.v_means2d), ("M", o.v_M), ("colors", o.v_colors), ("opac", o.v_opacities),
             ("normals", o.v_normals)] + ([("textures", o.v_textures)] if textured else [])
    for k, ref in pairs:
        assert rel_l2(to_np(g[k]), ref) < 1e-4, (k, rel_l2(to_np(g[k]), ref))


@pytest.mark.parametrize("tile,depth", [(8, 32), (8, 256), (16, 64), (16, 1024), (32, 256)])
def test_batch_depth_changes_nothing(tile, depth):
    """The staging depth only regroups the same front-to-back / back-to-front sweep:
    forward outputs bit-exact, gradients equal up to float-atomic order."""
    s = scenes.small()
    s.tile_size = tile
    d = _raster_inputs(s)
    g0, _, out0 = _grads_gpu(s, d, True, "bilinear_exact")
    g1, _, out1 = _grads_gpu(s, d, True, "bilinear_exact", depth=depth)
    for a, b in zip(out0[:5], out1[:5]):  # per-pixel outputs (the statistics are float atomics)
        assert torch.equal(a, b)
    for k in ("means2d", "M", "colors", "opac", "normals", "textures", "densify"):
        assert rel_l2(to_np(g1[k]), to_np(g0[k])) < 1e-6, k


@pytest.mark.parametrize("tile,textured", [(8, True), (16, True), (32, True), (16, False)])
def test_persistent_launch_changes_nothing(tile, textured):
    """CTAs taking tiles from a device work counter compute every tile exactly as one CTA per tile does."""
    s = scenes.small()
    s.tile_size = tile
    d = _raster_inputs(s)
    f = "bilinear" if textured else None
    g0, _, out0 = _grads_gpu(s, d, textured, f)
    g1, _, out1 = _grads_gpu(s, d, textured, f, persistent=True)
    for a, b in zip(out0[:5], out1[:5]):
        assert torch.equal(a, b)
    assert torch.equal(out0[6], out1[6])  # contribution counts
    for k in ("means2d", "M", "colors", "opac", "normals", "densify") + (("textures",) if textured else ()):
        assert rel_l2(to_np(g1[k]), to_np(g0[k])) < 1e-6, k


def _near_degenerate_splats(n=4000, seed=0):
    """Large splats close to the camera whose plane passes near the camera centre:
    s0^2 t1z^2 + s1^2 t2z^2 = z^2 (1 + eps), eps in +-[1e-7, 1e-1] (log-uniform), so the
    projection's `distance` cancels to a relative 1e-7..1e-1 of its terms."""
    rng = np.random.default_rng(seed)
    means, quats, scales = [], [], []
    while len(means) < n:
        mean = np.array([rng.uniform(-0.5, 0.5), rng.uniform(-0.5, 0.5), rng.uniform(0.5, 2.0)])
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        w, x, y, z = q
        t1z, t2z = 2 * (x * z - w * y), 2 * (y * z + w * x)
        if abs(t1z) < 0.3:
            continue
        eps = 10 ** rng.uniform(-7, -1) * rng.choice([-1, 1])
        s1 = abs(rng.normal(0.1, 0.05))
        rem = mean[2] ** 2 * (1 + eps) - (s1 * t2z) ** 2
        if rem <= 0:
            continue
        means.append(mean)
        quats.append(q)
        scales.append([np.sqrt(rem) / abs(t1z), s1, s1])
    f = lambda a: np.asarray(a, np.float32)
    return f(means), f(quats), f(scales)


def test_near_degenerate_projection_is_solved_in_fp64():
    """Where the FP32 solve cancels (the IEEE-FP32 oracle is off by up to ~1e-2 relative and flips most radii),
    the GPU's FP64 step matches the FP64 oracle to FP32 output rounding."""
    means, quats, scales = _near_degenerate_splats()
    V = np.eye(4, dtype=np.float32)[None]
    K = np.array([[[1200, 0, 800], [0, 1200, 600], [0, 0, 1]]], np.float32)
    radii, m2d, depths, M, nrm = fully_fused_projection_2dgs(T(means), T(quats), T(scales), T(V), T(K), 1600, 1200,
                                                             0.3, 0.01, 100.0, 0.0)
    r64, m64, d64, M64, n64 = O.project_fwd(means, quats, scales, V, K, 1600, 1200, 0.01, 100.0, dtype=F64)
    r32, m32, _, _, _ = O.project_fwd(means, quats, scales, V, K, 1600, 1200, 0.01, 100.0, dtype=np.float32)
    Mo = M64[0]
    rel = np.abs(Mo[:, 2, 0] ** 2 + Mo[:, 2, 1] ** 2 - Mo[:, 2, 2] ** 2) / (Mo[:, 2] ** 2).sum(1)
    deg = rel < 1.0 / 128  # safely inside the FP64 branch
    radii = radii.cpu().numpy()[0]
    # radii the oracle represents (its float -> int32 conversion of larger values is undefined in C++)
    vis = deg & (r64[0] > 0) & (r64[0] < (1 << 30))
    assert vis.sum() > 1000
    assert (radii[vis] == r64[0][vis]).mean() > 0.99
    both = vis & (radii > 0)
    g = to_np(m2d)[0][both]
    ref = m64[0][both]
    err = np.abs(g - ref).max(1) / (np.abs(ref).max(1) + 1)
    assert err.max() < 1e-6, err.max()
    e32 = np.abs(m32[0][both] - ref).max(1) / (np.abs(ref).max(1) + 1)
    assert e32.max() > 1e-4  # the FP32 chain really has cancelled on this set
    assert_close(to_np(M)[0][both], M64[0][both], 1e-6 * np.abs(M64[0][both]).max(), 1e-6, 0, "ray transforms")


def _sh_scene(seed=31, N=500, n_cams=3, K=16):
    s = scenes.tiny(seed=seed, N=N, n_cams=n_cams)
    rng = np.random.default_rng(seed)
    sh = np.concatenate([rng.uniform(0, 1, size=(N, 1, 3)), rng.normal(0, 0.25, size=(N, K - 1, 3))], 1)
    s.colors = sh.astype(np.float32)  # strong higher bands: some colours hit the clamp at 0
    return s


@pytest.mark.parametrize("packed", [False, True])
def test_fused_sh_matches_unfused_path(packed):
    """SH evaluated inside the projection (camera centre by cofactors in-kernel) against the separate SH op fed
    by torch's inverse: images to 1e-5, gradients to 1e-5 relative, dense and packed."""
    from textured_gaussians_b200 import rasterization_textured_gaussians

    s = _sh_scene()
    rng = np.random.default_rng(5)
    w = T(rng.normal(size=(3, s.height, s.width, 3)))
    res = []
    for fuse in (True, False):
        L = [T(x).requires_grad_() for x in (s.means, s.quats, s.scales, s.opacities, s.colors, s.textures)]
        out = rasterization_textured_gaussians(*L, T(s.viewmats), T(s.Ks), s.width, s.height, sh_degree=3,
                                               far_plane=s.far_plane, packed=packed, fuse_sh=fuse)
        (out[0] * w).sum().backward()
        res.append((out, [t.grad.to_dense() if t.grad.is_sparse else t.grad for t in L]))
    (of, gf), (ou, gu) = res
    assert torch.allclose(of[0], ou[0], atol=1e-5, rtol=0)
    assert torch.allclose(of[1], ou[1], atol=1e-6, rtol=0)
    for name, a, b in zip(("means", "quats", "scales", "opacities", "sh", "textures"), gf, gu):
        assert rel_l2(to_np(a), to_np(b)) < 1e-5, (name, rel_l2(to_np(a), to_np(b)))


def test_fused_sh_degree3_end_to_end_matches_oracle_pipeline():
    from textured_gaussians_b200 import rasterization_textured_gaussians

    s = _sh_scene(seed=32)
    L = [T(x).requires_grad_() for x in (s.means, s.quats, s.scales, s.opacities, s.colors, s.textures)]
    out = rasterization_textured_gaussians(*L, T(s.viewmats), T(s.Ks), s.width, s.height, sh_degree=3,
                                           far_plane=s.far_plane)
    rng = np.random.default_rng(0)
    vc = rng.normal(size=tuple(out[0].shape)).astype(np.float32)
    (out[0] * T(vc)).sum().backward()
    meta = out[-1]
    proj = tuple(to_np(meta[k]) if k != "radii" else meta[k].cpu().numpy()
                 for k in ("radii", "means2d", "depths", "ray_transforms", "normals"))
    rc, ra, rn, cache = P.render(s.means, s.quats, s.scales, s.opacities, s.colors, s.textures, s.viewmats, s.Ks,
                                 s.width, s.height, sh_degree=3, far_plane=s.far_plane, proj_override=proj, dtype=F64)
    assert_close(to_np(out[0]), rc, 1e-5, 1e-5, 1e-4, "colors")
    g = P.render_backward(cache, s.means, s.quats, s.scales, s.opacities, s.colors, s.textures, s.viewmats, s.Ks,
                          s.width, s.height, vc, sh_degree=3)
    for nm, t in zip(("means", "quats", "scales", "opacities", "colors", "textures"), L):
        assert rel_l2(to_np(t.grad), g[nm]) < 1e-4, (nm, rel_l2(to_np(t.grad), g[nm]))
