"""Golden vectors from the reference's own CUDA path (run on a CUDA machine).

Runs the UNMODIFIED reference -- its Python package (``rendering.py``,
``cuda/_wrapper.py``) installed under ``baseline/_ref`` and its kernels built
from its own sources by ``oracle/build_ref.py`` into ``oracle/_ref`` -- on the
seeded synthetic workloads, one camera per call (the reference's textured
kernels index the texture array with the flattened camera-major element index,
``rasterize_to_pixels_textured_gaussians_2dgs_fwd.cu:318``, so only C = 1 is
defined), and writes ``tests/golden/ref_<case>.npz``:

  small    the 10,000-splat, 8x8-texture, 200x200 workload, SH degree 0, white
           background, tile 16: the renderer end to end
           (``rendering.py:1342`` rasterization_textured_gaussians, bilinear and
           bilinear_bwd2) with leaf gradients, plus each stage on the
           reference's own intermediate tensors: projection, SH, intersections
           and offsets, the textured compositor forward / adjoint
           (``_wrapper.py:1806``) and the plain 2DGS compositor;
  adjoint  the 2,000-splat, 16x16-texture, 128x128 workload: the same, plus
           the mipmapped2 compositor; and, in ref_adjoint_aniso.npz, the
           anisotropic_bilinear compositor on the rows whose footprints stay
           convex (aniso_safe_rows: the reference's clipping is undefined for
           self-intersecting footprints);
  views8   camera 0 of the 300,000-splat, 50x50-texture (drawn on the GPU,
           seeded), SH degree 3, 800x800 workload, tile 16; compositor
           outputs on a sample of tiles (upstream gradients only there), with
           the sampled tiles' splat lists and the projected rows they use;
  mix1m    camera 0 of the benchmark workload (bench.py's make_scene and
           gpu_textures: 1,000,000 splats, 32x32 FP32 textures drawn on the
           GPU, 1600x1200, tile 8), sampled the same way;
  mix1m_bwd2, mix1m_mip  the same camera and textures with the bilinear_bwd2
           adjoint and with the mipmapped2 compositor, on other sampled tile
           rows;
  mix1m_aniso  the same camera and textures with the anisotropic_bilinear
           compositor, on other sampled tile rows, the splat lists keeping
           only the rows whose footprints stay convex (aniso_safe_rows).

For views8 and mix1m the reference's compositor runs on the sampled tiles'
sub-problem (see sampled_case): with the whole texture tensor it refuses the
call, which exceeds its 32-bit accessors.  Its mipmapped2 adjoint returns a
background gradient for a None background (see ref_backgrounds), so that
filter gets a zero background.

Large per-texel gradients are stored for a deterministic subset of rows plus
every row's L2 norm.  Upstream gradients are regenerated from the seeds
stored in the file.  The reference's ``_C`` module is replaced by the one
built in ``oracle/_ref`` before the reference package is imported (the
reference's own loader would try to compile every kernel it ships).

Usage:  python tests/golden/make_ref_golden.py [--out DIR] [--cases small,adjoint,views8,mix1m]
"""
from __future__ import annotations

import argparse
import hashlib
import os
import sys
import types

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import torch  # noqa: E402

from textured_gaussians_b200 import scenes  # noqa: E402

DEV = "cuda:0"
ROWS_KEPT = 1500        # texture-gradient rows kept per small case
ROWS_KEPT_LARGE = 24    # per sampled large case (50x50 / 32x32 textures)


def reference():
    """The reference package from baseline/_ref, its _C bound to oracle/_ref's build."""
    from oracle import build_ref

    mod = build_ref.load()
    if mod is None:
        raise RuntimeError("oracle/_ref holds no build of the reference's kernels (run oracle/build_ref.py)")
    sys.path.insert(0, os.path.join(ROOT, "baseline", "_ref"))
    stub = types.ModuleType("textured_gaussians.cuda._backend")
    stub._C = mod
    sys.modules["textured_gaussians.cuda._backend"] = stub
    from textured_gaussians import rendering
    from textured_gaussians.cuda import _wrapper

    return rendering, _wrapper


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def npy(t):
    return t.detach().cpu().numpy()


def upstream(seed, shapes):
    rng = np.random.default_rng(seed)
    return [rng.normal(size=s).astype(np.float32) for s in shapes]


def proj_upstream(seed, cn):
    """Upstream gradients of the projection's outputs means2d [C,N,2], depths [C,N], ray transforms
    [C,N,3,3] and normals [C,N,3]."""
    rng = np.random.default_rng(seed)
    C, N = cn
    return [rng.normal(size=sh).astype(np.float32) for sh in ((C, N, 2), (C, N), (C, N, 3, 3), (C, N, 3))]


def keep_rows(v, n_keep, seed=0):
    """A deterministic subset of the nonzero rows of v [G, ...], and every row's L2 norm."""
    flat = v.reshape(v.shape[0], -1)
    norms = np.linalg.norm(flat.astype(np.float64), axis=1)
    nz = np.flatnonzero(norms > 0)
    rng = np.random.default_rng(seed)
    rows = np.sort(rng.choice(nz, min(n_keep, nz.size), replace=False)) if nz.size else nz
    return rows.astype(np.int64), v[rows], norms


def T(x, dtype=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(x)).to(DEV, dtype)


def project_and_shade(W, s, means, quats, scales, colors):
    """The reference's projection, SH shading (rendering.py:1572-1583) and intersections, C = 1."""
    viewmats, Ks = T(s.viewmats), T(s.Ks)
    radii, means2d, depths, M, normals = W.fully_fused_projection_2dgs(
        means, quats, scales, viewmats, Ks, s.width, s.height, 0.3, s.near_plane, s.far_plane, 0.0)
    cam = torch.inverse(viewmats)[:, :3, 3]
    dirs = means[None] - cam[:, None]
    C = viewmats.shape[0]
    coeffs = colors.expand(C, *([-1] * colors.dim()))
    sh = W.spherical_harmonics(s.sh_degree, dirs, coeffs, masks=radii > 0)
    shaded = torch.clamp_min(sh + 0.5, 0.0)
    tw, th = -(-s.width // s.tile_size), -(-s.height // s.tile_size)
    tpg, isect_ids, flatten_ids = W.isect_tiles(means2d, radii, depths, s.tile_size, tw, th)
    offsets = W.isect_offset_encode(isect_ids, C, tw, th)
    return dict(radii=radii, means2d=means2d, depths=depths, M=M, normals=normals, colors=shaded, tpg=tpg,
                isect_ids=isect_ids, flatten_ids=flatten_ids, offsets=offsets, tw=tw, th=th)


def ref_backgrounds(s, filtering):
    """Backgrounds handed to the reference.  Its mipmapped2 adjoint gates the background gradient on
    needs_input_grad[8] (the normals, _wrapper.py:3554) and so returns one for a None background, which
    torch's autograd rejects; a zero background renders and differentiates identically, so that filter
    gets zeros(1, D) where the workload has none."""
    if s.backgrounds is not None:
        return T(s.backgrounds)
    if filtering == "mipmapped2":
        return torch.zeros((1, 3), device=DEV)
    return None


def compositor(W, p, s, textures, opacities, filtering, ups, masks=None):
    """One reference compositor forward + adjoint on the given stage inputs (_wrapper.py:1806)."""
    leaves = dict(means2d=p["means2d"].detach().clone(), M=p["M"].detach().clone(),
                  colors=p["colors"].detach().clone(), opacities=opacities.detach().clone(),
                  textures=textures.detach().clone(), normals=p["normals"].detach().clone())
    for v in leaves.values():
        v.requires_grad_(True)
    densify = torch.zeros_like(leaves["means2d"], requires_grad=True)
    bg = ref_backgrounds(s, filtering)
    out = W.rasterize_to_pixels_textured_gaussians(
        leaves["means2d"], leaves["M"], leaves["colors"], leaves["opacities"], leaves["textures"], 3.0, 3.0,
        leaves["normals"], densify, s.width, s.height, s.tile_size, p["offsets"], p["flatten_ids"], backgrounds=bg,
        masks=masks, filtering=filtering)
    loss = sum((o * T(u)).sum() for o, u in zip(out[:5], ups))
    loss.backward()
    res = {f"out{i}": npy(o) for i, o in enumerate(out)}
    for k, v in leaves.items():
        res[f"v_{k}"] = npy(v.grad) if v.grad is not None else np.zeros(v.shape, np.float32)
    return res


def plain_compositor(W, p, s, opacities, ups):
    leaves = dict(means2d=p["means2d"].detach().clone(), M=p["M"].detach().clone(),
                  colors=p["colors"].detach().clone(), opacities=opacities.detach().clone(),
                  normals=p["normals"].detach().clone())
    for v in leaves.values():
        v.requires_grad_(True)
    densify = torch.zeros_like(leaves["means2d"], requires_grad=True)
    bg = T(s.backgrounds) if s.backgrounds is not None else None
    out = W.rasterize_to_pixels_2dgs(leaves["means2d"], leaves["M"], leaves["colors"], leaves["opacities"],
                                     leaves["normals"], densify, s.width, s.height, s.tile_size, p["offsets"],
                                     p["flatten_ids"], backgrounds=bg)
    loss = sum((o * T(u)).sum() for o, u in zip(out[:5], ups))
    loss.backward()
    res = {f"out{i}": npy(o) for i, o in enumerate(out)}
    for k, v in leaves.items():
        res[f"v_{k}"] = npy(v.grad)
    return res


def pixel_shapes(s):
    C, H, Wd = 1, s.height, s.width
    return [(C, H, Wd, 3), (C, H, Wd, 1), (C, H, Wd, 3), (C, H, Wd, 1), (C, H, Wd, 1)]


def store_compositor(d, prefix, res, n_keep):
    for k, v in res.items():
        if k == "v_textures":
            rows, vals, norms = keep_rows(v, n_keep)
            d[f"{prefix}__v_textures_rows"] = rows
            d[f"{prefix}__v_textures_vals"] = vals
            d[f"{prefix}__v_textures_norms"] = norms
        else:
            d[f"{prefix}__{k}"] = v


def small_case(R, W, s, filters):
    """End to end and stage by stage on one small scene (C = 1)."""
    d = {"inputs_sha256": np.array(digest(s.means, s.quats, s.scales, s.opacities, s.colors, s.textures,
                                          s.viewmats, s.Ks))}
    means, quats, scales = T(s.means), T(s.quats), T(s.scales)
    opac, colors, tex = T(s.opacities), T(s.colors), T(s.textures)
    with torch.no_grad():
        p = project_and_shade(W, s, means, quats, scales, colors)
    for k in ("radii", "means2d", "depths", "M", "normals", "colors", "tpg", "isect_ids", "flatten_ids", "offsets"):
        d[f"stage__{k}"] = npy(p[k])
    # the projection's adjoint on its own (_wrapper.py:1267 fully_fused_projection_2dgs): seeded upstream
    # gradients on every visible entry's outputs (culled entries' outputs are left unwritten by the reference)
    pleaves = [x.detach().clone().requires_grad_(True) for x in (means, quats, scales)]
    pr = W.fully_fused_projection_2dgs(*pleaves, T(s.viewmats), T(s.Ks), s.width, s.height, 0.3, s.near_plane,
                                       s.far_plane, 0.0)
    d["projvjp_seed"] = np.array(77)
    pups = proj_upstream(77, pr[0].shape)
    vis = (pr[0] > 0).float()
    loss = sum((o * T(u) * vis.view(vis.shape + (1,) * (o.dim() - 2))).sum() for o, u in zip(pr[1:], pups))
    loss.backward()
    for k, leaf in zip(("means", "quats", "scales"), pleaves):
        d[f"projvjp__v_{k}"] = npy(leaf.grad)
    seeds = {"up": 101}
    d["up_seed"] = np.array(seeds["up"])
    ups = upstream(seeds["up"], pixel_shapes(s))
    op_c = opac[None].contiguous()
    for f in filters:
        res = compositor(W, p, s, tex, op_c, f, ups)
        store_compositor(d, f"comp_{f}", res, ROWS_KEPT)
    # plain 2DGS compositor on the same stage inputs
    store_compositor(d, "plain", plain_compositor(W, p, s, op_c, ups), ROWS_KEPT)
    # the renderer end to end, leaf gradients (the public entry point, rendering.py:1342)
    for f in filters:
        leaves = [x.detach().clone().requires_grad_(True) for x in (means, quats, scales, opac, colors, tex)]
        bg = ref_backgrounds(s, f)
        out = R.rasterization_textured_gaussians(*leaves, T(s.viewmats), T(s.Ks), s.width, s.height,
                                                 near_plane=s.near_plane, far_plane=s.far_plane,
                                                 sh_degree=s.sh_degree, tile_size=s.tile_size, backgrounds=bg,
                                                 filtering=f)
        outs = [out[0], out[1], out[2], out[4], out[5]]
        loss = sum((o * T(u)).sum() for o, u in zip(outs, ups))
        loss.backward()
        pre = f"e2e_{f}"
        for i, o in enumerate(outs):
            d[f"{pre}__out{i}"] = npy(o)
        d[f"{pre}__contrib_sum"] = npy(out[6])
        d[f"{pre}__contrib_count"] = npy(out[7])
        for name, leaf in zip(("means", "quats", "scales", "opacities", "colors"), leaves[:5]):
            d[f"{pre}__v_{name}"] = npy(leaf.grad)
        rows, vals, norms = keep_rows(npy(leaves[5].grad), ROWS_KEPT)
        d[f"{pre}__v_textures_rows"], d[f"{pre}__v_textures_vals"], d[f"{pre}__v_textures_norms"] = rows, vals, norms
    return d


def aniso_safe_rows(W, s):
    """Rows of scene s whose footprint quads stay convex on every pixel the compositor visits.

    The reference's anisotropic_bilinear clipping (filters/anisotropic_bilinear.cuh:80-160) keeps
    up to 8 vertices in fixed arrays; a self-intersecting quad -- a pixel whose corner rays meet
    the splat's plane on both sides, i.e. a pixel crossing the image line where rays run parallel
    to the plane -- can need more (undefined behaviour, possibly an out-of-bounds write).  That
    line is z(px, py) = 0 for z the third component of (px M2 - M0) x (py M2 - M1), affine in the
    pixel position; a splat is kept only if the line stays 1.5 (radius + tile + 2) pixels from its
    centre, beyond every pixel of every tile it touches.  Computed on the reference's own FP32
    projection, in FP64."""
    with torch.no_grad():
        radii, means2d, _, M, _ = W.fully_fused_projection_2dgs(T(s.means), T(s.quats), T(s.scales),
                                                                T(s.viewmats), T(s.Ks), s.width, s.height, 0.3,
                                                                s.near_plane, s.far_plane, 0.0)
    r = npy(radii)[0].astype(np.float64)
    M = npy(M)[0].astype(np.float64)
    c = npy(means2d)[0].astype(np.float64)
    M0, M1, M2 = M[:, 0], M[:, 1], M[:, 2]

    def cz(u, v):
        return u[:, 0] * v[:, 1] - u[:, 1] * v[:, 0]

    a, b, c0 = -cz(M2, M1), -cz(M0, M2), cz(M0, M1)
    dist = np.abs(a * c[:, 0] + b * c[:, 1] + c0) / np.maximum(np.hypot(a, b), 1e-300)
    keep = (r <= 0) | (dist >= 1.5 * (r + s.tile_size + 2))
    return np.flatnonzero(keep).astype(np.int64)


def subset(s, rows):
    import copy

    t = copy.copy(s)
    for k in ("means", "quats", "scales", "opacities", "colors", "textures"):
        setattr(t, k, np.ascontiguousarray(getattr(s, k)[rows]))
    return t


def sampled_case(W, s, tex, sample_rows, every, seed, filtering="bilinear", safe_rows=None):
    """Camera 0 of a large scene; outputs on sampled tiles, upstream gradients only there.

    The reference projects, shades and intersects the whole scene.  Its compositor cannot take the
    whole texture tensor (over 2^31 elements: it indexes textures through a 32-bit packed accessor and
    refuses the call), so it runs on the sampled tiles' sub-problem: the Gaussians their splat lists
    use, in ascending id order, and offsets that give every other tile an empty list.  A tile's result
    depends only on its own list, so this is the reference's result for those tiles.  safe_rows (sorted
    Gaussian ids): the splat lists keep only those (anisotropic_bilinear: the rows aniso_safe_rows allows)."""
    means, quats, scales, colors = T(s.means), T(s.quats), T(s.scales), T(s.colors)
    with torch.no_grad():
        p = project_and_shade(W, s, means, quats, scales, colors)
    ts, tw, th = s.tile_size, p["tw"], p["th"]
    mask = np.zeros((1, th, tw), bool)
    for r in sample_rows:
        mask[0, r, ::every] = True
    H, Wd = s.height, s.width
    pix = np.repeat(np.repeat(mask, ts, 1), ts, 2)[:, :H, :Wd].astype(np.float32)[..., None]
    ups = [u * pix for u in upstream(seed, pixel_shapes(s))]
    # the sampled tiles' splat lists and the rows they use
    off = npy(p["offsets"]).reshape(-1)
    fl = npy(p["flatten_ids"])
    tiles = np.flatnonzero(mask.reshape(-1))
    lists = [fl[off[t]:(off[t + 1] if t + 1 < off.size else fl.size)] for t in tiles]
    if safe_rows is not None:
        lists = [x[np.isin(x, safe_rows)] for x in lists]
    rows = np.unique(np.concatenate(lists))
    d = {"inputs_sha256": np.array(digest(s.means, s.quats, s.scales, s.opacities, s.colors, s.viewmats, s.Ks)),
         "up_seed": np.array(seed), "sample_rows": np.array(sample_rows), "sample_every": np.array(every),
         "tiles": tiles, "tile_counts": np.array([x.size for x in lists]), "tile_lists": np.concatenate(lists),
         "rows": rows}
    from tests import _refgold

    sub_off, sub_fl = _refgold.sampled_layout(d, th, tw)
    rt = T(rows, torch.int64)
    sub_tex = tex[rt].contiguous()
    d["tex_sha256_rows"] = np.array(digest(npy(sub_tex)))
    sub = {k: p[k][:, rt].contiguous() for k in ("means2d", "M", "normals", "colors")}
    sub["offsets"] = T(sub_off, torch.int32)
    sub["flatten_ids"] = T(sub_fl, torch.int32)
    op_c = T(s.opacities[rows])[None].contiguous()
    res = compositor(W, sub, s, sub_tex, op_c, filtering, ups)
    for k in ("radii", "means2d", "depths", "M", "normals", "colors"):
        d[f"stage__{k}"] = npy(p[k])[0, rows]
    d["stage__n_isects"] = np.array(fl.size)
    d["stage__isect_digest"] = np.array(digest(npy(p["isect_ids"]), fl, off))
    sel = pix[..., 0] > 0
    pre = f"comp_{filtering}"
    for i in range(5):
        d[f"{pre}__out{i}"] = res[f"out{i}"][sel]
    for k in ("means2d", "M", "colors", "opacities", "normals"):
        d[f"{pre}__v_{k}"] = res[f"v_{k}"][0]
    keep, vals, norms = keep_rows(res["v_textures"], ROWS_KEPT_LARGE)
    d[f"{pre}__v_textures_rows"], d[f"{pre}__v_textures_vals"] = keep, vals
    d[f"{pre}__v_textures_norms"] = norms
    return d

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    ap.add_argument("--cases", default="small,adjoint,views8,mix1m")
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    R, W = reference()
    cases = a.cases.split(",")
    if "small" in cases:
        d = small_case(R, W, scenes.small(), ("bilinear", "bilinear_bwd2"))
        np.savez_compressed(os.path.join(a.out, "ref_small.npz"), **d)
        print("small done", flush=True)
    if "adjoint" in cases:
        s = scenes.adjoint()
        d = small_case(R, W, s, ("bilinear", "bilinear_bwd2", "mipmapped2"))
        np.savez_compressed(os.path.join(a.out, "ref_adjoint.npz"), **d)
        keep = aniso_safe_rows(W, s)
        d = small_case(R, W, subset(s, keep), ("anisotropic_bilinear",))
        d["kept_rows"] = keep
        np.savez_compressed(os.path.join(a.out, "ref_adjoint_aniso.npz"), **d)
        print("adjoint done", flush=True)
    if "views8" in cases:
        s = scenes.views8(with_textures=False)
        N, Rt = s.means.shape[0], s.extra["texture_res"]
        s.viewmats, s.Ks = s.viewmats[:1], s.Ks[:1]
        g = torch.Generator(device=DEV)
        g.manual_seed(1)
        tex = torch.rand((N, Rt, Rt, 4), generator=g, device=DEV)
        d = sampled_case(W, s, tex, (20, 25), 6, 202)
        np.savez_compressed(os.path.join(a.out, "ref_views8.npz"), **d)
        del tex
        torch.cuda.empty_cache()
        print("views8 done", flush=True)
    if any(c.startswith("mix1m") for c in cases):
        import bench

        sc = bench.make_scene(0, 1, 1_000_000, 4)
        s = scenes.Scene(sc["means"], sc["quats"], sc["scales"], sc["opacities"], sc["colors"], None,
                         sc["viewmats"][:1], sc["Ks"][:1], sc["width"], sc["height"], 0, far_plane=100.0,
                         tile_size=8, name="mix1m")
        tex = bench.gpu_textures(s.means.shape[0], 32, torch.device(DEV))
        if "mix1m" in cases:
            d = sampled_case(W, s, tex, (60, 95), 10, 303)
            np.savez_compressed(os.path.join(a.out, "ref_mix1m.npz"), **d)
            print("mix1m done", flush=True)
        if "mix1m_bwd2" in cases:
            d = sampled_case(W, s, tex, (30, 120), 10, 306, "bilinear_bwd2")
            np.savez_compressed(os.path.join(a.out, "ref_mix1m_bwd2.npz"), **d)
            print("mix1m_bwd2 done", flush=True)
        if "mix1m_mip" in cases:
            d = sampled_case(W, s, tex, (50, 85), 10, 305, "mipmapped2")
            np.savez_compressed(os.path.join(a.out, "ref_mix1m_mip.npz"), **d)
            print("mix1m_mip done", flush=True)
        if "mix1m_aniso" in cases:
            d = sampled_case(W, s, tex, (40, 75, 110), 10, 304, "anisotropic_bilinear", aniso_safe_rows(W, s))
            np.savez_compressed(os.path.join(a.out, "ref_mix1m_aniso.npz"), **d)
            print("mix1m_aniso done", flush=True)

if __name__ == "__main__":
    main()
