"""Whole-pipeline CPU oracle -- TEST INFRASTRUCTURE ONLY.

``render`` follows rasterization_textured_gaussians / rasterization_2dgs
(textured_gaussians/rendering.py:1474-1685, :1135-1338) stage by stage on the
CPU oracle, for render modes "RGB" and "RGB+D" and the dense layout.
``render_backward`` chains the stage adjoints by hand (the reference relies on
torch autograd for the glue: opacity repeat, SH + 0.5 clamp, the depth
channel, and the rotation of normals to world space).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import oracle as O


@dataclass
class Cache:
    dtype: object
    C: int
    N: int
    radii: np.ndarray
    means2d: np.ndarray
    depths: np.ndarray
    M: np.ndarray
    normals: np.ndarray
    tiles_per_gauss: np.ndarray
    isect_ids: np.ndarray
    flatten_ids: np.ndarray
    offsets: np.ndarray
    opac_rep: np.ndarray
    colors: np.ndarray      # per-camera colours fed to the compositor [C,N,D]
    sh_pre: Optional[np.ndarray]  # SH output before the +0.5 clamp
    dirs: Optional[np.ndarray]
    fwd: O.RasterFwdOut
    rot_c2w: np.ndarray     # [C,3,3] rotation of inv(viewmats)


def render(means, quats, scales, opacities, colors, textures, viewmats, Ks, W, H, sh_degree=None, tile_size=16,
           near_plane=0.01, far_plane=1e10, radius_clip=0.0, backgrounds=None, render_mode="RGB", range_x=3.0,
           range_y=3.0, g_weight=1.0, contrib_threshold=0.0, dtype=np.float32, proj_override=None):
    """Returns (render_colors, render_alphas, render_normals_world, cache).

    ``textures=None`` renders the plain 2DGS compositor.  ``proj_override``
    (radii, means2d, depths, M, normals) replaces the oracle projection, so
    downstream stages can be compared on identical inputs.
    """
    assert render_mode in ("RGB", "RGB+D")
    C, N = viewmats.shape[0], means.shape[0]
    if proj_override is None:
        radii, means2d, depths, M, normals = O.project_fwd(means, quats, scales, viewmats, Ks, W, H, near_plane,
                                                           far_plane, radius_clip, dtype=dtype)
    else:
        radii, means2d, depths, M, normals = (np.asarray(x) for x in proj_override)
        means2d, depths, M, normals = (x.astype(dtype) for x in (means2d, depths, M, normals))
    tw, th = -(-W // tile_size), -(-H // tile_size)
    tpg, isect_ids, flatten_ids = O.isect_tiles(means2d, radii, depths, tile_size, tw, th, C)
    offsets = O.isect_offset_encode(isect_ids, C, tw, th)
    opac_rep = np.tile(np.asarray(opacities, dtype)[None], (C, 1))
    sh_pre, dirs = None, None
    if sh_degree is not None:
        c2w = np.linalg.inv(np.asarray(viewmats, np.float64))
        dirs = (np.asarray(means, np.float64)[None] - c2w[:, None, :3, 3]).astype(dtype)
        coeffs = np.broadcast_to(np.asarray(colors, dtype)[None], (C,) + colors.shape)
        sh_pre = O.sh_fwd(sh_degree, dirs, coeffs, masks=radii > 0, dtype=dtype)
        cols = np.maximum(sh_pre + dtype(0.5), dtype(0))
    else:
        cols = np.broadcast_to(np.asarray(colors, dtype)[None], (C,) + colors.shape).copy() if colors.ndim == 2 \
            else np.asarray(colors, dtype)
    if render_mode == "RGB+D":
        cols = np.concatenate([cols, depths[..., None]], -1)
    fwd = O.raster_fwd(means2d, M, cols, opac_rep, normals, textures, offsets, flatten_ids, W, H, tile_size,
                       range_x, range_y, backgrounds, contrib_threshold=contrib_threshold, g_weight=g_weight,
                       dtype=dtype)
    rot = np.linalg.inv(np.asarray(viewmats, np.float64))[:, :3, :3].astype(dtype)
    normals_world = np.einsum("cij,chwj->chwi", rot, fwd.normals)
    cache = Cache(dtype, C, N, radii, means2d, depths, M, normals, tpg, isect_ids, flatten_ids, offsets, opac_rep,
                  cols, sh_pre, dirs, fwd, rot)
    return fwd.colors, fwd.alphas, normals_world, cache


def render_backward(cache: Cache, means, quats, scales, opacities, colors, textures, viewmats, Ks, W, H,
                    v_colors, v_alphas=None, v_normals_world=None, v_distort=None, v_median=None, sh_degree=None,
                    tile_size=16, backgrounds=None, range_x=3.0, range_y=3.0, g_weight=1.0, raster_mode=0,
                    proj_mode=0):
    """Gradients w.r.t. means, quats, scales, opacities, colors (or SH coefficients) and textures."""
    dt = cache.dtype
    C, N = cache.C, cache.N
    z = lambda shape: np.zeros(shape, dt)
    v_alphas = z((C, H, W, 1)) if v_alphas is None else np.asarray(v_alphas, dt)
    v_distort = z((C, H, W, 1)) if v_distort is None else np.asarray(v_distort, dt)
    v_median = z((C, H, W, 1)) if v_median is None else np.asarray(v_median, dt)
    if v_normals_world is None:
        v_ncam = z((C, H, W, 3))
    else:
        v_ncam = np.einsum("cji,chwj->chwi", cache.rot_c2w, np.asarray(v_normals_world, dt))
    g = O.raster_bwd(cache.means2d, cache.M, cache.colors, cache.opac_rep, cache.normals, textures, cache.offsets,
                     cache.flatten_ids, W, H, tile_size, cache.fwd, v_colors, v_alphas, v_ncam, v_distort, v_median,
                     range_x, range_y, backgrounds, g_weight=g_weight, mode=raster_mode, dtype=dt)
    v_opacities = g.v_opacities.sum(0)
    v_cols = g.v_colors
    v_depths = z((C, N))
    if v_cols.shape[-1] == 4 and cache.colors.shape[-1] == 4:  # RGB+D: last channel is the depth
        v_depths = v_depths + v_cols[..., 3]
        v_cols = v_cols[..., :3]
    v_means_extra = z((N, 3))
    if sh_degree is not None:
        v_sh = v_cols * (cache.sh_pre + dt(0.5) >= 0)
        coeffs = np.broadcast_to(np.asarray(colors, dt)[None], (C,) + colors.shape)
        v_coeffs, v_dirs = O.sh_bwd(sh_degree, cache.dirs, coeffs, v_sh, masks=cache.radii > 0, dtype=dt)
        v_color_param = v_coeffs.sum(0)
        v_means_extra = v_dirs.sum(0)
    else:
        v_color_param = v_cols.sum(0) if np.asarray(colors).ndim == 2 else v_cols
    v_means, v_quats, v_scales = O.project_bwd(means, quats, scales, viewmats, Ks, cache.radii, cache.M, g.v_means2d,
                                               v_depths, g.v_normals, g.v_M, mode=proj_mode, dtype=dt)
    return {
        "means": v_means + v_means_extra,
        "quats": v_quats,
        "scales": v_scales,
        "opacities": v_opacities,
        "colors": v_color_param,
        "textures": g.v_textures,
        "raster": g,
    }
