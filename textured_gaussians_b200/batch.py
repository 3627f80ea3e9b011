"""Batching form: many views of uneven size over several scenes in one pass.

The reference renders C cameras of one image size and one scene per call
(``rasterization_textured_gaussians``, textured_gaussians/rendering.py:1342-1685).
Here a batch is any number of views, each with its own resolution and its own
scene.  The scenes' Gaussians live in one concatenated parameter store
(scene s owns rows ``[scene_offsets[s], scene_offsets[s+1])``), and one pass
renders every view:

* one packed projection over every (view, Gaussian of the view's scene)
  pair, each view with its own image size (``tg_project_packed_*`` with a
  view table and per-view Gaussian ranges);
* one intersection pass and one key sort over all views (per-view tile grids,
  view-local tile ids in the keys);
* one offsets pass over the flat list of every view's tiles, and one
  compositor launch forward and one backward over that list, taking the
  tiles heaviest first (a permutation sorted by intersection count), so the
  long tiles of large views do not form the launch's tail.

Forward results equal per-view calls of the drop-in bit for bit (same
per-entry arithmetic, same per-tile splat order); gradients equal the sum of
the per-view gradients up to float-atomic summation order.
"""
from __future__ import annotations

import math
from typing import List, Optional, Sequence

import numpy as np
import torch
from torch import Tensor

from . import _backend as B
from .cuda._wrapper import (
    _FILTER_ADJOINT,
    _FullyFusedProjectionPacked2DGS,
    isect_offset_encode_views,
    isect_tiles,
    n_isects_of,
    rasterize_to_pixels_2dgs,
    rasterize_to_pixels_textured_gaussians,
    spherical_harmonics,
    tile_order_heaviest_first,
)
from .rendering import _inverse
from .utils import depth_to_normal

# layout of tg_view (include/tg2dgs.h)
TG_VIEW = np.dtype([("width", "<i4"), ("height", "<i4"), ("tile_width", "<i4"), ("tile_height", "<i4"),
                    ("tile_base", "<i8"), ("pix_base", "<i8")])
assert TG_VIEW.itemsize == 32


class ViewTable:
    """Per-view image sizes, tile grids and flat tile / pixel bases (host
    lists) plus their device copies (the tg_view array and tile -> view map)."""

    def __init__(self, widths: Sequence[int], heights: Sequence[int], tile_size: int, device):
        assert len(widths) == len(heights) and len(widths) > 0
        self.widths = [int(w) for w in widths]
        self.heights = [int(h) for h in heights]
        self.tile_size = int(tile_size)
        self.n_views = len(self.widths)
        self.tile_w = [math.ceil(w / tile_size) for w in self.widths]
        self.tile_h = [math.ceil(h / tile_size) for h in self.heights]
        tiles = [tw * th for tw, th in zip(self.tile_w, self.tile_h)]
        self.pix_count = [w * h for w, h in zip(self.widths, self.heights)]
        self.tile_base = [0] + list(np.cumsum(tiles)[:-1].tolist())
        self.pix_base = [0] + list(np.cumsum(self.pix_count)[:-1].tolist())
        self.n_tiles = int(sum(tiles))
        self.n_pixels = int(sum(self.pix_count))
        self.key_tiles = int(max(tiles))  # sets the tile bits of the intersection keys
        arr = np.zeros(self.n_views, TG_VIEW)
        arr["width"], arr["height"] = self.widths, self.heights
        arr["tile_width"], arr["tile_height"] = self.tile_w, self.tile_h
        arr["tile_base"], arr["pix_base"] = self.tile_base, self.pix_base
        self.device = device
        self.views = torch.from_numpy(arr.view(np.uint8).copy()).to(device)
        self.tile_view = torch.from_numpy(np.repeat(np.arange(self.n_views, dtype=np.int32), tiles)).to(device)
        self._ranges = {}

    def gauss_ranges(self, scene_offsets: Sequence[int], view_scenes: Sequence[int]):
        """[C,2] int64 device tensor of each view's Gaussian range, and the longest
        range (cached, so a captured step makes no host-to-device copy)."""
        key = (tuple(int(o) for o in scene_offsets), tuple(int(v) for v in view_scenes))
        if key not in self._ranges:
            offs = key[0]
            rng = [(offs[v], offs[v + 1]) for v in key[1]]
            t = torch.tensor(rng, dtype=torch.int64).to(self.device)
            self._ranges[key] = (t, max(b - a for a, b in rng))
        return self._ranges[key]

    def split(self, flat: Tensor) -> List[Tensor]:
        """Per-view [H, W, ...] views of a flat per-pixel tensor [n_pixels, ...]."""
        return [flat[b:b + n].view(h, w, *flat.shape[1:])
                for b, n, h, w in zip(self.pix_base, self.pix_count, self.heights, self.widths)]


def rasterization_textured_gaussians_batch(
    means: Tensor,
    quats: Tensor,
    scales: Tensor,
    opacities: Tensor,
    colors: Tensor,
    textures: Optional[Tensor],
    scene_offsets: Sequence[int],
    viewmats: Tensor,
    Ks: Tensor,
    widths: Sequence[int],
    heights: Sequence[int],
    view_scenes: Sequence[int],
    texture_range_x: float = 3.0,
    texture_range_y: float = 3.0,
    near_plane: float = 0.01,
    far_plane: float = 1e10,
    radius_clip: float = 0.0,
    eps2d: float = 0.3,
    sh_degree: Optional[int] = None,
    tile_size: int = 16,
    backgrounds: Optional[Tensor] = None,
    render_mode: str = "RGB",
    absgrad: bool = False,
    norm_rot_grad: bool = False,
    depth_mode: str = "expected",
    gs_contrib_threshold: float = 0.0,
    filtering: str = "bilinear",
    g_weight: float = 1.0,
    *,
    texture_storage: Optional[Tensor] = None,
    texture_scales: Optional[Tensor] = None,
    adjoint: str = "reference",
    tile_order: str = "heaviest_first",
    view_table: Optional[ViewTable] = None,
    batch_depth: int = 0,
    persistent: bool = False,
    fuse_sh: bool = True,
):
    """Render C views of uneven size, view c showing scene ``view_scenes[c]``.

    Parameters are those of ``rasterization_textured_gaussians`` over the
    concatenated scenes (means [N,3] ... textures [N,R,R,4], N = sum of the
    scenes' sizes; ``textures=None`` renders plain 2DGS), plus
    ``scene_offsets`` [S+1], the per-view ``widths`` / ``heights`` and
    ``view_scenes``.  ``tile_order`` is "heaviest_first" or "launch".

    Returns ``(colors, alphas, normals, normals_from_depth, distort, median,
    gs_contrib_sum, gs_contrib_count, meta)`` where the per-pixel entries are
    lists of per-view [H_c, W_c, ...] tensors (views into flat buffers kept in
    ``meta``), normals in world space as in the drop-in, and the statistics
    per Gaussian of the concatenated store [N].
    """
    N = means.shape[0]
    C = viewmats.shape[0]
    dev = means.device
    assert Ks.shape == (C, 3, 3) and len(widths) == len(heights) == len(view_scenes) == C
    assert render_mode in ("RGB", "D", "ED", "RGB+D", "RGB+ED"), render_mode
    offs = [int(o) for o in scene_offsets]
    assert offs[0] == 0 and offs[-1] == N and all(a <= b for a, b in zip(offs, offs[1:])), offs
    vt = view_table or ViewTable(widths, heights, tile_size, dev)
    assert vt.widths == [int(w) for w in widths] and vt.heights == [int(h) for h in heights]
    assert vt.tile_size == tile_size
    ranges, max_range = vt.gauss_ranges(offs, view_scenes)
    mode = B.TG_ADJ_EXACT if adjoint == "exact" else (B.TG_ADJ_BWD2 if norm_rot_grad else B.TG_ADJ_REFERENCE)

    fuse = fuse_sh and sh_degree is not None
    sh = (colors.float().contiguous(), int(sh_degree)) if fuse else (None, 0)
    proj = _FullyFusedProjectionPacked2DGS.apply(
        means.contiguous(), quats.contiguous(), scales.contiguous(), viewmats.contiguous(), Ks.contiguous(), 0, 0,
        eps2d, near_plane, far_plane, radius_clip, False, mode, (vt.views, ranges, max_range), *sh)
    camera_ids, gaussian_ids, radii, means2d, depths, ray_transforms, normals = proj[:7]
    opac = opacities[gaussian_ids]
    if fuse:
        cols = proj[-1]
    elif sh_degree is not None:
        camtoworlds = _inverse(viewmats)
        dirs = means[gaussian_ids, :] - camtoworlds[camera_ids, :3, 3]
        cols = spherical_harmonics(sh_degree, dirs, colors[gaussian_ids], masks=radii > 0)
        cols = torch.clamp_min(cols + 0.5, 0.0)
    else:
        cols = colors[gaussian_ids]
    if render_mode in ("RGB+D", "RGB+ED"):
        cols = torch.cat((cols, depths[..., None]), dim=-1)
    elif render_mode in ("D", "ED"):
        cols = depths[..., None]
    densify = torch.zeros_like(means2d, dtype=means.dtype, requires_grad=True)

    tiles_per_gauss, isect_ids, flatten_ids = isect_tiles(
        means2d, radii, depths, tile_size, 0, 0, packed=True, n_cameras=C, camera_ids=camera_ids,
        gaussian_ids=gaussian_ids, view_table=vt)
    isect_offsets = isect_offset_encode_views(isect_ids, vt)
    order = (tile_order_heaviest_first(isect_offsets, n_isects_of(flatten_ids)) if tile_order == "heaviest_first"
             else None)

    common = dict(backgrounds=backgrounds, packed=True, absgrad=absgrad, gs_contrib_threshold=gs_contrib_threshold,
                  gaussian_ids=gaussian_ids, tile_order=order, view_table=vt, batch_depth=batch_depth,
                  persistent=persistent)
    if textures is not None:
        if filtering not in _FILTER_ADJOINT:
            raise Exception(f"Unsupported filter type {filtering}")
        outs = rasterize_to_pixels_textured_gaussians(
            means2d, ray_transforms, cols, opac, textures, texture_range_x, texture_range_y, normals, densify, 0, 0,
            tile_size, isect_offsets, flatten_ids, filtering=filtering, g_weight=g_weight,
            texture_storage=texture_storage, texture_scales=texture_scales, **common)
    else:
        outs = rasterize_to_pixels_2dgs(means2d, ray_transforms, cols, opac, normals, densify, 0, 0, tile_size,
                                        isect_offsets, flatten_ids, n_gaussians=N, **common)
    flat_colors, flat_alphas, flat_normals, flat_distort, flat_median, contrib_sum, contrib_count = outs
    if render_mode in ("ED", "RGB+ED"):
        flat_colors = torch.cat([flat_colors[..., :-1], flat_colors[..., -1:] / flat_alphas.clamp(min=1e-10)], dim=-1)

    camtoworlds = _inverse(viewmats)
    colors_v, alphas_v = vt.split(flat_colors), vt.split(flat_alphas)
    median_v = vt.split(flat_median)
    normals_v = [torch.einsum("ij,hwj->hwi", camtoworlds[c, :3, :3], n)
                 for c, n in enumerate(vt.split(flat_normals))]
    normals_from_depth = None
    if render_mode in ("RGB+ED", "RGB+D"):
        normals_from_depth = []
        for c in range(C):
            d = colors_v[c][..., -1:] if depth_mode == "expected" else median_v[c]
            normals_from_depth.append(depth_to_normal(d[None], camtoworlds[c:c + 1], Ks[c:c + 1])[0])
    meta = {
        "camera_ids": camera_ids, "gaussian_ids": gaussian_ids, "radii": radii, "means2d": means2d,
        "depths": depths, "ray_transforms": ray_transforms, "opacities": opac, "normals": normals,
        "tiles_per_gauss": tiles_per_gauss, "isect_ids": isect_ids, "flatten_ids": flatten_ids,
        "isect_offsets": isect_offsets, "tile_order": order, "view_table": vt, "tile_size": tile_size,
        "n_cameras": C, "gradient_2dgs": densify, "flat_colors": flat_colors, "flat_alphas": flat_alphas,
        "flat_normals": flat_normals, "render_distort": flat_distort,
    }
    return (colors_v, alphas_v, normals_v, normals_from_depth, vt.split(flat_distort), median_v, contrib_sum,
            contrib_count, meta)
