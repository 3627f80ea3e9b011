"""Renderer API: drop-in ``rasterization_2dgs`` and ``rasterization_textured_gaussians``.

Same arguments, defaults, return 9-tuple and ``meta`` keys as
textured_gaussians/rendering.py:1009-1338 and :1342-1685 of the reference:
projection -> tile intersection (+ sort) -> offsets -> SH colours -> compositor
-> expected-depth normalisation / depth normals -> normals to world space.
Every stage runs this package's sm_100a kernels; the glue between them
(repeat of opacities, camera centres, clamps, ED division, normal rotation)
is torch on the same device.

``packed=True`` runs the packed layout end to end (visible (camera, Gaussian)
entries only, ``meta["camera_ids"]`` / ``meta["gaussian_ids"]``), with
``sparse_grad`` giving COO gradients for means, quats and scales.

Extensions (keyword-only, default off): ``texture_storage`` /
``texture_scales`` (sample BF16 / FP16 / FP8 textures, gradients to the FP32
``textures``), ``filtering="bilinear_exact"`` and ``adjoint="exact"`` (exact
adjoint end to end), ``tile_order`` ("heaviest_first", the default: compositor
tiles taken by descending intersection count, so the longest tiles do not form
the launch's tail; "launch": tile index order; the results are the same),
``batch_depth`` (splats staged per compositor batch; 0 = tile_size^2),
``persistent`` (compositor CTAs take tiles from a device work counter),
``tile_size`` 32 besides the reference's 8 and 16, ``fuse_sh`` (default
on: the SH colours are computed inside the projection kernels instead of the
reference's separate SH op + camera-centre inverse + clamp glue), and, for
the textured renderer, ``transmittance`` ("divide", the reference's scheme, or
"checkpoint": per-batch transmittance kept by the forward, see
``rasterize_to_pixels_textured_gaussians``).
"""
from __future__ import annotations

import math
from typing import Dict, Optional, Tuple

import torch
from torch import Tensor

from .cuda._wrapper import (
    fully_fused_projection_2dgs,
    isect_offset_encode,
    isect_tiles,
    n_isects_of,
    tile_order_heaviest_first,
    rasterize_to_pixels_2dgs,
    rasterize_to_pixels_textured_gaussians,
    spherical_harmonics,
    spherical_harmonics_shared,
)
from .utils import depth_to_normal

_RENDER_MODES = ["RGB", "D", "ED", "RGB+D", "RGB+ED"]


def _inverse(m: Tensor) -> Tensor:
    """Batched 4x4 inverse without the host-side error check of torch.inverse
    (the same kernel; no synchronisation, so it can sit inside a CUDA graph)."""
    return torch.linalg.inv_ex(m)[0]


def _prepare(means, quats, scales, opacities, colors, viewmats, Ks, width, height, near_plane, far_plane,
             radius_clip, eps2d, sh_degree, packed, tile_size, render_mode, sparse_grad, norm_rot_grad, distloss,
             adjoint, tile_order="heaviest_first", fuse_sh=True):
    assert tile_order in ("launch", "heaviest_first"), tile_order
    N = means.shape[0]
    C = viewmats.shape[0]
    assert means.shape == (N, 3), means.shape
    assert quats.shape == (N, 4), quats.shape
    assert scales.shape == (N, 3), scales.shape
    assert opacities.shape == (N,), opacities.shape
    assert viewmats.shape == (C, 4, 4), viewmats.shape
    assert Ks.shape == (C, 3, 3), Ks.shape
    assert render_mode in _RENDER_MODES, render_mode
    if distloss:
        assert render_mode in ["D", "ED", "RGB+D", "RGB+ED"], (
            f"distloss requires depth rendering, render_mode should be D, ED, RGB+D, RGB+ED, but got {render_mode}")
    if sh_degree is None:
        assert (colors.dim() == 2 and colors.shape[0] == N) or (
            colors.dim() == 3 and colors.shape[:2] == (C, N)), colors.shape
    else:
        assert colors.dim() == 3 and colors.shape[0] == N and colors.shape[2] == 3, colors.shape
        assert (sh_degree + 1) ** 2 <= colors.shape[1], colors.shape

    fuse = fuse_sh and sh_degree is not None
    proj = fully_fused_projection_2dgs(
        means, quats, scales, viewmats, Ks, width, height, eps2d, near_plane, far_plane, radius_clip, packed,
        sparse_grad, norm_rot_grad, adjoint=adjoint, sh_coeffs=colors if fuse else None,
        sh_degree=sh_degree if fuse else None)
    if packed:
        camera_ids, gaussian_ids, radii, means2d, depths, ray_transforms, normals = proj[:7]
        opacities = opacities[gaussian_ids]
    else:
        radii, means2d, depths, ray_transforms, normals = proj[:5]
        opacities = opacities.repeat(C, 1)
        camera_ids, gaussian_ids = None, None

    densify = torch.zeros_like(means2d, dtype=means.dtype, requires_grad=True, device=means.device)
    tile_width = math.ceil(width / float(tile_size))
    tile_height = math.ceil(height / float(tile_size))
    tiles_per_gauss, isect_ids, flatten_ids = isect_tiles(
        means2d, radii, depths, tile_size, tile_width, tile_height, packed=packed, n_cameras=C,
        camera_ids=camera_ids, gaussian_ids=gaussian_ids)
    isect_offsets = isect_offset_encode(isect_ids, C, tile_width, tile_height)
    order = (tile_order_heaviest_first(isect_offsets, n_isects_of(flatten_ids)) if tile_order == "heaviest_first"
             else None)

    if fuse:
        colors = proj[-1]  # SH colours computed inside the projection, +0.5 and clamp applied
    elif sh_degree is not None:
        camtoworlds = _inverse(viewmats)
        if packed:
            dirs = means[gaussian_ids, :] - camtoworlds[camera_ids, :3, 3]
            colors = spherical_harmonics(sh_degree, dirs, colors[gaussian_ids], masks=radii > 0)  # [nnz, 3]
        else:
            dirs = means[None, :, :] - camtoworlds[:, None, :3, 3]
            colors = spherical_harmonics_shared(sh_degree, dirs, colors, masks=radii > 0)  # [C, N, 3]
        colors = torch.clamp_min(colors + 0.5, 0.0)
    elif colors.dim() == 2:
        colors = colors[gaussian_ids] if packed else colors.expand(C, *([-1] * colors.dim()))
    elif packed:
        colors = colors[camera_ids, gaussian_ids, :]

    if render_mode in ["RGB+D", "RGB+ED"]:
        colors = torch.cat((colors, depths[..., None]), dim=-1)
    elif render_mode in ["D", "ED"]:
        colors = depths[..., None]

    return dict(C=C, radii=radii, means2d=means2d, depths=depths, ray_transforms=ray_transforms, normals=normals,
                opacities=opacities, colors=colors, densify=densify, tile_width=tile_width, tile_height=tile_height,
                tiles_per_gauss=tiles_per_gauss, isect_ids=isect_ids, flatten_ids=flatten_ids,
                isect_offsets=isect_offsets, camera_ids=camera_ids, gaussian_ids=gaussian_ids, tile_order=order)


def _finish(p, render_colors, render_alphas, render_normals, render_distort, render_median, gs_contrib_sum,
            gs_contrib_count, viewmats, Ks, width, height, tile_size, render_mode, depth_mode):
    render_normals_from_depth = None
    if render_mode in ["ED", "RGB+ED"]:
        render_colors = torch.cat(
            [render_colors[..., :-1], render_colors[..., -1:] / render_alphas.clamp(min=1e-10)], dim=-1)
    if render_mode in ["RGB+ED", "RGB+D"]:
        depth_for_normal = render_colors[..., -1:] if depth_mode == "expected" else render_median
        render_normals_from_depth = depth_to_normal(depth_for_normal, _inverse(viewmats), Ks).squeeze(0)
    meta = {
        "camera_ids": p["camera_ids"],
        "gaussian_ids": p["gaussian_ids"],
        "radii": p["radii"],
        "means2d": p["means2d"],
        "depths": p["depths"],
        "ray_transforms": p["ray_transforms"],
        "opacities": p["opacities"],
        "normals": p["normals"],
        "tile_width": p["tile_width"],
        "tile_height": p["tile_height"],
        "tiles_per_gauss": p["tiles_per_gauss"],
        "isect_ids": p["isect_ids"],
        "flatten_ids": p["flatten_ids"],
        "isect_offsets": p["isect_offsets"],
        "width": width,
        "height": height,
        "tile_size": tile_size,
        "n_cameras": p["C"],
        "render_distort": render_distort,
        "gradient_2dgs": p["densify"],
    }
    render_normals = torch.einsum("...ij,...hwj->...hwi", _inverse(viewmats)[..., :3, :3], render_normals)
    return (render_colors, render_alphas, render_normals, render_normals_from_depth, render_distort, render_median,
            gs_contrib_sum, gs_contrib_count, meta)


def rasterization_2dgs(
    means: Tensor,
    quats: Tensor,
    scales: Tensor,
    opacities: Tensor,
    colors: Tensor,
    viewmats: Tensor,
    Ks: Tensor,
    width: int,
    height: int,
    near_plane: float = 0.01,
    far_plane: float = 1e10,
    radius_clip: float = 0.0,
    eps2d: float = 0.3,
    sh_degree: Optional[int] = None,
    packed: bool = False,
    tile_size: int = 16,
    backgrounds: Optional[Tensor] = None,
    render_mode: str = "RGB",
    sparse_grad: bool = False,
    absgrad: bool = False,
    distloss: bool = False,
    norm_rot_grad: bool = False,
    depth_mode: str = "expected",
    gs_contrib_threshold: float = 0.0,
    *,
    adjoint: str = "reference",
    tile_order: str = "heaviest_first",
    batch_depth: int = 0,
    persistent: bool = False,
    fuse_sh: bool = True,
) -> Tuple[Tensor, Tensor, Tensor, Optional[Tensor], Tensor, Tensor, Tensor, Tensor, Dict]:
    """Rasterize 2D Gaussian surfels (N) to C image planes (reference: rendering.py:1009-1338).

    Returns ``(render_colors, render_alphas, render_normals,
    render_normals_from_depth, render_distort, render_median, gs_contrib_sum,
    gs_contrib_count, meta)``.
    """
    p = _prepare(means, quats, scales, opacities, colors, viewmats, Ks, width, height, near_plane, far_plane,
                 radius_clip, eps2d, sh_degree, packed, tile_size, render_mode, sparse_grad, norm_rot_grad, distloss,
                 adjoint, tile_order, fuse_sh)
    outs = rasterize_to_pixels_2dgs(
        p["means2d"], p["ray_transforms"], p["colors"], p["opacities"], p["normals"], p["densify"], width, height,
        tile_size, p["isect_offsets"], p["flatten_ids"], backgrounds=backgrounds, packed=packed, absgrad=absgrad,
        distloss=distloss, gs_contrib_threshold=gs_contrib_threshold, gaussian_ids=p["gaussian_ids"],
        n_gaussians=means.shape[0] if packed else None, tile_order=p["tile_order"], batch_depth=batch_depth,
        persistent=persistent)
    return _finish(p, *outs, viewmats, Ks, width, height, tile_size, render_mode, depth_mode)


def rasterization_textured_gaussians(
    means: Tensor,
    quats: Tensor,
    scales: Tensor,
    opacities: Tensor,
    colors: Tensor,
    textures: Tensor,
    viewmats: Tensor,
    Ks: Tensor,
    width: int,
    height: int,
    texture_range_x: float = 3.0,
    texture_range_y: float = 3.0,
    near_plane: float = 0.01,
    far_plane: float = 1e10,
    radius_clip: float = 0.0,
    eps2d: float = 0.3,
    sh_degree: Optional[int] = None,
    packed: bool = False,
    tile_size: int = 16,
    backgrounds: Optional[Tensor] = None,
    render_mode: str = "RGB",
    sparse_grad: bool = False,
    absgrad: bool = False,
    distloss: bool = False,
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
    batch_depth: int = 0,
    persistent: bool = False,
    fuse_sh: bool = True,
    transmittance: str = "divide",
) -> Tuple[Tensor, Tensor, Tensor, Optional[Tensor], Tensor, Tensor, Tensor, Tensor, Dict]:
    """Rasterize textured 2D Gaussian surfels (reference: rendering.py:1342-1685).

    ``textures`` is [N, th, tw, 4] RGBA per Gaussian, sampled bilinearly over
    the splat's [-texture_range, texture_range]^2 UV square.  Returns the same
    9-tuple as :func:`rasterization_2dgs`.
    """
    N = means.shape[0]
    assert textures.shape[0] == N and textures.shape[-1] == 4 and textures.dim() == 4, textures.shape
    p = _prepare(means, quats, scales, opacities, colors, viewmats, Ks, width, height, near_plane, far_plane,
                 radius_clip, eps2d, sh_degree, packed, tile_size, render_mode, sparse_grad, norm_rot_grad, distloss,
                 adjoint, tile_order, fuse_sh)
    outs = rasterize_to_pixels_textured_gaussians(
        p["means2d"], p["ray_transforms"], p["colors"], p["opacities"], textures, texture_range_x, texture_range_y,
        p["normals"], p["densify"], width, height, tile_size, p["isect_offsets"], p["flatten_ids"],
        backgrounds=backgrounds, packed=packed, absgrad=absgrad, distloss=distloss,
        gs_contrib_threshold=gs_contrib_threshold, filtering=filtering, g_weight=g_weight,
        texture_storage=texture_storage, texture_scales=texture_scales, gaussian_ids=p["gaussian_ids"],
        tile_order=p["tile_order"], batch_depth=batch_depth,
        persistent=persistent, transmittance=transmittance)
    return _finish(p, *outs, viewmats, Ks, width, height, tile_size, render_mode, depth_mode)
