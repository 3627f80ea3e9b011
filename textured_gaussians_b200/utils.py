"""Depth-to-normal helpers used by the renderer's RGB+D / RGB+ED modes.

Behaviour of textured_gaussians/utils.py:81-168 (depth_to_points,
depth_to_normal): back-project a z-depth map through the pinhole intrinsics,
then take the normalised cross product of central differences, zero-padded at
the border.  Plain torch on the GPU tensors (post-processing glue).
"""
from __future__ import annotations

import torch
import torch.nn.functional as F
from torch import Tensor


def depth_to_points(depths: Tensor, camtoworlds: Tensor, Ks: Tensor, z_depth: bool = True) -> Tensor:
    """Depth maps [..., H, W, 1] -> world points [..., H, W, 3]."""
    assert depths.shape[-1] == 1, f"Invalid depth shape: {depths.shape}"
    assert camtoworlds.shape[-2:] == (4, 4), f"Invalid viewmats shape: {camtoworlds.shape}"
    assert Ks.shape[-2:] == (3, 3), f"Invalid Ks shape: {Ks.shape}"
    assert depths.shape[:-3] == camtoworlds.shape[:-2] == Ks.shape[:-2], (depths.shape, camtoworlds.shape, Ks.shape)
    device = depths.device
    height, width = depths.shape[-3:-1]
    x, y = torch.meshgrid(torch.arange(width, device=device), torch.arange(height, device=device), indexing="xy")
    fx, fy = Ks[..., 0, 0], Ks[..., 1, 1]
    cx, cy = Ks[..., 0, 2], Ks[..., 1, 2]
    dirs = torch.stack(
        [(x - cx[..., None, None] + 0.5) / fx[..., None, None], (y - cy[..., None, None] + 0.5) / fy[..., None, None]],
        dim=-1)
    dirs = F.pad(dirs, (0, 1), value=1.0)  # [..., H, W, 3]
    dirs = torch.einsum("...ij,...hwj->...hwi", camtoworlds[..., :3, :3], dirs)
    if not z_depth:
        dirs = F.normalize(dirs, dim=-1)
    origins = camtoworlds[..., :3, -1]
    return origins[..., None, None, :] + depths * dirs


def depth_to_normal(depths: Tensor, camtoworlds: Tensor, Ks: Tensor, z_depth: bool = True) -> Tensor:
    """Depth maps [..., H, W, 1] -> world-space surface normals [..., H, W, 3]."""
    points = depth_to_points(depths, camtoworlds, Ks, z_depth=z_depth)
    dx = points[..., 2:, 1:-1, :] - points[..., :-2, 1:-1, :]
    dy = points[..., 1:-1, 2:, :] - points[..., 1:-1, :-2, :]
    normals = F.normalize(torch.cross(dx, dy, dim=-1), dim=-1)
    return F.pad(normals, (0, 0, 1, 1, 1, 1), value=0.0)
