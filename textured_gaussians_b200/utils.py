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
    """Depth maps [..., H, W, 1] -> world points [..., H, W, 3] (pixel centres back-projected through Ks)."""
    if depths.shape[-1] != 1:
        raise AssertionError(f"depth maps need a trailing channel of 1, got {tuple(depths.shape)}")
    if camtoworlds.shape[-2:] != (4, 4):
        raise AssertionError(f"camera-to-world matrices must be 4x4, got {tuple(camtoworlds.shape)}")
    if Ks.shape[-2:] != (3, 3):
        raise AssertionError(f"intrinsics must be 3x3, got {tuple(Ks.shape)}")
    lead = depths.shape[:-3]
    if not (lead == camtoworlds.shape[:-2] == Ks.shape[:-2]):
        raise AssertionError(f"batch shapes differ: depths {tuple(depths.shape)}, cameras {tuple(camtoworlds.shape)}, "
                             f"intrinsics {tuple(Ks.shape)}")
    dev = depths.device
    rows, cols = depths.shape[-3:-1]
    u, v = torch.meshgrid(torch.arange(cols, device=dev), torch.arange(rows, device=dev), indexing="xy")
    f_u, f_v = Ks[..., 0, 0, None, None], Ks[..., 1, 1, None, None]
    c_u, c_v = Ks[..., 0, 2, None, None], Ks[..., 1, 2, None, None]
    rays = torch.stack([(u - c_u + 0.5) / f_u, (v - c_v + 0.5) / f_v, torch.ones_like(f_u * u)], dim=-1)
    rays = torch.einsum("...ij,...hwj->...hwi", camtoworlds[..., :3, :3], rays)
    if not z_depth:  # depth along the ray rather than along the optical axis
        rays = F.normalize(rays, dim=-1)
    centre = camtoworlds[..., :3, 3]
    return centre[..., None, None, :] + depths * rays


def depth_to_normal(depths: Tensor, camtoworlds: Tensor, Ks: Tensor, z_depth: bool = True) -> Tensor:
    """Depth maps [..., H, W, 1] -> world-space surface normals [..., H, W, 3]: the normalised cross product
    of central differences of the back-projected points, zero on the one-pixel border."""
    pts = depth_to_points(depths, camtoworlds, Ks, z_depth=z_depth)
    d_rows = pts[..., 2:, 1:-1, :] - pts[..., :-2, 1:-1, :]
    d_cols = pts[..., 1:-1, 2:, :] - pts[..., 1:-1, :-2, :]
    n = F.normalize(torch.cross(d_rows, d_cols, dim=-1), dim=-1)
    return F.pad(n, (0, 0, 1, 1, 1, 1), value=0.0)
