"""Drop-in op surface of the textured 2DGS path, backed by libtg2dgs.so.

Names, signatures, return tuples, dtypes and layouts follow the reference's
``textured_gaussians/cuda/_wrapper.py``:

=================================================  ====================================
this module                                        reference (textured_gaussians/...)
=================================================  ====================================
``spherical_harmonics``                            cuda/_wrapper.py:54-80, 1233-1263
``fully_fused_projection_2dgs``                    cuda/_wrapper.py:1267-1371, 1374-1484
``isect_tiles``                                    cuda/_wrapper.py:349-420
``isect_offset_encode``                            cuda/_wrapper.py:423-440
``rasterize_to_pixels_2dgs``                       cuda/_wrapper.py:1647-1784, 2767-2944
``rasterize_to_pixels_textured_gaussians``         cuda/_wrapper.py:1806-2002, 2947-3155
=================================================  ====================================

Every op runs hand-written sm_100a kernels through the C ABI; none has a CPU
path.  Additions beyond the reference are keyword-only and default off:
``filtering="bilinear_exact"`` (exact adjoint), ``texture_storage`` /
``texture_scales`` (BF16 / FP16 / FP8-E4M3 texture sampling with FP32
gradients), and ``adjoint="exact"`` on the projection.
"""
from __future__ import annotations

import ctypes
import math
from typing import Optional, Tuple

import torch
from torch import Tensor

from .. import _backend as B
from ..graph import active_plan

_FILTER_ADJOINT = {
    "bilinear": B.TG_ADJ_REFERENCE,
    "bilinear_bwd2": B.TG_ADJ_BWD2,
    "bilinear_exact": B.TG_ADJ_EXACT,
    "mipmapped2": B.TG_ADJ_REFERENCE,
    "anisotropic_bilinear": B.TG_ADJ_REFERENCE,
}
_MIP_FILTERS = ("mipmapped2",)
_FILTER_CODE = {"mipmapped2": B.TG_FILTER_MIPMAPPED2, "anisotropic_bilinear": B.TG_FILTER_ANISO_BILINEAR}


def _bit_width(n: int) -> int:
    return int(n).bit_length()


# --------------------------------------------------------------------------- SH
def spherical_harmonics(degrees_to_use: int, dirs: Tensor, coeffs: Tensor, masks: Optional[Tensor] = None) -> Tensor:
    """Computes spherical harmonics (reference: cuda/_wrapper.py:54-80).

    Args:
        degrees_to_use: The degree to be used.
        dirs: Directions. [..., 3]
        coeffs: Coefficients. [..., K, 3]
        masks: Optional boolean masks to skip some computation. [...,]

    Returns:
        Spherical harmonics. [..., 3]
    """
    assert (degrees_to_use + 1) ** 2 <= coeffs.shape[-2], coeffs.shape
    assert dirs.shape[:-1] == coeffs.shape[:-2], (dirs.shape, coeffs.shape)
    assert dirs.shape[-1] == 3, dirs.shape
    assert coeffs.shape[-1] == 3, coeffs.shape
    if masks is not None:
        assert masks.shape == dirs.shape[:-1], masks.shape
        masks = masks.contiguous()
    return _SphericalHarmonics.apply(degrees_to_use, dirs.contiguous(), coeffs.contiguous(), masks, 1)


def spherical_harmonics_shared(degrees_to_use: int, dirs: Tensor, coeffs: Tensor,
                               masks: Optional[Tensor] = None) -> Tensor:
    """SH colours for C cameras sharing one coefficient table.

    dirs [C, N, 3], coeffs [N, K, 3] -> colours [C, N, 3]; the same values as
    ``spherical_harmonics(d, dirs, coeffs.expand(C, ...), masks)`` without
    materialising C copies of the coefficients.
    """
    C = dirs.shape[0]
    assert dirs.dim() == 3 and coeffs.dim() == 3 and dirs.shape[1] == coeffs.shape[0], (dirs.shape, coeffs.shape)
    assert (degrees_to_use + 1) ** 2 <= coeffs.shape[-2], coeffs.shape
    if masks is not None:
        masks = masks.contiguous()
    return _SphericalHarmonics.apply(degrees_to_use, dirs.contiguous(), coeffs.contiguous(), masks, C)


class _SphericalHarmonics(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sh_degree: int, dirs: Tensor, coeffs: Tensor, masks: Optional[Tensor], share: int) -> Tensor:
        dirs_f = dirs.float().contiguous()
        coeffs_f = coeffs.float().contiguous()
        n = dirs_f.numel() // 3
        K = coeffs_f.shape[-2]
        rows = coeffs_f.numel() // (3 * K) if coeffs_f.numel() else 0
        colors = torch.empty(dirs_f.shape, dtype=torch.float32, device=dirs.device)
        m = None if masks is None else masks.to(torch.uint8).contiguous()
        if n:
            st = B.stream_of(dirs)
            B.call("tg_sh_fwd", st, B.lib().tg_sh_fwd, n, rows, sh_degree, K, B.ptr(dirs_f), B.ptr(coeffs_f), B.ptr(m),
                   B.ptr(colors), st)
        ctx.save_for_backward(dirs_f, coeffs_f, m)
        ctx.sh_degree = sh_degree
        ctx.share = share
        return colors

    @staticmethod
    def backward(ctx, v_colors: Tensor):
        dirs, coeffs, m = ctx.saved_tensors
        n = dirs.numel() // 3
        K = coeffs.shape[-2]
        rows = coeffs.numel() // (3 * K) if coeffs.numel() else 0
        compute_v_dirs = ctx.needs_input_grad[1]
        v_coeffs = torch.empty_like(coeffs)
        v_dirs = torch.empty_like(dirs) if compute_v_dirs else None
        vc = v_colors.float().contiguous()
        if n:
            st = B.stream_of(dirs)
            B.call("tg_sh_bwd", st, B.lib().tg_sh_bwd, n, rows, ctx.sh_degree, K, B.ptr(dirs), B.ptr(coeffs), B.ptr(m),
                   B.ptr(vc), B.ptr(v_coeffs), B.ptr(v_dirs), st)
        else:
            v_coeffs.zero_()
        return None, v_dirs, v_coeffs, None, None


# --------------------------------------------------------------------------- projection
def fully_fused_projection_2dgs(
    means: Tensor,
    quats: Tensor,
    scales: Tensor,
    viewmats: Tensor,
    Ks: Tensor,
    width: int,
    height: int,
    eps2d: float = 0.3,
    near_plane: float = 0.01,
    far_plane: float = 1e10,
    radius_clip: float = 0.0,
    packed: bool = False,
    sparse_grad: bool = False,
    norm_rot_grad: bool = False,
    *,
    adjoint: str = "reference",
    sh_coeffs: Optional[Tensor] = None,
    sh_degree: Optional[int] = None,
) -> Tuple[Tensor, ...]:
    """Ray-splat transforms, 2D means, depths, screen radii and normals
    (reference: cuda/_wrapper.py:1267-1371).

    Returns ``(radii, means2d, depths, ray_transforms, normals)`` for the dense
    layout and ``(camera_ids, gaussian_ids, radii, means2d, depths,
    ray_transforms, normals)`` for the packed one (visible entries only,
    ordered by camera then Gaussian; reference: cuda/_wrapper.py:1487-1644).
    With ``sparse_grad`` the packed backward returns the gradients of means,
    quats and scales as sparse COO tensors with one row per entry.
    ``adjoint="exact"`` selects the exact derivative of means2d with respect
    to the ray transform in the backward (the reference keeps only its
    diagonal terms).

    ``sh_coeffs`` [N,K,3] with ``sh_degree`` fuses the renderer's SH colour
    step into the projection (reference glue: rendering.py:1573-1583): one
    more output, the colours ``max(SH(degree, mean - camera centre) + 0.5, 0)``
    per visible entry ([C,N,3] or [nnz,3]; 0.5 for culled entries), whose
    adjoint reaches ``sh_coeffs`` and ``means``.
    """
    C = viewmats.size(0)
    N = means.size(0)
    assert means.size() == (N, 3), means.size()
    assert viewmats.size() == (C, 4, 4), viewmats.size()
    assert Ks.size() == (C, 3, 3), Ks.size()
    assert quats is not None, "quats is required"
    assert scales is not None, "scales is required"
    assert quats.size() == (N, 4), quats.size()
    assert scales.size() == (N, 3), scales.size()
    if sparse_grad:
        assert packed, "sparse_grad is only supported when packed is True"
    mode = B.TG_ADJ_EXACT if adjoint == "exact" else (B.TG_ADJ_BWD2 if norm_rot_grad else B.TG_ADJ_REFERENCE)
    if sh_coeffs is not None:
        assert sh_degree is not None and sh_coeffs.dim() == 3 and sh_coeffs.shape[0] == N, sh_coeffs.shape
        assert sh_coeffs.shape[2] == 3 and (sh_degree + 1) ** 2 <= sh_coeffs.shape[1] <= 25, sh_coeffs.shape
        sh_coeffs = sh_coeffs.float().contiguous()
    sh = (sh_coeffs, int(sh_degree or 0))
    if packed:
        return _FullyFusedProjectionPacked2DGS.apply(
            means.contiguous(), quats.contiguous(), scales.contiguous(), viewmats.contiguous(), Ks.contiguous(),
            width, height, eps2d, near_plane, far_plane, radius_clip, sparse_grad, mode, None, *sh)
    return _FullyFusedProjection2DGS.apply(
        means.contiguous(), quats.contiguous(), scales.contiguous(), viewmats.contiguous(), Ks.contiguous(),
        width, height, eps2d, near_plane, far_plane, radius_clip, mode, *sh)


class _FullyFusedProjection2DGS(torch.autograd.Function):
    """Projects Gaussians to 2D (reference: cuda/_wrapper.py:1374-1484)."""

    @staticmethod
    def forward(ctx, means, quats, scales, viewmats, Ks, width, height, eps2d, near_plane, far_plane, radius_clip,
                mode, sh_coeffs=None, sh_degree=0):
        C, N = viewmats.shape[0], means.shape[0]
        dev = means.device
        radii = torch.empty((C, N), dtype=torch.int32, device=dev)
        means2d = torch.empty((C, N, 2), dtype=torch.float32, device=dev)
        depths = torch.empty((C, N), dtype=torch.float32, device=dev)
        ray_transforms = torch.empty((C, N, 3, 3), dtype=torch.float32, device=dev)
        normals = torch.empty((C, N, 3), dtype=torch.float32, device=dev)
        a = B.ProjectFwdArgs(C, N, B.ptr(means), B.ptr(quats), B.ptr(scales), B.ptr(viewmats), B.ptr(Ks),
                             int(width), int(height), float(near_plane), float(far_plane), float(radius_clip),
                             B.ptr(radii), B.ptr(means2d), B.ptr(depths), B.ptr(ray_transforms), B.ptr(normals))
        colors = None
        if sh_coeffs is not None:
            colors = torch.empty((C, N, 3), dtype=torch.float32, device=dev)
            a.sh_degree, a.sh_K, a.sh_coeffs, a.colors = sh_degree, sh_coeffs.shape[1], B.ptr(sh_coeffs), B.ptr(colors)
        if C * N:
            st = B.stream_of(means)
            B.call("tg_project_fwd", st, B.lib().tg_project_fwd, ctypes.byref(a), st)
        ctx.save_for_backward(means, quats, scales, viewmats, Ks, radii, ray_transforms, sh_coeffs)
        ctx.mode = mode
        ctx.sh_degree = sh_degree
        ctx.mark_non_differentiable(radii)
        if colors is not None:
            return radii, means2d, depths, ray_transforms, normals, colors
        return radii, means2d, depths, ray_transforms, normals

    @staticmethod
    def backward(ctx, v_radii, v_means2d, v_depths, v_ray_transforms, v_normals, v_colors=None):
        means, quats, scales, viewmats, Ks, radii, ray_transforms, sh_coeffs = ctx.saved_tensors
        C, N = viewmats.shape[0], means.shape[0]

        def z(t, shape):
            return torch.zeros(shape, dtype=torch.float32, device=means.device) if t is None else t.float().contiguous()

        v_means2d = z(v_means2d, (C, N, 2))
        v_depths = z(v_depths, (C, N))
        v_ray_transforms = z(v_ray_transforms, (C, N, 3, 3))
        v_normals = z(v_normals, (C, N, 3))
        v_means = torch.empty_like(means)
        v_quats = torch.empty_like(quats)
        v_scales = torch.empty_like(scales)
        a = B.ProjectBwdArgs(C, N, B.ptr(means), B.ptr(quats), B.ptr(scales), B.ptr(viewmats), B.ptr(Ks),
                             B.ptr(radii), B.ptr(ray_transforms), B.ptr(v_means2d), B.ptr(v_depths),
                             B.ptr(v_normals), B.ptr(v_ray_transforms), ctx.mode, B.ptr(v_means), B.ptr(v_quats),
                             B.ptr(v_scales))
        v_sh = None
        if sh_coeffs is not None:
            v_col = z(v_colors, (C, N, 3))
            v_sh = torch.empty_like(sh_coeffs)
            a.sh_degree, a.sh_K, a.sh_coeffs = ctx.sh_degree, sh_coeffs.shape[1], B.ptr(sh_coeffs)
            a.v_colors, a.v_sh_coeffs = B.ptr(v_col), B.ptr(v_sh)
        if N:
            st = B.stream_of(means)
            B.call("tg_project_bwd", st, B.lib().tg_project_bwd, ctypes.byref(a), st)
        v_viewmats = torch.zeros_like(viewmats) if ctx.needs_input_grad[3] else None  # never written (reference)
        return (v_means if ctx.needs_input_grad[0] else None, v_quats if ctx.needs_input_grad[1] else None,
                v_scales if ctx.needs_input_grad[2] else None, v_viewmats,
                None, None, None, None, None, None, None, None, v_sh, None)


class _FullyFusedProjectionPacked2DGS(torch.autograd.Function):
    """Packed projection (reference: cuda/_wrapper.py:1487-1644).

    Two passes split at one host read of nnz, as in the reference.  Every
    camera uses its own intrinsics (the reference's packed forward reads
    Ks[0] for all cameras).
    """

    @staticmethod
    def forward(ctx, means, quats, scales, viewmats, Ks, width, height, eps2d, near_plane, far_plane, radius_clip,
                sparse_grad, mode, batch, sh_coeffs=None, sh_degree=0):
        C, N = viewmats.shape[0], means.shape[0]
        dev = means.device
        ws = torch.empty((B.lib().tg_project_packed_workspace_bytes(C, N),), dtype=torch.uint8, device=dev)
        nnz_dev = torch.empty((1,), dtype=torch.int64, device=dev)
        indptr = torch.empty((C + 1,), dtype=torch.int32, device=dev)
        a = B.ProjectPackedArgs(C, N, B.ptr(means), B.ptr(quats), B.ptr(scales), B.ptr(viewmats), B.ptr(Ks),
                                int(width), int(height), float(near_plane), float(far_plane), float(radius_clip),
                                B.ptr(ws), B.ptr(nnz_dev), B.ptr(indptr), 0)
        if batch is not None:  # (view table bytes, [C,2] Gaussian ranges, longest range)
            a.views, a.gauss_ranges, a.max_range = B.ptr(batch[0]), B.ptr(batch[1]), int(batch[2])
        st = B.stream_of(means)
        B.call("tg_project_packed_count", st, B.lib().tg_project_packed_count, ctypes.byref(a), st)
        plan = active_plan()
        if plan is not None and plan.mode == "capture":  # no host read: capacity-sized outputs, overflow flag
            nnz = plan.next_capacity()
            a.overflow = B.ptr(plan.new_flag(dev))
        else:
            nnz = int(nnz_dev.item())  # the one host synchronisation, as in the reference
            if plan is not None:
                plan.sizes.append(nnz)
        camera_ids = torch.empty((nnz,), dtype=torch.int64, device=dev)
        gaussian_ids = torch.empty((nnz,), dtype=torch.int64, device=dev)
        radii = torch.empty((nnz,), dtype=torch.int32, device=dev)
        means2d = torch.empty((nnz, 2), dtype=torch.float32, device=dev)
        depths = torch.empty((nnz,), dtype=torch.float32, device=dev)
        ray_transforms = torch.empty((nnz, 3, 3), dtype=torch.float32, device=dev)
        normals = torch.empty((nnz, 3), dtype=torch.float32, device=dev)
        a.nnz_host = nnz
        a.camera_ids, a.gaussian_ids, a.radii = B.ptr(camera_ids), B.ptr(gaussian_ids), B.ptr(radii)
        a.means2d, a.depths, a.ray_transforms, a.normals = (B.ptr(means2d), B.ptr(depths), B.ptr(ray_transforms),
                                                            B.ptr(normals))
        colors = None
        if sh_coeffs is not None:
            colors = torch.empty((nnz, 3), dtype=torch.float32, device=dev)
            a.sh_degree, a.sh_K, a.sh_coeffs, a.colors = sh_degree, sh_coeffs.shape[1], B.ptr(sh_coeffs), B.ptr(colors)
        B.call("tg_project_packed_emit", st, B.lib().tg_project_packed_emit, ctypes.byref(a), st)
        ctx.save_for_backward(camera_ids, gaussian_ids, means, quats, scales, viewmats, Ks, ray_transforms, sh_coeffs)
        ctx.sparse_grad = bool(sparse_grad)
        ctx.mode = mode
        ctx.sh_degree = sh_degree
        ctx.mark_non_differentiable(camera_ids, gaussian_ids, radii)
        if colors is not None:
            return camera_ids, gaussian_ids, radii, means2d, depths, ray_transforms, normals, colors
        return camera_ids, gaussian_ids, radii, means2d, depths, ray_transforms, normals

    @staticmethod
    def backward(ctx, v_camera_ids, v_gaussian_ids, v_radii, v_means2d, v_depths, v_ray_transforms, v_normals,
                 v_colors=None):
        camera_ids, gaussian_ids, means, quats, scales, viewmats, Ks, ray_transforms, sh_coeffs = ctx.saved_tensors
        C, N, nnz = viewmats.shape[0], means.shape[0], camera_ids.shape[0]
        dev = means.device

        def z(t, shape):
            return torch.zeros(shape, dtype=torch.float32, device=dev) if t is None else t.float().contiguous()

        v_means2d = z(v_means2d, (nnz, 2))
        v_depths = z(v_depths, (nnz,))
        v_ray_transforms = z(v_ray_transforms, (nnz, 3, 3))
        v_normals = z(v_normals, (nnz, 3))
        rows = nnz if ctx.sparse_grad else N
        v_means = torch.empty((rows, 3), dtype=torch.float32, device=dev)
        v_quats = torch.empty((rows, 4), dtype=torch.float32, device=dev)
        v_scales = torch.empty((rows, 3), dtype=torch.float32, device=dev)
        a = B.ProjectPackedBwdArgs(C, N, nnz, B.ptr(means), B.ptr(quats), B.ptr(scales), B.ptr(viewmats), B.ptr(Ks),
                                   B.ptr(camera_ids), B.ptr(gaussian_ids), B.ptr(ray_transforms), B.ptr(v_means2d),
                                   B.ptr(v_depths), B.ptr(v_normals), B.ptr(v_ray_transforms), ctx.mode,
                                   int(ctx.sparse_grad), B.ptr(v_means), B.ptr(v_quats), B.ptr(v_scales))
        v_sh = None
        if sh_coeffs is not None:
            v_col = z(v_colors, (nnz, 3))
            v_sh = torch.empty_like(sh_coeffs)
            a.sh_degree, a.sh_K, a.sh_coeffs = ctx.sh_degree, sh_coeffs.shape[1], B.ptr(sh_coeffs)
            a.v_colors, a.v_sh_coeffs = B.ptr(v_col), B.ptr(v_sh)
        st = B.stream_of(means)
        B.call("tg_project_packed_bwd", st, B.lib().tg_project_packed_bwd, ctypes.byref(a), st)

        def out(v, like, need):
            if not need:
                return None
            if ctx.sparse_grad:
                return torch.sparse_coo_tensor(indices=gaussian_ids[None], values=v, size=like.size(),
                                               is_coalesced=len(viewmats) == 1)
            return v

        # the reference gates the (never written, zero) viewmats gradient on the Ks input (index 4)
        v_viewmats = torch.zeros_like(viewmats) if ctx.needs_input_grad[4] else None
        return (out(v_means, means, ctx.needs_input_grad[0]), out(v_quats, quats, ctx.needs_input_grad[1]),
                out(v_scales, scales, ctx.needs_input_grad[2]), v_viewmats,
                None, None, None, None, None, None, None, None, None, None, v_sh, None)


# --------------------------------------------------------------------------- intersection
@torch.no_grad()
def isect_tiles(
    means2d: Tensor,
    radii: Tensor,
    depths: Tensor,
    tile_size: int,
    tile_width: int,
    tile_height: int,
    sort: bool = True,
    packed: bool = False,
    n_cameras: Optional[int] = None,
    camera_ids: Optional[Tensor] = None,
    gaussian_ids: Optional[Tensor] = None,
    *,
    view_table=None,
) -> Tuple[Tensor, Tensor, Tensor]:
    """Maps projected Gaussians to intersecting tiles (reference: cuda/_wrapper.py:349-420).

    Returns ``(tiles_per_gauss int32 [C,N] or [nnz], isect_ids int64 [n_isects],
    flatten_ids int32 [n_isects])``, sorted stably by isect id when ``sort``.
    ``view_table`` (batching form, :class:`textured_gaussians_b200.batch.ViewTable`)
    gives every camera its own tile grid; tile_width / tile_height are then
    ignored and the key's tile bits come from the largest grid.
    """
    if view_table is not None:
        tile_width, tile_height = view_table.key_tiles, 1
    if packed:
        nnz = means2d.size(0)
        assert means2d.shape == (nnz, 2), means2d.size()
        assert radii.shape == (nnz,), radii.size()
        assert depths.shape == (nnz,), depths.size()
        assert camera_ids is not None, "camera_ids is required if packed is True"
        assert gaussian_ids is not None, "gaussian_ids is required if packed is True"
        assert n_cameras is not None, "n_cameras is required if packed is True"
        C, N, E = n_cameras, 0, nnz
        cam = camera_ids.contiguous().long()
    else:
        C, N, _ = means2d.shape
        assert means2d.shape == (C, N, 2), means2d.size()
        assert radii.shape == (C, N), radii.size()
        assert depths.shape == (C, N), depths.size()
        E = C * N
        cam = None
    dev = means2d.device
    means2d = means2d.float().contiguous()
    radii = radii.int().contiguous()
    depths = depths.float().contiguous()
    tiles_per_gauss = torch.empty(radii.shape, dtype=torch.int32, device=dev)
    cum = torch.empty((max(E, 1),), dtype=torch.int64, device=dev)
    n_dev = torch.empty((1,), dtype=torch.int64, device=dev)
    ws = torch.empty((B.lib().tg_scan_workspace_bytes(E),), dtype=torch.uint8, device=dev)
    a = B.IsectArgs(E, N, B.ptr(cam), B.ptr(means2d), B.ptr(radii), B.ptr(depths), int(tile_size), int(tile_width),
                    int(tile_height), int(C), B.ptr(tiles_per_gauss), B.ptr(cum), B.ptr(n_dev), B.ptr(ws), None, None,
                    None if view_table is None else B.ptr(view_table.views))
    stream = B.stream_of(means2d)
    B.call("tg_isect_count", stream, B.lib().tg_isect_count, ctypes.byref(a), stream)
    end_bit = 32 + _bit_width(tile_width * tile_height) + _bit_width(C)
    plan = active_plan()
    if plan is not None and plan.mode == "capture":
        # no host read: capacity-sized keys (tail padded to sort last), device count attached to flatten_ids
        cap = plan.next_capacity()
        isect_ids = torch.empty((cap,), dtype=torch.int64, device=dev)
        flatten_ids = torch.empty((cap,), dtype=torch.int32, device=dev)
        a.isect_ids, a.flatten_ids = B.ptr(isect_ids), B.ptr(flatten_ids)
        a.capacity, a.overflow = cap, B.ptr(plan.new_flag(dev))
        B.call("tg_isect_emit", stream, B.lib().tg_isect_emit, ctypes.byref(a), stream)
        if sort:
            isect_ids, flatten_ids = sort_pairs(isect_ids, flatten_ids, end_bit)
        flatten_ids._tg_n_isects = n_dev
        return tiles_per_gauss, isect_ids, flatten_ids
    n_isects = int(n_dev.item())  # the one host synchronisation, as in the reference
    if plan is not None:
        plan.sizes.append(n_isects)
    isect_ids = torch.empty((n_isects,), dtype=torch.int64, device=dev)
    flatten_ids = torch.empty((n_isects,), dtype=torch.int32, device=dev)
    if n_isects:
        a.isect_ids = B.ptr(isect_ids)
        a.flatten_ids = B.ptr(flatten_ids)
        B.call("tg_isect_emit", stream, B.lib().tg_isect_emit, ctypes.byref(a), stream)
        if sort:
            isect_ids, flatten_ids = sort_pairs(isect_ids, flatten_ids, end_bit)
    return tiles_per_gauss, isect_ids, flatten_ids


def n_isects_of(flatten_ids: Tensor):
    """Valid intersection count: a device tensor [1] for capacity-sized
    intersections (graph capture), else the length of ``flatten_ids``."""
    return getattr(flatten_ids, "_tg_n_isects", flatten_ids.numel())


def sort_pairs(keys: Tensor, vals: Tensor, end_bit: int, check: bool = False) -> Tuple[Tensor, Tensor]:
    """Stable radix sort of (int64 key, int32 value) pairs on key bits [0, end_bit).

    ``check=True`` waits for the sort and raises if one of its bounded
    look-back waits gave up (``tg_sort_status``)."""
    n = keys.numel()
    if n <= 1:
        return keys, vals
    keys_alt = torch.empty_like(keys)
    vals_alt = torch.empty_like(vals)
    wsb = B.lib().tg_sort_workspace_bytes(n, end_bit)
    ws = torch.empty((wsb,), dtype=torch.uint8, device=keys.device)
    in_alt = ctypes.c_int32(0)
    st = B.stream_of(keys)
    B.call("tg_sort_pairs", st, B.lib().tg_sort_pairs, B.ptr(keys), B.ptr(vals), B.ptr(keys_alt), B.ptr(vals_alt), n,
           end_bit, B.ptr(ws), wsb, ctypes.byref(in_alt), st)
    if check:
        B.check(B.lib().tg_sort_status(B.ptr(ws), n, end_bit, st), "tg_sort_status")
    return (keys_alt, vals_alt) if in_alt.value else (keys, vals)


@torch.no_grad()
def isect_offset_encode(isect_ids: Tensor, n_cameras: int, tile_width: int, tile_height: int) -> Tensor:
    """Encodes intersection ids to offsets (reference: cuda/_wrapper.py:423-440). [C, tile_height, tile_width]"""
    isect_ids = isect_ids.contiguous()
    offsets = torch.empty((n_cameras, tile_height, tile_width), dtype=torch.int32, device=isect_ids.device)
    st = B.stream_of(isect_ids)
    B.call("tg_isect_offset_encode", st, B.lib().tg_isect_offset_encode, B.ptr(isect_ids), isect_ids.numel(),
           int(n_cameras), int(tile_width), int(tile_height), B.ptr(offsets), st)
    return offsets


@torch.no_grad()
def isect_offset_encode_views(isect_ids: Tensor, view_table) -> Tensor:
    """Batching form of :func:`isect_offset_encode`: one offset per flat tile of
    all views ([n_tiles] int32)."""
    vt = view_table
    isect_ids = isect_ids.contiguous()
    offsets = torch.empty((vt.n_tiles,), dtype=torch.int32, device=isect_ids.device)
    st = B.stream_of(isect_ids)
    B.call("tg_isect_offset_encode_views", st, B.lib().tg_isect_offset_encode_views, B.ptr(isect_ids),
           isect_ids.numel(), vt.n_views, vt.key_tiles, B.ptr(vt.views), B.ptr(vt.tile_view), vt.n_tiles,
           B.ptr(offsets), st)
    return offsets


@torch.no_grad()
def tile_order_heaviest_first(isect_offsets: Tensor, n_isects: int) -> Tensor:
    """Permutation of the flat tiles by descending intersection count (stable),
    so the longest tiles start first and the tail of the launch is short."""
    flat = isect_offsets.reshape(-1).to(torch.int64)
    n = flat.numel()
    if isinstance(n_isects, Tensor):  # device count (graph capture)
        tail = n_isects.reshape(1).to(torch.int64)
    else:
        tail = torch.full((1,), int(n_isects), dtype=torch.int64, device=flat.device)
    counts = torch.diff(flat, append=tail)
    keys = ((1 << 31) - 1) - counts.clamp(0, (1 << 31) - 1)
    vals = torch.arange(n, dtype=torch.int32, device=flat.device)
    _, order = sort_pairs(keys.contiguous(), vals, 31)
    return order


# --------------------------------------------------------------------------- compositor
_SUPPORTED_PADDED = (1, 2, 3, 4, 8, 16, 32, 64, 128, 256, 512)


def _pad_channels(colors: Tensor, backgrounds: Optional[Tensor]):
    """Channel padding rule of the reference (cuda/_wrapper.py:1880-1899)."""
    channels = colors.shape[-1]
    if channels > 512 or channels == 0:
        raise ValueError(f"Unsupported number of color channels: {channels}")
    if channels not in _SUPPORTED_PADDED:
        padded = (1 << (channels - 1).bit_length()) - channels
        colors = torch.cat([colors, torch.zeros(*colors.shape[:-1], padded, device=colors.device)], dim=-1)
        if backgrounds is not None:
            backgrounds = torch.cat(
                [backgrounds, torch.zeros(*backgrounds.shape[:-1], padded, device=backgrounds.device)], dim=-1)
    else:
        padded = 0
    return colors, backgrounds, padded


def _tex_format(storage: Tensor) -> int:
    if storage.dtype == torch.float32:
        return B.TG_TEX_F32
    if storage.dtype == torch.bfloat16:
        return B.TG_TEX_BF16
    if storage.dtype == torch.float16:
        return B.TG_TEX_F16
    if storage.dtype == torch.float8_e4m3fn:
        return B.TG_TEX_FP8_E4M3
    raise TypeError(f"unsupported texture dtype {storage.dtype}")


def make_texture_storage(textures: Tensor, fmt: str) -> Tuple[Tensor, Optional[Tensor]]:
    """Low-precision copy of FP32 textures for sampling: "bf16", "fp16" or "fp8".

    FP8-E4M3 uses one scale per Gaussian, max|texel| / 448, returned as the
    second element (None for the 16-bit forms).
    """
    if fmt == "bf16":
        return textures.to(torch.bfloat16).contiguous(), None
    if fmt == "fp16":
        return textures.to(torch.float16).contiguous(), None
    if fmt == "fp8":
        amax = textures.detach().abs().flatten(1).amax(dim=1).clamp_min(1e-12)
        scales = (amax / 448.0).float().contiguous()
        q = (textures.detach() / scales[:, None, None, None]).to(torch.float8_e4m3fn).contiguous()
        return q, scales
    if fmt == "fp32":
        return textures.float().contiguous(), None
    raise ValueError(f"unknown texture storage format {fmt!r}")


def mip_levels_of(textures: Tensor) -> int:
    """L of square 2^L x 2^L textures [G, R, R, 4] (the mipmapped2 filter's requirement, reference
    cuda/_wrapper.py:1946-1950)."""
    R = int(textures.shape[1])
    L = R.bit_length() - 1
    if textures.dim() != 4 or textures.shape[2] != R or R != 1 << L or L < 1:
        raise ValueError(f"mipmapped2 needs square power-of-two textures of side >= 2, got {tuple(textures.shape)}")
    return L


def _coarse_pyramid(textures: Tensor, L: int) -> Tensor:
    """Levels 1..L of the textures' mip pyramid, [G, (4^L - 1) / 3, 4] FP32, coarsest first."""
    src = textures.detach().float().contiguous()
    G = src.shape[0]
    coarse = torch.empty((G, (4 ** L - 1) // 3, 4), dtype=torch.float32, device=src.device)
    st = B.stream_of(src)
    B.call("tg_generate_mipmap", st, B.lib().tg_generate_mipmap, B.ptr(src), B.ptr(coarse), G, L, st)
    return coarse


class _GenerateMipmap(torch.autograd.Function):
    """Full mip pyramid [G, (4^(L+1) - 1) / 3, 4] of 2^L textures in the reference's layout (coarse levels, then
    level 0), mirroring _GenerateMipmap (reference cuda/_wrapper.py:4015-4058)."""

    @staticmethod
    def forward(ctx, textures, L):
        G, R = textures.shape[0], textures.shape[1]
        coarse = _coarse_pyramid(textures, L)
        ctx.L, ctx.shape = L, textures.shape
        return torch.cat([coarse, textures.detach().float().reshape(G, R * R, -1)], dim=1)

    @staticmethod
    def backward(ctx, v_mip):
        L = ctx.L
        G, R = ctx.shape[0], ctx.shape[1]
        clen = (4 ** L - 1) // 3
        v_mip = v_mip.float()
        v_coarse = v_mip[:, :clen].contiguous().clone()
        v_tex = v_mip[:, clen:].reshape(G, R, R, -1).contiguous().clone()
        st = B.stream_of(v_tex)
        B.call("tg_generate_mipmap_bwd", st, B.lib().tg_generate_mipmap_bwd, B.ptr(v_coarse), B.ptr(v_tex), G, L, st)
        return v_tex, None


def generate_mipmap(textures: Tensor, log_texture_res: int, log_reduce: int = 4, tile_size: int = 16) -> Tensor:
    """Mip pyramid of 2^L textures (reference ``generate_mipmap``, cuda/_wrapper.py:4052-4058).  ``log_reduce`` and
    ``tile_size`` only set the reference's launch shape and are accepted for compatibility."""
    assert textures.shape[1] == textures.shape[2] == 1 << log_texture_res, textures.shape
    return _GenerateMipmap.apply(textures, int(log_texture_res))


# How the anisotropic_bilinear filter integrates a footprint: "boundary" (a convex footprint along its
# boundary, over row-prefix tables built per call by tg_aniso_prefix; the others cell by cell) or "cells"
# (every footprint cell by cell, as the reference does).  The same integral up to FP32 rounding.
ANISO_INTEGRATION = "boundary"
# Footprint integrals per pixel the forward keeps for the adjoint with the boundary integration (0: none;
# the adjoint then integrates every footprint again).  Each pixel's first ANISO_RECORDS are kept, within
# ANISO_RECORDS_BYTES of device memory for the call (fewer per pixel on very large calls).
ANISO_RECORDS = 32
ANISO_RECORDS_BYTES = 8 << 30
# Splats staged per compositor batch for the anisotropic_bilinear filter when the caller leaves batch_depth at
# 0: its per-pair work dwarfs the staging, and a small batch leaves more of the L1 to the boundary walk's
# texture reads (1M splats x four 1600x1200 views, tile 8: 382 ms per step at 32, 391 at 64).
ANISO_BATCH_DEPTH = 32


def _aniso_prefix(tex_store, tex_scales, st):
    """Row-prefix table [G, ry, rx, 4] FP32 of the texture storage (tg_aniso_prefix), or None."""
    if tex_store is None or ANISO_INTEGRATION == "cells":
        return None
    if ANISO_INTEGRATION != "boundary":
        raise ValueError(f"ANISO_INTEGRATION must be 'boundary' or 'cells', got {ANISO_INTEGRATION!r}")
    G, ry, rx = tex_store.shape[:3]
    prefix = torch.empty((G, ry, rx, 4), dtype=torch.float32, device=tex_store.device)
    B.call("tg_aniso_prefix", st, B.lib().tg_aniso_prefix, B.ptr(tex_store), _tex_format(tex_store),
           B.ptr(tex_scales), G, ry, rx, B.ptr(prefix), st)
    return prefix


def _fwd_args(means2d, ray_transforms, colors, opacities, normals, textures_store, tex_scales, range_x, range_y,
              backgrounds, masks, width, height, tile_size, isect_offsets, flatten_ids, gaussian_ids, n_contrib,
              gs_contrib_threshold, g_weight, C, N, layout=None, n_isects_dev=None, mip_levels=0, tex_coarse=None,
              filter_code=0):
    D = colors.shape[-1]
    vt = None if layout is None else layout.get("view_table")
    th, tw = (1, 1) if vt is not None else isect_offsets.shape[1:3]
    if vt is not None:
        width = height = 0
    if textures_store is None:
        fmt, ry, rx = B.TG_TEX_NONE, 0, 0
    else:
        fmt, ry, rx = _tex_format(textures_store), textures_store.shape[1], textures_store.shape[2]
    return B.RasterFwdArgs(
        C, N, D, int(width), int(height), int(tile_size), int(tw), int(th), flatten_ids.numel(), B.ptr(means2d),
        B.ptr(ray_transforms), B.ptr(colors), B.ptr(opacities), B.ptr(normals), fmt, B.ptr(textures_store),
        B.ptr(tex_scales), ry, rx, float(range_x), float(range_y), B.ptr(backgrounds), B.ptr(masks),
        B.ptr(isect_offsets), B.ptr(flatten_ids), B.ptr(gaussian_ids), float(gs_contrib_threshold), float(g_weight),
        int(n_contrib), None, None, None, None, None, None, None, None, None,
        None if layout is None else B.ptr(layout.get("tile_order")),
        None if vt is None else B.ptr(vt.views), None if vt is None else B.ptr(vt.tile_view),
        0 if vt is None else vt.n_tiles, 0 if vt is None else vt.n_pixels, B.ptr(n_isects_dev),
        0 if layout is None else layout.get("batch_depth", 0),
        None if layout is None else B.ptr(layout.get("work_queue")), int(mip_levels), B.ptr(tex_coarse),
        int(filter_code))


class _RasterizeToPixelsTextured(torch.autograd.Function):
    """Compositor forward/adjoint for both the textured and the plain form.

    Mirrors _RasterizeToPixelsTexturedGaussians (reference cuda/_wrapper.py:2947-3155)
    and _RasterizeToPixels2DGS (:2767-2944): saves the inputs plus the final
    colours, alphas, last and median ids -- no per-splat transmittance.
    With ``mip_levels`` L > 0 (the mipmapped2 filter, reference
    _RasterizeToPixelsMip2TexturedGaussians) the forward builds the coarse
    levels of the FP32 textures, and the backward folds their gradient into
    the texture gradient in place (no full-pyramid tensor in either pass).
    ``filter_code`` TG_FILTER_ANISO_BILINEAR selects the anisotropic_bilinear
    filter (reference _RasterizeToPixelsTexturedGaussians with the
    ``aniso_bilinear`` kernels).
    """

    @staticmethod
    def forward(ctx, means2d, ray_transforms, colors, opacities, textures, normals, densify, backgrounds, masks,
                tex_store, tex_scales, range_x, range_y, width, height, tile_size, isect_offsets, flatten_ids,
                absgrad, gs_contrib_threshold, g_weight, adjoint, bg_grad_index_ok, gaussian_ids, n_rows, layout,
                mip_levels=0, filter_code=0):
        dev = means2d.device
        coarse = _coarse_pyramid(textures, mip_levels) if mip_levels else None
        vt = None if layout is None else layout.get("view_table")
        C = isect_offsets.shape[0] if vt is None else vt.n_views
        # per-pixel output shape: [C, H, W] for one image size, [n_pixels] over the flat views
        pshape = (C, height, width) if vt is None else (vt.n_pixels,)
        # N: row modulus of the dense layout, or the packed entry count (row = entry) without gaussian_ids
        N = means2d.shape[1] if means2d.dim() == 3 else means2d.shape[0]
        n_contrib = N if gaussian_ids is None else n_rows
        D = colors.shape[-1]
        m = None if masks is None else masks.to(torch.uint8).contiguous()
        n_dev = getattr(flatten_ids, "_tg_n_isects", None)
        a = _fwd_args(means2d, ray_transforms, colors, opacities, normals, tex_store, tex_scales, range_x, range_y,
                      backgrounds, m, width, height, tile_size, isect_offsets, flatten_ids, gaussian_ids, n_contrib,
                      gs_contrib_threshold, g_weight, C, N, layout, n_dev, mip_levels, coarse, filter_code)
        render_colors = torch.empty(pshape + (D,), dtype=torch.float32, device=dev)
        render_alphas = torch.empty(pshape + (1,), dtype=torch.float32, device=dev)
        render_normals = torch.empty(pshape + (3,), dtype=torch.float32, device=dev)
        render_distort = torch.empty(pshape + (1,), dtype=torch.float32, device=dev)
        render_median = torch.empty(pshape + (1,), dtype=torch.float32, device=dev)
        last_ids = torch.empty(pshape, dtype=torch.int32, device=dev)
        median_ids = torch.empty(pshape, dtype=torch.int32, device=dev)
        contrib_sum = torch.empty((n_contrib,), dtype=torch.float32, device=dev)
        contrib_count = torch.empty((n_contrib,), dtype=torch.float32, device=dev)
        a.out_colors, a.out_alphas, a.out_normals = B.ptr(render_colors), B.ptr(render_alphas), B.ptr(render_normals)
        a.out_distort, a.out_median = B.ptr(render_distort), B.ptr(render_median)
        a.last_ids, a.median_ids = B.ptr(last_ids), B.ptr(median_ids)
        a.contrib_sum, a.contrib_count = B.ptr(contrib_sum), B.ptr(contrib_count)
        ckpt = _checkpoint_buffer(layout, isect_offsets, flatten_ids, tile_size, C, dev)
        a.t_checkpoints = B.ptr(ckpt)
        st = B.stream_of(means2d)
        prefix = _aniso_prefix(tex_store, tex_scales, st) if filter_code == B.TG_FILTER_ANISO_BILINEAR else None
        a.aniso_prefix = B.ptr(prefix)
        # the footprint integrals, kept for the adjoint (which then need not integrate them again)
        records = counts = None
        n_pix = math.prod(pshape)
        cap = min(ANISO_RECORDS, ANISO_RECORDS_BYTES // max(1, 16 * n_pix))
        if prefix is not None and cap > 0 and any(ctx.needs_input_grad):
            records = torch.empty((n_pix, cap, 4), dtype=torch.float32, device=dev)
            counts = torch.empty((n_pix,), dtype=torch.int32, device=dev)
            a.aniso_records, a.aniso_record_count, a.aniso_record_cap = B.ptr(records), B.ptr(counts), cap
        B.call("tg_rasterize_fwd", st, B.lib().tg_rasterize_fwd, ctypes.byref(a), st)
        ctx.save_for_backward(means2d, ray_transforms, colors, opacities, textures, normals, densify, backgrounds, m,
                              tex_store, tex_scales, isect_offsets, flatten_ids, render_colors, render_alphas,
                              last_ids, median_ids, gaussian_ids)
        ctx.cfg = (range_x, range_y, width, height, tile_size, absgrad, g_weight, adjoint, bg_grad_index_ok,
                   gs_contrib_threshold, N, n_contrib, C, pshape)
        ctx.layout = layout
        ctx.n_isects_dev = n_dev
        ctx.mip = (mip_levels, coarse, filter_code)
        ctx.t_checkpoints = ckpt
        ctx.aniso_prefix = prefix
        ctx.aniso_records = (records, counts)
        ctx.mark_non_differentiable(contrib_sum, contrib_count)
        return render_colors, render_alphas, render_normals, render_distort, render_median, contrib_sum, contrib_count

    @staticmethod
    def backward(ctx, v_render_colors, v_render_alphas, v_render_normals, v_render_distort, v_render_median,
                 v_contrib_sum, v_contrib_count):
        (means2d, ray_transforms, colors, opacities, textures, normals, densify, backgrounds, m, tex_store, tex_scales,
         isect_offsets, flatten_ids, render_colors, render_alphas, last_ids, median_ids,
         gaussian_ids) = ctx.saved_tensors
        (range_x, range_y, width, height, tile_size, absgrad, g_weight, adjoint, bg_grad_index_ok,
         gs_contrib_threshold, N, n_contrib, C, pshape) = ctx.cfg
        dev = means2d.device
        D = colors.shape[-1]

        def g(t, shape):
            return torch.zeros(shape, dtype=torch.float32, device=dev) if t is None else t.float().contiguous()

        v_rc = g(v_render_colors, pshape + (D,))
        v_ra = g(v_render_alphas, pshape + (1,))
        v_rn = g(v_render_normals, pshape + (3,))
        v_rd = g(v_render_distort, pshape + (1,))
        v_rm = g(v_render_median, pshape + (1,))
        f = _fwd_args(means2d, ray_transforms, colors, opacities, normals, tex_store, tex_scales, range_x, range_y,
                      backgrounds, m, width, height, tile_size, isect_offsets, flatten_ids, gaussian_ids, n_contrib,
                      0.0, g_weight, C, N, ctx.layout, ctx.n_isects_dev, *ctx.mip)
        f.t_checkpoints = B.ptr(ctx.t_checkpoints)
        f.aniso_prefix = B.ptr(ctx.aniso_prefix)
        if ctx.aniso_records[0] is not None:
            f.aniso_records, f.aniso_record_count = B.ptr(ctx.aniso_records[0]), B.ptr(ctx.aniso_records[1])
            f.aniso_record_cap = ctx.aniso_records[0].shape[1]
        v_means2d = torch.empty_like(means2d)
        v_means2d_abs = torch.empty_like(means2d) if absgrad else None
        v_ray_transforms = torch.empty_like(ray_transforms)
        v_colors = torch.empty_like(colors)
        v_opacities = torch.empty_like(opacities)
        v_normals = torch.empty_like(normals)
        want_tex = tex_store is not None and ctx.needs_input_grad[4]
        v_textures = torch.empty(textures.shape, dtype=torch.float32, device=dev) if want_tex else None
        v_densify = torch.empty_like(densify)
        a = B.RasterBwdArgs(f, B.ptr(render_colors), B.ptr(render_alphas), B.ptr(last_ids), B.ptr(median_ids),
                            B.ptr(v_rc), B.ptr(v_ra), B.ptr(v_rn), B.ptr(v_rd), B.ptr(v_rm), int(adjoint),
                            means2d.numel() // 2, B.ptr(v_means2d), B.ptr(v_means2d_abs),
                            B.ptr(v_ray_transforms), B.ptr(v_colors), B.ptr(v_opacities), B.ptr(v_normals),
                            B.ptr(v_textures), B.ptr(v_densify))
        L = ctx.mip[0]
        v_coarse = torch.empty_like(ctx.mip[1]) if L and want_tex else None
        a.v_tex_coarse = B.ptr(v_coarse)
        v_prefix = torch.empty_like(ctx.aniso_prefix) if ctx.aniso_prefix is not None and want_tex else None
        a.v_aniso_prefix = B.ptr(v_prefix)
        st = B.stream_of(means2d)
        B.call("tg_rasterize_bwd", st, B.lib().tg_rasterize_bwd, ctypes.byref(a), st)
        if v_coarse is not None:
            B.call("tg_generate_mipmap_bwd", st, B.lib().tg_generate_mipmap_bwd, B.ptr(v_coarse), B.ptr(v_textures),
                   textures.shape[0], L, st)
        if absgrad:
            means2d.absgrad = v_means2d_abs
        v_backgrounds = None
        if bg_grad_index_ok and backgrounds is not None and ctx.needs_input_grad[7]:
            if len(pshape) == 3:
                v_backgrounds = (v_rc * (1.0 - render_alphas).float()).sum(dim=(1, 2))
            else:
                vt = ctx.layout["view_table"]
                v_backgrounds = torch.stack([(v_rc[b:b + n] * (1.0 - render_alphas[b:b + n])).sum(0)
                                             for b, n in zip(vt.pix_base, vt.pix_count)])
        if v_textures is not None and textures.dtype != torch.float32:
            v_textures = v_textures.to(textures.dtype)
        return (v_means2d, v_ray_transforms, v_colors, v_opacities, v_textures, v_normals, v_densify, v_backgrounds,
                None, None, None, None, None, None, None, None, None, None, None, None, None, None, None, None, None,
                None, None, None)


_TRANSMITTANCE = ("divide", "checkpoint")


def _layout(tile_order, view_table, batch_depth=0, persistent=False, device=None, transmittance="divide"):
    if transmittance not in _TRANSMITTANCE:
        raise ValueError(f"transmittance must be one of {_TRANSMITTANCE}, got {transmittance!r}")
    ckpt = transmittance == "checkpoint"
    if tile_order is None and view_table is None and not batch_depth and not persistent and not ckpt:
        return None
    if tile_order is not None:
        tile_order = tile_order.to(torch.int32).contiguous()
    queue = torch.zeros((1,), dtype=torch.int32, device=device) if persistent else None
    return {"tile_order": tile_order, "view_table": view_table, "batch_depth": int(batch_depth or 0),
            "work_queue": queue, "checkpoints": ckpt}


def _checkpoint_buffer(layout, isect_offsets, flatten_ids, tile_size, C, device):
    """The transmittance checkpoints of tg_raster_fwd_args: [n_tiles + n_isects / bs + 1, tile_size^2] FP32,
    or None when the layout does not ask for them."""
    if layout is None or not layout.get("checkpoints"):
        return None
    vt = layout.get("view_table")
    n_tiles = vt.n_tiles if vt is not None else C * isect_offsets.shape[1] * isect_offsets.shape[2]
    bs = layout.get("batch_depth") or tile_size * tile_size
    return torch.empty((n_tiles + flatten_ids.numel() // bs + 1, tile_size * tile_size), dtype=torch.float32,
                       device=device)


def _check_common(means2d, ray_transforms, colors, opacities, isect_offsets, tile_size, image_width, image_height,
                  backgrounds, packed, view_table=None):
    C = isect_offsets.size(0) if view_table is None else view_table.n_views
    if packed:
        nnz = means2d.size(0)
        assert means2d.shape == (nnz, 2), means2d.shape
        assert ray_transforms.shape == (nnz, 3, 3), ray_transforms.shape
        assert colors.shape[0] == nnz, colors.shape
        assert opacities.shape == (nnz,), opacities.shape
    else:
        N = means2d.size(1)
        assert means2d.shape == (C, N, 2), means2d.shape
        assert ray_transforms.shape == (C, N, 3, 3), ray_transforms.shape
        assert colors.shape[:2] == (C, N), colors.shape
        assert opacities.shape == (C, N), opacities.shape
    if backgrounds is not None:
        assert backgrounds.shape == (C, colors.shape[-1]), backgrounds.shape
    if view_table is not None:
        assert packed, "the batching form takes packed inputs"
        assert isect_offsets.shape == (view_table.n_tiles,), isect_offsets.shape
        assert tile_size == view_table.tile_size, (tile_size, view_table.tile_size)
        return
    tile_height, tile_width = isect_offsets.shape[1:3]
    assert tile_height * tile_size >= image_height, f"Assert Failed: {tile_height} * {tile_size} >= {image_height}"
    assert tile_width * tile_size >= image_width, f"Assert Failed: {tile_width} * {tile_size} >= {image_width}"


def rasterize_to_pixels_textured_gaussians(
    means2d: Tensor,
    ray_transforms: Tensor,
    colors: Tensor,
    opacities: Tensor,
    textures: Tensor,
    texture_range_x: float,
    texture_range_y: float,
    normals: Tensor,
    densify: Tensor,
    image_width: int,
    image_height: int,
    tile_size: int,
    isect_offsets: Tensor,
    flatten_ids: Tensor,
    backgrounds: Optional[Tensor] = None,
    masks: Optional[Tensor] = None,
    packed: bool = False,
    absgrad: bool = False,
    distloss: bool = False,
    gs_contrib_threshold: float = 0.0,
    filtering: str = "bilinear",
    g_weight: float = 1.0,
    *,
    texture_storage: Optional[Tensor] = None,
    texture_scales: Optional[Tensor] = None,
    gaussian_ids: Optional[Tensor] = None,
    tile_order: Optional[Tensor] = None,
    view_table=None,
    batch_depth: int = 0,
    persistent: bool = False,
    transmittance: str = "divide",
) -> Tuple[Tensor, ...]:
    """Rasterize textured 2D Gaussians to pixels (reference: cuda/_wrapper.py:1806-2002).

    Returns the reference's 7-tuple ``(render_colors, render_alphas,
    render_normals, render_distort, render_median, gs_contrib_sum,
    gs_contrib_count)``.  ``texture_storage`` (BF16 / FP16 / FP8-E4M3, same
    [N, th, tw, 4] layout, plus ``texture_scales`` [N] for FP8) is sampled in
    place of ``textures``; gradients still flow to ``textures`` in FP32.

    Packed inputs ([nnz, ...]) need ``gaussian_ids`` [nnz] (the packed
    projection's output): entry e samples texture row ``gaussian_ids[e]`` and
    the contribution statistics are per Gaussian, [N].  The reference indexes
    textures and statistics with the packed entry index, out of range for
    packed inputs, so it is not followed there.

    ``tile_order`` (a permutation of the tiles, e.g. from
    :func:`tile_order_heaviest_first`) sets the order in which tiles are
    taken; ``view_table`` selects the batching form (views of uneven size,
    flat ``isect_offsets`` from :func:`isect_offset_encode_views`, flat
    per-pixel outputs [n_pixels, ...]).  ``batch_depth`` sets how many splats
    are staged in shared memory per batch (0: tile_size^2, the reference's).
    ``persistent=True`` launches as many CTAs as fit on the device, which take
    tiles from a device work counter instead of one CTA per tile.

    ``transmittance``: "divide" (the reference's scheme: the adjoint recovers
    each splat's transmittance by dividing the final one by (1 - alpha), back
    to front over the whole list) or "checkpoint" (the forward also keeps
    every pixel's transmittance at the end of each batch of its tile, and the
    adjoint restarts the division from it at every batch, so rounding
    accumulates over one batch instead of up to thousands of splats; closer to
    exact arithmetic at pixels with many contributors, for a buffer of
    (n_tiles + n_isects / batch_depth) x tile_size^2 floats).
    """
    _check_common(means2d, ray_transforms, colors, opacities, isect_offsets, tile_size, image_width, image_height,
                  backgrounds, packed, view_table)
    if filtering not in _FILTER_ADJOINT:
        raise Exception(f"Unsupported filter type {filtering}")
    assert textures.dim() == 4 and textures.shape[-1] == 4, textures.shape
    mip_levels = mip_levels_of(textures) if filtering in _MIP_FILTERS else 0
    filter_code = _FILTER_CODE.get(filtering, B.TG_FILTER_BILINEAR)
    if packed:
        if gaussian_ids is None:
            raise ValueError("packed textured rasterization needs gaussian_ids (texture row of each packed entry)")
        assert gaussian_ids.shape == (means2d.shape[0],), gaussian_ids.shape
        gaussian_ids = gaussian_ids.to(torch.int64).contiguous()
    else:
        gaussian_ids = None
    colors, backgrounds, padded = _pad_channels(colors, backgrounds)
    store = textures if texture_storage is None else texture_storage
    store = store.contiguous()
    if store.dtype == torch.float8_e4m3fn:
        assert texture_scales is not None, "FP8 texture storage needs texture_scales"
        texture_scales = texture_scales.float().contiguous()
    if store.dtype == torch.float64:
        store = store.float()
    out = _RasterizeToPixelsTextured.apply(
        means2d.contiguous(), ray_transforms.contiguous(), colors.contiguous().float(), opacities.contiguous(),
        textures, normals.contiguous(), densify.contiguous(),
        None if backgrounds is None else backgrounds.contiguous(), masks, store, texture_scales,
        float(texture_range_x), float(texture_range_y), int(image_width), int(image_height), int(tile_size),
        isect_offsets.contiguous(), flatten_ids.contiguous(), absgrad, gs_contrib_threshold, g_weight,
        _FILTER_ADJOINT[filtering], False, gaussian_ids, textures.shape[0],
        _layout(tile_order, view_table,
                batch_depth or (ANISO_BATCH_DEPTH if filter_code == B.TG_FILTER_ANISO_BILINEAR else 0), persistent,
                means2d.device, transmittance), mip_levels,
        filter_code)
    render_colors = out[0]
    if padded > 0:
        render_colors = render_colors[..., :-padded]
    return (render_colors,) + tuple(out[1:])


def rasterize_to_pixels_2dgs(
    means2d: Tensor,
    ray_transforms: Tensor,
    colors: Tensor,
    opacities: Tensor,
    normals: Tensor,
    densify: Tensor,
    image_width: int,
    image_height: int,
    tile_size: int,
    isect_offsets: Tensor,
    flatten_ids: Tensor,
    backgrounds: Optional[Tensor] = None,
    masks: Optional[Tensor] = None,
    packed: bool = False,
    absgrad: bool = False,
    distloss: bool = False,
    gs_contrib_threshold: float = 0.0,
    *,
    gaussian_ids: Optional[Tensor] = None,
    n_gaussians: Optional[int] = None,
    tile_order: Optional[Tensor] = None,
    view_table=None,
    batch_depth: int = 0,
    persistent: bool = False,
) -> Tuple[Tensor, ...]:
    """Rasterize plain 2D Gaussians to pixels (reference: cuda/_wrapper.py:1647-1784).

    Same 7-tuple as the textured form; the background gradient is computed
    when the backgrounds require it (reference: cuda/_wrapper.py:2920-2925).
    Packed inputs: the contribution statistics are per entry, [nnz], or per
    Gaussian, [n_gaussians], when ``gaussian_ids`` and ``n_gaussians`` are
    given (the reference sizes them [0] for packed inputs).  ``tile_order``,
    ``view_table``, ``batch_depth`` and ``persistent`` as in
    :func:`rasterize_to_pixels_textured_gaussians`.
    """
    _check_common(means2d, ray_transforms, colors, opacities, isect_offsets, tile_size, image_width, image_height,
                  backgrounds, packed, view_table)
    if packed and gaussian_ids is not None:
        if n_gaussians is None:
            raise ValueError("gaussian_ids needs n_gaussians")
        assert gaussian_ids.shape == (means2d.shape[0],), gaussian_ids.shape
        gaussian_ids = gaussian_ids.to(torch.int64).contiguous()
    else:
        gaussian_ids, n_gaussians = None, 0
    colors, backgrounds, padded = _pad_channels(colors, backgrounds)
    dummy = torch.empty((0, 1, 1, 4), dtype=torch.float32, device=means2d.device)
    out = _RasterizeToPixelsTextured.apply(
        means2d.contiguous(), ray_transforms.contiguous(), colors.contiguous().float(), opacities.contiguous(), dummy,
        normals.contiguous(), densify.contiguous(), None if backgrounds is None else backgrounds.contiguous(), masks,
        None, None, 3.0, 3.0, int(image_width), int(image_height), int(tile_size), isect_offsets.contiguous(),
        flatten_ids.contiguous(), absgrad, gs_contrib_threshold, 1.0, B.TG_ADJ_REFERENCE, True, gaussian_ids,
        int(n_gaussians), _layout(tile_order, view_table, batch_depth, persistent, means2d.device))
    render_colors = out[0]
    if padded > 0:
        render_colors = render_colors[..., :-padded]
    return (render_colors,) + tuple(out[1:])


# --------------------------------------------------------------------------- gradient consumers
_SHADOW_FORMAT = {None: B.TG_TEX_NONE, torch.bfloat16: B.TG_TEX_BF16, torch.float16: B.TG_TEX_F16}


@torch.no_grad()
def selective_adam_update(param: Tensor, param_grad: Tensor, exp_avg: Tensor, exp_avg_sq: Tensor,
                          tiles_touched: Tensor, lr: float, b1: float, b2: float, eps: float, N: int, M: int, *,
                          shadow: Optional[Tensor] = None) -> None:
    """Adam step on the rows whose ``tiles_touched`` flag is set (reference: cuda/_wrapper.py:26-40,
    csrc/adam.cu:17-45; no bias correction).  ``shadow`` (BF16 / FP16, same number of elements) receives the
    updated rows in the same pass, e.g. the low-precision texture storage the compositor samples."""
    for t in (param, param_grad, exp_avg, exp_avg_sq):
        assert t.dtype == torch.float32 and t.is_contiguous() and t.numel() == N * M, (t.dtype, t.shape)
    vis = tiles_touched.reshape(-1)
    assert vis.numel() == N, vis.shape
    vis = vis.to(torch.uint8).contiguous()
    if shadow is not None:
        assert shadow.dtype in (torch.bfloat16, torch.float16) and shadow.is_contiguous() and shadow.numel() == N * M
    fmt = _SHADOW_FORMAT[None if shadow is None else shadow.dtype]
    st = B.stream_of(param)
    B.call("tg_selective_adam", st, B.lib().tg_selective_adam, B.ptr(param), B.ptr(param_grad), B.ptr(exp_avg),
           B.ptr(exp_avg_sq), B.ptr(vis), float(lr), float(b1), float(b2), float(eps), int(N), int(M), fmt,
           B.ptr(shadow), st)


@torch.no_grad()
def densify_stats(grads2d: Tensor, radii: Tensor, width: int, height: int, n_cameras: int, grad2d: Tensor,
                  count: Tensor, max_radii: Optional[Tensor] = None, gaussian_ids: Optional[Tensor] = None) -> None:
    """Running densification statistics in place (reference: strategy/default.py:213-261): per entry with
    radius > 0, ``grad2d[g] += |grad * (width/2 * C, height/2 * C)|``, ``count[g] += 1`` and
    ``max_radii[g] = max(max_radii[g], radius / max(width, height))``.  Dense inputs are [C,N,...];
    packed ones [nnz,...] with ``gaussian_ids``."""
    N = grad2d.numel()
    grads2d = grads2d.float().contiguous()
    radii = radii.int().contiguous()
    for t in (grad2d, count) + (() if max_radii is None else (max_radii,)):
        assert t.dtype == torch.float32 and t.is_contiguous() and t.numel() == N
    if gaussian_ids is None:
        assert radii.shape == (n_cameras, N) and grads2d.shape == (n_cameras, N, 2), (radii.shape, grads2d.shape)
        E = n_cameras * N
    else:
        E = radii.numel()
        gaussian_ids = gaussian_ids.to(torch.int64).contiguous()
        assert gaussian_ids.shape == (E,) and grads2d.shape == (E, 2)
    a = B.DensifyStatsArgs(int(n_cameras), N, E, B.ptr(grads2d), B.ptr(radii), B.ptr(gaussian_ids), int(width),
                           int(height), B.ptr(grad2d), B.ptr(count), B.ptr(max_radii))
    st = B.stream_of(grad2d)
    B.call("tg_densify_stats", st, B.lib().tg_densify_stats, ctypes.byref(a), st)
