"""numpy front end of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loads oracle/libtg_oracle.so (built by oracle/build.py) through ctypes and
exposes the stages of the textured 2DGS path plus a whole-pipeline
``render`` / ``render_backward`` pair that mirrors
``rasterization_textured_gaussians`` (textured_gaussians/rendering.py:1474-1685)
and ``rasterization_2dgs`` (textured_gaussians/rendering.py:1135-1338).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only as the checker.  The product package never does.

Parity status: projection, intersection, offsets and SH are pinned against
golden vectors from the reference's pure-torch twins; the plain compositor is
pinned against the reference's torch ``accumulate_2dgs``; the textured
compositor is a restatement with no executable reference ("parity unpinned").
Its adjoints are checked by FP64 finite differences instead: the exact
bilinear adjoint (tests/test_adjoint_fd.py), the reference and bwd2 adjoints
against it (tests/test_oracle_adjoint_modes.py), the mipmapped2 and
anisotropic_bilinear adjoints (tests/test_oracle_filter_adjoint.py) and the SH
adjoint (tests/test_oracle_sh_adjoint.py).
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import build as _build

_LIB = None

c_int = ctypes.c_int
c_i64 = ctypes.c_int64
c_dbl = ctypes.c_double
c_ptr = ctypes.c_void_p


def lib():
    global _LIB
    if _LIB is None:
        path = _build.build()
        _LIB = ctypes.CDLL(path)
        for suf in ("f32", "f64"):
            getattr(_LIB, f"tgo_project_fwd_{suf}").argtypes = [c_int, c_int] + [c_ptr] * 5 + [c_int, c_int, c_dbl, c_dbl, c_dbl] + [c_ptr] * 5
            getattr(_LIB, f"tgo_project_bwd_{suf}").argtypes = [c_int, c_int] + [c_ptr] * 11 + [c_int] + [c_ptr] * 3
            getattr(_LIB, f"tgo_isect_count_{suf}").argtypes = [c_i64, c_ptr, c_ptr, c_int, c_int, c_int, c_ptr]
            getattr(_LIB, f"tgo_isect_emit_{suf}").argtypes = [c_i64, c_i64] + [c_ptr] * 5 + [c_int] * 4 + [c_ptr] * 2
            getattr(_LIB, f"tgo_sh_fwd_{suf}").argtypes = [c_i64, c_int, c_int] + [c_ptr] * 4
            getattr(_LIB, f"tgo_sh_bwd_{suf}").argtypes = [c_i64, c_int, c_int] + [c_ptr] * 6
            getattr(_LIB, f"tgo_raster_fwd_{suf}").argtypes = (
                [c_int] * 8 + [c_i64] + [c_ptr] * 6 + [c_int] * 4 + [c_dbl, c_dbl] + [c_ptr] * 5 + [c_dbl, c_dbl]
                + [c_ptr] * 11
            )
            getattr(_LIB, f"tgo_raster_bwd_{suf}").argtypes = (
                [c_int] * 8 + [c_i64, c_i64] + [c_ptr] * 6 + [c_int] * 4 + [c_dbl, c_dbl] + [c_ptr] * 5 + [c_dbl]
                + [c_ptr] * 9 + [c_int] + [c_ptr] * 8
            )
        _LIB.tgo_sort_pairs.argtypes = [c_i64, c_ptr, c_ptr, c_int]
        _LIB.tgo_aniso_sample.argtypes = [c_ptr, c_int, c_int, c_ptr, c_ptr]
        _LIB.tgo_aniso_sample.restype = c_dbl
        _LIB.tgo_offset_encode.argtypes = [c_i64, c_ptr, c_int, c_int, c_int, c_ptr]
    return _LIB


def _p(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "oracle arrays must be C-contiguous"
    return a.ctypes.data_as(ctypes.c_void_p)


def _suf(dtype) -> str:
    return "f64" if np.dtype(dtype) == np.float64 else "f32"


def _c(a, dtype):
    return None if a is None else np.ascontiguousarray(a, dtype=dtype)


def tile_bits(n: int) -> int:
    """floor(log2(n)) + 1, the bit width the reference uses (isect_tiles.cu:156-157)."""
    return int(math.floor(math.log2(n))) + 1


# ------------------------------------------------------------------ projection
def project_fwd(means, quats, scales, viewmats, Ks, W, H, near_plane=0.01, far_plane=1e10, radius_clip=0.0,
                dtype=np.float32):
    means, quats, scales, viewmats, Ks = (_c(x, dtype) for x in (means, quats, scales, viewmats, Ks))
    C, N = viewmats.shape[0], means.shape[0]
    radii = np.zeros((C, N), np.int32)
    means2d = np.zeros((C, N, 2), dtype)
    depths = np.zeros((C, N), dtype)
    M = np.zeros((C, N, 3, 3), dtype)
    normals = np.zeros((C, N, 3), dtype)
    getattr(lib(), f"tgo_project_fwd_{_suf(dtype)}")(
        C, N, _p(means), _p(quats), _p(scales), _p(viewmats), _p(Ks), int(W), int(H), near_plane, far_plane,
        radius_clip, _p(radii), _p(means2d), _p(depths), _p(M), _p(normals))
    return radii, means2d, depths, M, normals


def project_bwd(means, quats, scales, viewmats, Ks, radii, M, v_means2d, v_depths, v_normals, v_M, mode=0,
                dtype=np.float32):
    """mode 0: reference adjoint, 1: reference norm_rot_grad adjoint, 2: exact."""
    args = [_c(x, dtype) for x in (means, quats, scales, viewmats, Ks)]
    C, N = args[3].shape[0], args[0].shape[0]
    radii = np.ascontiguousarray(radii, np.int32)
    rest = [_c(x, dtype) for x in (M, v_means2d, v_depths, v_normals, v_M)]
    v_means = np.zeros((N, 3), dtype)
    v_quats = np.zeros((N, 4), dtype)
    v_scales = np.zeros((N, 3), dtype)
    getattr(lib(), f"tgo_project_bwd_{_suf(dtype)}")(
        C, N, *[_p(x) for x in args], _p(radii), *[_p(x) for x in rest], int(mode), _p(v_means), _p(v_quats),
        _p(v_scales))
    return v_means, v_quats, v_scales


# ------------------------------------------------------------------ intersection
def isect_tiles(means2d, radii, depths, tile_size, tile_width, tile_height, n_cameras, camera_ids=None,
                sort=True):
    """Tile counts, 64-bit keys and flatten ids; sorted stably on the reference's bit range."""
    fdt = np.float64 if np.asarray(means2d).dtype == np.float64 else np.float32
    means2d = np.ascontiguousarray(means2d, fdt)
    radii = np.ascontiguousarray(radii, np.int32)
    depths32 = np.ascontiguousarray(depths, np.float32)
    packed = means2d.ndim == 2
    E = means2d.shape[0] if packed else means2d.shape[0] * means2d.shape[1]
    N = 0 if packed else means2d.shape[1]
    tpg = np.zeros(radii.shape, np.int32)
    L = lib()
    getattr(L, f"tgo_isect_count_{_suf(fdt)}")(E, _p(means2d), _p(radii), tile_size, tile_width, tile_height, _p(tpg))
    cum = np.cumsum(tpg.reshape(-1).astype(np.int64))
    n_isects = int(cum[-1]) if E else 0
    isect_ids = np.zeros(n_isects, np.int64)
    flatten_ids = np.zeros(n_isects, np.int32)
    tb = tile_bits(tile_width * tile_height)
    cb = tile_bits(n_cameras)
    cam = None if camera_ids is None else np.ascontiguousarray(camera_ids, np.int64)
    if n_isects:
        getattr(L, f"tgo_isect_emit_{_suf(fdt)}")(E, N, _p(cam), _p(means2d), _p(radii), _p(depths32), _p(cum),
                                                   tile_size, tile_width, tile_height, tb, _p(isect_ids),
                                                   _p(flatten_ids))
        if sort:
            L.tgo_sort_pairs(n_isects, _p(isect_ids), _p(flatten_ids), 32 + tb + cb)
    return tpg, isect_ids, flatten_ids


def sort_pairs(keys, vals, end_bit):
    keys = np.array(keys, np.int64, copy=True)
    vals = np.array(vals, np.int32, copy=True)
    lib().tgo_sort_pairs(keys.size, _p(keys), _p(vals), int(end_bit))
    return keys, vals


def isect_offset_encode(isect_ids, n_cameras, tile_width, tile_height):
    isect_ids = np.ascontiguousarray(isect_ids, np.int64)
    n_tiles = tile_width * tile_height
    offsets = np.zeros((n_cameras, tile_height, tile_width), np.int32)
    lib().tgo_offset_encode(isect_ids.size, _p(isect_ids), n_cameras, n_tiles, tile_bits(n_tiles), _p(offsets))
    return offsets


# ------------------------------------------------------------------ SH
def sh_fwd(degree, dirs, coeffs, masks=None, dtype=np.float32):
    dirs = _c(dirs, dtype)
    lead = dirs.shape[:-1]
    coeffs = _c(np.broadcast_to(coeffs, lead + coeffs.shape[-2:]), dtype)
    n = int(np.prod(lead))
    K = coeffs.shape[-2]
    m = None if masks is None else np.ascontiguousarray(np.broadcast_to(masks, lead), np.uint8)
    out = np.zeros(lead + (3,), dtype)
    getattr(lib(), f"tgo_sh_fwd_{_suf(dtype)}")(n, degree, K, _p(dirs), _p(coeffs), _p(m), _p(out))
    return out


def sh_bwd(degree, dirs, coeffs, v_colors, masks=None, dtype=np.float32):
    dirs = _c(dirs, dtype)
    lead = dirs.shape[:-1]
    coeffs = _c(np.broadcast_to(coeffs, lead + coeffs.shape[-2:]), dtype)
    n = int(np.prod(lead))
    K = coeffs.shape[-2]
    m = None if masks is None else np.ascontiguousarray(np.broadcast_to(masks, lead), np.uint8)
    v_colors = _c(v_colors, dtype)
    v_coeffs = np.zeros_like(coeffs)
    v_dirs = np.zeros_like(dirs)
    getattr(lib(), f"tgo_sh_bwd_{_suf(dtype)}")(n, degree, K, _p(dirs), _p(coeffs), _p(m), _p(v_colors),
                                                _p(v_coeffs), _p(v_dirs))
    return v_coeffs, v_dirs


# ------------------------------------------------------------------ compositor
@dataclass
class RasterFwdOut:
    colors: np.ndarray
    alphas: np.ndarray
    normals: np.ndarray
    distort: np.ndarray
    median: np.ndarray
    last_ids: np.ndarray
    median_ids: np.ndarray
    contrib_sum: np.ndarray
    contrib_count: np.ndarray
    pair_count: np.ndarray
    branch_sig: np.ndarray


def _tex_shape(textures, mip_levels):
    if textures is None:
        return 0, 0
    if mip_levels:
        assert textures.ndim == 3 and textures.shape[1] == (4 ** (mip_levels + 1) - 1) // 3, "expects the full pyramid"
        return 1 << mip_levels, 1 << mip_levels
    return textures.shape[1], textures.shape[2]


def aniso_sample(corners, texture):
    """anisotropic_bilinear filter of one footprint quad (corners [4,2] in texel coordinates) over a texture
    [ry, rx, 4], in FP64: the bilinear interpolant integrated over the quad's part inside the texel grid,
    divided by the quad's area.  Returns (rgba [4], area)."""
    c = np.ascontiguousarray(corners, np.float64).reshape(4, 2)
    t = np.ascontiguousarray(texture, np.float64)
    out = np.zeros(4, np.float64)
    area = lib().tgo_aniso_sample(_p(c), t.shape[1], t.shape[0], _p(t), _p(out))
    return out, area


def mip_level_base(L: int, t: int) -> int:
    """Texel index of level t (side 2^(L-t)) in the pyramid of a 2^L texture, coarsest first (filters/mip2.cuh:15-25)."""
    return (4 ** (L - t) - 1) // 3


def generate_mipmap(textures):
    """Full mip pyramid [G, (4^(L+1)-1)/3, 4] of square 2^L textures [G, R, R, 4], restating
    generate_mipmap_fwd.cu:19-57: level 0 is the texture itself; a texel of level t is ((a + b) + c + d) / 4 of its
    four children at level t - 1 (row-major order), in the textures' dtype."""
    G, R = textures.shape[0], textures.shape[1]
    L = R.bit_length() - 1
    assert textures.shape[2] == R and R == 1 << L
    out = np.empty((G, (4 ** (L + 1) - 1) // 3, textures.shape[3]), textures.dtype)
    lvl = np.ascontiguousarray(textures)
    out[:, mip_level_base(L, 0):] = lvl.reshape(G, R * R, -1)
    four = textures.dtype.type(4)
    for t in range(1, L + 1):
        lvl = (lvl[:, 0::2, 0::2] + lvl[:, 0::2, 1::2] + lvl[:, 1::2, 0::2] + lvl[:, 1::2, 1::2]) / four
        side = R >> t
        out[:, mip_level_base(L, t):mip_level_base(L, t) + side * side] = lvl.reshape(G, side * side, -1)
    return out


def generate_mipmap_bwd(v_pyramid, L: int):
    """Texture gradient [G, R, R, 4] from the full pyramid's, restating generate_mipmap_bwd.cu:19-60: coarsest first,
    each child adds its parent's (already complete) gradient / 4."""
    v = np.array(v_pyramid)
    G, four = v.shape[0], v.dtype.type(4)
    for t in range(L, 0, -1):
        side = 1 << (L - t)
        par = v[:, mip_level_base(L, t):mip_level_base(L, t) + side * side].reshape(G, side, side, -1) / four
        cb = mip_level_base(L, t - 1)
        ch = v[:, cb:cb + 4 * side * side].reshape(G, side, 2, side, 2, -1)
        ch += par[:, :, None, :, None, :]
        v[:, cb:cb + 4 * side * side] = ch.reshape(G, 4 * side * side, -1)
    R = 1 << L
    return v[:, mip_level_base(L, 0):].reshape(G, R, R, -1)


def raster_fwd(means2d, M, colors, opacities, normals, textures, offsets, flatten_ids, W, H, tile_size,
               range_x=3.0, range_y=3.0, backgrounds=None, masks=None, gaussian_ids=None, n_gauss=None,
               contrib_threshold=0.0, g_weight=1.0, mip_levels=0, aniso=False, dtype=np.float32):
    """Compositor forward.  ``textures=None`` selects the plain 2DGS compositor.

    Dense layout: means2d [C,N,2] ...; packed layout: [nnz,...] plus
    ``gaussian_ids`` [nnz] and ``n_gauss``.  ``mip_levels`` L > 0 selects the
    mipmapped2 filter on a 2^L x 2^L texture: ``textures`` is then the full
    pyramid [G, (4^(L+1)-1)/3, 4] of :func:`generate_mipmap`.  ``aniso``
    selects the anisotropic_bilinear filter (footprint-integrated bilinear).
    """
    means2d, M, colors, opacities, normals, textures, backgrounds = (
        _c(x, dtype) for x in (means2d, M, colors, opacities, normals, textures, backgrounds))
    offsets = np.ascontiguousarray(offsets, np.int32)
    flatten_ids = np.ascontiguousarray(flatten_ids, np.int32)
    C, th, tw = offsets.shape
    packed = means2d.ndim == 2
    N = n_gauss if packed else means2d.shape[1]
    D = colors.shape[-1]
    G = N if gaussian_ids is None else n_gauss
    gid = None if gaussian_ids is None else np.ascontiguousarray(gaussian_ids, np.int64)
    m = None if masks is None else np.ascontiguousarray(masks, np.uint8)
    ry, rx = _tex_shape(textures, mip_levels)
    o = RasterFwdOut(
        colors=np.zeros((C, H, W, D), dtype), alphas=np.zeros((C, H, W, 1), dtype), normals=np.zeros((C, H, W, 3), dtype),
        distort=np.zeros((C, H, W, 1), dtype), median=np.zeros((C, H, W, 1), dtype),
        last_ids=np.zeros((C, H, W), np.int32), median_ids=np.zeros((C, H, W), np.int32),
        contrib_sum=np.zeros((G,), dtype), contrib_count=np.zeros((G,), dtype), pair_count=np.zeros((C, H, W), np.int32),
        branch_sig=np.zeros((C, H, W), np.uint64))
    getattr(lib(), f"tgo_raster_fwd_{_suf(dtype)}")(
        C, N, D, int(W), int(H), tile_size, tw, th, flatten_ids.size, _p(means2d), _p(M), _p(colors), _p(opacities),
        _p(normals), _p(textures), ry, rx, int(mip_levels), int(bool(aniso)), float(range_x), float(range_y), _p(backgrounds), _p(m),
        _p(offsets), _p(flatten_ids), _p(gid), float(contrib_threshold), float(g_weight), _p(o.colors), _p(o.alphas),
        _p(o.normals), _p(o.distort), _p(o.median), _p(o.last_ids), _p(o.median_ids), _p(o.contrib_sum),
        _p(o.contrib_count), _p(o.pair_count), _p(o.branch_sig))
    return o


@dataclass
class RasterBwdOut:
    v_means2d: np.ndarray
    v_means2d_abs: np.ndarray
    v_M: np.ndarray
    v_colors: np.ndarray
    v_opacities: np.ndarray
    v_normals: np.ndarray
    v_textures: Optional[np.ndarray]
    v_densify: np.ndarray


def raster_bwd(means2d, M, colors, opacities, normals, textures, offsets, flatten_ids, W, H, tile_size, fwd,
               v_colors, v_alphas, v_normals, v_distort, v_median, range_x=3.0, range_y=3.0, backgrounds=None,
               masks=None, gaussian_ids=None, n_gauss=None, g_weight=1.0, mode=0, mip_levels=0, aniso=False,
               dtype=np.float32):
    """Compositor adjoint.  mode 0: reference "bilinear", 1: "bilinear_bwd2", 2: exact.  With ``mip_levels`` > 0
    (mipmapped2, mode 0 only, as the reference has no other) ``v_textures`` is the full pyramid's gradient."""
    means2d, M, colors, opacities, normals, textures, backgrounds = (
        _c(x, dtype) for x in (means2d, M, colors, opacities, normals, textures, backgrounds))
    offsets = np.ascontiguousarray(offsets, np.int32)
    flatten_ids = np.ascontiguousarray(flatten_ids, np.int32)
    C, th, tw = offsets.shape
    packed = means2d.ndim == 2
    N = n_gauss if packed else means2d.shape[1]
    D = colors.shape[-1]
    E = means2d.shape[0] if packed else C * N
    gid = None if gaussian_ids is None else np.ascontiguousarray(gaussian_ids, np.int64)
    m = None if masks is None else np.ascontiguousarray(masks, np.uint8)
    ry, rx = _tex_shape(textures, mip_levels)
    fc, fa = _c(fwd.colors, dtype), _c(fwd.alphas, dtype)
    li, mi = np.ascontiguousarray(fwd.last_ids, np.int32), np.ascontiguousarray(fwd.median_ids, np.int32)
    vc, va, vn, vd, vm = (_c(x, dtype) for x in (v_colors, v_alphas, v_normals, v_distort, v_median))
    o = RasterBwdOut(
        v_means2d=np.zeros(means2d.shape, dtype), v_means2d_abs=np.zeros(means2d.shape, dtype),
        v_M=np.zeros(M.shape, dtype), v_colors=np.zeros(colors.shape, dtype),
        v_opacities=np.zeros(opacities.shape, dtype), v_normals=np.zeros(normals.shape, dtype),
        v_textures=None if textures is None else np.zeros(textures.shape, dtype),
        v_densify=np.zeros(means2d.shape, dtype))
    getattr(lib(), f"tgo_raster_bwd_{_suf(dtype)}")(
        C, N, D, int(W), int(H), tile_size, tw, th, flatten_ids.size, E, _p(means2d), _p(M), _p(colors),
        _p(opacities), _p(normals), _p(textures), ry, rx, int(mip_levels), int(bool(aniso)), float(range_x), float(range_y), _p(backgrounds), _p(m),
        _p(offsets), _p(flatten_ids), _p(gid), float(g_weight), _p(fc), _p(fa), _p(li), _p(mi), _p(vc), _p(va),
        _p(vn), _p(vd), _p(vm), int(mode), _p(o.v_means2d), _p(o.v_means2d_abs), _p(o.v_M), _p(o.v_colors),
        _p(o.v_opacities), _p(o.v_normals), _p(o.v_textures), _p(o.v_densify))
    return o


# ---------------------------------------------------------------- gradient consumers (numpy)
def selective_adam(param, grad, exp_avg, exp_avg_sq, visibility, lr, b1, b2, eps, dtype=np.float64):
    """Selective Adam on rows of the first axis, restating textured_gaussians/cuda/csrc/adam.cu:29-44: rows with
    visibility False are untouched; m = b1 m + (1-b1) g, v = b2 v + (1-b2) g^2, p += -lr m / (sqrt(v) + eps), no
    bias correction.  The hyper-parameters are FP32 as in the reference's signature (adam.cu:25-28: const float lr,
    b1, b2, eps), so 1 - b2 is 1 - fp32(b2) (exact in FP32).  Returns new (param, exp_avg, exp_avg_sq)."""
    lr, b1, b2, eps = (float(np.float32(x)) for x in (lr, b1, b2, eps))
    p, g, m, v = (np.array(x, dtype) for x in (param, grad, exp_avg, exp_avg_sq))
    sel = np.asarray(visibility).reshape(-1).astype(bool)
    m[sel] = b1 * m[sel] + (1.0 - b1) * g[sel]
    v[sel] = b2 * v[sel] + (1.0 - b2) * g[sel] * g[sel]
    p[sel] = p[sel] + (-lr * m[sel] / (np.sqrt(v[sel]) + eps))
    return p, m, v


def densify_stats(grads2d, radii, width, height, n_cameras, N, gaussian_ids=None, dtype=np.float64):
    """Running densification statistics from zero, restating DefaultStrategy._update_state
    (textured_gaussians/strategy/default.py:225-261): per entry with radius > 0 the norm of
    (gx * width/2 * C, gy * height/2 * C) is added to grad2d[g], 1 to count[g], and max_radii[g] is the
    maximum of radius / max(width, height) computed as an FP32 division, as the reference's torch division does
    (a true maximum; the reference's indexed assignment keeps the last camera's value for a Gaussian seen by
    several cameras).  Dense: [C,N] entries, packed: gaussian_ids."""
    g = np.array(grads2d, dtype).reshape(-1, 2).copy()
    r = np.asarray(radii).reshape(-1)
    g[:, 0] *= width / 2.0 * n_cameras
    g[:, 1] *= height / 2.0 * n_cameras
    gid = (np.tile(np.arange(N), n_cameras) if gaussian_ids is None else np.asarray(gaussian_ids).reshape(-1))
    sel = r > 0
    grad2d = np.zeros(N, dtype)
    count = np.zeros(N, dtype)
    max_radii = np.zeros(N, np.float32)
    np.add.at(grad2d, gid[sel], np.linalg.norm(g[sel], axis=-1))
    np.add.at(count, gid[sel], 1.0)
    frac = r[sel].astype(np.float32) / np.float32(max(width, height))
    np.maximum.at(max_radii, gid[sel], frac)
    return grad2d, count, max_radii
