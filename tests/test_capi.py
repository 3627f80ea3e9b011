"""C-ABI library checks that need no GPU: it loads, exports every entry point
declared in include/tg2dgs.h, and rejects bad arguments with error codes
before touching a device."""
import ctypes
import os
import re
import subprocess

import pytest

from textured_gaussians_b200 import _backend as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "tg2dgs.h")


def declared_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^TG_API\s+[\w\s\*]+?\b(tg_\w+)\s*\(", src, flags=re.M)))


def test_library_loads_and_reports_version():
    assert B.lib().tg_version() >= 1


def test_every_declared_symbol_is_exported():
    syms = declared_symbols()
    assert len(syms) >= 14, syms
    out = subprocess.run(["nm", "-D", "--defined-only", B.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\sT\s+(tg_\w+)$", out, flags=re.M))
    missing = [s for s in syms if s not in exported]
    assert not missing, f"declared but not exported: {missing}"
    for s in syms:
        getattr(B.lib(), s)


def test_workspace_sizes_grow_with_n():
    L = B.lib()
    assert L.tg_sort_workspace_bytes(10, 40) > 0
    assert L.tg_sort_workspace_bytes(10_000_000, 48) > L.tg_sort_workspace_bytes(1_000_000, 48)
    assert L.tg_scan_workspace_bytes(1 << 20) >= 8 * ((1 << 20) // 4096)


def test_invalid_arguments_are_rejected_without_a_device():
    L = B.lib()
    # null args
    assert L.tg_project_fwd(None, None) == -1
    assert L.tg_rasterize_fwd(None, None) == -1
    # unsupported channel count
    a = B.RasterFwdArgs()
    a.C, a.N, a.D, a.width, a.height, a.tile_size, a.tile_width, a.tile_height = 1, 1, 9, 16, 16, 16, 1, 1
    assert L.tg_rasterize_fwd(ctypes.byref(a), None) == -2
    assert b"channels" in L.tg_last_error()
    # unsupported tile size
    a.D, a.tile_size = 3, 12
    assert L.tg_rasterize_fwd(ctypes.byref(a), None) == -2
    # tile grid that does not cover the image
    a.tile_size, a.width = 16, 64
    assert L.tg_rasterize_fwd(ctypes.byref(a), None) == -1
    # sort: too many pairs, bad bit range
    r = ctypes.c_int32(7)
    assert L.tg_sort_pairs(None, None, None, None, 1 << 31, 40, None, 0, ctypes.byref(r), None) == -1
    assert L.tg_sort_pairs(None, None, None, None, 10, 65, None, 0, ctypes.byref(r), None) == -1
    # trivially sorted sizes need no buffers
    assert L.tg_sort_pairs(None, None, None, None, 1, 40, None, 0, ctypes.byref(r), None) == 0 and r.value == 0
    # isect: camera + tile ids that do not fit 32 bits
    ia = B.IsectArgs()
    ia.n_elems, ia.tile_size, ia.tile_width, ia.tile_height, ia.n_cameras = 0, 16, 1 << 16, 1 << 10, 64
    assert L.tg_isect_count(ctypes.byref(ia), None) == -1
    # SH degree above 4
    assert L.tg_sh_fwd(1, 1, 5, 36, None, None, None, None, None) == -1
    # packed projection: null args, too many cameras, missing workspace, nnz beyond the int32 indptr, bad mode
    assert L.tg_project_packed_count(None, None) == -1
    pa = B.ProjectPackedArgs()
    pa.C, pa.N = 70_000, 10
    assert L.tg_project_packed_count(ctypes.byref(pa), None) == -2
    pa.C = 2
    assert L.tg_project_packed_count(ctypes.byref(pa), None) == -1 and b"workspace" in L.tg_last_error()
    buf = ctypes.create_string_buffer(256)
    pa.workspace = pa.nnz = pa.indptr = ctypes.cast(buf, ctypes.c_void_p)
    pa.N, pa.nnz_host = 0, 1 << 31
    assert L.tg_project_packed_emit(ctypes.byref(pa), None) == -2
    pb = B.ProjectPackedBwdArgs()
    pb.mode = 3
    assert L.tg_project_packed_bwd(ctypes.byref(pb), None) == -1
    assert L.tg_project_packed_workspace_bytes(4, 1 << 20) >= 8 * 4 * ((1 << 20) // 4096)


def test_product_path_fails_loudly_without_cuda():
    import torch

    from textured_gaussians_b200.cuda import isect_offset_encode

    if torch.cuda.is_available():
        pytest.skip("CUDA present")
    with pytest.raises(RuntimeError, match="CUDA"):
        isect_offset_encode(torch.zeros(4, dtype=torch.int64), 1, 2, 2)


def test_filter_arguments_are_rejected_without_a_device():
    """The mipmapped2 / anisotropic_bilinear checks run before any device work (host pointers stand in for
    device buffers: nothing is dereferenced before the checks fail)."""
    L = B.lib()
    buf = (ctypes.c_float * 4096)()
    p = ctypes.cast(buf, ctypes.c_void_p)

    def base():
        a = B.RasterFwdArgs()
        a.C, a.N, a.D, a.width, a.height, a.tile_size, a.tile_width, a.tile_height = 1, 4, 3, 16, 16, 16, 1, 1
        a.n_isects = 0
        a.means2d = a.ray_transforms = a.colors = a.opacities = a.normals = a.tile_offsets = p
        a.tex_format, a.textures, a.tex_ry, a.tex_rx, a.range_x, a.range_y = B.TG_TEX_F32, p, 8, 8, 3.0, 3.0
        return a

    def rejected(a, code, text):
        assert L.tg_rasterize_fwd(ctypes.byref(a), None) == code
        assert text in L.tg_last_error(), L.tg_last_error()

    a = base()
    a.mip_levels = 14
    rejected(a, -1, b"mip_levels")
    a = base()
    a.mip_levels = 2  # textures 8 x 8 are 2^3, not 2^2
    a.tex_coarse = p
    rejected(a, -1, b"2^L x 2^L")
    a = base()
    a.mip_levels = 3
    rejected(a, -1, b"coarse pyramid")
    a.tex_coarse, a.tile_size, a.width, a.height = p, 32, 32, 32
    rejected(a, -2, b"tile 8 or 16")
    a = base()
    a.filter = 7
    rejected(a, -1, b"unknown filter")
    a = base()
    a.filter = B.TG_FILTER_MIPMAPPED2
    rejected(a, -1, b"needs mip_levels")
    a = base()
    a.filter, a.tex_format, a.tex_scales = B.TG_FILTER_ANISO_BILINEAR, B.TG_TEX_FP8_E4M3, p
    rejected(a, -2, b"FP32 and BF16")
    a = base()
    a.filter, a.mip_levels, a.tex_coarse = B.TG_FILTER_ANISO_BILINEAR, 3, p
    rejected(a, -1, b"no mip levels")
    a = base()
    a.filter, a.work_queue = B.TG_FILTER_ANISO_BILINEAR, p
    rejected(a, -2, b"one CTA per tile")
    # pyramid entry points: level count out of range
    assert L.tg_generate_mipmap(p, p, 1, 0, None) == -1
    assert L.tg_generate_mipmap(p, p, 1, 14, None) == -1
    assert L.tg_generate_mipmap_bwd(p, p, 1, 14, None) == -1
    assert L.tg_generate_mipmap(p, p, 0, 3, None) == 0  # no textures: nothing to do
