"""ctypes binding of libtg2dgs.so, the C ABI declared in include/tg2dgs.h.

The library is built in-tree by textured_gaussians_b200/build.py.  There is no
fallback: if the library is missing or fails to load, every op raises.  All
calls enqueue on torch's current CUDA stream of the tensors' device.
"""
from __future__ import annotations

import ctypes
import os
import threading

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtg2dgs.so")

TG_TEX_NONE, TG_TEX_F32, TG_TEX_BF16, TG_TEX_F16, TG_TEX_FP8_E4M3 = 0, 1, 2, 3, 4
TG_ADJ_REFERENCE, TG_ADJ_BWD2, TG_ADJ_EXACT = 0, 1, 2
TG_FILTER_BILINEAR, TG_FILTER_MIPMAPPED2, TG_FILTER_ANISO_BILINEAR = 0, 1, 2
_ERRORS = {-1: "invalid argument", -2: "unsupported", -3: "CUDA error", -4: "workspace too small",
           -5: "device wait timed out"}

P = ctypes.c_void_p
I32 = ctypes.c_int32
I64 = ctypes.c_int64
F32 = ctypes.c_float


class ProjectFwdArgs(ctypes.Structure):
    _fields_ = [("C", I32), ("N", I32), ("means", P), ("quats", P), ("scales", P), ("viewmats", P), ("Ks", P),
                ("width", I32), ("height", I32), ("near_plane", F32), ("far_plane", F32), ("radius_clip", F32),
                ("radii", P), ("means2d", P), ("depths", P), ("ray_transforms", P), ("normals", P),
                ("sh_degree", I32), ("sh_K", I32), ("sh_coeffs", P), ("colors", P)]


class ProjectBwdArgs(ctypes.Structure):
    _fields_ = [("C", I32), ("N", I32), ("means", P), ("quats", P), ("scales", P), ("viewmats", P), ("Ks", P),
                ("radii", P), ("ray_transforms", P), ("v_means2d", P), ("v_depths", P), ("v_normals", P),
                ("v_ray_transforms", P), ("mode", I32), ("v_means", P), ("v_quats", P), ("v_scales", P),
                ("sh_degree", I32), ("sh_K", I32), ("sh_coeffs", P), ("v_colors", P), ("v_sh_coeffs", P)]


class ProjectPackedArgs(ctypes.Structure):
    _fields_ = [("C", I32), ("N", I32), ("means", P), ("quats", P), ("scales", P), ("viewmats", P), ("Ks", P),
                ("width", I32), ("height", I32), ("near_plane", F32), ("far_plane", F32), ("radius_clip", F32),
                ("workspace", P), ("nnz", P), ("indptr", P), ("nnz_host", I64), ("camera_ids", P),
                ("gaussian_ids", P), ("radii", P), ("means2d", P), ("depths", P), ("ray_transforms", P),
                ("normals", P), ("views", P), ("gauss_ranges", P), ("max_range", I32), ("overflow", P),
                ("sh_degree", I32), ("sh_K", I32), ("sh_coeffs", P), ("colors", P)]


class ProjectPackedBwdArgs(ctypes.Structure):
    _fields_ = [("C", I32), ("N", I32), ("nnz", I64), ("means", P), ("quats", P), ("scales", P), ("viewmats", P),
                ("Ks", P), ("camera_ids", P), ("gaussian_ids", P), ("ray_transforms", P), ("v_means2d", P),
                ("v_depths", P), ("v_normals", P), ("v_ray_transforms", P), ("mode", I32), ("sparse_grad", I32),
                ("v_means", P), ("v_quats", P), ("v_scales", P), ("sh_degree", I32), ("sh_K", I32),
                ("sh_coeffs", P), ("v_colors", P), ("v_sh_coeffs", P)]


class DensifyStatsArgs(ctypes.Structure):
    _fields_ = [("C", I32), ("N", I64), ("n_elems", I64), ("grads2d", P), ("radii", P), ("gaussian_ids", P),
                ("width", I32), ("height", I32), ("grad2d", P), ("count", P), ("max_radii", P)]


class IsectArgs(ctypes.Structure):
    _fields_ = [("n_elems", I64), ("N", I64), ("camera_ids", P), ("means2d", P), ("radii", P), ("depths", P),
                ("tile_size", I32), ("tile_width", I32), ("tile_height", I32), ("n_cameras", I32),
                ("tiles_per_gauss", P), ("cum_tiles", P), ("n_isects", P), ("scan_workspace", P),
                ("isect_ids", P), ("flatten_ids", P), ("views", P), ("capacity", I64), ("overflow", P)]


class RasterFwdArgs(ctypes.Structure):
    _fields_ = [("C", I32), ("N", I32), ("D", I32), ("width", I32), ("height", I32), ("tile_size", I32),
                ("tile_width", I32), ("tile_height", I32), ("n_isects", I64), ("means2d", P),
                ("ray_transforms", P), ("colors", P), ("opacities", P), ("normals", P), ("tex_format", I32),
                ("textures", P), ("tex_scales", P), ("tex_ry", I32), ("tex_rx", I32), ("range_x", F32),
                ("range_y", F32), ("backgrounds", P), ("masks", P), ("tile_offsets", P), ("flatten_ids", P),
                ("gaussian_ids", P), ("contrib_threshold", F32), ("g_weight", F32), ("n_contrib", I32),
                ("out_colors", P), ("out_alphas", P), ("out_normals", P), ("out_distort", P), ("out_median", P),
                ("last_ids", P), ("median_ids", P), ("contrib_sum", P), ("contrib_count", P), ("tile_order", P),
                ("views", P), ("tile_view", P), ("n_tiles", I64), ("n_pixels", I64), ("n_isects_dev", P),
                ("batch_depth", I32), ("work_queue", P), ("mip_levels", I32), ("tex_coarse", P),
                ("filter", I32), ("t_checkpoints", P), ("aniso_prefix", P),
                ("aniso_records", P), ("aniso_record_count", P), ("aniso_record_cap", I32)]


class RasterBwdArgs(ctypes.Structure):
    _fields_ = [("f", RasterFwdArgs), ("render_colors", P), ("render_alphas", P), ("last_ids", P),
                ("median_ids", P), ("v_render_colors", P), ("v_render_alphas", P), ("v_render_normals", P),
                ("v_render_distort", P), ("v_render_median", P), ("adjoint", I32), ("n_elems", I64),
                ("v_means2d", P), ("v_means2d_abs", P), ("v_ray_transforms", P), ("v_colors", P),
                ("v_opacities", P), ("v_normals", P), ("v_textures", P), ("v_densify", P), ("v_tex_coarse", P),
                ("v_aniso_prefix", P)]


_lib = None
_lock = threading.Lock()


def lib() -> ctypes.CDLL:
    """Load libtg2dgs.so (once).  Raises if it is missing: there is no CPU fallback."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"{LIB_PATH} is missing; build it with `python textured_gaussians_b200/build.py` "
                    "(this package has no CPU fallback)")
            L = ctypes.CDLL(LIB_PATH)
            L.tg_version.restype = ctypes.c_int
            L.tg_last_error.restype = ctypes.c_char_p
            for name, argt in [
                ("tg_project_fwd", [ctypes.POINTER(ProjectFwdArgs), P]),
                ("tg_project_bwd", [ctypes.POINTER(ProjectBwdArgs), P]),
                ("tg_project_packed_count", [ctypes.POINTER(ProjectPackedArgs), P]),
                ("tg_project_packed_emit", [ctypes.POINTER(ProjectPackedArgs), P]),
                ("tg_project_packed_bwd", [ctypes.POINTER(ProjectPackedBwdArgs), P]),
                ("tg_isect_count", [ctypes.POINTER(IsectArgs), P]),
                ("tg_isect_emit", [ctypes.POINTER(IsectArgs), P]),
                ("tg_sort_pairs", [P, P, P, P, I64, I32, P, ctypes.c_size_t, ctypes.POINTER(I32), P]),
                ("tg_sort_status", [P, I64, I32, P]),
                ("tg_sort_lookback_selftest", [P, P, P, P, P, ctypes.c_size_t, P]),
                ("tg_isect_offset_encode", [P, I64, I32, I32, I32, P, P]),
                ("tg_isect_offset_encode_views", [P, I64, I32, I64, P, P, I64, P, P]),
                ("tg_rasterize_fwd", [ctypes.POINTER(RasterFwdArgs), P]),
                ("tg_rasterize_bwd", [ctypes.POINTER(RasterBwdArgs), P]),
                ("tg_sh_fwd", [I64, I64, I32, I32, P, P, P, P, P]),
                ("tg_selective_adam", [P, P, P, P, P, F32, F32, F32, F32, I64, I64, I32, P, P]),
                ("tg_densify_stats", [ctypes.POINTER(DensifyStatsArgs), P]),
                ("tg_generate_mipmap", [P, P, I64, I32, P]),
                ("tg_generate_mipmap_bwd", [P, P, I64, I32, P]),
                ("tg_aniso_prefix", [P, I32, P, I64, I32, I32, P, P]),
                ("tg_sh_bwd", [I64, I64, I32, I32, P, P, P, P, P, P, P]),
            ]:
                fn = getattr(L, name)
                fn.argtypes = argt
                fn.restype = ctypes.c_int
            L.tg_kernel_launch_count.restype = ctypes.c_uint64
            L.tg_kernel_launch_count.argtypes = []
            for name in ("tg_scan_workspace_bytes", "tg_sort_workspace_bytes", "tg_project_packed_workspace_bytes"):
                getattr(L, name).restype = ctypes.c_size_t
            L.tg_project_packed_workspace_bytes.argtypes = [I32, I32]
            L.tg_scan_workspace_bytes.argtypes = [I64]
            L.tg_sort_workspace_bytes.argtypes = [I64, I32]
            _lib = L
    return _lib


class StageTimers:
    """CUDA-event timers around every C-ABI call, on the stream the call uses.

    Disabled by default (zero cost).  ``enable()`` starts recording; each
    entry point's (start, end) event pair is kept per name; ``summary()``
    synchronises and returns {name: [ms per call]}.
    """

    def __init__(self):
        self.on = False
        self.events = {}

    def enable(self, on: bool = True):
        self.on = on
        self.events = {}

    def record(self, name: str, stream_handle: int):
        if not self.on:
            return None
        s = torch.cuda.ExternalStream(stream_handle)
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(s)
        return (name, ev, s)

    def close(self, tok):
        if tok is None:
            return
        name, start, s = tok
        end = torch.cuda.Event(enable_timing=True)
        end.record(s)
        self.events.setdefault(name, []).append((start, end))

    def summary(self):
        torch.cuda.synchronize()
        return {k: [a.elapsed_time(b) for a, b in v] for k, v in self.events.items()}


TIMERS = StageTimers()


def call(name: str, stream_handle: int, fn, *args) -> None:
    """Invoke a C-ABI entry point, raising on a nonzero status; timed when TIMERS is on."""
    tok = TIMERS.record(name, stream_handle) if TIMERS.on else None
    rc = fn(*args)
    if tok is not None:
        TIMERS.close(tok)
    check(rc, name)


def check(rc: int, what: str) -> None:
    if rc != 0:
        msg = lib().tg_last_error().decode(errors="replace")
        raise RuntimeError(f"{what} failed ({_ERRORS.get(rc, rc)}): {msg}")


def ptr(t) -> int | None:
    """Device pointer of a tensor (None for None)."""
    if t is None:
        return None
    return t.data_ptr()


def stream_of(t: torch.Tensor) -> int:
    if not t.is_cuda:
        raise RuntimeError("textured_gaussians_b200 ops need CUDA tensors (there is no CPU path)")
    return torch.cuda.current_stream(t.device).cuda_stream
