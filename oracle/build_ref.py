"""Build recipe for the reference's own CUDA ops (test infrastructure only).

Compiles the UNMODIFIED reference kernels for the textured 2DGS path, straight
from the reference tree, into ``oracle/_ref/tgref*.so`` (a Python extension
module; ``oracle/_ref/`` is git-ignored, and the built module travels to the
GPU machine with the working tree).  Nothing in ``textured_gaussians_b200``
links or loads it: it exists to produce golden vectors and to time the
reference on the same GPU.

The reference's sources include ``<glm/glm.hpp>`` from an un-vendored, empty
git submodule (``textured_gaussians/cuda/csrc/third_party/glm``); the include
path puts ``oracle/glm_shim`` (a restatement of the small part of GLM's
documented API those kernels use) in its place.  Flags follow the reference's
own release build (``setup.py``: ``-O3 --use_fast_math``), for sm_100a only.

Sources compiled (paths inside the reference's project):
  textured_gaussians/cuda/csrc/compute_sh_{fwd,bwd}.cu
  textured_gaussians/cuda/csrc/fully_fused_projection_2dgs_{fwd,bwd}.cu
  textured_gaussians/cuda/csrc/isect_tiles.cu
  textured_gaussians/cuda/csrc/rasterize_to_pixels_2dgs_{fwd,bwd}.cu
  textured_gaussians/cuda/csrc/rasterize_to_pixels_textured_gaussians_2dgs_{fwd,bwd,bwd2}.cu
  textured_gaussians/cuda/csrc/generate_mipmap_{fwd,bwd}.cu
  textured_gaussians/cuda/csrc/rasterize_to_pixels_mip2_textured_gaussians_2dgs_{fwd,bwd}.cu
  textured_gaussians/cuda/csrc/rasterize_to_pixels_aniso_bilinear_textured_gaussians_2dgs_{fwd,bwd}.cu

Usage (in a tree where the reference is mounted; REFERENCE_ROOT overrides the
default location):  python oracle/build_ref.py
"""
from __future__ import annotations

import glob
import importlib.machinery
import importlib.util
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
SHIM = os.path.join(HERE, "glm_shim")
NAME = "tgref"

REF_SOURCES = [
    "compute_sh_fwd.cu",
    "compute_sh_bwd.cu",
    "fully_fused_projection_2dgs_fwd.cu",
    "fully_fused_projection_2dgs_bwd.cu",
    "isect_tiles.cu",
    "rasterize_to_pixels_2dgs_fwd.cu",
    "rasterize_to_pixels_2dgs_bwd.cu",
    "rasterize_to_pixels_textured_gaussians_2dgs_fwd.cu",
    "rasterize_to_pixels_textured_gaussians_2dgs_bwd.cu",
    "rasterize_to_pixels_textured_gaussians_2dgs_bwd2.cu",
    "generate_mipmap_fwd.cu",
    "generate_mipmap_bwd.cu",
    "rasterize_to_pixels_mip2_textured_gaussians_2dgs_fwd.cu",
    "rasterize_to_pixels_mip2_textured_gaussians_2dgs_bwd.cu",
    "rasterize_to_pixels_aniso_bilinear_textured_gaussians_2dgs_fwd.cu",
    "rasterize_to_pixels_aniso_bilinear_textured_gaussians_2dgs_bwd.cu",
]


def reference_root() -> str:
    return os.environ.get("REFERENCE_ROOT", "/root/reference")


def built_path() -> str | None:
    hits = sorted(glob.glob(os.path.join(OUT_DIR, NAME + "*.so")))
    return hits[0] if hits else None


def load():
    """Imports the built module from oracle/_ref without rebuilding (the
    reference tree need not exist where this runs).  Returns None if absent."""
    path = built_path()
    if path is None:
        return None
    import torch  # noqa: F401  (the module links against torch's libraries)

    loader = importlib.machinery.ExtensionFileLoader(NAME, path)
    spec = importlib.util.spec_from_file_location(NAME, path, loader=loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    return mod


def build(verbose: bool = False) -> str | None:
    """Compiles the module if the reference tree is present; returns its path
    (or None when the reference is not mounted and nothing was built)."""
    csrc = os.path.join(reference_root(), "textured_gaussians", "cuda", "csrc")
    if not os.path.isdir(csrc):
        return built_path()
    from torch.utils import cpp_extension

    os.makedirs(OUT_DIR, exist_ok=True)
    os.environ.setdefault("MAX_JOBS", str(max(1, min(16, os.cpu_count() or 1))))
    sources = [os.path.join(HERE, "ref_bind.cpp")] + [os.path.join(csrc, s) for s in REF_SOURCES]
    cpp_extension.load(
        name=NAME,
        sources=sources,
        extra_include_paths=[SHIM, csrc],
        extra_cflags=["-O3", "-Wno-sign-compare"],
        extra_cuda_cflags=["-O3", "--use_fast_math", "-gencode", "arch=compute_100a,code=sm_100a",
                           "--expt-relaxed-constexpr"],
        build_directory=OUT_DIR,
        with_cuda=True,
        is_python_module=True,
        verbose=verbose,
    )
    return built_path()


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
