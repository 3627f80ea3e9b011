"""Error of each texture storage form against the FP64 CPU oracle.

Workload: 30,000 splats from the 64-component mixture (the benchmark's
distribution), 32x32 low-frequency RGBA textures, one 800x600 camera, tile 16.
The GPU renders forward + exact adjoint with textures stored in FP32, BF16,
FP16 and FP8-E4M3 (per-Gaussian scale), FP32 arithmetic and FP32 gradient
accumulation; the oracle renders the same scene entirely in FP64 from the FP32
parameters.  Reported per form: image PSNR and max |error| of colours,
alphas and normals, and the cosine of every parameter gradient.

Thresholds: FP32 / FP16 >= 70 dB, BF16 >= 50 dB, FP8 >= 30 dB on colours;
gradient cosine >= 0.999 for FP32, FP16 and BF16, >= 0.98 for FP8 (its 3-bit
mantissa reaches the geometry gradients through the exact adjoint's texture-UV term).
"""
import json

import numpy as np
import pytest
import torch

from oracle import pipeline as P
from tests._util import cosine
from textured_gaussians_b200 import rasterization_textured_gaussians, scenes
from textured_gaussians_b200.cuda import make_texture_storage

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def psnr(a, b):
    mse = float(np.mean((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2))
    return float("inf") if mse == 0 else 10 * np.log10(1.0 / mse)


@pytest.fixture(scope="module")
def reference():
    s = scenes.mixture1m(N=30_000, n_cams=1, width=800, height=600)
    s.Ks[:, 0, 0] = s.Ks[:, 1, 1] = 600.0
    s.Ks[:, 0, 2], s.Ks[:, 1, 2] = 400.0, 300.0
    rng = np.random.default_rng(9)
    w = rng.normal(size=(1, s.height, s.width, 3))
    rc, ra, rn, cache = P.render(s.means, s.quats, s.scales, s.opacities, s.colors, s.textures, s.viewmats, s.Ks,
                                 s.width, s.height, sh_degree=0, far_plane=s.far_plane, dtype=np.float64)
    g = P.render_backward(cache, s.means, s.quats, s.scales, s.opacities, s.colors, s.textures, s.viewmats, s.Ks,
                          s.width, s.height, w, sh_degree=0, raster_mode=2, proj_mode=2)
    return s, w, (rc, ra, rn), g


@pytest.mark.parametrize("fmt,min_psnr,min_cos", [("fp32", 70, 0.999), ("fp16", 70, 0.999), ("bf16", 50, 0.999),
                                                  ("fp8", 30, 0.98)])
def test_texture_storage_error_vs_fp64_oracle(reference, fmt, min_psnr, min_cos):
    s, w, (rc, ra, rn), g = reference
    T = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(DEV)
    leaves = [T(x).requires_grad_() for x in (s.means, s.quats, s.scales, s.opacities, s.colors, s.textures)]
    store, scales = make_texture_storage(leaves[5].detach(), fmt)
    out = rasterization_textured_gaussians(*leaves, T(s.viewmats), T(s.Ks), s.width, s.height, sh_degree=0,
                                           far_plane=s.far_plane, filtering="bilinear_exact", adjoint="exact",
                                           texture_storage=None if fmt == "fp32" else store, texture_scales=scales)
    (out[0] * T(w.astype(np.float32))).sum().backward()
    row = {"form": fmt}
    for name, got, ref in (("colors", out[0], rc), ("alphas", out[1], ra), ("normals", out[2], rn)):
        got = got.detach().cpu().numpy()
        row[f"{name}_psnr_db"] = round(psnr(got, ref), 2)
        row[f"{name}_max_abs"] = float(np.abs(got - ref).max())
    for name, leaf in zip(("means", "quats", "scales", "opacities", "colors", "textures"), leaves):
        row[f"grad_cos_{name}"] = round(cosine(leaf.grad.cpu().numpy(), g[name]), 6)
    print("PRECISION", json.dumps(row))
    assert row["colors_psnr_db"] >= min_psnr, row
    for name in ("means", "quats", "scales", "opacities", "colors", "textures"):
        assert row[f"grad_cos_{name}"] >= min_cos, (name, row)
