"""Seeded synthetic scenes with the shapes and value distributions of the
benchmark workloads (there is no dataset on these machines).

Cameras use the OpenCV convention (x right, y down, z forward); a viewmat is
the world-to-camera [R | t; 0 0 0 1].  All arrays are numpy, FP32 unless
stated; callers move them to the GPU.

Workloads:
  small       seed 0, N=10,000, 8x8 textures, one 200x200 camera, SH degree 0
  views8      seed 1, N=300,000, 50x50 textures, eight 800x800 cameras, SH degree 3
  adjoint     seed 2, N=2,000, 16x16 textures, one 128x128 camera
  mixture1m   seed 3, N=1,000,000 from a 64-component mixture, 32x32 low-frequency
              textures, four 1600x1200 cameras
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np


@dataclass
class Scene:
    means: np.ndarray        # [N,3]
    quats: np.ndarray        # [N,4]
    scales: np.ndarray       # [N,3]
    opacities: np.ndarray    # [N] (post-sigmoid)
    colors: np.ndarray       # [N,K,3] SH coefficients (sh_degree set) or [N,3]
    textures: np.ndarray     # [N,R,R,4]
    viewmats: np.ndarray     # [C,4,4]
    Ks: np.ndarray           # [C,3,3]
    width: int
    height: int
    sh_degree: Optional[int]
    near_plane: float = 0.01
    far_plane: float = 1e10
    tile_size: int = 16
    backgrounds: Optional[np.ndarray] = None
    name: str = ""
    extra: dict = field(default_factory=dict)


def sigmoid(x):
    return 1.0 / (1.0 + np.exp(-x))


def look_at(center: np.ndarray, target=np.zeros(3)) -> np.ndarray:
    """World-to-camera matrix of a camera at `center` looking at `target`."""
    f = target - center
    f = f / np.linalg.norm(f)
    up = np.array([0.0, 0.0, 1.0])
    if abs(np.dot(f, up)) > 0.999:
        up = np.array([0.0, 1.0, 0.0])
    x = np.cross(f, up)
    x /= np.linalg.norm(x)
    y = np.cross(f, x)
    R = np.stack([x, y, f], 0)
    V = np.eye(4)
    V[:3, :3] = R
    V[:3, 3] = -R @ center
    return V


def fibonacci_dirs(n: int) -> np.ndarray:
    i = np.arange(n) + 0.5
    y = 1.0 - 2.0 * i / n
    r = np.sqrt(np.maximum(0.0, 1.0 - y * y))
    phi = i * np.pi * (3.0 - np.sqrt(5.0))
    return np.stack([np.cos(phi) * r, y, np.sin(phi) * r], -1)


def intrinsics(f: float, cx: float, cy: float) -> np.ndarray:
    return np.array([[f, 0, cx], [0, f, cy], [0, 0, 1]], np.float64)


def _gaussians(rng, N, log_scale_mu, log_scale_sd, opac_mu=0.0):
    ls = rng.normal(log_scale_mu, log_scale_sd, size=(N, 2))
    scales = np.exp(np.concatenate([ls, ls[:, 1:2]], 1))
    q = rng.normal(size=(N, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    opac = sigmoid(rng.normal(opac_mu, 1.0, size=N))
    return scales, q, opac


def dct_textures(rng, N, R, n_basis=4, sd=0.3):
    """0.5 + low-frequency cosine content (n_basis x n_basis DCT-II bases), clamped to [0,1]."""
    xs = np.arange(R)
    basis = np.cos(np.pi * (2 * xs[:, None] + 1) * np.arange(n_basis)[None, :] / (2 * R))  # [R, nb]
    out = np.empty((N, R, R, 4), np.float32)
    step = 65536
    for s in range(0, N, step):
        n = min(step, N - s)
        a = rng.normal(0, sd, size=(n, n_basis, n_basis, 4)).astype(np.float32)
        tex = 0.5 + np.einsum("yv,xu,nvuc->nyxc", basis, basis, a, optimize=True)
        out[s:s + n] = np.clip(tex, 0.0, 1.0)
    return out


def small(seed=0, N=10_000, R=8) -> Scene:
    rng = np.random.default_rng(seed)
    means = rng.uniform(-1, 1, size=(N, 3))
    scales, quats, opac = _gaussians(rng, N, -4.0, 0.5)
    colors = rng.uniform(0, 1, size=(N, 1, 3))
    textures = rng.uniform(0, 1, size=(N, R, R, 4))
    V = np.eye(4)
    V[2, 3] = 4.0
    return Scene(means.astype(np.float32), quats.astype(np.float32), scales.astype(np.float32),
                 opac.astype(np.float32), colors.astype(np.float32), textures.astype(np.float32),
                 V[None].astype(np.float32), intrinsics(200, 100, 100)[None].astype(np.float32), 200, 200, 0,
                 far_plane=100.0, backgrounds=np.ones((1, 3), np.float32), name="small")


def adjoint(seed=2, N=2_000, R=16) -> Scene:
    rng = np.random.default_rng(seed)
    means = rng.uniform(-1, 1, size=(N, 3))
    scales, quats, opac = _gaussians(rng, N, -4.0, 0.5)
    colors = rng.uniform(0, 1, size=(N, 1, 3))
    textures = rng.uniform(0, 1, size=(N, R, R, 4))
    V = np.eye(4)
    V[2, 3] = 4.0
    return Scene(means.astype(np.float32), quats.astype(np.float32), scales.astype(np.float32),
                 opac.astype(np.float32), colors.astype(np.float32), textures.astype(np.float32),
                 V[None].astype(np.float32), intrinsics(128, 64, 64)[None].astype(np.float32), 128, 128, 0,
                 far_plane=100.0, name="adjoint")


def views8(seed=1, N=300_000, R=50, n_cams=8, width=800, height=800, with_textures=True) -> Scene:
    """``with_textures=False`` leaves the 12 GB of uniform[0,1] textures to the caller (textures None,
    ``extra["texture_res"]`` = R), e.g. to draw them on the GPU."""
    rng = np.random.default_rng(seed)
    means = rng.uniform(-1, 1, size=(N, 3))
    scales, quats, opac = _gaussians(rng, N, -4.0, 0.5)
    sh = np.concatenate([rng.uniform(0, 1, size=(N, 1, 3)), rng.normal(0, 0.05, size=(N, 15, 3))], 1)
    textures = rng.uniform(0, 1, size=(N, R, R, 4)).astype(np.float32) if with_textures else None
    dirs = fibonacci_dirs(n_cams)
    V = np.stack([look_at(4.0 * d) for d in dirs])
    K = np.stack([intrinsics(1111, width / 2, height / 2)] * n_cams)
    return Scene(means.astype(np.float32), quats.astype(np.float32), scales.astype(np.float32),
                 opac.astype(np.float32), sh.astype(np.float32), textures, V.astype(np.float32),
                 K.astype(np.float32), width, height, 3, name="views8", extra={"texture_res": R})


def mixture1m(seed=3, N=1_000_000, R=32, n_cams=4, width=1600, height=1200, radius=25.0) -> Scene:
    rng = np.random.default_rng(seed)
    n_comp = 64
    u = rng.normal(size=(n_comp, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    centres = u * (10.0 * rng.uniform(0, 1, size=(n_comp, 1)) ** (1.0 / 3.0))
    comp = rng.integers(0, n_comp, size=N)
    means = centres[comp] + rng.normal(0, 0.5, size=(N, 3))
    scales, quats, opac = _gaussians(rng, N, -3.5, 0.6, opac_mu=0.5)
    colors = rng.uniform(0, 1, size=(N, 1, 3))
    textures = dct_textures(rng, N, R)
    dirs = fibonacci_dirs(n_cams)
    V = np.stack([look_at(radius * d) for d in dirs])
    K = np.stack([intrinsics(1200, width / 2, height / 2)] * n_cams)
    return Scene(means.astype(np.float32), quats.astype(np.float32), scales.astype(np.float32),
                 opac.astype(np.float32), colors.astype(np.float32), textures, V.astype(np.float32),
                 K.astype(np.float32), width, height, 0, far_plane=100.0, name="mixture1m",
                 extra={"camera_radius": radius})


def tiny(seed=5, N=300, R=8, width=64, height=48, n_cams=1) -> Scene:
    """A few hundred splats for fast parity / edge-case tests."""
    rng = np.random.default_rng(seed)
    means = rng.uniform(-1, 1, size=(N, 3))
    scales, quats, opac = _gaussians(rng, N, -2.5, 0.5)
    colors = rng.uniform(0, 1, size=(N, 1, 3))
    textures = rng.uniform(0, 1, size=(N, R, R, 4))
    if n_cams == 1:
        V = np.eye(4)[None]
        V[0, 2, 3] = 4.0
    else:
        V = np.stack([look_at(4.0 * d) for d in fibonacci_dirs(n_cams)])
    K = np.stack([intrinsics(60, width / 2, height / 2)] * n_cams)
    return Scene(means.astype(np.float32), quats.astype(np.float32), scales.astype(np.float32),
                 opac.astype(np.float32), colors.astype(np.float32), textures.astype(np.float32),
                 V.astype(np.float32), K.astype(np.float32), width, height, 0, far_plane=100.0, name="tiny")
