"""Loading the golden vectors the reference's own CUDA path produced
(tests/golden/ref_*.npz, written by tests/golden/make_ref_golden.py) and
rebuilding the inputs they were made from.

Each fixture holds the reference's outputs on one camera (C = 1) of a seeded
workload; the inputs are regenerated here from the same seeds and checked
against the SHA-256 digests stored beside the outputs.
"""
from __future__ import annotations

import copy
import hashlib
import os

import numpy as np

from textured_gaussians_b200 import scenes

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def path(case: str) -> str:
    return os.path.join(GOLDEN, f"ref_{case}.npz")


def load(case: str) -> dict:
    with np.load(path(case)) as z:
        return {k: z[k] for k in z.files}


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def upstream(seed: int, s) -> list:
    """The five per-pixel upstream gradients (colours, alphas, normals, distortion, median) of the fixture."""
    rng = np.random.default_rng(int(seed))
    H, W = s.height, s.width
    shapes = [(1, H, W, 3), (1, H, W, 1), (1, H, W, 3), (1, H, W, 1), (1, H, W, 1)]
    return [rng.normal(size=sh).astype(np.float32) for sh in shapes]


def proj_upstream(seed: int, C: int, N: int) -> list:
    """Upstream gradients of the projection's means2d, depths, ray transforms and normals (the fixture's)."""
    rng = np.random.default_rng(int(seed))
    return [rng.normal(size=sh).astype(np.float32) for sh in ((C, N, 2), (C, N), (C, N, 3, 3), (C, N, 3))]


def scene(case: str, g: dict):
    """The scene a small fixture was made from, verified against its input digest."""
    if case == "small":
        s = scenes.small()
    elif case in ("adjoint", "adjoint_aniso"):
        s = scenes.adjoint()
    else:
        raise KeyError(case)
    if case == "adjoint_aniso":
        rows = g["kept_rows"]
        s = copy.copy(s)
        for k in ("means", "quats", "scales", "opacities", "colors", "textures"):
            setattr(s, k, np.ascontiguousarray(getattr(s, k)[rows]))
    got = digest(s.means, s.quats, s.scales, s.opacities, s.colors, s.textures, s.viewmats, s.Ks)
    assert got == str(g["inputs_sha256"]), f"{case}: regenerated inputs differ from the fixture's"
    return s


def sampled_layout(g: dict, th: int, tw: int):
    """Offsets [1, th, tw] and flatten ids over the fixture's sub-rows for its sampled tiles only.

    The fixture stores each sampled tile's splat list (global Gaussian ids, C = 1); every other
    tile gets an empty range, so a render over the sub-rows reproduces the sampled tiles exactly."""
    rows, tiles, counts, lists = g["rows"], g["tiles"], g["tile_counts"], g["tile_lists"]
    sub = np.searchsorted(rows, lists).astype(np.int32)
    assert np.array_equal(rows[sub], lists)
    start = np.zeros(th * tw, np.int64)
    per_tile = np.zeros(th * tw, np.int64)
    per_tile[tiles] = counts
    start[1:] = np.cumsum(per_tile)[:-1]
    return start.reshape(1, th, tw).astype(np.int32), sub


def pixel_mask(g: dict, tile: int, th: int, tw: int, H: int, W: int):
    mask = np.zeros(th * tw, bool)
    mask[g["tiles"]] = True
    mask = mask.reshape(1, th, tw)
    return np.repeat(np.repeat(mask, tile, 1), tile, 2)[:, :H, :W]


def texture_rows_check(g: dict, prefix: str, v_tex: np.ndarray):
    """(rows kept, reference values, reference per-row norms) of a texture gradient, and ours on them."""
    rows = g[f"{prefix}__v_textures_rows"]
    return rows, g[f"{prefix}__v_textures_vals"], g[f"{prefix}__v_textures_norms"], v_tex[rows]
