"""depth_to_points / depth_to_normal (the RGB+D / RGB+ED post-processing of
the renderer) against the reference's own functions
(textured_gaussians/utils.py:81-168), imported from its install under
baseline/_ref where that exists, and against a plain restatement otherwise."""
import os
import sys

import numpy as np
import pytest
import torch

from textured_gaussians_b200 import utils as U

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _inputs(seed=0):
    g = torch.Generator().manual_seed(seed)
    d = torch.rand((2, 7, 9, 1), generator=g) + 1.0
    c2w = torch.eye(4).repeat(2, 1, 1)
    c2w[:, :3, :3] = torch.linalg.qr(torch.randn((2, 3, 3), generator=g))[0]
    c2w[:, :3, 3] = torch.randn((2, 3), generator=g)
    K = torch.tensor([[5.0, 0, 4], [0, 6, 3], [0, 0, 1]]).repeat(2, 1, 1)
    return d, c2w, K


def test_depth_to_normal_matches_a_restatement():
    d, c2w, K = _inputs()
    n = U.depth_to_normal(d, c2w, K).numpy()
    dn, cw, k = d.double().numpy(), c2w.double().numpy(), K.double().numpy()
    H, W = dn.shape[1:3]
    pts = np.zeros((2, H, W, 3))
    for b in range(2):
        for i in range(H):
            for j in range(W):
                ray = np.array([(j - k[b, 0, 2] + 0.5) / k[b, 0, 0], (i - k[b, 1, 2] + 0.5) / k[b, 1, 1], 1.0])
                pts[b, i, j] = cw[b, :3, 3] + dn[b, i, j, 0] * (cw[b, :3, :3] @ ray)
    ref = np.zeros_like(pts)
    for b in range(2):
        for i in range(1, H - 1):
            for j in range(1, W - 1):
                c = np.cross(pts[b, i + 1, j] - pts[b, i - 1, j], pts[b, i, j + 1] - pts[b, i, j - 1])
                ref[b, i, j] = c / np.linalg.norm(c)
    assert np.abs(n - ref).max() < 1e-5


def test_depth_to_normal_matches_the_reference():
    pkg = os.path.join(ROOT, "baseline", "_ref")
    if not os.path.isdir(os.path.join(pkg, "textured_gaussians")):
        pytest.skip("the reference is not installed under baseline/_ref")
    sys.path.append(pkg)
    from textured_gaussians.utils import depth_to_normal, depth_to_points

    for z in (True, False):
        d, c2w, K = _inputs(1)
        assert torch.equal(U.depth_to_points(d, c2w, K, z), depth_to_points(d, c2w, K, z))
        assert torch.equal(U.depth_to_normal(d, c2w, K, z), depth_to_normal(d, c2w, K, z))
    with pytest.raises(AssertionError):
        U.depth_to_normal(d[..., 0], c2w, K)
