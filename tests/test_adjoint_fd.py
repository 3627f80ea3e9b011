"""FP64 central finite differences against the exact adjoint (CPU oracle).

Workload: 2,000 Gaussians with 16x16 textures, one 128x128 camera, loss
L = sum(w * colors), w ~ N(0,1) (the adjoint-check workload).  For each
parameter (means, quats, scales, opacity logits, SH coefficients, textures)
random coordinates of contributing splats are perturbed by +-h; a coordinate
is kept only when the per-pixel branch signature (alpha cut, 1e-4 stop,
2D/3D kernel choice, texture range and taps, alpha clamp), the radii and the
intersection list are identical at x+h and x-h, since the derivative is not
defined across those kinks.

The exact adjoint must agree with FD (cosine >= 0.999 per parameter and a
small median relative error); the reference adjoint is expected to differ
where it drops terms (texture-UV dependence, off-diagonal d means2d / d M).
"""
import numpy as np
import pytest

from oracle import pipeline as P
from textured_gaussians_b200 import scenes
from tests._util import cosine

F64 = np.float64
H_STEP = 1e-4


def _setup(n_coords, seed=2):
    s = scenes.adjoint(seed=seed)
    rng = np.random.default_rng(123)
    logits = np.log(s.opacities / (1 - s.opacities)).astype(F64)
    params = dict(means=s.means.astype(F64), quats=s.quats.astype(F64), scales=s.scales.astype(F64),
                  logits=logits, colors=s.colors.astype(F64), textures=s.textures.astype(F64))
    w = rng.normal(size=(1, s.height, s.width, 3))
    return s, params, w, rng


def _render(s, p):
    op = 1.0 / (1.0 + np.exp(-p["logits"]))
    rc, ra, rn, cache = P.render(p["means"], p["quats"], p["scales"], op, p["colors"], p["textures"], s.viewmats,
                                 s.Ks, s.width, s.height, sh_degree=0, far_plane=s.far_plane, dtype=F64)
    return rc, cache


def _signature(cache):
    return (cache.radii.tobytes(), cache.isect_ids.tobytes(), cache.fwd.branch_sig.tobytes())


def _analytic(s, p, w, raster_mode, proj_mode):
    rc, cache = _render(s, p)
    op = 1.0 / (1.0 + np.exp(-p["logits"]))
    g = P.render_backward(cache, p["means"], p["quats"], p["scales"], op, p["colors"], p["textures"], s.viewmats,
                          s.Ks, s.width, s.height, w, sh_degree=0, raster_mode=raster_mode, proj_mode=proj_mode)
    g["logits"] = g["opacities"] * op * (1 - op)
    return g, cache


def _fd_check(n_coords=25):
    s, p, w, rng = _setup(n_coords)
    exact, cache = _analytic(s, p, w, raster_mode=2, proj_mode=2)
    ref, _ = _analytic(s, p, w, raster_mode=0, proj_mode=0)
    visible = np.nonzero(cache.radii[0] > 0)[0]
    contributing = np.unique(cache.flatten_ids)
    live = np.intersect1d(visible, contributing)
    results = {}
    for name in ("means", "quats", "scales", "logits", "colors", "textures"):
        arr = p[name]
        fd, an, an_ref = [], [], []
        tries = 0
        while len(fd) < n_coords and tries < 20 * n_coords:
            tries += 1
            gi = int(rng.choice(live))
            if name == "scales":
                idx = (gi, int(rng.integers(0, 2)))
            elif name == "textures":
                idx = (gi,) + tuple(int(rng.integers(0, d)) for d in arr.shape[1:])
            else:
                idx = (gi,) + tuple(int(rng.integers(0, d)) for d in arr.shape[1:])
            if exact[name][idx] == 0 and name == "textures":
                continue
            x0 = arr[idx]
            sigs, Ls = [], []
            for sgn in (1, -1):
                arr[idx] = x0 + sgn * H_STEP
                rc, c = _render(s, p)
                sigs.append(_signature(c))
                Ls.append(float((rc * w).sum()))
            arr[idx] = x0
            if sigs[0] != sigs[1]:
                continue
            fd.append((Ls[0] - Ls[1]) / (2 * H_STEP))
            an.append(exact[name][idx])
            an_ref.append(ref[name][idx])
        results[name] = (np.array(fd), np.array(an), np.array(an_ref))
    return results


@pytest.fixture(scope="module")
def fd_results():
    return _fd_check()


@pytest.mark.parametrize("name", ["means", "quats", "scales", "logits", "colors", "textures"])
def test_exact_adjoint_matches_finite_differences(fd_results, name):
    fd, an, _ = fd_results[name]
    assert len(fd) >= 10, f"only {len(fd)} usable coordinates for {name}"
    assert cosine(an, fd) >= 0.999, (name, cosine(an, fd))
    rel = np.abs(an - fd) / (np.abs(fd) + np.abs(an) + 1e-6 * np.abs(fd).max())
    assert np.median(rel) < 1e-3, (name, np.median(rel))


def test_reference_adjoint_drops_geometry_terms(fd_results):
    # The reference "bilinear" adjoint ignores d(texture sample)/d(uv) and keeps only the diagonal of
    # d means2d / d M, so on geometry parameters it departs from the true derivative.
    fd, an, an_ref = fd_results["means"]
    assert cosine(an_ref, fd) < cosine(an, fd)
