"""GPU parity of the gradient consumers: selective Adam (with its fused BF16 /
FP16 shadow write) and the densification statistics.

Tolerances: Adam state and parameters within 2e-6 relative (+1e-7 of the
tensor's scale where the FP32 update cancels) of the FP64 oracle on the same
FP32 inputs and FP32 hyper-parameters; statistics: counts and radius maxima
exact, sums within 1e-5 relative (float atomics in the packed layout).
"""
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O
from textured_gaussians_b200 import rasterization_textured_gaussians, scenes
from textured_gaussians_b200.cuda import densify_stats, selective_adam_update
from textured_gaussians_b200.optimizers import SelectiveAdam
from textured_gaussians_b200.strategy import update_state

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def T(x, dtype=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(x)).to(DEV, dtype)


def _close(got, ref, rel=2e-6):
    """|got - ref| <= rel |ref| + 1e-7 max|ref|: relative, except where the FP32 update cancels (m = b1 m +
    (1-b1) g or p + step close to zero), where FP32 rounding at the inputs' scale is the floor."""
    got = got.detach().double().cpu().numpy()
    bound = rel * np.abs(ref) + 1e-7 * np.abs(ref).max()
    assert (np.abs(got - ref) <= bound).all(), np.max(np.abs(got - ref) / bound)


@pytest.mark.parametrize("shape,shadow", [((700, 16, 16, 4), None), ((700, 16, 16, 4), torch.bfloat16),
                                          ((700, 8, 8, 4), torch.float16), ((1001, 3), None),
                                          ((1001, 3), torch.bfloat16)])
def test_selective_adam_matches_oracle(shape, shadow):
    rng = np.random.default_rng(3)
    N = shape[0]
    M = int(np.prod(shape[1:]))
    p0 = rng.normal(size=shape).astype(np.float32)
    g = rng.normal(size=shape).astype(np.float32)
    m0 = rng.normal(size=shape).astype(np.float32) * 0.1
    v0 = rng.uniform(0, 0.1, size=shape).astype(np.float32)
    vis = rng.uniform(size=N) < 0.6
    p, m, v = T(p0), T(m0), T(v0)
    sh = None if shadow is None else torch.full(shape, -7.0, dtype=shadow, device=DEV)
    selective_adam_update(p, T(g), m, v, T(vis, torch.bool), 1e-3, 0.9, 0.999, 1e-15, N, M, shadow=sh)
    rp, rm, rv = O.selective_adam(p0, g, m0, v0, vis, 1e-3, 0.9, 0.999, 1e-15)
    _close(m, rm)
    _close(v, rv)
    _close(p, rp)
    hidden = ~T(vis, torch.bool)
    assert torch.equal(p[hidden], T(p0)[hidden])  # hidden rows untouched
    if sh is not None:
        assert torch.equal(sh[~hidden], p[~hidden].to(shadow))
        assert bool((sh[hidden] == -7.0).all())


def test_selective_adam_optimizer_two_steps():
    rng = np.random.default_rng(4)
    N, R = 300, 8
    tex0 = rng.uniform(0, 1, size=(N, R, R, 4)).astype(np.float32)
    tex = T(tex0).requires_grad_()
    store = tex.detach().to(torch.bfloat16)
    opt = SelectiveAdam([{"params": [tex], "lr": 1e-2}], eps=1e-15, betas=(0.9, 0.999), shadows={tex: store})
    p, m, v = tex0.astype(np.float64), np.zeros_like(tex0, np.float64), np.zeros_like(tex0, np.float64)
    for _ in range(2):
        g = rng.normal(size=tex0.shape).astype(np.float32)
        vis = rng.uniform(size=N) < 0.5
        tex.grad = T(g)
        opt.step(T(vis, torch.bool))
        p, m, v = O.selective_adam(p.astype(np.float32), g, m.astype(np.float32), v.astype(np.float32), vis, 1e-2,
                                   0.9, 0.999, 1e-15)
    _close(tex, p, 1e-5)
    # every row's shadow is the BF16 rounding of its current FP32 master (updated rows refreshed in the step)
    assert torch.equal(store, tex.detach().to(torch.bfloat16))


@pytest.mark.parametrize("tag,C", [("dense3", 3), ("dense1", 1), ("packed", 3)])
def test_densify_stats_match_reference_fixture(tag, C):
    d = np.load(os.path.join(GOLDEN, "densify_stats.npz"))
    W, H, N = int(d["width"]), int(d["height"]), int(d["N"])
    gid = d[f"{tag}_gaussian_ids"] if f"{tag}_gaussian_ids" in d.files else None
    grad2d = torch.zeros(N, device=DEV)
    count = torch.zeros(N, device=DEV)
    mr = torch.zeros(N, device=DEV)
    densify_stats(T(d[f"{tag}_grads"]), T(d[f"{tag}_radii"], torch.int32), W, H, C, grad2d, count, mr,
                  gaussian_ids=None if gid is None else T(gid, torch.int64))
    np.testing.assert_allclose(grad2d.cpu().numpy(), d[f"{tag}_grad2d"], rtol=1e-5, atol=1e-7)
    np.testing.assert_array_equal(count.cpu().numpy(), d[f"{tag}_count"])
    _, _, ref_mr = O.densify_stats(d[f"{tag}_grads"], d[f"{tag}_radii"], W, H, C, N, gaussian_ids=gid)
    np.testing.assert_array_equal(mr.cpu().numpy(), ref_mr)


@pytest.mark.parametrize("packed", [False, True])
def test_update_state_after_a_render(packed):
    s = scenes.tiny(seed=17, N=600, n_cams=3)
    L = [T(x).requires_grad_() for x in (s.means, s.quats, s.scales, s.opacities, s.colors, s.textures)]
    out = rasterization_textured_gaussians(*L, T(s.viewmats), T(s.Ks), s.width, s.height, sh_degree=0,
                                           far_plane=s.far_plane, packed=packed)
    meta = out[-1]
    rng = np.random.default_rng(1)
    (out[0] * T(rng.normal(size=tuple(out[0].shape)))).sum().backward()
    state = {"grad2d": None, "count": None, "radii": None}
    N = s.means.shape[0]
    update_state(state, meta, N, packed=packed, track_radii=True)
    update_state(state, meta, N, packed=packed, track_radii=True)  # accumulates
    g = meta["gradient_2dgs"].grad.cpu().numpy()
    gid = meta["gaussian_ids"].cpu().numpy() if packed else None
    r2, rc, rr = O.densify_stats(g, meta["radii"].cpu().numpy(), s.width, s.height, 3, N, gaussian_ids=gid)
    np.testing.assert_allclose(state["grad2d"].cpu().numpy(), 2 * r2, rtol=1e-5, atol=1e-9)
    np.testing.assert_array_equal(state["count"].cpu().numpy(), 2 * rc)
    np.testing.assert_array_equal(state["radii"].cpu().numpy(), rr)
