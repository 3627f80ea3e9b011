"""CUDA-graph capture of forward + backward (textured_gaussians_b200.graph).

A captured step must give what the eager step gives on the same inputs:
rendered images bit for bit (capacity-sized intersection buffers change
nothing but the unused, padded tail), gradients within 1e-6 relative (float
atomics), for the drop-in and for the batching form, after the inputs are
updated in place between replays, and it must report -- not silently
truncate -- a replay that needs more intersections than were captured.
"""
import numpy as np
import pytest
import torch

from tests._util import rel_l2, to_np
from textured_gaussians_b200 import rasterization_textured_gaussians, scenes
from textured_gaussians_b200.batch import ViewTable, rasterization_textured_gaussians_batch
from textured_gaussians_b200.graph import GraphedStep

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def T(x):
    return torch.from_numpy(np.ascontiguousarray(x)).to(DEV, torch.float32)


class DropInStep:
    """Static inputs + one render / loss / backward of the drop-in."""

    def __init__(self, seed=7, n_cams=3):
        s = scenes.tiny(seed=seed, N=400, n_cams=n_cams)
        self.s = s
        self.leaves = [T(x).requires_grad_() for x in (s.means, s.quats, s.scales, s.opacities, s.colors,
                                                        s.textures)]
        self.V, self.K = T(s.viewmats), T(s.Ks)
        rng = np.random.default_rng(1)
        self.w = T(rng.normal(size=(n_cams, s.height, s.width, 3)))

    def __call__(self):
        for t in self.leaves:
            t.grad = None
        out = rasterization_textured_gaussians(*self.leaves, self.V, self.K, self.s.width, self.s.height,
                                               sh_degree=0, far_plane=100.0)
        loss = (out[0] * self.w).sum()
        loss.backward()
        return out[0].detach(), out[1].detach(), loss.detach()

    def grads(self):
        return [t.grad.clone() for t in self.leaves]


def _eager(step):
    img, alpha, loss = step()
    return img.clone(), alpha.clone(), loss.clone(), step.grads()


def _check(replayed, eager, grads_now):
    img, alpha, loss = replayed
    e_img, e_alpha, e_loss, e_grads = eager
    assert torch.equal(img, e_img) and torch.equal(alpha, e_alpha)
    assert abs(float(loss) - float(e_loss)) <= 1e-5 * max(1.0, abs(float(e_loss)))
    for a, b in zip(grads_now, e_grads):
        assert rel_l2(to_np(a), to_np(b)) < 1e-6


def test_graph_replay_matches_eager_and_follows_inputs():
    step = DropInStep()
    eager = _eager(step)
    g = GraphedStep(step)
    assert len(g.sizes) == 1 and g.capacities[0] >= g.sizes[0]
    _check(g.replay(), eager, step.grads())
    assert not g.overflowed()
    # update the inputs in place: the replay follows them
    with torch.no_grad():
        step.leaves[0].add_(0.01)
        step.leaves[5].mul_(0.9)
    out = tuple(t.clone() for t in g.replay())
    grads = step.grads()
    assert not g.overflowed()
    _check(out, _eager(step), grads)


def test_graph_overflow_is_reported_and_recapture_fixes_it():
    step = DropInStep(seed=8)
    g = GraphedStep(step, slack=1.0, floor=0)
    with torch.no_grad():
        step.leaves[2].mul_(2.5)  # larger splats: more tiles each than the captured capacity holds
    g.replay()
    assert g.overflowed()
    g.recapture()
    out = tuple(t.clone() for t in g.replay())
    grads = step.grads()
    assert not g.overflowed()
    _check(out, _eager(step), grads)


SIZES = [(64, 48), (40, 30), (80, 60), (33, 21)]


class BatchStep:
    def __init__(self):
        parts = [scenes.tiny(seed=s, N=n) for s, n in ((21, 250), (22, 400))]
        self.offs = np.cumsum([0] + [p.means.shape[0] for p in parts]).tolist()
        cat = {k: np.concatenate([getattr(p, k) for p in parts]) for k in
               ("means", "quats", "scales", "opacities", "colors", "textures")}
        self.leaves = [T(cat[k]).requires_grad_() for k in ("means", "quats", "scales", "opacities", "colors",
                                                              "textures")]
        dirs = scenes.fibonacci_dirs(len(SIZES))
        self.V = T(np.stack([scenes.look_at(4.0 * d) for d in dirs]))
        self.K = T(np.stack([scenes.intrinsics(0.9 * w, w / 2, h / 2) for w, h in SIZES]))
        self.vt = ViewTable([w for w, _ in SIZES], [h for _, h in SIZES], 16, DEV)
        self.vs = [c % 2 for c in range(len(SIZES))]
        rng = np.random.default_rng(2)
        self.w = T(rng.normal(size=(self.vt.n_pixels, 3)))

    def __call__(self):
        for t in self.leaves:
            t.grad = None
        out = rasterization_textured_gaussians_batch(*self.leaves, self.offs, self.V, self.K, self.vt.widths,
                                                     self.vt.heights, self.vs, sh_degree=0, far_plane=100.0,
                                                     view_table=self.vt)
        flat = out[-1]["flat_colors"]
        loss = (flat * self.w).sum()
        loss.backward()
        return flat.detach(), out[-1]["flat_alphas"].detach(), loss.detach()

    def grads(self):
        return [t.grad.clone() for t in self.leaves]


def test_graph_batch_form_matches_eager():
    step = BatchStep()
    eager = _eager(step)
    g = GraphedStep(step)
    assert len(g.sizes) == 2  # packed entries, then intersections
    _check(g.replay(), eager, step.grads())
    assert not g.overflowed()
