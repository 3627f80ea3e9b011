"""GPU parity of the batching form: views of uneven size over several scenes
in one pass against one drop-in call per view.

Tolerances: compositor outputs bit-exact (the same per-entry arithmetic and
the same per-tile splat order as the per-view calls); world-space normals
within 1e-6 (the camera-to-world rotation is a separate torch op); gradients
and contribution sums within 1e-5 relative (float atomics add the views' terms
in a different order).
"""
import numpy as np
import pytest
import torch

from tests._util import rel_l2, to_np
from textured_gaussians_b200 import rasterization_2dgs, rasterization_textured_gaussians, scenes
from textured_gaussians_b200.batch import ViewTable, rasterization_textured_gaussians_batch

pytestmark = pytest.mark.gpu
DEV = "cuda:0"

SIZES = [(64, 48), (40, 30), (80, 60), (64, 48), (33, 21), (48, 64), (17, 95)]


def T(x):
    return torch.from_numpy(np.ascontiguousarray(x)).to(DEV, torch.float32)


def make_batch():
    parts = [scenes.tiny(seed=s, N=n) for s, n in ((11, 200), (12, 350), (13, 500))]
    offs = np.cumsum([0] + [p.means.shape[0] for p in parts]).tolist()
    cat = {k: np.concatenate([getattr(p, k) for p in parts]) for k in
           ("means", "quats", "scales", "opacities", "colors", "textures")}
    dirs = scenes.fibonacci_dirs(len(SIZES))
    V = np.stack([scenes.look_at(4.0 * d) for d in dirs]).astype(np.float32)
    K = np.stack([scenes.intrinsics(0.9 * w, w / 2, h / 2) for w, h in SIZES]).astype(np.float32)
    view_scenes = [i % 3 for i in range(len(SIZES))]
    return cat, offs, V, K, view_scenes


def leaves(cat):
    return {k: T(v).requires_grad_() for k, v in cat.items()}


def run_batch(cat, offs, V, K, vs, textured=True, mode="RGB", tile=16, order="heaviest_first", persistent=False):
    L = leaves(cat)
    out = rasterization_textured_gaussians_batch(
        L["means"], L["quats"], L["scales"], L["opacities"], L["colors"], L["textures"] if textured else None, offs,
        T(V), T(K), [w for w, _ in SIZES], [h for _, h in SIZES], vs, sh_degree=0, tile_size=tile, render_mode=mode,
        far_plane=100.0, tile_order=order, persistent=persistent)
    return out, L


def run_per_view(cat, offs, V, K, vs, textured=True, mode="RGB", tile=16):
    L = leaves(cat)
    outs = []
    for c, (w, h) in enumerate(SIZES):
        a, b = offs[vs[c]], offs[vs[c] + 1]
        args = [L[k][a:b] for k in ("means", "quats", "scales", "opacities", "colors")]
        if textured:
            o = rasterization_textured_gaussians(*args, L["textures"][a:b], T(V[c:c + 1]), T(K[c:c + 1]), w, h,
                                                 sh_degree=0, tile_size=tile, render_mode=mode, far_plane=100.0)
        else:
            o = rasterization_2dgs(*args, T(V[c:c + 1]), T(K[c:c + 1]), w, h, sh_degree=0, tile_size=tile,
                                   render_mode=mode, far_plane=100.0)
        outs.append(o)
    return outs, L


def loss_weights(shapes, seed=4):
    rng = np.random.default_rng(seed)
    return [T(rng.normal(size=s)) for s in shapes]


@pytest.mark.parametrize("textured,mode,tile,persistent", [(True, "RGB", 16, False), (True, "RGB+ED", 8, False),
                                                           (False, "RGB", 16, False), (True, "RGB", 8, True)])
def test_batch_matches_per_view_calls(textured, mode, tile, persistent):
    cat, offs, V, K, vs = make_batch()
    bo, bl = run_batch(cat, offs, V, K, vs, textured, mode, tile, persistent=persistent)
    po, pl = run_per_view(cat, offs, V, K, vs, textured, mode, tile)
    for c in range(len(SIZES)):
        ref = po[c]
        assert torch.equal(bo[0][c], ref[0][0]), ("colors", c)
        assert torch.equal(bo[1][c], ref[1][0]), ("alphas", c)
        # world normals: the same camera-space normals rotated by an einsum that may
        # group the three products differently for one view and for a batch of views
        assert torch.allclose(bo[2][c], ref[2][0], rtol=0, atol=1e-6), ("normals", c)
        assert torch.equal(bo[4][c], ref[4][0]), ("distort", c)
        assert torch.equal(bo[5][c], ref[5][0]), ("median", c)
        if mode == "RGB+ED":
            assert torch.allclose(bo[3][c], ref[3], rtol=0, atol=1e-5), ("normals from depth", c)
    # contribution statistics: per Gaussian, summed over the views of its scene
    N = cat["means"].shape[0]
    cs = torch.zeros(N, device=DEV)
    cc = torch.zeros(N, device=DEV)
    for c in range(len(SIZES)):
        a, b = offs[vs[c]], offs[vs[c] + 1]
        cs[a:b] += po[c][6]
        cc[a:b] += po[c][7]
    assert torch.allclose(bo[6], cs, rtol=1e-5, atol=1e-6) and torch.equal(bo[7], cc)
    # gradients of one loss over every view
    ws = loss_weights([tuple(x.shape) for x in bo[0]])
    sum((x * w).sum() for x, w in zip(bo[0], ws)).backward()
    sum((p[0][0] * w).sum() for p, w in zip(po, ws)).backward()
    names = ["means", "quats", "scales", "opacities", "colors"] + (["textures"] if textured else [])
    for k in names:
        r = rel_l2(to_np(bl[k].grad), to_np(pl[k].grad))
        assert r < 1e-5, (k, r)


def test_tile_order_does_not_change_results():
    cat, offs, V, K, vs = make_batch()
    a, _ = run_batch(cat, offs, V, K, vs, order="heaviest_first")
    b, _ = run_batch(cat, offs, V, K, vs, order="launch")
    for c in range(len(SIZES)):
        for i in (0, 1, 2, 4, 5):
            assert torch.equal(a[i][c], b[i][c]), (i, c)
    order = a[-1]["tile_order"]
    vt = a[-1]["view_table"]
    assert sorted(order.tolist()) == list(range(vt.n_tiles))
    off = a[-1]["isect_offsets"].long()
    counts = torch.diff(off, append=torch.tensor([a[-1]["flatten_ids"].numel()], device=DEV))
    taken = counts[order.long()]
    assert bool((taken[:-1] >= taken[1:]).all())  # heaviest first


def test_view_table_reuse_and_flat_layout():
    cat, offs, V, K, vs = make_batch()
    vt = ViewTable([w for w, _ in SIZES], [h for _, h in SIZES], 16, DEV)
    L = leaves(cat)
    out = rasterization_textured_gaussians_batch(
        L["means"], L["quats"], L["scales"], L["opacities"], L["colors"], L["textures"], offs, T(V), T(K),
        vt.widths, vt.heights, vs, sh_degree=0, far_plane=100.0, view_table=vt)
    flat = out[-1]["flat_colors"]
    assert flat.shape == (vt.n_pixels, 3)
    for c, img in enumerate(out[0]):
        assert img.data_ptr() == flat[vt.pix_base[c]:].data_ptr()
