"""The batching form at full size: three scenes of 200,000, 500,000 and
1,000,000 splats (32x32 RGBA textures, BF16 storage), 64 views of uneven
resolution drawn from {400x300, 800x600, 1297x840, 1600x1200}, forward and
adjoint of all views in one call (tile 8, batch depth 64, heaviest tiles
first) -- checked against the FP64 oracle on sampled tiles of two views of
every resolution.

The oracle gets each sampled view's own projection (the dense per-view
projection, whose entries equal the batch's packed ones bit for bit), the
BF16-stored textures as the compositor samples them, and upstream gradients
that are nonzero only on the sampled tiles.  Tolerances: colours and alphas
1e-5 absolute with the 1e-3 flip budget; texture and opacity gradients (summed
over the sampled views by the batch's atomics) 1e-4 relative L2, or 1.5x the
IEEE-FP32 oracle's own distance from FP64 where that is larger (pixels with
many contributors, where recovering transmittance by division leaves any FP32
evaluation that far from FP64).
"""
import numpy as np
import pytest
import torch

import bench
from oracle import oracle as O
from tests._util import assert_close, rel_l2, to_np
from textured_gaussians_b200.batch import ViewTable, rasterization_textured_gaussians_batch
from textured_gaussians_b200.cuda import (
    fully_fused_projection_2dgs,
    isect_offset_encode,
    isect_tiles,
    make_texture_storage,
    spherical_harmonics,
)

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
TILE, DEPTH = 8, 64


def T(x, dtype=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(x)).to(DEV, dtype)


def _sampled_views(sizes):
    """Two views of every resolution (the first two in view order)."""
    picks = []
    for res in bench.BATCH_SIZES:
        picks += [c for c, s in enumerate(sizes) if tuple(s) == tuple(res)][:2]
    return sorted(picks)


@pytest.fixture(scope="module")
def batch():
    cat, offs, V, K, sizes, vs = bench.make_batch_workload(n_views=64)
    dev = torch.device(DEV)
    N = offs[-1]
    tex32 = torch.cat([bench.gpu_textures(offs[s + 1] - offs[s], 32, dev, seed=4 + s) for s in range(len(offs) - 1)])
    store, _ = make_texture_storage(tex32, "bf16")
    widths, heights = [w for w, _ in sizes], [h for _, h in sizes]
    vt = ViewTable(widths, heights, TILE, dev)
    picks = _sampled_views(sizes)
    # upstream gradients: nonzero only on every 10th tile of the middle tile row of each sampled view
    rng = np.random.default_rng(44)
    up = np.zeros((vt.n_pixels, 4), np.float32)
    masks = {}
    for c in picks:
        w, h = sizes[c]
        tw, th = -(-w // TILE), -(-h // TILE)
        m = np.zeros((1, th, tw), np.uint8)
        m[0, th // 2, ::10] = 1
        masks[c] = m
        pix = np.repeat(np.repeat(m, TILE, 1), TILE, 2)[0, :h, :w].reshape(-1)
        base = vt.pix_base[c]
        up[base:base + w * h] = rng.normal(size=(w * h, 4)).astype(np.float32) * pix[:, None]
    leaves = {k: T(v).requires_grad_() for k, v in cat.items()}
    tex = tex32.detach().clone().requires_grad_()
    out = rasterization_textured_gaussians_batch(
        leaves["means"], leaves["quats"], leaves["scales"], leaves["opacities"], leaves["colors"], tex, offs,
        T(V), T(K), widths, heights, vs, sh_degree=0, far_plane=100.0, tile_size=TILE, texture_storage=store,
        tile_order="heaviest_first", view_table=vt, batch_depth=DEPTH)
    meta = out[-1]
    upt = T(up)
    ((meta["flat_colors"] * upt[:, :3]).sum() + (meta["flat_alphas"] * upt[:, 3:]).sum()).backward()
    torch.cuda.synchronize()
    yield dict(cat=cat, offs=offs, V=V, K=K, sizes=sizes, vs=vs, vt=vt, picks=picks, masks=masks, up=up, store=store,
               flat_colors=to_np(meta["flat_colors"]), flat_alphas=to_np(meta["flat_alphas"]),
               v_tex=tex.grad, v_opac=to_np(leaves["opacities"].grad), N=N)
    del tex, tex32, store, leaves, out, meta
    torch.cuda.empty_cache()


def test_config4_batch_matches_the_oracle_on_sampled_tiles(batch):
    d = batch
    offs, vs = d["offs"], d["vs"]
    assert len(d["picks"]) == 8 and d["N"] == 1_700_000 and len(d["sizes"]) == 64
    # every sampled view against the FP64 (and IEEE-FP32) oracle on its own inputs
    rows_all, vtex64, vtex32 = [], [], []
    vop64, vop32 = np.zeros(d["N"]), np.zeros(d["N"])
    n_sel = 0
    for c in d["picks"]:
        w, h = d["sizes"][c]
        a, b = offs[vs[c]], offs[vs[c] + 1]
        n = b - a
        cat = {k: v[a:b] for k, v in d["cat"].items()}
        radii, m2d, dep, M, nrm = fully_fused_projection_2dgs(
            T(cat["means"]), T(cat["quats"]), T(cat["scales"]), T(d["V"][c:c + 1]), T(d["K"][c:c + 1]), w, h, 0.3,
            0.01, 100.0, 0.0)
        tw, th = -(-w // TILE), -(-h // TILE)
        _, ids, fl = isect_tiles(m2d, radii, dep, TILE, tw, th)
        off = isect_offset_encode(ids, 1, tw, th)
        cam = torch.linalg.inv(T(d["V"][c:c + 1]))[:, :3, 3]
        cols = torch.clamp_min(spherical_harmonics(0, T(cat["means"])[None] - cam[:, None], T(cat["colors"])[None],
                                                   masks=radii > 0) + 0.5, 0.0)
        mask = d["masks"][c]
        offn, fln = off.cpu().numpy().reshape(-1), fl.cpu().numpy()
        touched = [fln[offn[t]:(offn[t + 1] if t + 1 < offn.size else fln.size)] for t in np.flatnonzero(mask)]
        rows = np.unique(np.concatenate(touched))
        remap = np.zeros(n, np.int64)
        remap[rows] = np.arange(rows.size)
        tex_sub = d["store"][T(a + rows, torch.int64)].float().cpu().numpy()
        args = (to_np(m2d), to_np(M), to_np(cols), cat["opacities"][None], to_np(nrm), tex_sub, off.cpu().numpy(),
                fln, w, h, TILE)
        base = d["vt"].pix_base[c]
        up = d["up"][base:base + w * h].reshape(1, h, w, 4)
        z3, z1 = np.zeros((1, h, w, 3), np.float32), np.zeros((1, h, w, 1), np.float32)
        res = {}
        for dt in (np.float64, np.float32):
            kw = dict(masks=mask, gaussian_ids=remap, n_gauss=rows.size, dtype=dt)
            fo = O.raster_fwd(*args, **kw)
            res[dt] = (fo, O.raster_bwd(*args, fo, up[..., :3], up[..., 3:], z3, z1, z1, mode=0, **kw))
        fo, bo = res[np.float64]
        sel = np.repeat(np.repeat(mask, TILE, 1), TILE, 2)[0, :h, :w] > 0
        n_sel += int(sel.sum())
        got_c = d["flat_colors"][base:base + w * h].reshape(h, w, 3)
        got_a = d["flat_alphas"][base:base + w * h].reshape(h, w, 1)
        assert_close(got_c[sel], fo.colors[0][sel], 1e-5, 1e-5, 1e-3, f"view {c} ({w}x{h}) colors")
        assert_close(got_a[sel], fo.alphas[0][sel], 1e-5, 0.0, 1e-3, f"view {c} ({w}x{h}) alphas")
        rows_all.append(a + rows)
        vtex64.append((a + rows, res[np.float64][1].v_textures))
        vtex32.append((a + rows, res[np.float32][1].v_textures))
        vop64[a:b] += res[np.float64][1].v_opacities[0]
        vop32[a:b] += res[np.float32][1].v_opacities[0]
    assert n_sel >= 5_000
    # texture gradients: the oracle's per-view rows summed into the global rows
    rows = np.unique(np.concatenate(rows_all))
    pos = {int(r): i for i, r in enumerate(rows)}
    ref64 = np.zeros((rows.size, 32, 32, 4))
    ref32 = np.zeros((rows.size, 32, 32, 4))
    for (rr, v64), (_, v32) in zip(vtex64, vtex32):
        idx = np.array([pos[int(r)] for r in rr])
        np.add.at(ref64, idx, v64)
        np.add.at(ref32, idx, v32)
    got = d["v_tex"][T(rows, torch.int64)].cpu().numpy()
    bound = max(1e-4, 1.5 * rel_l2(ref32, ref64))
    assert rel_l2(got, ref64) < bound, ("textures", rel_l2(got, ref64), bound)
    bound = max(1e-4, 1.5 * rel_l2(vop32, vop64))
    assert rel_l2(d["v_opac"], vop64) < bound, ("opacities", rel_l2(d["v_opac"], vop64), bound)
    # no gradient reaches a texture no sampled tile touches
    untouched = torch.ones(d["N"], dtype=torch.bool, device=DEV)
    untouched[T(rows, torch.int64)] = False
    assert float(d["v_tex"][untouched].abs().max()) == 0.0
