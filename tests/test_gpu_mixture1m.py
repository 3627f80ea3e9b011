"""The benchmark workload at full size on the GPU -- 1,000,000 Gaussians from a
64-component mixture, 32x32 low-frequency RGBA textures, four 1600x1200
cameras, tile 8 -- against the oracle where it can follow at this size:

  * intersections, sorted keys, flatten ids and offsets of the four cameras:
    bit-exact against the oracle's on the same projected inputs;
  * the compositor forward and reference adjoint, with the textures stored in
    FP32, BF16, FP16 and FP8-E4M3 (per-Gaussian scale), against the FP64
    oracle on the FP32 textures, on a sample of 80 tiles (20 of one tile row
    per camera; the oracle's tile masks select them, the textures they touch
    are gathered on the GPU; upstream gradients are nonzero only there).
    FP32 storage: colours and alphas to 1e-5 with the 1e-3 flip budget,
    gradients to 1e-4 relative L2 (or 1.5x the IEEE-FP32 oracle's own error
    where that is larger).  Every form: render PSNR and gradient cosine are
    printed; BF16 and FP16 must reach 50 dB and 0.999, FP8 35 dB and 0.99;
  * the anisotropic_bilinear filter (FP32 storage) on the same sampled tiles,
    against the oracle's cell-by-cell footprint integration, at the FP32
    tolerances above.
"""
import numpy as np
import pytest
import torch

import bench
from oracle import oracle as O
from tests._util import assert_close, cosine, rel_l2, to_np
from textured_gaussians_b200.cuda import (
    fully_fused_projection_2dgs,
    isect_offset_encode,
    isect_tiles,
    make_texture_storage,
    rasterize_to_pixels_textured_gaussians,
)

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
TILE = 8
ROW = 75  # sampled tile row of every camera (of 150); every 10th tile of it


def T(x, dtype=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(x)).to(DEV, dtype)


@pytest.fixture(scope="module")
def mixture():
    sc = bench.make_scene(0, 1, 1_000_000, 4)
    N, C, W, H = 1_000_000, 4, sc["width"], sc["height"]
    tex = bench.gpu_textures(N, 32, torch.device(DEV))
    radii, means2d, depths, M, normals = fully_fused_projection_2dgs(
        T(sc["means"]), T(sc["quats"]), T(sc["scales"]), T(sc["viewmats"]), T(sc["Ks"]), W, H, 0.3, 0.01, 100.0,
        0.0)
    tw, th = -(-W // TILE), -(-H // TILE)
    tpg, ids, fl = isect_tiles(means2d, radii, depths, TILE, tw, th)
    off = isect_offset_encode(ids, C, tw, th)
    colors = T(np.broadcast_to(sc["colors"][:, 0][None], (C, N, 3)))
    opac = np.tile(sc["opacities"][None], (C, 1))
    yield dict(sc=sc, tex=tex, radii=radii, means2d=means2d, depths=depths, M=M, normals=normals, tpg=tpg, ids=ids,
               fl=fl, off=off, colors=colors, opac=opac, N=N, C=C, W=W, H=H, tw=tw, th=th)
    del tex
    torch.cuda.empty_cache()


def test_mixture1m_intersections_bit_exact(mixture):
    d = mixture
    o_tpg, o_ids, o_fl = O.isect_tiles(to_np(d["means2d"]), d["radii"].cpu().numpy(), to_np(d["depths"]), TILE,
                                       d["tw"], d["th"], d["C"])
    assert d["ids"].numel() > 20_000_000
    np.testing.assert_array_equal(d["tpg"].cpu().numpy(), o_tpg)
    np.testing.assert_array_equal(d["ids"].cpu().numpy(), o_ids)
    np.testing.assert_array_equal(d["fl"].cpu().numpy(), o_fl)
    np.testing.assert_array_equal(d["off"].cpu().numpy(), O.isect_offset_encode(o_ids, d["C"], d["tw"], d["th"]))


def _psnr(a, b):
    mse = float(np.mean((np.asarray(a, np.float64) - b) ** 2))
    return float("inf") if mse == 0 else 10.0 * np.log10(1.0 / mse)


@pytest.fixture(scope="module")
def sampled_oracle(mixture):
    d = mixture
    C, N, W, H, tw, th = d["C"], d["N"], d["W"], d["H"], d["tw"], d["th"]
    mask = np.zeros((C, th, tw), np.uint8)
    mask[:, ROW, ::10] = 1
    off = d["off"].cpu().numpy().reshape(-1)
    fl = d["fl"].cpu().numpy()
    touched = []
    for t in np.flatnonzero(mask.reshape(-1)):
        end = off[t + 1] if t + 1 < off.size else fl.size
        touched.append(fl[off[t]:end] % N)
    rows = np.unique(np.concatenate(touched))
    remap = np.zeros(N, np.int64)
    remap[rows] = np.arange(rows.size)
    gid = remap[np.arange(C * N) % N]
    pix = np.repeat(np.repeat(mask, TILE, 1), TILE, 2)[:, :H, :W].astype(np.float32)[..., None]
    rng = np.random.default_rng(4)
    up_c = rng.normal(size=(C, H, W, 3)).astype(np.float32) * pix
    up_a = rng.normal(size=(C, H, W, 1)).astype(np.float32) * pix
    tex_sub = d["tex"][T(rows, torch.int64)].cpu().numpy()
    args = (to_np(d["means2d"]), to_np(d["M"]), to_np(d["colors"]), d["opac"], to_np(d["normals"]), tex_sub,
            d["off"].cpu().numpy(), fl, W, H, TILE)
    z3, z1 = np.zeros((C, H, W, 3), np.float32), np.zeros((C, H, W, 1), np.float32)
    out = {}
    for dt in (np.float64, np.float32):
        kw = dict(masks=mask, gaussian_ids=gid, n_gauss=rows.size, dtype=dt)
        fo = O.raster_fwd(*args, **kw)
        out[dt] = (fo, O.raster_bwd(*args, fo, up_c, up_a, z3, z1, z1, mode=0, **kw))
    return dict(rows=rows, sel=pix[..., 0] > 0, up_c=up_c, up_a=up_a, ref=out[np.float64], ref32=out[np.float32])


@pytest.mark.parametrize("fmt", ["fp32", "bf16", "fp16", "fp8"])
def test_mixture1m_storage_forms_on_sampled_tiles(mixture, sampled_oracle, fmt):
    d, o = mixture, sampled_oracle
    assert o["sel"].sum() >= 5_000
    store, scales = make_texture_storage(d["tex"], fmt)
    m2d = d["means2d"].detach().clone().requires_grad_()
    M = d["M"].detach().clone().requires_grad_()
    cols = d["colors"].detach().clone().requires_grad_()
    op = T(d["opac"]).requires_grad_()
    tex = d["tex"].detach().requires_grad_()
    out = rasterize_to_pixels_textured_gaussians(
        m2d, M, cols, op, tex, 3.0, 3.0, d["normals"], torch.zeros_like(m2d), d["W"], d["H"], TILE, d["off"],
        d["fl"], texture_storage=None if fmt == "fp32" else store, texture_scales=scales)
    ((out[0] * T(o["up_c"])).sum() + (out[1] * T(o["up_a"])).sum()).backward()
    (fo, ob), (_, ob32) = o["ref"], o["ref32"]
    sel = o["sel"]
    rc, ra = to_np(out[0])[sel], to_np(out[1])[sel]
    grads = [("means2d", m2d.grad, ob.v_means2d, ob32.v_means2d), ("M", M.grad, ob.v_M, ob32.v_M),
             ("colors", cols.grad, ob.v_colors, ob32.v_colors), ("opacities", op.grad, ob.v_opacities,
                                                                  ob32.v_opacities),
             ("textures", tex.grad[T(o["rows"], torch.int64)], ob.v_textures, ob32.v_textures)]
    psnr = _psnr(rc, fo.colors[sel])
    cos = {k: cosine(to_np(g), ref) for k, g, ref, _ in grads}
    print(f"\n{fmt}: colour max abs {np.abs(rc - fo.colors[sel]).max():.3g}, PSNR {psnr:.1f} dB, "
          f"alpha max abs {np.abs(ra - fo.alphas[sel]).max():.3g}, gradient cosine "
          + ", ".join(f"{k} {v:.6f}" for k, v in cos.items()))
    if fmt == "fp32":
        assert_close(rc, fo.colors[sel], 1e-5, 1e-5, 1e-3, "colors")
        assert_close(ra, fo.alphas[sel], 1e-5, 0.0, 1e-3, "alphas")
        for k, g, ref, ref32 in grads:
            bound = max(1e-4, 1.5 * rel_l2(ref32, ref))
            assert rel_l2(to_np(g), ref) < bound, (k, rel_l2(to_np(g), ref), bound)
    else:
        floor_db, floor_cos = (35.0, 0.99) if fmt == "fp8" else (50.0, 0.999)
        assert psnr >= floor_db, psnr
        assert min(cos.values()) >= floor_cos, cos


@pytest.fixture(scope="module")
def sampled_oracle_aniso(mixture, sampled_oracle):
    """The FP64 and IEEE-FP32 oracle of the anisotropic_bilinear filter on the same sampled tiles."""
    d, o = mixture, sampled_oracle
    C, N, W, H, tw, th = d["C"], d["N"], d["W"], d["H"], d["tw"], d["th"]
    mask = np.zeros((C, th, tw), np.uint8)
    mask[:, ROW, ::10] = 1
    rows = o["rows"]
    remap = np.zeros(N, np.int64)
    remap[rows] = np.arange(rows.size)
    gid = remap[np.arange(C * N) % N]
    tex_sub = d["tex"][T(rows, torch.int64)].cpu().numpy()
    args = (to_np(d["means2d"]), to_np(d["M"]), to_np(d["colors"]), d["opac"], to_np(d["normals"]), tex_sub,
            d["off"].cpu().numpy(), d["fl"].cpu().numpy(), W, H, TILE)
    z3, z1 = np.zeros((C, H, W, 3), np.float32), np.zeros((C, H, W, 1), np.float32)
    out = {}
    for dt in (np.float64, np.float32):
        kw = dict(masks=mask, gaussian_ids=gid, n_gauss=rows.size, aniso=True, dtype=dt)
        fo = O.raster_fwd(*args, **kw)
        out[dt] = (fo, O.raster_bwd(*args, fo, o["up_c"], o["up_a"], z3, z1, z1, mode=0, **kw))
    return out


def test_mixture1m_anisotropic_bilinear_on_sampled_tiles(mixture, sampled_oracle, sampled_oracle_aniso):
    """The anisotropic_bilinear filter at full size (boundary integration, forward integral records, prefix
    fold), FP32 texture storage, against the FP64 oracle's cell-by-cell integration on the sampled tiles."""
    d, o = mixture, sampled_oracle
    m2d = d["means2d"].detach().clone().requires_grad_()
    M = d["M"].detach().clone().requires_grad_()
    cols = d["colors"].detach().clone().requires_grad_()
    op = T(d["opac"]).requires_grad_()
    tex = d["tex"].detach().requires_grad_()
    out = rasterize_to_pixels_textured_gaussians(
        m2d, M, cols, op, tex, 3.0, 3.0, d["normals"], torch.zeros_like(m2d), d["W"], d["H"], TILE, d["off"],
        d["fl"], filtering="anisotropic_bilinear")
    ((out[0] * T(o["up_c"])).sum() + (out[1] * T(o["up_a"])).sum()).backward()
    (fo, ob), (_, ob32) = sampled_oracle_aniso[np.float64], sampled_oracle_aniso[np.float32]
    sel = o["sel"]
    assert_close(to_np(out[0])[sel], fo.colors[sel], 1e-5, 1e-5, 1e-3, "colors")
    assert_close(to_np(out[1])[sel], fo.alphas[sel], 1e-5, 0.0, 1e-3, "alphas")
    grads = [("means2d", m2d.grad, ob.v_means2d, ob32.v_means2d), ("M", M.grad, ob.v_M, ob32.v_M),
             ("colors", cols.grad, ob.v_colors, ob32.v_colors),
             ("opacities", op.grad, ob.v_opacities, ob32.v_opacities),
             ("textures", tex.grad[T(o["rows"], torch.int64)], ob.v_textures, ob32.v_textures)]
    for k, g, ref, ref32 in grads:
        assert np.abs(ref).max() > 0, k
        bound = max(1e-4, 1.5 * rel_l2(ref32, ref))
        assert rel_l2(to_np(g), ref) < bound, (k, rel_l2(to_np(g), ref), bound)
