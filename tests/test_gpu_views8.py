"""The "views8" workload at full size on the GPU: 300,000 Gaussians, 50x50
FP32 RGBA textures, SH degree 3, eight 800x800 cameras, tile 16 -- the FP32
plain drop-in -- checked against the oracle where the oracle can follow at
this size:

  * intersections, sorted keys, flatten ids and tile offsets of all eight
    cameras: bit-exact against the oracle's on the same projected inputs;
  * SH colours (degree 3) of a sample of visible entries: 1e-5 against the
    FP64 oracle;
  * compositor forward on a sample of tiles of two cameras: 1e-5 absolute
    with the 1e-3 branch-flip budget against the FP64 oracle on the same
    inputs (the oracle's tile masks select the sample; the textures of the
    Gaussians those tiles touch are gathered on the GPU);
  * compositor adjoint with upstream gradients nonzero only on the sampled
    tiles: per tensor, relative L2 to the FP64 oracle within 1e-4 or within
    1.5x that of the IEEE-FP32 oracle (the same algorithm evaluated in FP32),
    whichever is larger.  Tiles here hold up to 3,400 splats and pixels up
    to ~190 contributors; the adjoint recovers each contributor's
    transmittance by division (the reference's scheme, no per-splat storage),
    so an FP32 evaluation itself lands 1e-4 .. 4e-3 from FP64 on this
    workload (measured: means2d 2.5e-4, M 3.7e-3).

The textures are drawn on the GPU (uniform [0, 1], seeded): 12 GB that the
host never holds.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests._util import assert_close, rel_l2, to_np
from textured_gaussians_b200 import scenes
from textured_gaussians_b200.cuda import (
    fully_fused_projection_2dgs,
    isect_offset_encode,
    isect_tiles,
    rasterize_to_pixels_textured_gaussians,
    spherical_harmonics,
)

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
TILE = 16
SAMPLE = {0: 25, 5: 12}  # camera -> tile row; every 6th tile of the row is compared


def T(x, dtype=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(x)).to(DEV, dtype)


@pytest.fixture(scope="module")
def views8():
    s = scenes.views8(with_textures=False)
    N, R = s.means.shape[0], s.extra["texture_res"]
    g = torch.Generator(device=DEV)
    g.manual_seed(1)
    tex = torch.rand((N, R, R, 4), generator=g, device=DEV)
    radii, means2d, depths, M, normals = fully_fused_projection_2dgs(
        T(s.means), T(s.quats), T(s.scales), T(s.viewmats), T(s.Ks), s.width, s.height, 0.3, s.near_plane,
        s.far_plane, 0.0)
    C = radii.shape[0]
    tw, th = -(-s.width // TILE), -(-s.height // TILE)
    tpg, ids, fl = isect_tiles(means2d, radii, depths, TILE, tw, th)
    off = isect_offset_encode(ids, C, tw, th)
    cam = torch.linalg.inv(T(s.viewmats))[:, :3, 3]
    dirs = T(s.means)[None] - cam[:, None]
    coeffs = T(s.colors)[None].expand(C, -1, -1, -1)
    sh = spherical_harmonics(3, dirs, coeffs, masks=radii > 0)
    colors = torch.clamp_min(sh + 0.5, 0.0)
    yield dict(s=s, tex=tex, radii=radii, means2d=means2d, depths=depths, M=M, normals=normals, tpg=tpg, ids=ids,
               fl=fl, off=off, dirs=dirs, sh=sh, colors=colors, C=C, N=N, R=R, tw=tw, th=th)
    del tex
    torch.cuda.empty_cache()


def test_views8_intersections_bit_exact(views8):
    d = views8
    o_tpg, o_ids, o_fl = O.isect_tiles(to_np(d["means2d"]), d["radii"].cpu().numpy(), to_np(d["depths"]), TILE,
                                       d["tw"], d["th"], d["C"])
    assert d["ids"].numel() > 10_000_000  # the workload's scale: tens of millions of (tile, splat) pairs
    np.testing.assert_array_equal(d["tpg"].cpu().numpy(), o_tpg)
    np.testing.assert_array_equal(d["ids"].cpu().numpy(), o_ids)
    np.testing.assert_array_equal(d["fl"].cpu().numpy(), o_fl)
    np.testing.assert_array_equal(d["off"].cpu().numpy(), O.isect_offset_encode(o_ids, d["C"], d["tw"], d["th"]))


def test_views8_sh_degree3(views8):
    d = views8
    rng = np.random.default_rng(0)
    pick = rng.choice(d["N"], 20_000, replace=False)
    ref = O.sh_fwd(3, to_np(d["dirs"])[:, pick].astype(np.float64), d["s"].colors[pick].astype(np.float64),
                   masks=(d["radii"] > 0).cpu().numpy()[:, pick], dtype=np.float64)
    assert_close(to_np(d["sh"])[:, pick], ref, 1e-5, 0.0, 0.0, "sh")


def _sampled(d):
    """Tile mask of the sample, the Gaussians its tiles touch, and the per-element texture row map."""
    C, N, tw, th = d["C"], d["N"], d["tw"], d["th"]
    mask = np.zeros((C, th, tw), np.uint8)
    for c, row in SAMPLE.items():
        mask[c, row, ::6] = 1
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
    return mask, rows, gid


def test_views8_compositor_forward_and_adjoint_on_sampled_tiles(views8):
    d = views8
    s, C, N = d["s"], d["C"], d["N"]
    W, H = s.width, s.height
    mask, rows, gid = _sampled(d)
    opac = np.tile(s.opacities[None], (C, 1))
    # GPU: the whole render; upstream gradients only on the sampled tiles' pixels
    pix = np.repeat(np.repeat(mask, TILE, 1), TILE, 2)[:, :H, :W].astype(np.float32)[..., None]
    rng = np.random.default_rng(2)
    up_c = rng.normal(size=(C, H, W, 3)).astype(np.float32) * pix
    up_a = rng.normal(size=(C, H, W, 1)).astype(np.float32) * pix
    m2d = d["means2d"].detach().clone().requires_grad_()
    M = d["M"].detach().clone().requires_grad_()
    cols = d["colors"].detach().clone().requires_grad_()
    op = T(opac).requires_grad_()
    tex = d["tex"].requires_grad_()
    out = rasterize_to_pixels_textured_gaussians(m2d, M, cols, op, tex, 3.0, 3.0, d["normals"],
                                                 torch.zeros_like(m2d), W, H, TILE, d["off"], d["fl"])
    ((out[0] * T(up_c)).sum() + (out[1] * T(up_a)).sum()).backward()
    # oracle: FP64 on the same inputs, sampled tiles only, textures of the touched Gaussians
    tex_sub = d["tex"].detach()[T(rows, torch.int64)].cpu().numpy()
    args = (to_np(d["means2d"]), to_np(d["M"]), to_np(d["colors"]), opac, to_np(d["normals"]), tex_sub,
            d["off"].cpu().numpy(), d["fl"].cpu().numpy(), W, H, TILE)
    kw = dict(masks=mask, gaussian_ids=gid, n_gauss=rows.size, dtype=np.float64)
    fo = O.raster_fwd(*args, **kw)
    sel = pix[..., 0] > 0
    assert sel.sum() >= 4000
    assert_close(to_np(out[0])[sel], fo.colors[sel], 1e-5, 1e-5, 1e-3, "colors")
    assert_close(to_np(out[1])[sel], fo.alphas[sel], 1e-5, 0.0, 1e-3, "alphas")
    assert_close(to_np(out[2])[sel], fo.normals[sel], 1e-5, 1e-5, 1e-3, "normals")
    zeros = np.zeros((C, H, W, 3)), np.zeros((C, H, W, 1))
    ob = O.raster_bwd(*args, fo, up_c, up_a, zeros[0], zeros[1], zeros[1], mode=0, **kw)
    kw32 = dict(kw, dtype=np.float32)
    ob32 = O.raster_bwd(*args, O.raster_fwd(*args, **kw32), up_c, up_a, zeros[0], zeros[1], zeros[1], mode=0,
                        **kw32)
    pairs = [("means2d", m2d.grad, ob.v_means2d, ob32.v_means2d), ("M", M.grad, ob.v_M, ob32.v_M),
             ("colors", cols.grad, ob.v_colors, ob32.v_colors),
             ("opacities", op.grad, ob.v_opacities, ob32.v_opacities),
             ("textures", tex.grad[T(rows, torch.int64)], ob.v_textures, ob32.v_textures)]
    for k, got, ref, ref32 in pairs:
        got = to_np(got)
        assert np.abs(ref).max() > 0, k
        bound = max(1e-4, 1.5 * rel_l2(ref32, ref))
        assert rel_l2(got, ref) < bound, (k, rel_l2(got, ref), bound)
    # no gradient reaches a texture the sampled tiles do not touch
    untouched = torch.ones(N, dtype=torch.bool, device=DEV)
    untouched[T(rows, torch.int64)] = False
    assert float(tex.grad[untouched].abs().max()) == 0.0


def test_views8_transmittance_checkpoints_bring_gradients_closer_to_fp64(views8):
    """transmittance="checkpoint": the forward keeps every pixel's transmittance at the end of each batch
    and the adjoint restarts its back-to-front division there, instead of dividing the final transmittance
    back over the whole list (up to ~3,400 splats per tile here).  On the sampled tiles every gradient must
    come out at least as close to the FP64 oracle as with the reference's division scheme, and the
    per-Gaussian ones (colours, opacities, textures) within 1e-4 relative L2 of it."""
    d = views8
    s, C, N = d["s"], d["C"], d["N"]
    W, H = s.width, s.height
    mask, rows, gid = _sampled(d)
    opac = np.tile(s.opacities[None], (C, 1))
    pix = np.repeat(np.repeat(mask, TILE, 1), TILE, 2)[:, :H, :W].astype(np.float32)[..., None]
    rng = np.random.default_rng(2)
    up_c = rng.normal(size=(C, H, W, 3)).astype(np.float32) * pix
    up_a = rng.normal(size=(C, H, W, 1)).astype(np.float32) * pix
    tex_sub = d["tex"].detach()[T(rows, torch.int64)].cpu().numpy()
    args = (to_np(d["means2d"]), to_np(d["M"]), to_np(d["colors"]), opac, to_np(d["normals"]), tex_sub,
            d["off"].cpu().numpy(), d["fl"].cpu().numpy(), W, H, TILE)
    kw = dict(masks=mask, gaussian_ids=gid, n_gauss=rows.size, dtype=np.float64)
    fo = O.raster_fwd(*args, **kw)
    zeros = np.zeros((C, H, W, 3)), np.zeros((C, H, W, 1))
    ob = O.raster_bwd(*args, fo, up_c, up_a, zeros[0], zeros[1], zeros[1], mode=0, **kw)
    errs = {}
    for mode in ("divide", "checkpoint"):
        m2d = d["means2d"].detach().clone().requires_grad_()
        M = d["M"].detach().clone().requires_grad_()
        cols = d["colors"].detach().clone().requires_grad_()
        op = T(opac).requires_grad_()
        tex = d["tex"].detach().requires_grad_()
        out = rasterize_to_pixels_textured_gaussians(m2d, M, cols, op, tex, 3.0, 3.0, d["normals"],
                                                     torch.zeros_like(m2d), W, H, TILE, d["off"], d["fl"],
                                                     transmittance=mode)
        ((out[0] * T(up_c)).sum() + (out[1] * T(up_a)).sum()).backward()
        errs[mode] = {"means2d": rel_l2(to_np(m2d.grad), ob.v_means2d), "M": rel_l2(to_np(M.grad), ob.v_M),
                      "colors": rel_l2(to_np(cols.grad), ob.v_colors),
                      "opacities": rel_l2(to_np(op.grad), ob.v_opacities),
                      "textures": rel_l2(to_np(tex.grad[T(rows, torch.int64)]), ob.v_textures)}
        tex.grad = None
    print("\nrelative L2 to FP64, divide:", {k: f"{v:.2e}" for k, v in errs["divide"].items()},
          "\ncheckpoint:", {k: f"{v:.2e}" for k, v in errs["checkpoint"].items()})
    for k, e in errs["checkpoint"].items():
        assert e <= 1.05 * errs["divide"][k] + 1e-7, (k, e, errs["divide"][k])
    for k in ("colors", "opacities", "textures"):
        assert errs["checkpoint"][k] < 1e-4, (k, errs["checkpoint"][k])
