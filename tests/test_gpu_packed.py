"""GPU parity of the packed layout (``packed=True``, ``sparse_grad``).

The reference checks its packed path against its dense path
(tests/test_basic.py: test_fully_fused_projection_packed,
test_rasterize_to_pixels with packed=True); these tests do the same and add the
CPU oracle on the packed entries themselves.

Tolerances:
  * packed projection entries, ids and indptr: bit-exact against the dense
    entries with radii > 0 (one device function computes both);
  * packed compositor forward: bit-exact against the dense compositor on the
    same scene (same intersections in the same order), and within the dense
    tests' bounds of the FP64 oracle run on the packed entries;
  * gradients: 1e-5 relative in L2 norm against the dense path (float atomics
    sum the per-camera terms in a different order).
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests._util import assert_close, rel_l2, to_np
from textured_gaussians_b200 import rasterization_2dgs, rasterization_textured_gaussians, scenes
from textured_gaussians_b200.cuda import (
    fully_fused_projection_2dgs,
    isect_offset_encode,
    isect_tiles,
    rasterize_to_pixels_textured_gaussians,
)

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def T(x, dtype=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(x)).to(DEV, dtype)


def scene3():
    """Three cameras with different intrinsics, so a wrong camera's K shows."""
    s = scenes.tiny(seed=7, n_cams=3)
    s.Ks[1, 0, 0] *= 1.2
    s.Ks[1, 1, 1] *= 1.2
    s.Ks[2, 0, 2] += 5.0
    s.Ks[2, 1, 2] -= 3.0
    return s


def scene_multi_chunk():
    """20,000 Gaussians, 3 cameras: several 4096-entry chunks per camera row."""
    s = scenes.mixture1m(N=20_000, n_cams=3, width=320, height=240, radius=25.0)
    s.Ks[2, 0, 0] *= 0.8
    return s


def _leaves(s):
    return [T(x).requires_grad_() for x in (s.means, s.quats, s.scales)]


@pytest.mark.parametrize("make", [scene3, scene_multi_chunk])
def test_packed_projection_matches_dense_entries_bit_exact(make):
    s = make()
    args = (T(s.viewmats), T(s.Ks), s.width, s.height, 0.3, s.near_plane, s.far_plane, 0.0)
    radii, m2d, depths, M, nrm = fully_fused_projection_2dgs(T(s.means), T(s.quats), T(s.scales), *args)
    cids, gids, p_radii, p_m2d, p_depths, p_M, p_nrm = fully_fused_projection_2dgs(
        T(s.means), T(s.quats), T(s.scales), *args, packed=True)
    sel = (radii > 0).nonzero()
    assert cids.dtype == torch.int64 and gids.dtype == torch.int64 and p_radii.dtype == torch.int32
    assert torch.equal(cids, sel[:, 0]) and torch.equal(gids, sel[:, 1])
    for dense, packed in ((radii, p_radii), (m2d, p_m2d), (depths, p_depths), (M, p_M), (nrm, p_nrm)):
        assert torch.equal(dense[sel[:, 0], sel[:, 1]], packed)
    # every camera's intrinsics are used: the entries differ from a projection with Ks[0] everywhere
    assert not torch.equal(p_m2d, fully_fused_projection_2dgs(
        T(s.means), T(s.quats), T(s.scales), T(s.viewmats), T(np.repeat(s.Ks[:1], 3, 0)), s.width, s.height, 0.3,
        s.near_plane, s.far_plane, 0.0)[1][sel[:, 0], sel[:, 1]])


def test_packed_projection_empty_and_indptr():
    s = scene3()
    # near plane beyond every Gaussian: nnz = 0
    out = fully_fused_projection_2dgs(T(s.means), T(s.quats), T(s.scales), T(s.viewmats), T(s.Ks), s.width,
                                      s.height, 0.3, 1e9, 1e10, 0.0, packed=True)
    assert all(t.shape[0] == 0 for t in out)
    # indptr (exposed through the C ABI) against per-camera counts
    import ctypes
    from textured_gaussians_b200 import _backend as B
    C, N = s.viewmats.shape[0], s.means.shape[0]
    means, quats, scales, vm, Ks = (T(x) for x in (s.means, s.quats, s.scales, s.viewmats, s.Ks))
    ws = torch.empty((B.lib().tg_project_packed_workspace_bytes(C, N),), dtype=torch.uint8, device=DEV)
    nnz = torch.empty((1,), dtype=torch.int64, device=DEV)
    indptr = torch.empty((C + 1,), dtype=torch.int32, device=DEV)
    a = B.ProjectPackedArgs(C, N, B.ptr(means), B.ptr(quats), B.ptr(scales), B.ptr(vm), B.ptr(Ks), s.width,
                            s.height, s.near_plane, s.far_plane, 0.0, B.ptr(ws), B.ptr(nnz), B.ptr(indptr), 0)
    st = torch.cuda.current_stream().cuda_stream
    assert B.lib().tg_project_packed_count(ctypes.byref(a), st) == 0
    radii = fully_fused_projection_2dgs(means, quats, scales, vm, Ks, s.width, s.height, 0.3, s.near_plane,
                                        s.far_plane, 0.0)[0]
    counts = (radii > 0).sum(1)
    expect = torch.cat([torch.zeros(1, dtype=torch.int64, device=DEV), counts.cumsum(0)]).int()
    assert torch.equal(indptr, expect)
    assert int(nnz.item()) == int(counts.sum())


@pytest.mark.parametrize("norm_rot_grad,adjoint", [(False, "reference"), (True, "reference"), (False, "exact")])
def test_packed_projection_backward_dense_and_sparse(norm_rot_grad, adjoint):
    s = scene3()
    rng = np.random.default_rng(5)
    vm, Ks = T(s.viewmats), T(s.Ks)
    kw = dict(norm_rot_grad=norm_rot_grad, adjoint=adjoint)
    # dense reference
    lm, lq, ls = _leaves(s)
    radii, m2d, depths, M, nrm = fully_fused_projection_2dgs(lm, lq, ls, vm, Ks, s.width, s.height, 0.3,
                                                             s.near_plane, s.far_plane, 0.0, **kw)
    w = [T(rng.normal(size=t.shape)) for t in (m2d, depths, M, nrm)]
    mask = (radii > 0)
    sum((t * wt * (mask[..., None, None] if t.dim() == 4 else mask[..., None] if t.dim() == 3 else mask)).sum()
        for t, wt in zip((m2d, depths, M, nrm), w)).backward()
    dense = [t.grad.clone() for t in (lm, lq, ls)]
    sel = mask.nonzero()
    for sparse in (False, True):
        pm, pq, ps = _leaves(s)
        cids, gids, _, p_m2d, p_d, p_M, p_n = fully_fused_projection_2dgs(
            pm, pq, ps, vm, Ks, s.width, s.height, 0.3, s.near_plane, s.far_plane, 0.0, packed=True,
            sparse_grad=sparse, **kw)
        pw = [x[sel[:, 0], sel[:, 1]] for x in w]
        sum((t * wt).sum() for t, wt in zip((p_m2d, p_d, p_M, p_n), pw)).backward()
        for name, leaf, ref in zip(("means", "quats", "scales"), (pm, pq, ps), dense):
            g = leaf.grad
            if sparse:
                assert g.is_sparse and torch.equal(g._indices()[0], gids), name
                assert g._values().shape == (gids.shape[0], ref.shape[1]), name
                g = g.to_dense()
            assert rel_l2(to_np(g), to_np(ref)) < 1e-5, (name, sparse, rel_l2(to_np(g), to_np(ref)))


def test_packed_textured_compositor_vs_oracle():
    s = scene3()
    C, N = s.viewmats.shape[0], s.means.shape[0]
    cids, gids, radii, m2d, depths, M, nrm = fully_fused_projection_2dgs(
        T(s.means), T(s.quats), T(s.scales), T(s.viewmats), T(s.Ks), s.width, s.height, 0.3, s.near_plane,
        s.far_plane, 0.0, packed=True)
    ts = s.tile_size
    tw, th = -(-s.width // ts), -(-s.height // ts)
    _, ids, fl = isect_tiles(m2d, radii, depths, ts, tw, th, packed=True, n_cameras=C, camera_ids=cids,
                             gaussian_ids=gids)
    off = isect_offset_encode(ids, C, tw, th)
    nnz = cids.shape[0]
    rng = np.random.default_rng(2)
    colors = rng.uniform(0, 1, size=(nnz, 3)).astype(np.float32)
    opac = s.opacities[gids.cpu().numpy()]
    g = rasterize_to_pixels_textured_gaussians(m2d, M, T(colors), T(opac), T(s.textures), 3.0, 3.0, nrm,
                                               torch.zeros_like(m2d), s.width, s.height, ts, off, fl, packed=True,
                                               gaussian_ids=gids)
    o = O.raster_fwd(to_np(m2d), to_np(M), colors, opac, to_np(nrm), s.textures, off.cpu().numpy(),
                     fl.cpu().numpy(), s.width, s.height, ts, gaussian_ids=gids.cpu().numpy(), n_gauss=N,
                     dtype=np.float64)
    rc, ra, rn, rd, rm, cs, cc = (to_np(x) for x in g)
    assert cs.shape == (N,) and cc.shape == (N,)
    assert_close(rc, o.colors, 1e-5, 1e-5, 1e-4, "colors")
    assert_close(ra, o.alphas, 1e-5, 0, 1e-4, "alphas")
    assert_close(rn, o.normals, 1e-5, 1e-5, 1e-4, "normals")
    assert_close(rd, o.distort, 1e-5, 1e-4, 1e-4, "distort")
    assert_close(rm, o.median, 1e-5, 1e-5, 1e-4, "median")
    assert_close(cs, o.contrib_sum, 1e-4, 1e-5, 1e-4, "contrib_sum")
    assert_close(cc, o.contrib_count, 0, 0, 1e-4, "contrib_count")


def test_packed_textured_needs_gaussian_ids():
    s = scene3()
    z = torch.zeros((4, 2), device=DEV)
    with pytest.raises(ValueError):
        rasterize_to_pixels_textured_gaussians(z, torch.zeros((4, 3, 3), device=DEV), torch.zeros((4, 3), device=DEV),
                                               torch.zeros((4,), device=DEV), T(s.textures), 3.0, 3.0,
                                               torch.zeros((4, 3), device=DEV), z, 16, 16, 16,
                                               torch.zeros((1, 1, 1), dtype=torch.int32, device=DEV),
                                               torch.zeros((0,), dtype=torch.int32, device=DEV), packed=True)


def _render(fn, s, packed, textured, sh, mode, sparse=False):
    leaves = [T(x).requires_grad_() for x in (s.means, s.quats, s.scales, s.opacities)]
    cols = T(s.colors if sh else s.colors[:, 0, :]).requires_grad_()
    tex = T(s.textures).requires_grad_()
    kw = dict(sh_degree=int(round(np.sqrt(s.colors.shape[1]))) - 1 if sh else None,
              far_plane=s.far_plane, packed=packed, sparse_grad=sparse, render_mode=mode,
              backgrounds=None)
    if textured:
        out = fn(*leaves, cols, tex, T(s.viewmats), T(s.Ks), s.width, s.height, **kw)
    else:
        out = fn(*leaves, cols, T(s.viewmats), T(s.Ks), s.width, s.height, **kw)
    rng = np.random.default_rng(11)
    loss = sum((t * T(rng.normal(size=t.shape))).sum() for t in (out[0], out[1], out[2]))
    loss.backward()
    grads = [t.grad.to_dense() if t.grad.is_sparse else t.grad for t in leaves + [cols]]
    if textured:
        grads.append(tex.grad)
    return out, grads


@pytest.mark.parametrize("textured,sh,mode,sparse", [(True, True, "RGB", False), (True, False, "RGB+ED", False),
                                                     (True, True, "RGB", True), (False, True, "RGB+D", False),
                                                     (False, False, "RGB", True)])
def test_packed_render_matches_dense(textured, sh, mode, sparse):
    s = scene3()
    fn = rasterization_textured_gaussians if textured else rasterization_2dgs
    dense, gd = _render(fn, s, False, textured, sh, mode)
    packed, gp = _render(fn, s, True, textured, sh, mode, sparse)
    meta = packed[-1]
    assert meta["camera_ids"] is not None and meta["gaussian_ids"] is not None
    for i in (0, 1, 2, 4, 5):  # colours, alphas, normals, distortion, median
        assert torch.equal(dense[i], packed[i]), i
    # per-Gaussian contribution statistics in both layouts
    assert dense[6].shape == packed[6].shape == (s.means.shape[0],)
    assert torch.allclose(dense[6], packed[6], rtol=1e-5, atol=1e-6)
    assert torch.equal(dense[7], packed[7])
    for k, (a, b) in enumerate(zip(gd, gp)):
        assert rel_l2(to_np(b), to_np(a)) < 1e-5, (k, rel_l2(to_np(b), to_np(a)))
