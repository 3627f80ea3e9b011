"""Generate tests/golden/*.npz from the reference's own pure-torch code.

Run where the reference's source tree is mounted (read-only), naming its
root:  python tests/golden/make_golden.py --reference PATH  (or set
REFERENCE_ROOT).

The reference's CUDA extension cannot be built (its GLM submodule is empty),
but these pure-torch twins import and run on the CPU:
  * _fully_fused_projection_2dgs   textured_gaussians/cuda/_torch_impl_2dgs.py:9-75
  * _isect_tiles                   textured_gaussians/cuda/_torch_impl.py:331-400
  * _isect_offset_encode           textured_gaussians/cuda/_torch_impl.py:403-429
  * _spherical_harmonics           textured_gaussians/cuda/_torch_impl.py:704-714
  * accumulate_2dgs                textured_gaussians/cuda/_torch_impl_2dgs.py:78-168
  * DefaultStrategy._update_state  textured_gaussians/strategy/default.py:213-261
accumulate_2dgs needs two functions of the third-party package nerfacc
(not installed): render_weight_from_alpha and accumulate_along_rays.  A
stand-in module below restates their published semantics (nerfacc 0.5:
weights_i = alpha_i * prod_{j<i on the same ray}(1 - alpha_j); accumulation =
per-ray sum of weights * values).  The contributing (Gaussian, pixel) pairs fed
to accumulate_2dgs are enumerated here in numpy, front to back, with the
reference compositor's alpha cut (1/255) and stop rule (T <= 1e-4).

The fixtures are small and committed; nothing on the GPU machine reads the
reference tree.
"""
import os
import sys
import types

import numpy as np
import torch

def _reference_root() -> str:
    if "--reference" in sys.argv:
        return sys.argv[sys.argv.index("--reference") + 1]
    root = os.environ.get("REFERENCE_ROOT")
    if not root:
        raise SystemExit("name the reference's source tree: --reference PATH or REFERENCE_ROOT")
    return root


REF = _reference_root()
HERE = os.path.dirname(os.path.abspath(__file__))
sys.dont_write_bytecode = True
sys.path.insert(0, REF)
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def nerfacc_standin():
    m = types.ModuleType("nerfacc")

    def render_weight_from_alpha(alphas, ray_indices=None, n_rays=None):
        order = torch.arange(alphas.numel())
        w = torch.empty_like(alphas)
        trans = torch.empty_like(alphas)
        T = {}
        for i in order.tolist():
            r = int(ray_indices[i])
            t = T.get(r, torch.tensor(1.0, dtype=alphas.dtype))
            trans[i] = t
            w[i] = alphas[i] * t
            T[r] = t * (1 - alphas[i])
        return w, trans

    def accumulate_along_rays(weights, values=None, ray_indices=None, n_rays=None):
        src = weights[:, None] if values is None else weights[:, None] * values
        out = torch.zeros((n_rays, src.shape[-1]), dtype=weights.dtype)
        out.index_add_(0, ray_indices.long(), src)
        return out

    m.render_weight_from_alpha = render_weight_from_alpha
    m.accumulate_along_rays = accumulate_along_rays
    return m


def main():
    sys.modules["nerfacc"] = nerfacc_standin()
    from textured_gaussians.cuda._torch_impl import _isect_offset_encode, _isect_tiles, _spherical_harmonics
    from textured_gaussians.cuda._torch_impl_2dgs import _fully_fused_projection_2dgs, accumulate_2dgs

    from textured_gaussians_b200 import scenes

    torch.manual_seed(0)
    # ---------------------------------------------------------------- projection + isect
    s = scenes.tiny(seed=21, N=400, width=120, height=90, n_cams=3)
    args = [torch.from_numpy(x) for x in (s.means, s.quats, s.scales, s.viewmats, s.Ks)]
    radii, means2d, depths, M, normals = _fully_fused_projection_2dgs(*args, s.width, s.height, s.near_plane,
                                                                      s.far_plane)
    ts = 16
    tw, th = -(-s.width // ts), -(-s.height // ts)
    tpg, isect_ids, flatten_ids = _isect_tiles(means2d, radii, depths, ts, tw, th, sort=True)
    offsets = _isect_offset_encode(isect_ids, s.viewmats.shape[0], tw, th)
    np.savez_compressed(
        os.path.join(HERE, "projection_isect.npz"), means=s.means, quats=s.quats, scales=s.scales,
        viewmats=s.viewmats, Ks=s.Ks, width=s.width, height=s.height, near=s.near_plane, far=s.far_plane,
        radii=radii.numpy(), means2d=means2d.numpy(), depths=depths.numpy(), M=M.numpy(), normals=normals.numpy(),
        tile_size=ts, tiles_per_gauss=tpg.numpy(), isect_ids=isect_ids.numpy(), flatten_ids=flatten_ids.numpy(),
        offsets=offsets.numpy())

    # ---------------------------------------------------------------- spherical harmonics
    rng = np.random.default_rng(4)
    dirs = rng.normal(size=(96, 3)).astype(np.float64)
    coeffs = rng.normal(size=(96, 25, 3)).astype(np.float64)
    sh = {}
    for deg in range(5):
        sh[f"deg{deg}"] = _spherical_harmonics(deg, torch.from_numpy(dirs), torch.from_numpy(coeffs)).numpy()
    np.savez_compressed(os.path.join(HERE, "sh.npz"), dirs=dirs, coeffs=coeffs, **sh)

    # ---------------------------------------------------------------- plain 2DGS compositing
    from oracle import oracle as O

    s = scenes.tiny(seed=22, N=250, width=48, height=32)
    C = 1
    radii, m2d, dep, Mo, nrm = O.project_fwd(s.means, s.quats, s.scales, s.viewmats, s.Ks, s.width, s.height,
                                             s.near_plane, s.far_plane)
    tw, th = -(-s.width // ts), -(-s.height // ts)
    _, ids, fl = O.isect_tiles(m2d, radii, dep, ts, tw, th, C)
    off = O.isect_offset_encode(ids, C, tw, th)
    opac = s.opacities[None].astype(np.float32)
    colors = rng.uniform(0, 1, size=(C, s.means.shape[0], 3)).astype(np.float32)
    n_isects = ids.size
    g_ids, p_ids = [], []
    for i in range(s.height):
        for j in range(s.width):
            t = (i // ts) * tw + (j // ts)
            start = off.reshape(-1)[t]
            end = n_isects if t == tw * th - 1 else off.reshape(-1)[t + 1]
            px, py = np.float32(j + 0.5), np.float32(i + 0.5)
            T = np.float32(1)
            for k in range(start, end):
                g = fl[k]
                Mg = Mo.reshape(-1, 3, 3)[g]
                hu = px * Mg[2] - Mg[0]
                hv = py * Mg[2] - Mg[1]
                z = np.cross(hu, hv).astype(np.float32)
                if z[2] == 0:
                    continue
                u, v = z[0] / z[2], z[1] / z[2]
                d = m2d.reshape(-1, 2)[g] - np.array([px, py], np.float32)
                sig = np.float32(0.5) * min(u * u + v * v, np.float32(2) * (d[0] * d[0] + d[1] * d[1]))
                a = min(np.float32(0.999), opac.reshape(-1)[g] * np.exp(-sig))
                if sig < 0 or a < np.float32(1) / np.float32(255):
                    continue
                nT = T * (np.float32(1) - a)
                if nT <= np.float32(1e-4):
                    break
                g_ids.append(g)
                p_ids.append(i * s.width + j)
                T = nT
    gi = torch.tensor(g_ids, dtype=torch.long)
    pi = torch.tensor(p_ids, dtype=torch.long)
    ci = torch.zeros_like(gi)
    renders, alphas, rnormals = accumulate_2dgs(
        torch.from_numpy(m2d), torch.from_numpy(Mo), torch.from_numpy(opac), torch.from_numpy(colors),
        torch.from_numpy(nrm), gi, pi, ci, s.width, s.height)
    np.savez_compressed(
        os.path.join(HERE, "plain_accumulate.npz"), means=s.means, quats=s.quats, scales=s.scales,
        opacities=s.opacities, viewmats=s.viewmats, Ks=s.Ks, width=s.width, height=s.height, near=s.near_plane,
        far=s.far_plane, colors=colors, tile_size=ts, pair_gaussian_ids=gi.numpy(), pair_pixel_ids=pi.numpy(),
        renders=renders.numpy(), alphas=alphas.numpy(), normals=rnormals.numpy())
    densify_golden()
    print("wrote", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))


def densify_golden():
    """Running densification statistics of the reference's DefaultStrategy on seeded gradients and radii:
    dense [C=3], dense [C=1] (where its radius statistic is a plain maximum) and packed."""
    from textured_gaussians.strategy.default import DefaultStrategy

    rng = np.random.default_rng(41)
    W, H, N = 120, 90, 500
    out = {}
    for tag, C, packed in (("dense3", 3, False), ("dense1", 1, False), ("packed", 3, True)):
        radii = rng.integers(0, 6, size=(C, N)).astype(np.int32) * (rng.uniform(size=(C, N)) < 0.7)
        grads = rng.normal(size=(C, N, 2)).astype(np.float32) * 1e-3
        if packed:
            cam, gid = np.nonzero(radii > 0)
            radii_in, grads_in = radii[cam, gid].astype(np.int32), grads[cam, gid]
        else:
            gid, radii_in, grads_in = None, radii.astype(np.int32), grads
        g2 = torch.from_numpy(grads_in.copy()).requires_grad_()
        g2.grad = torch.from_numpy(grads_in.copy())
        strat = DefaultStrategy(refine_scale2d_stop_iter=1)
        state = {"grad2d": None, "count": None, "radii": None}
        info = {"width": W, "height": H, "n_cameras": C, "radii": torch.from_numpy(radii_in),
                "gaussian_ids": None if gid is None else torch.from_numpy(gid.astype(np.int64)),
                strat.key_for_gradient: g2}
        strat._update_state({"means": torch.zeros(N, 3)}, state, info, packed=packed)
        out.update({f"{tag}_radii": radii_in, f"{tag}_grads": grads_in, f"{tag}_grad2d": state["grad2d"].numpy(),
                    f"{tag}_count": state["count"].numpy(), f"{tag}_max_radii": state["radii"].numpy()})
        if gid is not None:
            out[f"{tag}_gaussian_ids"] = gid.astype(np.int64)
    np.savez_compressed(os.path.join(HERE, "densify_stats.npz"), width=W, height=H, N=N, **out)


if __name__ == "__main__":
    main()
