"""The CPU oracle pinned to the reference's OWN CUDA path: golden vectors from
the unmodified reference run on a B200, one camera per call
(tests/golden/make_ref_golden.py), compared with the oracle on the same inputs
-- the reference's intermediate tensors for every stage.

This is what pins the oracle's restatement of the textured compositor
(bilinear, bilinear_bwd2, mipmapped2, anisotropic_bilinear: forward and
adjoint) and of the plain 2DGS compositor, the projection, SH and the tile
intersection.  The oracle runs in FP64 on the FP32 inputs; tolerances:
intersections bit-exact; forward outputs 1e-5 absolute (+1e-5 relative) with a
1e-3 fraction of branch flips between the FP32 reference and the FP64 oracle;
gradients 1e-4 relative L2 per tensor.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests import _refgold as RG
from tests._util import assert_close, rel_l2

F64 = np.float64
FLIPS = 1e-3
CASES = {"small": ("bilinear", "bilinear_bwd2"), "adjoint": ("bilinear", "bilinear_bwd2", "mipmapped2"),
         "adjoint_aniso": ("anisotropic_bilinear",)}
MODE = {"bilinear": 0, "bilinear_bwd2": 1, "mipmapped2": 0, "anisotropic_bilinear": 0}

_CACHE = {}


def fixture(case):
    if case not in _CACHE:
        g = RG.load(case)
        _CACHE[case] = (g, RG.scene(case, g))
    return _CACHE[case]


def check_grad(name, got, ref, tol=1e-4):
    assert np.abs(ref).max() > 0, f"{name}: reference gradient is all zero"
    r = rel_l2(got, ref)
    assert r < tol, f"{name}: relative L2 {r:.3g} >= {tol}"


@pytest.mark.parametrize("case", list(CASES))
def test_oracle_projection_and_sh_match_reference(case):
    g, s = fixture(case)
    radii, m2d, dep, M, nrm = O.project_fwd(s.means, s.quats, s.scales, s.viewmats, s.Ks, s.width, s.height,
                                            s.near_plane, s.far_plane, dtype=F64)
    ref_r = g["stage__radii"]
    diff = radii != ref_r
    assert diff.sum() <= max(2, 5e-3 * diff.size), f"{diff.sum()} radius flips"
    vis = (radii > 0) & (ref_r > 0)
    assert_close(m2d[vis], g["stage__means2d"][vis], 1e-5, 1e-5, name="means2d")
    assert_close(dep[vis], g["stage__depths"][vis], 1e-5, 1e-6, name="depths")
    assert_close(M[vis], g["stage__M"][vis], 1e-5, 1e-5, name="ray_transforms")
    assert_close(nrm[vis], g["stage__normals"][vis], 1e-5, 0.0, name="normals")
    cam = np.linalg.inv(s.viewmats.astype(F64))[:, :3, 3]
    dirs = s.means.astype(F64)[None] - cam[:, None]
    sh = O.sh_fwd(s.sh_degree, dirs, s.colors.astype(F64), masks=ref_r > 0, dtype=F64)
    assert_close(np.maximum(sh + 0.5, 0.0)[vis], g["stage__colors"][vis], 1e-5, 1e-6, name="sh colours")


@pytest.mark.parametrize("case", list(CASES))
def test_oracle_intersections_bit_exact_against_reference(case):
    g, s = fixture(case)
    tw, th = -(-s.width // s.tile_size), -(-s.height // s.tile_size)
    tpg, ids, fl = O.isect_tiles(g["stage__means2d"], g["stage__radii"], g["stage__depths"], s.tile_size, tw, th, 1)
    np.testing.assert_array_equal(tpg, g["stage__tpg"])
    np.testing.assert_array_equal(ids, g["stage__isect_ids"])
    np.testing.assert_array_equal(fl, g["stage__flatten_ids"])
    np.testing.assert_array_equal(O.isect_offset_encode(ids, 1, tw, th), g["stage__offsets"])


def _oracle(g, s, filtering):
    """Oracle forward + adjoint of one compositor on the fixture's stage inputs."""
    L = 0
    tex = None if filtering is None else s.textures.astype(np.float32)
    if filtering == "mipmapped2":
        L = s.textures.shape[1].bit_length() - 1
        tex = O.generate_mipmap(tex)
    aniso = filtering == "anisotropic_bilinear"
    args = (g["stage__means2d"], g["stage__M"], g["stage__colors"], s.opacities[None], g["stage__normals"], tex,
            g["stage__offsets"], g["stage__flatten_ids"], s.width, s.height, s.tile_size)
    bg = s.backgrounds
    fo = O.raster_fwd(*args, backgrounds=bg, mip_levels=L, aniso=aniso, dtype=F64)
    ups = RG.upstream(g["up_seed"], s)
    bo = O.raster_bwd(*args, fo, *ups, backgrounds=bg, mode=MODE.get(filtering, 0), mip_levels=L, aniso=aniso,
                      dtype=F64)
    v_tex = bo.v_textures
    if L:
        v_tex = O.generate_mipmap_bwd(v_tex, L)
    return fo, bo, v_tex


def _check(g, prefix, fo, bo, v_tex):
    outs = (fo.colors, fo.alphas, fo.normals, fo.distort, fo.median)
    for i, (o, name) in enumerate(zip(outs, ("colors", "alphas", "normals", "distort", "median"))):
        assert_close(o, g[f"{prefix}__out{i}"], 1e-5, 1e-5, FLIPS, f"{prefix} {name}")
    cnt = g[f"{prefix}__out6"]
    off = np.abs(fo.contrib_count - cnt) > 0
    assert off.sum() <= max(1, 0.01 * off.size) and np.abs(fo.contrib_count - cnt).max() <= 2
    assert rel_l2(fo.contrib_sum, g[f"{prefix}__out5"]) < 1e-4
    for k, v in (("means2d", bo.v_means2d), ("M", bo.v_M), ("colors", bo.v_colors),
                 ("opacities", bo.v_opacities), ("normals", bo.v_normals)):
        check_grad(f"{prefix} v_{k}", v, g[f"{prefix}__v_{k}"])
    if v_tex is not None:
        rows, vals, norms, ours = RG.texture_rows_check(g, prefix, v_tex)
        check_grad(f"{prefix} texture rows", ours, vals)
        check_grad(f"{prefix} texture row norms", np.linalg.norm(v_tex.reshape(v_tex.shape[0], -1), axis=1), norms)


@pytest.mark.parametrize("case,filtering", [(c, f) for c, fs in CASES.items() for f in fs])
def test_oracle_textured_compositor_matches_reference(case, filtering):
    g, s = fixture(case)
    _check(g, f"comp_{filtering}", *_oracle(g, s, filtering))


@pytest.mark.parametrize("case", ["small", "adjoint"])
def test_oracle_plain_compositor_matches_reference(case):
    g, s = fixture(case)
    _check(g, "plain", *_oracle(g, s, None))
