"""CPU check of the drop-in boundary's Python surface: every public function of
the reference on this path (textured_gaussians/rendering.py:1009-1372 and the
op wrappers in textured_gaussians/cuda/_wrapper.py) has a counterpart here
whose leading parameters are the reference's -- same names, order, kinds and
defaults (a parameter the reference requires may have a default here) -- so
calls written for the reference, positional or by keyword, bind the same way.
Parameters added here come after them and all have defaults.  The renderers
return the reference's 9-tuple with the same ``meta`` keys.
The reference's signatures and ``meta`` keys are the committed fixture
tests/golden/api_signatures.json (written by tests/golden/make_api_signatures.py).
"""
import inspect
import json
import os

import pytest

import textured_gaussians_b200.cuda._wrapper as ours_wrapper
import textured_gaussians_b200.rendering as ours_rendering

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, "golden", "api_signatures.json")))
MODULES = {"textured_gaussians.rendering": ours_rendering, "textured_gaussians.cuda._wrapper": ours_wrapper}


SIGNATURES = sorted(k for k in GOLDEN if not k.startswith("meta_keys:"))


def test_fixture_covers_the_path():
    assert len(SIGNATURES) >= 10
    assert "textured_gaussians.rendering.rasterization_textured_gaussians" in GOLDEN


@pytest.mark.parametrize("renderer", ["rasterization_textured_gaussians", "rasterization_2dgs"])
def test_meta_has_the_reference_keys(renderer):
    """Both renderers build their ``meta`` in one place (the reference's rendering.py:1301-1322, 1648-1669);
    run it on tiny CPU tensors and compare the keys, in order."""
    import torch
    C, N, H, W = 1, 2, 4, 4
    p = {k: torch.zeros(1) for k in ("camera_ids", "gaussian_ids", "radii", "means2d", "depths", "ray_transforms",
                                     "opacities", "normals", "tiles_per_gauss", "isect_ids", "flatten_ids",
                                     "isect_offsets", "densify")}
    p.update(tile_width=1, tile_height=1, C=C)
    viewmats, Ks = torch.eye(4)[None], torch.eye(3)[None]
    out = ours_rendering._finish(p, torch.zeros(C, H, W, 3), torch.ones(C, H, W, 1), torch.zeros(C, H, W, 3),
                                 torch.zeros(C, H, W, 1), torch.zeros(C, H, W, 1), torch.zeros(N), torch.zeros(N),
                                 viewmats, Ks, W, H, 16, "RGB", "expected")
    assert len(out) == 9
    assert list(out[-1].keys()) == GOLDEN[f"meta_keys:{renderer}"]


@pytest.mark.parametrize("qualname", SIGNATURES)
def test_signature_extends_the_reference(qualname):
    mod, name = qualname.rsplit(".", 1)
    fn = getattr(MODULES[mod], name, None)
    assert fn is not None, f"{name} missing"
    params = list(inspect.signature(fn).parameters.values())
    ref = GOLDEN[qualname]
    assert [p.name for p in params[:len(ref)]] == [r["name"] for r in ref]
    for p, r in zip(params, ref):
        assert p.kind.name == r["kind"], (name, p.name)
        if r["default"] is not None:  # a reference default is kept; a required parameter may gain one here
            assert p.default is not inspect.Parameter.empty and repr(p.default) == r["default"], (name, p.name)
    for p in params[len(ref):]:
        assert p.default is not inspect.Parameter.empty or p.kind in (
            inspect.Parameter.VAR_POSITIONAL, inspect.Parameter.VAR_KEYWORD), (name, p.name)
