"""CPU check of the drop-in's error behaviour: bad arguments are rejected the
way the reference rejects them (its assertions and exceptions, quoted with
file:line), before any device work, so these run with CPU tensors.
"""
import pytest
import torch

from textured_gaussians_b200 import rasterization_textured_gaussians
from textured_gaussians_b200.cuda import rasterize_to_pixels_textured_gaussians

N, C, R = 3, 1, 4


def renderer_args(**over):
    a = dict(means=torch.zeros(N, 3), quats=torch.tensor([[1.0, 0, 0, 0]] * N), scales=torch.ones(N, 3),
             opacities=torch.ones(N), colors=torch.zeros(N, 3), textures=torch.zeros(N, R, R, 4),
             viewmats=torch.eye(4)[None], Ks=torch.eye(3)[None], width=16, height=16)
    a.update(over)
    return a


@pytest.mark.parametrize("over,match", [
    (dict(render_mode="XYZ"), "XYZ"),                                   # rendering.py:1485
    (dict(distloss=True), "distloss requires depth rendering"),          # rendering.py:1486-1492
    (dict(textures=torch.zeros(N, R, R, 3)), r"torch.Size"),             # rendering.py:1482-1484
    (dict(textures=torch.zeros(N + 1, R, R, 4)), r"torch.Size"),
    (dict(colors=torch.zeros(N + 1, 3)), r"torch.Size"),                 # rendering.py:1494-1499
    (dict(quats=torch.zeros(N, 3)), r"torch.Size"),                      # rendering.py:1477
    (dict(Ks=torch.eye(3)), r"torch.Size"),                              # rendering.py:1481
    (dict(sh_degree=3, colors=torch.zeros(N, 4, 3)), r"torch.Size"),     # (degree + 1)^2 coefficients needed
])
def test_renderer_rejects_bad_arguments(over, match):
    with pytest.raises(AssertionError, match=match):
        rasterization_textured_gaussians(**renderer_args(**over))


def op_args(**over):
    a = dict(means2d=torch.zeros(C, N, 2), ray_transforms=torch.zeros(C, N, 3, 3), colors=torch.zeros(C, N, 3),
             opacities=torch.zeros(C, N), textures=torch.zeros(N, R, R, 4), texture_range_x=3.0,
             texture_range_y=3.0, normals=torch.zeros(C, N, 3), densify=torch.zeros(C, N, 2), image_width=32,
             image_height=32, tile_size=16, isect_offsets=torch.zeros(C, 2, 2, dtype=torch.int32),
             flatten_ids=torch.zeros(0, dtype=torch.int32))
    a.update(over)
    return a


def test_op_rejects_an_unknown_filter():
    # cuda/_wrapper.py:1989 and :2156: raise Exception(f"Unsupported filter type {filtering}")
    with pytest.raises(Exception, match="Unsupported filter type bogus"):
        rasterize_to_pixels_textured_gaussians(**op_args(filtering="bogus"))


def test_op_rejects_a_tile_grid_smaller_than_the_image():
    # cuda/_wrapper.py:1904-1909: the tile grid must cover the image
    with pytest.raises(AssertionError, match="Assert Failed"):
        rasterize_to_pixels_textured_gaussians(**op_args(image_width=48))


@pytest.mark.parametrize("over", [dict(means2d=torch.zeros(C, N, 3)), dict(opacities=torch.zeros(C, N + 1)),
                                  dict(ray_transforms=torch.zeros(C, N, 9)), dict(backgrounds=torch.zeros(C, 4))])
def test_op_rejects_mismatched_shapes(over):
    # cuda/_wrapper.py:1872-1877: the per-splat inputs share [C, N]
    with pytest.raises(AssertionError):
        rasterize_to_pixels_textured_gaussians(**op_args(**over))
