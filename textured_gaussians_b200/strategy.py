"""Densification statistics: the running-state update of the reference's
DefaultStrategy (textured_gaussians/strategy/default.py:213-261), one fused
kernel instead of its clone / scale / norm / index_add chain.

Only the statistics step is here (what consumes the renderer's gradients);
growing, splitting and pruning Gaussians are outside this package.
"""
from __future__ import annotations

from typing import Any, Dict

import torch

from .cuda._wrapper import densify_stats


def update_state(state: Dict[str, Any], info: Dict[str, Any], n_gaussians: int, packed: bool = False,
                 absgrad: bool = False, key_for_gradient: str = "gradient_2dgs", track_radii: bool = False) -> None:
    """In-place update of state["grad2d"], state["count"] (and state["radii"] with ``track_radii``), created
    as zeros [N] on first use, from the renderer's ``meta`` dict after ``loss.backward()``.

    The radius statistic is a true per-Gaussian maximum; the reference's indexed assignment
    (default.py:256-260) keeps the last camera's value when a Gaussian is seen by several cameras.
    """
    for key in ("width", "height", "n_cameras", "radii", "gaussian_ids", key_for_gradient):
        assert key in info, f"{key} is required but missing."
    g = info[key_for_gradient]
    grads = g.absgrad if absgrad else g.grad
    dev = grads.device
    if state.get("grad2d") is None:
        state["grad2d"] = torch.zeros(n_gaussians, device=dev)
    if state.get("count") is None:
        state["count"] = torch.zeros(n_gaussians, device=dev)
    if track_radii and state.get("radii") is None:
        state["radii"] = torch.zeros(n_gaussians, device=dev)
    densify_stats(grads, info["radii"], info["width"], info["height"], info["n_cameras"], state["grad2d"],
                  state["count"], state["radii"] if track_radii else None,
                  gaussian_ids=info["gaussian_ids"] if packed else None)
