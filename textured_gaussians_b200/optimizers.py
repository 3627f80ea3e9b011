"""SelectiveAdam, as the reference's textured_gaussians/optimizers/selective_adam.py:6-91.

Each parameter group holds one tensor whose leading dimension is the
Gaussian count N; ``step(visibility)`` updates only the rows of the visible
Gaussians with the fused kernel (no bias correction, as in the reference).
B200 addition: ``shadows`` maps a parameter to its BF16 / FP16 storage copy
(e.g. the texture storage the compositor samples), which the same kernel
refreshes for the updated rows.
"""
from __future__ import annotations

from typing import Dict, Optional

import torch

from .cuda._wrapper import selective_adam_update


class SelectiveAdam(torch.optim.Adam):
    def __init__(self, params, eps, betas, shadows: Optional[Dict[torch.Tensor, torch.Tensor]] = None):
        super().__init__(params=params, eps=eps, betas=betas)
        self.shadows = shadows or {}

    @torch.no_grad()
    def step(self, visibility):
        N = visibility.numel()
        for group in self.param_groups:
            lr = group["lr"]
            eps = group["eps"]
            beta1, beta2 = group["betas"]
            assert len(group["params"]) == 1, "more than one tensor in group"
            param = group["params"][0]
            if param.grad is None:
                continue
            state = self.state[param]
            if len(state) == 0:
                state["step"] = torch.tensor(0.0, dtype=torch.float32)
                state["exp_avg"] = torch.zeros_like(param, memory_format=torch.preserve_format)
                state["exp_avg_sq"] = torch.zeros_like(param, memory_format=torch.preserve_format)
            M = param.numel() // N
            selective_adam_update(param, param.grad, state["exp_avg"], state["exp_avg_sq"], visibility, lr, beta1,
                                  beta2, eps, N, M, shadow=self.shadows.get(param))
