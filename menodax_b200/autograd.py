"""torch.autograd front end over the C ABI: the discrete adjoint of a solve."""

from __future__ import annotations

import torch


def needs_grad(*xs) -> bool:
    return torch.is_grad_enabled() and any(isinstance(x, torch.Tensor) and x.requires_grad for x in xs)


def solve_with_grad(*args, **kwargs):
    raise NotImplementedError("the discrete adjoint is not built yet")
