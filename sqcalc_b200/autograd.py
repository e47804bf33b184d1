"""PyTorch autograd entry point for S(q) of one frame.

``structure_factor(pos, plan)`` returns S(q) (nq shells, float64) of the
positions ``pos`` (natoms x 3, float64, CPU or CUDA) as a differentiable torch
tensor.  The backward pass calls the library's adjoint (sqn_sq_grad: three
type-2 NUFFTs of i h_i dL/dS conj(T) / den, interpolated at the atoms) and
recomputes the forward transform instead of storing the fine grid.  The plan
must be created with ``grad=True`` and q-independent weights.

Example (the differentiation form: a loss over shells against a target)::

    plan = Plan(cell, origin, types, qmin=0.5, qmax=8.0, nq=150, eps=1e-12, grad=True)
    S = structure_factor(pos, plan)
    loss = ((S - S_target) ** 2).sum()
    loss.backward()          # pos.grad = dLoss/dr
"""
from __future__ import annotations

import numpy as np
import torch


class _StructureFactor(torch.autograd.Function):
    @staticmethod
    def forward(ctx, pos, plan):
        S, _ = plan.sq_grad(_library_positions(pos))
        ctx.plan = plan
        ctx.save_for_backward(pos)
        return torch.as_tensor(S, dtype=torch.float64, device=pos.device)

    @staticmethod
    def backward(ctx, grad_S):
        (pos,) = ctx.saved_tensors
        dLdS = grad_S.detach().to("cpu", torch.float64).numpy()
        _, grad = ctx.plan.sq_grad(_library_positions(pos), np.ascontiguousarray(dLdS))
        if not torch.is_tensor(grad):
            grad = torch.from_numpy(grad)
        return grad.to(device=pos.device, dtype=pos.dtype), None


def _library_positions(pos):
    p = pos.detach().to(torch.float64)
    if p.is_cuda:
        return p.contiguous()
    return p.contiguous().numpy()


def structure_factor(pos: torch.Tensor, plan) -> torch.Tensor:
    """S(q) of one frame, differentiable with respect to ``pos``."""
    return _StructureFactor.apply(pos, plan)
