"""Checkpointed gradients of iterated maps on the GPU (``src/checkpoint.rs:67-126``).

``grad_checkpointed(ctx, step, loss, X0, num_steps, num_checkpoints)``: for every
row x_0 of ``X0`` (a device tensor [B, n]), the gradient of ``loss(x_T)`` with
``x_{t+1} = step(x_t)``; ``step`` and ``loss`` are uploaded tapes (``step`` maps n
inputs to n outputs, ``loss`` n inputs to one output).  Only the states at the
evenly spread checkpoint positions are stored; each reverse segment recomputes
its states and pulls the adjoint back with vector-Jacobian products.
"""
from __future__ import annotations

from . import _lib
from .gpu import _check


def grad_checkpointed(ctx, step, loss, X0, num_steps: int, num_checkpoints: int):
    import torch
    X0 = X0.contiguous()
    grads = torch.empty_like(X0)
    torch.cuda.synchronize()
    _check(_lib.load().ech_grad_checkpointed_device(ctx._h, step._h, loss._h, int(step.f64), X0.data_ptr(),
                                                    int(X0.shape[0]), int(num_steps), int(num_checkpoints),
                                                    grads.data_ptr()))
    return grads
