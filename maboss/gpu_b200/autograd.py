"""torch.autograd binding of the engine's window probabilities and their score-function gradients.

    probs = window_probabilities(theta, ctx, model, ["$u_0", "$d_0"], n_traj=10**6, seed=0)
    loss = (probs * weights).sum(); loss.backward()      # theta.grad = d loss / d theta

Forward: the batched fast-mode kernel with the parameter values of `theta` (no recompilation).
Backward: the adjoint kernel on the same random streams (the same trajectories as the forward),
which accumulates the likelihood-ratio estimate of the vector-Jacobian product. Both run through
the C ABI on one batch per (context, model, parameter names, trajectory count), kept across calls:
a new theta only re-uploads the variant's rate tables (mb_batch_set_variables), so device buffers,
launch shapes and CUDA graphs are reused. torch only carries the tensors.
"""
from __future__ import annotations

import numpy as np
import torch

from .engine import Batch, Context, Model

_ENGINES: dict = {}  # (id(ctx), id(model), names, n_traj) -> (Batch, variant); holds ctx and model


def _engine(ctx: Context, model: Model, names: tuple, n_traj: int, params: dict):
    key = (id(ctx), id(model), names, n_traj)
    hit = _ENGINES.get(key)
    if hit is None:
        if len(_ENGINES) >= 8:
            _ENGINES.pop(next(iter(_ENGINES)))
        b = Batch(ctx)
        v = b.add_variant(b.add_model(model), n_traj, params, grad_params=list(names))
        hit = _ENGINES[key] = (b, v)
    else:
        hit[0].set_variables(hit[1], params)
    return hit


class _WindowProbabilities(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, engine_ctx, model, names, n_traj, seed):
        params = {n: float(v) for n, v in zip(names, theta.detach().cpu().tolist())}
        b, v = _engine(engine_ctx, model, tuple(names), int(n_traj), params)
        b.run(seed)
        probs = torch.from_numpy(b.result(v).window_probs)
        ctx.engine = (engine_ctx, model, tuple(names), int(n_traj), int(seed), params)
        ctx.theta_device, ctx.theta_dtype = theta.device, theta.dtype
        return probs.to(device=theta.device, dtype=theta.dtype)

    @staticmethod
    def backward(ctx, grad_probs):
        engine_ctx, model, names, n_traj, seed, params = ctx.engine
        cot = grad_probs.detach().to("cpu", torch.float64).numpy()
        b, v = _engine(engine_ctx, model, names, n_traj, params)  # the forward's values (another call may have moved them)
        b.run_gradient(seed, {v: cot})
        g = b.gradient(v)
        grad_theta = torch.from_numpy(np.asarray(g)).to(device=ctx.theta_device, dtype=ctx.theta_dtype)
        return grad_theta, None, None, None, None, None


def window_probabilities(theta: torch.Tensor, ctx: Context, model: Model, names: list[str], n_traj: int,
                         seed: int = 0) -> torch.Tensor:
    """Window probabilities [windows, 2^k] as a differentiable function of the $variables `names`."""
    return _WindowProbabilities.apply(theta, ctx, model, names, n_traj, seed)
