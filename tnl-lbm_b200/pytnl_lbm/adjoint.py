"""The discrete adjoint as a torch.autograd.Function.

``objective(force, lattice, f0, nsteps, samples, target)`` runs the lattice
from the populations ``f0`` (ghost layout, at iteration 0) for ``nsteps`` A-A
steps with the per-site body force ``force`` (a float64 tensor [3, Z, Y, X])
and returns the objective J of ``LBM.adjoint_forward`` as a 0-d tensor;
``J.backward()`` fills ``force.grad`` with the gradient the C-ABI computes
(lbm_adjoint_backward: exact discrete adjoint with checkpointing, FP64
accumulation).  PyTorch only carries the tensors; the forward and adjoint
steps run in the library's sm_100a kernels.  A CUDA ``force`` stays on the
device: the library reads it in place and writes the gradient into a device
tensor.
"""
from __future__ import annotations

import numpy as np
import torch

from . import LBM


class _AdjointObjective(torch.autograd.Function):
    @staticmethod
    def forward(ctx, force, lattice: LBM, f0, nsteps, samples, target, checkpoint_every, rho_weight):
        lattice.set_populations(f0)
        lattice.iteration = 0
        src = force.detach() if force.is_cuda else force.detach().cpu().numpy()
        loss = lattice.adjoint_forward(src, nsteps, samples, target, checkpoint_every=checkpoint_every,
                                       rho_weight=rho_weight)
        ctx.lattice = lattice
        ctx.device = force.device
        return torch.tensor(loss, dtype=torch.float64, device=force.device)

    @staticmethod
    def backward(ctx, grad_out):
        if ctx.device.type == "cuda":
            g = torch.empty((3,) + ctx.lattice.shape, dtype=torch.float64, device=ctx.device)
            ctx.lattice.adjoint_backward(seed=float(grad_out), out=g)
        else:
            g = torch.from_numpy(ctx.lattice.adjoint_backward(seed=float(grad_out)))
        return g, None, None, None, None, None, None, None


def objective(force, lattice: LBM, f0: np.ndarray, nsteps: int, samples, target, checkpoint_every: int = 0,
              rho_weight: float = 0.0):
    return _AdjointObjective.apply(force, lattice, f0, nsteps, samples, target, checkpoint_every, rho_weight)
