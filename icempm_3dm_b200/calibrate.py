"""Calibration of ice strength from an indenter force history with the
hand-written adjoint (icempm_3dm_b200.autograd).

Fits two log-scale factors, one on the per-particle cohesion field and one on
Young's modulus, minimising the squared error between the simulated and the
measured (nsteps, 3) force history with L-BFGS. Each objective evaluation is
one checkpointed forward and one reverse sweep on the GPU.
"""
import numpy as np
import torch

from ._lib import PRECISION_FP64_SVD64
from .autograd import indenter_force_history


def calibrate_strength(state, cohesion, youngs_modulus, prms, measured, nsteps, ckpt_every=20, iters=30,
                       device=0, tol=1e-10, precision=PRECISION_FP64_SVD64):
    """Returns (cohesion_scale, youngs_modulus_scale, history of the loss).

    state (28, n) and cohesion (n,) are numpy or float64 tensors, measured the
    (nsteps, 3) force history to fit. The loss is normalised by the squared
    norm of the measurement. precision=PRECISION_MIXED runs the forward in
    mixed precision (the adjoint recomputes in FP64 from its checkpoints)."""
    state = torch.as_tensor(np.asarray(state), dtype=torch.float64)
    c0 = torch.as_tensor(np.asarray(cohesion), dtype=torch.float64)
    E0 = float(youngs_modulus)
    meas = torch.as_tensor(np.asarray(measured), dtype=torch.float64)
    norm = float((meas ** 2).sum())
    theta = torch.zeros(2, dtype=torch.float64, requires_grad=True)
    opt = torch.optim.LBFGS([theta], lr=1.0, max_iter=iters, tolerance_grad=tol, tolerance_change=tol,
                            line_search_fn="strong_wolfe")
    losses = []

    def closure():
        opt.zero_grad()
        hist = indenter_force_history(state, c0 * torch.exp(theta[0]), E0 * torch.exp(theta[1]), prms, nsteps,
                                      ckpt_every, device, precision)
        loss = ((hist - meas) ** 2).sum() / norm
        loss.backward()
        losses.append(loss.item())
        return loss

    opt.step(closure)
    s = torch.exp(theta.detach())
    return float(s[0]), float(s[1]), losses
