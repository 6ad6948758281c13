"""torch.autograd wrapper of the hand-written adjoint of the step.

    hist = indenter_force_history(state, cohesion, youngs_modulus, prms, nsteps)
    loss = ((hist - measured) ** 2).sum()
    loss.backward()        # cohesion.grad, youngs_modulus.grad, state.grad

The forward runs mpm_adjoint_forward (nsteps substeps of Model3D::Step,
model_3d.cpp:35-51, a device checkpoint every ckpt_every substeps) in FP64
with the FP64 SVD, or with precision=PRECISION_MIXED in mixed precision (the
checkpoints are then FP64 copies of the mixed state); the backward runs
mpm_adjoint_backward (each segment recomputed in FP64 from its checkpoint,
then reverse G2P, reverse grid update, reverse P2G as a gather) with
grad_output as dL/d(force history). With a mixed forward the gradient is
that of the FP64 step along the mixed trajectory, restarted at every
checkpoint.

Inputs are float64 tensors on any device (they are staged through host
memory to the C-ABI, which takes host buffers):
  state           (28, n) particle SoA in the HostSideSOA row layout
                  (parameters_sim_3d.h:29-38); its gradient fills the rows
                  x, v, Fe, Bp and Jp_inv, zero elsewhere
  cohesion        (n,) per-particle cohesion c (apex shift p0 = c / tan phi)
  youngs_modulus  0-d tensor; mu, kappa follow it (parameters_sim_3d.cpp:65-70)
Non-smooth switches (crushed flag, contact test, min() in the return map)
are differentiated on the side the forward took.
"""
import ctypes

import numpy as np
import torch
from torch.autograd.function import once_differentiable

from ._lib import BP00, FE00, IDX_JP_INV, LIB, N_PTS_ARRAYS, POSX, PRECISION_FP64_SVD64, VELX
from .simulation import MPMHandle

# rows of mpm_adjoint_state -> rows of the particle SoA
_ADJ_TO_SOA = ((0, POSX, 3), (3, VELX, 3), (6, BP00, 9), (15, FE00, 9), (24, IDX_JP_INV, 1))


def _params_with_E(prms, E):
    p = prms.copy()
    p.YoungsModulus = float(E)
    LIB.mpm_params_compute_camclay(ctypes.byref(p))
    LIB.mpm_params_compute_helper_variables(ctypes.byref(p))
    return p


class IndenterForceHistory(torch.autograd.Function):
    @staticmethod
    def forward(ctx, state, cohesion, youngs_modulus, prms, nsteps, ckpt_every, device, precision):
        if state.dtype != torch.float64 or cohesion.dtype != torch.float64:
            raise TypeError("state and cohesion must be float64")
        if state.dim() != 2 or state.shape[0] != N_PTS_ARRAYS or cohesion.shape != (state.shape[1],):
            raise ValueError("state must be (28, n) and cohesion (n,)")
        n = state.shape[1]
        h = MPMHandle(_params_with_E(prms, youngs_modulus.item()), n, precision, device)
        try:
            h.upload(state.detach().cpu().numpy(), cohesion=cohesion.detach().cpu().numpy())
            hist = h.adjoint_forward(int(nsteps), int(ckpt_every))
        except Exception:
            h.close()
            raise
        ctx.handle = h
        ctx.n = n
        ctx.out_device = cohesion.device
        return torch.from_numpy(hist).to(cohesion.device)

    @staticmethod
    @once_differentiable
    def backward(ctx, grad_hist):
        h = ctx.handle
        try:
            dc, dE = h.adjoint_backward(grad_hist.detach().cpu().numpy())
            g_state = None
            if ctx.needs_input_grad[0]:
                adj = h.adjoint_state()
                g = np.zeros((N_PTS_ARRAYS, ctx.n))
                for a, s, k in _ADJ_TO_SOA:
                    g[s:s + k] = adj[a:a + k]
                g_state = torch.from_numpy(g).to(ctx.out_device)
        finally:
            h.close()
            ctx.handle = None
        dev = ctx.out_device
        return (g_state, torch.from_numpy(dc).to(dev), torch.tensor(dE, dtype=torch.float64, device=dev),
                None, None, None, None, None)


def indenter_force_history(state, cohesion, youngs_modulus, prms, nsteps, ckpt_every=20, device=0,
                           precision=PRECISION_FP64_SVD64):
    """(nsteps, 3) indenter force of each substep, differentiable with respect
    to state, cohesion and youngs_modulus (see the module docstring)."""
    if not torch.is_tensor(youngs_modulus):
        youngs_modulus = torch.tensor(float(youngs_modulus), dtype=torch.float64)
    return IndenterForceHistory.apply(state, cohesion, youngs_modulus, prms, nsteps, ckpt_every, device, precision)
