"""torch.autograd wrapper (icempm_3dm_b200.autograd) over the C-ABI adjoint:
a squared-error loss on the indenter force history backpropagates to
cohesion, Young's modulus and the initial state. Checked against the direct
C-ABI calls (identical numbers) and against the oracle's FP64 dual-number
forward mode of the same loss (1e-6 relative)."""
import numpy as np
import pytest
import torch

from icempm_3dm_b200 import MPMHandle, PRECISION_FP64_SVD64
from icempm_3dm_b200.autograd import indenter_force_history
from oracle import pyoracle as po
from tests.test_gpu_adjoint import case

pytestmark = pytest.mark.gpu


def test_autograd_matches_c_abi_and_dual_forward_mode():
    nsteps, every = 8, 3
    prms, soa, coh = case()
    n = soa.shape[1]
    state = torch.tensor(soa, dtype=torch.float64, requires_grad=True)
    c = torch.tensor(coh, dtype=torch.float64, requires_grad=True)
    E = torch.tensor(prms.YoungsModulus, dtype=torch.float64, requires_grad=True)
    rng = np.random.default_rng(3)
    target = torch.tensor(rng.standard_normal((nsteps, 3)) * 50.0)

    hist = indenter_force_history(state, c, E, prms, nsteps, ckpt_every=every)
    loss = ((hist - target) ** 2).sum()
    loss.backward()
    assert c.grad is not None and E.grad is not None and state.grad is not None

    # the same sweep through the C-ABI directly
    with MPMHandle(prms, n, PRECISION_FP64_SVD64) as h:
        h.upload(soa, cohesion=coh)
        h2 = h.adjoint_forward(nsteps, every)
        dc, dE = h.adjoint_backward(2.0 * (h2 - target.numpy()))
    # two GPU runs differ only by the summation order of FP64 atomics
    assert np.allclose(hist.detach().numpy(), h2, rtol=1e-10, atol=1e-10 * np.abs(h2).max())
    assert np.allclose(c.grad.numpy(), dc, rtol=1e-8, atol=1e-8 * np.abs(dc).max())
    assert E.grad.item() == pytest.approx(dE, rel=1e-8)

    # dual forward mode of the same loss along a cohesion direction and E
    p0 = coh / prms.DP_tan_phi
    r = coh * rng.standard_normal(n)
    hv, dh, _, _ = po.dual_steps(prms, soa, nsteps, p0=p0, dp0=r / prms.DP_tan_phi, dE=1.0)
    resid = 2.0 * (hv - target.numpy())
    # tangent of the loss along (r, dE = 1) = r . dL/dc + dL/dE
    t = float(np.sum(resid * dh))
    a = float(r @ c.grad.numpy()) + E.grad.item()
    assert t != 0.0
    assert abs(t - a) <= 1e-6 * abs(t), (t, a)
    assert torch.count_nonzero(state.grad[0:3]) == 0       # utility, p, q rows carry no gradient
    assert torch.count_nonzero(state.grad[4:10]) > 0


@pytest.mark.parametrize("forward", ["fp64", "mixed"])
def test_calibration_recovers_strength_scales(forward):
    """The target history comes from the FP64 forward (c x 1.2, E x 0.9);
    the fit runs its forward in FP64 or, as the calibration workload asks,
    in mixed precision (gradients from the FP64 recompute of each segment)."""
    from icempm_3dm_b200 import PRECISION_MIXED
    """Force history measured with cohesion x1.2 and E x0.9 (the calibration
    workload's targets) on a 20k-particle copy of that block; the fit starts at
    x1. Crush flags switch inside the fit, so the loss is piecewise smooth and
    the fit lands within 1e-2 of the targets rather than on them."""
    from icempm_3dm_b200 import generator as gen
    from icempm_3dm_b200._lib import IDX_UTILITY, LIB
    from icempm_3dm_b200.calibrate import calibrate_strength
    nsteps = 200
    prms, soa, coh = gen.calibration_block()
    p_true = prms.copy()
    p_true.YoungsModulus = 0.9 * prms.YoungsModulus
    LIB.mpm_params_compute_camclay(p_true)
    LIB.mpm_params_compute_helper_variables(p_true)
    with MPMHandle(p_true, soa.shape[1], PRECISION_FP64_SVD64) as h:
        h.upload(soa, cohesion=1.2 * coh)
        measured = h.step(nsteps)
        crushed = float(np.mean((h.download()[IDX_UTILITY].view(np.int64) & 0x10000) != 0))
    assert crushed > 0.02            # cohesion must matter
    # L-BFGS runs to convergence here (its evaluation cap is 1.25 x iters): with 40
    # iterations it could stop at the cap, 1 % away along the shallow c/E trade-off
    sc, sE, losses = calibrate_strength(soa, coh, prms.YoungsModulus, prms, measured, nsteps, ckpt_every=20,
                                        iters=100,
                                        precision=PRECISION_MIXED if forward == "mixed" else PRECISION_FP64_SVD64)
    print(f"\n{forward} forward: crushed {crushed:.3f}; cohesion scale {sc:.5f}  E scale {sE:.5f}  "
          f"loss {losses[0]:.3e} -> {losses[-1]:.3e} in {len(losses)} evaluations")
    assert losses[-1] < 1e-2 * losses[0]
    assert abs(sc - 1.2) < 1e-2 and abs(sE - 0.9) < 1e-2
