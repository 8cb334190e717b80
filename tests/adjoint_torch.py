"""torch.autograd wrapper of the discrete adjoint, for the test harness only.

``MaxwellStressMean.apply(lin0, solver, mf0, kx0, nsteps, checkpoint_every)``
returns J (the fluctuation Maxwell stress averaged over nsteps steps of the
GPU step); its backward is qlgpu_adjoint_maxwell.  lin0 is a complex128 CPU
tensor; the gradient follows torch's convention for real-valued functions of
complex inputs (conj-free: dJ = Re sum conj(grad) d lin0).
"""
import numpy as np
import torch


class MaxwellStressMean(torch.autograd.Function):
    @staticmethod
    def forward(ctx, lin0, solver, mf0, kx0, nsteps, checkpoint_every):
        x = lin0.detach().cpu().numpy()
        J, g, gm = solver.adjoint_maxwell(0.0, x, mf0, kx0, nsteps, checkpoint_every)
        ctx.save_for_backward(torch.from_numpy(g))
        return torch.tensor(J, dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        return grad_out * g, None, None, None, None, None


def maxwell_stress_mean(lin0, solver, mf0, kx0, nsteps, checkpoint_every=100):
    return MaxwellStressMean.apply(lin0, solver, np.asarray(mf0), np.asarray(kx0), nsteps, checkpoint_every)
