"""torch.autograd binding of the discrete adjoint, used by the gradient tests.

FRSteps.apply(U0, solver, nsteps, checkpoint_every) runs nsteps of the
solver's update from U0 (a float64 CPU tensor in the reference layout
[spt][ele][field]) and returns U_N; its backward is the solver's reverse RK
sweep (frg_adjoint_backward) seeded with dL/dU_N.
"""
import numpy as np
import torch


class FRSteps(torch.autograd.Function):
    @staticmethod
    def forward(ctx, U0, solver, nsteps, checkpoint_every):
        solver.set("U_spts", U0.detach().cpu().numpy())
        solver.adjoint_forward(nsteps, checkpoint_every)
        ctx.solver = solver
        return torch.from_numpy(solver.get("U_spts"))

    @staticmethod
    def backward(ctx, gUN):
        lam0, _ = ctx.solver.adjoint_backward(np.ascontiguousarray(gUN.detach().cpu().numpy(), np.float64))
        return torch.from_numpy(lam0), None, None, None
