"""Fermion action S_f = Re psi^dag (M^dag M)^{-1} psi with a hand-written adjoint.

``FermionAction.apply(phi, psi, solver, Lx, dtau)`` returns S_f per batch row;
its backward is the fused force kernel (``qedf_force_f_*``):
dS_f/dphi = -F, with F the reference's fermion force (``force_f_fast``,
``hmc_sampler_batch.py:2150-2227``).  Only xi = (M^dag M)^{-1} psi is kept
between forward and backward; the per-slice partial products the reference
stores are recomputed inside the kernel.
"""
from __future__ import annotations

import torch

from . import ops


class FermionAction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, phi, psi, solver, Lx, dtau):
        # phi: kernel-layout angles [bs, N*2]; psi: [bs, N] complex
        res = solver.solve(phi.detach().to(solver.angle_dtype), psi.detach().to(solver.vec_dtype))
        xi = res.x.view(psi.shape[0], -1)
        ctx.save_for_backward(phi.detach(), xi)
        ctx.Lx, ctx.dtau = Lx, dtau
        ctx.iters, ctx.status = res.iters, res.status
        return ops.cdot(psi.detach().to(xi.dtype), xi).to(phi.dtype)

    @staticmethod
    def backward(ctx, g):
        phi, xi = ctx.saved_tensors
        if phi.dtype == torch.float64:
            F = ops.fermion_force(phi, xi.to(torch.complex128), ctx.Lx, ctx.dtau)
        else:
            F = ops.fermion_force(phi.to(torch.float32), xi.to(torch.complex64), ctx.Lx, ctx.dtau).to(phi.dtype)
        return -F * g.view(-1, 1).to(F.dtype), None, None, None, None


def fermion_action(phi, psi, solver, Lx, dtau=0.1):
    return FermionAction.apply(phi, psi, solver, Lx, dtau)
