"""Stochastic-estimator solves: G_eta = (M^dag M)^{-1} M^dag eta for Nrv noise
vectors sharing one gauge field, as one multi-right-hand-side batched PCG.

Mirrors ``StochaticEstimator.random_vec_bin`` / ``set_eta_G_eta`` /
``set_eta_G_eta_inner`` (``qed_fermion/stochastic_estimator.py:210-224,
409-433``).  The reference repeats the boson Nrv times and solves with
``bs = Nrv``; here the Nrv right-hand sides reference one angle array.
"""
from __future__ import annotations

import math

import torch

from . import ops
from .hmc import ref_to_kernel
from .observables import BondBond
from .solver import PcgSolver, System


class StochaticEstimator:
    def __init__(self, Lx, Ltau, Nrv=20, dtau=0.1, precision="mixed", cg_rtol=1e-10, max_iter=20000,
                 use_precon=True, device=None, seed=None, noise="z2z2", autotune=True, corr_dtype=None):
        self.Lx, self.Ly, self.Ltau, self.Nrv, self.dtau = Lx, Lx, Ltau, Nrv, dtau
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        self.noise = noise
        self.generator = torch.Generator(device=self.device)
        if seed is not None:
            self.generator.manual_seed(seed)
        mode = precision
        self.solver = PcgSolver([System(Lx, Ltau, Nrv, True)], mode=mode, rtol=cg_rtol, max_iter=max_iter,
                                dtau=dtau, use_precon=use_precon and Ltau >= 26, device=self.device,
                                tune=autotune)
        self.eta = None
        self.G_eta = None
        # complex dtype of the bond-bond correlators' arithmetic: None keeps
        # that of eta / G_eta; torch.complex64 is the reference estimator's
        # own precision and halves their memory traffic
        self.corr_dtype = corr_dtype

    def random_vec_bin(self):
        """Nrv vectors with entries (+-1 +- i)/sqrt(2) (reference :210-224); with
        ``noise="z2"`` real +-1 entries instead."""
        n = self.Lx * self.Ly * self.Ltau
        re = torch.randint(0, 2, (self.Nrv, n), device=self.device, generator=self.generator) * 2 - 1
        if self.noise == "z2":
            return re.to(torch.complex128)
        im = torch.randint(0, 2, (self.Nrv, n), device=self.device, generator=self.generator) * 2 - 1
        return (re + 1j * im).to(torch.complex128) / math.sqrt(2.0)

    def set_eta_G_eta(self, boson, eta):
        """boson: ``[1, 2, Lx, Ly, Ltau]``; eta: ``[Nrv, N]``.  Sets ``self.G_eta``."""
        self.eta = eta
        phi = ref_to_kernel(boson)[0]
        vdt = self.solver.vec_dtype
        adt = torch.float64 if vdt == torch.complex128 else torch.float32
        psi = ops.apply_operator("mh", phi.to(adt), eta.to(vdt), self.Lx, self.dtau, rhs_per_boson=self.Nrv)
        res = self.solver.solve(phi.to(self.solver.angle_dtype), psi)
        self.G_eta = res.x.view(self.Nrv, -1)
        self.iters, self.relres, self.status = res.iters, res.relres, res.status
        return self.G_eta

    # ---- bond-bond correlators (reference :1393-1652, :2594-2651) -------------
    def _bb(self):
        if getattr(self, "_bond_bond", None) is None:
            self._bond_bond = BondBond(self.Lx, self.Ltau)
        return self._bond_bond

    def T1(self, eta, G_eta, boson):
        return self._bb().T1(eta, G_eta, boson)

    def T21(self, eta, G_eta, boson):
        return self._bb().T21(eta, G_eta, boson)

    def T2(self, eta, G_eta, boson):
        return self._bb().T2(eta, G_eta, boson)

    def T4(self, eta, G_eta, boson):
        return self._bb().T4(eta, G_eta, boson)

    def Tvv(self, eta, G_eta, boson):
        return self._bb().Tvv(eta, G_eta, boson)

    def get_bond_bond_per_b2(self, boson):
        """The observables of the current eta / G_eta (after set_eta_G_eta), in
        ``corr_dtype`` when it is set."""
        eta, g = self.eta, self.G_eta
        if self.corr_dtype is not None:
            eta, g = eta.to(self.corr_dtype), g.to(self.corr_dtype)
        return self._bb().get_bond_bond_per_b2(eta, g, boson)

    def bond_corr(self, BB_r_mean, B_r_mean):
        return self._bb().bond_corr(BB_r_mean, B_r_mean)
