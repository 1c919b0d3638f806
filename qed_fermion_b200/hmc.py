"""Hybrid Monte Carlo for the fermion-coupled U(1) gauge field on the B200 kernels.

``HmcSampler`` keeps the reference's call signatures
(``qed_fermion/hmc_sampler_batch.py``): ``draw_momentum`` (:1247),
``draw_psudo_fermion`` (:1279), ``preconditioned_cg_fast_test`` (:751),
``Ot_inv_psi_fast`` (:2112), ``force_f_fast`` (:2150), ``leapfrog_cmp``
(:2332), ``leapfrog_proposer5`` (:2366), ``metropolis_update`` (:2886) and the
boson action/force methods (:1338-1459).  Bosons, momenta and forces use the
reference layout ``[bs, 2, Lx, Ly, Ltau]`` at this interface; internally the
trajectory runs in the kernels' layout ``[bs, Ltau, Ly, Lx, 2]``.

Precision ("precision" argument):
  "fp64"  plain double path: float64 angles/momenta, complex128 vectors,
          double PCG and force;
  "mixed" float32 angles and momenta (as the reference stores them), PCG in
          float with double reliable updates, float force, and the
          Hamiltonian, Delta H and the Metropolis test in double;
  "mixed_bf16" as "mixed", with the PCG's p and z stored as bf16;
  "mixed_f16" as "mixed", with the PCG's p and z stored as scaled fp16;
  "fp32"  everything in single precision (the reference's own GPU choice).

``chrono_guess`` ("last" or "linear") starts each leapfrog solve after the
first from the previous solution or the linear extrapolation of the last two,
instead of the reference's zero.  The solves end at the same tolerance, so
the integrator stays reversible to that tolerance.  On L=48, Ltau=480 at a
step of 0.05 the guesses' residuals are 1-2 % of |psi|, and they save about
5 % ("last") and 6 % ("linear") of the iterations: the error left in the
guess lies in the slow modes that take CG the most iterations.

``graph=True`` replays each trajectory from a CUDA graph captured on the first
proposal (``TrajectoryGraph``).  With or without it, a Metropolis update never
waits for the GPU: the accept test runs on the device and the threshold queue
is read back only when it is used.
"""
from __future__ import annotations

import collections
import math
import os

import torch

from . import _lib, ops
from .fourier_mass import FourierMass
from .solver import PcgSolver, System

PRECISIONS = ("fp64", "mixed", "mixed_bf16", "mixed_f16", "fp32")


def ref_to_kernel(boson: torch.Tensor) -> torch.Tensor:
    """``[bs, 2, Lx, Ly, Ltau] -> [bs, Ltau*Ly*Lx*2]`` (``permute([0, 4, 3, 2, 1])``)."""
    return boson.permute(0, 4, 3, 2, 1).reshape(boson.shape[0], -1).contiguous()


def metropolis_accept(H_old: torch.Tensor, H_new: torch.Tensor, u: torch.Tensor):
    """The accept test of ``metropolis_update`` (``hmc_sampler_batch.py:2910``)
    in double precision: ``u < exp(H_old - H_new)`` per chain, with ``u``
    uniform in [0, 1).  Returns (accept mask, min(exp(H_old - H_new), 1)), the
    second being the value each chain's threshold queue records (:2921).  A
    non-finite Delta H is rejected."""
    w = torch.exp(H_old.double() - H_new.double())
    accept = u.double() < w
    return accept, torch.clamp(torch.nan_to_num(w, nan=0.0), max=1.0)


def kernel_to_ref(phi: torch.Tensor, Lx: int, Ltau: int) -> torch.Tensor:
    bs = phi.shape[0]
    return phi.view(bs, Ltau, Lx, Lx, 2).permute(0, 4, 3, 2, 1).contiguous()


class HmcSampler:
    def __init__(self, Lx=6, Ltau=10, J=1.0, K=1.0, dtau=0.1, bs=1, delta_t=0.06, N_leapfrog=5, m=1.0,
                 compact=False, precision="mixed", cg_rtol=1e-10, max_iter=20000, use_precon=True,
                 ru_interval=100, ru_delta=0.01, device=None, seed=None, solver_impl="persistent",
                 max_tau_block_idx=1, autotune=True, graph=False, chrono_guess=None):
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {PRECISIONS}")
        if chrono_guess not in (None, "last", "linear"):
            raise ValueError("chrono_guess must be None, 'last' or 'linear'")
        if Lx % 2:
            raise ValueError("Lx must be even")
        self.Lx = self.Ly = Lx
        self.Ltau = Ltau
        self.Vs = Lx * Lx
        self.bs = bs
        self.dtau = dtau
        self.Nf = 2
        # couplings as HmcSampler.__init__ scales them (hmc_sampler_batch.py:166-175)
        self.J = J / dtau * self.Nf / 4
        self.K = K * dtau * self.Nf / 2
        self.t = 1
        self.m = m
        self.compact = compact
        self.N_leapfrog = N_leapfrog
        self.precision = precision
        self.cg_rtol = cg_rtol
        self.max_iter = max_iter
        self.use_precon = use_precon and Ltau >= 26
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        self.dtype = torch.float64 if precision == "fp64" else torch.float32
        self.cdtype = torch.complex128 if precision in ("fp64", "mixed", "mixed_bf16", "mixed_f16") else torch.complex64
        self.delta_t_tensor = torch.full((bs,), float(delta_t), device=self.device, dtype=torch.float64)
        self.generator = torch.Generator(device=self.device)
        if seed is not None:
            self.generator.manual_seed(seed)
        solver_mode = {"fp64": "fp64", "mixed": "mixed", "mixed_bf16": "mixed_bf16", "mixed_f16": "mixed_f16",
                       "fp32": "fp32"}[precision]
        self.solver = PcgSolver([System(Lx, Ltau, bs, False)], mode=solver_mode, rtol=cg_rtol, max_iter=max_iter,
                                dtau=dtau, use_precon=self.use_precon, ru_interval=ru_interval,
                                ru_delta=ru_delta, device=self.device, tune=autotune)
        # "persistent": one cooperative PCG kernel per solve; "reference_loop": the
        # reference's per-iteration launch sequence (preconditioned_cg_fast_test) on
        # this library's _C kernels -- the drop-in path
        if solver_impl not in ("persistent", "reference_loop"):
            raise ValueError("solver_impl must be 'persistent' or 'reference_loop'")
        self.solver_impl = solver_impl
        self._precon_tau = None
        self.boson = None
        self.last_cg_iters = None
        # tau-block updates and step-size adaptation (hmc_sampler_batch.py:158-163,
        # 263-268): blocks only when Ltau >= 10 Lx; per chain a queue of the last
        # 5 x blocks clipped acceptance probabilities
        self.tau_block_idx = 0
        self.max_tau_block_idx = max_tau_block_idx if Ltau // Lx // 10 >= 1 else 1
        self.tau_block_size = Ltau // self.max_tau_block_idx
        self._threshold_queue = [collections.deque(maxlen=5 * self.max_tau_block_idx) for _ in range(bs)]
        self._thr_pending = []
        # trajectories replayed from CUDA graphs (one per masked / unmasked proposal)
        self.use_graph = bool(graph)
        # initial guesses of the leapfrog's solves (None: zero, as the reference)
        self.chrono_guess = chrono_guess
        self._graphs = {}
        self.lower_limit = 0.25
        self.upper_limit = 0.5

    @property
    def threshold_queue(self):
        """Per chain, the clipped acceptance probabilities of the latest
        proposals (a deque of ``5 x max_tau_block_idx``).  Proposals leave
        theirs on the device; reading the queue moves them here in one copy."""
        if self._thr_pending:
            rows = torch.stack(self._thr_pending).cpu().tolist()
            self._thr_pending.clear()
            for row in rows:
                for q, v in zip(self._threshold_queue, row):
                    q.append(v)
        return self._threshold_queue

    # ---- couplings ---------------------------------------------------------
    @property
    def tau_coeff(self):
        return 1.0 / self.J / self.dtau ** 2

    # ---- initial fields (reference :1026-1043) --------------------------------
    def initialize_boson_pi_flux_randn_matfree(self):
        x = torch.arange(self.Lx, device=self.device).view(-1, 1)
        y = torch.arange(self.Ly, device=self.device).view(1, -1)
        sign = (1 - 2 * ((x + y) % 2)).to(self.dtype)
        stag = torch.zeros(1, 2, self.Lx, self.Ly, self.Ltau, device=self.device, dtype=self.dtype)
        stag[0, 0] = (sign * math.pi / 4).unsqueeze(-1)
        stag[0, 1] = (-sign * math.pi / 4).unsqueeze(-1)
        if self.bs > 1:
            noise = torch.randn(self.bs - 1, 2, self.Lx, self.Ly, 1, device=self.device, dtype=self.dtype,
                                generator=self.generator)
            lev = torch.linspace(0.02, 0.08, self.bs - 1, device=self.device, dtype=self.dtype).view(-1, 1, 1, 1, 1)
            self.boson = torch.cat([stag.repeat(self.bs - 1, 1, 1, 1, 1) + noise * lev, stag], dim=0)
        else:
            self.boson = stag
        return self.boson

    # ---- boson checkpoints (reference :971-1016, :3164-3181, :3211-3215) -------
    # The reference saves {'boson': [bs, 2, Lx, Ly, Ltau] on the CPU,
    # 'delta_t_tensor': [bs]} with torch.save as "<folder>/<name>.pt", and reads
    # either that dict or a bare boson tensor back.
    def save_boson_checkpoint(self, data_folder, file_name):
        """Write the current field and step sizes in the reference's format and
        return the file path (``<data_folder>/<file_name>.pt``)."""
        if self.boson is None:
            raise RuntimeError("no boson field to save")
        os.makedirs(data_folder, exist_ok=True)
        path = os.path.join(data_folder, f"{file_name}.pt")
        # the reference keeps delta_t_tensor in its field dtype
        torch.save({"boson": self.boson.detach().cpu(),
                    "delta_t_tensor": self.delta_t_tensor.detach().to(self.dtype).cpu()}, path)
        return path

    def load_boson_checkpoint(self, path):
        """Read a field written by the reference or by ``save_boson_checkpoint``
        (a dict with 'boson' and optionally 'delta_t_tensor', or a bare tensor)."""
        loaded = torch.load(path, map_location="cpu")
        boson = loaded["boson"] if isinstance(loaded, dict) else loaded
        if tuple(boson.shape) != (self.bs, 2, self.Lx, self.Ly, self.Ltau):
            raise RuntimeError(f"checkpoint field has shape {tuple(boson.shape)}, expected [{self.bs}, 2, "
                               f"{self.Lx}, {self.Ly}, {self.Ltau}] (the sampler's chains)")
        dt = None
        if isinstance(loaded, dict) and "delta_t_tensor" in loaded:
            dt = loaded["delta_t_tensor"].reshape(-1)
            if dt.numel() != self.bs:
                raise RuntimeError(f"checkpoint has {dt.numel()} step sizes for {self.bs} chains")
        self.boson = boson.to(device=self.device, dtype=self.dtype)
        if dt is not None:
            self.delta_t_tensor = dt.to(device=self.device, dtype=torch.float64)
        return self.boson

    def initialize_boson_ensemble(self, data_folder, specifics, steps=range(4000, 10001, 500)):
        """Warm start from saved ensemble members (reference :971-1016): the
        files ``boson_<specifics>_<step>.pt`` that exist in ``data_folder``; one
        field and one step-size tensor are drawn at random with the sampler's
        generator.  Without any file the pi-flux start is used."""
        bosons, dts = [], []
        for step in steps:
            path = os.path.join(data_folder, f"boson_{specifics}_{step}.pt")
            if not os.path.exists(path):
                continue
            loaded = torch.load(path, map_location="cpu")
            if isinstance(loaded, dict):
                bosons.append(loaded["boson"])
                if "delta_t_tensor" in loaded:
                    dts.append(loaded["delta_t_tensor"])
            else:
                bosons.append(loaded)
        if not bosons:
            return self.initialize_boson_pi_flux_randn_matfree()
        pick = int(torch.randint(len(bosons), (1,), generator=self._cpu_generator()).item())
        self.boson = bosons[pick].to(device=self.device, dtype=self.dtype)
        if dts:
            pick = int(torch.randint(len(dts), (1,), generator=self._cpu_generator()).item())
            self.delta_t_tensor = dts[pick].to(device=self.device, dtype=torch.float64)
        return self.boson

    def _cpu_generator(self):
        g = torch.Generator()
        g.manual_seed(int(torch.randint(0, 2 ** 31 - 1, (1,), device=self.device, generator=self.generator).item()))
        return g

    # ---- adaptive Fourier mass (reference :272-285, 1133-1277) -----------------
    # The reference computes these but its leapfrog does not call the draw or
    # M^{-1} (the call sites are commented out); they are kept for the API.
    @property
    def fourier_mass(self):
        if getattr(self, "_fourier_mass", None) is None:
            self._fourier_mass = FourierMass(self.bs, self.Lx, self.Ltau, dtype=self.dtype, device=self.device)
        return self._fourier_mass

    def update_sigma_hat_cpu(self, boson_cpu, i):
        self.fourier_mass.update_sigma_hat_cpu(boson_cpu, i)

    def apply_sigma_hat_cpu(self, i):
        self.fourier_mass.apply_sigma_hat_cpu(i)

    def draw_momentum_fft(self):
        return self.fourier_mass.draw_momentum_fft(self.generator)

    def apply_m_inv(self, p):
        return self.fourier_mass.apply_m_inv(p)

    # ---- random draws (reference :1247-1252, :1279-1287) ----------------------
    def draw_momentum(self):
        return torch.randn(self.bs, 2, self.Lx, self.Ly, self.Ltau, device=self.device, dtype=self.dtype,
                           generator=self.generator) * math.sqrt(self.m)

    def draw_psudo_fermion(self):
        # the reference's active line: complex randn (E|z|^2 = 1) divided by sqrt(2)
        return torch.randn(self.bs, self.Vs * self.Ltau, device=self.device, dtype=self.cdtype,
                           generator=self.generator) / math.sqrt(2)

    # ---- boson action and forces (reference layout) ---------------------------
    def action_boson_tau(self, x):
        phi = ref_to_kernel(x)
        return ops.boson_action(phi, self.Lx, 0.0, self.tau_coeff, self.compact)

    def action_boson_plaq_matfree(self, x):
        phi = ref_to_kernel(x)
        return ops.boson_action(phi, self.Lx, self.K, 0.0, self.compact)

    def force_b_plaq_matfree(self, x):
        phi = ref_to_kernel(x)
        return kernel_to_ref(ops.boson_force(phi, self.Lx, self.K, 0.0), self.Lx, self.Ltau)

    def force_b_tau_noncmp(self, x):
        phi = ref_to_kernel(x)
        return kernel_to_ref(ops.boson_force(phi, self.Lx, 0.0, self.tau_coeff, False), self.Lx, self.Ltau)

    def force_b_tau_cmp(self, x):
        phi = ref_to_kernel(x)
        return kernel_to_ref(ops.boson_force(phi, self.Lx, 0.0, self.tau_coeff, True), self.Lx, self.Ltau)

    # ---- solver ---------------------------------------------------------------
    def _angles_for_solver(self, phi_k):
        return phi_k.to(self.solver.angle_dtype)

    def Ot_inv_psi_fast(self, psi, boson_k, MhM=None, x0=None):
        """xi = (M^dag M)^{-1} psi with the persistent batched PCG.
        ``boson_k``: kernel-layout angles ``[bs, ...]``; ``x0``: optional
        initial guess like ``psi`` (the reference starts from 0); returns
        (xi, iters, relres)."""
        if self.solver_impl == "reference_loop":
            if self._precon_tau is None and self.use_precon:
                from . import precon
                self._precon_tau = precon.to_device(precon.builtin_tau_csr(self.Ltau), self.device)
            adt = torch.float64 if self.cdtype == torch.complex128 else torch.float32
            x, it, err = self.preconditioned_cg_fast_test(boson_k.to(adt), psi.to(self.cdtype),
                                                          precon_tau=self._precon_tau)
            self.last_cg_iters = it
            return x.view(self.bs, -1), it, err
        res = self.solver.solve(self._angles_for_solver(boson_k), psi.to(self.solver.vec_dtype),
                                x0=None if x0 is None else x0.to(self.solver.vec_dtype))
        self.last_cg_iters = res.iters
        self.last_status = res.status
        return res.x.view(self.bs, -1), res.iters, res.relres

    def preconditioned_cg_fast_test(self, boson, b, MhM_inv=None, matL=None, b_idx=None, axs=None,
                                    cg_dtype=None, MhM=None, precon_tau=None):
        """The reference's batched masked PCG loop (``hmc_sampler_batch.py:751-846``),
        one torch/_C launch sequence per iteration, on this library's kernels.
        ``boson``: ``[bs, Ltau, Vs*2]`` angles; ``b``: ``[bs, N]``.  Runs until
        every system converged or ``max_iter``; returns (x, iterations, error)."""
        bs = b.shape[0]
        boson = boson.reshape(bs, -1)
        dt = self.dtau
        norm_b = torch.linalg.vector_norm(b, dim=1)
        active = torch.ones((bs, 1), device=b.device, dtype=b.dtype)
        x = torch.zeros_like(b)

        def P(r):
            return ops.precon_apply(r, precon_tau, self.Lx) if precon_tau is not None else r.clone()

        r = b - ops.apply_operator("mhm", boson, x, self.Lx, dt)
        z = P(r)
        p = z
        rz_old = torch.einsum("bj,bj->b", r.conj(), z).real
        iterations = torch.zeros(bs, dtype=torch.int64, device=b.device)
        error = torch.ones(bs, dtype=norm_b.dtype, device=b.device)
        for _ in range(self.max_iter):
            Op = ops.apply_operator("mhm", boson, p, self.Lx, dt)
            alpha = (rz_old / torch.einsum("bj,bj->b", p.conj(), Op).real).unsqueeze(-1)
            x = x + alpha * p * active
            r = r - alpha * Op * active
            error = torch.linalg.vector_norm(r, dim=1) / norm_b
            active = torch.where(error.view(-1, 1) > self.cg_rtol, active, torch.zeros_like(active))
            if bool((active == 0).all()):
                break
            iterations += (active == 1).view(-1).long()
            z = P(r)
            rz_new = torch.einsum("bj,bj->b", r.conj(), z).real
            beta = rz_new / rz_old
            p = z + beta.unsqueeze(-1) * p * active
            rz_old = rz_new
        return x, iterations, error

    # ---- fermion force (reference :2150-2227) ---------------------------------
    def force_f_fast(self, psi, boson, MhM=None):
        """Returns (Ft [bs, 2, Lx, Ly, Ltau], xi [bs, N], cg_iters, r_err)."""
        phi_k = ref_to_kernel(boson)
        xi, it, err = self.Ot_inv_psi_fast(psi, phi_k)
        F = self._force_from_xi(phi_k, xi)
        return kernel_to_ref(F, self.Lx, self.Ltau), xi, it, err

    def _force_from_xi(self, phi_k, xi):
        if self.precision == "fp64":
            return ops.fermion_force(phi_k, xi, self.Lx, self.dtau)
        return ops.fermion_force(phi_k.to(torch.float32), xi.to(torch.complex64), self.Lx, self.dtau).to(self.dtype)

    # ---- trajectory -------------------------------------------------------------
    def _Sb_kin(self, phi_k, p_k):
        # S_tau + S_plaq + sum p^2 / 2m in double
        return ops.boson_action(phi_k, self.Lx, self.K, self.tau_coeff, self.compact, momenta=p_k, mass=self.m)

    def leapfrog_proposer5(self, boson, tau_mask=None, p0=None, R=None):
        """One trajectory from ``boson`` (reference layout); ``p0`` / ``R`` may
        be given (reference layout / ``[bs, N]``) instead of drawn.
        Returns (x, H0, H_fin, cg_iters_mean, r_err_mean) like the reference."""
        Lx, Ltau = self.Lx, self.Ltau
        if p0 is None:
            p0 = self.draw_momentum()
        if R is None:
            R = self.draw_psudo_fermion()
        if self.use_graph and self.solver_impl == "persistent":
            key = tau_mask is not None
            if key not in self._graphs:
                self._graphs[key] = TrajectoryGraph(self, masked=key)
            x, p, H0, H_fin, it, err = self._graphs[key].run(boson, p0, R, self.delta_t_tensor, tau_mask)
        else:
            x = ref_to_kernel(boson.to(self.dtype))
            p = ref_to_kernel(p0.to(self.dtype))
            mask = None
            if tau_mask is not None:
                mask = tau_mask.reshape(-1).to(torch.float32).contiguous()
            H0, H_fin, it, err = self._integrate(x, p, R, self.delta_t_tensor, mask)
        self._last_p = p
        return kernel_to_ref(x, Lx, Ltau), H0, H_fin, it, err

    def _chrono_guess(self, hist):
        """Initial guess of the next solve along a trajectory from the latest
        solutions ``hist`` (same psi, the field moved by one step): none (the
        reference's zero start), the last solution, or the linear
        extrapolation of the last two (Brower, Ivanenko, Levi and Orginos,
        "Chronological inversion method for the Dirac matrix in hybrid Monte
        Carlo", 1997)."""
        if self.chrono_guess is None or not hist:
            return None
        if self.chrono_guess == "linear" and len(hist) >= 2:
            return 2 * hist[-1] - hist[-2]
        return hist[-1]

    def _integrate(self, x, p, R, dt, mask):
        """The trajectory body of ``leapfrog_proposer5`` (reference :2366-2460)
        on kernel-layout angles ``x`` and momenta ``p`` (both ``[bs, Ltau*Vs*2]``,
        advanced in place), the pseudofermion noise ``R`` (``[bs, N]``), the
        per-chain step sizes ``dt`` (``[bs]`` float64) and an optional tau mask
        (``[Ltau]`` float32).  Only device work: nothing here waits for the GPU,
        so the whole body can be captured in a CUDA graph.
        Returns (H0, H_fin, cg_iters_mean, r_err_mean)."""
        Lx = self.Lx
        # psi = M(x0)^dag R, in the solver's vector precision
        vdt = self.solver.vec_dtype
        adt = torch.float64 if vdt == torch.complex128 else torch.float32
        psi = ops.apply_operator("mh", x.to(adt), R.to(vdt).reshape(self.bs, -1), Lx, self.dtau)
        xi, it, err = self.Ot_inv_psi_fast(psi, x)
        iters, errs = [it.to(torch.float64)], [err]
        hist = [xi]
        Ff = self._force_from_xi(x, xi)
        Sf0 = ops.cdot(psi, xi)
        H0 = self._Sb_kin(x, p) + Sf0
        Fb = ops.boson_force(x, Lx, self.K, self.tau_coeff, self.compact)
        M = 5
        for _ in range(self.N_leapfrog):
            ops.kick_drift(p, Ff, None, dt, mask, 0.5, 0.0, Lx)
            for _ in range(M):
                ops.kick_drift(p, Fb, x, dt, mask, 0.5 / M, 1.0 / M / self.m, Lx)
                ops.boson_force(x, Lx, self.K, self.tau_coeff, self.compact, out=Fb)
                ops.kick_drift(p, Fb, None, dt, mask, 0.5 / M, 0.0, Lx)
            xi, it, err = self.Ot_inv_psi_fast(psi, x, x0=self._chrono_guess(hist))
            hist = (hist + [xi])[-2:]
            iters.append(it.to(torch.float64))
            errs.append(err)
            Ff = self._force_from_xi(x, xi)
            ops.kick_drift(p, Ff, None, dt, mask, 0.5, 0.0, Lx)
        Sf = ops.cdot(psi, xi)
        H_fin = self._Sb_kin(x, p) + Sf
        return H0, H_fin, torch.stack(iters).mean(dim=0), torch.stack(errs).mean(dim=0)

    def _metropolis_step(self, tau_mask):
        boson_new, H_old, H_new, it, err = self.leapfrog_proposer5(self.boson, tau_mask)
        u = torch.rand(self.bs, device=self.device, dtype=torch.float64, generator=self.generator)
        accp, thr = metropolis_accept(H_old, H_new, u)
        self.boson = torch.where(accp.view(-1, 1, 1, 1, 1), boson_new.to(self.boson.dtype), self.boson)
        # the queue entry stays on the device until the queue is read; entries
        # older than the queue's length would have left it anyway
        self._thr_pending.append(thr)
        del self._thr_pending[:-self._threshold_queue[0].maxlen]
        return accp, it, err, H_old, H_new

    def metropolis_update(self, tau_mask=None):
        """Metropolis update of ``self.boson`` (reference :2886-2930).  Without
        ``tau_mask``, one proposal per tau block (``max_tau_block_idx`` blocks of
        ``tau_block_size`` slices, each moving only its own slices) with its own
        accept test; with ``tau_mask`` (``[1, 1, 1, 1, Ltau]`` or ``[Ltau]``), one
        proposal under that mask.  The accept test ``u < exp(H_old - H_new)`` is
        evaluated in double; every test appends min(exp(H_old - H_new), 1) to the
        chain's threshold queue.  Returns (boson, accp, iters, err, H_old, H_new)
        of the last proposal."""
        if tau_mask is not None:
            accp, it, err, H_old, H_new = self._metropolis_step(tau_mask)
            return self.boson, accp, it, err, H_old, H_new
        if self.max_tau_block_idx == 1:
            accp, it, err, H_old, H_new = self._metropolis_step(None)
            return self.boson, accp, it, err, H_old, H_new
        while self.tau_block_idx < self.max_tau_block_idx:
            t0 = self.tau_block_idx * self.tau_block_size
            mask = torch.zeros((1, 1, 1, 1, self.Ltau), device=self.device, dtype=self.dtype)
            mask[..., t0:t0 + self.tau_block_size] = 1.0
            accp, it, err, H_old, H_new = self._metropolis_step(mask)
            self.tau_block_idx += 1
        self.tau_block_idx = 0
        return self.boson, accp, it, err, H_old, H_new

    def adjust_delta_t(self):
        """Per chain, once its threshold queue is full: shrink delta_t by 0.9 when
        the mean clipped acceptance is below ``lower_limit``, grow it by 1.1 when
        above ``upper_limit``, and clear the queue (reference :699-724)."""
        for b in range(self.bs):
            q = self.threshold_queue[b]
            if len(q) < q.maxlen:
                continue
            rate = sum(q) / len(q)
            if rate < self.lower_limit:
                self.delta_t_tensor[b] *= 0.9
            elif self.upper_limit < rate:
                self.delta_t_tensor[b] *= 1.1
            else:
                continue
            q.clear()


class TrajectoryGraph:
    """One trajectory of ``HmcSampler._integrate`` captured in a CUDA graph.

    The first ``run`` integrates eagerly on the current stream (so every
    first-call setup and the solver's tuning happen outside the capture), then
    captures the same launches into a graph.  Later runs copy the proposal's
    field, momenta, pseudofermion noise, step sizes and tau mask into the
    captured buffers and replay: the ~24 launches of each leapfrog step (one
    persistent PCG solve, the fermion force, the boson sub-steps) become one
    graph launch per trajectory, and nothing returns to the host.

    The captured buffers belong to this object; ``run`` returns fresh copies
    of the results, so they stay valid across later runs."""

    def __init__(self, sampler: "HmcSampler", masked: bool):
        s = sampler
        n = s.Vs * s.Ltau
        self.s = s
        self.x = torch.empty(s.bs, 2 * n, dtype=s.dtype, device=s.device)
        self.p = torch.empty_like(self.x)
        self.R = torch.empty(s.bs, n, dtype=s.cdtype, device=s.device)
        self.dt = torch.empty(s.bs, dtype=torch.float64, device=s.device)
        self.mask = torch.empty(s.Ltau, dtype=torch.float32, device=s.device) if masked else None
        self.graph = None
        self.out = None
        self.launches = 0

    def _load(self, boson, p0, R, dt, tau_mask):
        self.x.copy_(ref_to_kernel(boson.to(self.s.dtype)))
        self.p.copy_(ref_to_kernel(p0.to(self.s.dtype)))
        self.R.copy_(R.reshape(self.R.shape))
        self.dt.copy_(dt.reshape(-1))
        if self.mask is not None:
            self.mask.copy_(tau_mask.reshape(-1))

    def run(self, boson, p0, R, dt, tau_mask=None):
        """Returns (x, p, H0, H_fin, cg_iters_mean, r_err_mean); x and p in the
        kernel layout."""
        if (tau_mask is None) != (self.mask is None):
            raise ValueError("tau_mask must be given exactly when the graph was made for a masked proposal")
        self._load(boson, p0, R, dt, tau_mask)
        if self.graph is None:
            out = self.s._integrate(self.x, self.p, self.R, self.dt, self.mask)
            res = (self.x.clone(), self.p.clone()) + tuple(out)
            g = torch.cuda.CUDAGraph()
            n0 = _lib.LAUNCHES["count"]
            with torch.cuda.graph(g):
                self.out = self.s._integrate(self.x, self.p, self.R, self.dt, self.mask)
            # the capture launched nothing; each replay launches what it recorded
            self.launches = _lib.LAUNCHES["count"] - n0
            _lib.LAUNCHES["count"] = n0
            self.graph = g
            return res
        self.graph.replay()
        _lib.LAUNCHES["count"] += self.launches
        return (self.x.clone(), self.p.clone()) + tuple(t.clone() for t in self.out)
