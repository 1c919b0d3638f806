"""Fourier-space adaptive mass of the boson momenta.

The reference keeps, per chain and bond direction, a spectrum sigma_hat over
the rfft grid ``[bs, 2, Lx, Ly, Ltau // 2 + 1]`` (``hmc_sampler_batch.py``
:272-285).  Every step it accumulates the running mean of |rfftn(boson -
mean)|^2 (``update_sigma_hat_cpu`` :1202-1210).  Every ``sigma_mini_batch_size``
steps it turns that spectrum into a mass:
- clamp at the 0.99 quantile;
- a Box-Cox transform with lambda = 0.05;
- rescale into [sig_min, sig_max];
- shift the mean to 1;
- shrink towards 1 by lmd;
- and, in mass mode -1, invert (``apply_sigma_hat_cpu`` :1133-1200).

``draw_momentum_fft`` (:1254-1265) and ``apply_m_inv`` (:1267-1277) draw
momenta with that mass and apply its inverse.  Their call sites in the
reference's leapfrog are commented out, so the sampler's trajectories do not
depend on it.  The routines are provided with the reference's names,
arguments and arithmetic.  FFTs are cuFFT's through torch; the statistics
live on the CPU, as in the reference.
"""
from __future__ import annotations

import torch


class FourierMass:
    def __init__(self, bs, Lx, Ltau, dtype=torch.float32, device=None, sigma_mini_batch_size=1000, lmd=0.9,
                 lambda_=0.05, sig_min=0.8, sig_max=1.2, mass_mode=0):
        self.bs, self.Lx, self.Ly, self.Ltau = bs, Lx, Lx, Ltau
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        shape = (bs, 2, Lx, Lx, Ltau // 2 + 1)
        self.sigma_hat = torch.ones(shape, device=self.device, dtype=dtype)
        self.sigma_hat_cpu = torch.ones(shape, dtype=dtype)
        self.boson_mean_cpu = torch.zeros((bs, 2, Lx, Lx, Ltau), dtype=dtype)
        self.sigma_mini_batch_size = sigma_mini_batch_size
        self.sigma_hat_mini_batch_last_i = 0
        self.annealing_step = max(50, sigma_mini_batch_size)
        self.anneal_times = 10
        # the non-redundant rfft modes along tau count twice, k = 0 and Nyquist once
        self.multiplier = torch.full_like(self.sigma_hat, 2)
        self.multiplier[..., torch.tensor([0, -1], device=self.device)] = 1
        self.lmd, self.lambda_, self.sig_min, self.sig_max = lmd, lambda_, sig_min, sig_max
        self.mass_mode = mass_mode

    def update_sigma_hat_cpu(self, boson_cpu, i):
        """Fold step i's field (reference layout, on the CPU) into the running
        mean and the running mean spectrum; restart the window at each
        annealing step while annealing steps remain."""
        if i % self.annealing_step == 0 and i > 0 and self.anneal_times > 0:
            self.sigma_hat_mini_batch_last_i = i
            self.anneal_times -= 1
        cnt = i - self.sigma_hat_mini_batch_last_i
        self.boson_mean_cpu = (self.boson_mean_cpu * cnt + boson_cpu) / (cnt + 1)
        d = torch.fft.rfftn(boson_cpu - self.boson_mean_cpu, (self.Lx, self.Ly, self.Ltau), norm="ortho").abs() ** 2
        self.sigma_hat_cpu = (self.sigma_hat_cpu * cnt + d) / (cnt + 1)

    def stabilize_sigma_hat(self, method="shrink", **kw):
        if method == "shrink":
            lmd = kw.get("lmd", 0.8)
            self.sigma_hat = (1 - lmd) * self.sigma_hat + lmd * torch.ones_like(self.sigma_hat)
        elif method == "pow":
            self.sigma_hat = self.sigma_hat.pow(kw.get("beta", 0.5))
        elif method == "clamp":
            self.sigma_hat = self.sigma_hat.clamp(kw.get("sgm_min", 0.5), kw.get("sgm_max", 2.0))
        elif method == "clamp_shrink":
            sgm_min, sgm_max = kw.get("sgm_min", 0.5), kw.get("sgm_max", 2.0)
            mx = self.sigma_hat.amax(dim=(2, 3, 4), keepdim=True)
            mn = self.sigma_hat.amin(dim=(2, 3, 4), keepdim=True)
            self.sigma_hat = torch.where(self.sigma_hat > 1, 1 + (self.sigma_hat - 1) * ((sgm_max - 1) / (mx - 1)),
                                         1 - (1 - self.sigma_hat) * ((sgm_min - 1) / (mn - 1)))
        elif method == "log_inter":
            lmd = kw.get("lmd", 0.8)
            self.sigma_hat = (1 - lmd) * torch.log1p(self.sigma_hat) + lmd * torch.ones_like(self.sigma_hat)
        else:
            raise ValueError(f"unknown method {method}")

    def apply_sigma_hat_cpu(self, i):
        """Every sigma_mini_batch_size steps: the accumulated spectrum becomes the
        mass (see the module docstring for the steps)."""
        if not (i % self.sigma_mini_batch_size == 0 and i > 0):
            return
        self.sigma_hat = self.sigma_hat_cpu.to(self.sigma_hat.device)
        flat = self.sigma_hat.view(self.sigma_hat.size(0), self.sigma_hat.size(1), -1)
        q = torch.quantile(flat, 0.99, dim=-1, keepdim=True).view(self.sigma_hat.size(0), self.sigma_hat.size(1),
                                                                  1, 1, 1)
        self.stabilize_sigma_hat(method="clamp", sgm_min=0, sgm_max=q.mean())
        lam = self.lambda_
        self.sigma_hat = (self.sigma_hat ** lam - 1) / lam
        mn = self.sigma_hat.amin(dim=(2, 3, 4), keepdim=True)
        mx = self.sigma_hat.amax(dim=(2, 3, 4), keepdim=True)
        self.sigma_hat = (self.sigma_hat - mn) / (mx - mn).clamp(min=1e-8) * (self.sig_max - self.sig_min) + self.sig_min
        self.sigma_hat = self.sigma_hat - self.sigma_hat.mean(dim=(2, 3, 4), keepdim=True) + 1
        self.stabilize_sigma_hat(method="shrink", lmd=self.lmd)
        if self.mass_mode == -1:
            self.sigma_hat = self.sigma_hat ** (-1)

    def draw_momentum_fft(self, generator=None):
        """Momenta [bs, 2, Lx, Ly, Ltau] with the Fourier mass.  The normal draws
        are float32, as the reference's (torch's default dtype)."""
        shape = self.sigma_hat.shape
        x = torch.randn(shape, device=self.device, dtype=torch.float32, generator=generator)
        y = torch.randn(shape, device=self.device, dtype=torch.float32, generator=generator)
        z = (x + 1j * y) / torch.sqrt(self.sigma_hat * self.multiplier)
        return torch.fft.irfftn(z, (self.Lx, self.Ly, self.Ltau), norm="ortho")

    def apply_m_inv(self, p):
        """M^{-1} p = F^{-1} sigma_hat F p."""
        pf = torch.fft.rfftn(p, (self.Lx, self.Ly, self.Ltau)) * self.sigma_hat
        return torch.fft.irfftn(pf, (self.Lx, self.Ly, self.Ltau))
