"""Adaptive Fourier mass of the boson momenta (``hmc_sampler_batch.py:1133-1277``).

Per chain and bond direction the sampler estimates the power spectrum of the
field's fluctuations on the real-FFT grid ``[Lx, Ly, Ltau // 2 + 1]`` and
turns it into a mass per mode; momenta drawn with that mass, and the inverse
mass applied to them, move the slow modes faster.  The arithmetic around the
FFTs runs in this library's kernels (``qedf_fm_*``), the FFTs are cuFFT's
through torch, and the statistics stay on the device:

* ``update(boson, i)``: the running mean of the field and of the orthonormal
  power spectrum of the centred field, averaged over a window that restarts
  at every ``annealing_step``-th step while restarts remain (10 of them);
* ``apply(i)``: every ``sigma_mini_batch_size`` steps the spectrum becomes
  the mass spectrum ``sigma_hat`` (clamp at the mean row 0.99 quantile,
  Box-Cox with ``lambda_``, rescale each row into ``[sig_min, sig_max]``,
  shift its mean to 1, shrink towards 1 by ``lmd``; inverted for
  ``mass_mode == -1``);
* ``draw_momentum_fft`` and ``apply_m_inv``.

The reference's method names (``update_sigma_hat_cpu``,
``apply_sigma_hat_cpu``) are kept as aliases; its leapfrog does not call the
draw or M^-1 (those call sites are commented out), so trajectories do not
depend on this module.
"""
from __future__ import annotations

import torch

from . import _lib
from .ops import ptr, stream_handle


class FourierMass:
    def __init__(self, bs, Lx, Ltau, dtype=torch.float32, device=None, sigma_mini_batch_size=1000, lmd=0.9,
                 lambda_=0.05, sig_min=0.8, sig_max=1.2, mass_mode=0):
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        if self.device.type != "cuda":
            raise RuntimeError("FourierMass runs on the GPU kernels (no CPU fallback)")
        if dtype not in (torch.float32, torch.float64):
            raise ValueError("dtype must be float32 or float64")
        self.bs, self.Lx, self.Ly, self.Ltau = bs, Lx, Lx, Ltau
        self.dtype = dtype
        self.grid = (Lx, Lx, Ltau)
        self.nk = Ltau // 2 + 1
        kshape = (bs, 2, Lx, Lx, self.nk)
        self.sigma_hat = torch.ones(kshape, device=self.device, dtype=dtype)
        self.spectrum = torch.ones(kshape, device=self.device, dtype=dtype)
        self.field_mean = torch.zeros((bs, 2, Lx, Lx, Ltau), device=self.device, dtype=dtype)
        self.sigma_mini_batch_size = sigma_mini_batch_size
        self.annealing_step = max(50, sigma_mini_batch_size)
        self.restarts_left = 10
        self.window_start = 0
        self.lmd, self.lambda_, self.sig_min, self.sig_max = lmd, lambda_, sig_min, sig_max
        self.mass_mode = mass_mode
        self._sfx = "f32" if dtype == torch.float32 else "f64"

    # ---- running statistics -------------------------------------------------
    def update(self, boson, i):
        """Fold step ``i``'s field (reference layout ``[bs, 2, Lx, Ly, Ltau]``)
        into the running mean and the running mean spectrum."""
        if i % self.annealing_step == 0 and i > 0 and self.restarts_left > 0:
            self.window_start = i
            self.restarts_left -= 1
        cnt = float(i - self.window_start)
        x = boson.to(device=self.device, dtype=self.dtype).contiguous()
        d = torch.empty_like(x)
        _lib.call(f"qedf_fm_accumulate_{self._sfx}", ptr(self.field_mean), ptr(x), ptr(d), x.numel(), cnt,
                  stream_handle())
        X = torch.fft.rfftn(d, self.grid, norm="ortho").contiguous()
        _lib.call(f"qedf_fm_spectrum_{self._sfx}", ptr(self.spectrum), ptr(torch.view_as_real(X)),
                  self.spectrum.numel(), cnt, stream_handle())

    def apply(self, i):
        """At every ``sigma_mini_batch_size``-th step (``i > 0``) the spectrum
        becomes the mass spectrum ``sigma_hat``."""
        if not (i % self.sigma_mini_batch_size == 0 and i > 0):
            return
        rows = self.spectrum.reshape(self.bs * 2, -1)
        clamp_hi = torch.quantile(rows, 0.99, dim=-1).mean().reshape(1).contiguous()
        _lib.call(f"qedf_fm_mass_{self._sfx}", ptr(self.spectrum), ptr(self.sigma_hat), rows.shape[0], rows.shape[1],
                  ptr(clamp_hi), float(self.lambda_), float(self.sig_min), float(self.sig_max), float(self.lmd),
                  1 if self.mass_mode == -1 else 0, stream_handle())

    # the reference's names (its statistics live on the host; here on the device)
    def update_sigma_hat_cpu(self, boson, i):
        self.update(boson, i)

    def apply_sigma_hat_cpu(self, i):
        self.apply(i)

    @property
    def sigma_hat_cpu(self):
        return self.spectrum.cpu()

    @property
    def boson_mean_cpu(self):
        return self.field_mean.cpu()

    # ---- momenta ------------------------------------------------------------
    def draw_momentum_fft(self, generator=None, noise=None):
        """Momenta ``[bs, 2, Lx, Ly, Ltau]`` with the Fourier mass.  The two
        normal draws are float32 like the reference's (torch's default dtype);
        ``noise = (a, b)`` supplies them instead."""
        shape = self.sigma_hat.shape
        if noise is None:
            a = torch.randn(shape, device=self.device, dtype=torch.float32, generator=generator)
            b = torch.randn(shape, device=self.device, dtype=torch.float32, generator=generator)
        else:
            a, b = noise
        a = a.to(device=self.device, dtype=self.dtype).contiguous()
        b = b.to(device=self.device, dtype=self.dtype).contiguous()
        cdt = torch.complex64 if self.dtype == torch.float32 else torch.complex128
        z = torch.empty(shape, device=self.device, dtype=cdt)
        _lib.call(f"qedf_fm_noise_{self._sfx}", ptr(a), ptr(b), ptr(self.sigma_hat), ptr(torch.view_as_real(z)),
                  a.numel(), self.nk, stream_handle())
        return torch.fft.irfftn(z, self.grid, norm="ortho")

    def apply_m_inv(self, p):
        """``M^-1 p = F^-1 (sigma_hat F p)``."""
        P = torch.fft.rfftn(p.to(device=self.device, dtype=self.dtype), self.grid).contiguous()
        _lib.call(f"qedf_fm_scale_{self._sfx}", ptr(torch.view_as_real(P)), ptr(self.sigma_hat), P.numel(),
                  stream_handle())
        return torch.fft.irfftn(P, self.grid)
