"""Bond-bond correlators of the stochastic estimator on the GPU.

These are the observables the reference computes from the noise vectors eta
and G_eta = (M^dag M)^-1 M^dag eta of one gauge field
(``qed_fermion/stochastic_estimator.py``: ``T1`` :1393, ``T21`` :1447, ``T2``
:1504, ``T4`` :1561, ``Tvv`` :1612, ``get_bond_bond_per_b2`` :2594,
``bond_corr`` :2643), with the same names, arguments and return values.

Each ``T`` averages, over all noise pairs s < s' (``torch.combinations``
order) and over tau, the spatial correlation of two bond products,
    C(d) = (1 / Vs) sum_r a(r) b(r + d),
evaluated with 2-D FFTs over (y, x).  Because the inverse transform is linear,
the products of the transforms are summed over pairs and tau first and only
one inverse FFT per observable remains; the reference instead transforms back
per batch.  Pairs are processed in chunks sized by ``chunk_bytes``.

Layouts as in the reference: eta, G_eta ``[Nrv, Ltau * Ly * Lx]`` (index
tau Vs + x + Lx y); boson ``[1, 2, Lx, Ly, Ltau]``.  Inputs must be CUDA
tensors; the transforms are cuFFT's (through torch).
"""
from __future__ import annotations

import torch


class BondBond:
    def __init__(self, Lx: int, Ltau: int, chunk_bytes: int = 1 << 30):
        self.Lx = self.Ly = Lx
        self.Ltau = Ltau
        self.chunk_bytes = int(chunk_bytes)

    # ---- helpers ----------------------------------------------------------
    def _fields(self, eta, G_eta, boson):
        for t in (eta, G_eta, boson):
            if not t.is_cuda:
                raise RuntimeError("bond-bond correlators need CUDA tensors")
        ec = eta.conj().reshape(-1, self.Ltau, self.Ly, self.Lx)
        g = G_eta.reshape(-1, self.Ltau, self.Ly, self.Lx).to(ec.dtype)
        ph = boson.permute(0, 1, 4, 3, 2)[0, 0].to(ec.real.dtype)  # [Ltau, Ly, Lx], x-bond angles
        return ec, g, ph

    @staticmethod
    def _sx(a, k):
        """value at x + k (the reference's torch.roll(a, shifts=-k, dims=-1))"""
        return torch.roll(a, shifts=-k, dims=-1)

    def _chunk(self, ec, n_arrays=4):
        per = ec[0].numel() * ec.element_size() * n_arrays
        return max(1, self.chunk_bytes // max(1, per))

    def _pair_mean(self, ec, fa, fb):
        nrv = ec.shape[0]
        pairs = torch.combinations(torch.arange(nrv, device=ec.device), r=2, with_replacement=False)
        S = torch.zeros((self.Ly, self.Lx), dtype=ec.dtype, device=ec.device)
        for ch in pairs.split(self._chunk(ec)):
            s, t = ch[:, 0], ch[:, 1]
            aF = torch.fft.ifft2(fa(s, t), norm="backward")
            bF = torch.fft.fft2(fb(s, t), norm="forward")
            S += (aF * bF).sum(dim=(0, 1))
        return torch.fft.ifft2(S, norm="forward") / (len(pairs) * self.Ltau)

    # ---- the correlators ----------------------------------------------------
    def T1(self, eta, G_eta, boson):
        ec, g, ph = self._fields(eta, G_eta, boson)
        e = torch.exp(1j * ph)
        sx = self._sx
        out = -self._pair_mean(ec, lambda s, t: ec[s] * sx(g[t], 1) * e, lambda s, t: sx(g[s], 1) * ec[t] * e)
        out[0, -1] += (sx(g, 1) * torch.roll(ec, 1, dims=-1) * e * torch.exp(1j * torch.roll(ph, 1, dims=-1))).mean()
        return out

    def T21(self, eta, G_eta, boson):
        ec, g, ph = self._fields(eta, G_eta, boson)
        em, ep = torch.exp(-1j * ph), torch.exp(1j * ph)
        sx = self._sx
        out = -self._pair_mean(
            ec, lambda s, t: (sx(ec[s], 1) * g[t] + sx(ec[t], 1) * g[s]) * em / 2,
            lambda s, t: (sx(g[s], 1) * ec[t] + sx(g[t], 1) * ec[s]) * ep / 2)
        out[0, 0] += (g * ec).mean()
        return out

    def T2(self, eta, G_eta, boson):
        ec, g, ph = self._fields(eta, G_eta, boson)
        em, ep = torch.exp(-1j * ph), torch.exp(1j * ph)
        sx = self._sx
        out = -self._pair_mean(
            ec, lambda s, t: (ec[s] * sx(g[t], 1) + ec[t] * sx(g[s], 1)) * ep / 2,
            lambda s, t: (g[s] * sx(ec[t], 1) + g[t] * sx(ec[s], 1)) * em / 2)
        out[0, 0] += (g * ec).mean()
        return out

    def T4(self, eta, G_eta, boson):
        ec, g, ph = self._fields(eta, G_eta, boson)
        e = torch.exp(-1j * ph)
        sx = self._sx
        out = -self._pair_mean(ec, lambda s, t: sx(ec[s], 1) * g[t] * e, lambda s, t: g[s] * sx(ec[t], 1) * e)
        out[0, 1] += (g * sx(ec, 2) * e * torch.exp(-1j * sx(ph, 1))).mean()
        return out

    def Tvv(self, eta, G_eta, boson):
        ec, g, ph = self._fields(eta, G_eta, boson)
        sx = self._sx
        ep, em = torch.exp(1j * ph), torch.exp(-1j * ph)
        S = torch.zeros((self.Ly, self.Lx), dtype=ec.dtype, device=ec.device)
        Tv = torch.zeros((self.Ly, self.Lx), dtype=ec.dtype, device=ec.device)
        nrv = ec.shape[0]
        for idx in torch.arange(nrv, device=ec.device).split(self._chunk(ec, 3)):
            v = sx(g[idx], 1) * ec[idx] * ep + g[idx] * sx(ec[idx], 1) * em
            S += (torch.fft.ifft2(v, norm="backward") * torch.fft.fft2(v, norm="forward")).sum(dim=(0, 1))
            Tv += v.sum(dim=(0, 1))
        return torch.fft.ifft2(S, norm="forward") / (nrv * self.Ltau), Tv / (nrv * self.Ltau)

    def get_bond_bond_per_b2(self, eta, G_eta, boson):
        """BB0_r, BB_r, B_r and BB_k (real parts; BB_k in ascending momentum order)."""
        T = self.T1(eta, G_eta, boson) + self.T21(eta, G_eta, boson) + self.T2(eta, G_eta, boson) + \
            self.T4(eta, G_eta, boson)
        Tvv, Tv = self.Tvv(eta, G_eta, boson)
        BB_r = T * 2 + Tvv * 4
        BB_k = torch.fft.ifft2(BB_r, norm="forward")
        BB_k = torch.roll(BB_k, shifts=(self.Ly // 2, self.Lx // 2), dims=(-2, -1))
        return {"BB0_r": (T * 2).real, "BB_r": BB_r.real, "B_r": Tv.real, "BB_k": BB_k.real}

    def bond_corr(self, BB_r_mean, B_r_mean):
        """BB_r minus the disconnected part 4 (B_r correlated with itself)."""
        vF_neg = torch.fft.ifftn(B_r_mean, (self.Ly, self.Lx), norm="backward")
        vF = torch.fft.fftn(B_r_mean, (self.Ly, self.Lx), norm="forward")
        return BB_r_mean - 4 * torch.fft.ifftn(vF_neg * vF, (self.Ly, self.Lx), norm="forward")
