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
per batch.  Pairs are processed in chunks sized by ``chunk_bytes``: per chunk
one kernel writes both fields of every pair (``ops.bb_pair_fields``), cuFFT
transforms them, and one kernel adds the products of the transforms into a
double-precision k-space sum (``ops.bb_kspace_acc``).

Layouts as in the reference: eta, G_eta ``[Nrv, Ltau * Ly * Lx]`` (index
tau Vs + x + Lx y); boson ``[1, 2, Lx, Ly, Ltau]``.  Inputs must be CUDA
tensors; the transforms are cuFFT's (through torch).
"""
from __future__ import annotations

import torch

from . import ops


class BondBond:
    def __init__(self, Lx: int, Ltau: int, chunk_bytes: int = 1 << 30, fused: bool = False):
        self.Lx = self.Ly = Lx
        self.Ltau = Ltau
        self.chunk_bytes = int(chunk_bytes)
        # fused=True: one-pass pair sums (ops.bb_corr, fields and transforms in
        # shared memory) where the lattice fits that kernel.  Measured at
        # L = 36, Ltau = 360, 64 vectors: 113 ms per correlator against 35 ms for
        # the two-pass path (pair fields, cuFFT, k-space sum), so off by default
        self.fused = bool(fused)

    # ---- helpers ----------------------------------------------------------
    def _chunk(self, ec, n_arrays=4):
        per = ec[0].numel() * ec.element_size() * n_arrays
        return max(1, self.chunk_bytes // max(1, per))

    def _pair_mean(self, kind, eta, G_eta, boson):
        """mean over pairs s < t and tau of ifft2(a_st) * fft2(b_st), transformed
        back to real space; a_st, b_st are the fields of correlator ``kind``."""
        dt = eta.dtype
        nrv = eta.shape[0]
        if nrv < 2:
            raise RuntimeError("bond-bond correlators need at least two noise vectors")
        e = eta.resolve_conj().reshape(nrv, -1).contiguous()
        g = G_eta.to(dt).resolve_conj().reshape(nrv, -1).contiguous()
        ph = boson.permute(0, 1, 4, 3, 2)[0, 0].to(e.real.dtype)
        ep = torch.exp(1j * ph).to(dt).contiguous()
        Vs = self.Lx * self.Ly
        pairs = torch.combinations(torch.arange(nrv, device=e.device), r=2, with_replacement=False).to(torch.int32)
        S = torch.zeros(Vs, dtype=torch.complex128, device=e.device)
        if self.fused and ops.bb_corr(kind, e, g, ep, pairs[:, 0].contiguous(), pairs[:, 1].contiguous(), self.Lx, S):
            S = S.view(self.Ly, self.Lx) / (Vs * Vs)
            return (torch.fft.ifft2(S, norm="forward") / (len(pairs) * self.Ltau)).to(dt)
        chunk = min(65535, self._chunk(e.reshape(nrv, self.Ltau, self.Ly, self.Lx)), len(pairs))
        fa = torch.empty((chunk, self.Ltau, self.Ly, self.Lx), dtype=dt, device=e.device)
        fb = torch.empty_like(fa)
        for ch in pairs.split(chunk):
            n = len(ch)
            a, b = fa[:n], fb[:n]
            ops.bb_pair_fields(kind, e, g, ep, ch[:, 0].contiguous(), ch[:, 1].contiguous(), self.Lx, a, b)
            # unnormalised transforms; the 1 / Vs of each is applied to S once
            ops.bb_kspace_acc(torch.fft.ifft2(a, norm="forward"), torch.fft.fft2(b, norm="backward"), S)
        S = S.view(self.Ly, self.Lx) / (Vs * Vs)
        return (torch.fft.ifft2(S, norm="forward") / (len(pairs) * self.Ltau)).to(dt)

    def _inputs(self, eta, G_eta, boson):
        """eta, G_eta as contiguous [Nrv, N] of one dtype and e^{i phi_x} [Ltau, Ly, Lx]."""
        dt = eta.dtype
        nrv = eta.shape[0]
        e = eta.resolve_conj().reshape(nrv, -1).contiguous()
        g = G_eta.to(dt).resolve_conj().reshape(nrv, -1).contiguous()
        ph = boson.permute(0, 1, 4, 3, 2)[0, 0].to(e.real.dtype)
        return e, g, torch.exp(1j * ph).to(dt).contiguous()

    def _diag(self, eta, G_eta, boson):
        """The three short-distance terms as means (kernel ``bb_diag``)."""
        e, g, ep = self._inputs(eta, G_eta, boson)
        return ops.bb_diag(e, g, ep, self.Lx) / e.numel()

    # ---- the correlators ----------------------------------------------------
    def T1(self, eta, G_eta, boson):
        out = -self._pair_mean("T1", eta, G_eta, boson)
        out[0, -1] += self._diag(eta, G_eta, boson)[0].to(out.dtype)
        return out

    def T21(self, eta, G_eta, boson):
        out = -self._pair_mean("T21", eta, G_eta, boson)
        out[0, 0] += self._diag(eta, G_eta, boson)[1].to(out.dtype)
        return out

    @staticmethod
    def _reflect(a):
        """a at -d: element (-dy mod Ly, -dx mod Lx) at (dy, dx)"""
        return torch.roll(torch.flip(a, dims=(-2, -1)), shifts=(1, 1), dims=(-2, -1))

    def T2(self, eta, G_eta, boson):
        """T2's two pair fields are T21's with a and b exchanged:
        (ec_s g_t(r+x) + ec_t g_s(r+x)) e/2 is T21's b, and (g_s ec_t(r+x) +
        g_t ec_s(r+x)) e*/2 is T21's a.  Its pair correlation is therefore T21's
        at -d, and both add the same term at d = 0, so T2 is T21 reflected."""
        return self._reflect(self.T21(eta, G_eta, boson))

    def T2_direct(self, eta, G_eta, boson):
        """T2 from its own pair fields (the reference's computation)."""
        out = -self._pair_mean("T2", eta, G_eta, boson)
        out[0, 0] += self._diag(eta, G_eta, boson)[1].to(out.dtype)
        return out

    def T4(self, eta, G_eta, boson):
        out = -self._pair_mean("T4", eta, G_eta, boson)
        out[0, 1] += self._diag(eta, G_eta, boson)[2].to(out.dtype)
        return out

    def Tvv(self, eta, G_eta, boson):
        """The current-current correlation and the mean current: each vector's
        field v (kernel ``bb_vfield``, which also sums it), the products of its
        transforms summed in k-space (``bb_kspace_acc``), one inverse FFT."""
        e, g, ep = self._inputs(eta, G_eta, boson)
        nrv = e.shape[0]
        Vs = self.Lx * self.Ly
        S = torch.zeros(Vs, dtype=torch.complex128, device=e.device)
        Tv = torch.zeros(Vs, dtype=torch.complex128, device=e.device)
        per = max(1, self.chunk_bytes // max(1, 3 * e[0].numel() * e.element_size()))
        v = torch.empty((min(per, nrv), self.Ltau, self.Ly, self.Lx), dtype=e.dtype, device=e.device)
        for lo in range(0, nrv, per):
            n = min(per, nrv - lo)
            vb = v[:n]
            ops.bb_vfield(e[lo:lo + n], g[lo:lo + n], ep, self.Lx, vb, Tv)
            # the reference's ifft2(v, "backward") * fft2(v, "forward"): unnormalised
            # transforms here, their two 1 / Vs applied to the sum once
            ops.bb_kspace_acc(torch.fft.ifft2(vb, norm="forward"), torch.fft.fft2(vb, norm="backward"), S)
        S = S.view(self.Ly, self.Lx) / (Vs * Vs)
        dt = eta.dtype
        return ((torch.fft.ifft2(S, norm="forward") / (nrv * self.Ltau)).to(dt),
                (Tv.view(self.Ly, self.Lx) / (nrv * self.Ltau)).to(dt))

    def get_bond_bond_per_b2(self, eta, G_eta, boson):
        """BB0_r, BB_r, B_r and BB_k (real parts; BB_k in ascending momentum order)."""
        t21 = self.T21(eta, G_eta, boson)
        T = self.T1(eta, G_eta, boson) + t21 + self._reflect(t21) + self.T4(eta, G_eta, boson)
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
