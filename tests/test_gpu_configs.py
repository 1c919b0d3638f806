"""The benchmark configurations beyond C1/C3 on the GPU, checked against the oracle.

C2  L=24, Ltau=240, uniform angles, b = M^dag eta: M^dag M in complex64 and
    complex128, PCG to 1e-8 with float iterations (mixed) and in double.
C4a L=36, Ltau=360, one configuration, 64 Z2 noise vectors solved jointly.
C4b 16 lattices L in {12, 18, 24, 30} x 4, Ltau = 10 L, one launch, one mask each.
C5  L=66, Ltau=660: the adjoint force against central differences of the action
    (h = 1e-5, 32 seeded bonds) and against the oracle's force, and one
    trajectory of 30 leapfrog steps.
The oracle checks use its operator on the same angles (true residuals) and its
force on a few slices, which keeps the CPU side to seconds.
"""
import math

import numpy as np
import pytest
import torch

from oracle import qedf_oracle as O

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0") if torch.cuda.is_available() else None


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from qed_fermion_b200 import build
    build.build()
    torch.cuda.set_device(DEV)


def piflux(rng, L, Nt, bs, noise=0.1):
    x = np.arange(L)[:, None]
    y = np.arange(L)[None, :]
    sg = 1 - 2 * ((x + y) % 2)
    b = np.zeros((bs, 2, L, L, Nt))
    b[:, 0] = (sg * np.pi / 4)[None, :, :, None]
    b[:, 1] = (-sg * np.pi / 4)[None, :, :, None]
    return b + noise * rng.standard_normal(b.shape)


def true_relres(phi_k, x, b, L, Nt):
    n = b.shape[0]
    r = b - O.mhm_vec(phi_k, x.reshape(n, Nt, L * L), L, 0.1).reshape(n, -1)
    return np.linalg.norm(r, axis=1) / np.linalg.norm(b, axis=1)


def test_c2_matvec_and_pcg():
    from qed_fermion_b200 import ops
    from qed_fermion_b200.solver import PcgSolver, System
    L, Nt = 24, 240
    rng = np.random.default_rng(2)
    boson = rng.uniform(-np.pi, np.pi, size=(1, 2, L, L, Nt))
    phi = O.ref_to_kernel_layout(boson)
    eta = (rng.standard_normal((1, Nt * L * L)) + 1j * rng.standard_normal((1, Nt * L * L))) / math.sqrt(2)
    b = O.mh_vec(phi, eta.reshape(1, Nt, L * L), L, 0.1).reshape(1, -1)
    want = O.mhm_vec(phi, b.reshape(1, Nt, L * L), L, 0.1).reshape(1, -1)
    for cdt, rdt, tol in ((torch.complex64, torch.float32, 1e-6), (torch.complex128, torch.float64, 1e-13)):
        got = ops.apply_operator("mhm", torch.tensor(phi.reshape(1, -1), dtype=rdt, device=DEV),
                                 torch.tensor(b, dtype=cdt, device=DEV), L, 0.1).cpu().numpy()
        assert np.abs(got - want).max() / np.abs(want).max() < tol
    for mode in ("mixed", "fp64"):
        s = PcgSolver([System(L, Nt, 1)], mode=mode, rtol=1e-8, max_iter=200000, device=DEV)
        res = s.solve(torch.tensor(phi.reshape(-1), dtype=s.angle_dtype, device=DEV),
                      torch.tensor(b.reshape(-1), dtype=s.vec_dtype, device=DEV))
        assert res.status.cpu().tolist() == [0], (mode, res.iters.cpu().tolist(), res.relres.cpu().tolist())
        ph = phi.astype(np.float32).astype(np.float64) if mode == "mixed" else phi
        assert true_relres(ph, res.x.cpu().numpy(), b, L, Nt)[0] < 2e-8


def test_c4a_64_noise_vectors_one_field():
    from qed_fermion_b200.estimator import StochaticEstimator
    L, Nt, nrv = 36, 360, 64
    rng = np.random.default_rng(4)
    boson = piflux(rng, L, Nt, 1)
    se = StochaticEstimator(L, Nt, Nrv=nrv, precision="mixed", cg_rtol=1e-10, device=DEV, seed=5, noise="z2")
    eta = se.random_vec_bin()  # +-1 complex128 entries
    assert set(np.unique(eta.real.cpu().numpy())) == {-1.0, 1.0} and float(eta.imag.abs().max()) == 0.0
    G = se.set_eta_G_eta(torch.tensor(boson, device=DEV), eta)
    assert se.status.cpu().tolist() == [0] * nrv
    assert float(se.relres.max()) <= 1e-10
    # two of the 64 against the oracle: M G = eta  <=>  M^dag M G = M^dag eta
    phi = O.ref_to_kernel_layout(boson).astype(np.float32).astype(np.float64)
    for k in (0, 63):
        Gk = G[k].cpu().numpy().reshape(1, Nt, L * L)
        MG = O.m_vec(phi, Gk, L, 0.1).reshape(-1)
        e = eta[k].cpu().numpy()
        assert np.linalg.norm(MG - e) / np.linalg.norm(e) < 1e-8


def test_c4b_sixteen_uneven_lattices_one_launch():
    from qed_fermion_b200.solver import PcgSolver, System
    rng = np.random.default_rng(44)
    Ls = [12, 18, 24, 30] * 4
    systems = [System(L, 10 * L, 1) for L in Ls]
    phis, bs_ = [], []
    for L in Ls:
        bos = piflux(rng, L, 10 * L, 1)
        phis.append(O.ref_to_kernel_layout(bos).reshape(-1))
        bs_.append(((rng.standard_normal(10 * L ** 3) + 1j * rng.standard_normal(10 * L ** 3)) / math.sqrt(2)))
    s = PcgSolver(systems, mode="mixed", rtol=1e-10, max_iter=20000, device=DEV)
    res = s.solve(torch.tensor(np.concatenate(phis), dtype=torch.float32, device=DEV),
                  torch.tensor(np.concatenate(bs_), device=DEV))
    assert res.status.cpu().tolist() == [0] * 16
    x = res.x.cpu().numpy()
    off = 0
    for k, L in enumerate(Ls):
        n = 10 * L ** 3
        ph = phis[k].astype(np.float32).astype(np.float64).reshape(1, 10 * L, -1)
        assert true_relres(ph, x[off:off + n].reshape(1, -1), bs_[k].reshape(1, -1), L, 10 * L)[0] < 2e-10
        off += n
    assert len(set(res.iters.cpu().tolist())) > 1


def test_c5_force_finite_differences_and_trajectory():
    from qed_fermion_b200 import ops
    from qed_fermion_b200.force import fermion_action
    from qed_fermion_b200.hmc import HmcSampler, kernel_to_ref
    from qed_fermion_b200.solver import PcgSolver, System
    L, Nt = 66, 660
    rng = np.random.default_rng(66)
    boson = piflux(rng, L, Nt, 1, noise=0.05)
    phi = torch.tensor(O.ref_to_kernel_layout(boson).reshape(1, -1), dtype=torch.float32, device=DEV)
    psi = torch.tensor((rng.standard_normal((1, Nt * L * L)) + 1j * rng.standard_normal((1, Nt * L * L)))
                       / math.sqrt(2), device=DEV)
    solver = PcgSolver([System(L, Nt, 1)], mode="mixed", rtol=1e-12, max_iter=50000, device=DEV)
    phi_g = phi.clone().requires_grad_(True)
    S = fermion_action(phi_g, psi, solver, L, 0.1)
    (g,) = torch.autograd.grad(S.sum(), phi_g)
    # against the oracle's force on three slices (F_t needs xi_t, xi_{t+1}, phi_t)
    xi = solver.solve(phi, psi).x.view(1, Nt, L * L).cpu().numpy()
    ph = phi.double().cpu().numpy().reshape(1, Nt, -1)
    for t in (0, 331, Nt - 1):
        tn = (t + 1) % Nt
        if t != Nt - 1:
            # ring [t, t+1, t]: slice 0 carries sign -1 and sees slice t+1 next
            sel, pos = [t, tn, t], 0
        else:
            # ring [0, Nt-1]: the last slice carries the antiperiodic +1 and sees slice 0
            sel, pos = [0, t], 1
        Fo = O.force_f_from_xi(ph[:, sel], xi[:, sel], L, 0.1)[:, pos]
        Fg = -g.view(1, Nt, -1)[:, t].double().cpu().numpy()
        assert np.abs(Fg - Fo).max() / np.abs(Fo).max() < 2e-5, t
    # central differences: S(phi+h) - S(phi-h) = xi_+^dag (A(phi-h) - A(phi+h)) xi_-
    h = 1e-5
    idx = rng.choice(phi.numel(), 32, replace=False)
    for k in idx:
        pp = phi.double().clone()
        pm = phi.double().clone()
        pp[0, k] += h
        pm[0, k] -= h
        s64 = PcgSolver([System(L, Nt, 1)], mode="fp64", rtol=1e-12, max_iter=50000, device=DEV)
        xp = s64.solve(pp, psi).x.view(1, -1)
        xm = s64.solve(pm, psi).x.view(1, -1)
        dA = ops.apply_operator("mhm", pm, xm, L, 0.1) - ops.apply_operator("mhm", pp, xm, L, 0.1)
        fd = float(torch.vdot(xp.view(-1), dA.view(-1)).real) / (2 * h)
        # the mixed path's force is computed in float; tolerance of the reference's
        # own force test (unit_test/test_force_f.py:73: atol 1e-4, rtol 1e-5)
        assert abs(fd - float(g[0, k])) <= 1e-4 + 1e-5 * abs(fd), (int(k), fd, float(g[0, k]))
    # one trajectory of 30 leapfrog steps, Delta H in double
    hmc = HmcSampler(Lx=L, Ltau=Nt, bs=1, precision="mixed", cg_rtol=1e-10, max_iter=50000, delta_t=0.02,
                     N_leapfrog=30, device=DEV, seed=6)
    x1, H0, H1, it, err = hmc.leapfrog_proposer5(torch.tensor(boson, dtype=torch.float32, device=DEV))
    assert torch.isfinite(H1).all() and int(hmc.last_status.max()) == 0
    assert abs(float(H1 - H0)) < 1e-3 * abs(float(H0))
