"""Generate golden vectors by running the reference's own CPU path in complex128.

Run where the reference source tree is present, giving its root directory:

    python tests/golden/make_golden.py <reference-root>          # golden_ref.npz, golden_traj.npz
    python tests/golden/make_golden.py <reference-root> bond     # golden_bond.npz
    python tests/golden/make_golden.py <reference-root> fourier  # golden_fourier_mass.npz
    python tests/golden/make_golden.py <reference-root> mid      # golden_traj_L12.npz

The reference module ``qed_fermion.hmc_sampler_batch`` imports ``matplotlib``
and ``matlab.engine`` at module level; neither is needed for the CPU path, so
both are replaced by empty stub modules before the import.  The reference's
module-level dtypes are switched to float64/complex128 and its preconditioner
writer is redirected to a temporary directory (it otherwise writes into its
own source tree).  Nothing here is used at run time by the library; the
``.npz`` files it writes are the fixtures ``tests/test_oracle_golden.py`` pins
the oracle against.
"""
from __future__ import annotations

import math
import os
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _stub_modules():
    for name in ["matplotlib", "matplotlib.pyplot", "matlab", "matlab.engine"]:
        sys.modules[name] = types.ModuleType(name)
    mpl = sys.modules["matplotlib"]
    mpl.use = lambda *a, **k: None
    mpl.rcParams = {}
    plt = sys.modules["matplotlib.pyplot"]
    plt.ion = lambda *a, **k: None
    mpl.pyplot = plt


def import_reference(ref_root: str):
    _stub_modules()
    sys.path.insert(0, ref_root)
    import torch  # noqa: F401
    import qed_fermion.hmc_sampler_batch as H
    import qed_fermion.preconditioners_orig.precon_manual as PM
    H.dtype = torch.float64
    H.cdtype = torch.complex128
    H.cg_dtype = torch.complex128
    H.Nstep = 4
    tmp = tempfile.mkdtemp(prefix="qedf_golden_")
    PM.script_path = os.path.join(tmp, "sub")
    os.makedirs(PM.script_path, exist_ok=True)
    return H, PM


def make_sampler(H, L, Nt, J=1.0):
    import torch
    hmc = H.HmcSampler(Lx=L, Ltau=Nt, J=J, Nstep=4)
    hmc.dtype = torch.float64
    hmc.cdtype = torch.complex128
    hmc.delta_t_tensor = hmc.delta_t_tensor.to(torch.float64)
    return hmc


def uniform_boson(rng, L, Nt):
    return rng.uniform(-math.pi, math.pi, size=(1, 2, L, L, Nt))


def pi_flux_boson(rng, L, Nt, noise=0.1):
    b = np.zeros((1, 2, L, L, Nt))
    for x in range(L):
        for y in range(L):
            sign = (-1) ** (x + y)
            b[0, 0, x, y, :] = sign * math.pi / 4
            b[0, 1, x, y, :] = -sign * math.pi / 4
    return b + noise * rng.standard_normal(b.shape)


def cvec(rng, n):
    return (rng.standard_normal(n) + 1j * rng.standard_normal(n)) / math.sqrt(2)


def gen_geometry(H, out):
    for L in (2, 4, 6, 12, 24):
        hmc = make_sampler(H, L, 10)
        for g in range(1, 5):
            out[f"geom_L{L}_i{g}"] = getattr(hmc, f"i_list_{g}").numpy()
            out[f"geom_L{L}_j{g}"] = getattr(hmc, f"j_list_{g}").numpy()
            out[f"geom_L{L}_b{g}"] = getattr(hmc, f"boson_idx_list_{g}").numpy()


def gen_operators(H, out, rng):
    import torch
    for (L, Nt, kind) in ((4, 10, "uniform"), (6, 20, "uniform"), (4, 30, "piflux")):
        hmc = make_sampler(H, L, Nt)
        b = uniform_boson(rng, L, Nt) if kind == "uniform" else pi_flux_boson(rng, L, Nt)
        boson = torch.tensor(b, dtype=torch.float64)
        MhM, B_list, _, M = H.HmcSampler.get_M_sparse(hmc, boson)
        N = L * L * Nt
        x = torch.tensor(cvec(rng, N), dtype=torch.complex128).view(-1, 1)
        tag = f"L{L}_T{Nt}"
        out[f"op_{tag}_boson"] = b
        out[f"op_{tag}_x"] = x.view(-1).numpy()
        out[f"op_{tag}_Mx"] = torch.sparse.mm(M, x).view(-1).numpy()
        out[f"op_{tag}_MHx"] = torch.sparse.mm(M.t().conj().coalesce(), x).view(-1).numpy()
        out[f"op_{tag}_MHMx"] = torch.sparse.mm(MhM, x).view(-1).numpy()
        # B partial products on slice tau = 1 (F4 v, F3F4 v, ..., B v)
        Vs = L * L
        v = torch.tensor(cvec(rng, Vs), dtype=torch.complex128).view(-1, 1)
        tau = 1
        seq = [B_list[3][tau], B_list[2][tau], B_list[1][tau], B_list[0][tau],
               B_list[1][tau], B_list[2][tau], B_list[3][tau]]
        w = v
        rows = []
        for mat in seq:
            w = torch.sparse.mm(mat, w)
            rows.append(w.view(-1).numpy())
        out[f"bvec_{tag}_v"] = v.view(-1).numpy()
        out[f"bvec_{tag}_tau"] = np.array(tau)
        out[f"bvec_{tag}_rows"] = np.stack(rows)


def gen_precon(H, PM, out):
    import torch
    for (L, Nt) in ((2, 26), (2, 30), (4, 60)):
        PM.get_precon_man(L, Nt)
        path = os.path.join(PM.script_path, "..", "preconditioners",
                            f"precon_ckpt_L_{L}_Ltau_{Nt}_dtau_0.1_t_1.pt")
        d = torch.load(path)
        out[f"precon_L{L}_T{Nt}_indices"] = d["indices"].numpy()
        out[f"precon_L{L}_T{Nt}_values"] = d["values"].numpy()


def gen_cg(H, PM, out, rng):
    import torch
    L, Nt = 4, 30
    hmc = make_sampler(H, L, Nt)
    b = pi_flux_boson(rng, L, Nt)
    boson = torch.tensor(b, dtype=torch.float64)
    MhM, _, _, M = H.HmcSampler.get_M_sparse(hmc, boson)
    N = L * L * Nt
    rhs = torch.tensor(cvec(rng, N), dtype=torch.complex128)
    PM.get_precon_man(L, Nt)
    path = os.path.join(PM.script_path, "..", "preconditioners",
                        f"precon_ckpt_L_{L}_Ltau_{Nt}_dtau_0.1_t_1.pt")
    d = torch.load(path)
    P = torch.sparse_coo_tensor(d["indices"], d["values"], size=d["size"]).coalesce().to(torch.complex128)
    x_cg, cnt_cg, err_cg = hmc.preconditioned_cg(MhM, rhs, None, rtol=1e-10, max_iter=3000,
                                                 cg_dtype=torch.complex128)
    x_pcg, cnt_pcg, err_pcg = hmc.preconditioned_cg(MhM, rhs, P, rtol=1e-10, max_iter=3000,
                                                    cg_dtype=torch.complex128)
    out["cg_boson"] = b
    out["cg_rhs"] = rhs.numpy()
    out["cg_x"] = x_cg.view(-1).numpy()
    out["cg_cnt"] = np.array(cnt_cg)
    out["cg_err"] = np.array(err_cg)
    out["pcg_x"] = x_pcg.view(-1).numpy()
    out["pcg_cnt"] = np.array(cnt_pcg)
    out["pcg_err"] = np.array(err_pcg)


def gen_force(H, out, rng):
    import torch
    for (L, Nt) in ((4, 10), (6, 20)):
        hmc = make_sampler(H, L, Nt)
        hmc.cg_rtol = 1e-13
        hmc.max_iter = 20000
        b = uniform_boson(rng, L, Nt)
        boson = torch.tensor(b, dtype=torch.float64)
        MhM, B_list, _, M = H.HmcSampler.get_M_sparse(hmc, boson)
        N = L * L * Nt
        R = torch.tensor(cvec(rng, N), dtype=torch.complex128).view(-1, 1)
        psi = torch.sparse.mm(M.t().conj().coalesce(), R)
        F, xi, cnt = hmc.force_f_sparse(psi, MhM, boson, B_list)
        tag = f"L{L}_T{Nt}"
        out[f"force_{tag}_boson"] = b
        out[f"force_{tag}_psi"] = psi.view(-1).numpy()
        out[f"force_{tag}_F"] = F.numpy()
        out[f"force_{tag}_xi"] = xi.view(-1).numpy()
        if L == 4:
            # known answer from the reference's own test intent (unit_test/test_force_f.py):
            # F = -dS_f/dphi with S_f = psi^dag (M^dag M)^{-1} psi from the dense M
            with torch.inference_mode(False):
                bb = boson.clone().requires_grad_(True)
                Md, _ = hmc.get_M(bb)
                Ot = Md.conj().T @ Md
                Sf = (psi.view(-1).conj() @ torch.linalg.solve(Ot, psi.view(-1))).real
                Fa = -torch.autograd.grad(Sf, bb)[0]
            out[f"force_{tag}_F_autograd"] = Fa.detach().numpy()


def gen_boson(H, out, rng):
    import torch
    L, Nt = 6, 20
    hmc = make_sampler(H, L, Nt)
    b = rng.uniform(-math.pi, math.pi, size=(2, 2, L, L, Nt))
    boson = torch.tensor(b, dtype=torch.float64)
    out["boson_b"] = b
    out["boson_S_tau"] = hmc.action_boson_tau(boson).numpy()
    out["boson_S_plaq"] = hmc.action_boson_plaq_matfree(boson).numpy()
    out["boson_F_plaq"] = hmc.force_b_plaq_matfree(boson).numpy()
    out["boson_F_tau"] = hmc.force_b_tau_noncmp(boson).numpy()
    out["boson_F_tau_cmp"] = hmc.force_b_tau_cmp(boson).numpy()
    out["boson_J_int"] = np.array(hmc.J)
    out["boson_K_int"] = np.array(hmc.K)
    # curl-matrix form of the plaquette action (unit_test/test_matrix_free.py intent)
    hmc.initialize_curl_mat()
    hmc.bs = 2
    out["boson_S_plaq_curlmat"] = hmc.action_boson_plaq(boson).numpy()


def gen_trajectory(H, out, rng):
    import torch
    L, Nt = 6, 20
    hmc = make_sampler(H, L, Nt)
    hmc.cg_rtol = 1e-10
    hmc.max_iter = 20000
    hmc.N_leapfrog = 10
    b = uniform_boson(rng, L, Nt)
    p0 = rng.standard_normal((1, 2, L, L, Nt))
    R = cvec(rng, L * L * Nt)[None, :] / math.sqrt(2)
    hmc.draw_momentum = lambda: torch.tensor(p0, dtype=torch.float64)
    hmc.draw_psudo_fermion = lambda: torch.tensor(R, dtype=torch.complex128)
    tau_mask = torch.ones((1, 1, 1, 1, Nt), dtype=torch.float64)
    x, H0, H_fin, its, errs = hmc.leapfrog_proposer5(torch.tensor(b, dtype=torch.float64), tau_mask)
    out["traj_boson"] = b
    out["traj_p0"] = p0
    out["traj_R"] = R
    out["traj_x"] = x.numpy()
    out["traj_H0"] = H0.numpy()
    out["traj_Hfin"] = H_fin.numpy()
    out["traj_delta_t"] = np.array(float(hmc.delta_t_tensor[0]))
    out["traj_n_leapfrog"] = np.array(hmc.N_leapfrog)
    out["traj_cg_iters_mean"] = its.numpy()


def gen_trajectory_mid(H, rng):
    """A trajectory at the benchmark's step size (20 leapfrog steps of 0.05)
    on a mid-size lattice, L = 12, Ltau = 120, from the reference's physical
    start (staggered pi-flux plus noise), PCG to 1e-10."""
    import torch
    L, Nt = 12, 120
    hmc = make_sampler(H, L, Nt)
    hmc.cg_rtol = 1e-10
    hmc.max_iter = 50000
    hmc.N_leapfrog = 20
    hmc.delta_t_tensor = torch.full((1,), 0.05, dtype=torch.float64)
    b = pi_flux_boson(rng, L, Nt, noise=0.05)
    p0 = rng.standard_normal((1, 2, L, L, Nt))
    R = cvec(rng, L * L * Nt)[None, :] / math.sqrt(2)
    hmc.draw_momentum = lambda: torch.tensor(p0, dtype=torch.float64)
    hmc.draw_psudo_fermion = lambda: torch.tensor(R, dtype=torch.complex128)
    tau_mask = torch.ones((1, 1, 1, 1, Nt), dtype=torch.float64)
    x, H0, H_fin, its, errs = hmc.leapfrog_proposer5(torch.tensor(b, dtype=torch.float64), tau_mask)
    return {"mid_boson": b, "mid_p0": p0, "mid_R": R, "mid_x": x.numpy(), "mid_H0": H0.numpy(),
            "mid_Hfin": H_fin.numpy(), "mid_delta_t": np.array(0.05), "mid_n_leapfrog": np.array(20),
            "mid_cg_iters_mean": its.numpy()}


def main_mid(ref_root):
    H, _ = import_reference(ref_root)
    out = gen_trajectory_mid(H, np.random.default_rng(20261204))
    np.savez_compressed(os.path.join(HERE, "golden_traj_L12.npz"), **out)
    print("wrote", sorted(out))


def gen_estimator(H, out, rng):
    import torch
    L, Nt, nrv = 4, 10, 6
    hmc = make_sampler(H, L, Nt)
    b = pi_flux_boson(rng, L, Nt)
    boson = torch.tensor(b, dtype=torch.float64)
    _, _, _, M = H.HmcSampler.get_M_sparse(hmc, boson)
    Md = M.to_dense()
    N = L * L * Nt
    re = rng.integers(0, 2, size=(nrv, N)) * 2 - 1
    im = rng.integers(0, 2, size=(nrv, N)) * 2 - 1
    eta = (re + 1j * im) / math.sqrt(2)
    G = torch.linalg.solve(Md, torch.tensor(eta.T, dtype=torch.complex128)).T
    out["se_boson"] = b
    out["se_eta"] = eta
    out["se_G_eta"] = G.numpy()


def main():
    ref_root = sys.argv[1]
    H, PM = import_reference(ref_root)
    rng = np.random.default_rng(20240611)
    out = {}
    gen_geometry(H, out)
    gen_operators(H, out, rng)
    gen_precon(H, PM, out)
    gen_cg(H, PM, out, rng)
    gen_force(H, out, rng)
    gen_boson(H, out, rng)
    gen_estimator(H, out, rng)
    np.savez_compressed(os.path.join(HERE, "golden_ref.npz"), **out)
    traj = {}
    gen_trajectory(H, traj, rng)
    np.savez_compressed(os.path.join(HERE, "golden_traj.npz"), **traj)
    print("wrote", sorted(out.keys()) + sorted(traj.keys()))





def gen_bond_observables(ref_root, rng):
    """The reference estimator's bond-bond correlators (stochastic_estimator.py
    T1 :1393, T21 :1447, T2 :1504, T4 :1561, Tvv :1612, get_bond_bond_per_b2
    :2594, bond_corr :2643) on L=6, Ltau=12 with 12 noise vectors, G_eta from a
    dense solve of M in complex128.  The estimator's constructor would load the
    sampler's preconditioner from the reference's source tree; the correlators do
    not use it, so a placeholder stands in."""
    import torch
    import qed_fermion.hmc_sampler_batch as H
    import qed_fermion.stochastic_estimator as SE
    L, Nt, nrv = 6, 12, 12
    hmc = make_sampler(H, L, Nt)
    hmc.precon_csr = "unused"
    b = pi_flux_boson(rng, L, Nt)
    boson = torch.tensor(b, dtype=torch.float64)
    _, _, _, M = H.HmcSampler.get_M_sparse(hmc, boson)
    N = L * L * Nt
    re = rng.integers(0, 2, size=(nrv, N)) * 2 - 1
    im = rng.integers(0, 2, size=(nrv, N)) * 2 - 1
    eta = torch.tensor((re + 1j * im) / math.sqrt(2), dtype=torch.complex128)
    G = torch.linalg.solve(M.to_dense(), eta.T).T.contiguous()
    SE.Nrv = nrv
    se = SE.StochaticEstimator(hmc)
    se.Nrv = nrv
    se.initialize()
    se.eta, se.G_eta = eta, G
    out = {"bb_boson": b, "bb_eta": eta.numpy(), "bb_G_eta": G.numpy()}
    for name in ("T1", "T21", "T2", "T4"):
        out[f"bb_{name}"] = getattr(se, name)(eta, G, boson).numpy()
    tvv, tv = se.Tvv(eta, G, boson)
    out["bb_Tvv"], out["bb_Tv"] = tvv.numpy(), tv.numpy()
    obsr = se.get_bond_bond_per_b2(boson)
    for k in ("BB0_r", "BB_r", "B_r", "BB_k"):
        out[f"bb_obsr_{k}"] = obsr[k].numpy()
    out["bb_bond_corr"] = se.bond_corr(obsr["BB_r"], obsr["B_r"]).numpy()
    return out


def main_bond(ref_root):
    import_reference(ref_root)
    rng = np.random.default_rng(20241203)
    out = gen_bond_observables(ref_root, rng)
    np.savez_compressed(os.path.join(HERE, "golden_bond.npz"), **out)
    print("wrote", sorted(out))


def gen_fourier_mass(rng):
    """The reference's adaptive Fourier mass (hmc_sampler_batch.py:272-285,
    1133-1277) on L=4, Ltau=10: 12 fields folded into the statistics with a
    window of 5 and annealing every 4 steps, the mass formed at step 10 in mass
    modes 1 and -1, M^{-1} applied to a momentum, and a momentum drawn with a
    seeded torch generator."""
    import torch
    import qed_fermion.hmc_sampler_batch as H
    out = {}
    L, Nt = 4, 10
    fields = rng.standard_normal((12, 1, 2, L, L, Nt))
    p = rng.standard_normal((1, 2, L, L, Nt))
    out["fm_fields"], out["fm_p"] = fields, p
    for mode in (1, -1):
        H.mass_mode = mode
        hmc = make_sampler(H, L, Nt)
        hmc.sigma_mini_batch_size = 5
        hmc.annealing_step = 4
        for i in range(12):
            hmc.update_sigma_hat_cpu(torch.tensor(fields[i]), i)
        out[f"fm{mode}_sigma_hat_cpu"] = hmc.sigma_hat_cpu.numpy()
        out[f"fm{mode}_boson_mean_cpu"] = hmc.boson_mean_cpu.numpy()
        hmc.apply_sigma_hat_cpu(10)
        out[f"fm{mode}_sigma_hat"] = hmc.sigma_hat.numpy()
        out[f"fm{mode}_m_inv_p"] = hmc.apply_m_inv(torch.tensor(p)).numpy()
        torch.manual_seed(77)
        out[f"fm{mode}_p_fft"] = hmc.draw_momentum_fft().numpy()
    H.mass_mode = 0
    return out


def main_fourier(ref_root):
    import_reference(ref_root)
    out = gen_fourier_mass(np.random.default_rng(20241204))
    np.savez_compressed(os.path.join(HERE, "golden_fourier_mass.npz"), **out)
    print("wrote", sorted(out))


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: make_golden.py <reference-root> [bond|fourier]")
    if len(sys.argv) > 2 and sys.argv[2] == "bond":
        main_bond(sys.argv[1])
    elif len(sys.argv) > 2 and sys.argv[2] == "fourier":
        main_fourier(sys.argv[1])
    elif len(sys.argv) > 2 and sys.argv[2] == "mid":
        main_mid(sys.argv[1])
    else:
        main()
