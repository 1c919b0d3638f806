"""Run the reference's own HmcSampler and StochaticEstimator (installed under
baseline/_ref) on this library's drop-in ``qed_fermion._C`` and compare
their results with the oracle.  Called as a script by
tests/test_gpu_reference_dropin.py (a fresh process, since the reference
reads its configuration from the environment when it is imported); prints
one JSON line with the measured errors.

The reference calls checked are ``force_f_fast`` (hmc_sampler_batch.py:2150-2227:
its per-slice loop of _C.b_vec_per_tau and df_dot_bs1, around
Ot_inv_psi_fast -> preconditioned_cg_fast_test, :751-846, with _C.mhm_vec and
_C.precon_vec) and ``StochaticEstimator.set_eta_G_eta``
(stochastic_estimator.py:409-433: _C.mh_vec and the same solver with Nrv
right-hand sides).  The reference's GPU solver is complex64 only (it asserts
so), so its results are compared at single-precision tolerances.
"""
import json
import os
import sys
import tempfile
import types

import numpy as np

L, LTAU, BS, NRV = 6, 60, 2, 4


def main(ref_dir, repo):
    os.environ.update({"L": str(L), "bs": str(BS), "cuda_graph": "0", "max_iter": "5000", "precon": "1",
                       "debug": "0", "Nrv": str(NRV), "max_iter_se": "5000", "seed": "42"})
    sys.path.insert(0, repo)
    import torch
    import qed_fermion_b200
    from qed_fermion_b200 import build
    build.build()
    qed_fermion_b200.install_as_reference_C()
    for name in ["matplotlib", "matplotlib.pyplot", "matlab", "matlab.engine"]:
        sys.modules[name] = types.ModuleType(name)
    sys.modules["matplotlib"].use = lambda *a, **k: None
    sys.modules["matplotlib"].rcParams = {}
    sys.modules["matplotlib.pyplot"].ion = lambda *a, **k: None
    sys.modules["matplotlib"].pyplot = sys.modules["matplotlib.pyplot"]
    sys.path.insert(0, ref_dir)
    import qed_fermion.hmc_sampler_batch as H
    import qed_fermion.preconditioners_orig.precon_manual as PM
    from qed_fermion.stochastic_estimator import StochaticEstimator
    from oracle import qedf_oracle as O
    assert H._C is qed_fermion_b200._C, "the reference did not bind the drop-in _C"
    H.Nstep = 4  # a module global the reference's __main__ block defines and its sampler reads
    # the reference writes its preconditioner file next to its sources; keep it in a temp dir
    tmp = tempfile.mkdtemp(prefix="qedf_dropin_")
    H.script_path = tmp
    PM.script_path = os.path.join(tmp, "sub")
    os.makedirs(PM.script_path, exist_ok=True)

    hmc = H.HmcSampler(Lx=L, Ltau=LTAU, J=1.0, Nstep=4)
    hmc.cg_rtol = 1e-6
    hmc.max_iter = 5000
    hmc.reset_precon()
    dev = torch.device("cuda")
    rng = np.random.default_rng(11)
    x = np.arange(L)[:, None]
    y = np.arange(L)[None, :]
    sg = 1 - 2 * ((x + y) % 2)
    b64 = np.zeros((BS, 2, L, L, LTAU))
    b64[:, 0] = (sg * np.pi / 4)[None, :, :, None]
    b64[:, 1] = (-sg * np.pi / 4)[None, :, :, None]
    b64 += 0.1 * rng.standard_normal(b64.shape)
    boson = torch.tensor(b64, dtype=torch.float32, device=dev)
    b64 = boson.double().cpu().numpy()  # the angles the GPU sees
    N = L * L * LTAU
    psi64 = (rng.standard_normal((BS, N)) + 1j * rng.standard_normal((BS, N))) / np.sqrt(2)
    psi = torch.tensor(psi64, dtype=torch.complex64, device=dev)
    psi64 = psi.cpu().numpy().astype(np.complex128)

    out = {}
    # 1. the reference's fermion force on the drop-in kernels
    Ft, xi, it, err = hmc.force_f_fast(psi, boson, None)
    torch.cuda.synchronize()
    cp = O.Couplings()
    P = O.precon_tau_matrix(LTAU)
    F_ref, xi_ref, _, _ = O.fermion_force(b64, psi64.reshape(BS, LTAU, L * L), L, cp, 1e-12, 20000, P)
    out["force_rel_err"] = float(np.abs(Ft.double().cpu().numpy() - F_ref).max() / np.abs(F_ref).max())
    out["xi_rel_err"] = float(np.abs(xi.cpu().numpy() - xi_ref.reshape(BS, -1)).max() / np.abs(xi_ref).max())
    out["force_cg_iters"] = it.cpu().tolist()

    # 2. its PCG loop alone: the true residual of its solution
    phi_k = boson.permute([0, 4, 3, 2, 1]).reshape(BS, LTAU, -1)
    xs, its, errs = hmc.preconditioned_cg_fast_test(phi_k, psi.clone())
    x_np = xs.cpu().numpy().astype(np.complex128)
    r = psi64 - O.mhm_vec(O.ref_to_kernel_layout(b64), x_np.reshape(BS, LTAU, L * L), L, 0.1).reshape(BS, -1)
    out["pcg_true_rel_residual"] = (np.linalg.norm(r, axis=1) / np.linalg.norm(psi64, axis=1)).tolist()
    out["pcg_iters"] = its.cpu().tolist()

    # 3. the estimator's noise solves
    se = StochaticEstimator(hmc)
    eta = se.random_vec_bin()
    se.set_eta_G_eta(boson[:1], eta)
    torch.cuda.synchronize()
    G_ref, _, _ = O.g_eta(O.ref_to_kernel_layout(b64[:1])[0], eta.cpu().numpy().astype(np.complex128), L, cp,
                          1e-12, 20000, P)
    G = se.G_eta.cpu().numpy()
    out["g_eta_rel_err"] = float(np.abs(G - G_ref).max() / np.abs(G_ref).max())
    out["bs_restored"] = int(hmc.bs)
    print(json.dumps(out))


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
