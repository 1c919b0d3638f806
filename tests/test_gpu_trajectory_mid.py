"""A trajectory at the benchmark's step size (20 leapfrog steps of 0.05) on a
mid-size lattice, L = 12, Ltau = 120, against the reference's own
leapfrog_proposer5 run in complex128 on the same start, momenta and
pseudofermion draw (tests/golden/golden_traj_L12.npz; the reference's CPU
path, PCG to rtol 1e-10).

Tolerances: the plain FP64 path reproduces Delta H to 1e-9 of |H0|; the mixed
paths meet the stated bar, Delta H within 1e-6 of |H0|.  The error is also
bounded relative to Delta H itself (1e-3 mixed, 1e-7 FP64), which is the
stricter measure when Delta H is O(1)."""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
DEV = torch.device("cuda:0") if torch.cuda.is_available() else None


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from qed_fermion_b200 import build
    build.build()
    torch.cuda.set_device(DEV)


@pytest.mark.parametrize("precision,chrono", [("fp64", None), ("mixed", None), ("mixed_bf16", None), ("mixed_f16", None),
                                              ("fp64", "linear"), ("mixed", "last"), ("mixed", "linear")])
def test_mid_size_trajectory_matches_reference(precision, chrono):
    """``chrono``: the leapfrog's solves start from the previous solutions
    instead of zero; the same tolerances hold."""
    from qed_fermion_b200.hmc import HmcSampler
    T = dict(np.load(os.path.join(HERE, "golden", "golden_traj_L12.npz")))
    hmc = HmcSampler(Lx=12, Ltau=120, bs=1, precision=precision, cg_rtol=1e-10, max_iter=50000,
                     delta_t=float(T["mid_delta_t"]), N_leapfrog=int(T["mid_n_leapfrog"]), device=DEV,
                     chrono_guess=chrono)
    x, H0, H1, it, err = hmc.leapfrog_proposer5(torch.tensor(T["mid_boson"], device=DEV),
                                                p0=torch.tensor(T["mid_p0"], device=DEV),
                                                R=torch.tensor(T["mid_R"], device=DEV))
    H0r, H1r = float(T["mid_H0"][0]), float(T["mid_Hfin"][0])
    dH, dHr = float(H1 - H0), float(H1r - H0r)
    err_abs = abs(dH - dHr)
    print(f"{precision}: dH {dH:.9f} reference {dHr:.9f}; |error| {err_abs:.3e} = "
          f"{err_abs / abs(H0r):.2e} of |H0|, {err_abs / abs(dHr):.2e} of dH")
    xr = T["mid_x"]
    x_err = float(np.abs(x.cpu().numpy() - xr).max() / np.abs(xr).max())
    if precision == "fp64":
        assert abs(float(H0) - H0r) < 1e-11 * abs(H0r)
        assert err_abs < 1e-9 * abs(H0r) and err_abs < 1e-7 * abs(dHr)
        assert x_err < 1e-9
    else:
        assert err_abs < 1e-6 * abs(H0r), (dH, dHr)
        assert err_abs < 1e-3 * abs(dHr), (dH, dHr)
        assert x_err < 1e-4
