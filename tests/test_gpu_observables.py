"""Bond-bond correlators of the stochastic estimator on the GPU, against the
reference's own values (golden fixture) and the oracle."""
import os

import numpy as np
import pytest
import torch

from oracle import qedf_oracle as O

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
DEV = torch.device("cuda:0") if torch.cuda.is_available() else None


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from qed_fermion_b200 import build
    build.build()


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max()


@pytest.mark.parametrize("chunk_bytes", [1 << 30, 20000])
def test_correlators_match_reference_fixture(chunk_bytes):
    from qed_fermion_b200.observables import BondBond
    G = dict(np.load(os.path.join(HERE, "golden", "golden_bond.npz")))
    bb = BondBond(6, 12, chunk_bytes=chunk_bytes)
    eta, g, bos = (torch.tensor(G[k], device=DEV) for k in ("bb_eta", "bb_G_eta", "bb_boson"))
    for name in ("T1", "T21", "T2", "T4"):
        assert rel(getattr(bb, name)(eta, g, bos).cpu(), G[f"bb_{name}"]) < 1e-12, name
    tvv, tv = bb.Tvv(eta, g, bos)
    assert rel(tvv.cpu(), G["bb_Tvv"]) < 1e-12 and rel(tv.cpu(), G["bb_Tv"]) < 1e-12
    ob = bb.get_bond_bond_per_b2(eta, g, bos)
    for k in ("BB0_r", "BB_r", "B_r", "BB_k"):
        assert rel(ob[k].cpu(), G[f"bb_obsr_{k}"]) < 1e-12, k
    bc = bb.bond_corr(torch.tensor(G["bb_obsr_BB_r"], device=DEV), torch.tensor(G["bb_obsr_B_r"], device=DEV))
    assert rel(bc.cpu(), G["bb_bond_corr"]) < 1e-12


@pytest.mark.parametrize("cdt,tol", [(torch.complex128, 1e-11), (torch.complex64, 2e-5)])
def test_estimator_observables_match_oracle(cdt, tol):
    """G_eta from the library's own solve at L=12, Ltau=30, 10 Z2 vectors; the
    observables in both precisions against the oracle on the same inputs."""
    from qed_fermion_b200.estimator import StochaticEstimator
    L, Nt, nrv = 12, 30, 10
    rng = np.random.default_rng(12)
    x = np.arange(L)[:, None]
    y = np.arange(L)[None, :]
    sg = 1 - 2 * ((x + y) % 2)
    boson = np.zeros((1, 2, L, L, Nt))
    boson[:, 0] = (sg * np.pi / 4)[None, :, :, None]
    boson[:, 1] = (-sg * np.pi / 4)[None, :, :, None]
    boson += 0.1 * rng.standard_normal(boson.shape)
    se = StochaticEstimator(L, Nt, Nrv=nrv, precision="fp64", cg_rtol=1e-12, device=DEV, seed=7)
    eta = se.random_vec_bin()
    bos = torch.tensor(boson, device=DEV)
    se.set_eta_G_eta(bos, eta)
    se.eta, se.G_eta = se.eta.to(cdt), se.G_eta.to(cdt)
    ob = se.get_bond_bond_per_b2(bos)
    want = O.bb_observables(se.eta.cpu().numpy().astype(np.complex128), se.G_eta.cpu().numpy().astype(np.complex128),
                            boson, L, Nt)
    for k in ("BB0_r", "BB_r", "B_r", "BB_k"):
        assert rel(ob[k].double().cpu(), want[k]) < tol, k


def test_cpu_tensors_are_refused():
    from qed_fermion_b200.observables import BondBond
    bb = BondBond(4, 6)
    with pytest.raises(RuntimeError):
        bb.T1(torch.zeros(3, 96, dtype=torch.complex128), torch.zeros(3, 96, dtype=torch.complex128),
              torch.zeros(1, 2, 4, 4, 6))
