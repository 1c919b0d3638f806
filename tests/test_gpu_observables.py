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


def _fields_torch(kind, eta, g, ep, s, t):
    """the two pair fields of a correlator, written with torch for the check
    (x-shift by one site: roll by -1 along x)"""
    ec = eta.conj()
    sx = lambda a: torch.roll(a, shifts=-1, dims=-1)
    em = ep.conj()
    if kind == "T1":
        return ec[s] * sx(g[t]) * ep, sx(g[s]) * ec[t] * ep
    if kind == "T4":
        return sx(ec[s]) * g[t] * em, g[s] * sx(ec[t]) * em
    if kind == "T21":
        return ((sx(ec[s]) * g[t] + sx(ec[t]) * g[s]) * em / 2, (sx(g[s]) * ec[t] + sx(g[t]) * ec[s]) * ep / 2)
    return ((ec[s] * sx(g[t]) + ec[t] * sx(g[s])) * ep / 2, (g[s] * sx(ec[t]) + g[t] * sx(ec[s])) * em / 2)


@pytest.mark.parametrize("kind", ["T1", "T21", "T2", "T4"])
@pytest.mark.parametrize("cdt,tol", [(torch.complex128, 1e-14), (torch.complex64, 1e-6)])
def test_pair_fields_and_kspace_sum_kernels(kind, cdt, tol):
    """The pair-field kernel against torch products for every correlator, with
    an out-of-range pair index giving zero fields; the k-space sum against a
    torch sum of the transforms' products."""
    from qed_fermion_b200 import ops
    L, Nt, nrv = 6, 5, 4
    gen = torch.Generator(device="cpu").manual_seed(3)
    mk = lambda *sh: torch.complex(torch.randn(*sh, generator=gen, dtype=torch.float64),
                                    torch.randn(*sh, generator=gen, dtype=torch.float64)).to(cdt).to(DEV)
    eta, g = mk(nrv, Nt, L, L), mk(nrv, Nt, L, L)
    ep = torch.exp(1j * torch.rand(Nt, L, L, generator=gen, dtype=torch.float64) * 6.2832).to(cdt).to(DEV)
    pairs = torch.combinations(torch.arange(nrv), r=2).to(torch.int32)
    pairs = torch.cat([pairs, torch.tensor([[0, nrv]], dtype=torch.int32)]).to(DEV)  # last: not a noise vector
    n = len(pairs)
    fa = torch.full((n, Nt, L, L), 7.0, dtype=cdt, device=DEV)
    fb = torch.full_like(fa, 7.0)
    ops.bb_pair_fields(kind, eta.reshape(nrv, -1), g.reshape(nrv, -1), ep, pairs[:, 0].contiguous(),
                       pairs[:, 1].contiguous(), L, fa, fb)
    wa, wb = _fields_torch(kind, eta, g, ep, pairs[:-1, 0].long(), pairs[:-1, 1].long())
    assert rel(fa[:-1].cpu(), wa.cpu()) < tol and rel(fb[:-1].cpu(), wb.cpu()) < tol
    assert torch.count_nonzero(fa[-1]) == 0 and torch.count_nonzero(fb[-1]) == 0
    A, B = torch.fft.ifft2(fa, norm="forward"), torch.fft.fft2(fb, norm="backward")
    S = torch.zeros(L * L, dtype=torch.complex128, device=DEV)
    ops.bb_kspace_acc(A, B, S)
    ops.bb_kspace_acc(A, B, S)  # accumulates
    want = 2 * (A.to(torch.complex128) * B.to(torch.complex128)).sum(dim=(0, 1)).reshape(-1)
    assert rel(S.cpu(), want.cpu()) < 1e-12


@pytest.mark.parametrize("cdt,tol", [(torch.complex128, 1e-12), (torch.complex64, 1e-5)])
def test_t2_is_t21_reflected(cdt, tol):
    """T2 from T21 at -d (its pair fields are T21's exchanged) against T2 from its own pair
    fields, on random noise vectors at L=8, Ltau=10."""
    from qed_fermion_b200.observables import BondBond
    L, Nt, nrv = 8, 10, 6
    gen = torch.Generator(device="cpu").manual_seed(11)
    mk = lambda *sh: torch.complex(torch.randn(*sh, generator=gen, dtype=torch.float64),
                                    torch.randn(*sh, generator=gen, dtype=torch.float64)).to(cdt).to(DEV)
    eta, g = mk(nrv, Nt * L * L), mk(nrv, Nt * L * L)
    bos = (torch.rand(1, 2, L, L, Nt, generator=gen, dtype=torch.float64) * 6.2832).to(DEV)
    bb = BondBond(L, Nt)
    want = bb.T2_direct(eta, g, bos)
    assert rel(bb.T2(eta, g, bos).cpu(), want.cpu()) < tol


@pytest.mark.parametrize("L,Lt,nrv,cdt,tol", [(12, 20, 6, torch.complex128, 1e-12), (18, 8, 5, torch.complex128, 1e-12),
                                             (36, 6, 4, torch.complex64, 2e-5), (10, 12, 4, torch.complex128, 1e-12),
                                             (34, 4, 3, torch.complex128, 1e-12)])
def test_fused_pair_sums_match_two_pass(L, Lt, nrv, cdt, tol):
    """The one-pass correlator kernel (fields, transforms and k-space product in
    shared memory) against the two-pass path (pair fields, cuFFT, k-space sum);
    L = 34 = 2 x 17 does not split into factors <= 8 and takes the two-pass path."""
    from qed_fermion_b200.observables import BondBond
    g = torch.Generator(device=DEV).manual_seed(L + Lt)
    N = L * L * Lt
    eta = torch.randn((nrv, N), dtype=cdt, device=DEV, generator=g)
    G = torch.randn((nrv, N), dtype=cdt, device=DEV, generator=g)
    bos = torch.rand((1, 2, L, L, Lt), dtype=torch.float64, device=DEV, generator=g) * 6.28
    for name in ("T1", "T21", "T2_direct", "T4"):
        a = getattr(BondBond(L, Lt, fused=True), name)(eta, G, bos)
        b = getattr(BondBond(L, Lt, fused=False), name)(eta, G, bos)
        assert float((a - b).abs().max() / b.abs().max()) < tol, name
