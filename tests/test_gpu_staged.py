"""The PCG's staged operator engine (input slices copied whole into shared
memory by bulk copies, one slice ahead) against the engine that loads them
directly: the same arithmetic on the same values, so the solutions agree bit
for bit; and the bf16 vector storage mode, which runs on the staged engine."""
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


def _case(L, Nt, nrhs, seed):
    rng = np.random.default_rng(seed)
    x = np.arange(L)[:, None]
    y = np.arange(L)[None, :]
    sg = 1 - 2 * ((x + y) % 2)
    boson = np.zeros((nrhs, 2, L, L, Nt))
    boson[:, 0] = (sg * np.pi / 4)[None, :, :, None]
    boson[:, 1] = (-sg * np.pi / 4)[None, :, :, None]
    boson += 0.1 * rng.standard_normal(boson.shape)
    b = (rng.standard_normal((nrhs, Nt * L * L)) + 1j * rng.standard_normal((nrhs, Nt * L * L))) / np.sqrt(2)
    return O.ref_to_kernel_layout(boson).reshape(-1), b.reshape(-1)


@pytest.mark.parametrize("mode", ["mixed", "fp32"])
@pytest.mark.parametrize("systems", [
    [(48, 24, 2)],               # the engine compiled for L = 48
    [(12, 40, 2)],               # run-time L, preconditioned
    [(20, 14, 3)],               # no preconditioner (Ltau < 26)
    [(12, 30, 1), (18, 36, 2)],  # two lattices in one launch
])
def test_pcg_staged_engine_is_bit_identical(mode, systems):
    from qed_fermion_b200 import _lib
    from qed_fermion_b200.solver import PcgSolver, System
    sysl = [System(L, Nt, k) for L, Nt, k in systems]
    phis, bs = zip(*[_case(L, Nt, k, seed=L + Nt + k) for L, Nt, k in systems])
    out = []
    for stage in (True, False):
        s = PcgSolver(sysl, mode=mode, rtol=1e-14, max_iter=60, device=DEV, stage=stage, timeout_ms=500.0)
        res = s.solve(torch.tensor(np.concatenate(phis), dtype=s.angle_dtype, device=DEV),
                      torch.tensor(np.concatenate(bs), dtype=s.vec_dtype, device=DEV))
        torch.cuda.synchronize()
        out.append((res.x.clone(), res.iters.clone(), res.relres.clone(), res.status.clone()))
    assert out[0][3].cpu().tolist() == out[1][3].cpu().tolist()
    assert set(out[0][3].cpu().tolist()) <= {0, _lib.QEDF_ERR_MAXITER}
    assert torch.equal(out[0][0], out[1][0])
    assert torch.equal(out[0][1], out[1][1])
    # the residual norms are double sums that blocks add atomically in a
    # run-dependent order, so they agree to rounding rather than bit for bit
    assert torch.allclose(out[0][2], out[1][2], rtol=1e-12, atol=0)


@pytest.mark.parametrize("mode", ["mixed_bf16", "mixed_f16"])
@pytest.mark.parametrize("stage", [False, True])
@pytest.mark.parametrize("L,Nt,nrhs,kind", [(12, 40, 2, "piflux"), (48, 48, 2, "piflux"), (20, 14, 1, "piflux")])
def test_pcg_bf16_storage_meets_rtol_on_true_residual(L, Nt, nrhs, kind, stage, mode):
    """p and z stored as bf16 pairs or scaled fp16 pairs, float arithmetic,
    double reliable updates, on either operator engine: the returned x meets
    rtol = 1e-10 on the true residual (the oracle's operator on the same
    angles) and agrees with the plain mixed solution."""
    from qed_fermion_b200.solver import PcgSolver, System
    phi, b = _case(L, Nt, nrhs, seed=L * Nt)
    s = PcgSolver([System(L, Nt, nrhs)], mode=mode, rtol=1e-10, max_iter=20000, device=DEV,
                  timeout_ms=500.0, stage=stage)
    res = s.solve(torch.tensor(phi, dtype=torch.float32, device=DEV), torch.tensor(b, device=DEV))
    assert res.status.cpu().tolist() == [0] * nrhs
    x = res.x.cpu().numpy().reshape(nrhs, -1)
    phi32 = phi.astype(np.float32).astype(np.float64).reshape(nrhs, Nt, -1)
    bb = b.reshape(nrhs, -1)
    r = bb - O.mhm_vec(phi32, x.reshape(nrhs, Nt, L * L), L, 0.1).reshape(nrhs, -1)
    true_rel = np.linalg.norm(r, axis=1) / np.linalg.norm(bb, axis=1)
    assert np.all(true_rel < 2e-10), true_rel
    # same system in plain mixed precision: same solution to the solver tolerance
    m = PcgSolver([System(L, Nt, nrhs)], mode="mixed", rtol=1e-10, max_iter=20000, device=DEV)
    xm = m.solve(torch.tensor(phi, dtype=torch.float32, device=DEV), torch.tensor(b, device=DEV)).x
    xm = xm.cpu().numpy().reshape(nrhs, -1)
    assert np.abs(x - xm).max() / np.abs(xm).max() < 1e-7


@pytest.mark.parametrize("mode", ["mixed_f16", "mixed_bf16"])
def test_pcg_narrow_storage_ill_conditioned(mode):
    """Uniform random angles (the ill-conditioned case, thousands of
    iterations): the search direction grows far above the residual.  The
    narrow storages then lose z's contribution to p in rounding and may stall,
    which the solve reports as QEDF_ERR_MAXITER; the fp16 storage's scale
    follows p's growth, so nothing overflows into a NaN.  Float storage
    converges on the same system."""
    from qed_fermion_b200.solver import PcgSolver, System
    L, Nt, nrhs = 12, 120, 2
    rng = np.random.default_rng(17)
    boson = rng.uniform(-np.pi, np.pi, size=(nrhs, 2, L, L, Nt))
    phi = O.ref_to_kernel_layout(boson).reshape(-1)
    b = ((rng.standard_normal((nrhs, Nt * L * L)) + 1j * rng.standard_normal((nrhs, Nt * L * L))) / np.sqrt(2))
    res = {}
    for m in (mode, "mixed"):
        s = PcgSolver([System(L, Nt, nrhs)], mode=m, rtol=1e-8, max_iter=20000, device=DEV)
        r = s.solve(torch.tensor(phi, dtype=torch.float32, device=DEV), torch.tensor(b.reshape(-1), device=DEV))
        res[m] = (r.status.cpu().tolist(), r.x.cpu().numpy(), r.relres.cpu().numpy(), r.iters.cpu().numpy())
    st, x, rel, its = res[mode]
    assert all(v in (0, 4) for v in st), st  # converged or out of iterations, never NaN
    assert np.all(np.isfinite(x)) and np.all(np.isfinite(rel))
    stm, _, _, itm = res["mixed"]
    assert stm == [0] * nrhs and itm.min() > 1000
