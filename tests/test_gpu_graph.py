"""The solver and the operators inside a CUDA graph: the persistent PCG (one
cooperative launch plus its preparation kernel) and M^dag M are captured once
and replayed on new inputs written into the captured buffers."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from qed_fermion_b200 import build
    build.build()


def _inputs(L, Nt, bs, seed, dev):
    from qed_fermion_b200.hmc import ref_to_kernel
    rng = np.random.default_rng(seed)
    x = np.arange(L)[:, None]
    y = np.arange(L)[None, :]
    sg = 1 - 2 * ((x + y) % 2)
    boson = np.zeros((bs, 2, L, L, Nt))
    boson[:, 0] = (sg * np.pi / 4)[None, :, :, None]
    boson[:, 1] = (-sg * np.pi / 4)[None, :, :, None]
    boson += 0.1 * rng.standard_normal(boson.shape)
    phi = ref_to_kernel(torch.tensor(boson, device=dev)).reshape(-1)
    b = torch.tensor((rng.standard_normal(bs * Nt * L * L) + 1j * rng.standard_normal(bs * Nt * L * L)) / np.sqrt(2),
                     device=dev)
    return phi, b


@pytest.mark.parametrize("mode", ["mixed", "fp64"])
def test_pcg_solve_replays_in_cuda_graph(mode):
    from qed_fermion_b200.solver import PcgSolver, SolveResult, System
    dev = torch.device("cuda:0")
    L, Nt, bs = 6, 30, 2
    s = PcgSolver([System(L, Nt, bs)], mode=mode, rtol=1e-10, max_iter=5000, device=dev)
    phi0, b0 = _inputs(L, Nt, bs, 1, dev)
    phi1, b1 = _inputs(L, Nt, bs, 2, dev)
    phi = phi0.to(s.angle_dtype).clone()
    b = b0.to(s.vec_dtype).clone()
    out = SolveResult(torch.empty(s.vec_len, dtype=s.vec_dtype, device=dev),
                      torch.empty(s.nrhs, dtype=torch.int32, device=dev),
                      torch.empty(s.nrhs, dtype=torch.float64, device=dev),
                      torch.empty(s.nrhs, dtype=torch.int32, device=dev))
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        s.solve(phi, b, out=out)
    torch.cuda.current_stream().wait_stream(side)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        s.solve(phi, b, out=out)
    # replay on the second input, written into the captured buffers
    phi.copy_(phi1.to(s.angle_dtype))
    b.copy_(b1.to(s.vec_dtype))
    g.replay()
    torch.cuda.synchronize()
    ref = PcgSolver([System(L, Nt, bs)], mode=mode, rtol=1e-10, max_iter=5000, device=dev).solve(
        phi1.to(s.angle_dtype), b1.to(s.vec_dtype))
    assert out.status.tolist() == [0, 0] == ref.status.tolist()
    xa, xb = out.x.cpu().numpy(), ref.x.cpu().numpy()
    assert np.abs(xa - xb).max() / np.abs(xb).max() < 1e-8
    assert np.all(np.abs(out.iters.cpu().numpy() - ref.iters.cpu().numpy()) <= 1)


def test_operator_replays_in_cuda_graph():
    from qed_fermion_b200 import ops
    dev = torch.device("cuda:0")
    L, Nt, bs = 12, 24, 2
    phi0, x0 = _inputs(L, Nt, bs, 3, dev)
    phi1, x1 = _inputs(L, Nt, bs, 4, dev)
    phi, x = phi0.float().view(bs, -1).clone(), x0.to(torch.complex64).view(bs, -1).clone()
    out = torch.empty_like(x)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        ops.apply_operator("mhm", phi, x, L, 0.1, out=out)
    torch.cuda.current_stream().wait_stream(side)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        ops.apply_operator("mhm", phi, x, L, 0.1, out=out)
    phi.copy_(phi1.float().view(bs, -1))
    x.copy_(x1.to(torch.complex64).view(bs, -1))
    g.replay()
    torch.cuda.synchronize()
    want = ops.apply_operator("mhm", phi1.float().view(bs, -1), x1.to(torch.complex64).view(bs, -1), L, 0.1)
    assert torch.equal(out, want)


@pytest.mark.parametrize("precision,chrono", [("mixed", None), ("fp64", None), ("mixed_f16", "linear")])
def test_trajectory_graph_matches_eager(precision, chrono):
    """Metropolis updates with the trajectory replayed from a CUDA graph give
    the eager sampler's fields, Hamiltonians and decisions: same seed, so the
    same draws; the first proposal runs eagerly and captures, the later ones
    replay.  Tau-block proposals use their own (masked) graph."""
    from qed_fermion_b200 import _lib
    from qed_fermion_b200.hmc import HmcSampler
    dev = torch.device("cuda:0")
    kw = dict(Lx=6, Ltau=60, bs=2, delta_t=0.02, N_leapfrog=3, precision=precision, cg_rtol=1e-10,
              device=dev, seed=7, max_tau_block_idx=1, autotune=False, chrono_guess=chrono)
    runs = {}
    for graph in (False, True):
        h = HmcSampler(graph=graph, **kw)
        h.initialize_boson_pi_flux_randn_matfree()
        out = []
        for _ in range(3):
            n0 = _lib.LAUNCHES["count"]
            boson, accp, it, err, H0, H1 = h.metropolis_update()
            out.append((boson.clone(), accp.clone(), H0.clone(), H1.clone(), it.clone(), _lib.LAUNCHES["count"] - n0))
        mask = torch.zeros((1, 1, 1, 1, h.Ltau), device=dev, dtype=h.dtype)
        mask[..., :20] = 1.0
        for _ in range(2):
            boson, accp, it, err, H0, H1 = h.metropolis_update(tau_mask=mask)
            out.append((boson.clone(), accp.clone(), H0.clone(), H1.clone(), it.clone(), 0))
        torch.cuda.synchronize()
        runs[graph] = (out, [list(q) for q in h.threshold_queue], h)
    (e, qe, he), (g, qg, hg) = runs[False], runs[True]
    assert len(hg._graphs) == 2 and all(tg.graph is not None for tg in hg._graphs.values())
    for (b0, a0, h00, h10, i0, n0), (b1, a1, h01, h11, i1, n1) in zip(e, g):
        assert torch.equal(a0, a1)
        assert torch.allclose(h00, h01, rtol=1e-12, atol=0) and torch.allclose(h10, h11, rtol=1e-12, atol=0)
        assert torch.allclose(b0, b1, rtol=0, atol=1e-9 if precision == "fp64" else 1e-5)
        assert torch.all((i0 - i1).abs() <= 1)
    # the launch counter sees the replays' kernels
    assert [o[5] for o in g[:3]] == [o[5] for o in e[:3]]
    assert len(qe) == len(qg)
    for a, b in zip(qe, qg):
        assert a == pytest.approx(b, rel=1e-9, abs=1e-12)
