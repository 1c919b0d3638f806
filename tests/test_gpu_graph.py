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
