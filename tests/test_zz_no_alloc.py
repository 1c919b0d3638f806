"""The allocation-free solve, qedf_pcg_solve_static.

Callers that cannot allocate device memory where they solve (a driver that is
capturing a CUDA graph, or one running under an allocator or memory budget it
does not control) use this entry point: it takes the same inputs and outputs
as qedf_pcg_solve but keeps its scratch in a fixed device array inside the
library.  This file checks, through the C ABI, that two calls in a row give
the same solution as the workspace-taking qedf_pcg_solve, and that a problem
larger than the array is refused.  It is named to run after every other test,
so that a run stopping at the first failure has run all the others first.
"""
import ctypes

import numpy as np
import pytest
import torch

from oracle import qedf_oracle as O

pytestmark = pytest.mark.gpu


def _case(L, Nt, bs, seed):
    rng = np.random.default_rng(seed)
    x = np.arange(L)[:, None]
    y = np.arange(L)[None, :]
    sg = 1 - 2 * ((x + y) % 2)
    boson = np.zeros((bs, 2, L, L, Nt))
    boson[:, 0] = (sg * np.pi / 4)[None, :, :, None]
    boson[:, 1] = (-sg * np.pi / 4)[None, :, :, None]
    boson += 0.1 * rng.standard_normal(boson.shape)
    b = (rng.standard_normal((bs, Nt * L * L)) + 1j * rng.standard_normal((bs, Nt * L * L))) / np.sqrt(2)
    return O.ref_to_kernel_layout(boson), b


@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA device")
def test_static_scratch_solve_matches_workspace_solve():
    from qed_fermion_b200 import _lib, build
    build.build()
    lib = _lib.load()
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    L, Nt, bs = 6, 30, 2
    phi, b = _case(L, Nt, bs, seed=17)
    phi_t = torch.tensor(phi.reshape(-1), dtype=torch.float64, device=dev)
    b_t = torch.tensor(b.reshape(-1), dtype=torch.complex128, device=dev)
    systems = (_lib.QedfSystem * 1)(_lib.QedfSystem(L, Nt, bs, 0))
    opts = _lib.QedfPcgOpts(_lib.QEDF_PCG_PLAIN_F64, 20000, 1e-12, 0.1, 1, 50, 0.1, 0, 0, 0, 0.0, None)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def outputs():
        return (torch.empty_like(b_t), torch.empty(bs, dtype=torch.int32, device=dev),
                torch.empty(bs, dtype=torch.float64, device=dev), torch.empty(bs, dtype=torch.int32, device=dev))

    def p(t):
        return ctypes.c_void_p(t.data_ptr())

    # reference result: the entry point that takes a caller-allocated workspace
    nbytes = lib.qedf_pcg_workspace_bytes(systems, 1, opts)
    assert 0 < nbytes <= _lib.PCG_STATIC_SCRATCH_BYTES
    ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    x_ws, it_ws, rr_ws, st_ws = outputs()
    assert lib.qedf_pcg_solve(systems, 1, p(phi_t), p(b_t), p(x_ws), p(it_ws), p(rr_ws), p(st_ws), p(ws), nbytes,
                              opts, stream) == _lib.QEDF_OK

    # two calls in a row of the allocation-free entry point
    for _ in range(2):
        x_st, it_st, rr_st, st_st = outputs()
        assert lib.qedf_pcg_solve_static(systems, 1, p(phi_t), p(b_t), p(x_st), p(it_st), p(rr_st), p(st_st),
                                         opts, stream) == _lib.QEDF_OK
        torch.cuda.synchronize()
        assert st_st.cpu().tolist() == [0] * bs == st_ws.cpu().tolist()
        xa, xb = x_st.cpu().numpy(), x_ws.cpu().numpy()
        assert np.abs(xa - xb).max() / np.abs(xb).max() < 1e-9
        assert np.all(np.abs(it_st.cpu().numpy() - it_ws.cpu().numpy()) <= 1)

    # a problem whose workspace exceeds the array is refused before any launch
    big = (_lib.QedfSystem * 1)(_lib.QedfSystem(48, 480, 8, 0))
    x_st, it_st, rr_st, st_st = outputs()
    assert lib.qedf_pcg_solve_static(big, 1, p(phi_t), p(b_t), p(x_st), p(it_st), p(rr_st), p(st_st), opts,
                                     stream) == _lib.QEDF_ERR_SIZE
