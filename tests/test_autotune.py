"""The autotuner's candidate sets (CPU) and, on the GPU, that every candidate it
may pick solves to the stated tolerance against the oracle, and that its
choice is cached in memory and on disk."""
import json
import os

import numpy as np
import pytest
import torch

from oracle import qedf_oracle as O
from qed_fermion_b200 import autotune
from qed_fermion_b200.solver import System


def test_tile_heights_follow_the_library_rule():
    assert autotune.tile_heights([48]) == [2, 4, 6]
    assert autotune.tile_heights([36]) == [2, 4, 6]
    assert autotune.tile_heights([66]) == [6]          # 33 x 33 tiles of 2 x 2 exceed 576 threads
    assert autotune.tile_heights([12, 18, 24, 30]) == [2, 6]
    assert autotune.tile_heights([10]) == [2]


def test_slab_candidates():
    # two chains x 480 slices over 148 blocks: 1, 2 and 3 rounds of units
    assert autotune.slab_candidates([System(48, 480, 2)]) == [0, 7, 4, 3]
    assert autotune.slab_candidates([System(36, 360, 64, True)]) == [0, 156, 78, 52]
    assert autotune.slab_candidates([System(4, 10, 1)]) == [0, 1]


def _solve_case(L, Nt, nrhs, seed):
    rng = np.random.default_rng(seed)
    x = np.arange(L)[:, None]
    y = np.arange(L)[None, :]
    sg = 1 - 2 * ((x + y) % 2)
    boson = np.zeros((nrhs, 2, L, L, Nt))
    boson[:, 0] = (sg * np.pi / 4)[None, :, :, None]
    boson[:, 1] = (-sg * np.pi / 4)[None, :, :, None]
    boson += 0.1 * rng.standard_normal(boson.shape)
    b = (rng.standard_normal((nrhs, Nt * L * L)) + 1j * rng.standard_normal((nrhs, Nt * L * L))) / np.sqrt(2)
    return O.ref_to_kernel_layout(boson), b


@pytest.mark.gpu
@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA device")
@pytest.mark.parametrize("mode", ["mixed", "fp64", "mixed_bf16", "mixed_f16"])
def test_every_pcg_candidate_meets_rtol(mode, tmp_path, monkeypatch):
    from qed_fermion_b200 import build
    from qed_fermion_b200.solver import PcgSolver
    build.build()
    monkeypatch.setenv("QEDF_TUNE_CACHE", str(tmp_path / "tune.json"))
    L, Nt, nrhs = 12, 40, 2
    systems = [System(L, Nt, nrhs)]
    choice = autotune.pcg_choice(systems, mode, force=True)
    assert len(choice["candidates"]) >= 2
    assert autotune.pcg_choice(systems, mode) is choice            # in memory
    disk = json.load(open(tmp_path / "tune.json"))
    assert any(v["by"] == choice["by"] and v["slab"] == choice["slab"] for v in disk.values())
    phi, b = _solve_case(L, Nt, nrhs, seed=5)
    dev = torch.device("cuda")
    for c in choice["candidates"]:
        s = PcgSolver(systems, mode=mode, rtol=1e-10, max_iter=20000, by=c["by"], slab=c["slab"],
                      stage=c["stage"], chunk=c["chunk"], device=dev)
        res = s.solve(torch.tensor(phi.reshape(-1), dtype=s.angle_dtype, device=dev),
                      torch.tensor(b.reshape(-1), dtype=s.vec_dtype, device=dev))
        assert res.status.cpu().tolist() == [0] * nrhs, c
        x = res.x.cpu().numpy().reshape(nrhs, Nt, L * L)
        ph = phi.astype(np.float32).astype(np.float64) if s.angle_dtype == torch.float32 else phi
        r = b - O.mhm_vec(ph, x, L, 0.1).reshape(nrhs, -1)
        assert np.all(np.linalg.norm(r, axis=1) / np.linalg.norm(b, axis=1) < 2e-10), c
    # a tuned solver uses the choice
    t = PcgSolver(systems, mode=mode, rtol=1e-10, device=dev, tune=True)
    assert t.tuned is choice


@pytest.mark.gpu
@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA device")
def test_every_operator_candidate_matches_oracle(tmp_path, monkeypatch):
    from qed_fermion_b200 import build, ops
    build.build()
    monkeypatch.setenv("QEDF_TUNE_CACHE", str(tmp_path / "tune.json"))
    L, Nt, nv = 24, 16, 2
    choice = autotune.operator_choice(L, Nt, nv, torch.complex64, force=True)
    phi, v = _solve_case(L, Nt, nv, seed=9)
    want = O.mhm_vec(phi, v.reshape(nv, Nt, L * L), L, 0.1).reshape(nv, -1)
    dev = torch.device("cuda")
    for c in choice["candidates"]:
        got = ops.apply_operator("mhm", torch.tensor(phi.reshape(nv, -1), dtype=torch.float32, device=dev),
                                 torch.tensor(v, dtype=torch.complex64, device=dev), L, 0.1, by=c["by"],
                                 slab=c["slab"]).cpu().numpy()
        assert np.abs(got - want).max() / np.abs(want).max() < 1e-6, c
