"""Adaptive Fourier mass (hmc_sampler_batch.py:272-285, 1133-1277) against the
reference's own values (fixture golden_fourier_mass.npz): the oracle's
restatement on the CPU, and the library's kernels on the GPU."""
import os

import numpy as np
import pytest
import torch

from oracle import qedf_oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))


def _fixture():
    return dict(np.load(os.path.join(HERE, "golden", "golden_fourier_mass.npz")))


def _noise(shape):
    """The two normal draws the fixture's draw_momentum_fft took (torch generator 77, float32)."""
    g = torch.Generator().manual_seed(77)
    a = torch.randn(shape, dtype=torch.float32, generator=g)
    b = torch.randn(shape, dtype=torch.float32, generator=g)
    return a, b


@pytest.mark.parametrize("mode", [1, -1])
def test_oracle_fourier_mass_matches_reference(mode):
    """12 steps with a window of 5 restarting every 4 steps, the mass at step 10."""
    G = _fixture()
    fields = G["fm_fields"]
    mean = np.zeros_like(fields[0])
    spec = np.ones(fields[0].shape[:-1] + (fields[0].shape[-1] // 2 + 1,))
    start, restarts = 0, 10
    for i in range(12):
        if i % 4 == 0 and i > 0 and restarts > 0:
            start, restarts = i, restarts - 1
        mean, spec = O.fm_accumulate(mean, spec, fields[i], i - start)
    np.testing.assert_allclose(spec, G[f"fm{mode}_sigma_hat_cpu"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(mean, G[f"fm{mode}_boson_mean_cpu"], rtol=1e-12, atol=1e-14)
    sigma = O.fm_mass(spec, invert=(mode == -1))
    np.testing.assert_allclose(sigma, G[f"fm{mode}_sigma_hat"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(O.fm_m_inv(G["fm_p"], sigma), G[f"fm{mode}_m_inv_p"], rtol=1e-12, atol=1e-14)
    a, b = _noise(sigma.shape)
    np.testing.assert_allclose(O.fm_draw(sigma, a.double().numpy(), b.double().numpy(), fields[0].shape[-3:]),
                               G[f"fm{mode}_p_fft"], rtol=1e-12, atol=1e-14)


@pytest.mark.gpu
@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA device")
@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-12), (torch.float32, 1e-4)])
@pytest.mark.parametrize("mode", [1, -1])
def test_fourier_mass_kernels_match_reference(mode, dtype, tol):
    from qed_fermion_b200 import build
    from qed_fermion_b200.fourier_mass import FourierMass
    build.build()
    G = _fixture()
    dev = torch.device("cuda")
    fm = FourierMass(1, 4, 10, dtype=dtype, device=dev, sigma_mini_batch_size=5, mass_mode=mode)
    fm.annealing_step = 4
    for i in range(12):
        fm.update_sigma_hat_cpu(torch.tensor(G["fm_fields"][i]), i)
    scale = lambda a: np.abs(a).max()
    for got, key in ((fm.sigma_hat_cpu, "sigma_hat_cpu"), (fm.boson_mean_cpu, "boson_mean_cpu")):
        want = G[f"fm{mode}_{key}"]
        assert np.abs(got.double().numpy() - want).max() <= tol * scale(want)
    fm.apply_sigma_hat_cpu(7)  # not a window boundary: unchanged
    assert torch.equal(fm.sigma_hat, torch.ones_like(fm.sigma_hat))
    fm.apply_sigma_hat_cpu(10)
    want = G[f"fm{mode}_sigma_hat"]
    assert np.abs(fm.sigma_hat.double().cpu().numpy() - want).max() <= tol * scale(want)
    got = fm.apply_m_inv(torch.tensor(G["fm_p"])).double().cpu().numpy()
    want = G[f"fm{mode}_m_inv_p"]
    assert np.abs(got - want).max() <= 10 * tol * scale(want)
    got = fm.draw_momentum_fft(noise=_noise(fm.sigma_hat.shape)).double().cpu().numpy()
    want = G[f"fm{mode}_p_fft"]
    assert np.abs(got - want).max() <= 10 * tol * scale(want)
