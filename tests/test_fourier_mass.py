"""Adaptive Fourier mass against the reference's own values
(hmc_sampler_batch.py:272-285, 1133-1277; fixture golden_fourier_mass.npz)."""
import os

import numpy as np
import pytest
import torch

from qed_fermion_b200.fourier_mass import FourierMass

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("mode", [1, -1])
def test_fourier_mass_matches_reference(mode):
    G = dict(np.load(os.path.join(HERE, "golden", "golden_fourier_mass.npz")))
    fm = FourierMass(1, 4, 10, dtype=torch.float64, device="cpu", sigma_mini_batch_size=5, mass_mode=mode)
    fm.annealing_step = 4
    for i in range(12):
        fm.update_sigma_hat_cpu(torch.tensor(G["fm_fields"][i]), i)
    np.testing.assert_allclose(fm.sigma_hat_cpu.numpy(), G[f"fm{mode}_sigma_hat_cpu"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(fm.boson_mean_cpu.numpy(), G[f"fm{mode}_boson_mean_cpu"], rtol=1e-12, atol=1e-14)
    fm.apply_sigma_hat_cpu(7)  # not a window boundary: unchanged
    assert torch.equal(fm.sigma_hat, torch.ones_like(fm.sigma_hat))
    fm.apply_sigma_hat_cpu(10)
    np.testing.assert_allclose(fm.sigma_hat.numpy(), G[f"fm{mode}_sigma_hat"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(fm.apply_m_inv(torch.tensor(G["fm_p"])).numpy(), G[f"fm{mode}_m_inv_p"],
                               rtol=1e-12, atol=1e-14)
    g = torch.Generator().manual_seed(77)
    np.testing.assert_allclose(fm.draw_momentum_fft(g).numpy(), G[f"fm{mode}_p_fft"], rtol=1e-12, atol=1e-14)
