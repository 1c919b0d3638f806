"""Momentum and pseudofermion draws and the Metropolis accept decision
(hmc_sampler_batch.py:1247-1252, 1279-1287, 2886-2930).

The draws keep the reference's normalisations: p ~ N(0, m) per component,
and R = complex randn / sqrt(2), whose E|R|^2 is 1/2 (torch's complex normal
already has E|z|^2 = 1).  The accept test is u < exp(H_old - H_new) in
double with u drawn from the sampler's generator; the threshold queues
record min(exp(H_old - H_new), 1)."""
import math

import numpy as np
import pytest
import torch

from oracle import qedf_oracle as O
from qed_fermion_b200.hmc import HmcSampler, metropolis_accept


def _devices():
    devs = ["cpu"]
    if torch.cuda.is_available():
        devs.append(pytest.param("cuda", marks=pytest.mark.gpu))
    return devs


@pytest.mark.parametrize("device", _devices())
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_draw_normalisations(device, precision):
    h = HmcSampler(Lx=8, Ltau=80, bs=4, m=2.5, precision=precision, device=device, seed=17)
    p = torch.cat([h.draw_momentum().double().reshape(-1) for _ in range(8)])   # 163,840 samples
    R = torch.cat([h.draw_psudo_fermion().reshape(-1) for _ in range(8)])      # 81,920 samples
    n_p, n_r = p.numel(), R.numel()
    assert abs(float(p.mean())) < 5 * math.sqrt(2.5 / n_p)
    # Var p = m; the sample variance of a normal has standard error m sqrt(2/n)
    assert abs(float(p.var()) - 2.5) < 5 * 2.5 * math.sqrt(2.0 / n_p)
    # |R|^2 = (a^2 + b^2) / 2 with a, b ~ N(0, 1/2): mean 1/2, standard deviation 1/2
    r2 = R.abs().double() ** 2
    assert abs(float(r2.mean()) - 0.5) < 5 * 0.5 / math.sqrt(n_r)
    assert abs(float(R.real.double().var()) - 0.25) < 5 * 0.25 * math.sqrt(2.0 / n_r)
    assert R.dtype == (torch.complex128 if precision in ("fp64", "mixed") else torch.complex64)
    assert p.shape[0] == 8 * 4 * 2 * 8 * 8 * 80


def test_accept_rule_matches_oracle_and_edges():
    H_old = torch.tensor([10.0, 10.0, 10.0, 10.0, 10.0, 10.0], dtype=torch.float64)
    H_new = torch.tensor([9.0, 10.5, 10.5, 1e4, float("nan"), 10.0 + 1e-300], dtype=torch.float64)
    u = torch.tensor([0.999999, 0.6, 0.61, 0.0, 0.0, 0.5], dtype=torch.float64)
    acc, thr = metropolis_accept(H_old, H_new, u)
    want = O.metropolis_accept(H_old.numpy(), H_new.numpy(), u.numpy())
    assert acc.tolist() == want.tolist() == [True, True, False, False, False, True]
    assert thr.tolist() == pytest.approx([1.0, math.exp(-0.5), math.exp(-0.5), 0.0, 0.0, 1.0])


def test_metropolis_update_with_fixed_u(monkeypatch):
    """The sampler's own update with the leapfrog replaced by fixed proposals:
    the u it draws (the next draws of its generator) decides each chain as the
    reference's rule says, accepted chains take the proposal, rejected ones
    keep their field, and every test feeds the threshold queue."""
    bs = 4
    h = HmcSampler(Lx=4, Ltau=10, bs=bs, device="cpu", seed=123)
    h.initialize_boson_pi_flux_randn_matfree()
    b0 = h.boson.clone()
    prop = b0 + 1.0
    H_old = torch.tensor([5.0, 5.0, 5.0, 5.0], dtype=torch.float64)
    H_new = torch.tensor([4.0, 5.7, 5.05, 40.0], dtype=torch.float64)
    monkeypatch.setattr(h, "leapfrog_proposer5",
                        lambda boson, tau_mask=None: (prop, H_old, H_new, torch.zeros(bs), torch.zeros(bs)))
    g = torch.Generator().manual_seed(0)
    g.set_state(h.generator.get_state())
    u = torch.rand(bs, dtype=torch.float64, generator=g)
    _, accp, _, _, _, _ = h.metropolis_update()
    want = u.numpy() < np.exp(H_old.numpy() - H_new.numpy())
    assert accp.tolist() == want.tolist()
    assert bool(accp[0]) and not bool(accp[3])
    for c in range(bs):
        assert torch.equal(h.boson[c], prop[c] if want[c] else b0[c])
    assert [q[-1] for q in h.threshold_queue] == pytest.approx(
        np.minimum(np.exp(H_old.numpy() - H_new.numpy()), 1.0).tolist())
