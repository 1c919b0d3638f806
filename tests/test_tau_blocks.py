"""tau-block Metropolis updates and the step-size adaptation of the sampler
(hmc_sampler_batch.py:158-163, 263-268, 699-724, 2886-2930)."""
import pytest
import torch

from qed_fermion_b200.hmc import HmcSampler


def test_block_layout():
    h = HmcSampler(Lx=4, Ltau=40, bs=2, device="cpu", max_tau_block_idx=4)
    assert (h.max_tau_block_idx, h.tau_block_size, h.threshold_queue[0].maxlen) == (4, 10, 20)
    # blocks only when Ltau >= 10 Lx
    h = HmcSampler(Lx=6, Ltau=40, bs=1, device="cpu", max_tau_block_idx=4)
    assert (h.max_tau_block_idx, h.tau_block_size) == (1, 40)


def test_adjust_delta_t():
    h = HmcSampler(Lx=4, Ltau=40, bs=3, device="cpu", delta_t=0.1, max_tau_block_idx=1)
    for v, q in zip((0.1, 0.9, 0.4), h.threshold_queue):
        q.extend([v] * q.maxlen)
    h.threshold_queue[2].pop()  # not full yet: untouched
    h.adjust_delta_t()
    assert torch.allclose(h.delta_t_tensor, torch.tensor([0.09, 0.11, 0.1], dtype=torch.float64))
    assert [len(q) for q in h.threshold_queue] == [0, 0, 4]
    h.threshold_queue[2].append(0.4)  # full, inside [0.25, 0.5]: kept
    h.adjust_delta_t()
    assert float(h.delta_t_tensor[2]) == pytest.approx(0.1) and len(h.threshold_queue[2]) == 5


@pytest.mark.gpu
@pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA device")
def test_tau_block_update_moves_only_its_block():
    from qed_fermion_b200 import build
    build.build()
    h = HmcSampler(Lx=4, Ltau=40, bs=2, precision="fp64", cg_rtol=1e-10, delta_t=0.05, N_leapfrog=3,
                   device="cuda", seed=4, max_tau_block_idx=2)
    h.initialize_boson_pi_flux_randn_matfree()
    b0 = h.boson.clone()
    mask = torch.zeros((1, 1, 1, 1, 40), device="cuda", dtype=torch.float64)
    mask[..., 20:] = 1
    x, H0, H1, it, err = h.leapfrog_proposer5(b0, mask)
    assert torch.equal(x[..., :20], b0[..., :20]) and not torch.equal(x[..., 20:], b0[..., 20:])
    h.metropolis_update()
    assert [len(q) for q in h.threshold_queue] == [2, 2] and h.tau_block_idx == 0
    assert all(0.0 <= v <= 1.0 for q in h.threshold_queue for v in q)


def test_threshold_queue_reads_pending_entries_in_order():
    """Proposals leave their clipped acceptance probabilities on the device;
    reading the queue appends them in order, and entries older than the
    queue's length (which the deque would drop anyway) are not kept pending."""
    h = HmcSampler(Lx=4, Ltau=40, bs=2, device="cpu", max_tau_block_idx=1)
    maxlen = h.threshold_queue[0].maxlen
    for k in range(maxlen + 3):
        h._thr_pending.append(torch.tensor([k / 100, 1 - k / 100], dtype=torch.float64))
        del h._thr_pending[:-maxlen]
    assert len(h._thr_pending) == maxlen
    q = h.threshold_queue
    assert list(q[0]) == pytest.approx([k / 100 for k in range(3, maxlen + 3)])
    assert list(q[1]) == pytest.approx([1 - k / 100 for k in range(3, maxlen + 3)])
    assert h._thr_pending == []


def test_sampler_option_validation():
    with pytest.raises(ValueError):
        HmcSampler(Lx=4, Ltau=40, bs=1, device="cpu", chrono_guess="quadratic")
    with pytest.raises(ValueError):
        HmcSampler(Lx=4, Ltau=40, bs=1, device="cpu", precision="bf16")
    h = HmcSampler(Lx=4, Ltau=40, bs=1, device="cpu", chrono_guess="linear", graph=True, precision="mixed_f16")
    assert h.chrono_guess == "linear" and h.use_graph and h.solver.mode == "mixed_f16"
    # the guesses along a trajectory: none for the first solve, then the last
    # solution or the linear extrapolation of the last two
    a, b = torch.tensor([1.0, 2.0]), torch.tensor([3.0, 5.0])
    assert h._chrono_guess([]) is None
    assert torch.equal(h._chrono_guess([a]), a)
    assert torch.equal(h._chrono_guess([a, b]), 2 * b - a)
    h.chrono_guess = "last"
    assert torch.equal(h._chrono_guess([a, b]), b)
