"""Boson checkpoints in the reference's format (hmc_sampler_batch.py:971-1016,
3164-3181, 3211-3215): torch.save of {'boson': [bs, 2, Lx, Ly, Ltau] on the CPU,
'delta_t_tensor': [bs]} as <folder>/<name>.pt; a bare boson tensor is read too."""
import pytest
import torch

from qed_fermion_b200.hmc import HmcSampler


def _sampler(seed=3, **kw):
    return HmcSampler(Lx=4, Ltau=10, bs=2, device="cpu", seed=seed, **kw)


def test_save_load_round_trip(tmp_path):
    h = _sampler()
    h.initialize_boson_pi_flux_randn_matfree()
    h.delta_t_tensor = torch.tensor([0.05, 0.07], dtype=torch.float64)
    path = h.save_boson_checkpoint(str(tmp_path / "boson_ensemble"), "boson_spec_4000")
    assert path.endswith("boson_spec_4000.pt")
    d = torch.load(path)
    assert set(d) == {"boson", "delta_t_tensor"}
    assert d["boson"].shape == (2, 2, 4, 4, 10) and d["boson"].device.type == "cpu"
    assert d["delta_t_tensor"].dtype == torch.float32  # the reference's field dtype
    g = _sampler(seed=9)
    g.load_boson_checkpoint(path)
    assert torch.equal(g.boson, h.boson)
    assert torch.allclose(g.delta_t_tensor, torch.tensor([0.05, 0.07], dtype=torch.float64))


def test_reads_reference_written_files(tmp_path):
    """A dict written the way the reference writes it, and a bare tensor."""
    b = torch.randn(2, 2, 4, 4, 10)
    torch.save({"boson": b, "delta_t_tensor": torch.full((2,), 0.03)}, tmp_path / "a.pt")
    torch.save(b * 2, tmp_path / "b.pt")
    h = _sampler()
    h.load_boson_checkpoint(str(tmp_path / "a.pt"))
    assert torch.equal(h.boson, b) and float(h.delta_t_tensor[0]) == pytest.approx(0.03)
    h.load_boson_checkpoint(str(tmp_path / "b.pt"))
    assert torch.equal(h.boson, b * 2)
    with pytest.raises(RuntimeError):
        HmcSampler(Lx=6, Ltau=10, bs=2, device="cpu").load_boson_checkpoint(str(tmp_path / "a.pt"))


def test_initialize_from_ensemble(tmp_path):
    folder = tmp_path / "check_points" / "boson_ensemble"
    h = _sampler()
    members = {}
    for step in (4000, 5500):
        h.initialize_boson_pi_flux_randn_matfree()
        h.boson = h.boson + step * 1e-4
        h.save_boson_checkpoint(str(folder), f"boson_spec_{step}")
        members[step] = h.boson.clone()
    g = _sampler(seed=11)
    g.initialize_boson_ensemble(str(folder), "spec")
    assert any(torch.equal(g.boson, m) for m in members.values())
    # no files: the pi-flux start
    e = _sampler(seed=11)
    e.initialize_boson_ensemble(str(tmp_path / "empty"), "spec")
    ref = _sampler(seed=11)
    assert torch.equal(e.boson, ref.initialize_boson_pi_flux_randn_matfree())


def test_rejects_other_chain_counts(tmp_path):
    """A field saved with another number of chains, or step sizes that do not
    match its chains, is refused rather than broadcast."""
    torch.save({"boson": torch.randn(3, 2, 4, 4, 10), "delta_t_tensor": torch.full((3,), 0.03)},
               tmp_path / "three.pt")
    torch.save({"boson": torch.randn(2, 2, 4, 4, 10), "delta_t_tensor": torch.full((3,), 0.03)},
               tmp_path / "bad_dt.pt")
    h = _sampler()
    with pytest.raises(RuntimeError, match="chains"):
        h.load_boson_checkpoint(str(tmp_path / "three.pt"))
    with pytest.raises(RuntimeError, match="step sizes"):
        h.load_boson_checkpoint(str(tmp_path / "bad_dt.pt"))
    assert h.boson is None
