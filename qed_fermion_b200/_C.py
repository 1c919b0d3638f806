"""Drop-in for the reference's native extension ``qed_fermion._C``.

The reference imports ``from qed_fermion import _C`` when CUDA is available
(``hmc_sampler_batch.py:98-99``, ``stochastic_estimator.py:17-18``) and calls
the five functions below.  Registering this module under that name
(``qed_fermion_b200.install_as_reference_C()``) runs the reference's
``HmcSampler`` / ``StochaticEstimator`` unchanged on the sm_100a kernels.

Semantics, reconstructed from the call sites:

* ``mhm_vec(boson, x, Lx, dtau, bx, by)`` -> ``M^dag M x`` per batch row
  (``hmc_sampler_batch.py:772, 799``);
* ``mh_vec(boson, v, Lx, dtau, bx, by)`` -> ``M^dag v``
  (``hmc_sampler_batch.py:2406``, ``stochastic_estimator.py:430``);
* ``precon_vec(r, precon_csr, Lx)`` -> ``P r`` (``hmc_sampler_batch.py:773, 838``);
* ``b_vec_per_tau(boson_tau, v, Lx, dtau, interm, bx, by)`` -> ``B_t v`` or the
  six partial products (``hmc_sampler_batch.py:2174-2189``), reading the raw
  storage of ``v`` (a lazy ``.conj()`` on the argument is not applied).

``bx, by`` (the reference's ``BLOCK_SIZE = (4, 8)``) are launch hints of the
original kernels; this implementation chooses its own tiles and ignores them.
The float32 angles / complex64 vectors of the reference and float64 /
complex128 (the plain FP64 path) are both accepted.  Errors (wrong dtype,
shape, odd Lx, a non-CUDA tensor) raise ``RuntimeError``.
"""
from __future__ import annotations

import torch

from . import ops, precon

_tau_cache: dict = {}


def mhm_vec(boson, x, Lx, dtau, bx=4, by=8):
    return ops.apply_operator("mhm", boson.reshape(boson.shape[0], -1), x, int(Lx), float(dtau))


def mh_vec(boson, v, Lx, dtau, bx=4, by=8):
    return ops.apply_operator("mh", boson.reshape(boson.shape[0], -1), v, int(Lx), float(dtau))


def m_vec(boson, v, Lx, dtau, bx=4, by=8):
    """M v (no call site in the reference; provided for completeness)."""
    return ops.apply_operator("m", boson.reshape(boson.shape[0], -1), v, int(Lx), float(dtau))


def b_vec_per_tau(boson_tau, v, Lx, dtau, interm, bx=4, by=8):
    return ops.b_vec_per_tau(boson_tau.reshape(-1), v, int(Lx), float(dtau), bool(interm))


def _tau_part(precon_csr, Lx):
    key = (id(precon_csr), precon_csr.values().data_ptr(), int(precon_csr.values().numel()), int(Lx))
    hit = _tau_cache.get(key)
    if hit is None:
        hit = precon.to_device(precon.tau_csr_from_full(precon_csr, int(Lx)), precon_csr.device)
        _tau_cache[key] = hit
    return hit


def precon_vec(r, precon_csr, Lx):
    if precon_csr is None or not precon_csr.is_sparse_csr:
        raise RuntimeError("precon_vec: expected a torch sparse CSR preconditioner")
    return ops.precon_apply(r, _tau_part(precon_csr, Lx), int(Lx))


def prec_vec(r, precon_csr, Lx):
    """Older name of ``precon_vec`` that appears in the reference's comments."""
    return precon_vec(r, precon_csr, Lx)
