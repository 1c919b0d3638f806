"""qed_fermion_b200: the hybrid-QMC fermion hot path of qed_fermion on B200 (sm_100a).

Native code: ``libqedf.so`` (C ABI in ``include/qedf.h``), built in-tree by
``qed_fermion_b200.build.build()``.  Python modules:

* ``_C``         drop-in for the reference's ``qed_fermion._C`` extension
* ``ops``        tensor wrappers of the operators, force, boson kernels
* ``solver``     batched persistent PCG (multi-system, multi-RHS, mixed precision)
* ``force``      fermion action with its adjoint force as an autograd.Function
* ``hmc``        ``HmcSampler`` with the reference's method names
* ``estimator``  ``StochaticEstimator`` noise solves
"""
from __future__ import annotations

import sys

__version__ = "0.1.0"


def install_as_reference_C():
    """Register ``qed_fermion_b200._C`` as ``qed_fermion._C`` so that the
    reference's modules pick up these kernels when they import it."""
    from . import _C
    sys.modules["qed_fermion._C"] = _C
    pkg = sys.modules.get("qed_fermion")
    if pkg is not None:
        setattr(pkg, "_C", _C)
    return _C
