"""The tau-banded preconditioner P = P_tau (x) I_Vs.

The coefficient table lives in the native library (``qedf_precon_tau_csr``),
restating the reference's hand-built preconditioner
(``preconditioners_orig/precon_manual.py:15-186``).  This module turns it into
tau-space CSR arrays, and reduces a full ``N x N`` CSR matrix as the
reference passes it to ``_C.precon_vec`` (``hmc_sampler_batch.py:547, 838``)
to its tau part after checking that it has the ``P_tau (x) I`` structure.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib

MIN_LTAU = 26


def builtin_tau_csr(Ltau: int):
    """Host numpy arrays ``(row_ptr, col, val)`` of the builtin P_tau."""
    lib = _lib.load()
    nnz = ctypes.c_int(0)
    row_ptr = (ctypes.c_int * (Ltau + 1))()
    st = lib.qedf_precon_tau_csr(Ltau, row_ptr, None, None, ctypes.byref(nnz))
    if st != _lib.QEDF_OK:
        raise ValueError(f"builtin preconditioner is defined for Ltau >= {MIN_LTAU}, got {Ltau}")
    col = (ctypes.c_int * nnz.value)()
    val = (ctypes.c_double * nnz.value)()
    lib.qedf_precon_tau_csr(Ltau, row_ptr, col, val, ctypes.byref(nnz))
    return (np.frombuffer(row_ptr, dtype=np.int32).copy(), np.frombuffer(col, dtype=np.int32).copy(),
            np.frombuffer(val, dtype=np.float64).copy())


def builtin_tau_dense(Ltau: int) -> np.ndarray:
    rp, col, val = builtin_tau_csr(Ltau)
    P = np.zeros((Ltau, Ltau))
    for t in range(Ltau):
        for k in range(rp[t], rp[t + 1]):
            P[t, col[k]] += val[k]
    return P


def to_device(tau_csr, device):
    rp, col, val = tau_csr
    return (torch.as_tensor(rp, dtype=torch.int32, device=device),
            torch.as_tensor(col, dtype=torch.int32, device=device),
            torch.as_tensor(val, dtype=torch.float64, device=device))


def tau_csr_from_full(precon_csr: torch.Tensor, Lx: int):
    """Reduce an ``N x N`` sparse CSR ``P`` to ``P_tau`` if ``P = P_tau (x) I_Vs``.

    Raises ``RuntimeError`` when the matrix does not have that structure.
    Returns host numpy ``(row_ptr, col, val)``.
    """
    crow = precon_csr.crow_indices().cpu().numpy().astype(np.int64)
    cols = precon_csr.col_indices().cpu().numpy().astype(np.int64)
    vals = precon_csr.values().cpu().numpy()
    N = precon_csr.shape[0]
    Vs = Lx * Lx
    if N % Vs or precon_csr.shape[1] != N:
        raise RuntimeError("precon_vec: preconditioner shape does not match the lattice")
    Ltau = N // Vs
    rows = np.repeat(np.arange(N), np.diff(crow))
    if np.any(np.abs(np.imag(vals)) > 0):
        raise RuntimeError("precon_vec: preconditioner must be real")
    if np.any(rows % Vs != cols % Vs):
        raise RuntimeError("precon_vec: preconditioner is not of the form P_tau (x) I")
    tr, tc = rows // Vs, cols // Vs
    P = np.zeros((Ltau, Ltau))
    np.add.at(P, (tr[rows % Vs == 0], tc[rows % Vs == 0]), np.real(vals[rows % Vs == 0]))
    if not np.array_equal(P[tr, tc], np.real(vals)) or len(vals) != Vs * np.count_nonzero(P):
        raise RuntimeError("precon_vec: preconditioner is not of the form P_tau (x) I")
    rp = np.zeros(Ltau + 1, dtype=np.int32)
    col_l, val_l = [], []
    for t in range(Ltau):
        nz = np.nonzero(P[t])[0]
        col_l.append(nz)
        val_l.append(P[t, nz])
        rp[t + 1] = rp[t] + len(nz)
    return rp, np.concatenate(col_l).astype(np.int32), np.concatenate(val_l).astype(np.float64)
