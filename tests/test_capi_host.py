"""CPU-only checks of the C-ABI library: it loads without a GPU, exports every
symbol ``include/qedf.h`` declares, rejects bad arguments on the host, and its
builtin preconditioner table equals the oracle's restatement of the
reference's table.  No compute entry point is launched here."""
import ctypes
import os
import re

import numpy as np
import pytest
import torch

from oracle import qedf_oracle as O
from qed_fermion_b200 import _lib, precon

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "qedf.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(qedf_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    syms = header_symbols()
    assert len(syms) >= 25
    for s in syms:
        assert hasattr(lib, s), s
    # and the ctypes signature table covers the same set
    assert set(syms) == set(_lib.SIGNATURES), set(syms) ^ set(_lib.SIGNATURES)


def test_version_and_status_strings():
    lib = _lib.load()
    assert b"sm_100a" in lib.qedf_version()
    assert _lib.status_string(_lib.QEDF_ERR_TIMEOUT) == "device-side wait timed out"


def test_host_validation_rejects_before_launch():
    lib = _lib.load()
    # null pointers, odd L, bad rhs grouping: rejected on the host
    assert lib.qedf_mhm_vec_c64(None, None, None, 1, 4, 10, 0.1, 1, 0, 0, None) == _lib.QEDF_ERR_ARG
    buf = ctypes.create_string_buffer(64 + 16)
    p = ctypes.c_void_p((ctypes.addressof(buf) + 15) // 16 * 16)
    q = ctypes.c_void_p(p.value + 32)
    assert lib.qedf_mhm_vec_c64(p, p, q, 1, 5, 10, 0.1, 1, 0, 0, None) == _lib.QEDF_ERR_ARG
    assert lib.qedf_mhm_vec_c64(p, p, q, 3, 4, 10, 0.1, 2, 0, 0, None) == _lib.QEDF_ERR_ARG
    assert lib.qedf_mhm_vec_c64(p, p, p, 1, 4, 10, 0.1, 1, 0, 0, None) == _lib.QEDF_ERR_ARG  # in place
    assert lib.qedf_mh_vec_c128(p, p, q, 1, 4, 10, 0.1, 1, 3, 0, None) == _lib.QEDF_ERR_ARG  # by=3
    # no tile of an L = 80 slice fits one thread block: size error
    assert lib.qedf_mhm_vec_c64(p, p, q, 1, 80, 10, 0.1, 1, 0, 0, None) == _lib.QEDF_ERR_SIZE
    # L = 66 needs 2 x 6 tiles; asking for 2 x 2 is an argument error
    assert lib.qedf_mhm_vec_c64(p, p, q, 1, 66, 10, 0.1, 1, 2, 0, None) == _lib.QEDF_ERR_ARG
    # correlator passes: unknown kind, null pointers, too many pairs or slices, one noise
    # vector, negative row count
    bb = lib.qedf_bb_pair_fields_c64
    assert bb(3, p, p, p, p, p, 1, 4, 4, 10, p, q, None) == _lib.QEDF_ERR_ARG
    assert bb(1, None, p, p, p, p, 1, 4, 4, 10, p, q, None) == _lib.QEDF_ERR_ARG
    assert bb(21, p, p, p, p, p, 70000, 4, 4, 10, p, q, None) == _lib.QEDF_ERR_ARG
    assert lib.qedf_bb_pair_fields_c128(2, p, p, p, p, p, 1, 4, 4, 70000, p, q, None) == _lib.QEDF_ERR_ARG
    assert bb(4, p, p, p, p, p, 1, 1, 4, 10, p, q, None) == _lib.QEDF_ERR_ARG
    assert bb(1, p, p, p, p, p, 0, 4, 4, 10, p, q, None) == _lib.QEDF_OK  # nothing to do
    assert lib.qedf_bb_kspace_acc_c64(p, p, -1, 16, p, None) == _lib.QEDF_ERR_ARG
    assert lib.qedf_bb_kspace_acc_c128(p, None, 4, 16, p, None) == _lib.QEDF_ERR_ARG
    assert lib.qedf_bb_kspace_acc_c128(p, p, 0, 16, p, None) == _lib.QEDF_OK  # nothing to do


def test_pcg_workspace_query():
    sys_ = (_lib.QedfSystem * 2)(_lib.QedfSystem(12, 120, 4, 0), _lib.QedfSystem(18, 180, 4, 1))
    opts = _lib.QedfPcgOpts(_lib.QEDF_PCG_MIXED, 100, 1e-10, 0.1, 1, 50, 0.1, 0, 0, 0, 0.0, None)
    nb = _lib.load().qedf_pcg_workspace_bytes(sys_, 2, opts)
    nvec = 4 * 12 * 12 * 120 + 4 * 18 * 18 * 180
    assert nb >= 6 * nvec * 8
    bad = _lib.QedfPcgOpts(7, 100, 1e-10, 0.1, 1, 50, 0.1, 0, 0, 0, 0.0, None)
    assert _lib.load().qedf_pcg_workspace_bytes(sys_, 2, bad) < 0


@pytest.mark.parametrize("Nt", [26, 27, 30, 60, 480])
def test_builtin_precon_table_matches_oracle(Nt):
    P = precon.builtin_tau_dense(Nt)
    np.testing.assert_array_equal(P, O.precon_tau_matrix(Nt))


def test_builtin_precon_rejects_short_ltau():
    with pytest.raises(ValueError):
        precon.builtin_tau_csr(25)


def test_tau_csr_from_full_roundtrip():
    L, Nt = 2, 30
    P_tau = O.precon_tau_matrix(Nt)
    full = np.kron(P_tau, np.eye(L * L)).astype(np.complex64)
    csr = torch.tensor(full).to_sparse_csr()
    rp, col, val = precon.tau_csr_from_full(csr, L)
    dense = np.zeros((Nt, Nt))
    for t in range(Nt):
        dense[t, col[rp[t]:rp[t + 1]]] = val[rp[t]:rp[t + 1]]
    np.testing.assert_array_equal(dense, P_tau)
    bad = full.copy()
    bad[0, 1] = 0.5  # couples different sites
    with pytest.raises(RuntimeError):
        precon.tau_csr_from_full(torch.tensor(bad).to_sparse_csr(), L)


def test_ops_refuse_cpu_tensors():
    from qed_fermion_b200 import ops
    x = torch.zeros(1, 4 * 4 * 10, dtype=torch.complex64)
    b = torch.zeros(1, 2 * 4 * 4 * 10, dtype=torch.float32)
    with pytest.raises(RuntimeError):
        ops.apply_operator("mhm", b, x, 4, 0.1)
