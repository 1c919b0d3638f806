"""The C/OpenMP restatement (oracle/qedf_cpu.c) that bench.py times as the CPU
baseline, against the numpy oracle that the reference's golden vectors pin."""
import numpy as np
import pytest

from oracle import cpu_port as C
from oracle import qedf_oracle as O


@pytest.fixture(scope="module", autouse=True)
def _lib():
    C.build()


def _case(L, Nt, seed):
    rng = np.random.default_rng(seed)
    phi = rng.uniform(-np.pi, np.pi, size=(Nt, 2 * L * L))
    x = (rng.standard_normal((Nt, L * L)) + 1j * rng.standard_normal((Nt, L * L))) / np.sqrt(2)
    return phi, x


@pytest.mark.parametrize("L,Nt", [(2, 4), (4, 10), (6, 26)])
def test_mhm_and_force_match_oracle(L, Nt):
    phi, x = _case(L, Nt, L + Nt)
    want = O.mhm_vec(phi[None], x[None], L, 0.1)[0]
    assert np.abs(C.mhm(phi, x, L, 0.1) - want).max() / np.abs(want).max() < 1e-13
    Fw = O.force_f_from_xi(phi[None], x[None], L, 0.1)[0]
    assert np.abs(C.force(phi, x, L, 0.1) - Fw).max() / np.abs(Fw).max() < 1e-12


def test_pcg_iterations_match_oracle():
    L, Nt = 4, 30
    phi, b = _case(L, Nt, 7)
    P = O.precon_tau_matrix(Nt)
    csr = C.csr_of(P)
    z = C.precon(b, csr)
    assert np.abs(z - O.precon_vec(b[None], P)[0]).max() < 1e-13
    s = C.Pcg(phi, b, L, 0.1, csr)
    for _ in range(300):
        s.step()
        if np.sqrt(s.rr / np.vdot(b, b).real) < 1e-10:
            break
    r = b - O.mhm_vec(phi[None], s.x[None], L, 0.1)[0]
    assert np.linalg.norm(r) / np.linalg.norm(b) < 2e-10
    assert C.threads() >= 1
