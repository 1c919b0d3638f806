"""Build and call the C/OpenMP restatement of the fermion path (qedf_cpu.c).

Test infrastructure: the CPU baseline of bench.py times it on all host cores,
and tests/test_cpu_port.py checks it against the numpy oracle (qedf_oracle.py),
which the reference's golden vectors pin.  The library never uses it.
"""
from __future__ import annotations

import ctypes
import os
import shutil
import subprocess
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "qedf_cpu.c")
LIB = os.path.join(HERE, "libqedf_cpu.so")
# portable: the GPU box's host need not be this machine's CPU model
FLAGS = ["-O3", "-march=x86-64-v3", "-fopenmp", "-shared", "-fPIC", "-std=c11"]
_LIB = None


def build(force: bool = False) -> str:
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    cc = shutil.which("gcc") or "cc"
    subprocess.run([cc] + FLAGS + [SRC, "-o", LIB, "-lm"], check=True)
    return LIB


def load():
    global _LIB
    if _LIB is None:
        lib = ctypes.CDLL(LIB)
        d, i, p = ctypes.c_double, ctypes.c_int, ctypes.c_void_p
        lib.qedf_cpu_threads.restype = i
        lib.qedf_cpu_mhm.argtypes = [p, p, p, i, i, d]
        lib.qedf_cpu_precon.argtypes = [p, p, i, i, p, p, p]
        lib.qedf_cpu_pcg_iter.argtypes = [p, p, p, p, p, p, i, i, d, d, p, p, p, p]
        lib.qedf_cpu_pcg_iter.restype = d
        lib.qedf_cpu_force.argtypes = [p, p, p, i, i, d]
        _LIB = lib
    return _LIB


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def threads() -> int:
    return load().qedf_cpu_threads()


def mhm(phi, x, L, dtau):
    """M^dag M x; phi float64 [Nt, 2Vs], x complex128 [Nt, Vs]."""
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.complex128)
    out = np.empty_like(x)
    load().qedf_cpu_mhm(_p(phi), _p(x), _p(out), L, x.shape[-2], dtau)
    return out


def csr_of(P_tau):
    rows, cols = np.nonzero(P_tau)
    row_ptr = np.zeros(P_tau.shape[0] + 1, dtype=np.int32)
    np.add.at(row_ptr, rows + 1, 1)
    return np.cumsum(row_ptr).astype(np.int32), cols.astype(np.int32), P_tau[rows, cols].astype(np.float64)


def precon(r, csr):
    r = np.ascontiguousarray(r, dtype=np.complex128)
    z = np.empty_like(r)
    rp, col, val = csr
    load().qedf_cpu_precon(_p(r), _p(z), r.shape[-2], r.shape[-1], _p(rp), _p(col), _p(val))
    return z


def force(phi, xi, L, dtau):
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    xi = np.ascontiguousarray(xi, dtype=np.complex128)
    F = np.empty_like(phi)
    load().qedf_cpu_force(_p(phi), _p(xi), _p(F), L, xi.shape[-2], dtau)
    return F


class Pcg:
    """State of one PCG solve advanced an iteration at a time (for timing)."""

    def __init__(self, phi, b, L, dtau, csr=None):
        self.phi = np.ascontiguousarray(phi, dtype=np.float64)
        self.L, self.dtau = L, dtau
        self.x = np.zeros_like(b, dtype=np.complex128)
        self.r = np.array(b, dtype=np.complex128)
        self.z = precon(self.r, csr) if csr is not None else self.r.copy()
        self.p = self.z.copy()
        self.Op = np.empty_like(self.r)
        self.csr = csr
        self.rz = float(np.vdot(self.r, self.z).real)
        self.rr = float(np.vdot(self.r, self.r).real)

    def step(self):
        rr = ctypes.c_double()
        rp, col, val = self.csr if self.csr is not None else (None, None, None)
        nul = ctypes.c_void_p()
        self.rz = load().qedf_cpu_pcg_iter(
            _p(self.phi), _p(self.x), _p(self.r), _p(self.p), _p(self.z), _p(self.Op), self.L, self.r.shape[-2],
            self.dtau, self.rz, _p(rp) if rp is not None else nul, _p(col) if col is not None else nul,
            _p(val) if val is not None else nul, ctypes.byref(rr))
        self.rr = rr.value


def time_sample(phi, b, L, dtau, csr, seconds):
    """Seconds per PCG iteration and per force on this input, each timed for
    about the given share of ``seconds``."""
    s = Pcg(phi, b, L, dtau, csr)
    s.step()  # warm the caches and the thread pool
    t0 = time.perf_counter()
    n_it = 0
    while n_it < 1 or time.perf_counter() - t0 < 0.6 * seconds:
        s.step()
        n_it += 1
    t_it = (time.perf_counter() - t0) / n_it
    force(phi, b, L, dtau)
    t1 = time.perf_counter()
    n_f = 0
    while n_f < 1 or time.perf_counter() - t1 < 0.3 * seconds:
        force(phi, b, L, dtau)
        n_f += 1
    return t_it, (time.perf_counter() - t1) / n_f, n_it, n_f


def solve(phi, b, L, dtau, csr, rtol, max_iter):
    """PCG on M^dag M x = b until the iterated relative residual is at most
    ``rtol``: the C port's iteration, the stopping test of ``pcg_single``.
    Returns (x, iterations, relative residual)."""
    s = Pcg(phi, b, L, dtau, csr)
    bb = float(np.vdot(b, b).real)
    it = 0
    while it < max_iter and s.rr > rtol * rtol * bb:
        s.step()
        it += 1
    return s.x, it, (s.rr / bb) ** 0.5


def inner_boson_step(x, p, dt, fb, cp, M=5):
    """One of the M boson-only substeps of ``leapfrog_cmp``
    (``hmc_sampler_batch.py:2332-2347``), numpy, reference layout."""
    from . import qedf_oracle as O
    p = p + fb * dt / 2 / M
    x = x + p / cp.m * dt / M
    fb = O.force_b_plaq(x, cp) + O.force_b_tau(x, cp)
    p = p + fb * dt / 2 / M
    return x, p, fb


def trajectory(boson_ref, p0, R, L, cp, delta_t, n_leapfrog, rtol, max_iter, csr, M=5):
    """One HMC trajectory of one chain (``leapfrog_proposer5``,
    ``hmc_sampler_batch.py:2366-2625``, as ``qedf_oracle.trajectory``): the
    fermion solves and forces on the C port, the boson parts in numpy.
    ``boson_ref`` / ``p0``: ``[1, 2, L, L, Nt]``; ``R``: ``[Nt*Vs]``.
    Returns (H0, H_fin, PCG iterations per solve, seconds by part)."""
    from . import qedf_oracle as O
    Nt = boson_ref.shape[-1]
    Vs = L * L
    secs = {"solve": 0.0, "force": 0.0, "boson": 0.0}

    def fermion(x):
        phi = O.ref_to_kernel_layout(x)[0]
        t0 = time.perf_counter()
        xi, it, _ = solve(phi, psi, L, cp.dtau, csr, rtol, max_iter)
        t1 = time.perf_counter()
        F = force(phi, xi, L, cp.dtau)
        secs["solve"] += t1 - t0
        secs["force"] += time.perf_counter() - t1
        return O.kernel_to_ref_layout(F[None], L), xi, it

    def H(x, p, xi):
        return float(O.action_boson_tau(x, cp)[0] + O.action_boson_plaq(x, cp)[0] + (p ** 2).sum() / (2 * cp.m)
                     + np.vdot(psi, xi).real)

    x = boson_ref.copy()
    p = p0.copy()
    psi = O.mh_vec(O.ref_to_kernel_layout(x), R.reshape(1, Nt, Vs), L, cp.dtau, cp.t)[0]
    Ff, xi, it = fermion(x)
    iters = [it]
    H0 = H(x, p, xi)
    t0 = time.perf_counter()
    fb = O.force_b_plaq(x, cp) + O.force_b_tau(x, cp)
    secs["boson"] += time.perf_counter() - t0
    for _ in range(n_leapfrog):
        p = p + delta_t / 2 * Ff
        t0 = time.perf_counter()
        for _ in range(M):
            x, p, fb = inner_boson_step(x, p, delta_t, fb, cp, M)
        secs["boson"] += time.perf_counter() - t0
        Ff, xi, it = fermion(x)
        iters.append(it)
        p = p + delta_t / 2 * Ff
    return H0, H(x, p, xi), iters, secs
