"""CPU oracle for the qed_fermion hybrid-QMC fermion hot path (numpy restatement).

TEST INFRASTRUCTURE ONLY.  This module is the checker that the CUDA path is
compared against.  Only the test suite, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import it; the product package
(``qed_fermion_b200``) never imports, links or executes anything here.

Every function restates, in vectorised numpy, an algorithm of the reference
project KexinFeng/qed_fermion; the docstring names the reference file:line it
follows.  Parity of this restatement is pinned against golden vectors that the
reference itself produced in complex128 (``tests/golden/make_golden.py``,
fixtures ``tests/golden/*.npz``, checked by ``tests/test_oracle_golden.py``).

Conventions (identical to the reference's ``_C`` call sites):

* lattice ``L x L`` (``Lx == Ly == L``, L even), ``Vs = L*L`` sites per slice,
  site index ``s = x + L*y``; ``Nt`` imaginary-time slices; vector index
  ``t*Vs + s`` (``hmc_sampler_batch.py:1741-1753``).
* gauge angles in "kernel layout" ``[..., Nt, Ly, Lx, 2]`` flattened to
  ``[..., Nt, 2*Vs]``: angle of bond ``(site s, component c)`` at ``2*s + c``,
  c=0 the x-bond ``s -> s+x``, c=1 the y-bond ``s -> s+y``
  (``boson.permute([0, 4, 3, 2, 1])``, ``hmc_sampler_batch.py:2166``).
* "reference layout" of bosons, momenta and forces: ``[bs, 2, Lx, Ly, Nt]``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

# ----------------------------------------------------------------------------
# geometry (checkerboard bond groups)
# ----------------------------------------------------------------------------


def geometry(L: int):
    """Checkerboard bond groups g=1..4 as (i_list, j_list, boson_idx_list).

    Restates ``HmcSampler.initialize_geometry`` (``hmc_sampler_batch.py:937-969``):
    sites ``(x, y)`` with ``x, y`` both even (row-major over (y, x)), then both
    odd, are the "A" sites.  g1: x-bond A -> A+x; g2: y-bond A -> A+y;
    g3: x-bond (A-x) -> A; g4: y-bond (A-y) -> A.  ``boson_idx = 2*i + c``.
    Returns int64 arrays, each of length ``Vs/2``.
    """
    assert L % 2 == 0 and L >= 2
    Lx = Ly = L
    out_i, out_j = [[], [], [], []], [[], [], [], []]
    for parity in (0, 1):
        xs = np.arange(parity, Lx, 2, dtype=np.int64)[None, :]
        ys = np.arange(parity, Ly, 2, dtype=np.int64)[:, None]
        a = (xs + ys * Lx).reshape(-1)
        out_i[0].append(a)
        out_j[0].append(((xs + 1) % Lx + ys * Lx).reshape(-1))
        out_i[1].append(a)
        out_j[1].append((xs + (ys + 1) % Ly * Lx).reshape(-1))
        out_i[2].append(((xs - 1) % Lx + ys * Lx).reshape(-1))
        out_j[2].append(a)
        out_i[3].append((xs + (ys - 1) % Ly * Lx).reshape(-1))
        out_j[3].append(a)
    i_list = [np.concatenate(v) for v in out_i]
    j_list = [np.concatenate(v) for v in out_j]
    comp = [0, 1, 0, 1]
    b_idx = [i_list[g] * 2 + comp[g] for g in range(4)]
    return i_list, j_list, b_idx


_GEOM_CACHE: dict = {}


def _geom(L):
    if L not in _GEOM_CACHE:
        _GEOM_CACHE[L] = geometry(L)
    return _GEOM_CACHE[L]


def factor_coeffs(dtau: float, t: float = 1.0):
    """(c_g, s_g) of the four bond factors.

    g1 uses ``cosh/sinh(t*dtau)``, g2..g4 ``cosh/sinh(t*dtau/2)``
    (``get_dB``/``get_dB1`` ``hmc_sampler_batch.py:1508-1550``, off-diagonals
    ``:1770-1866``).
    """
    c = [math.cosh(t * dtau)] + [math.cosh(t * dtau / 2)] * 3
    s = [math.sinh(t * dtau)] + [math.sinh(t * dtau / 2)] * 3
    return c, s


# ----------------------------------------------------------------------------
# one-slice operators
# ----------------------------------------------------------------------------


def apply_factor(v, phi, g, L, dtau, t=1.0):
    """F_g v for every slice in the batch.

    ``v``: complex ``[..., Vs]``; ``phi``: real ``[..., 2*Vs]`` (same leading
    shape).  ``F_g = c_g I + s_g (e^{i phi} E_ij + e^{-i phi} E_ji)`` over the
    pairs of group g (``get_M_sparse`` ``hmc_sampler_batch.py:1770-1866``).
    """
    i_l, j_l, b_l = _geom(L)
    c, s = factor_coeffs(dtau, t)
    ang = phi[..., b_l[g]]
    ph = np.exp(1j * ang)
    vi = v[..., i_l[g]]
    vj = v[..., j_l[g]]
    out = np.empty_like(v)
    out[..., i_l[g]] = c[g] * vi + s[g] * ph * vj
    out[..., j_l[g]] = s[g] * np.conj(ph) * vi + c[g] * vj
    return out


# order in which B_tau = F4 F3 F2 F1 F2 F3 F4 acts on a column vector
B_SEQUENCE = (3, 2, 1, 0, 1, 2, 3)


def b_vec_per_tau(phi_slice, v, L, dtau, interm=False, t=1.0):
    """B_tau v, or the six partial products.

    Restates the semantics of ``_C.b_vec_per_tau`` as used by ``force_f_fast``
    (``hmc_sampler_batch.py:2174-2189``): with ``interm`` the rows are
    ``[F4 v, F3F4 v, F2F3F4 v, F1F2F3F4 v, F2F1F2F3F4 v, F3F2F1F2F3F4 v]``.
    The raw values of ``v`` are used (a conjugation flag on the caller's
    tensor is not applied), which is what the reference's call sites rely on.
    """
    w = np.asarray(v)
    rows = []
    for k, g in enumerate(B_SEQUENCE):
        w = apply_factor(w, phi_slice, g, L, dtau, t)
        if k < 6:
            rows.append(w)
    if interm:
        return np.stack(rows, axis=-2)
    return w


def apply_B(v, phi, L, dtau, t=1.0):
    """B_tau v slice by slice: ``v`` ``[..., Nt, Vs]``, ``phi`` ``[..., Nt, 2Vs]``."""
    w = v
    for g in B_SEQUENCE:
        w = apply_factor(w, phi, g, L, dtau, t)
    return w


# ----------------------------------------------------------------------------
# full operators M, M^dagger, M^dagger M
# ----------------------------------------------------------------------------


def m_vec(phi, x, L, dtau, t=1.0):
    """M x with ``M = I - sum_{t<Nt-1} E_{t+1,t} B_t + E_{0,Nt-1} B_{Nt-1}``.

    Restates ``get_M_sparse`` (``hmc_sampler_batch.py:1884-1903``).
    ``phi``: ``[..., Nt, 2Vs]`` real; ``x``: ``[..., Nt, Vs]`` complex.
    """
    w = apply_B(x, phi, L, dtau, t)
    y = x.copy()
    y[..., 1:, :] -= w[..., :-1, :]
    y[..., 0, :] += w[..., -1, :]
    return y


def mh_vec(phi, y, L, dtau, t=1.0):
    """M^dagger y (B_t is Hermitian), the semantics of ``_C.mh_vec``
    (``hmc_sampler_batch.py:2406``, ``stochastic_estimator.py:430``)."""
    u = apply_B(np.roll(y, -1, axis=-2), phi, L, dtau, t)
    z = y.copy()
    z[..., :-1, :] -= u[..., :-1, :]
    z[..., -1, :] += u[..., -1, :]
    return z


def mhm_vec(phi, x, L, dtau, t=1.0):
    """M^dagger M x, the semantics of ``_C.mhm_vec``
    (``hmc_sampler_batch.py:772, 799``; sparse form ``:1905``)."""
    return mh_vec(phi, m_vec(phi, x, L, dtau, t), L, dtau, t)


# ----------------------------------------------------------------------------
# preconditioner P = P_tau (x) I_Vs
# ----------------------------------------------------------------------------

# Coefficient table of the hand-built banded-in-tau preconditioner
# (``preconditioners_orig/precon_manual.py:36-166``): per tau-distance r, the
# values at the first rows ("edge"), the repeated bulk value ("middle") and the
# last rows ("tail"); plus the wrap-around corner values for r = 1..5.
PRECON_DIAG_EDGE = (0.91698223, 1.02107012, 1.1740706, 1.24646831, 1.28092396,
                    1.29741096, 1.30534041, 1.30917168, 1.3110323, 1.31193936)
PRECON_DIAG_TAIL = (1.31167626, 1.31074941, 1.30885756, 1.30498219, 1.29699361,
                    1.28042281, 1.24588311, 1.17343438, 1.02052784)
PRECON_DIAG_MIDDLE = 1.312381281
PRECON_BAND_EDGE = (
    (0.475227, 0.69804072, 0.80315554, 0.85303694, 0.87684089, 0.88826168,
     0.89376724, 0.89643389, 0.89773124, 0.89836514, 0.89867532, 0.89882821),
    (0.32525402, 0.47824016, 0.550632, 0.58508581, 0.60157132, 0.60949975,
     0.61333305, 0.61519265),
    (0.22288805, 0.32804558, 0.3779504, 0.40176818, 0.41319385, 0.4187026,
     0.42137364, 0.42267111),
    (0.15300766, 0.22541766, 0.25988016, 0.27637246, 0.28430402, 0.28813654,
     0.29000109, 0.29090756, 0.291352),
    (0.10518534, 0.15511395, 0.17894313, 0.190377, 0.19588688, 0.1985613,
     0.19986567, 0.20050026, 0.20081173, 0.20096488, 0.20104057),
    (0.10691644, 0.12341493, 0.13135427, 0.13519259, 0.13706173, 0.13796897,
     0.13841458),
)
PRECON_BAND_TAIL = (
    (0.89785033, 0.89652652, 0.89382064, 0.88826007, 0.87676316, 0.85285789,
     0.80287397, 0.69771057),
    (0.61507541, 0.61318511, 0.60930747, 0.60131705, 0.58475631, 0.5502165,
     0.47778079),
    (0.42132217, 0.41861743, 0.41305307, 0.40155935, 0.37766892, 0.3276957),
    (0.29132634, 0.29086968, 0.28994057, 0.28805143, 0.28417516, 0.27618375,
     0.25962788, 0.22511749),
    (0.20103745, 0.20095888, 0.20079921, 0.20047785, 0.19982809, 0.19850214,
     0.19579838, 0.19023941, 0.17874525, 0.15486649),
    (0.13839549, 0.13793865, 0.13701266, 0.13511762, 0.13124515, 0.12326149,
     0.10670882),
)
PRECON_BAND_MIDDLE = (0.8989771, 0.616974, 0.42391914, 0.29178312, 0.20111492,
                      0.13884714)
PRECON_CORNER = (-0.47505581, -0.32495788, -0.22264314, -0.15278356, -0.10501137)


def precon_min_ltau() -> int:
    """Smallest Nt for which the table defines every band (``n_middle >= 0``)."""
    need = len(PRECON_DIAG_EDGE) + len(PRECON_DIAG_TAIL)
    for r in range(1, 7):
        need = max(need, len(PRECON_BAND_EDGE[r - 1]) + len(PRECON_BAND_TAIL[r - 1])
                   + r + (1 if r == 6 else 0))
    return need


def precon_tau_matrix(Nt: int, value_dtype=np.complex64) -> np.ndarray:
    """Dense ``Nt x Nt`` tau-part of the preconditioner, P = P_tau (x) I_Vs.

    Restates ``get_precon_man`` (``precon_manual.py:15-186``): diagonal, bands
    at tau-distance 1..6 (band 6 starts at row 1), corners (0, Nt-r) and
    (Nt-r, 0) for r = 1..5; duplicates are summed as ``coalesce`` does.  The
    reference stores the values as complex64 (``precon_manual.py:27``), so the
    float32-rounded values are returned unless ``value_dtype`` says otherwise.
    """
    if Nt < precon_min_ltau():
        raise ValueError(f"preconditioner table needs Nt >= {precon_min_ltau()}, got {Nt}")

    def q(v):
        return np.asarray(v, dtype=value_dtype).real.astype(np.float64)

    P = np.zeros((Nt, Nt), dtype=np.float64)
    diag = np.concatenate([q(PRECON_DIAG_EDGE),
                           np.full(Nt - len(PRECON_DIAG_EDGE) - len(PRECON_DIAG_TAIL),
                                   q(PRECON_DIAG_MIDDLE)),
                           q(PRECON_DIAG_TAIL)])
    np.add.at(P, (np.arange(Nt), np.arange(Nt)), diag)
    for r in range(1, 7):
        edge, tail = PRECON_BAND_EDGE[r - 1], PRECON_BAND_TAIL[r - 1]
        n_mid = Nt - len(edge) - len(tail) - r - (1 if r == 6 else 0)
        vals = np.concatenate([q(edge), np.full(n_mid, q(PRECON_BAND_MIDDLE[r - 1])), q(tail)])
        rows = np.arange(0 if r < 6 else 1, Nt - r)
        assert rows.size == vals.size
        np.add.at(P, (rows, rows + r), vals)
        np.add.at(P, (rows + r, rows), vals)
    for r in range(1, 6):
        v = q(PRECON_CORNER[r - 1])
        np.add.at(P, (np.array([0]), np.array([Nt - r])), v)
        np.add.at(P, (np.array([Nt - r]), np.array([0])), v)
    return P


def precon_vec(r, P_tau):
    """z = (P_tau (x) I) r for ``r`` ``[..., Nt, Vs]`` (``_C.precon_vec``,
    ``hmc_sampler_batch.py:773, 838``)."""
    return np.einsum("tu,...us->...ts", P_tau, r)


# ----------------------------------------------------------------------------
# conjugate gradient
# ----------------------------------------------------------------------------


def pcg_single(apply_A, b, apply_P=None, rtol=1e-8, max_iter=100, reference_alias=None):
    """Single-system (P)CG; restates ``HmcSampler.preconditioned_cg``
    (``hmc_sampler_batch.py:848-930``).

    Returns ``(x, cnt, err)`` with the reference's counting: ``cnt`` is the
    number of completed non-final iterations, ``err = ||r||/||b||`` last seen.

    ``reference_alias`` (default: on exactly when no preconditioner is given)
    reproduces an aliasing effect of the reference: without a preconditioner
    ``z = r`` and ``p = z`` are the same tensor as ``r`` (``:864-867``), so the
    in-place ``r -= alpha * Op`` (``:884``) also rewrites ``p`` during the
    first iteration and the next direction becomes ``(1 + beta) r_1``.  The
    converged solution is unchanged; only the iteration count differs from
    textbook CG.
    """
    if reference_alias is None:
        reference_alias = apply_P is None
    P = (lambda r: r) if apply_P is None else apply_P
    x = np.zeros_like(b)
    r = b - apply_A(x)
    z = P(r)
    p = z
    rz_old = np.vdot(r, z).real
    nb = np.linalg.norm(b)
    err = np.inf
    cnt = 0
    for it in range(max_iter):
        Op = apply_A(p)
        alpha = rz_old / np.vdot(p, Op).real
        x = x + alpha * p
        r = r - alpha * Op
        if reference_alias and it == 0:
            p = r
        err = np.linalg.norm(r) / nb
        if err < rtol:
            break
        z = P(r)
        rz_new = np.vdot(r, z).real
        beta = rz_new / rz_old
        p = z + beta * p
        rz_old = rz_new
        cnt += 1
    return x, cnt, err


def pcg_batched_masked(apply_A, b, apply_P=None, rtol=1e-8, max_iter=100, reference_alias=None):
    """Batched masked PCG; restates ``preconditioned_cg_fast_test``
    (``hmc_sampler_batch.py:751-846``) for ``b`` ``[bs, N]``.

    A system stops updating x and r once ``||r||/||b|| <= rtol``; its ``p`` is
    reset to ``z`` from then on.  Returns ``(x, iterations, error)`` where
    ``iterations[b]`` counts the iterations the system was still active after
    (the reference's non-graph counter).  ``reference_alias`` as in
    ``pcg_single`` (without a preconditioner ``z = r`` at ``:774``, and the
    in-place ``r -= ...`` at ``:803`` rewrites ``p`` in the first iteration).
    """
    if reference_alias is None:
        reference_alias = apply_P is None
    P = (lambda r: r) if apply_P is None else apply_P
    bs = b.shape[0]
    nb = np.linalg.norm(b, axis=1)
    active = np.ones((bs, 1))
    x = np.zeros_like(b)
    r = b - apply_A(x)
    z = P(r)
    p = z
    rz_old = np.einsum("bj,bj->b", r.conj(), z).real
    iters = np.zeros(bs, dtype=np.int64)
    error = np.full(bs, np.inf)
    for it in range(max_iter):
        Op = apply_A(p)
        alpha = (rz_old / np.einsum("bj,bj->b", p.conj(), Op).real)[:, None]
        x = x + alpha * p * active
        r = r - alpha * Op * active
        if reference_alias and it == 0:
            p = r
        error = np.linalg.norm(r, axis=1) / nb
        active = np.where(error[:, None] > rtol, active, 0.0)
        if (active == 0).all():
            break
        iters += (active[:, 0] == 1)
        z = P(r)
        rz_new = np.einsum("bj,bj->b", r.conj(), z).real
        beta = rz_new / rz_old
        p = z + beta[:, None] * p * active
        rz_old = rz_new
    return x, iters, error


# ----------------------------------------------------------------------------
# fermion force
# ----------------------------------------------------------------------------


def _df_dot(angle, lft_row, rgt, i_l, j_l, s):
    """``df_dot_bs1`` (``hmc_sampler_batch.py:1987-2006``): per bond
    ``lft_i rgt_j v + lft_j rgt_i conj(v)``, ``v = s e^{i(phi + pi/2)}``;
    ``lft_row`` is already a row vector (conjugated)."""
    v = s * np.exp(1j * (angle + np.pi / 2))
    return lft_row[..., i_l] * rgt[..., j_l] * v + lft_row[..., j_l] * rgt[..., i_l] * np.conj(v)


def force_f_from_xi(phi, xi, L, dtau, t=1.0):
    """Fermion force F = -dS_f/dphi given xi = (M^dag M)^{-1} psi.

    Restates ``force_f_sparse`` (``hmc_sampler_batch.py:2230-2330``), whose
    partial products are the same as ``force_f_fast`` (``:2150-2227``), slice
    by slice and vectorised over all slices and batch rows.
    ``phi`` ``[..., Nt, 2Vs]``, ``xi`` ``[..., Nt, Vs]``; returns the force in
    kernel layout ``[..., Nt, 2Vs]``.
    """
    i_l, j_l, b_l = _geom(L)
    _, s = factor_coeffs(dtau, t)
    Nt = xi.shape[-2]
    xi_c = xi
    xi_n = np.roll(xi, -1, axis=-2)

    # right partial products R_k = (F ... ) xi_c, k factors applied
    R = [xi_c]
    for g in B_SEQUENCE:
        R.append(apply_factor(R[-1], phi, g, L, dtau, t))
    Bxi = R[7]
    # left partial products as row vectors: lft_k = u^dag F4 F3 ... (k factors)
    def left_rows(u_col):
        rows = [np.conj(u_col)]
        w = u_col
        for g in B_SEQUENCE[:6]:
            w = apply_factor(w, phi, g, L, dtau, t)
            rows.append(np.conj(w))
        return rows
    ln = left_rows(xi_n)
    lb = left_rows(Bxi)
    sign_B = np.full(Nt, -1.0)
    sign_B[-1] = 1.0
    sign_B = sign_B[:, None]
    F = np.zeros(phi.shape, dtype=np.float64)
    # (group, [(left index k-1, right index 7-k)]) over the occurrences of F_g
    occ = {0: [(3, 3)], 1: [(2, 4), (4, 2)], 2: [(1, 5), (5, 1)], 3: [(0, 6), (6, 0)]}
    for g in range(4):
        ang = phi[..., b_l[g]]
        acc = 0
        for (kl, kr) in occ[g]:
            acc = acc + _df_dot(ang, ln[kl], R[kr], i_l[g], j_l[g], s[g]) * sign_B
            acc = acc + _df_dot(ang, lb[kl], R[kr], i_l[g], j_l[g], s[g])
        F[..., b_l[g]] = 2.0 * np.real(acc)
    return F


# ----------------------------------------------------------------------------
# layouts
# ----------------------------------------------------------------------------


def ref_to_kernel_layout(boson):
    """``[bs, 2, Lx, Ly, Nt] -> [bs, Nt, 2*Vs]`` (``permute([0, 4, 3, 2, 1])``)."""
    bs, _, Lx, Ly, Nt = boson.shape
    return np.ascontiguousarray(np.transpose(boson, (0, 4, 3, 2, 1))).reshape(bs, Nt, 2 * Lx * Ly)


def kernel_to_ref_layout(phi, L):
    """``[bs, Nt, 2*Vs] -> [bs, 2, Lx, Ly, Nt]``."""
    bs, Nt, _ = phi.shape
    return np.ascontiguousarray(np.transpose(phi.reshape(bs, Nt, L, L, 2), (0, 4, 3, 2, 1)))


# ----------------------------------------------------------------------------
# boson action and forces (reference layout [bs, 2, Lx, Ly, Nt])
# ----------------------------------------------------------------------------


@dataclass
class Couplings:
    """Physical couplings as ``HmcSampler.__init__`` scales them
    (``hmc_sampler_batch.py:166-175``): ``J_int = J/dtau * Nf/4``,
    ``K_int = K * dtau * Nf/2``, Nf = 2."""

    J: float = 1.0
    K: float = 1.0
    dtau: float = 0.1
    t: float = 1.0
    m: float = 1.0
    compact: bool = False

    @property
    def J_int(self):
        return self.J / self.dtau * 2 / 4

    @property
    def K_int(self):
        return self.K * self.dtau * 2 / 2

    @property
    def tau_coeff(self):
        return 1.0 / self.J_int / self.dtau ** 2


def curl_phi(boson):
    """``phi_x(r) + phi_y(r+x) - phi_x(r+y) - phi_y(r)`` (``hmc_sampler_batch.py:1409-1426``)."""
    px, py = boson[:, 0], boson[:, 1]
    return px + np.roll(py, -1, axis=1) - np.roll(px, -1, axis=2) - py


def action_boson_plaq(boson, cp: Couplings):
    """``K_int * sum cos(curl)`` (``hmc_sampler_batch.py:1428-1436``)."""
    return cp.K_int * np.cos(curl_phi(boson)).sum(axis=(1, 2, 3))


def force_b_plaq(boson, cp: Couplings):
    """``-dS_plaq/dphi`` (``force_b_plaq_matfree``, ``hmc_sampler_batch.py:1438-1459``)."""
    sc = np.sin(curl_phi(boson))
    gx = cp.K_int * (sc - np.roll(sc, 1, axis=2))
    gy = cp.K_int * (-sc + np.roll(sc, 1, axis=1))
    return np.stack([gx, gy], axis=1)


def action_boson_tau(boson, cp: Couplings):
    """Temporal action (``action_boson_tau``, ``hmc_sampler_batch.py:1363-1372``)."""
    d = np.roll(boson, -1, axis=-1) - boson
    if cp.compact:
        return cp.tau_coeff * (1 - np.cos(d)).sum(axis=(1, 2, 3, 4))
    return cp.tau_coeff * (0.5 * d ** 2).sum(axis=(1, 2, 3, 4))


def force_b_tau(boson, cp: Couplings):
    """``-dS_tau/dphi`` (``force_b_tau_noncmp`` ``:1350-1360``, ``force_b_tau_cmp`` ``:1338-1348``)."""
    d1 = np.roll(boson, -1, axis=-1) - boson
    d2 = boson - np.roll(boson, 1, axis=-1)
    if cp.compact:
        f = -np.sin(d1) + np.sin(d2)
    else:
        f = -d1 + d2
    return -cp.tau_coeff * f


# ----------------------------------------------------------------------------
# HMC trajectory
# ----------------------------------------------------------------------------


def solve_xi(phi_k, psi, L, cp: Couplings, rtol, max_iter, P_tau=None):
    """xi = (M^dag M)^{-1} psi per batch row with the masked batched PCG."""
    bs, Nt, Vs = psi.shape

    def A(v):
        return mhm_vec(phi_k, v.reshape(bs, Nt, Vs), L, cp.dtau, cp.t).reshape(bs, -1)

    Pf = None
    if P_tau is not None:
        def Pf(v):
            return precon_vec(v.reshape(bs, Nt, Vs), P_tau).reshape(bs, -1)
    x, it, err = pcg_batched_masked(A, psi.reshape(bs, -1), Pf, rtol, max_iter)
    return x.reshape(bs, Nt, Vs), it, err


def fermion_force(boson_ref, psi, L, cp, rtol, max_iter, P_tau=None):
    """(F_f in reference layout, xi, iterations, error) for ``boson_ref`` ``[bs,2,L,L,Nt]``."""
    phi_k = ref_to_kernel_layout(boson_ref)
    xi, it, err = solve_xi(phi_k, psi, L, cp, rtol, max_iter, P_tau)
    Fk = force_f_from_xi(phi_k, xi, L, cp.dtau, cp.t)
    return kernel_to_ref_layout(Fk, L), xi, it, err


def leapfrog_cmp(x, p, dt, tau_mask, fb_plaq, fb_tau, cp: Couplings, M=5):
    """Inner boson-only multi-step (``leapfrog_cmp``, ``hmc_sampler_batch.py:2332-2347``)."""
    for _ in range(M):
        p = p + (fb_plaq + fb_tau) * dt / 2 / M * tau_mask
        x = x + p / cp.m * dt / M * tau_mask
        fb_plaq = force_b_plaq(x, cp)
        fb_tau = force_b_tau(x, cp)
        p = p + (fb_plaq + fb_tau) * dt / 2 / M * tau_mask
    return x, p, fb_plaq, fb_tau


def trajectory(boson_ref, p0, R, L, cp: Couplings, delta_t, n_leapfrog,
               rtol, max_iter, P_tau=None, tau_mask=None):
    """One HMC trajectory given the momentum ``p0`` and the Gaussian ``R``.

    Restates ``leapfrog_proposer5`` (``hmc_sampler_batch.py:2366-2625``):
    psi = M(x0)^dag R; H = S_b + sum p^2/2m + Re psi^dag xi; outer leapfrog
    with fermion half-kicks around ``leapfrog_cmp``.  ``delta_t`` is a scalar
    or ``[bs]``.  Returns ``(x, H0, H_fin, cg_iters)``.
    """
    bs, _, Lx, Ly, Nt = boson_ref.shape
    Vs = Lx * Ly
    if tau_mask is None:
        tau_mask = np.ones((1, 1, 1, 1, Nt))
    dt = np.broadcast_to(np.asarray(delta_t, dtype=np.float64).reshape(-1), (bs,)).reshape(bs, 1, 1, 1, 1)
    x = boson_ref.copy()
    p = p0.copy()
    phi0 = ref_to_kernel_layout(x)
    psi = mh_vec(phi0, R.reshape(bs, Nt, Vs), L, cp.dtau, cp.t)
    Ff, xi, it, _ = fermion_force(x, psi, L, cp, rtol, max_iter, P_tau)
    iters = [it]
    Sf0 = np.einsum("bi,bi->b", psi.reshape(bs, -1).conj(), xi.reshape(bs, -1)).real
    H0 = action_boson_tau(x, cp) + action_boson_plaq(x, cp) + (p0 ** 2).sum(axis=(1, 2, 3, 4)) / (2 * cp.m) + Sf0
    fb_plaq = force_b_plaq(x, cp)
    fb_tau = force_b_tau(x, cp)
    for _ in range(n_leapfrog):
        p = p + dt / 2 * Ff * tau_mask
        x, p, fb_plaq, fb_tau = leapfrog_cmp(x, p, dt, tau_mask, fb_plaq, fb_tau, cp)
        Ff, xi, it, _ = fermion_force(x, psi, L, cp, rtol, max_iter, P_tau)
        iters.append(it)
        p = p + dt / 2 * Ff * tau_mask
    Sf = np.einsum("bi,bi->b", psi.reshape(bs, -1).conj(), xi.reshape(bs, -1)).real
    H_fin = action_boson_tau(x, cp) + action_boson_plaq(x, cp) + (p ** 2).sum(axis=(1, 2, 3, 4)) / (2 * cp.m) + Sf
    return x, H0, H_fin, np.stack(iters)


def metropolis_accept(H_old, H_new, u):
    """``u < exp(H_old - H_new)`` per chain (``metropolis_update``, ``hmc_sampler_batch.py:2910``)."""
    return u < np.exp(H_old - H_new)


# ----------------------------------------------------------------------------
# stochastic-estimator solves
# ----------------------------------------------------------------------------


def random_vec_bin(rng: np.random.Generator, nrv: int, n_site: int):
    """Z2 x Z2 noise ``(+-1 +- i)/sqrt(2)`` (``random_vec_bin``, ``stochastic_estimator.py:210-224``)."""
    re = rng.integers(0, 2, size=(nrv, n_site)) * 2 - 1
    im = rng.integers(0, 2, size=(nrv, n_site)) * 2 - 1
    return (re + 1j * im) / np.sqrt(2.0)


def g_eta(phi_slice_k, eta, L, cp: Couplings, rtol, max_iter, P_tau=None):
    """G_eta = (M^dag M)^{-1} M^dag eta for Nrv noise rows sharing one gauge
    field (``set_eta_G_eta_inner``, ``stochastic_estimator.py:427-433``).
    ``phi_slice_k`` ``[Nt, 2Vs]``; ``eta`` ``[Nrv, Nt*Vs]``."""
    nrv = eta.shape[0]
    Nt = phi_slice_k.shape[0]
    Vs = L * L
    phi = np.broadcast_to(phi_slice_k, (nrv,) + phi_slice_k.shape)
    psi = mh_vec(phi, eta.reshape(nrv, Nt, Vs), L, cp.dtau, cp.t)
    x, it, err = solve_xi(np.ascontiguousarray(phi), psi, L, cp, rtol, max_iter, P_tau)
    return x.reshape(nrv, -1), it, err


# ----------------------------------------------------------------------------
# bond-bond correlators of the stochastic estimator
# (stochastic_estimator.py T1 :1393, T21 :1447, T2 :1504, T4 :1561, Tvv :1612,
#  get_bond_bond_per_b2 :2594, bond_corr :2643)
# ----------------------------------------------------------------------------
#
# eta, G_eta: [Nrv, Ltau * L * L] (index tau Vs + x + L y); boson: reference
# layout [1, 2, Lx, Ly, Ltau].  Each T sums, over the noise pairs s < s'
# (itertools order) and over tau, the spatial correlation
#     C(d) = (1 / Vs) sum_r a(r) b(r + d)
# of two bond products, as the FFT identity ifft(ifft(a) fft(b)) with the
# reference's norms, and averages; "shift k" is a roll along x by -k (the value
# at x + k), as torch.roll(..., shifts=-k, dims=-1).


def _bb_fields(eta, G, boson, L, Nt):
    ec = np.conj(eta).reshape(-1, Nt, L, L)
    g = G.reshape(-1, Nt, L, L)
    phx = np.transpose(boson, (0, 1, 4, 3, 2))[0, 0]  # [Ltau, Ly, Lx]
    return ec, g, phx


def _sx(a, k):
    return np.roll(a, -k, axis=-1)


def _corr(a, b):
    aF = np.fft.ifft2(a, norm="backward")
    bF = np.fft.fft2(b, norm="forward")
    return np.fft.ifft2(aF * bF, norm="forward")


def _pairs(nrv):
    return [(s, t) for s in range(nrv) for t in range(s + 1, nrv)]


def _pair_mean(fa, fb, nrv, L):
    acc = np.zeros((L, L), dtype=complex)
    P = _pairs(nrv)
    for s, t in P:
        acc += _corr(fa(s, t), fb(s, t)).mean(axis=0)
    return acc / len(P)


def bb_T1(eta, G, boson, L, Nt):
    ec, g, ph = _bb_fields(eta, G, boson, L, Nt)
    e = np.exp(1j * ph)
    out = -_pair_mean(lambda s, t: ec[s] * _sx(g[t], 1) * e, lambda s, t: _sx(g[s], 1) * ec[t] * e, len(ec), L)
    out[0, -1] += (_sx(g, 1) * np.roll(ec, 1, axis=-1) * e * np.exp(1j * np.roll(ph, 1, axis=-1))).mean()
    return out


def bb_T21(eta, G, boson, L, Nt):
    ec, g, ph = _bb_fields(eta, G, boson, L, Nt)
    fa = lambda s, t: (_sx(ec[s], 1) * g[t] + _sx(ec[t], 1) * g[s]) * np.exp(-1j * ph) / 2
    fb = lambda s, t: (_sx(g[s], 1) * ec[t] + _sx(g[t], 1) * ec[s]) * np.exp(1j * ph) / 2
    out = -_pair_mean(fa, fb, len(ec), L)
    out[0, 0] += (g * ec).mean()
    return out


def bb_T2(eta, G, boson, L, Nt):
    ec, g, ph = _bb_fields(eta, G, boson, L, Nt)
    fa = lambda s, t: (ec[s] * _sx(g[t], 1) + ec[t] * _sx(g[s], 1)) * np.exp(1j * ph) / 2
    fb = lambda s, t: (g[s] * _sx(ec[t], 1) + g[t] * _sx(ec[s], 1)) * np.exp(-1j * ph) / 2
    out = -_pair_mean(fa, fb, len(ec), L)
    out[0, 0] += (g * ec).mean()
    return out


def bb_T4(eta, G, boson, L, Nt):
    ec, g, ph = _bb_fields(eta, G, boson, L, Nt)
    e = np.exp(-1j * ph)
    out = -_pair_mean(lambda s, t: _sx(ec[s], 1) * g[t] * e, lambda s, t: g[s] * _sx(ec[t], 1) * e, len(ec), L)
    out[0, 1] += (g * _sx(ec, 2) * e * np.exp(-1j * _sx(ph, 1))).mean()
    return out


def bb_Tvv(eta, G, boson, L, Nt):
    ec, g, ph = _bb_fields(eta, G, boson, L, Nt)
    v = _sx(g, 1) * ec * np.exp(1j * ph) + g * _sx(ec, 1) * np.exp(-1j * ph)
    return _corr(v, v).mean(axis=(0, 1)), v.mean(axis=(0, 1))


def bb_observables(eta, G, boson, L, Nt):
    """get_bond_bond_per_b2: BB0_r, BB_r, B_r, BB_k (real parts, BB_k reordered
    to ascending momenta)."""
    T = bb_T1(eta, G, boson, L, Nt) + bb_T21(eta, G, boson, L, Nt) + bb_T2(eta, G, boson, L, Nt) + \
        bb_T4(eta, G, boson, L, Nt)
    Tvv, Tv = bb_Tvv(eta, G, boson, L, Nt)
    BB_r = T * 2 + Tvv * 4
    BB_k = np.roll(np.fft.ifft2(BB_r, norm="forward"), (L // 2, L // 2), axis=(0, 1))
    return {"BB0_r": (T * 2).real, "BB_r": BB_r.real, "B_r": Tv.real, "BB_k": BB_k.real}


def bb_bond_corr(BB_r_mean, B_r_mean):
    return BB_r_mean - 4 * _corr(B_r_mean, B_r_mean)


# ----------------------------------------------------------------------------
# adaptive Fourier mass (hmc_sampler_batch.py:1133-1277)
# ----------------------------------------------------------------------------


def fm_accumulate(mean, spec, field, cnt):
    """One step of the running statistics (``update_sigma_hat_cpu`` :1202-1210):
    the field mean and the mean power spectrum of the centred field under the
    orthonormal real FFT over the last three axes, each averaged over the
    ``cnt + 1`` steps of the window.  Returns (mean, spec)."""
    mean = (mean * cnt + field) / (cnt + 1)
    X = np.fft.rfftn(field - mean, axes=(-3, -2, -1), norm="ortho")
    return mean, (spec * cnt + np.abs(X) ** 2) / (cnt + 1)


def fm_mass(spec, lam=0.05, smin=0.8, smax=1.2, lmd=0.9, invert=False):
    """The mass spectrum from the accumulated spectrum (``apply_sigma_hat_cpu``
    :1133-1200) for ``spec`` of shape [bs, 2, ...]: clamp to [0, c] with c the
    mean over (chain, direction) rows of the rows' 0.99 quantiles; Box-Cox
    (s^lam - 1) / lam; per row, rescale into [smin, smax] and shift the mean
    to 1; shrink towards 1 by lmd; invert for mass mode -1."""
    rows = spec.reshape(spec.shape[0] * spec.shape[1], -1)
    c = np.quantile(rows, 0.99, axis=-1).mean()
    s = (np.clip(rows, 0.0, c) ** lam - 1.0) / lam
    lo = s.min(axis=-1, keepdims=True)
    hi = s.max(axis=-1, keepdims=True)
    s = (s - lo) / np.maximum(hi - lo, 1e-8) * (smax - smin) + smin
    s = s - s.mean(axis=-1, keepdims=True) + 1.0
    s = (1.0 - lmd) * s + lmd
    if invert:
        s = 1.0 / s
    return s.reshape(spec.shape)


def fm_draw(sigma, a, b, shape):
    """Momenta with the Fourier mass (``draw_momentum_fft`` :1254-1265): the
    inverse orthonormal real FFT of (a + i b) / sqrt(sigma m_k), m_k = 1 for
    the first and last tau frequency and 2 otherwise."""
    m = np.full(sigma.shape[-1], 2.0)
    m[[0, -1]] = 1.0
    return np.fft.irfftn((a + 1j * b) / np.sqrt(sigma * m), s=shape, axes=(-3, -2, -1), norm="ortho")


def fm_m_inv(p, sigma):
    """``M^-1 p = F^-1 (sigma F p)`` (``apply_m_inv`` :1267-1277, unnormalised FFT pair)."""
    return np.fft.irfftn(np.fft.rfftn(p, axes=(-3, -2, -1)) * sigma, s=p.shape[-3:], axes=(-3, -2, -1))
