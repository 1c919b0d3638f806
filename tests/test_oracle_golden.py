"""Pin the CPU oracle against golden vectors produced by the reference itself.

The fixtures come from ``tests/golden/make_golden.py``, which ran the
reference's CPU path (``get_M_sparse``, ``preconditioned_cg``,
``force_f_sparse``, ``leapfrog_proposer5``, ``get_precon_man``) in complex128.
"""
import math
import os

import numpy as np
import pytest

from oracle import qedf_oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def G():
    return dict(np.load(os.path.join(HERE, "golden", "golden_ref.npz")))


@pytest.fixture(scope="module")
def T():
    return dict(np.load(os.path.join(HERE, "golden", "golden_traj.npz")))


@pytest.mark.parametrize("L", [2, 4, 6, 12, 24])
def test_geometry_bit_exact(G, L):
    i_l, j_l, b_l = O.geometry(L)
    for g in range(4):
        np.testing.assert_array_equal(i_l[g], G[f"geom_L{L}_i{g + 1}"])
        np.testing.assert_array_equal(j_l[g], G[f"geom_L{L}_j{g + 1}"])
        np.testing.assert_array_equal(b_l[g], G[f"geom_L{L}_b{g + 1}"])


@pytest.mark.parametrize("tag", ["L4_T10", "L6_T20", "L4_T30"])
def test_operators(G, tag):
    L = int(tag.split("_")[0][1:])
    Nt = int(tag.split("_")[1][1:])
    phi = O.ref_to_kernel_layout(G[f"op_{tag}_boson"])
    x = G[f"op_{tag}_x"].reshape(1, Nt, L * L)
    for name, fn in (("Mx", O.m_vec), ("MHx", O.mh_vec), ("MHMx", O.mhm_vec)):
        got = fn(phi, x, L, 0.1).reshape(-1)
        want = G[f"op_{tag}_{name}"]
        err = np.abs(got - want).max() / np.abs(want).max()
        assert err < 1e-13, (name, err)


@pytest.mark.parametrize("tag", ["L4_T10", "L6_T20", "L4_T30"])
def test_b_vec_per_tau_rows(G, tag):
    L = int(tag.split("_")[0][1:])
    Nt = int(tag.split("_")[1][1:])
    phi = O.ref_to_kernel_layout(G[f"op_{tag}_boson"])[0]
    tau = int(G[f"bvec_{tag}_tau"])
    v = G[f"bvec_{tag}_v"]
    rows = O.b_vec_per_tau(phi[tau], v, L, 0.1, interm=True)
    np.testing.assert_allclose(rows, G[f"bvec_{tag}_rows"][:6], rtol=0, atol=1e-13)
    np.testing.assert_allclose(O.b_vec_per_tau(phi[tau], v, L, 0.1), G[f"bvec_{tag}_rows"][6],
                               rtol=0, atol=1e-13)


@pytest.mark.parametrize("L,Nt", [(2, 26), (2, 30), (4, 60)])
def test_precon_table_equals_reference(G, L, Nt):
    idx = G[f"precon_L{L}_T{Nt}_indices"]
    val = G[f"precon_L{L}_T{Nt}_values"]
    N = L * L * Nt
    dense = np.zeros((N, N), dtype=np.complex128)
    np.add.at(dense, (idx[0], idx[1]), val)
    P_tau = O.precon_tau_matrix(Nt)
    want = np.kron(P_tau, np.eye(L * L))
    np.testing.assert_array_equal(dense.real, want)
    assert np.all(dense.imag == 0)


def test_precon_rejects_short_ltau():
    assert O.precon_min_ltau() == 26
    with pytest.raises(ValueError):
        O.precon_tau_matrix(25)


def test_cg_and_pcg(G):
    L, Nt = 4, 30
    phi = O.ref_to_kernel_layout(G["cg_boson"])
    b = G["cg_rhs"]
    A = lambda v: O.mhm_vec(phi, v.reshape(1, Nt, L * L), L, 0.1).reshape(-1)
    x, cnt, err = O.pcg_single(A, b, None, rtol=1e-10, max_iter=3000)
    assert abs(cnt - int(G["cg_cnt"])) <= 1
    np.testing.assert_allclose(x, G["cg_x"], rtol=0, atol=1e-8 * np.abs(G["cg_x"]).max())
    P_tau = O.precon_tau_matrix(Nt)
    Pf = lambda v: O.precon_vec(v.reshape(1, Nt, L * L), P_tau).reshape(-1)
    x, cnt, err = O.pcg_single(A, b, Pf, rtol=1e-10, max_iter=3000)
    assert abs(cnt - int(G["pcg_cnt"])) <= 1
    assert cnt < int(G["cg_cnt"])
    np.testing.assert_allclose(x, G["pcg_x"], rtol=0, atol=1e-8 * np.abs(G["pcg_x"]).max())


def test_batched_masked_pcg_matches_single(G):
    L, Nt = 4, 30
    phi = O.ref_to_kernel_layout(G["cg_boson"])
    rng = np.random.default_rng(3)
    b = np.stack([G["cg_rhs"], (rng.standard_normal(L * L * Nt) + 1j) * 1e-3])
    phib = np.broadcast_to(phi, (2,) + phi.shape[1:])
    A = lambda v: O.mhm_vec(phib, v.reshape(2, Nt, L * L), L, 0.1).reshape(2, -1)
    x, it, err = O.pcg_batched_masked(A, b, None, rtol=1e-10, max_iter=3000)
    assert np.all(err <= 1e-10)
    np.testing.assert_allclose(x[0], G["cg_x"], rtol=0, atol=1e-8 * np.abs(G["cg_x"]).max())


@pytest.mark.parametrize("tag", ["L4_T10", "L6_T20"])
def test_force_matches_reference(G, tag):
    L = int(tag.split("_")[0][1:])
    Nt = int(tag.split("_")[1][1:])
    phi = O.ref_to_kernel_layout(G[f"force_{tag}_boson"])
    xi = G[f"force_{tag}_xi"].reshape(1, Nt, L * L)
    F = O.kernel_to_ref_layout(O.force_f_from_xi(phi, xi, L, 0.1), L)
    want = G[f"force_{tag}_F"].reshape(F.shape)
    np.testing.assert_allclose(F, want, rtol=0, atol=1e-11 * np.abs(want).max())
    if f"force_{tag}_F_autograd" in G:
        np.testing.assert_allclose(F, G[f"force_{tag}_F_autograd"], rtol=0, atol=1e-8)


def test_force_solve_end_to_end(G):
    tag = "L6_T20"
    L, Nt = 6, 20
    cp = O.Couplings()
    psi = G[f"force_{tag}_psi"].reshape(1, Nt, L * L)
    F, xi, it, err = O.fermion_force(G[f"force_{tag}_boson"], psi, L, cp, 1e-13, 20000)
    np.testing.assert_allclose(xi.reshape(-1), G[f"force_{tag}_xi"], rtol=0,
                               atol=1e-9 * np.abs(G[f"force_{tag}_xi"]).max())
    want = G[f"force_{tag}_F"].reshape(F.shape)
    np.testing.assert_allclose(F, want, rtol=0, atol=1e-9 * np.abs(want).max())


def test_boson_actions_forces(G):
    b = G["boson_b"]
    cp = O.Couplings()
    assert math.isclose(cp.J_int, float(G["boson_J_int"]))
    assert math.isclose(cp.K_int, float(G["boson_K_int"]))
    np.testing.assert_allclose(O.action_boson_tau(b, cp), G["boson_S_tau"], rtol=1e-13)
    np.testing.assert_allclose(O.action_boson_plaq(b, cp), G["boson_S_plaq"], rtol=1e-13)
    np.testing.assert_allclose(O.action_boson_plaq(b, cp), G["boson_S_plaq_curlmat"], rtol=1e-12)
    np.testing.assert_allclose(O.force_b_plaq(b, cp), G["boson_F_plaq"], rtol=0, atol=1e-13)
    np.testing.assert_allclose(O.force_b_tau(b, cp), G["boson_F_tau"], rtol=0, atol=1e-11)
    cpc = O.Couplings(compact=True)
    np.testing.assert_allclose(O.force_b_tau(b, cpc), G["boson_F_tau_cmp"], rtol=0, atol=1e-11)


def test_estimator_g_eta(G):
    L, Nt = 4, 10
    phi = O.ref_to_kernel_layout(G["se_boson"])[0]
    eta = G["se_eta"]
    cp = O.Couplings()
    Gx, it, err = O.g_eta(phi, eta, L, cp, 1e-12, 5000)
    np.testing.assert_allclose(Gx, G["se_G_eta"], rtol=0, atol=1e-8 * np.abs(G["se_G_eta"]).max())


def test_trajectory_matches_reference(T):
    L, Nt = 6, 20
    cp = O.Couplings()
    x, H0, H1, iters = O.trajectory(T["traj_boson"], T["traj_p0"], T["traj_R"], L, cp,
                                    float(T["traj_delta_t"]), int(T["traj_n_leapfrog"]),
                                    rtol=1e-10, max_iter=20000)
    np.testing.assert_allclose(H0, T["traj_H0"], rtol=1e-12)
    np.testing.assert_allclose(H1, T["traj_Hfin"], rtol=1e-9)
    dH_ref = T["traj_Hfin"] - T["traj_H0"]
    assert abs((H1 - H0)[0] - dH_ref[0]) < 1e-6 * abs(T["traj_H0"][0])
    np.testing.assert_allclose(x, T["traj_x"], rtol=0, atol=1e-8)


def test_bond_bond_correlators_match_reference():
    """The oracle's T1, T21, T2, T4, Tvv, get_bond_bond_per_b2 and bond_corr
    against the reference's own (stochastic_estimator.py:1393-1652, 2594-2651)."""
    G = dict(np.load(os.path.join(HERE, "golden", "golden_bond.npz")))
    L, Nt = 6, 12
    args = (G["bb_eta"], G["bb_G_eta"], G["bb_boson"], L, Nt)

    def rel(a, b):
        return np.abs(a - b).max() / np.abs(b).max()
    for name, f in (("T1", O.bb_T1), ("T21", O.bb_T21), ("T2", O.bb_T2), ("T4", O.bb_T4)):
        assert rel(f(*args), G[f"bb_{name}"]) < 1e-12, name
    tvv, tv = O.bb_Tvv(*args)
    assert rel(tvv, G["bb_Tvv"]) < 1e-12 and rel(tv, G["bb_Tv"]) < 1e-12
    ob = O.bb_observables(*args)
    for k in ("BB0_r", "BB_r", "B_r", "BB_k"):
        assert rel(ob[k], G[f"bb_obsr_{k}"]) < 1e-12, k
    assert rel(O.bb_bond_corr(G["bb_obsr_BB_r"], G["bb_obsr_B_r"]), G["bb_bond_corr"]) < 1e-12
