"""Pins the C restatement (oracle/) against golden vectors produced by the
reference itself (tests/golden/make_golden.py)."""
import numpy as np
import pytest

from oracle.oracle import REP_ADJ, REP_FUND, REP_GENERAL, LEAPFROG, OMELYAN

FIXTURES = ["su3_fund_d4", "su2_fund_d4", "su3_adj_d3", "su2_adj_d4", "su3_sextet_d3", "su3_octet_d3",
            "su3_27plet_d2", "su3_gauge_d4", "su2_gauge_d3"]


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300))


def oracle_rep(orc, golden, fx):
    spec = str(fx["spec"])
    N = int(fx["N"])
    if spec == "none":
        return None
    if spec == "fund":
        return orc.rep(REP_FUND, N)
    if spec == "adj":
        return orc.rep(REP_ADJ, N)
    reps = golden("reps")
    tag = f"N{N}_{spec.replace(',', '-').replace(':', '_')}"
    d, real, n, dimT, _ = reps[tag + "_info"]
    return orc.rep(REP_GENERAL, N, int(d), int(real), int(n), int(dimT), reps[tag + "_T"], reps[tag + "_W"])


def test_rng_against_reference(orc, golden):
    g = golden("rng")
    for i, seed in enumerate(g["seeds"]):
        seed = int(seed)
        keys = g["keys"][i]
        u = np.array([orc.uniform(seed, int(k)) for k in keys])
        assert np.array_equal(u, g["uniform"][i])           # bit-exact
        gs = np.array([orc.gauss(seed, int(k)) for k in keys])
        assert np.abs(gs - g["gauss"][i]).max() < 1e-15
    for args, out in zip(g["key_args"], g["key_out"]):
        assert orc.key(*[int(x) for x in args]) == int(out)


@pytest.mark.parametrize("name", FIXTURES)
def test_fields_forces_steps(orc, golden, name):
    fx = golden(name)
    D, N = int(fx["D"]), int(fx["N"])
    L = [int(x) for x in fx["L"]]
    beta, kappa, lam = float(fx["beta"]), float(fx["kappa"]), float(fx["lam"])
    U0 = fx["U0"]
    assert np.abs(orc.hot_start(D, N, L, int(fx["seed"]), 0.8) - U0).max() < 1e-15
    assert abs(orc.avg_plaquette(D, N, L, U0) - fx["plaq"]) < 1e-14
    assert abs(orc.gauge_action(D, N, L, U0, beta) - fx["S_g"]) < 1e-12 * max(1, abs(fx["S_g"]))
    assert abs(orc.polyakov(D, N, L, U0) - fx["poly"]) < 1e-14
    assert rel(orc.gauge_force(D, N, L, U0, beta), fx["F_gauge"]) < 1e-13
    rep = oracle_rep(orc, golden, fx)
    if rep is not None:
        phi = fx["phi0"]
        assert rel(orc.matter_force(D, N, L, rep, U0, phi, kappa), fx["F_matter"]) < 1e-13
        assert rel(orc.scalar_force(D, N, L, rep, U0, phi, kappa, lam), fx["F_phi"]) < 1e-13
        assert abs(orc.scalar_action(D, N, L, rep, U0, phi, kappa, lam) - fx["S_H"]) < 1e-12 * max(1, abs(fx["S_H"]))
        assert abs(orc.link_energy(D, N, L, rep, U0, phi) - fx["L_link"]) < 1e-14
    # the HMC object
    integ = LEAPFROG if int(fx["integ"]) == 0 else OMELYAN
    h = orc.hmc(D, N, L, rep, seed=int(fx["seed"]), beta=beta, kappa=kappa, lam=lam, nmd=int(fx["nmd"]), integ=integ)

    def reset():
        h.U[:] = U0
        h.P[:] = fx["P0"]
        if rep is not None:
            h.phi[:] = fx["phi0"]
            h.pi[:] = fx["pi0"]
    reset()
    assert abs(h.hamiltonian() - fx["H0"]) < 1e-12 * abs(fx["H0"])
    h.P[:] = 0
    h.refresh_momenta()
    assert np.abs(h.P - fx["refresh_P"]).max() < 1e-15
    reset()
    h.kick(float(fx["eps"]))
    assert rel(h.P, fx["kick_P"]) < 1e-13
    if rep is not None:
        assert rel(h.pi, fx["kick_pi"]) < 1e-13
    reset()
    h.drift(float(fx["eps"]))
    assert rel(h.U, fx["drift_U"]) < 1e-13
    reset()
    h.md_evolve()
    assert rel(h.U, fx["md_U"]) < 1e-12 and rel(h.P, fx["md_P"]) < 1e-12
    h.reunitarize_all()
    assert rel(h.U, fx["reunit_U"]) < 1e-12
    reset()
    h.h.traj_count = 0
    acc = h.trajectory()
    assert abs(h.h.last_dH - fx["traj_dH"]) < 1e-12 * abs(fx["H0"]) + 1e-12
    assert acc == bool(fx["traj_acc"])
    assert rel(h.U, fx["traj_U"]) < 1e-12


@pytest.mark.parametrize("N", [2, 3])
def test_group_kernels(orc, golden, N):
    reps = golden("reps")
    T = orc.generators(N)
    assert np.abs(T - reps[f"gen{N}"]).max() == 0.0
    # Tr T^a T^b = delta/2, Hermitian, traceless (test/test_math.cpp:17-34)
    G = np.einsum("aij,bji->ab", T, T)
    assert np.abs(G - 0.5 * np.eye(N * N - 1)).max() < 1e-14
    rng = np.random.default_rng(N)
    for _ in range(10):
        H = np.einsum("a,aij->ij", rng.normal(size=N * N - 1), T)
        U = orc.expi(H)
        assert np.abs(U.conj().T @ U - np.eye(N)).max() < 1e-12
        assert abs(np.linalg.det(U) - 1) < 1e-12
        Ur = orc.reunitarize(U + 1e-6 * rng.normal(size=(N, N)))
        assert np.abs(Ur.conj().T @ Ur - np.eye(N)).max() < 1e-14
        assert abs(np.linalg.det(Ur) - 1) < 1e-14
