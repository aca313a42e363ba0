"""Generate the golden fixtures under tests/golden/ from the reference itself.

Run in the development container, where the reference tree exists and
`make -C oracle ref` has built oracle/_ref/libghref.so (the unmodified
reference headers compiled with the reference Makefile's flags):

    python tests/golden/make_golden.py

Every number in the .npz files is an output of the reference's own code
(GaugeField::hot, LinkMom::refresh, add_gauge_force, scalar_force,
GaugeHiggsHMC::trajectory, GeneralRep tables, ...).  The tests pin the C
restatement (oracle/) and the product against these files.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle.oracle import Reference, LEAPFROG, OMELYAN  # noqa: E402

R = Reference()
R.set_threads(1)  # deterministic reduction order


def rng_fixture():
    seeds = [1, 7, 0x1234567890ABCDEF]
    rows = []
    for seed in seeds:
        keys = [R.key(1, s, mu, a) for s in range(40) for mu in range(4) for a in range(8)]
        keys += [R.key(0xC3, R.key(0xC3, t), s, mu, a) for t in range(3) for s in range(8) for mu in range(4) for a in range(3)]
        keys += [R.key(12345, s, k) for s in range(64) for k in range(6)]
        keys += list(range(200))
        keys = np.array(keys, np.uint64)
        rows.append((seed, keys, R.uniform_many(seed, keys), R.gauss_many(seed, keys)))
    key_args = np.array([[1, 2, 3, 4, 5], [0xC3, 7, 0, 0, 0], [0xE5, 12, 0, 0, 0], [2**63, 2**64 - 1, 0, 1, 2]], np.uint64)
    key_out = np.array([R.key(*[int(x) for x in k]) for k in key_args], np.uint64)
    np.savez_compressed(os.path.join(HERE, "rng.npz"),
                        seeds=np.array([r[0] for r in rows], np.uint64),
                        keys=np.stack([r[1] for r in rows]), uniform=np.stack([r[2] for r in rows]),
                        gauss=np.stack([r[3] for r in rows]), key_args=key_args, key_out=key_out)


def rep_fixture():
    out = {}
    for N, spec in [(2, "2:real"), (2, "3"), (3, "1,1"), (3, "2"), (3, "2,1:real"), (3, "4,2:real")]:
        T, W, info = R.rep_tables(N, spec)
        tag = f"N{N}_{spec.replace(',', '-').replace(':', '_')}"
        out[tag + "_T"] = T
        out[tag + "_W"] = W
        out[tag + "_info"] = np.array([info["d"], info["real"], info["n"], info["dimT"], info["use_fast"]])
        rng = np.random.default_rng(11)
        a = rng.uniform(-1.2, 1.2, size=N * N - 1)
        H = np.einsum("a,aij->ij", a, R.generators(N))
        U = R.expi(H)
        d = info["d"]
        phi = rng.normal(size=d) + 1j * rng.normal(size=d)
        phy = rng.normal(size=d) + 1j * rng.normal(size=d)
        out[tag + "_U"] = U
        out[tag + "_phi"] = phi
        out[tag + "_phiy"] = phy
        out[tag + "_rot"] = R.rep_rotate(N, spec, U, phi)
        out[tag + "_rotdag"] = R.rep_rotate(N, spec, U, phi, dag=True)
        out[tag + "_hop"] = R.rep_hop(N, spec, U, phi, phy)
    for N in (2, 3):
        out[f"gen{N}"] = R.generators(N)
    np.savez_compressed(os.path.join(HERE, "reps.npz"), **out)


def field_fixture(name, D, N, L, spec, beta, kappa, lam, nmd, integ, seed=1, eps=0.0625):
    """Initial fields, forces, actions, one kick/drift, md_evolve, one trajectory."""
    out = dict(D=D, N=N, L=np.array(L), beta=beta, kappa=kappa, lam=lam, nmd=nmd, integ=integ, seed=seed, eps=eps)
    out["spec"] = np.array(spec)
    U = R.hot_start(D, N, L, seed, 0.8)
    out["U0"] = U
    out["plaq"] = R.avg_plaquette(D, N, L, U)
    out["S_g"] = R.gauge_action(D, N, L, U, beta)
    out["poly"] = R.polyakov(D, N, L, U)
    out["F_gauge"] = R.gauge_force(D, N, L, U, beta)
    V = int(np.prod(L))
    ngen = N * N - 1
    P0 = R.mom_refresh(D, N, L, seed, R.key(0xC3 if spec != "none" else 0xA1, 0))
    out["P0"] = P0
    if spec != "none":
        info = R.rep_info(N, spec)
        d = info["d"]
        phi = R.phi_gaussian(D, L, d, seed, 12345, info["real"], 0.3)
        out["phi0"] = phi
        out["F_matter"] = R.matter_force(D, N, L, spec, U, phi, kappa)
        out["F_phi"] = R.scalar_force(D, N, L, spec, U, phi, kappa, lam)
        out["S_H"] = R.scalar_action(D, N, L, spec, U, phi, kappa, lam)
        out["L_link"] = R.link_energy(D, N, L, spec, U, phi)
        out["L_phi"] = float(np.sum(np.abs(phi) ** 2) / V)
        pi0 = R.phi_gaussian(D, L, d, seed, R.key(0xD4, 0), info["real"], 1.0)
        out["pi0"] = pi0
    else:
        d = 1
        phi = np.zeros((V, 1), np.complex128)
        pi0 = np.zeros((V, 1), np.complex128)
    base = dict(U=U.copy(), P=P0.copy(), phi=phi.copy(), pi=pi0.copy())
    kw = dict(seed=seed, beta=beta, kappa=kappa, lam=lam, nmd=nmd, integ=integ)
    # refresh via the HMC object itself (keys 0xC3/0xD4 or 0xA1 at traj_count 0)
    st = {k: v.copy() for k, v in base.items()}
    st["P"][:] = 0
    st["pi"][:] = 0
    R.hmc_op("refresh", D, N, L, spec, st, **kw)
    out["refresh_P"] = st["P"]
    out["refresh_pi"] = st["pi"]
    out["H0"] = R.hmc_op("hamiltonian", D, N, L, spec, {k: v.copy() for k, v in base.items()}, **kw)[0]
    st = {k: v.copy() for k, v in base.items()}
    R.hmc_op("kick", D, N, L, spec, st, eps=eps, **kw)
    out["kick_P"], out["kick_pi"] = st["P"], st["pi"]
    st = {k: v.copy() for k, v in base.items()}
    R.hmc_op("drift", D, N, L, spec, st, eps=eps, **kw)
    out["drift_U"], out["drift_phi"] = st["U"], st["phi"]
    st = {k: v.copy() for k, v in base.items()}
    R.hmc_op("md_evolve", D, N, L, spec, st, **kw)
    out["md_U"], out["md_P"], out["md_phi"], out["md_pi"] = st["U"], st["P"], st["phi"], st["pi"]
    out["md_H"] = R.hmc_op("hamiltonian", D, N, L, spec, {k: v.copy() for k, v in st.items()}, **kw)[0]
    st = dict(U=out["md_U"].copy(), P=out["md_P"].copy(), phi=out["md_phi"].copy(), pi=out["md_pi"].copy())
    R.hmc_op("reunitarize", D, N, L, spec, st, **kw)
    out["reunit_U"] = st["U"]
    st = {k: v.copy() for k, v in base.items()}
    res = R.hmc_op("trajectory", D, N, L, spec, st, **kw)
    out["traj_dH"], out["traj_acc"] = res[0], res[1]
    out["traj_U"], out["traj_phi"] = st["U"], st["phi"]
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)


def multi_fixture():
    """Multi-invariant onsite potential (src/action/scalar_invariants.hpp): channels,
    the combined superoperator, V and dV/dphibar of single vectors, and the scalar
    force and action of small lattices with that potential."""
    out = {}
    cases = [(2, "fund"), (2, "adj"), (3, "fund"), (3, "adj"), (2, "6"), (3, "2"), (3, "2,1:real")]
    rng = np.random.default_rng(2026)
    for N, spec in cases:
        tag = f"N{N}_{spec.replace(',', '-').replace(':', '_')}"
        c2 = R.casimir_channels(N, spec)
        f = np.round(rng.uniform(0.2, 1.5, size=len(c2)), 3)
        mu2 = 0.7
        A = R.multi_superop(N, spec, f, mu2)
        d = int(round(np.sqrt(A.shape[0])))
        phis = rng.normal(size=(4, d)) + 1j * rng.normal(size=(4, d))
        vals, dvs = [], []
        for ph in phis:
            v, g = R.multi_value_dV(N, spec, f, mu2, ph)
            vals.append(v)
            dvs.append(g)
        out.update({tag + "_c2": c2, tag + "_f": f, tag + "_mu2": np.array(mu2), tag + "_A": A,
                    tag + "_phi": phis, tag + "_value": np.array(vals), tag + "_dV": np.array(dvs)})
    # lattices: scalar force and action with the potential
    for name, D, N, L, spec in [("lat_su2_fund", 3, 2, [3, 4, 2], "fund"), ("lat_su3_adj", 3, 3, [2, 3, 2], "adj"),
                                ("lat_su2_spin3", 2, 2, [3, 2], "6")]:
        c2 = R.casimir_channels(N, spec)
        f = np.round(rng.uniform(0.2, 1.5, size=len(c2)), 3)
        U = R.hot_start(D, N, L, 5, 0.8)
        d = R.multi_superop(N, spec, f, 0.0).shape[0]
        d = int(round(np.sqrt(d)))
        phi = R.phi_gaussian(D, L, d, 5, 12345, False, 0.6)
        out.update({name + "_f": f, name + "_U": U, name + "_phi": phi, name + "_L": np.array(L),
                    name + "_Fphi": R.scalar_force_multi(D, N, L, spec, U, phi, 0.17, f, 0.4),
                    name + "_SH": np.array(R.scalar_action_multi(D, N, L, spec, U, phi, 0.17, f, 0.4))})
    np.savez_compressed(os.path.join(HERE, "multi_potential.npz"), **out)


def frozen_fixture():
    """Frozen-length scalar (GaugeHiggsHMC::frozen_phi): normalize_phi, the tangent-space
    refresh, one kick (radial force dropped), one geodesic drift and a whole MD evolution
    of the reference, from one start state."""
    out = {}
    for name, D, N, L, spec, kappa in [("su2_fund", 3, 2, [3, 4, 2], "fund", 0.3), ("su3_adj", 3, 3, [2, 3, 2], "adj", 0.2),
                                       ("su2_spin3", 2, 2, [3, 2], "6", 0.25)]:
        d = {"fund": N, "adj": N * N - 1}.get(spec) or R.rep_info(N, spec)["d"]
        V = int(np.prod(L))
        st = {"U": R.hot_start(D, N, L, 3, 0.6), "P": np.zeros((V, D, N * N - 1)),
              "phi": R.phi_gaussian(D, L, d, 3, 12345, spec == "adj", 0.7), "pi": np.zeros((V, d), np.complex128)}
        kw = dict(seed=3, beta=2.1, kappa=kappa, lam=0.5, nmd=3, tau=0.5, integ=OMELYAN)
        R.hmc_op_frozen("normalize", D, N, L, spec, st, **kw)
        out[name + "_U0"], out[name + "_phi0"], out[name + "_L"] = st["U"].copy(), st["phi"].copy(), np.array(L)
        R.hmc_op_frozen("refresh", D, N, L, spec, st, **kw)
        out[name + "_P0"], out[name + "_pi0"] = st["P"].copy(), st["pi"].copy()
        s1 = {k: v.copy() for k, v in st.items()}
        R.hmc_op_frozen("kick", D, N, L, spec, s1, eps=0.07, **kw)
        out[name + "_kick_P"], out[name + "_kick_pi"] = s1["P"], s1["pi"]
        s2 = {k: v.copy() for k, v in st.items()}
        R.hmc_op_frozen("drift", D, N, L, spec, s2, eps=0.07, **kw)
        out[name + "_drift_U"], out[name + "_drift_phi"], out[name + "_drift_pi"] = s2["U"], s2["phi"], s2["pi"]
        s3 = {k: v.copy() for k, v in st.items()}
        R.hmc_op_frozen("md_evolve", D, N, L, spec, s3, **kw)
        out[name + "_md_U"], out[name + "_md_phi"], out[name + "_md_pi"] = s3["U"], s3["phi"], s3["pi"]
        out[name + "_H0"] = R.hmc_op_frozen("hamiltonian", D, N, L, spec, {k: v.copy() for k, v in st.items()}, **kw)[0]
    np.savez_compressed(os.path.join(HERE, "frozen_phi.npz"), **out)


def loops_fixture():
    """Wilson loops (fundamental and in probe irreps) and Polyakov loops in probe irreps
    of the reference (src/measure/observables.hpp:36-101) on hot configurations."""
    out = {}
    for name, D, N, L, sigma in [("su2_d4", 4, 2, [4, 3, 4, 5], 0.5), ("su3_d4", 4, 3, [3, 4, 2, 4], 0.4),
                                 ("su3_d3", 3, 3, [4, 4, 3], 0.7)]:
        U = R.hot_start(D, N, L, 7, sigma)
        out[name + "_U"], out[name + "_L"] = U, np.array(L)
        specs = ["fund0", "fund", "adj", "2", "3"] + (["2,1", "1,1", "3,1"] if N == 3 else ["4", "6"])
        for spec in specs:
            for Ra, Rb in [(1, 1), (2, 1), (2, 3)]:
                out[f"{name}_W_{spec}_{Ra}x{Rb}"] = np.array(R.wilson_loop(D, N, L, spec, U, Ra, Rb))
            if spec != "fund0":
                for tdir in range(D):
                    out[f"{name}_P_{spec}_{tdir}"] = np.array(R.polyakov_rep(D, N, L, spec, U, tdir))
    np.savez_compressed(os.path.join(HERE, "loops.npz"), **out)


if __name__ == "__main__" and sys.argv[1:] == ["loops"]:
    loops_fixture()
elif __name__ == "__main__" and sys.argv[1:] == ["multi"]:
    multi_fixture()
elif __name__ == "__main__" and sys.argv[1:] == ["frozen"]:
    frozen_fixture()
elif __name__ == "__main__":
    loops_fixture()
    frozen_fixture()
    multi_fixture()
    rng_fixture()
    rep_fixture()
    field_fixture("su3_fund_d4", 4, 3, [4, 3, 2, 3], "fund", 5.7, 0.10, 0.5, 4, OMELYAN)
    field_fixture("su2_fund_d4", 4, 2, [3, 4, 2, 3], "fund", 2.3, 0.20, 0.5, 5, LEAPFROG)
    field_fixture("su3_adj_d3", 3, 3, [3, 4, 3], "adj", 5.7, 0.15, 0.5, 4, OMELYAN)
    field_fixture("su2_adj_d4", 4, 2, [3, 2, 3, 2], "adj", 2.3, 0.3, 0.4, 4, LEAPFROG)
    field_fixture("su3_sextet_d3", 3, 3, [3, 2, 3], "2", 5.7, 0.1, 0.5, 3, OMELYAN)
    field_fixture("su3_octet_d3", 3, 3, [2, 3, 2], "2,1:real", 5.7, 0.1, 0.5, 3, OMELYAN)
    field_fixture("su3_27plet_d2", 2, 3, [2, 3], "4,2:real", 5.7, 0.1, 0.5, 2, OMELYAN)
    field_fixture("su3_gauge_d4", 4, 3, [3, 2, 3, 4], "none", 5.7, 0.0, 0.0, 4, OMELYAN)
    field_fixture("su2_gauge_d3", 3, 2, [4, 4, 4], "none", 2.3, 0.0, 0.0, 6, LEAPFROG)
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))
