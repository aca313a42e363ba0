"""Integrator-level and statistical checks on the GPU, mirroring the reference's
own tests: test/test_gauge.cpp (force FD, reversibility, dH scaling, <exp(-dH)>),
test/test_scalar.cpp (scalar / link force FD, combined reversibility and
<exp(-dH)>), test/test_general.cpp (general irreps), with the same tolerances,
run in FP64 and in the FP32-MD mode."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def cube(D, n):
    return [n] * D


def expi_np(H):
    w, v = np.linalg.eigh(H)
    return (v * np.exp(1j * w)) @ v.conj().T


def gens(N):
    from oracle.oracle import Oracle
    return Oracle().generators(N)


def make(kind, D, N, precision="fp64", seed=1, **kw):
    import gauge_higgs_b200 as gh
    if kind == "none":
        kw.pop("kappa", None)
        kw.pop("lam", None)
        return gh.GaugeHMC(cube(D, 4), N, seed=seed, precision=precision, **kw)
    rep = {"fund": lambda: gh.FundamentalRep(N), "adj": lambda: gh.AdjointRep(N),
           "gen2": lambda: gh.GeneralRep(N, [2]), "gen2r": lambda: gh.GeneralRep(N, [2], real=True)}[kind]()
    return gh.GaugeHiggsHMC(cube(D, 4), rep, seed=seed, precision=precision, **kw)


# ---------------------------------------------------------------------------
# finite differences (test_gauge.cpp:12-49, test_scalar.cpp:64-120)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("D,N,kind", [(2, 2, "none"), (3, 2, "none"), (4, 2, "none"), (3, 3, "none"),
                                      (3, 2, "fund"), (3, 2, "adj"), (3, 3, "fund"), (3, 3, "gen2")])
def test_link_force_finite_difference(D, N, kind):
    h = make(kind, D, N, beta=2.0, kappa=0.35, lam=0.4)
    h.hot(0.5)
    if kind != "none":
        h.phi_gaussian(77, 0.7)
    U0 = h.U
    F = h.gauge_force() + (h.matter_link_force() if kind != "none" else 0.0)
    T = gens(N)
    eps = 1e-5
    worst = 0.0
    V = U0.shape[0]
    for s in (0, V // 2, V - 1):
        for mu in range(D):
            for a in range(N * N - 1):
                U = U0.copy()
                U[s, mu] = expi_np(eps * T[a]) @ U0[s, mu]
                h.U = U
                m = h.measure()
                Sp = m["S_g"] + m["S_H"]
                U[s, mu] = expi_np(-eps * T[a]) @ U0[s, mu]
                h.U = U
                m = h.measure()
                Sm = m["S_g"] + m["S_H"]
                worst = max(worst, abs((Sp - Sm) / (2 * eps) - F[s, mu, a]))
    assert worst < 1e-5 if kind != "none" else worst < 1e-6
    h.close()


@pytest.mark.parametrize("N,kind", [(2, "fund"), (2, "adj"), (3, "fund"), (3, "adj"), (3, "gen2")])
def test_scalar_force_finite_difference(N, kind):
    h = make(kind, 3, N, kappa=0.3, lam=0.4)
    h.hot(0.5)
    h.phi_gaussian(99, 0.7)
    phi0 = h.phi
    F = h.scalar_force()
    eps = 1e-5
    worst = 0.0
    real = h.rep.real
    for s in (0, 3, phi0.shape[0] - 1):
        for k in range(phi0.shape[1]):
            for unit in ((1.0,) if real else (1.0, 1j)):
                p = phi0.copy()
                p[s, k] += eps * unit
                h.phi = p
                Sp = h.measure()["S_H"]
                p[s, k] -= 2 * eps * unit
                h.phi = p
                Sm = h.measure()["S_H"]
                fd = -(Sp - Sm) / (2 * eps)
                got = F[s, k].real if unit == 1.0 else F[s, k].imag
                worst = max(worst, abs(fd - got))
    assert worst < 1e-5
    h.close()


# ---------------------------------------------------------------------------
# reversibility (test_gauge.cpp:65-85, test_scalar.cpp:122-141)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("fp32", 2e-4), ("fp32-all", 2e-4)])
@pytest.mark.parametrize("N,kind", [(2, "none"), (3, "none"), (2, "fund"), (2, "adj"), (3, "fund"), (3, "gen2")])
def test_reversibility(N, kind, precision, tol):
    h = make(kind, 3, N, precision=precision, seed=999, beta=2.3, kappa=0.3, lam=0.5, nmd=12)
    h.hot(0.5)
    if kind != "none":
        h.phi_gaussian(1, 0.6)
        h.refresh_momenta()
    else:
        h.mom_refresh(7)
    U0 = h.U
    phi0 = h.phi if kind != "none" else None
    h.md_evolve()
    h.P = -h.P
    if kind != "none":
        h.pi = -h.pi
    h.md_evolve()
    U1 = h.U
    worst = np.abs(U1 - U0).max()
    if kind != "none":
        worst = max(worst, np.abs(h.phi - phi0).max())
    assert worst < tol, worst
    h.close()


def test_fp64_refresh_equals_host_draws_bit_for_bit():
    """The FP64 refresh on the device draws every momentum with the two-phase correctly
    rounded log and cos; the host entry point gh_rng_gauss runs the same code, so the
    device momenta equal the host draws bit for bit (P^a = gauss(key(key(0xC3, traj),
    s, mu, a)), pi_k = gauss(key(key(0xD4, traj), s, 2k)) + i gauss(.., 2k + 1))."""
    import gauge_higgs_b200 as gh
    from gauge_higgs_b200._lib import LIB
    seed, L = 5, [4, 4, 4, 4]
    h = gh.GaugeHiggsHMC(L, gh.FundamentalRep(3), seed=seed, precision="fp64", beta=5.7, kappa=0.1, lam=0.5)
    h.hot(0.5)
    h.refresh_momenta()
    P, pi = np.asarray(h.P), np.asarray(h.pi)
    h.close()
    V = int(np.prod(L))
    sp, sq = LIB.gh_rng_key(0xC3, 0, 0, 0, 0), LIB.gh_rng_key(0xD4, 0, 0, 0, 0)
    want = np.array([[[LIB.gh_rng_gauss(seed, LIB.gh_rng_key(sp, s, mu, a, 0)) for a in range(8)] for mu in range(4)]
                     for s in range(V)])
    assert np.array_equal(P.reshape(V, 4, 8), want)
    wpi = np.array([[complex(LIB.gh_rng_gauss(seed, LIB.gh_rng_key(sq, s, 2 * k, 0, 0)),
                             LIB.gh_rng_gauss(seed, LIB.gh_rng_key(sq, s, 2 * k + 1, 0, 0))) for k in range(3)]
                    for s in range(V)])
    assert np.array_equal(pi.reshape(V, 3), wpi)


def test_fp32_refresh_equals_rounded_fp64():
    """The FP32-MD refresh draws with the CUDA math library's FP64 log and cos; rounded
    to FP32 its momenta equal the FP64 mode's correctly rounded draws, bar a few."""
    import gauge_higgs_b200 as gh
    out = {}
    for p in ("fp64", "fp32"):
        h = gh.GaugeHiggsHMC([8, 8, 8, 8], gh.FundamentalRep(3), seed=5, precision=p, beta=5.7, kappa=0.1, lam=0.5)
        h.hot(0.5)
        h.refresh_momenta()
        out[p] = (h.P, h.pi)
        h.close()
    for a, b in zip(out["fp64"], out["fp32"]):
        a, b = np.asarray(a), np.asarray(b)
        if np.iscomplexobj(a):          # pi: compare real and imaginary parts
            a, b = a.view(np.float64), b.view(np.float64)
        a32, b32 = a.astype(np.float32), b.astype(np.float32)
        assert int(np.sum(a32 != b32)) <= 2
        assert np.abs(a32.astype(np.float64) - b32).max() < 1e-6


# ---------------------------------------------------------------------------
# dH second-order scaling (test_gauge.cpp:88-107)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp32-all"])
def test_dH_scaling(precision):
    def run(nmd):
        h = make("none", 3, 2, precision=precision, seed=31415, beta=2.3, nmd=nmd)
        h.hot(0.4)
        h.mom_refresh(5)
        Hi = h.hamiltonian()
        h.md_evolve()
        d = abs(h.hamiltonian() - Hi)
        h.close()
        return d
    ratio = run(8) / run(16)
    assert 3.0 < ratio < 5.0, ratio


# ---------------------------------------------------------------------------
# <exp(-dH)> = 1 and acceptance (test_gauge.cpp:110-129, test_scalar.cpp:143-156,
# test_general.cpp:183-195)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("N,kind,seed", [(2, "none", 2024), (3, "none", 2025), (2, "fund", 501), (2, "adj", 502),
                                         (3, "gen2", 42)])
def test_exp_minus_dH(N, kind, seed, precision):
    import gauge_higgs_b200 as gh
    if kind == "none":
        h = make(kind, 3, N, precision=precision, seed=seed, beta=2.3, nmd=16)
        h.hot(0.3)
        tol, amin = 0.12, 0.55
    else:
        kap = 0.15 if kind == "gen2" else 0.2
        h = make(kind, 3, N, precision=precision, seed=seed, beta=2.3, kappa=kap, lam=0.5, nmd=20)
        h.hot(0.3)
        h.phi_cold(0.4 if kind == "gen2" else 0.5)
        tol, amin = 0.15, 0.5
    ntraj = 300 if kind == "gen2" else 400
    rec = h.run(ntraj)[:, 0]
    mean = float(np.mean(np.exp(-rec["dH"])))
    acc = float(np.mean(rec["accepted"]))
    assert abs(mean - 1.0) < tol, (mean, acc)
    if kind != "gen2":
        assert acc > amin, acc
    t, a, nonfinite = h.traj_counts(0)
    assert t == ntraj and a == int(np.sum(rec["accepted"])) and nonfinite == 0
    h.close()


# ---------------------------------------------------------------------------
# FP32-MD against FP64: forces, one MD trajectory, statistics at equal couplings
# ---------------------------------------------------------------------------
def test_fp32_force_error():
    import gauge_higgs_b200 as gh
    L = [6, 6, 6, 6]
    hs = {p: gh.GaugeHiggsHMC(L, gh.FundamentalRep(3), seed=5, precision=p, beta=5.7, kappa=0.1, lam=0.5)
          for p in ("fp64", "fp32")}
    hs["fp64"].hot(0.8)
    hs["fp64"].phi_gaussian(12345, 0.3)
    U, phi = hs["fp64"].U, hs["fp64"].phi
    hs["fp32"].U = U
    hs["fp32"].phi = phi
    for f in ("gauge_force", "matter_link_force", "scalar_force"):
        a = getattr(hs["fp64"], f)()
        b = getattr(hs["fp32"], f)()
        rel = np.abs(a - b).max() / np.abs(a).max()
        assert rel < 5e-6, (f, rel)
    for h in hs.values():
        h.close()


@pytest.mark.parametrize("N", [2, 3])
def test_fp32_md_drift_is_fp64_arithmetic(N):
    """FP32-MD drift: exp(i eps P), its product with U and the SU(N) projection run in
    FP64 on the FP32 fields, so one drift equals the FP64 drift of the same (rounded)
    inputs followed by one projection to SU(N), up to the final rounding to FP32.  The
    all-FP32 variant is only FP32-accurate."""
    import gauge_higgs_b200 as gh
    L = [6, 4, 4, 6]
    rep = gh.FundamentalRep(N)
    hs = {p: gh.GaugeHiggsHMC(L, rep, seed=11, precision=p, beta=5.7, kappa=0.1, lam=0.5)
          for p in ("fp64", "fp32", "fp32-all")}
    hs["fp64"].hot(0.8)
    hs["fp64"].phi_gaussian(12345, 0.3)
    hs["fp64"].refresh_momenta()
    U = hs["fp64"].U.astype(np.complex64).astype(np.complex128)
    P = hs["fp64"].P.astype(np.float32).astype(np.float64)
    for h in hs.values():
        h.U = U
        h.P = P
        h.phi = hs["fp64"].phi
        h.drift(0.0625)
    ref = hs["fp64"].U
    # the FP64 reference projected to SU(N) in numpy (Gram-Schmidt, det 1)
    M = ref.reshape(-1, N, N).copy()
    for k in range(N - 1):
        for j in range(k):
            M[:, k] -= np.einsum("v,vi->vi", np.einsum("vi,vi->v", M[:, j].conj(), M[:, k]), M[:, j])
        M[:, k] /= np.linalg.norm(M[:, k], axis=1)[:, None]
    if N == 3:
        M[:, 2] = np.cross(M[:, 0], M[:, 1]).conj()
    else:
        M[:, 1] = np.stack([-M[:, 0, 1].conj(), M[:, 0, 0].conj()], axis=1)
    ref = M.reshape(ref.shape)
    err_md = np.abs(hs["fp32"].U - ref).max()
    err_all = np.abs(hs["fp32-all"].U - ref).max()
    assert err_md < 1.5e-7, err_md              # one FP32 rounding of O(1) entries
    assert err_all < 3e-6, err_all
    for h in hs.values():
        h.close()


@pytest.mark.parametrize("p32", ["fp32", "fp32-all"])
def test_fp32_fp64_trajectory_agreement(p32):
    """Same start, same momenta (bit-identical RNG in both modes): dH and the final
    fields of one trajectory agree to FP32 accuracy."""
    import gauge_higgs_b200 as gh
    L = [8, 8, 8, 8]
    out = {}
    for p in ("fp64", p32):
        h = gh.GaugeHiggsHMC(L, gh.FundamentalRep(3), seed=7, precision=p, beta=5.7, kappa=0.1, lam=0.5, nmd=16)
        h.cold()
        h.phi_gaussian(12345, 0.3)
        for _ in range(3):
            h.trajectory()   # leave the cold start
        h.set_traj_count(0, 0, 0)
        acc = h.trajectory()
        out[p] = (h.last_dH, acc, h.U, h.measure()["plaquette"])
        h.close()
    assert abs(out["fp64"][0] - out[p32][0]) < 0.05 + 0.02 * abs(out["fp64"][0])
    assert abs(out["fp64"][3] - out[p32][3]) < 1e-4


# ---------------------------------------------------------------------------
# ensembles: one context of many lattices == independent single-lattice contexts
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_ensemble_equals_independent(precision):
    import gauge_higgs_b200 as gh
    ext = [[4, 4, 4, 4], [6, 4, 4, 6], [5, 5, 3, 4]]
    kappas = [0.22, 0.25, 0.28]
    seeds = [11, 12, 13]
    ens = gh.Ensemble(ext, gh.FundamentalRep(2), seeds=seeds, precision=precision, beta=2.3, kappa=kappas, lam=0.5,
                      nmd=10, integ="leapfrog")
    ens.hot(0.8)
    ens.phi_gaussian(12345, 0.3)
    rec = ens.run(6)
    for i in range(3):
        h = gh.GaugeHiggsHMC(ext[i], gh.FundamentalRep(2), seed=seeds[i], precision=precision, beta=2.3,
                             kappa=kappas[i], lam=0.5, nmd=10, integ="leapfrog")
        h.hot(0.8)
        h.phi_gaussian(12345, 0.3)
        r1 = h.run(6)[:, 0]
        assert np.array_equal(r1["dH"], rec[:, i]["dH"])
        assert np.array_equal(r1["accepted"], rec[:, i]["accepted"])
        assert np.array_equal(h.U, ens.get("U", i))
        h.close()
    ens.close()


def test_tempering_toggle_and_swaps():
    import gauge_higgs_b200 as gh
    ext = [[4, 4, 4, 4]] * 4
    kappas = [0.24, 0.25, 0.26, 0.27]
    mk = lambda: gh.Ensemble(ext, gh.FundamentalRep(2), seeds=[1, 2, 3, 4], beta=2.3, kappa=kappas, lam=0.5,
                             nmd=10, precision="fp32")
    a = mk()
    a.hot(0.8)
    a.phi_gaussian(12345, 0.3)
    ra = a.run(20)
    b = mk()
    b.hot(0.8)
    b.phi_gaussian(12345, 0.3)
    b.enable_tempering(False)
    rb = b.run(20)
    assert np.array_equal(ra["dH"], rb["dH"])     # toggle off: bit-identical to no tempering
    c = mk()
    c.hot(0.8)
    c.phi_gaussian(12345, 0.3)
    c.enable_tempering(True, swap_seed=0x5A7AB1EC)
    c.run(60)
    att, acc, kap = c.tempering_stats()
    assert att.sum() > 0 and acc.sum() > 0
    assert sorted(np.round(kap, 12).tolist()) == sorted(kappas)   # a permutation of the ladder
    for x in (a, b, c):
        x.close()


def _temper_ensemble(tempered, ntraj, seed0=31, precision="fp64"):
    import gauge_higgs_b200 as gh
    ext = [[4, 4, 4, 4]] * 4
    kappas = [0.20, 0.235, 0.27, 0.305]     # across the SU(2) transition at beta = 2.3, lambda = 0.5
    e = gh.Ensemble(ext, gh.FundamentalRep(2), seeds=[seed0 + i for i in range(4)], beta=2.3, kappa=kappas, lam=0.5,
                    nmd=10, precision=precision)
    e.hot(0.8)
    e.phi_gaussian(12345, 0.3)
    if tempered:
        e.enable_tempering(True, swap_seed=0x5A7AB1EC)
    rec = e.run(ntraj)
    e.close()
    return kappas, rec


def test_tempering_swaps_replayed_on_host():
    """Every swap decision of the device pass, replayed on the host from the trajectory
    records: ladder order, even then odd pairs, Delta = (k_i - k_j)(B_i - B_j) with
    B = 2 V D L_link, acceptance min(1, exp(-Delta)) with the swap stream
    uniform(seed, key(0x57A9, attempt)) (src/hmc/replica_tempering.hpp:157-205)."""
    import math
    from gauge_higgs_b200._lib import LIB
    kappas, rec = _temper_ensemble(True, 400)
    V, D, seed = 4 ** 4, 4, 0x5A7AB1EC
    kap = np.array(kappas)                         # kappa of each lattice before the first pass
    assert np.array_equal(rec[0]["kappa"], kap)
    attempt = 0
    nswaps = 0
    for t in range(len(rec) - 1):
        B = 2.0 * rec[t]["L_link"] * float(V) * D
        order = list(np.argsort(kap, kind="stable"))
        for start in (0, 1):
            for k in range(start, 3, 2):
                li, lj = order[k], order[k + 1]
                delta = (kap[li] - kap[lj]) * (B[li] - B[lj])
                attempt += 1
                acc = delta <= 0.0 or LIB.gh_rng_uniform(seed, LIB.gh_rng_key(0x57A9, attempt, 0, 0, 0)) < math.exp(-delta)
                if acc:
                    kap[li], kap[lj] = kap[lj], kap[li]
                    order[k], order[k + 1] = lj, li
                    nswaps += 1
        assert np.array_equal(rec[t + 1]["kappa"], kap), t
    assert 0 < nswaps < attempt


def test_tempering_is_canonical():
    """kappa tempering leaves every rung's distribution unchanged: <L_link> and <L_phi>
    per kappa from the tempered ensemble agree with independent chains at fixed kappa
    (binned errors, 4.5 sigma)."""
    from gauge_higgs_b200.stats import Stats
    n, nth = 6000, 300
    kappas, rt = _temper_ensemble(True, n + nth, seed0=31)
    _, ru = _temper_ensemble(False, n + nth, seed0=71)
    rt, ru = rt[nth:], ru[nth:]
    worst = 0.0
    for i, k in enumerate(kappas):
        for obs in ("L_link", "L_phi"):
            xt = rt[obs][rt["kappa"] == k]        # every trajectory run at this kappa, whichever lattice held it
            xu = ru[obs][:, i]
            assert len(xt) == n
            st, su = Stats(xt.astype(float)), Stats(xu.astype(float))
            z = (st.mean() - su.mean()) / np.hypot(st.binned_error(), su.binned_error())
            worst = max(worst, abs(z))
    assert worst < 4.5, worst


def _beta_ensemble(tempered, ntraj, seed0=11, n_sweep=1, higgs=True, precision="fp64"):
    import gauge_higgs_b200 as gh
    ext = [[4, 4, 4, 4]] * 4
    betas = [2.2, 2.25, 2.3, 2.35]
    rep = gh.FundamentalRep(2) if higgs else None
    e = gh.Ensemble(ext, rep, seeds=[seed0 + 1000003 * i for i in range(4)], N=2, beta=betas, kappa=0.25, lam=0.5,
                    nmd=10, precision=precision)
    e.hot(0.8)
    if higgs:
        e.phi_gaussian(12345, 0.3)
    if tempered:
        e.enable_tempering(True, swap_seed=0x5A7AB1EC, coupling="beta")
        e.set_temper_interval(n_sweep)
    rec = e.run(ntraj)
    e.close()
    return betas, rec


@pytest.mark.parametrize("n_sweep,higgs", [(1, True), (2, False)])
def test_beta_tempering_replayed_on_host(n_sweep, higgs):
    """The reference's tempering (src/hmc/replica_tempering.hpp:157-205): beta ladder,
    Delta = (beta_i - beta_j)(P_i - P_j), P = n_plaq (plaquette - 1), one even + odd
    pass after every n_sweep trajectories, coin uniform(key(0x57A9, ++counter)) --
    every decision replayed on the host from the trajectory records."""
    import math
    from gauge_higgs_b200._lib import LIB
    betas, rec = _beta_ensemble(True, 300, n_sweep=n_sweep, higgs=higgs)
    nplaq, seed = 4 ** 4 * 6, 0x5A7AB1EC
    b = np.array(betas)
    assert np.array_equal(rec[0]["beta"], b)
    attempt = nswaps = 0
    for t in range(len(rec) - 1):
        if (t + 1) % n_sweep == 0:
            P = nplaq * (rec[t]["plaquette"] - 1.0)
            order = list(np.argsort(b, kind="stable"))
            for start in (0, 1):
                for k in range(start, 3, 2):
                    li, lj = order[k], order[k + 1]
                    delta = (b[li] - b[lj]) * (P[li] - P[lj])
                    attempt += 1
                    if delta <= 0.0 or LIB.gh_rng_uniform(seed, LIB.gh_rng_key(0x57A9, attempt, 0, 0, 0)) < math.exp(-delta):
                        b[li], b[lj] = b[lj], b[li]
                        order[k], order[k + 1] = lj, li
                        nswaps += 1
        assert np.array_equal(rec[t + 1]["beta"], b), t
    assert 0 < nswaps < attempt


def test_beta_tempering_is_canonical():
    """Per-beta <plaquette> and <L_link> of the tempered ensemble equal those of
    independent fixed-beta chains (binned errors, 4.5 sigma) -- the property that
    test/test_replica_tempering_canonical.cpp checks for the reference."""
    from gauge_higgs_b200.stats import Stats
    n, nth = 5000, 300
    betas, rt = _beta_ensemble(True, n + nth, seed0=21)
    _, ru = _beta_ensemble(False, n + nth, seed0=71)
    rt, ru = rt[nth:], ru[nth:]
    worst = 0.0
    for i, bv in enumerate(betas):
        for obs in ("plaquette", "L_link"):
            xt = rt[obs][rt["beta"] == bv]
            xu = ru[obs][:, i]
            assert len(xt) == n
            st, su = Stats(xt.astype(float)), Stats(xu.astype(float))
            worst = max(worst, abs(st.mean() - su.mean()) / np.hypot(st.binned_error(), su.binned_error()))
    assert worst < 4.5, worst


# ---------------------------------------------------------------------------
# kick tiles: results are independent of the block shape; the autotuner picks one
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_kick_tiles_bit_identical(precision):
    import gauge_higgs_b200 as gh
    L = [8, 6, 4, 6]
    h = gh.GaugeHiggsHMC(L, gh.FundamentalRep(3), seed=4, precision=precision, beta=5.7, kappa=0.1, lam=0.5)
    h.hot(0.8)
    h.phi_gaussian(12345, 0.3)
    h.refresh_momenta()
    P0, pi0 = h.P, h.pi
    outs = []
    for tile in ([8, 4, 4, 1], [4, 4, 4, 2], [2, 2, 2, 16], [1, 1, 1, 1], [8, 8, 2, 1]):
        h.set_tile(tile)
        assert h.get_tile() == tile
        h.P = P0
        h.pi = pi0
        h.kick(0.05)
        outs.append((h.P, h.pi))
    for P, pi in outs[1:]:
        assert np.array_equal(P, outs[0][0]) and np.array_equal(pi, outs[0][1])
    ms = h.autotune(reps=2)
    t = h.get_tile()
    assert ms > 0 and int(np.prod(t)) <= 128 and all(x & (x - 1) == 0 for x in t)
    h.close()


def test_large_single_row_irrep_su2_spin6():
    """SU(2) {12} (d = 13, N^n = 4096): the reference's GeneralRep fast-path case
    (src/rep/rep_general.hpp:161-179).  The engine applies the exact tensor path
    (fewer warps per block so the 4096-entry buffer fits in shared memory); its
    forces match the oracle's tensor path and finite differences of the action."""
    import gauge_higgs_b200 as gh
    from oracle.oracle import Oracle, REP_GENERAL
    orc = Oracle()
    rep = gh.GeneralRep(2, [12])
    D, N, L = 3, 2, [3, 2, 2]
    h = gh.GaugeHiggsHMC(L, rep, seed=2, beta=2.3, kappa=0.2, lam=0.5, nmd=6)
    h.hot(0.6)
    h.phi_gaussian(3, 0.4)
    U, phi = h.U, h.phi
    orep = orc.rep(REP_GENERAL, N, rep.d, 0, rep.n_boxes, rep.dimT, rep.T, rep.W)
    Fm = orc.matter_force(D, N, L, orep, U, phi, 0.2)
    Fs = orc.scalar_force(D, N, L, orep, U, phi, 0.2, 0.5)
    assert np.abs(h.matter_link_force() - Fm).max() < 1e-12 * np.abs(Fm).max()
    assert np.abs(h.scalar_force() - Fs).max() < 1e-12 * np.abs(Fs).max()
    assert abs(h.measure()["S_H"] - orc.scalar_action(D, N, L, orep, U, phi, 0.2, 0.5)) < 1e-10
    h.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_nonfinite_hamiltonian_is_rejected_and_counted(precision):
    """Failure injected on the host: an overflowing coupling makes H infinite, so
    dH = inf - inf is NaN.  The device Metropolis step rejects it (every comparison
    with NaN is false, as in the reference), counts it, and restores the fields;
    the chain then continues normally."""
    import gauge_higgs_b200 as gh
    h = gh.GaugeHiggsHMC([4, 4, 4, 4], gh.FundamentalRep(2), seed=9, precision=precision, beta=2.3, kappa=0.2,
                         lam=0.5, nmd=8)
    h.hot(0.5)
    h.phi_gaussian(12345, 0.3)
    h.run(2)
    U0, phi0 = h.U, h.phi
    h.lam = 1e308
    dH, acc = gh.Ensemble.trajectory(h)
    assert np.isnan(dH[0]) and not acc[0]
    assert np.array_equal(h.U, U0) and np.array_equal(h.phi, phi0)
    t, a, nonfinite = h.traj_counts(0)
    assert t == 3 and nonfinite == 1
    h.lam = 0.5
    rec = h.run(5)[:, 0]
    assert np.all(np.isfinite(rec["dH"]))
    assert h.traj_counts(0)[2] == 1
    h.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_trajectory_host_matches_device_chain(precision):
    """gh_trajectory_host (fields in host memory, uploaded and downloaded every
    trajectory; not downloaded after a rejection, which restores the uploaded state)
    against the same chain kept on the device: identical records, identical fields
    (FP32-MD: identical after rounding to FP32)."""
    import gauge_higgs_b200 as gh
    hs = []
    for _ in range(2):
        h = gh.GaugeHiggsHMC([4, 4, 4, 4], gh.FundamentalRep(3), seed=11, precision=precision, beta=5.7, kappa=0.1,
                             lam=0.5, nmd=4)
        h.hot(0.8)
        h.phi_gaussian(12345, 0.3)
        hs.append(h)
    hA, hB = hs
    U = np.ascontiguousarray(hA.U)
    phi = np.ascontiguousarray(hA.phi)
    recs = [hA.trajectory_host(U, phi) for _ in range(12)]
    rB = hB.run(12)[:, 0]
    assert [int(r.accepted) for r in recs] == [int(x) for x in rB["accepted"]]
    assert np.array_equal(np.array([r.dH for r in recs]), rB["dH"])
    if precision == "fp64":
        assert np.array_equal(U, hB.U) and np.array_equal(phi, hB.phi)
    else:
        assert np.array_equal(U.astype(np.complex64), hB.U.astype(np.complex64))
        assert np.array_equal(phi.astype(np.complex64), hB.phi.astype(np.complex64))
    hA.close()
    hB.close()


def test_contexts_on_concurrent_streams_match_sequential():
    """Independent contexts share no device state: two ensembles enqueued at once on two
    CUDA streams give bit for bit the records and fields of running them one after the
    other on their own streams."""
    import torch
    import gauge_higgs_b200 as gh

    def make(kappa0):
        ens = gh.Ensemble([[4, 4, 4, 4], [4, 4, 2, 6]], gh.FundamentalRep(2), seeds=[3, 4], precision="fp32",
                          beta=2.3, kappa=[kappa0, kappa0 + 0.02], lam=0.5, nmd=8)
        ens.hot(0.6)
        ens.phi_gaussian(12345, 0.4)
        return ens

    ref = []
    for k0 in (0.2, 0.25):
        e = make(k0)
        ref.append(e.run(6))
        e.close()
    a, b = make(0.2), make(0.25)
    sa, sb = torch.cuda.Stream(), torch.cuda.Stream()
    a.set_stream(sa.cuda_stream)
    b.set_stream(sb.cuda_stream)
    a.enqueue(6)
    b.enqueue(6)
    torch.cuda.synchronize()
    for e, rec in zip((a, b), ref):
        got = e.records(6)
        for k in ("dH", "accepted", "plaquette", "L_phi", "L_link"):
            assert np.array_equal(got[k], rec[k]), k
    a.close()
    b.close()
