"""FP64 parity with the reference itself at the benchmark configurations' sizes.

The reference's own code (its headers compiled unmodified into oracle/_ref) and
the device path through the C ABI start from identical fields and momenta:

  * SU(3) + fundamental Higgs on 16^4 (beta 5.7, kappa 0.10, lambda 0.5), with the
    kick tile the autotuner picks and with one fixed tile;
  * SU(3) 12^4 with the sextet {2}, the octet {2,1}:real and the 27-plet
    {4,2}:real (beta 5.7, kappa 0.1, lambda 0.5), the scalar field initialised as
    the reference driver does (Gaussian, sigma 0.3, stream 12345).

Compared (FP64 mode): the gauge, matter-link and scalar forces; one kick; one
drift; a two-step MD evolution; dH of a short trajectory from identical momenta.
Gates: forces, one kick and one drift 1e-12 relative to the largest entry; MD
fields 1e-11; dH within 1e-12 |H| (the reference sums H with an OpenMP
reduction).  The FP32-MD force and one-step errors against the FP64 reference
at 16^4 are printed and bounded.  The MD steps use eps = 1/16, the benchmark's
step (tau 1, nmd 16); the trajectory is two Omelyan steps of that size.

References: src/action/gauge_wilson.hpp:70-83, src/action/scalar_higgs.hpp:71-128,
src/rep/rep_general.hpp:196-220, src/hmc/gauge_higgs_hmc.hpp:112-192.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL = 1e-12
EPS = 1.0 / 16


def rel_err(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


@pytest.fixture(scope="module")
def ref():
    from oracle.oracle import Reference, have_reference
    if not have_reference():
        pytest.fail("oracle/_ref/libghref.so (the reference harness) is not built")
    r = Reference()
    r.set_threads(os.cpu_count() or 1)
    return r


def device_rep(ref, N, spec):
    import gauge_higgs_b200 as gh
    if spec == "fund":
        return gh.FundamentalRep(N)
    T, W, info = ref.rep_tables(N, spec)
    rows = [int(t) for t in spec.split(":")[0].split(",")]
    return gh.GeneralRep(N, rows, real=bool(info["real"]), T=T, W=W)


def start_state(ref, D, N, L, spec, rep):
    U = ref.hot_start(D, N, L, 1, 0.8)
    phi = ref.phi_gaussian(D, L, rep.d, 1, 12345, int(rep.real), 0.3)
    return U, phi


def check_config(ref, D, N, L, spec, beta, kappa, lam, tile=None, integ_nmd=2):
    import gauge_higgs_b200 as gh
    from oracle.oracle import OMELYAN
    rep = device_rep(ref, N, spec)
    U, phi = start_state(ref, D, N, L, spec, rep)
    h = gh.GaugeHiggsHMC(L, rep, seed=1, beta=beta, kappa=kappa, lam=lam, nmd=integ_nmd, tau=integ_nmd * EPS,
                         integ="omelyan")
    if tile == "auto":
        h.autotune(reps=2)
    elif tile is not None:
        h.set_tile(tile)
    h.U = U
    h.phi = phi
    out = {}
    out["gauge_force"] = rel_err(h.gauge_force(), ref.gauge_force(D, N, L, U, beta))
    out["matter_force"] = rel_err(h.matter_link_force(), ref.matter_force(D, N, L, spec, U, phi, kappa))
    out["scalar_force"] = rel_err(h.scalar_force(), ref.scalar_force(D, N, L, spec, U, phi, kappa, lam))
    # identical momenta: the device's heatbath, handed to the reference
    h.refresh_momenta()
    P, pi = h.P, h.pi
    kw = dict(seed=1, beta=beta, kappa=kappa, lam=lam, tau=integ_nmd * EPS, nmd=integ_nmd, integ=OMELYAN)

    def state():
        return dict(U=U.copy(), P=P.copy(), phi=phi.copy(), pi=pi.copy())

    def load(st):
        h.U, h.P, h.phi, h.pi = st["U"], st["P"], st["phi"], st["pi"]

    # one kick
    st = state()
    ref.hmc_op("kick", D, N, L, spec, st, eps=EPS, **kw)
    load(state())
    h.kick(EPS)
    out["kick_P"] = rel_err(h.P, st["P"])
    out["kick_pi"] = rel_err(h.pi, st["pi"])
    # one drift
    st = state()
    ref.hmc_op("drift", D, N, L, spec, st, eps=EPS, **kw)
    load(state())
    h.drift(EPS)
    out["drift_U"] = rel_err(h.U, st["U"])
    out["drift_phi"] = rel_err(h.phi, st["phi"])
    # a two-step Omelyan MD evolution
    st = state()
    ref.hmc_op("md_evolve", D, N, L, spec, st, **kw)
    load(state())
    h.md_evolve()
    out["md_U"] = rel_err(h.U, st["U"])
    out["md_P"] = rel_err(h.P, st["P"])
    out["md_phi"] = rel_err(h.phi, st["phi"])
    out["md_pi"] = rel_err(h.pi, st["pi"])
    # dH of the trajectory's deterministic part (H_i, MD, reunitarisation, H_f)
    st = state()
    Hi = ref.hmc_op("hamiltonian", D, N, L, spec, st, **kw)[0]
    ref.hmc_op("md_evolve", D, N, L, spec, st, **kw)
    ref.hmc_op("reunitarize", D, N, L, spec, st, **kw)
    dH_ref = ref.hmc_op("hamiltonian", D, N, L, spec, st, **kw)[0] - Hi
    load(state())
    Hi_d = h.hamiltonian()
    h.md_evolve()
    h.reunitarize_all()
    dH_dev = h.hamiltonian() - Hi_d
    out["H_i"] = abs(Hi_d - Hi) / abs(Hi)
    out["dH_dev"], out["dH_ref"], out["dH_gap_over_H"] = dH_dev, dH_ref, abs(dH_dev - dH_ref) / abs(Hi)
    out["tile"] = h.get_tile()
    h.close()
    print(f"\n{spec} {L}: " + ", ".join(f"{k} {v:.3g}" if isinstance(v, float) else f"{k} {v}" for k, v in out.items()))
    for k in ("gauge_force", "matter_force", "scalar_force", "kick_P", "kick_pi", "drift_U", "drift_phi", "H_i"):
        assert out[k] < REL, (k, out[k])
    for k in ("md_U", "md_P", "md_phi", "md_pi"):
        assert out[k] < 1e-11, (k, out[k])
    assert out["dH_gap_over_H"] < REL, out
    return out


@pytest.mark.parametrize("tile", ["auto", [8, 4, 2, 2]])
def test_su3_fund_16x4(ref, tile):
    check_config(ref, 4, 3, [16, 16, 16, 16], "fund", 5.7, 0.10, 0.5, tile=tile)


@pytest.mark.parametrize("spec", ["2", "2,1:real", "4,2:real"])
def test_su3_general_irreps_12x4(ref, spec):
    check_config(ref, 4, 3, [12, 12, 12, 12], spec, 5.7, 0.1, 0.5)


def test_fp32_md_error_against_fp64_reference_16x4(ref):
    """FP32-MD at 16^4: per-link force error and the error of one kick + drift against
    the reference's FP64 results on the same (FP32-representable) inputs."""
    import gauge_higgs_b200 as gh
    D, N, L, beta, kappa, lam = 4, 3, [16, 16, 16, 16], 5.7, 0.10, 0.5
    rep = gh.FundamentalRep(N)
    U, phi = start_state(ref, D, N, L, "fund", rep)
    U = U.astype(np.complex64).astype(np.complex128)
    phi = phi.astype(np.complex64).astype(np.complex128)
    h = gh.GaugeHiggsHMC(L, rep, seed=1, precision="fp32", beta=beta, kappa=kappa, lam=lam)
    h.autotune(reps=2)
    h.U = U
    h.phi = phi
    F = h.gauge_force() + h.matter_link_force()
    Fr = ref.gauge_force(D, N, L, U, beta) + ref.matter_force(D, N, L, "fund", U, phi, kappa)
    e_link = rel_err(F, Fr)
    e_phi = rel_err(h.scalar_force(), ref.scalar_force(D, N, L, "fund", U, phi, kappa, lam))
    h.refresh_momenta()
    P, pi = h.P, h.pi
    st = dict(U=U.copy(), P=P.copy(), phi=phi.copy(), pi=pi.copy())
    kw = dict(seed=1, beta=beta, kappa=kappa, lam=lam, tau=1.0, nmd=16)
    ref.hmc_op("kick", D, N, L, "fund", st, eps=EPS, **kw)
    ref.hmc_op("drift", D, N, L, "fund", st, eps=EPS, **kw)
    h.kick(EPS)
    h.drift(EPS)
    e_U = float(np.abs(h.U - st["U"]).max())
    e_P = rel_err(h.P, st["P"])
    h.close()
    print(f"\nFP32-MD vs FP64 reference, SU(3) fund 16^4: link force {e_link:.2e}, scalar force {e_phi:.2e}, "
          f"P after one kick {e_P:.2e}, U after kick + drift {e_U:.2e} (max abs)")
    assert e_link < 5e-6 and e_phi < 5e-6
    assert e_P < 5e-6
    assert e_U < 5e-7
