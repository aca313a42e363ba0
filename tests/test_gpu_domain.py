"""Domain decomposition on the device (gh_set_domain, gh_halo_pack/unpack and
gauge_higgs_b200.domain.DomainHMC) against one undivided lattice: the property the
reference prints for its MPI drivers ("identical for any procgrid",
src/mpi/gh_higgs_mpi.cpp:81) -- hot start and scalar initialisation equal the whole
lattice's draws bit for bit, the forces on every interior link equal, and a run of
trajectories takes the same accept decisions with the same fields (only dH's global
sum is ordered differently).  All subdomains run in one process on one GPU
(InProcessTransport); none of their kernels waits for another's."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_halo_pack_order_matches_host_planes():
    import torch
    import ctypes as C
    import gauge_higgs_b200 as gh
    from gauge_higgs_b200._lib import LIB
    from gauge_higgs_b200.domain import Subdomain
    p = Subdomain([4, 4, 4, 6], [1, 1, 2, 2], [1, 0, 1, 1])
    h = gh.GaugeHiggsHMC(p.L, gh.FundamentalRep(3), seed=1)
    ia = lambda v: (C.c_int * 4)(*v)
    assert LIB.gh_set_domain(h.ctx.h, 0, ia(p.G), ia(p.lo), ia(p.hi), ia(p.goff)) == 0
    V = p.V
    U = (np.arange(V)[:, None, None, None] + 1j * np.arange(36).reshape(1, 4, 3, 3)).astype(np.complex128)
    phi = (np.arange(V)[:, None] * 0.5 + 1j * np.arange(3)[None, :]).astype(np.complex128)
    for field, F, ncomp in ((0, U.reshape(V, 36), 36), (1, phi, 3)):
        for nu in p.split_dirs:
            h.U = U                   # the unpack below overwrites a plane
            h.phi = phi
            n = C.c_longlong()
            assert LIB.gh_halo_count(h.ctx.h, 0, field, nu, C.byref(n)) == 0
            sites = p.plane_sites(nu, 1)
            assert n.value == len(sites) * ncomp
            buf = torch.zeros(2 * n.value, dtype=torch.float64, device="cuda")
            assert LIB.gh_halo_pack(h.ctx.h, 0, field, nu, 1, buf.data_ptr()) == 0
            h.sync()
            got = buf.cpu().numpy().view(np.complex128).reshape(ncomp, len(sites))
            assert np.array_equal(got, F[sites].T)
            # unpack into layer 0 and read it back
            assert LIB.gh_halo_unpack(h.ctx.h, 0, field, nu, 0, buf.data_ptr()) == 0
            back = (h.U.reshape(V, 36) if field == 0 else h.phi)[p.plane_sites(nu, 0)]
            assert np.array_equal(back, F[sites])
    h.close()


def _whole(G, rep, N, precision, seed, beta, kappa, lam, nmd, integ):
    import gauge_higgs_b200 as gh
    if rep is None:
        return gh.GaugeHMC(G, N, seed=seed, precision=precision, beta=beta, nmd=nmd, integ=integ)
    return gh.GaugeHiggsHMC(G, rep, seed=seed, precision=precision, beta=beta, kappa=kappa, lam=lam, nmd=nmd,
                            integ=integ)


CASES = [("fund3", [4, 4, 4, 6], [1, 1, 1, 2], "fp64"), ("fund3", [4, 4, 4, 6], [1, 1, 2, 2], "fp64"),
         ("fund3", [4, 4, 4, 6], [1, 1, 2, 2], "fp32"), ("none2", [4, 4, 6, 4], [1, 2, 3, 1], "fp64"),
         ("adj2", [4, 4, 4, 4], [2, 1, 1, 2], "fp64"), ("27plet", [2, 2, 3, 4], [1, 1, 1, 2], "fp64"),
         ("sextet", [2, 2, 3, 4], [1, 1, 1, 2], "fp64")]


@pytest.mark.parametrize("kind,G,P,precision", CASES)
def test_decomposed_run_equals_whole_lattice(kind, G, P, precision):
    import gauge_higgs_b200 as gh
    from gauge_higgs_b200.domain import DomainHMC, InProcessTransport
    N = 2 if kind.endswith("2") else 3
    rep = {"fund3": gh.FundamentalRep(3), "none2": None, "adj2": gh.AdjointRep(2),
           "27plet": gh.GeneralRep(3, [4, 2], real=True), "sextet": gh.GeneralRep(3, [2])}[kind]
    beta, kappa, lam, nmd = (5.7, 0.1, 0.5, 6) if N == 3 else (2.3, 0.2, 0.5, 8)
    whole = _whole(G, rep, N, precision, 7, beta, kappa, lam, nmd, "omelyan")
    tr = InProcessTransport(G, P)
    dom = DomainHMC(G, tr, rep=rep, N=N, seed=7, precision=precision, beta=beta, kappa=kappa, lam=lam, nmd=nmd)
    for h in (whole, dom):
        h.hot(0.8)
        if rep is not None:
            h.phi_gaussian(12345, 0.3)
    dom.exchange()
    # every stored site of every subdomain (halos included) holds the whole lattice's value
    Uw = whole.U.reshape(int(np.prod(G)), -1)
    phw = whole.phi if rep is not None else None
    for p, h in zip(tr.local_parts(), dom.h):
        g = p.global_site(np.arange(p.V))
        assert np.array_equal(h.U.reshape(p.V, -1), Uw[g])
        if rep is not None:
            assert np.array_equal(h.phi, phw[g])
    # forces on the interior links
    Fw = whole.gauge_force() + (whole.matter_link_force() if rep is not None else 0)
    Fw = Fw.reshape(int(np.prod(G)), -1)
    for p, h in zip(tr.local_parts(), dom.h):
        s, g = p.interior_sites()
        F = (h.gauge_force() + (h.matter_link_force() if rep is not None else 0)).reshape(p.V, -1)
        assert np.abs(F[s] - Fw[g]).max() <= 1e-13 * max(1.0, np.abs(Fw).max())
    # a run of trajectories: the same decisions and fields
    m0, mw = dom.measure(), whole.measure()
    assert abs(m0["plaquette"] - mw["plaquette"]) < 1e-13
    assert abs(m0["H"] - mw["H"]) < 1e-12 * abs(mw["H"])
    for t in range(4):
        acc_w = whole.trajectory()
        acc_d = dom.trajectory()
        assert acc_w == acc_d, t
        assert abs(dom.last_dH - whole.last_dH) < 1e-9 * max(1.0, abs(mw["H"])) + 1e-9, (dom.last_dH, whole.last_dH)
    m1, mw1 = dom.measure(), whole.measure()
    for k in ("plaquette",) + (("L_link", "L_phi") if rep is not None else ()):
        assert abs(m1[k] - mw1[k]) < 1e-12, (k, m1[k], mw1[k])
    assert dom.acceptance() == whole.acceptance()
    dom.close()
    whole.close()


def test_device_metropolis_is_refused_on_a_subdomain():
    import gauge_higgs_b200 as gh
    from gauge_higgs_b200.domain import DomainHMC, InProcessTransport
    dom = DomainHMC([4, 4, 4, 6], InProcessTransport([4, 4, 4, 6], [1, 1, 1, 2]), rep=gh.FundamentalRep(3), seed=1)
    with pytest.raises(gh.GaugeHiggsError):
        dom.h[0].trajectory()
    dom.close()


def test_mpi_driver_output_does_not_depend_on_the_grid():
    """gauge_higgs_b200.mpi_driver (src/mpi/gh_higgs_mpi.cpp's command line) in one
    process: the hot and measured plaquette, L_link, L_phi lines agree for the undivided
    grid and a 2 x 2 split."""
    import re
    import subprocess
    import sys
    from conftest import ROOT
    out = {}
    for grid in ("1,1,1,1", "1,1,2,2"):
        r = subprocess.run([sys.executable, "-m", "gauge_higgs_b200.mpi_driver", "fund", "4", grid, "2.3", "0.2", "0.5",
                            "3", "4", "10", "1.0", "1"], capture_output=True, text=True, cwd=ROOT, timeout=300)
        assert r.returncode == 0, r.stderr
        out[grid] = [float(x) for x in re.findall(r"=(-?[0-9]+\.[0-9]+)", "\n".join(
            ln for ln in r.stdout.splitlines() if ln.startswith(("hot:", "meas:", "acceptance"))))]
    assert len(out["1,1,1,1"]) == 8
    assert np.allclose(out["1,1,1,1"], out["1,1,2,2"], rtol=0, atol=2e-10), out
