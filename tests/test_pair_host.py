"""The identities behind the two-slot register path (k_gen_pair), checked on the host
with the library's own irrep tables (gh_rep_general_build, the reference's basis
construction, src/rep/rep_general.hpp:54-84,338-411):

* every basis vector W_b, read as an N x N matrix (tensor index i*N + j), is symmetric
  ({2}) or antisymmetric ({1,1});
* the reference's tensor apply D = conj(W) (U (x) U) W^T equals lift / U Phi U^T /
  project, and D^dag the same with U^dag Phi conj(U);
* the generators T^a_R are conj(W) (T^a (x) 1 + 1 (x) T^a) W^T;
* phi_x^dag T^a_R D phi_y = 2 Tr(T^a Psi Phi_x^dag), Psi = U Phi_y U^T, so the matter
  force is 4 kappa Im Tr(T^a Psi Phi_x^dag)."""
import numpy as np
import pytest


def su3(rng):
    A = rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3))
    H = (A + A.conj().T) / 2
    w, v = np.linalg.eigh(H)
    U = v @ np.diag(np.exp(1j * w)) @ v.conj().T
    return U / np.linalg.det(U) ** (1 / 3)


@pytest.mark.parametrize("rows,sign", [([2], 1), ([1, 1], -1)])
def test_two_slot_identities(rows, sign):
    import gauge_higgs_b200 as gh
    rng = np.random.default_rng(3)
    rep = gh.GeneralRep(3, rows)
    d = rep.d
    W = np.asarray(rep.W).reshape(d, 9)
    T = np.asarray(rep.T).reshape(8, d, d)
    for b in range(d):
        M = W[b].reshape(3, 3)
        assert np.abs(M - sign * M.T).max() < 1e-14
    Tf = np.asarray(gh.GeneralRep(3, [1]).T).reshape(8, 3, 3)
    Wf = np.asarray(gh.GeneralRep(3, [1]).W).reshape(3, 3)
    Tg = np.array([Wf.T @ Tf[a] @ Wf.conj() for a in range(8)])     # the fundamental generators
    TR = np.array([W.conj() @ (np.kron(Tg[a], np.eye(3)) + np.kron(np.eye(3), Tg[a])) @ W.T for a in range(8)])
    assert np.abs(TR - T).max() < 1e-13
    for _ in range(20):
        U = su3(rng)
        D = W.conj() @ np.kron(U, U) @ W.T
        phy = rng.normal(size=d) + 1j * rng.normal(size=d)
        phx = rng.normal(size=d) + 1j * rng.normal(size=d)
        Phy, Phx = (phy @ W).reshape(3, 3), (phx @ W).reshape(3, 3)
        Psi = U @ Phy @ U.T
        assert np.abs(D @ phy - W.conj() @ Psi.reshape(9)).max() < 1e-13
        assert np.abs(D.conj().T @ phx - W.conj() @ (U.conj().T @ Phx @ U.conj()).reshape(9)).max() < 1e-13
        lhs = np.array([phx.conj() @ T[a] @ (D @ phy) for a in range(8)])
        rhs = np.array([2 * np.trace(Tg[a] @ Psi @ Phx.conj().T) for a in range(8)])
        assert np.abs(lhs - rhs).max() < 1e-13
