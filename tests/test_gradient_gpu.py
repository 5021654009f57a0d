"""Energy gradients through the adjoint of the apply (the differentiation form): dE/d scale of every MPO entry
from the single-site adjoint at every site (the orthogonality centre moved through the MPS), and dE/dh, dE/dV
through the QC MPO's integral provenance.  Checked against the exact FCI density matrices, the expectation-value
measurements (the oneptdm / twoptdm counterparts), the Euler identities of the energy (linear in the integrals,
and in each site tensor of the MPO) and central finite differences of FCI energies."""
import numpy as np
import pytest

from oracle.fci import FCI

from helpers import gauge_signed, qc_system

pytestmark = pytest.mark.gpu


def orbit_mean(X):
    """Average over the 8 index permutations of real (pq|rs)."""
    perms = [X, X.transpose(1, 0, 2, 3), X.transpose(0, 1, 3, 2), X.transpose(1, 0, 3, 2),
             X.transpose(2, 3, 0, 1), X.transpose(3, 2, 0, 1), X.transpose(2, 3, 1, 0), X.transpose(3, 2, 1, 0)]
    return sum(perms) / 8.0


def fci_rdms(h, V, e, n):
    f = FCI(h, V, e, n, n)
    w, Z = np.linalg.eigh(f.dense())
    c = Z[:, 0]
    L = h.shape[0]
    Ec = [[f.E[p][q] @ c for q in range(L)] for p in range(L)]
    g1 = np.array([[c @ Ec[p][q] for q in range(L)] for p in range(L)])
    G = np.zeros((L,) * 4)
    for p in range(L):
        for q in range(L):
            for r in range(L):
                for s in range(L):
                    G[p, q, r, s] = 0.5 * (Ec[q][p] @ Ec[r][s] - (g1[p, s] if q == r else 0.0))
    return w[0], g1, orbit_mean(G)


def test_integral_gradient_is_the_fci_density_matrix(gpu_ctx):
    """L=6 at a bond dimension where the MPS is exact: dE/dh is the FCI 1-RDM, dE/dV averaged over the
    integral symmetry is the FCI two-body gradient, both equal the expectation-value measurements, and
    sum h dh + sum V dV + ecore is the energy."""
    from qcmaquis_b200.dmrg import DMRG
    L, M = 6, 64
    h, V, e, m, ts, blob = qc_system(L)
    E_fci, g1, G_fci = fci_rdms(h, V, e, L // 2)
    d = DMRG(gpu_ctx, m, L // 2, L // 2, M, ecore=e)
    for _ in range(4):
        E, _ = d.sweep()
    assert abs(E.min() - E_fci) < 1e-9
    dh, dV = d.integral_gradient(h, V)
    assert np.abs(dh - g1).max() < 1e-8, np.abs(dh - g1).max()
    assert np.abs(orbit_mean(dV) - G_fci).max() < 1e-8
    assert abs(np.sum(h * dh) + np.sum(V * dV) + e - E_fci) < 1e-9
    assert np.abs(dh - d.measure_1rdm()).max() < 1e-10
    assert np.abs(orbit_mean(dV) - d.measure_2rdm_grad()).max() < 1e-10
    # central differences of FCI energies along a random direction of both integral sets (symmetric, as
    # the FCI Hamiltonian reads them)
    rng = np.random.default_rng(7)
    Dh = rng.standard_normal((L, L))
    Dh = Dh + Dh.T
    DV = orbit_mean(rng.standard_normal((L,) * 4))
    eps = 1e-5
    ep = np.linalg.eigvalsh(FCI(h + eps * Dh, V + eps * DV, e, L // 2, L // 2).dense())[0]
    em = np.linalg.eigvalsh(FCI(h - eps * Dh, V - eps * DV, e, L // 2, L // 2).dense())[0]
    fd = (ep - em) / (2 * eps)
    an = np.sum(Dh * dh) + np.sum(DV * dV)
    assert abs(fd - an) <= 1e-6 * abs(fd), (fd, an)


@pytest.mark.parametrize("gauge", [None, 3])
def test_mpo_gradient_site_identities(gpu_ctx, gauge):
    """L=8, M=24 (a truncated MPS): for every site k, sum_e scale_e dE/d scale_e over W[k]'s entries is the
    energy of the MPS (E is linear in each site tensor of the MPO), the same for every site, and the same as
    the integral Euler sum; with the MPO's Hermitian pairs and a sign gauge on the bond indices."""
    from qcmaquis_b200.dmrg import DMRG
    L, M = 8, 24
    h, V, e, m, ts, blob = qc_system(L, gauge=gauge)
    d = DMRG(gpu_ctx, m, L // 2, L // 2, M)
    for _ in range(2):
        d.sweep()
    grads = d.mpo_gradient(m)
    sums = np.array([np.dot(m.terms(k)["scale"], grads[k]) for k in range(L)])
    assert np.abs(sums - sums[0]).max() < 1e-11 * abs(sums[0]), sums
    dh, dV = d.integral_gradient(h, V)
    assert abs(np.sum(h * dh) + np.sum(V * dV) - sums[0]) < 1e-11 * abs(sums[0])
    assert np.abs(dh - d.measure_1rdm()).max() < 1e-10
    assert abs(np.trace(dh) - L) < 1e-9


def test_ladder_densities_from_the_adjoint(gpu_ctx):
    """The reference's own ladder local densities (test_fermiladder_ts.py, 'Local density up/down'; N_up =
    N_down, tolerance 1e-3 there) from dE/dh_ii of the adjoint gradient of the device MPS."""
    import json
    import os
    from qcmaquis_b200.dmrg import DMRG
    from qcmaquis_b200.fcidump import hubbard_ladder_integrals
    from qcmaquis_b200.mpo import MPO
    golden = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))
    h, V, e = hubbard_ladder_integrals(6)
    dev = DMRG(gpu_ctx, MPO.qc(h, V), 10, 10, 400, init_bond_dimension=5)
    for _ in range(3):
        dev.sweep()
    dh, _ = dev.integral_gradient(h, V, with_V=False)
    n_spin = np.diag(dh) / 2
    for spin in ("up", "down"):
        dref = np.array(golden[f"hubbard_ladder_6x2_local_density_{spin}_reference"])
        assert np.abs(n_spin - dref).max() < 1e-6, (n_spin, dref)
    assert np.abs(dh - dev.measure_1rdm()).max() < 1e-10
