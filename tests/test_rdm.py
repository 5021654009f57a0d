"""One-particle density matrix of the device MPS (the oneptdm measurement, lib/interface/cpp_maquis.cpp:235-366)
as dE/dh_ij: expectation values of the one-body operators through left boundary steps, against the exact FCI
density matrix and central finite differences of FCI energies (Hellmann-Feynman), at a bond dimension where the
MPS is exact."""
import numpy as np
import pytest

from oracle.fci import FCI

from helpers import qc_system

pytestmark = pytest.mark.gpu


def fci_ground(h, V, e, n):
    f = FCI(h, V, e, n, n)
    w, Z = np.linalg.eigh(f.dense())
    c = Z[:, 0]
    L = h.shape[0]
    gamma = np.array([[c @ (f.E[p][q] @ c) for q in range(L)] for p in range(L)])
    return w[0], gamma


def test_1rdm_matches_fci(gpu_ctx):
    from qcmaquis_b200.dmrg import DMRG
    L, M = 6, 64
    h, V, e, m, ts, blob = qc_system(L)
    E_fci, g_fci = fci_ground(h, V, e, L // 2)
    d = DMRG(gpu_ctx, m, L // 2, L // 2, M)
    for _ in range(4):
        E, _ = d.sweep()
    assert abs(E.min() - E_fci) < 1e-9
    g = d.measure_1rdm()
    assert np.abs(g - g.T).max() < 1e-12
    assert abs(np.trace(g) - L) < 1e-9  # N electrons
    assert np.abs(g - g_fci).max() < 1e-8, np.abs(g - g_fci).max()
    # Hellmann-Feynman: dE/dh along (e_ij + e_ji) is 2 gamma_ij (gamma_ii on the diagonal)
    eps = 1e-5
    for (i, j) in ((1, 1), (0, 3), (2, 5)):
        S = np.zeros_like(h)
        S[i, j] = S[j, i] = 1.0
        ep = np.linalg.eigvalsh(FCI(h + eps * S, V, e, L // 2, L // 2).dense())[0]
        em = np.linalg.eigvalsh(FCI(h - eps * S, V, e, L // 2, L // 2).dense())[0]
        fd = (ep - em) / (2 * eps)
        assert abs(fd - (g[i, i] if i == j else 2 * g[i, j])) < 1e-6, (i, j, fd)


def orbit_mean(X):
    """Average over the 8 index permutations of real (pq|rs)."""
    perms = [X, X.transpose(1, 0, 2, 3), X.transpose(0, 1, 3, 2), X.transpose(1, 0, 3, 2),
             X.transpose(2, 3, 0, 1), X.transpose(3, 2, 0, 1), X.transpose(2, 3, 1, 0), X.transpose(3, 2, 1, 0)]
    return sum(perms) / 8.0


def test_2rdm_grad_matches_fci(gpu_ctx):
    """dE/dV_pqrs = 1/2 (<E_pq E_rs> - delta_qr <E_ps>) symmetrised over the integral symmetry (FCI vector), and
    the derivative along a random symmetric V direction against central differences of FCI energies."""
    from qcmaquis_b200.dmrg import DMRG
    L, M = 6, 64
    h, V, e, m, ts, blob = qc_system(L)
    f = FCI(h, V, e, L // 2, L // 2)
    w, Z = np.linalg.eigh(f.dense())
    c = Z[:, 0]
    Ec = [[f.E[p][q] @ c for q in range(L)] for p in range(L)]
    g1 = np.array([[c @ Ec[p][q] for q in range(L)] for p in range(L)])
    G_fci = np.zeros((L,) * 4)
    for p in range(L):
        for q in range(L):
            for r in range(L):
                for s in range(L):
                    G_fci[p, q, r, s] = 0.5 * (Ec[q][p] @ Ec[r][s] - (g1[p, s] if q == r else 0.0))
    G_fci = orbit_mean(G_fci)
    d = DMRG(gpu_ctx, m, L // 2, L // 2, M)
    for _ in range(4):
        E, _ = d.sweep()
    assert abs(E.min() - w[0]) < 1e-9
    G = d.measure_2rdm_grad()
    assert np.abs(G - G_fci).max() < 1e-8, np.abs(G - G_fci).max()
    D = orbit_mean(np.random.default_rng(4).standard_normal((L,) * 4))
    eps = 1e-5
    ep = np.linalg.eigvalsh(FCI(h, V + eps * D, e, L // 2, L // 2).dense())[0]
    em = np.linalg.eigvalsh(FCI(h, V - eps * D, e, L // 2, L // 2).dense())[0]
    assert abs((ep - em) / (2 * eps) - np.sum(D * G)) < 1e-6
