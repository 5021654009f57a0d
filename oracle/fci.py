"""Exact diagonalisation (FCI) of the ab-initio Hamiltonian in one (N_up, N_down) sector.

TEST INFRASTRUCTURE ONLY (part of the oracle): used by tests/ and by the
pinning of the CPU restatement.  It is never called by the product path.

H = sum_{pq,s} h_pq a+_{ps} a_{qs}
  + 1/2 sum_{pqrs,s,t} (pq|rs) a+_{ps} a+_{rt} a_{st} a_{qs}  + ecore
  = sum_pq h_pq E_pq + 1/2 sum_pqrs (pq|rs) (E_pq E_rs - delta_qr E_ps) + ecore,
with E_pq = sum_s a+_{ps} a_{qs}.  Determinants are |alpha string> x
|beta string>; E_pq never changes the parity of either string, so no
alpha/beta cross sign appears.  This is the standard string-based FCI
sigma-vector construction; the lowest eigenvalue comes from ARPACK (eigsh).
"""
from __future__ import annotations

from itertools import combinations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


def _strings(L: int, n: int):
    out = []
    for occ in combinations(range(L), n):
        m = 0
        for o in occ:
            m |= 1 << o
        out.append(m)
    return out


def _single_excitations(L: int, n: int):
    """e[p][q]: sparse (nstr x nstr) matrix of a+_p a_q on n-electron strings."""
    strs = _strings(L, n)
    pos = {s: i for i, s in enumerate(strs)}
    ns = len(strs)
    e = [[None] * L for _ in range(L)]
    for p in range(L):
        for q in range(L):
            rows, cols, vals = [], [], []
            for j, s in enumerate(strs):
                if not (s >> q) & 1:
                    continue
                sign = -1 if bin(s & ((1 << q) - 1)).count("1") % 2 else 1
                s2 = s & ~(1 << q)
                if (s2 >> p) & 1:
                    continue
                sign *= -1 if bin(s2 & ((1 << p) - 1)).count("1") % 2 else 1
                s3 = s2 | (1 << p)
                rows.append(pos[s3])
                cols.append(j)
                vals.append(sign)
            e[p][q] = sp.csr_matrix((vals, (rows, cols)), shape=(ns, ns))
    return e, ns


class FCI:
    def __init__(self, h, V, ecore, nup, ndown):
        h = np.asarray(h, dtype=np.float64)
        V = np.asarray(V, dtype=np.float64)
        L = h.shape[0]
        self.L = L
        ea, na = _single_excitations(L, nup)
        eb, nb = _single_excitations(L, ndown)
        Ia, Ib = sp.identity(na, format="csr"), sp.identity(nb, format="csr")
        self.dim = na * nb
        self.E = [[(sp.kron(ea[p][q], Ib) + sp.kron(Ia, eb[p][q])).tocsr() for q in range(L)]
                  for p in range(L)]
        # h'_pq = h_pq - 1/2 sum_r (pr|rq)
        self.hp = h - 0.5 * np.einsum("prrq->pq", V)
        self.V2 = V.reshape(L * L, L * L)
        self.ecore = ecore

    def matvec(self, c):
        L = self.L
        D = np.empty((L * L, c.shape[0]))
        for p in range(L):
            for q in range(L):
                D[p * L + q] = self.E[p][q] @ c
        G = self.V2 @ D
        sigma = self.ecore * c
        for p in range(L):
            for q in range(L):
                sigma = sigma + self.E[p][q] @ (self.hp[p, q] * c + 0.5 * G[p * L + q])
        return sigma

    def lowest(self, k: int = 1, tol: float = 1e-13):
        op = spla.LinearOperator((self.dim, self.dim), matvec=self.matvec, dtype=np.float64)
        if self.dim <= 400:
            H = np.column_stack([self.matvec(col) for col in np.eye(self.dim)])
            return np.sort(np.linalg.eigvalsh(H))[:k]
        rng = np.random.default_rng(7)
        w = spla.eigsh(op, k=k, which="SA", tol=tol, v0=rng.standard_normal(self.dim),
                       return_eigenvectors=False)
        return np.sort(w)

    def ground_state(self, tol: float = 1e-13):
        """Lowest eigenpair (energy, normalised vector) by ARPACK."""
        op = spla.LinearOperator((self.dim, self.dim), matvec=self.matvec, dtype=np.float64)
        rng = np.random.default_rng(7)
        w, Z = spla.eigsh(op, k=1, which="SA", tol=tol, v0=rng.standard_normal(self.dim))
        c = Z[:, 0]
        return float(w[0]), c / np.linalg.norm(c)

    def one_rdm(self, c):
        """Spin-summed one-particle density matrix gamma_pq = <c| sum_s a+_ps a_qs |c>."""
        return np.array([[c @ (self.E[p][q] @ c) for q in range(self.L)] for p in range(self.L)])

    def dense(self):
        return np.column_stack([self.matvec(col) for col in np.eye(self.dim)])


def fci_energy(h, V, ecore, nup, ndown):
    return float(FCI(h, V, ecore, nup, ndown).lowest(1)[0])
