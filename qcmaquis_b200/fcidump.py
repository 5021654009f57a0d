"""Synthetic ab-initio integrals and FCIDUMP text I/O.

The integrals are the inputs of the two-site DMRG effective-Hamiltonian path;
the reference reads them from an FCIDUMP file
(models/chem/parse_integrals.h: four header lines, then ``value i j k l``
with 1-based orbital indices, ``k = l = 0`` for one-electron terms and
``0 0 0 0`` for the core energy).  The unique-index convention of the writer
follows lib/interface/cpp_maquis.cpp (prepare_integrals):
``h: i >= j`` and ``V: i >= j, k >= l, (i > k or (i == k and j >= l))``.

Synthetic recipe (seeded ``numpy.random.default_rng(seed)``), draw order:
  1. ``A = rng.standard_normal((L, L))``; ``h = triu(A) + triu(A, 1).T``;
     ``h *= exp(-|i - j| / 2)``; ``h[i, i] += -2 - 4 i / L`` (i 0-based).
  2. for P in 0 .. 2L-1: ``Bm = rng.normal(0, 0.3, (L, L))``;
     ``B[P] = triu(Bm) + triu(Bm, 1).T``.
  3. ``V[i, j, k, l] = sum_P B[P, i, j] * B[P, k, l]`` (chemist notation
     (ij|kl); 8-fold symmetric, positive semi-definite Coulomb matrix).
  Nuclear repulsion (core energy) 0.
"""
from __future__ import annotations

import numpy as np


def synthetic_integrals(L: int, seed: int):
    """Return (h, V, ecore) for the seeded synthetic Hamiltonian of L orbitals."""
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((L, L))
    h = np.triu(A) + np.triu(A, 1).T
    idx = np.arange(L)
    h = h * np.exp(-np.abs(idx[:, None] - idx[None, :]) / 2.0)
    h[idx, idx] += -2.0 - 4.0 * idx / L
    B = np.empty((2 * L, L, L))
    for P in range(2 * L):
        Bm = rng.normal(0.0, 0.3, (L, L))
        B[P] = np.triu(Bm) + np.triu(Bm, 1).T
    V = np.einsum("pij,pkl->ijkl", B, B, optimize=True)
    return np.ascontiguousarray(h), np.ascontiguousarray(V), 0.0


def hubbard_ladder_integrals(nrungs: int, t: float = 1.0, tp: float = 1.0, U: float = 8.0):
    """Open two-leg Hubbard ladder (nrungs x 2 sites) written as integrals.

    Site numbering is rung-major: site 2*r + leg.  Hopping ``-t`` along the
    legs, ``-tp`` across each rung, on-site ``U`` as ``V_iiii``.  This is the
    system of the reference's two-site TwoU1 regression test
    (regression/applications/dmrg/test_fermiladder_ts.py).
    """
    L = 2 * nrungs
    h = np.zeros((L, L))
    for r in range(nrungs):
        a, b = 2 * r, 2 * r + 1
        h[a, b] = h[b, a] = -tp
        if r + 1 < nrungs:
            for leg in range(2):
                i, j = 2 * r + leg, 2 * (r + 1) + leg
                h[i, j] = h[j, i] = -t
    V = np.zeros((L, L, L, L))
    for i in range(L):
        V[i, i, i, i] = U
    return h, V, 0.0


def write_fcidump(path: str, h: np.ndarray, V: np.ndarray, ecore: float, nelec: int,
                  ms2: int = 0, cutoff: float = 0.0) -> None:
    L = h.shape[0]
    lines = [f" &FCI NORB={L},NELEC={nelec},MS2={ms2},",
             "  ORBSYM=" + ",".join(["1"] * L) + ",",
             "  ISYM=1,",
             " &END"]
    for i in range(L):
        for j in range(i + 1):
            for k in range(L):
                for l in range(k + 1):
                    if i > k or (i == k and j >= l):
                        v = V[i, j, k, l]
                        if abs(v) > cutoff:
                            lines.append(f"{v: .16e} {i + 1} {j + 1} {k + 1} {l + 1}")
    for i in range(L):
        for j in range(i + 1):
            if abs(h[i, j]) > cutoff:
                lines.append(f"{h[i, j]: .16e} {i + 1} {j + 1} 0 0")
    lines.append(f"{ecore: .16e} 0 0 0 0")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def read_fcidump(path: str):
    """Parse an FCIDUMP file written as above (4 header lines skipped)."""
    with open(path) as f:
        text = f.read().splitlines()
    header = " ".join(text[:4])
    L = int(header.split("NORB=")[1].split(",")[0])
    h = np.zeros((L, L))
    V = np.zeros((L, L, L, L))
    ecore = 0.0
    for line in text[4:]:
        parts = line.split()
        if len(parts) != 5:
            continue
        v = float(parts[0])
        i, j, k, l = (int(x) - 1 for x in parts[1:])
        if i < 0:
            ecore = v
        elif k < 0:
            h[i, j] = h[j, i] = v
        else:
            for (a, b, c, d) in ((i, j, k, l), (j, i, k, l), (i, j, l, k), (j, i, l, k),
                                 (k, l, i, j), (l, k, i, j), (k, l, j, i), (l, k, j, i)):
                V[a, b, c, d] = v
    return h, V, ecore
