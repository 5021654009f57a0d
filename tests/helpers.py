"""Shared test helpers: seeded synthetic problems and frozen site problems from the oracle."""
from __future__ import annotations

import functools
import struct

import numpy as np

from qcmaquis_b200.fcidump import synthetic_integrals, hubbard_ladder_integrals
from qcmaquis_b200.mpo import MPO


def gauge_signed(tensors, seed):
    """The same MPO with a random sign on bond indices (column b of W[p] and row b of W[p+1]
    negated together); a Hermitian pair with one negated member gets phase -1, so boundaries
    built from it carry conjugate scales of -1 (BoundaryIndex::conjugate_scale)."""
    rng = np.random.default_rng(seed)
    ts = [dict(t) for t in tensors]
    for p in range(len(ts) - 1):
        n = ts[p]["cols"]
        s = np.where(rng.random(n) < 0.5, -1.0, 1.0)
        s[:1] = 1.0
        hr = ts[p]["herm_right"].copy()
        for b in range(n):
            if hr[b, 0] >= 0:
                hr[b, 1] = int(hr[b, 1] * s[b] * s[hr[b, 0]])
        ts[p]["scale"] = ts[p]["scale"] * s[ts[p]["b2"]]
        ts[p]["herm_right"] = hr
        ts[p + 1]["scale"] = ts[p + 1]["scale"] * s[ts[p + 1]["b1"]]
        ts[p + 1]["herm_left"] = hr.copy()
    return ts


@functools.lru_cache(maxsize=None)
def qc_system(L: int, seed: int = 0, gauge=None):
    """Integrals, single-site MPO, two-site MPO and MPO blob; gauge = seed of a sign gauge on the
    MPO's bond indices (gauge_signed), None for the plain MPO."""
    h, V, e = synthetic_integrals(L, seed)
    m = MPO.qc(h, V)
    if gauge is not None:
        m = MPO.from_tensors(gauge_signed(m.tensors(), gauge))
    return h, V, e, m, m.twosite(), m.blob()


@functools.lru_cache(maxsize=None)
def snapshot(L: int, M: int, sweeps_before: int, step: int, seed: int = 0, gauge=None):
    """Frozen site problem (QSPB blob) of `step` in sweep `sweeps_before` (oracle DMRG)."""
    from oracle.oracle import OracleDMRG
    h, V, e, m, ts, blob = qc_system(L, seed, gauge)
    d = OracleDMRG(blob, L, L // 2, L // 2, M)
    for s in range(sweeps_before):
        d.sweep(s)
    return d.snapshot(sweeps_before, step)


def site_of_step(L: int, step: int) -> int:
    """site1 of ts_optimize's step index (ts_optimize.hpp:128-150)."""
    return step if step < L - 1 else 2 * L - 2 - step - 1


def parse_schedule_export(sch: bytes):
    """Rows (lb_in, lb_out, ci, ci_eff, unit_offset, ms, b1, mps_offset, ci_right, col, alpha) of a QSCH blob."""
    off = 0

    def get(fmt):
        nonlocal off
        v = struct.unpack_from("<" + fmt, sch, off)
        off += struct.calcsize("<" + fmt)
        return v

    magic, nb = get("II")
    assert magic == 0x48435351
    rows = []
    for _ in range(nb):
        (ntj,) = get("I")
        tj = [get("IIII") for _ in range(ntj)]
        (nc,) = get("I")
        for _ in range(nc):
            lb, rb, ls, rs, ci, cie, nS, stripe, nu = get("IIIIIIIII")
            for _ in range(nu):
                uo, ms, nl, na = get("IIII")
                lines = [get("II") for _ in range(nl)]
                als = [get("dII") for _ in range(na)]
                k = 0
                for (b1, cnt) in lines:
                    for a in als[k:k + cnt]:
                        rows.append((lb, rb, ci, cie, uo, ms, b1, tj[a[1]][0], tj[a[1]][1], a[2], a[0]))
                    k += cnt
    return rows


# ---------------------------------------------------------------------------
# dense restatement of one boundary step (independent of the block bookkeeping)

def _offsets(idx):
    o, t = [], 0
    for (_, _, s) in idx:
        o.append(t)
        t += s
    return o, t


def dense_site_tensor(phys, left, right, blocks):
    """A[state, l, r] from right-paired blocks (columns ordered by ProductBasis(phys, right, -p + r))."""
    lo, ln = _offsets(left)
    ro, rn = _offsets(right)
    so, sn = _offsets(phys)
    rpos = {(a, b): i for i, (a, b, _) in enumerate(right)}
    lpos = {(a, b): i for i, (a, b, _) in enumerate(left)}
    A = np.zeros((sn, ln, rn))
    for (ch, blk) in blocks:
        lb = lpos[ch]
        col = 0
        for s, (pa, pb, d) in enumerate(phys):
            rc = (ch[0] + pa, ch[1] + pb)
            if rc not in rpos:
                continue
            rb = rpos[rc]
            rs = right[rb][2]
            for ss in range(d):
                A[so[s] + ss, lo[lb]:lo[lb] + left[lb][2], ro[rb]:ro[rb] + rs] = blk[:, col:col + rs]
                col += rs
        assert col == blk.shape[1]
    return A


def boundary_cohort_of(b):
    """(bra charge, ket charge) -> cohort index of a boundary dict."""
    return {(tuple(b["bra"][int(i)][:2]), tuple(b["ket"][int(j)][:2])): ci
            for ci, (i, j) in enumerate(zip(b["cohort_bra"], b["cohort_ket"]))}


def dense_boundary(b):
    """B[aux, bra, ket] of a boundary dict (cohort blocks bra size x ket size).

    A transposed cohort (tr) stores no data: its block k is conjugate_scale times the transpose
    of the block at offsets[k] of the partner cohort (bra and ket charges swapped), as
    BoundaryIndex::complement_transpose sets it up (boundary.h:161-191)."""
    bo, bn = _offsets(b["bra"])
    ko, kn = _offsets(b["ket"])
    aux = b["aux"]
    where = boundary_cohort_of(b)
    B = np.zeros((aux, bn, kn))
    for ci in range(len(b["cohort_bra"])):
        i, j = int(b["cohort_bra"][ci]), int(b["cohort_ket"][ci])
        r, c = b["bra"][i][2], b["ket"][j][2]
        if b["tr"][ci]:
            ce = where[(tuple(b["ket"][j][:2]), tuple(b["bra"][i][:2]))]
            assert not b["tr"][ce]
            base = int(b["data_offset"][ce])
            for k in range(aux):
                o = int(b["offsets"][ci * aux + k])
                if o >= 0:
                    blk = b["data"][base + o: base + o + r * c].reshape(r, c)  # partner block c x r, column-major
                    B[k, bo[i]:bo[i] + r, ko[j]:ko[j] + c] = b["cscale"][ci * aux + k] * blk
            continue
        base = int(b["data_offset"][ci])
        for k in range(aux):
            o = int(b["offsets"][ci * aux + k])
            if o >= 0:
                B[k, bo[i]:bo[i] + r, ko[j]:ko[j] + c] = b["data"][base + o: base + o + r * c].reshape(c, r).T
    return B


def dense_mpo_tensor(t):
    """W[b1, b2, out, in] of one MPO tensor dict (mpo.parse_blob)."""
    n = sum(s[2] for s in t["phys"])
    W = np.zeros((t["rows"], t["cols"], n, n))
    for e in range(len(t["b1"])):
        op = t["ops"][int(t["op"][e])]
        W[int(t["b1"][e]), int(t["b2"][e]), op["out"], op["inp"]] += t["scale"][e] * op["val"]
    return W


def dense_boundary_step(case, mpo_tensor):
    """New boundary of a QBSP case, dense: left  L'[b2, r', r] = A[s', l', r'] L[b1, l', l] W[b1, b2, s', s] A[s, l, r];
    right R'[b1, l, l'] = A[s, l, r] W[b1, b2, s', s] R[b2, r, r'] A[s', l', r']."""
    A = dense_site_tensor(case["phys"], case["left"], case["right"], case["blocks"])
    B = dense_boundary(case["B_in"])
    W = dense_mpo_tensor(mpo_tensor)
    if case["side"] == 0:
        return np.einsum("pak,xac,xypq,qcl->ykl", A, B, W, A, optimize=True)
    return np.einsum("qak,xypq,ykl,pbl->xab", A, W, B, A, optimize=True)
