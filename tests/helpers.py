"""Shared test helpers: seeded synthetic problems and frozen site problems from the oracle."""
from __future__ import annotations

import functools
import struct

import numpy as np

from qcmaquis_b200.fcidump import synthetic_integrals, hubbard_ladder_integrals
from qcmaquis_b200.mpo import MPO


@functools.lru_cache(maxsize=None)
def qc_system(L: int, seed: int = 0):
    h, V, e = synthetic_integrals(L, seed)
    m = MPO.qc(h, V)
    return h, V, e, m, m.twosite(), m.blob()


@functools.lru_cache(maxsize=None)
def snapshot(L: int, M: int, sweeps_before: int, step: int, seed: int = 0):
    """Frozen site problem (QSPB blob) of `step` in sweep `sweeps_before` (oracle DMRG)."""
    from oracle.oracle import OracleDMRG
    h, V, e, m, ts, blob = qc_system(L, seed)
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
