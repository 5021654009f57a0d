"""Excited states (ts_optimize.hpp:217-223, optimize.h:134-172): two-site sweeps whose every solution is kept
orthogonal to given ortho states, through overlap boundaries (mps.h:175-219) and the ortho states' projections
onto each step's two-site basis (site_ortho_boundaries, contractions/special.hpp:38-62).  The oracle is pinned
against FCI's first excited state at a bond dimension where the MPS is exact; the device against the oracle
step by step and against FCI."""
import functools

import numpy as np
import pytest

from oracle.oracle import OracleDMRG
from oracle.fci import FCI

from helpers import qc_system

L_EX = 6  # 400-determinant sector: at M = 64 every bond of the MPS is exact


@functools.lru_cache(maxsize=None)
def fci_levels(L):
    h, V, e, m, ts, blob = qc_system(L)
    return FCI(h, V, e, L // 2, L // 2).lowest(3)


@functools.lru_cache(maxsize=None)
def ground_state(L, M, sweeps=4):
    """Oracle ground state: (site blobs, lowest sweep energy)."""
    h, V, e, m, ts, blob = qc_system(L)
    g = OracleDMRG(blob, L, L // 2, L // 2, M)
    for s in range(sweeps):
        E = g.sweep(s)[0]
    return tuple(g.mps_export(i) for i in range(L)), float(E.min())


def test_oracle_excited_state_matches_fci():
    L, M = L_EX, 64
    h, V, e, m, ts, blob = qc_system(L)
    w = fci_levels(L)
    gs, E0 = ground_state(L, M)
    assert abs(E0 - w[0]) < 1e-9
    x = OracleDMRG(blob, L, L // 2, L // 2, M)
    x.set_ortho([list(gs)])
    for s in range(6):
        E = x.sweep(s)[0]
    assert abs(E.min() - w[1]) < 1e-8, E.min() - w[1]
    assert abs(E.max() - w[1]) < 1e-8, E.max() - w[1]  # every step of a converged sweep


@pytest.mark.gpu
def test_device_excited_sweeps_match_oracle(gpu_ctx):
    """Both engines start from the oracle's initial MPS with the same ortho state (an M = 24 ground state):
    step energies to 1e-10 Eh and identical kept dimensions over three sweeps."""
    from qcmaquis_b200.dmrg import DMRG
    from qcmaquis_b200.heff import parse_mps_tensor
    L, M = L_EX, 24
    h, V, e, m, ts, blob = qc_system(L)
    gs, _ = ground_state(L, M)
    ref = OracleDMRG(blob, L, L // 2, L // 2, M)
    sites = [parse_mps_tensor(ref.mps_export(i)) for i in range(L)]
    ref.set_ortho([list(gs)])
    dev = DMRG.from_mps(gpu_ctx, m, sites, M)
    dev.set_ortho([[parse_mps_tensor(b) for b in gs]])
    for s in range(3):
        E_ref, tw_ref, tf_ref, bd_ref = ref.sweep(s)
        E, tr = dev.sweep()
        assert np.abs(E - E_ref).max() < 1e-10, (s, np.abs(E - E_ref).max())
        assert np.array_equal(np.array([t["bond_dimension"] for t in tr]), bd_ref.astype(np.int64))


@pytest.mark.gpu
def test_device_excited_state_matches_fci(gpu_ctx):
    """The device's own ground state (const initial state) as the ortho state, then the excited-state sweeps
    from a fresh const state: the first excited FCI level to 1e-8."""
    from qcmaquis_b200.dmrg import DMRG
    from qcmaquis_b200.heff import parse_mps_tensor
    L, M = L_EX, 64
    h, V, e, m, ts, blob = qc_system(L)
    w = fci_levels(L)
    g = DMRG(gpu_ctx, m, L // 2, L // 2, M)
    for _ in range(4):
        E0, _ = g.sweep()
    assert abs(E0.min() - w[0]) < 1e-9
    gs = [parse_mps_tensor(b) for b in g.export_mps()]
    x = DMRG(gpu_ctx, m, L // 2, L // 2, M)
    x.set_ortho([gs])
    for _ in range(6):
        E1, _ = x.sweep()
    assert abs(E1.min() - w[1]) < 1e-8, E1.min() - w[1]
    with pytest.raises(RuntimeError, match="start of a sweep"):
        x.run(3)
        x.set_ortho([gs])
