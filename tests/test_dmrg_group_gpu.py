"""Whole DMRG runs in lockstep (qcm_dmrg_group_sweep): independent two-site FP64 runs of the same length
swept together, one merged plan group and one lockstep Jacobi-Davidson per step.  Each run must follow its
own separate sweeps (qcm_dmrg_sweep) and the oracle's step energies, whatever the other runs in the group
hold (different integrals, bond dimensions and gauges)."""
import numpy as np
import pytest

from helpers import qc_system

pytestmark = pytest.mark.gpu

# (integral seed, max bond dimension, gauge of the MPO's bond indices)
RUNS = [(0, 16, None), (1, 24, None), (2, 64, 5), (3, 12, None), (4, 16, 2)]


def make_runs(ctx, L, runs):
    """Device runs started from the oracle's initial MPS (the const initial state itself depends on the
    QR's rounding), with the oracle runs beside them."""
    from oracle.oracle import OracleDMRG
    from qcmaquis_b200.dmrg import DMRG
    from qcmaquis_b200.heff import parse_mps_tensor
    out = []
    for seed, M, gauge in runs:
        h, V, e, m, ts, blob = qc_system(L, seed, gauge)
        ref = OracleDMRG(blob, L, L // 2, L // 2, M)
        sites = [parse_mps_tensor(ref.mps_export(i)) for i in range(L)]
        out.append((DMRG.from_mps(ctx, m, sites, M), DMRG.from_mps(ctx, m, sites, M), ref))
    return out


def test_group_sweeps_follow_separate_sweeps_and_the_oracle(gpu_ctx):
    from qcmaquis_b200.dmrg import DMRG
    L, sweeps = 6, 3
    runs = make_runs(gpu_ctx, L, RUNS)
    for s in range(sweeps):
        Eg, Tg = DMRG.group_sweep([d for d, _, _ in runs])
        assert Eg.shape == (len(RUNS), 2 * L - 2)
        for i, (d, a, ref) in enumerate(runs):
            Ea, Ta = a.sweep()
            E_ref, tw_ref, tf_ref, bd_ref = ref.sweep(s)
            # the lockstep JD orthogonalises by classical Gram-Schmidt twice, the single solve by modified
            # Gram-Schmidt: the same ground states to the JD tolerance
            assert np.abs(Eg[i] - Ea).max() < 1e-9, (s, i, Eg[i] - Ea)
            assert np.abs(Eg[i] - E_ref).max() < 1e-9, (s, i, Eg[i] - E_ref)
            bd = [t["bond_dimension"] for t in Tg[i]]
            assert bd == [t["bond_dimension"] for t in Ta] == list(bd_ref.astype(int)), (s, i)
            assert np.allclose([t["truncated_weight"] for t in Tg[i]], tw_ref, rtol=1e-5, atol=1e-13)
            assert np.array_equal(d.bond_dimensions(), a.bond_dimensions())
    # the plan and boundary-step caches of every run work through the group form too
    for d, _, _ in runs:
        st = d.stats()
        assert st["plans_reused"] + st["plans_built"] == sweeps * (2 * L - 2)
        assert st["plans_reused"] > 0 and st["hpsi_count"] > 0


def test_group_sweep_of_one_run_is_a_sweep(gpu_ctx):
    """A group of one run converges to the FCI energy of an exact bond dimension like its own sweeps."""
    from oracle.fci import FCI
    from qcmaquis_b200.dmrg import DMRG
    L = 6
    h, V, e, m, ts, blob = qc_system(L, 0)
    E_fci = np.linalg.eigvalsh(FCI(h, V, e, L // 2, L // 2).dense())[0]
    d = DMRG(gpu_ctx, m, L // 2, L // 2, 64, ecore=e)
    for _ in range(4):
        E, _ = DMRG.group_sweep([d])
    assert abs(E.min() - E_fci) < 1e-9


def test_group_sweep_rejects_unlike_runs(gpu_ctx):
    from qcmaquis_b200._lib import QcmError
    from qcmaquis_b200.dmrg import DMRG
    h, V, e, m6, ts, blob = qc_system(6, 0)
    h, V, e, m8, ts, blob = qc_system(8, 0)
    a = DMRG(gpu_ctx, m6, 3, 3, 16)
    with pytest.raises(QcmError):
        DMRG.group_sweep([a, DMRG(gpu_ctx, m8, 4, 4, 16)])                       # different lengths
    with pytest.raises(QcmError):
        DMRG.group_sweep([a, DMRG(gpu_ctx, m6, 3, 3, 16, precision="mixed")])    # not FP64
    with pytest.raises(QcmError):
        DMRG.group_sweep([a, DMRG(gpu_ctx, m6, 3, 3, 16, jcd_tol=1e-8)])         # different JD tolerance
    with pytest.raises(QcmError):
        DMRG.group_sweep([a, a])                                                 # a run twice
    b = DMRG(gpu_ctx, m6, 3, 3, 16)
    b.run(3)
    with pytest.raises(QcmError):
        DMRG.group_sweep([a, b])                                                 # b is inside a sweep
    # the rejected calls left a untouched: a full group sweep of it still runs
    E, _ = DMRG.group_sweep([a])
    assert np.all(np.isfinite(E))
