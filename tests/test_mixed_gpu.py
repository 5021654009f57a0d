"""Mixed-precision form of H_eff . psi (S build as 3xTF32 on the tensor cores, FP32 accumulation;
T-GEMM and L.S in FP64) against the FP64 oracle: the apply itself, the Jacobi-Davidson eigenvalue
(FP64 Rayleigh quotient of the mixed solve's vector) and whole sweeps."""
import numpy as np
import pytest

from qcmaquis_b200 import heff
from oracle.oracle import heff_apply

from helpers import qc_system, snapshot, site_of_step

pytestmark = pytest.mark.gpu

# 3xTF32 products carry ~2^-21 relative error, summed in FP32: ~1e-7 of the largest output element
HPSI_TOL = 2e-6
# the eigenvalue is an FP64 Rayleigh quotient: its error is second order in the vector's
JD_TOL = 1e-8
# the precision form's target: per-step energies within 1e-6 Eh of the FP64 oracle
SWEEP_TOL = 1e-6


FORMS = ["mixed", "mixed_tc"]


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("L,M,sw,step", [(6, 16, 1, 2), (8, 64, 1, 3), (8, 64, 2, 12), (10, 48, 1, 4)])
def test_mixed_heff_matches_oracle(gpu_ctx, L, M, sw, step, form):
    snap = snapshot(L, M, sw, step)
    h, V, e, m, ts, blob = qc_system(L, 0)
    site = site_of_step(L, step)
    p = heff.parse_site_problem(snap)
    plan = heff.plan_from_problem(gpu_ctx, p, ts, site)
    x0 = heff.twin_vector(p)
    rng = np.random.default_rng(step)
    for x in (x0, rng.standard_normal(x0.size)):
        y_ref, fl, _ = heff_apply(snap, blob, site, x)
        y = plan.apply(x, precision=form)
        scale = np.abs(y_ref).max()
        err = np.abs(y - y_ref).max()
        assert err <= HPSI_TOL * scale, (err / scale)
        assert err > 0.0  # it is the mixed path, not the FP64 one
        # run to run the mixed form is deterministic too
        assert np.array_equal(plan.apply(x, precision=form), y)
        # the FP64 form on the same plan is unaffected by the mixed buffers
        assert np.abs(plan.apply(x) - y_ref).max() <= 1e-12 * scale


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("L,M,sw,step", [(6, 16, 1, 2), (8, 32, 1, 9)])
def test_mixed_jd_matches_oracle_step_energy(gpu_ctx, L, M, sw, step, form):
    from oracle.oracle import OracleDMRG
    from qcmaquis_b200.dmrg import jd_solve
    h, V, e, m, ts, blob = qc_system(L)
    prob = heff.parse_site_problem(snapshot(L, M, sw, step))
    plan = heff.plan_from_problem(gpu_ctx, prob, ts, site_of_step(L, step))
    ev, vec, it = jd_solve(plan, heff.twin_vector(prob), 1e-10, 8, precision=form)
    d = OracleDMRG(blob, L, L // 2, L // 2, M)
    for s in range(sw):
        d.sweep(s)
    E_ref = d.sweep(sw)[0][step]
    # the exact lowest eigenvalue of the frozen problem (FP64 applies)
    from scipy.sparse.linalg import LinearOperator, eigsh
    n = vec.size
    lam = eigsh(LinearOperator((n, n), matvec=lambda v: plan.apply(np.ascontiguousarray(v)), dtype=np.float64),
                k=1, which="SA", tol=1e-13, v0=heff.twin_vector(prob))[0][0]
    # ev is an FP64 Rayleigh quotient, so it is variational; it is no further from the exact
    # eigenvalue than the FP64 solve (which stops at maxiter = 8 too) plus JD_TOL
    assert ev >= lam - 1e-11, (ev - lam)
    assert ev - lam <= (E_ref - lam) + JD_TOL, (ev - lam, E_ref - lam)
    assert abs(vec @ plan.apply(vec) / (vec @ vec) - ev) < 1e-10


@pytest.mark.parametrize("L,M,sweeps", [(8, 32, 3), (12, 128, 4)])
def test_mixed_sweeps_match_oracle(gpu_ctx, L, M, sweeps):
    """Both engines start from the oracle's initial MPS; the device runs every JD in the mixed form (with
    its FP64 residual correction) and the oracle in FP64: every sweep's energy within 1e-6 Eh."""
    from oracle.oracle import OracleDMRG
    from qcmaquis_b200.dmrg import DMRG
    from qcmaquis_b200.heff import parse_mps_tensor
    h, V, e, m, ts, blob = qc_system(L)
    ref = OracleDMRG(blob, L, L // 2, L // 2, M)
    sites = [parse_mps_tensor(ref.mps_export(i)) for i in range(L)]
    dev = DMRG.from_mps(gpu_ctx, m, sites, M, precision="mixed")
    dev_steps = []
    for s in range(sweeps):
        E_ref, tw_ref, tf_ref, bd_ref = ref.sweep(s)
        E, tr = dev.sweep()
        # the sweep energy (minimum over its steps, as the reference reports it) within the target
        assert abs(E.min() - E_ref.min()) < SWEEP_TOL, (s, E.min() - E_ref.min())
        dev_steps.append(np.abs(E - E_ref).max())
        if M <= 32:
            # (at M = 128 the cut meets singular values that the mixed vectors move by ~1e-7)
            bd = np.array([t["bond_dimension"] for t in tr])
            assert np.array_equal(bd, bd_ref.astype(np.int64)), (s, bd, bd_ref)
    # step energies of a growing sweep follow the unconverged JD path (8 iterations), so they
    # differ more than the precision does; once converged every step is within the target
    assert dev_steps[-1] < SWEEP_TOL, dev_steps
    st = dev.stats()
    # the FP64 residual correction: the Rayleigh quotient of each step's final vector, and at most
    # one FP64 correction step (the default mixed_refine)
    nsteps = sweeps * (2 * L - 2)
    assert nsteps <= st["hpsi_count_fp64"] <= 2 * nsteps
