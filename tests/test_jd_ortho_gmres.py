"""Jacobi-Davidson beyond the plain solve: GMRES corrections (ietl_jcd_gmres; jcd_gmres_solver,
ietl/jacobi.h:126-164 and ietl_gmres, ietl/gmres.h:78-146) and ortho vectors (excited states;
DavidsonVS::project, solver/ietl_interface_dv.h:94-99), the oracle pinned against dense
diagonalisation on the CPU and the device solve (qcm_jd_solve_ex) against the oracle."""
import functools

import numpy as np
import pytest

from oracle.oracle import heff_apply, jd_solve as orc_jd

from helpers import qc_system, snapshot, site_of_step

CASE = (6, 16, 1, 2)  # L, M, sweeps before, step: a 400-dimensional site problem


@functools.lru_cache(maxsize=None)
def dense_problem(L, M, sw, step):
    h, V, e, m, ts, blob = qc_system(L, 0)
    snap = snapshot(L, M, sw, step)
    site = site_of_step(L, step)
    from qcmaquis_b200 import heff
    x0 = heff.twin_vector(heff.parse_site_problem(snap))
    n = x0.size
    H = np.column_stack([heff_apply(snap, blob, site, np.eye(n)[i])[0] for i in range(n)])
    w, Z = np.linalg.eigh(0.5 * (H + H.T))
    return snap, blob, site, x0, w, Z


def random_start(n, seed=3):
    return np.random.default_rng(seed).standard_normal(n)


def test_oracle_gmres_one_is_the_plain_correction():
    """ietl_gmres keeps the directions before its last inner step: with max_iter 1 the loop body never
    runs and the start t0 comes back after one operator apply, so the solve is the gmres = 0 solve
    with one extra H.psi per correction."""
    snap, blob, site, x0, w, Z = dense_problem(*CASE)
    e0, v0, it0, na0 = orc_jd(snap, blob, site, x0, 1e-10, 8, gmres=0)
    e1, v1, it1, na1 = orc_jd(snap, blob, site, x0, 1e-10, 8, gmres=1)
    assert e0 == e1 and np.array_equal(v0, v1) and it0 == it1
    assert na0 == it0 and na1 == it1 + (it1 - 1)


def test_oracle_gmres_converges_further():
    snap, blob, site, x0, w, Z = dense_problem(*CASE)
    errs = []
    for g in (0, 3, 6):
        ev, vec, it, na = orc_jd(snap, blob, site, x0, 1e-10, 8, gmres=g)
        assert ev >= w[0] - 1e-12
        errs.append(ev - w[0])
        # each correction costs at most g applies (one for the start residual, g - 1 Arnoldi steps)
        assert na <= it + (it - 1) * max(g, 0)
    assert errs[2] < errs[1] < errs[0]
    assert errs[2] < 1e-5


@pytest.mark.parametrize("gmres,maxiter", [(0, 64), (4, 40)])
def test_oracle_ortho_vectors_give_excited_states(gmres, maxiter):
    """From a random start (overlaps 0.03-0.06 with the low eigenvectors) the plain correction needs
    ~64 iterations for 1e-10, GMRES(4) converges in 33."""
    snap, blob, site, x0, w, Z = dense_problem(*CASE)
    xr = random_start(x0.size)
    ev, vec, it, na = orc_jd(snap, blob, site, xr, 1e-10, maxiter, ortho=[Z[:, 0]], gmres=gmres)
    assert abs(ev - w[1]) < 1e-8, ev - w[1]
    assert abs(vec @ Z[:, 0]) < 1e-12
    # non-normalised, non-orthogonal ortho vectors span the same space after Gram-Schmidt
    ev, vec, it, na = orc_jd(snap, blob, site, xr, 1e-10, maxiter, ortho=[3 * Z[:, 0], Z[:, 1] + 0.5 * Z[:, 0]],
                             gmres=gmres)
    assert abs(ev - w[2]) < 1e-8, ev - w[2]
    assert max(abs(vec @ Z[:, 0]), abs(vec @ Z[:, 1])) < 1e-12


JD_CASES = {
    # name: (start, ortho eigenvector indices, gmres, maxiter)
    "gmres6": ("twin", (), 6, 8),
    "gmres1": ("twin", (), 1, 8),
    "gmres3_it12": ("twin", (), 3, 12),
    "ortho1": ("random", (0,), 0, 24),
    "ortho2_gmres4": ("random", (0, 1), 4, 16),
}


@pytest.mark.gpu
@pytest.mark.parametrize("case", list(JD_CASES))
def test_device_jd_ex_matches_oracle(gpu_ctx, case):
    from qcmaquis_b200 import heff
    from qcmaquis_b200.dmrg import jd_solve
    start, oi, gmres, maxiter = JD_CASES[case]
    L, M, sw, step = CASE
    snap, blob, site, x0, w, Z = dense_problem(*CASE)
    h, V, e, m, ts, _ = qc_system(L, 0)
    plan = heff.plan_from_problem(gpu_ctx, heff.parse_site_problem(snap), ts, site)
    xs = x0 if start == "twin" else random_start(x0.size)
    ortho = [Z[:, i] * (1.0 + i) for i in oi]
    er, vr, itr, nar = orc_jd(snap, blob, site, xs, 1e-10, maxiter, ortho=ortho, gmres=gmres)
    ev, vec, it, na = jd_solve(plan, xs, 1e-10, maxiter, ortho=ortho, gmres=gmres, return_applies=True)
    # the same iteration path: counts equal, eigenvalue and vector to rounding
    assert (it, na) == (itr, nar)
    assert abs(ev - er) <= 1e-10 * abs(er), ev - er
    sg = np.sign(vec @ vr)
    assert np.abs(vec - sg * vr).max() < 1e-6
    for i in oi:
        assert abs(vec @ Z[:, i]) < 1e-10
    # variational within the complement of the ortho vectors (to the rounding of the projections)
    assert ev >= w[len(oi)] - 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["mixed", "mixed_tc"])
def test_device_jd_ex_mixed_excited_state(gpu_ctx, form):
    """Mixed H.psi with GMRES and an ortho vector: the FP64 Rayleigh quotient of the converged vector
    is the first excited eigenvalue to 1e-8."""
    from qcmaquis_b200 import heff
    from qcmaquis_b200.dmrg import jd_solve
    L, M, sw, step = CASE
    snap, blob, site, x0, w, Z = dense_problem(*CASE)
    h, V, e, m, ts, _ = qc_system(L, 0)
    plan = heff.plan_from_problem(gpu_ctx, heff.parse_site_problem(snap), ts, site)
    ev, vec, it, na = jd_solve(plan, random_start(x0.size), 1e-10, 24, precision=form, ortho=[Z[:, 0]], gmres=6,
                               return_applies=True)
    assert abs(ev - w[1]) < 1e-8, ev - w[1]
    assert abs(vec @ Z[:, 0]) < 1e-10


@pytest.mark.gpu
def test_device_jd_ex_rejects_bad_arguments(gpu_ctx):
    from qcmaquis_b200 import heff
    from qcmaquis_b200.dmrg import jd_solve
    L, M, sw, step = CASE
    snap, blob, site, x0, w, Z = dense_problem(*CASE)
    h, V, e, m, ts, _ = qc_system(L, 0)
    plan = heff.plan_from_problem(gpu_ctx, heff.parse_site_problem(snap), ts, site)
    with pytest.raises(RuntimeError, match="gmres"):
        jd_solve(plan, x0, 1e-10, 8, gmres=65)
    with pytest.raises(RuntimeError, match="zero norm"):
        jd_solve(plan, x0, 1e-10, 8, ortho=[Z[:, 0], np.zeros_like(x0)])


@pytest.mark.gpu
def test_sweeps_with_gmres_match_oracle(gpu_ctx):
    """ietl_jcd_gmres = 4 in every step: both engines from the oracle's initial MPS, step energies to
    1e-10 Eh, identical kept dimensions and H.psi counts.  jcd_maxiter 30 so that every step converges:
    the first step from the const state needs 23 iterations, and an iterate stopped before convergence
    carries the rounding differences of its inner solves into the energy (4.7e-10 Eh at 8 iterations)."""
    from oracle.oracle import OracleDMRG
    from qcmaquis_b200.dmrg import DMRG
    from qcmaquis_b200.heff import parse_mps_tensor
    L, M, sweeps, g, maxiter = 6, 24, 2, 4, 30
    h, V, e, m, ts, blob = qc_system(L)
    ref = OracleDMRG(blob, L, L // 2, L // 2, M, maxiter=maxiter)
    ref.set_gmres(g)
    sites = [parse_mps_tensor(ref.mps_export(i)) for i in range(L)]
    dev = DMRG.from_mps(gpu_ctx, m, sites, M, jcd_gmres=g, jcd_maxiter=maxiter)
    for s in range(sweeps):
        E_ref, tw_ref, tf_ref, bd_ref = ref.sweep(s)
        E, tr = dev.sweep()
        assert np.abs(E - E_ref).max() < 1e-10, (s, np.abs(E - E_ref).max())
        assert np.array_equal(np.array([t["bond_dimension"] for t in tr]), bd_ref.astype(np.int64))
    assert int(dev.stats()["hpsi_count"]) == int(ref.stats()["hpsi_count"])
