"""Adjoint of the H_eff apply (the differentiation form): for f = ybar . H_eff x, psi_bar = H_eff^T ybar
and the derivative of f with respect to the scale of every entry of the two-site MPO tensor.  The
oracle's gradient (per schedule coefficient alpha, site_hamil_tasks.hpp:41-137, through the transposes
of create_s_r and contract) is pinned by central finite differences of its own apply on the CPU; the
device's (qcm_heff_adjoint) against the oracle and against finite differences of its own apply and of
the lowest eigenvalue."""
import numpy as np
import pytest

from oracle.oracle import heff_adjoint as orc_adjoint
from oracle.oracle import heff_apply

from helpers import qc_system, snapshot, site_of_step

STEP = 1e-5        # central-difference step on the scales (relative to each scale)
N_DIRECTIONS = 20  # seeded random directions


def problem(L, M, sw, step, seed=0):
    from qcmaquis_b200 import heff
    h, V, e, m, ts, blob = qc_system(L, 0)
    snap = snapshot(L, M, sw, step)
    site = site_of_step(L, step)
    p = heff.parse_site_problem(snap)
    x = heff.twin_vector(p)
    rng = np.random.default_rng(seed)
    ybar = rng.standard_normal(x.size)
    return snap, site, p, x, ybar, ts, rng


def perturbed(ts, site, scale, D, h):
    t = ts.copy()
    t.set_scales(site, scale + h * D)
    return t


def test_oracle_scale_gradient_matches_finite_differences():
    L, M, sw, step = 6, 16, 1, 2
    snap, site, p, x, ybar, ts, rng = problem(L, M, sw, step)
    sc = ts.terms(site)["scale"]
    pb, g = orc_adjoint(snap, ts.blob(), site, x, ybar, sc.size)
    f0 = ybar @ heff_apply(snap, ts.blob(), site, x)[0]
    # psi_bar: d f / d x along random directions (f is linear in x)
    for _ in range(3):
        d = rng.standard_normal(x.size)
        fd = ybar @ heff_apply(snap, ts.blob(), site, d)[0]
        assert abs(pb @ d - fd) <= 1e-12 * np.abs(pb).sum() * np.abs(d).max()
    errs = []
    for _ in range(N_DIRECTIONS):
        D = rng.standard_normal(sc.size) * np.abs(sc)
        fp = ybar @ heff_apply(snap, perturbed(ts, site, sc, D, STEP).blob(), site, x)[0]
        fm = ybar @ heff_apply(snap, perturbed(ts, site, sc, D, -STEP).blob(), site, x)[0]
        fd = (fp - fm) / (2 * STEP)
        errs.append(abs(fd - g @ D) / max(abs(fd), 1e-3 * abs(f0)))
    assert max(errs) < 1e-6, max(errs)
    # single entries: the largest gradients one at a time
    for e in np.argsort(-np.abs(g))[:3]:
        D = np.zeros(sc.size)
        D[e] = 1.0
        fp = ybar @ heff_apply(snap, perturbed(ts, site, sc, D, 1.0).blob(), site, x)[0]
        assert abs((fp - f0) - g[e]) <= 1e-9 * abs(f0)


@pytest.mark.gpu
@pytest.mark.parametrize("L,M,sw,step", [(6, 16, 1, 2), (8, 64, 1, 3), (8, 64, 2, 12), (10, 48, 1, 4)])
def test_device_adjoint_matches_oracle(gpu_ctx, L, M, sw, step):
    from qcmaquis_b200 import heff
    snap, site, p, x, ybar, ts, rng = problem(L, M, sw, step)
    plan = heff.plan_from_problem(gpu_ctx, p, ts, site)
    pb, g = plan.adjoint(x, ybar)
    assert g.size == ts.terms(site)["scale"].size
    pb_r, g_r = orc_adjoint(snap, ts.blob(), site, x, ybar, g.size)
    assert np.abs(pb - pb_r).max() <= 1e-12 * np.abs(pb_r).max()
    # different summation orders (dense unit GEMMs vs per-alpha dots): agreement to rounding
    assert np.abs(g - g_r).max() <= 1e-11 * np.abs(g_r).max(), np.abs(g - g_r).max() / np.abs(g_r).max()
    # run to run the gradient is bitwise reproducible
    pb2, g2 = plan.adjoint(x, ybar)
    assert np.array_equal(g, g2) and np.array_equal(pb, pb2)


@pytest.mark.gpu
def test_device_adjoint_finite_differences(gpu_ctx):
    from qcmaquis_b200 import heff
    L, M, sw, step = 8, 64, 1, 3
    snap, site, p, x, ybar, ts, rng = problem(L, M, sw, step, seed=1)
    plan = heff.plan_from_problem(gpu_ctx, p, ts, site)
    pb, g = plan.adjoint(x, ybar)
    f0 = ybar @ plan.apply(x)
    sc = ts.terms(site)["scale"]
    errs = []
    for _ in range(N_DIRECTIONS):
        D = rng.standard_normal(sc.size) * np.abs(sc)
        pp = heff.plan_from_problem(gpu_ctx, p, perturbed(ts, site, sc, D, STEP), site)
        pm = heff.plan_from_problem(gpu_ctx, p, perturbed(ts, site, sc, D, -STEP), site)
        fd = (ybar @ pp.apply(x) - ybar @ pm.apply(x)) / (2 * STEP)
        errs.append(abs(fd - g @ D) / max(abs(fd), 1e-3 * abs(f0)))
    assert max(errs) < 1e-6, max(errs)
    # psi_bar = H^T ybar: f along x directions
    for _ in range(3):
        d = rng.standard_normal(x.size)
        assert abs(pb @ d - ybar @ plan.apply(d)) <= 1e-12 * np.abs(pb).sum() * np.abs(d).max()


@pytest.mark.gpu
def test_device_energy_gradient(gpu_ctx):
    """At the converged lowest eigenvector psi (unit norm) the adjoint with x = ybar = psi is dE/d scale
    (Hellmann-Feynman, boundaries fixed); central differences of the lowest eigenvalue agree."""
    from qcmaquis_b200 import heff
    from qcmaquis_b200.dmrg import jd_solve
    L, M, sw, step = 6, 16, 1, 2
    snap, site, p, x, ybar, ts, rng = problem(L, M, sw, step, seed=2)
    plan = heff.plan_from_problem(gpu_ctx, p, ts, site)
    E, psi, it = jd_solve(plan, x, 1e-13, 64, gmres=8)
    psi = psi / np.linalg.norm(psi)
    _, g = plan.adjoint(psi, psi)
    sc = ts.terms(site)["scale"]
    for _ in range(4):
        D = rng.standard_normal(sc.size) * np.abs(sc)
        Ep = jd_solve(heff.plan_from_problem(gpu_ctx, p, perturbed(ts, site, sc, D, STEP), site), psi, 1e-13, 64,
                      gmres=8)[0]
        Em = jd_solve(heff.plan_from_problem(gpu_ctx, p, perturbed(ts, site, sc, D, -STEP), site), psi, 1e-13, 64,
                      gmres=8)[0]
        fd = (Ep - Em) / (2 * STEP)
        assert abs(fd - g @ D) <= 1e-6 * max(abs(fd), 1.0), (fd, g @ D)


@pytest.mark.gpu
def test_config4_energy_gradient_finite_differences(gpu_ctx):
    """The differentiation form's configuration (L=16, N=16, TwoU1 Sz=0, M=256): after device sweeps, at the
    middle bond's converged lowest eigenvector psi the adjoint with x = ybar = psi is dE/d scale for every
    two-site MPO entry (Hellmann-Feynman, boundaries fixed).  Central differences of the lowest eigenvalue
    (step 1e-5 relative to each scale, 20 seeded random directions) agree to 1e-6 relative, for the FP64
    eigensolver and for the mixed one (mixed H.psi, FP64 Rayleigh quotient)."""
    from qcmaquis_b200 import heff
    from qcmaquis_b200.dmrg import DMRG, jd_solve
    L, M = 16, 256
    h, V, e, m, ts, blob = qc_system(L, 0)
    d = DMRG(gpu_ctx, m, L // 2, L // 2, M, 64)
    for _ in range(3):
        d.sweep()
    site = L // 2 - 1
    d.run(site)
    p = heff.parse_site_problem(d.pending_export())
    del d
    plan = heff.plan_from_problem(gpu_ctx, p, ts, site)
    x0 = heff.twin_vector(p)
    E, psi, it = jd_solve(plan, x0, 1e-13, 64, gmres=8)
    psi = psi / np.linalg.norm(psi)
    _, g = plan.adjoint(psi, psi)
    assert abs(g @ ts.terms(site)["scale"] - E) <= 1e-10 * abs(E)  # Euler: E is linear in the scales
    sc = ts.terms(site)["scale"]
    rng = np.random.default_rng(4)
    errs, errs_mixed = [], []
    for k in range(N_DIRECTIONS):
        D = rng.standard_normal(sc.size) * np.abs(sc)
        pp = heff.plan_from_problem(gpu_ctx, p, perturbed(ts, site, sc, D, STEP), site)
        pm = heff.plan_from_problem(gpu_ctx, p, perturbed(ts, site, sc, D, -STEP), site)
        Ep = jd_solve(pp, psi, 1e-13, 64, gmres=8)[0]
        Em = jd_solve(pm, psi, 1e-13, 64, gmres=8)[0]
        fd = (Ep - Em) / (2 * STEP)
        errs.append(abs(fd - g @ D) / max(abs(fd), 1e-3 * abs(E)))
        if k < 5:
            Ep = jd_solve(pp, psi, 1e-13, 64, precision="mixed")[0]
            Em = jd_solve(pm, psi, 1e-13, 64, precision="mixed")[0]
            fd = (Ep - Em) / (2 * STEP)
            errs_mixed.append(abs(fd - g @ D) / max(abs(fd), 1e-3 * abs(E)))
        del pp, pm
    assert max(errs) < 1e-6, errs
    assert max(errs_mixed) < 1e-6, errs_mixed
