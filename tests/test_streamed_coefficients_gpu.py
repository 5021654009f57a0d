"""Coefficient blocks streamed through a bounded scratch (qcm_heff_stream_coefficients and
qcm_dmrg_set_coefficient_budget): every FP64 apply generates the S-build blocks chunk by chunk instead of
keeping them.  The apply must give the same result to the bit as with the blocks kept, at every chunk size
down to one unit per chunk, and sweeps with a budget the same energies and truncations."""
import numpy as np
import pytest

from helpers import qc_system, site_of_step, snapshot

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("L,M,sw,step", [(8, 32, 1, 3), (10, 48, 1, 4)])
def test_streamed_apply_is_the_kept_apply(gpu_ctx, L, M, sw, step):
    from qcmaquis_b200._lib import QcmError
    from qcmaquis_b200.dmrg import jd_solve
    from qcmaquis_b200.heff import parse_site_problem, plan_from_problem, twin_vector
    h, V, e, m, ts, blob = qc_system(L)
    prob = parse_site_problem(snapshot(L, M, sw, step))
    plan = plan_from_problem(gpu_ctx, prob, ts, site_of_step(L, step))
    x = np.random.default_rng(3).standard_normal(plan.n)
    y_kept = plan.apply(x)
    ev_kept, vec_kept, it_kept = jd_solve(plan, twin_vector(prob), 1e-10, 8)
    w_bytes = 8 * int(plan.info["w_len"])
    launches_kept = int(plan.info["launches"])
    for parts in (3, 17, 10 ** 9):  # the last one: every unit a chunk of its own
        plan.stream_coefficients(max(8, w_bytes // parts))
        assert int(plan.info["launches"]) > launches_kept
        assert np.array_equal(plan.apply(x), y_kept), parts
        ev, vec, it = jd_solve(plan, twin_vector(prob), 1e-10, 8)
        assert ev == ev_kept and it == it_kept and np.array_equal(vec, vec_kept)
    with pytest.raises(QcmError):
        plan.apply(x, precision="mixed")
    plan.stream_coefficients(0)
    assert int(plan.info["launches"]) == launches_kept
    assert np.array_equal(plan.apply(x), y_kept)


@pytest.mark.parametrize("kw", [dict(), dict(heev=dict(alpha_initial=1e-3, alpha_main=1e-6, alpha_final=0.0,
                                                        ngrowsweeps=1, nmainsweeps=1),
                                             optimization="singlesite", init_bond_dimension=8)])
def test_sweeps_do_not_depend_on_the_coefficient_budget(gpu_ctx, kw):
    from qcmaquis_b200.dmrg import DMRG
    L, M = 8, 32
    h, V, e, m, ts, blob = qc_system(L)
    out = []
    for budget in (0, 64 * 1024):
        d = DMRG(gpu_ctx, m, L // 2, L // 2, M, ecore=e, **kw)
        d.set_coefficient_budget(budget)
        out.append([d.sweep() for _ in range(3)])
    for (E0, T0), (E1, T1) in zip(*out):
        assert np.array_equal(E0, E1)
        assert T0 == T1
