"""Boundary residency (qcm_dmrg_set_boundary_budget): boundaries no later step reads are released after every
step, and under a device budget the others move to pinned host memory and back.  The sweeps must not depend
on it: the same energies and truncations, bit for bit, with a budget that leaves only the next step's two
boundaries on the device, in two-site and single-site sweeps, and the pending step's site problem the same."""
import numpy as np
import pytest

from helpers import qc_system

pytestmark = pytest.mark.gpu

NOISE = dict(alpha_initial=1e-3, alpha_main=1e-6, alpha_final=0.0, ngrowsweeps=1, nmainsweeps=1)


def sweeps(ctx, L, M, n, budget, **kw):
    from qcmaquis_b200.dmrg import DMRG
    h, V, e, m, ts, blob = qc_system(L)
    d = DMRG(ctx, m, L // 2, L // 2, M, ecore=e, **kw)
    if budget is not None:
        d.set_boundary_budget(budget)
    out = [d.sweep() for _ in range(n)]
    return d, out, d.stats()


@pytest.mark.parametrize("kw", [dict(), dict(heev=NOISE, optimization="singlesite", init_bond_dimension=8)])
def test_sweeps_do_not_depend_on_the_boundary_budget(gpu_ctx, kw):
    L, M, n = 8, 32, 3
    d0, ref, st0 = sweeps(gpu_ctx, L, M, n, None, **kw)
    d1, out, st1 = sweeps(gpu_ctx, L, M, n, 1, **kw)
    for (E0, T0), (E1, T1) in zip(ref, out):
        assert np.array_equal(E0, E1)
        assert T0 == T1
    assert st0["boundaries_offloaded"] == 0 and st0["boundaries_fetched"] == 0
    assert st1["boundaries_offloaded"] > 0 and st1["boundaries_fetched"] > 0
    assert st1["boundary_bytes_peak"] < st0["boundary_bytes_peak"]


def test_pending_problem_after_offload(gpu_ctx):
    """Halfway through a sweep with everything but the pending step's boundaries in host memory, the pending
    site problem (plan and start vector) applies exactly as without a budget."""
    from qcmaquis_b200.dmrg import DMRG
    L, M = 8, 32
    h, V, e, m, ts, blob = qc_system(L)
    runs = []
    for budget in (None, 1):
        d = DMRG(gpu_ctx, m, L // 2, L // 2, M)
        if budget:
            d.set_boundary_budget(budget)
        d.sweep()
        d.run(L + 1)
        plan, x = d.pending_plan()
        runs.append((d, plan.apply(x), x))
    assert np.array_equal(runs[0][2], runs[1][2])
    assert np.array_equal(runs[0][1], runs[1][1])
    assert runs[1][0].stats()["boundaries_offloaded"] > 0
