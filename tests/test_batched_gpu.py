"""The batching form: independent site problems merged into one plan group (qcm_heff_group) -- one apply
for all, equal member by member to the separate applies, and a lockstep Jacobi-Davidson (each iteration a
CUDA graph) whose eigenpairs match the separate solves and the oracle's step energies."""
import numpy as np
import pytest

from qcmaquis_b200 import heff

from helpers import qc_system, snapshot, site_of_step

pytestmark = pytest.mark.gpu

# (L, M, sweeps before, step, integral seed): problems of different sizes and Hamiltonians
MEMBERS = [(6, 16, 1, 2, 1), (8, 32, 1, 3, 2), (8, 32, 1, 10, 3), (6, 16, 1, 7, 4), (8, 32, 1, 5, 5)]


def members(ctx):
    plans, xs, snaps = [], [], []
    for (L, M, sw, step, seed) in MEMBERS:
        snap = snapshot(L, M, sw, step, seed)
        h, V, e, m, ts, blob = qc_system(L, seed)
        p = heff.parse_site_problem(snap)
        plans.append(heff.plan_from_problem(ctx, p, ts, site_of_step(L, step)))
        xs.append(heff.twin_vector(p))
        snaps.append((snap, blob, site_of_step(L, step)))
    return plans, xs, snaps


def test_group_apply_equals_member_applies(gpu_ctx):
    plans, xs, _ = members(gpu_ctx)
    g = heff.HeffGroup(gpu_ctx, plans)
    assert g.info["flops"] == sum(p.info["flops"] for p in plans)
    rng = np.random.default_rng(0)
    ins = [rng.standard_normal(x.size) for x in xs]
    ys = g.unpack(g.apply(g.pack(ins)))
    for p, x, y in zip(plans, ins, ys):
        assert np.array_equal(y, p.apply(x))  # same kernels and summation order, member by member
    # the arena's gaps come back as zeros
    out = g.apply(g.pack(ins))
    mask = np.ones(g.n, bool)
    for o, l in zip(g.offsets, g.lengths):
        mask[int(o):int(o) + int(l)] = False
    assert np.all(out[mask] == 0.0)


@pytest.mark.parametrize("graphs", [True, False])
def test_batched_jd_matches_separate_solves(gpu_ctx, graphs):
    from qcmaquis_b200.dmrg import jd_solve
    from oracle.oracle import OracleDMRG
    plans, xs, snaps = members(gpu_ctx)
    g = heff.HeffGroup(gpu_ctx, plans)
    ev, out, it, napply = g.jd_solve(g.pack(xs), 1e-10, 8, graphs=graphs)
    vecs = g.unpack(out)
    for k, (p, x, v) in enumerate(zip(plans, xs, vecs)):
        e1, v1, it1 = jd_solve(p, x, 1e-10, 8)
        # the same Krylov-type subspace (t = -r + (r.u)/(u.u) u), orthogonalised differently
        assert abs(ev[k] - e1) <= 1e-10 * abs(e1), (k, ev[k] - e1)
        assert abs(int(it[k]) - it1) <= 1, (k, it[k], it1)
        assert abs(np.linalg.norm(v) - 1.0) < 1e-12
        assert abs(v @ p.apply(v) - ev[k]) <= 1e-9 * abs(ev[k])
    assert napply == int(it.max())
    # the oracle's step energies of the same problems
    for k, (L, M, sw, step, seed) in enumerate(MEMBERS):
        h, V, e, m, ts, blob = qc_system(L, seed)
        d = OracleDMRG(blob, L, L // 2, L // 2, M)
        for s in range(sw):
            d.sweep(s)
        assert abs(ev[k] - d.sweep(sw)[0][step]) < 1e-10


def test_batched_jd_graphs_replay_bitwise(gpu_ctx):
    plans, xs, _ = members(gpu_ctx)
    g = heff.HeffGroup(gpu_ctx, plans)
    a = g.jd_solve(g.pack(xs), 1e-10, 8, graphs=True)
    b = g.jd_solve(g.pack(xs), 1e-10, 8, graphs=False)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
