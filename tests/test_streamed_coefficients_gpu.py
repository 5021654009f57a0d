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


@pytest.mark.parametrize("L,M,sw,step", [(8, 32, 1, 3), (10, 48, 1, 4)])
def test_sector_chunked_apply_is_the_whole_apply(gpu_ctx, L, M, sw, step):
    """The apply cut by ket sector (qcm_heff_chunk_apply): T, coefficient blocks, S and the split-K partials of
    a chunk of ket sectors at a time, the partials summed at the end.  The same H.psi and JD to the bit at
    every chunk size down to one ket sector per chunk, and back."""
    from qcmaquis_b200._lib import QcmError
    from qcmaquis_b200.dmrg import jd_solve
    from qcmaquis_b200.heff import parse_site_problem, plan_from_problem, twin_vector
    h, V, e, m, ts, blob = qc_system(L)
    prob = parse_site_problem(snapshot(L, M, sw, step))
    plan = plan_from_problem(gpu_ctx, prob, ts, site_of_step(L, step))
    x = np.random.default_rng(4).standard_normal(plan.n)
    y_whole = plan.apply(x)
    ev_whole, vec_whole, it_whole = jd_solve(plan, twin_vector(prob), 1e-10, 8)
    i = plan.info
    whole = 8 * (int(i["t_len"]) + int(i["s_len"]) + int(i["w_len"]))
    launches_whole = int(i["launches"])
    for parts in (2, 5, 10 ** 9):
        plan.chunk_apply(max(8, whole // parts))
        assert int(plan.info["launches"]) > launches_whole
        assert np.array_equal(plan.apply(x), y_whole), parts
        ev, vec, it = jd_solve(plan, twin_vector(prob), 1e-10, 8)
        assert ev == ev_whole and it == it_whole and np.array_equal(vec, vec_whole)
    with pytest.raises(QcmError):
        plan.apply(x, precision="mixed")
    plan.chunk_apply(0)
    assert np.array_equal(plan.apply(x), y_whole)


def test_sweeps_do_not_depend_on_the_apply_budget(gpu_ctx):
    from qcmaquis_b200.dmrg import DMRG
    L, M = 8, 32
    h, V, e, m, ts, blob = qc_system(L)
    out = []
    for budget in (0, 256 * 1024):
        d = DMRG(gpu_ctx, m, L // 2, L // 2, M, ecore=e)
        d.set_apply_budget(budget)
        out.append([d.sweep() for _ in range(3)])
    for (E0, T0), (E1, T1) in zip(*out):
        assert np.array_equal(E0, E1)
        assert T0 == T1


def test_chunked_apply_at_the_bench_bond_shapes(gpu_ctx):
    """The bench's frozen L=16, M=256 middle-bond problem (its L.S output tiles take all three row shapes, whose
    split-K partials a chunked apply keeps apart until the end): chunked applies at two and eight chunks and
    the streamed coefficient blocks give the whole apply to the bit."""
    import argparse
    import importlib.util
    import os
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    spec = importlib.util.spec_from_file_location("qcm_bench", os.path.join(root, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    a = argparse.Namespace(L=16, M=256, seed=0)
    h, V, sites, site1, fixture = bench.problem_inputs(a)
    d, plan, x, mpo = bench.device_problem(gpu_ctx, h, V, sites, site1, a.M)
    y = plan.apply(x)
    i = plan.info
    whole = 8 * (int(i["t_len"]) + int(i["s_len"]) + int(i["w_len"]))
    for parts in (2, 8):
        plan.chunk_apply(whole // parts)
        assert np.array_equal(plan.apply(x), y), parts
    plan.chunk_apply(0)
    plan.stream_coefficients(8 * int(i["w_len"]) // 4)
    assert np.array_equal(plan.apply(x), y)
    plan.stream_coefficients(0)
    assert np.array_equal(plan.apply(x), y)


def test_chunked_apply_keeping_the_coefficient_blocks(gpu_ctx):
    """A budget of at least twice the coefficient blocks keeps them whole (generated once, no generation
    launches in the apply) while T and S still run in chunks: the same apply to the bit."""
    from qcmaquis_b200.heff import parse_site_problem, plan_from_problem
    L, M, sw, step = 10, 48, 1, 4
    h, V, e, m, ts, blob = qc_system(L)
    prob = parse_site_problem(snapshot(L, M, sw, step))
    plan = plan_from_problem(gpu_ctx, prob, ts, site_of_step(L, step))
    x = np.random.default_rng(5).standard_normal(plan.n)
    y = plan.apply(x)
    i = plan.info
    w, tsb = 8 * int(i["w_len"]), 8 * (int(i["t_len"]) + int(i["s_len"]))
    plan.chunk_apply(w + tsb // 3 if w + tsb // 3 >= 2 * w else 2 * w + tsb // 3)
    assert np.array_equal(plan.apply(x), y)
    plan.chunk_apply(0)
