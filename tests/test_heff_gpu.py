"""H_eff . psi on the B200 (C-ABI, DMMA FP64 kernels) against the oracle on frozen site problems."""
import numpy as np
import pytest

from qcmaquis_b200 import heff
from oracle.oracle import heff_apply

from helpers import qc_system, snapshot, site_of_step

pytestmark = pytest.mark.gpu

# (L, M, sweeps before, step, MPO sign gauge): left-to-right and right-to-left steps, ends and
# middle; the gauged MPO's Hermitian pairs carry phase -1 (conjugate scales of -1)
CASES = [(6, 16, 1, 0, None), (6, 16, 1, 2, None), (6, 16, 1, 7, None), (8, 64, 1, 3, None), (8, 64, 1, 10, None),
         (8, 64, 2, 12, None), (10, 48, 1, 4, None), (8, 64, 1, 3, 11), (10, 48, 1, 13, 5)]


def transposed_cohorts(b):
    """(transposed cohorts, blocks with conjugate scale != 1) of a boundary dict."""
    return int(np.sum(b["tr"])), int(np.sum(b["cscale"] != 1.0))


@pytest.mark.parametrize("L,M,sw,step,gauge", CASES)
def test_heff_matches_oracle(gpu_ctx, L, M, sw, step, gauge):
    snap = snapshot(L, M, sw, step, 0, gauge)
    h, V, e, m, ts, blob = qc_system(L, 0, gauge)
    site = site_of_step(L, step)
    p = heff.parse_site_problem(snap)
    if L >= 8:
        # the reference's storage: half the off-diagonal cohorts are transposed Hermitian partners
        ntr = [transposed_cohorts(p[k]) for k in ("L", "R")]
        assert ntr[0][0] > 0 and ntr[1][0] > 0
        if gauge is not None:
            assert ntr[0][1] + ntr[1][1] > 0
    plan = heff.plan_from_problem(gpu_ctx, p, ts, site)
    x0 = heff.twin_vector(p)
    rng = np.random.default_rng(step)
    for x in (x0, rng.standard_normal(x0.size)):
        y_ref, fl, _ = heff_apply(snap, blob, site, x)
        y = plan.apply(x)
        scale = np.abs(y_ref).max()
        assert np.abs(y - y_ref).max() <= 1e-12 * scale, (np.abs(y - y_ref).max(), scale)
        assert abs(plan.info["flops"] - fl) == 0
    # Rayleigh quotient of the current state agrees to 1e-12 relative
    e_ref = x0 @ heff_apply(snap, blob, site, x0)[0] / (x0 @ x0)
    e_gpu = x0 @ plan.apply(x0) / (x0 @ x0)
    assert abs(e_gpu - e_ref) <= 1e-12 * abs(e_ref)


def test_heff_deterministic_and_device_path(gpu_ctx):
    import torch
    L, M, sw, step = 8, 64, 1, 3
    snap = snapshot(L, M, sw, step)
    h, V, e, m, ts, blob = qc_system(L, 0)
    p = heff.parse_site_problem(snap)
    plan = heff.plan_from_problem(gpu_ctx, p, ts, site_of_step(L, step))
    x = np.random.default_rng(3).standard_normal(plan.n)
    y1 = plan.apply(x)
    y2 = plan.apply(x)
    assert np.array_equal(y1, y2)  # fixed reduction order, no atomics
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty_like(xd)
    torch.cuda.synchronize()
    plan.apply_device(xd.data_ptr(), yd.data_ptr())
    gpu_ctx.synchronize()
    assert np.array_equal(yd.cpu().numpy(), y1)


def test_heff_linear_symmetric(gpu_ctx):
    L, M, sw, step = 8, 64, 1, 10
    snap = snapshot(L, M, sw, step)
    h, V, e, m, ts, blob = qc_system(L, 0)
    p = heff.parse_site_problem(snap)
    plan = heff.plan_from_problem(gpu_ctx, p, ts, site_of_step(L, step))
    rng = np.random.default_rng(11)
    a, b = rng.standard_normal(plan.n), rng.standard_normal(plan.n)
    ya, yb = plan.apply(a), plan.apply(b)
    yab = plan.apply(2.0 * a - 0.5 * b)
    assert np.abs(yab - (2.0 * ya - 0.5 * yb)).max() <= 1e-12 * np.abs(yab).max()
    assert abs(a @ yb - b @ ya) <= 1e-12 * np.linalg.norm(a) * np.linalg.norm(yb)
    assert np.all(plan.apply(np.zeros(plan.n)) == 0.0)
