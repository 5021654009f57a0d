"""The allocation-free H_eff entry point (qcm_heff_apply_device_noalloc) through the C-ABI.

It exists for host codes that cannot call cudaMalloc where they need H.psi (their
HBM belongs to their own caching allocator, or their solver loop must not stall
on cudaFree's device-wide synchronisation).  Its scratch is the library's fixed
64 MiB device array instead of the plan's own buffers; the result must equal the
regular device apply's, call after call (the array keeps the previous call's
contents, so a stale buffer would show on the second call).  Collected last so a
run that stops at the first failure has already run every other test.
"""
import numpy as np
import pytest

from qcmaquis_b200 import heff

from helpers import qc_system, snapshot, site_of_step

pytestmark = pytest.mark.gpu


def _round32(n):
    return (n + 31) // 32 * 32


@pytest.mark.parametrize("L,M,sw,step", [(8, 64, 1, 3), (6, 16, 1, 7)])
def test_noalloc_matches_device_apply_twice(gpu_ctx, L, M, sw, step):
    import torch
    snap = snapshot(L, M, sw, step)
    h, V, e, m, ts, blob = qc_system(L, 0)
    p = heff.parse_site_problem(snap)
    plan = heff.plan_from_problem(gpu_ctx, p, ts, site_of_step(L, step))
    need = sum(_round32(plan.info[k]) for k in ("t_len", "s_len", "p_len"))
    assert 0 < need <= heff.NOALLOC_SCRATCH_DOUBLES
    rng = np.random.default_rng(5)
    xs = [torch.from_numpy(rng.standard_normal(plan.n)).cuda() for _ in range(3)]
    ys = [torch.empty_like(x) for x in xs]
    y_refs = [torch.empty_like(x) for x in xs]
    for x, y_ref in zip(xs, y_refs):
        plan.apply_device(x.data_ptr(), y_ref.data_ptr())
    gpu_ctx.synchronize()

    def noalloc_call(i):
        ys[i].fill_(float("nan"))
        torch.cuda.synchronize()
        plan.apply_device_noalloc(xs[i].data_ptr(), ys[i].data_ptr())
        gpu_ctx.synchronize()
        a, b = ys[i].cpu().numpy(), y_refs[i].cpu().numpy()
        assert np.all(np.isfinite(a))
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()

    # a first call (with the same checks) lets every module these calls and the checks use load
    # (CUDA loads kernels lazily, each module taking device memory at its first launch)
    noalloc_call(0)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for i in (1, 2):  # two calls in a row, different inputs
        noalloc_call(i)
    # nothing was allocated on the device by the two calls
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
