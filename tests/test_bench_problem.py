"""The bench's frozen problem: the oracle's site problem built from a given MPS (no optimisation) equals the
one its own sweep reaches, and the bench's synthetic MPS over recorded bond sectors is well formed."""
import importlib.util
import os

import numpy as np
import pytest

from qcmaquis_b200.heff import parse_mps_tensor, parse_site_problem
from oracle.oracle import OracleDMRG, site_problem, mpo_blob_qc

from helpers import qc_system

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def bench_module():
    spec = importlib.util.spec_from_file_location("qcm_bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _same_problem(a, b):
    pa, pb = parse_site_problem(a), parse_site_problem(b)
    for k in ("phys", "left", "right"):
        assert pa[k] == pb[k]
    assert [c for c, _ in pa["blocks"]] == [c for c, _ in pb["blocks"]]
    for (_, x), (_, y) in zip(pa["blocks"], pb["blocks"]):
        assert np.array_equal(x, y)
    for k in ("L", "R"):
        for f in ("cohort_bra", "cohort_ket", "tr", "n_blocks", "offsets", "cscale"):
            assert np.array_equal(pa[k][f], pb[k][f]), (k, f)
        assert np.abs(pa[k]["data"] - pb[k]["data"]).max() <= 1e-13 * np.abs(pb[k]["data"]).max()


def test_site_problem_from_mps_equals_sweep_snapshot():
    L, M, step = 8, 32, 3
    h, V, e, m, ts, blob = qc_system(L)
    d = OracleDMRG(blob, L, 4, 4, M)
    d.sweep(0)
    snap = d.snapshot(1, step)  # the sweep stopped before solving `step`
    sites = [d.mps_export(i) for i in range(L)]
    _same_problem(site_problem(blob, sites, step), snap)
    # the MPO built inside the oracle library is the package's
    assert mpo_blob_qc(h, V) == blob


def test_bench_synthetic_mps_and_problem():
    """The bench's MPS over the bond sectors of a converged state: one block per left sector, blocks
    matching the site's indices; its twin as the QSPB twin vector; QMPS blobs read back unchanged."""
    bench = bench_module()
    L, M = 8, 32
    h, V, e, m, ts, blob = qc_system(L)
    d = OracleDMRG(blob, L, 4, 4, M)
    d.sweep(0)
    ref = [parse_mps_tensor(d.mps_export(i)) for i in range(L)]
    phys = [tuple(p) for p in ref[0]["phys"]]
    bonds = [[tuple(s) for s in ref[0]["left"]]] + [[tuple(s) for s in r["right"]] for r in ref]
    sites = bench.synthetic_mps(phys, bonds, 5)
    for s, r in zip(sites, ref):
        back = parse_mps_tensor(bench.qmps_blob(s))
        assert back["left"] == [tuple(x) for x in r["left"]] and back["right"] == [tuple(x) for x in r["right"]]
        assert [b.shape for _, b in back["blocks"]] == [b.shape for _, b in r["blocks"]]
        for (_, x), (_, y) in zip(back["blocks"], s["blocks"]):
            assert np.array_equal(x, y)
    snap = site_problem(blob, [bench.qmps_blob(s) for s in sites], L // 2 - 1)
    p = parse_site_problem(snap)
    x = bench.twin_of_problem(snap)
    assert np.array_equal(x, np.concatenate([b.T.ravel() for _, b in p["blocks"]]))
    assert p["L"]["tr"].sum() > 0 and p["R"]["tr"].sum() > 0
    # same seed, same tensors
    again = bench.synthetic_mps(phys, bonds, 5)
    assert all(np.array_equal(x[1], y[1]) for s1, s2 in zip(sites, again) for x, y in zip(s1["blocks"], s2["blocks"]))


def test_bench_sector_fixtures_well_formed():
    """Every committed bond-sector fixture: L + 1 bonds from the vacuum to (N/2, N/2), bond dimensions at most
    M (plus the one degenerate state the truncation may keep), each bond's sectors reachable from the
    previous or the next bond's through one site's physical states (TwoU1 charges; a sector the truncation
    of the neighbouring bond cut off on one side may stay on the other), and the recorded sweep energies
    decreasing."""
    import glob
    import json
    files = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "bench_sectors_L*_M*.json")))
    assert len(files) >= 4
    for f in files:
        d = json.load(open(f))
        L, M, bonds, phys = d["L"], d["M"], d["bonds"], [tuple(p[:2]) for p in d["phys"]]
        assert len(bonds) == L + 1, f
        assert [tuple(s[:2]) for s in bonds[0]] == [(0, 0)] and [tuple(s[:2]) for s in bonds[-1]] == [(L // 2, L // 2)]
        for i in range(1, L):
            assert sum(s[2] for s in bonds[i]) <= M + 1, f
            fwd = {(a[0] + p[0], a[1] + p[1]) for a in bonds[i - 1] for p in phys}
            bwd = {(a[0] - p[0], a[1] - p[1]) for a in bonds[i + 1] for p in phys}
            assert all(tuple(s[:2]) in fwd or tuple(s[:2]) in bwd for s in bonds[i]), (f, i)
        E = d["energies_min_per_sweep"]
        assert all(e1 <= e0 + 1e-9 for e0, e1 in zip(E, E[1:])), f


@pytest.mark.gpu
def test_device_problem_from_mps_matches_oracle(gpu_ctx):
    """qcm_dmrg_create_from_mps_at on the bench's synthetic MPS (boundaries built on the device from the given
    MPS, Hermitian-paired) gives the oracle's site problem: same twin, same H.psi to 1e-12."""
    from oracle.oracle import heff_apply
    from qcmaquis_b200.dmrg import DMRG
    bench = bench_module()
    L, M = 8, 32
    h, V, e, m, ts, blob = qc_system(L)
    d = OracleDMRG(blob, L, 4, 4, M)
    d.sweep(0)
    ref = [parse_mps_tensor(d.mps_export(i)) for i in range(L)]
    phys = [tuple(p) for p in ref[0]["phys"]]
    bonds = [[tuple(s) for s in ref[0]["left"]]] + [[tuple(s) for s in r["right"]] for r in ref]
    sites = bench.synthetic_mps(phys, bonds, 9)
    for site1 in (0, L // 2 - 1, L - 2):
        snap = site_problem(blob, [bench.qmps_blob(s) for s in sites], site1)
        x_or = bench.twin_of_problem(snap)
        dev = DMRG.from_mps(gpu_ctx, m, sites, M, initial_site=site1)
        assert dev.next_step == site1
        plan, x = dev.pending_plan()
        assert np.abs(x - x_or).max() <= 1e-14 * np.abs(x_or).max()
        y = plan.apply(x_or)
        y_ref, fl, _ = heff_apply(snap, blob, site1, x_or)
        assert plan.info["flops"] == fl
        assert np.abs(y - y_ref).max() <= 1e-12 * np.abs(y_ref).max()
        del plan, dev
