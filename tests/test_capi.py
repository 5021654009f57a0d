"""C-ABI: symbol export, error behaviour, and host-side schedule parity with the oracle."""
import ctypes
import os
import re

import numpy as np
import pytest

import qcmaquis_b200
from qcmaquis_b200 import _lib, heff
from oracle.oracle import schedule_export

from helpers import qc_system, snapshot, site_of_step, parse_schedule_export

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names += re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(qcm_[a-z_0-9]+)\s*\(", txt, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    names = declared_symbols()
    assert len(names) >= 15
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_errors_are_status_codes():
    out = ctypes.c_void_p()
    rc = _lib.lib.qcm_mpo_build_qc(1, None, None, 0.0, ctypes.byref(out))
    assert rc == -1 and "bad arguments" in _lib.lib.qcm_last_error().decode()
    rc = _lib.lib.qcm_mpo_deserialize(b"garbage!" * 4, 32, ctypes.byref(out))
    assert rc < 0
    assert qcmaquis_b200.version().startswith("qcm_b200")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="only meaningful without a GPU")
def test_ctx_create_without_gpu_fails_loudly():
    with pytest.raises(_lib.QcmError, match="status -5"):
        heff.Context(0)


@pytest.mark.parametrize("L,M,sw,step", [(6, 16, 1, 0), (6, 16, 1, 5), (8, 64, 1, 3), (8, 64, 2, 11)])
def test_schedule_bookkeeping_matches_oracle(L, M, sw, step):
    """Host plan == oracle schedule: same cohorts, units, lines, T slices and coefficients."""
    snap = snapshot(L, M, sw, step)
    h, V, e, m, ts, blob = qc_system(L, 0)
    site = site_of_step(L, step)
    p = heff.parse_site_problem(snap)
    Lb, Rb = heff.Boundary(None, p["L"]), heff.Boundary(None, p["R"])
    plan = heff.HeffPlan(None, Lb, Rb, ts, site, p["phys"], p["left"], p["right"], bookkeeping=True)
    ints, al = plan.bookkeeping()
    sch, fl = schedule_export(snap, blob, site)
    ro = sorted(parse_schedule_export(sch))
    rp = sorted([tuple(int(v) for v in r) + (a,) for r, a in zip(ints, al)])
    assert len(ro) == len(rp) > 0
    assert [r[:10] for r in ro] == [r[:10] for r in rp]
    assert max(abs(a[10] - b[10]) for a, b in zip(ro, rp)) <= 1e-15 * max(abs(a[10]) for a in ro)
    assert plan.info["flops"] == fl
    if L == 8:
        # the Hermitian-paired MPO stores half the off-diagonal cohorts: transposed ones are read
        assert any(r[2] != r[3] for r in ro)
    with pytest.raises(_lib.QcmError, match="host-only"):
        plan.apply(np.zeros(plan.n))


def test_package_modules_import():
    import importlib
    for m in ("qcmaquis_b200.heff", "qcmaquis_b200.dmrg", "qcmaquis_b200.mpo", "qcmaquis_b200.fcidump"):
        importlib.import_module(m)
