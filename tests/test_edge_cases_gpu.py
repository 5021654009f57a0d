"""Edge cases of whole device sweeps against exact diagonalisation: the shortest chains (one two-site step per
half-sweep), empty and full orbitals (a single determinant), odd electron counts, a bond dimension of one,
and the single-site optimiser at the shortest length."""
import numpy as np
import pytest

from oracle.fci import FCI

from helpers import qc_system

pytestmark = pytest.mark.gpu

NOISE = dict(alpha_initial=1e-3, alpha_main=1e-6, alpha_final=0.0, ngrowsweeps=1, nmainsweeps=1)


def fci_energy(h, V, e, nup, ndown):
    return float(np.linalg.eigvalsh(FCI(h, V, e, nup, ndown).dense())[0])


@pytest.mark.parametrize("L,nup,ndown", [(2, 1, 1), (2, 2, 1), (3, 2, 1), (4, 0, 1), (4, 4, 4), (4, 4, 3), (5, 1, 0)])
def test_exact_sweeps_at_the_edges(gpu_ctx, L, nup, ndown):
    from qcmaquis_b200.dmrg import DMRG
    h, V, e, m, ts, blob = qc_system(L)
    E_fci = fci_energy(h, V, e, nup, ndown)
    d = DMRG(gpu_ctx, m, nup, ndown, 64, ecore=e)
    assert d.steps == 2 * L - 2
    for _ in range(3):
        E, tr = d.sweep()
    assert abs(E.min() - E_fci) < 1e-10, (E.min(), E_fci)
    assert np.all(np.isfinite(E))


def test_bond_dimension_one_follows_the_oracle(gpu_ctx):
    """M = 1 from the oracle's initial MPS: step energies and bond dimensions as the oracle's (the cut keeps the
    singular values tied with the M-th, so the spin-flip partner of a sector's state stays with it and bonds
    hold up to two states); the energy stays above the exact one."""
    from oracle.oracle import OracleDMRG
    from qcmaquis_b200.dmrg import DMRG
    from qcmaquis_b200.heff import parse_mps_tensor
    L, M = 6, 1
    h, V, e, m, ts, blob = qc_system(L)
    ref = OracleDMRG(blob, L, L // 2, L // 2, M)
    sites = [parse_mps_tensor(ref.mps_export(i)) for i in range(L)]
    dev = DMRG.from_mps(gpu_ctx, m, sites, M)
    for s in range(3):
        E_ref, tw_ref, tf_ref, bd_ref = ref.sweep(s)
        E, tr = dev.sweep()
        assert np.abs(E - E_ref).max() < 1e-10, (s, E - E_ref)
        assert [t["bond_dimension"] for t in tr] == list(bd_ref.astype(int))
        assert max(t["bond_dimension"] for t in tr) <= 2
    assert E.min() > fci_energy(h, V, 0.0, L // 2, L // 2)


@pytest.mark.parametrize("L,nup,ndown", [(2, 1, 1), (3, 1, 2)])
def test_single_site_at_the_shortest_lengths(gpu_ctx, L, nup, ndown):
    from qcmaquis_b200.dmrg import DMRG
    h, V, e, m, ts, blob = qc_system(L)
    d = DMRG(gpu_ctx, m, nup, ndown, 64, init_bond_dimension=8, ecore=e, heev=NOISE, optimization="singlesite")
    assert d.steps == 2 * L
    for _ in range(4):
        E, tr = d.sweep()
    assert abs(E.min() - fci_energy(h, V, e, nup, ndown)) < 1e-10
