"""Single-site optimiser (optimization = singlesite; ss_optimize.hpp:59-186): 2L steps per sweep, each site
solved with its single-site MPO tensor, then grown by the density-matrix prediction with noise alpha
(grow_l2r_sweep / grow_r2l_sweep, contractions/engine.hpp:85-123; prediction.hpp:41-148).  The oracle is
pinned against FCI and the device against the oracle step by step."""
import functools

import numpy as np
import pytest

from oracle.oracle import OracleDMRG
from oracle.fci import FCI

from helpers import qc_system

L_SS = 6
NOISE = dict(alpha_initial=1e-3, alpha_main=1e-5, alpha_final=1e-8, ngrowsweeps=2, nmainsweeps=2)


@functools.lru_cache(maxsize=None)
def fci_levels(L):
    h, V, e, m, ts, blob = qc_system(L)
    return FCI(h, V, e, L // 2, L // 2).lowest(2)


def oracle_ss(L, M, init_bd, cutoff=1e-16):
    h, V, e, m, ts, blob = qc_system(L)
    g = OracleDMRG(blob, L, L // 2, L // 2, M, init_bond_dimension=init_bd, cutoff=cutoff)
    g.set_heev(True, **NOISE)
    g.set_single_site(True)
    return g


def test_oracle_single_site_reaches_fci():
    """From an init_bond_dimension 4 state the growth with noise raises the bond dimensions and the sweeps
    reach the FCI ground state (M = 64 is exact for L = 6)."""
    L = L_SS
    w = fci_levels(L)
    g = oracle_ss(L, 64, 4)
    dims = []
    for s in range(8):
        E, tw, tf, bd = g.sweep(s)
        assert E.size == 2 * L
        dims.append(int(bd.max()))
        # the steps that end a half-sweep canonise without truncation
        assert bd[L - 1] == 0 and bd[2 * L - 1] == 0
    assert dims[0] > 4
    assert abs(E.min() - w[0]) < 1e-9, E.min() - w[0]
    # the Rayleigh quotients of a converged sweep stay within the JD tolerance of each other
    assert E.max() - E.min() < 1e-8


def test_oracle_single_site_bounded_by_mmax():
    g = oracle_ss(L_SS, 8, 4)
    for s in range(3):
        E, tw, tf, bd = g.sweep(s)
        assert bd.max() <= 8 + 2  # Mmax plus the ties estimate_truncation keeps
    assert tw[: L_SS - 1].max() > 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("M,cutoff", [(64, 1e-7), (12, 1e-7)])
def test_device_single_site_matches_oracle(gpu_ctx, M, cutoff):
    """Both engines from the oracle's init_bond_dimension 4 MPS: every step's energy to 1e-10 Eh and the
    same kept dimensions over four sweeps (growth, main and final noise), with and without Mmax binding."""
    from qcmaquis_b200.dmrg import DMRG
    from qcmaquis_b200.heff import parse_mps_tensor
    L = L_SS
    h, V, e, m, ts, blob = qc_system(L)
    ref = oracle_ss(L, M, 4, cutoff)
    sites = [parse_mps_tensor(ref.mps_export(i)) for i in range(L)]
    dev = DMRG.from_mps(gpu_ctx, m, sites, M, truncation_cutoff=cutoff, heev=NOISE, optimization="singlesite")
    assert dev.steps == 2 * L
    for s in range(4):
        E_ref, tw_ref, tf_ref, bd_ref = ref.sweep(s)
        E, tr = dev.sweep()
        assert np.abs(E - E_ref).max() < 1e-10, (s, np.abs(E - E_ref).max())
        assert np.array_equal(np.array([t["bond_dimension"] for t in tr]), bd_ref.astype(np.int64)), s
        # heev_truncate reports the truncated fraction, a sum of square roots of the discarded eigenvalues:
        # where those are at the rounding level of the density matrix (1e-16 of its largest) the two
        # eigensolvers' roundings show up as ~1e-8 in the fraction
        tw = np.array([t["truncated_weight"] for t in tr])
        assert np.allclose(tw, tw_ref, rtol=1e-6, atol=1e-6), s
    assert int(dev.stats()["hpsi_count"]) == int(ref.stats()["hpsi_count"])


@pytest.mark.gpu
def test_device_single_site_reaches_fci(gpu_ctx):
    """Const initial state at init_bond_dimension 8, single-site sweeps on the device: the FCI ground state
    to 1e-9, and the 1-RDM of the converged state equals the two-site DMRG's."""
    from qcmaquis_b200.dmrg import DMRG
    L = L_SS
    h, V, e, m, ts, blob = qc_system(L)
    w = fci_levels(L)
    d = DMRG(gpu_ctx, m, L // 2, L // 2, 64, init_bond_dimension=8, heev=NOISE, optimization="singlesite")
    for _ in range(8):
        E, tr = d.sweep()
    assert E.size == 2 * L
    assert abs(E.min() - w[0]) < 1e-9, E.min() - w[0]
    t = DMRG(gpu_ctx, m, L // 2, L // 2, 64)
    for _ in range(4):
        E2, _ = t.sweep()
    assert np.abs(d.measure_1rdm() - t.measure_1rdm()).max() < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("precision,gmres", [("mixed", 0), ("fp64", 4)])
def test_device_single_site_forms(gpu_ctx, precision, gmres):
    """The single-site sweep with the mixed H.psi (FP64 Rayleigh quotient per step) and with GMRES(4)
    corrections: the FCI ground state to 1e-8."""
    from qcmaquis_b200.dmrg import DMRG
    L = L_SS
    h, V, e, m, ts, blob = qc_system(L)
    w = fci_levels(L)
    d = DMRG(gpu_ctx, m, L // 2, L // 2, 64, init_bond_dimension=8, heev=NOISE, optimization="singlesite",
             precision=precision, jcd_gmres=gmres)
    for _ in range(8):
        E, tr = d.sweep()
    assert abs(E.min() - w[0]) < 1e-8, E.min() - w[0]


@pytest.mark.gpu
def test_device_single_site_excited_state_matches_oracle(gpu_ctx):
    """Single-site sweeps kept orthogonal to a ground state (ss_optimize.hpp:104-109): step energies equal
    the oracle's and converge to the first excited FCI level.  Near the chain's end the density matrix is
    rank-deficient; the cutoff 1e-7 drops its rounding-level eigenvectors, which each eigensolver would
    choose differently (with 1e-16 they are kept and enlarge the next site's space arbitrarily)."""
    from qcmaquis_b200.dmrg import DMRG
    from qcmaquis_b200.heff import parse_mps_tensor
    L = L_SS
    h, V, e, m, ts, blob = qc_system(L)
    w = fci_levels(L)
    g = OracleDMRG(blob, L, L // 2, L // 2, 64)
    for s in range(4):
        g.sweep(s)
    gs = [g.mps_export(i) for i in range(L)]
    ref = oracle_ss(L, 64, 8, 1e-7)
    ref.set_ortho([gs])
    sites = [parse_mps_tensor(ref.mps_export(i)) for i in range(L)]
    dev = DMRG.from_mps(gpu_ctx, m, sites, 64, truncation_cutoff=1e-7, heev=NOISE, optimization="singlesite")
    dev.set_ortho([[parse_mps_tensor(b) for b in gs]])
    for s in range(8):
        E_ref = ref.sweep(s)[0]
        E, _ = dev.sweep()
        assert np.abs(E - E_ref).max() < 1e-9, (s, np.abs(E - E_ref).max())
    assert abs(E.min() - w[1]) < 1e-8, E.min() - w[1]


@pytest.mark.gpu
def test_device_single_site_rejects_two_site_queries(gpu_ctx):
    import ctypes
    from qcmaquis_b200 import _lib
    from qcmaquis_b200.dmrg import DMRG, _params
    L = L_SS
    h, V, e, m, ts, blob = qc_system(L)
    d = DMRG(gpu_ctx, m, L // 2, L // 2, 16, optimization="singlesite")
    with pytest.raises(RuntimeError, match="two-site sweeps only"):
        d.pending_plan()
    with pytest.raises(ValueError):
        _params(16, 16, 1e-16, 1e-10, 8, 0.0, None, optimization="threesite")
    p = _params(16, 16, 1e-16, 1e-10, 8, 0.0, None)
    p.optimization = 7
    h_out = ctypes.c_void_p()
    assert _lib.lib.qcm_dmrg_create(gpu_ctx.h, m.handle, L // 2, L // 2, ctypes.byref(p), ctypes.byref(h_out)) != 0
