"""QC MPO (input prep): exactness against FCI spectra by dense contraction."""
import numpy as np
import pytest

from qcmaquis_b200.fcidump import synthetic_integrals, write_fcidump, read_fcidump
from qcmaquis_b200.mpo import MPO, dense_operator, parse_blob
from oracle.fci import FCI

from helpers import gauge_signed


def dense_mpo(ts):
    A, charges = None, None
    for t in ts:
        n = sum(s[2] for s in t["phys"])
        T = np.zeros((t["rows"], t["cols"], n, n))
        for b1, b2, op, sc in zip(t["b1"], t["b2"], t["op"], t["scale"]):
            T[b1, b2] += sc * dense_operator(t, op)
        ch = np.array([(a, b) for (a, b, sz) in t["phys"] for _ in range(sz)])
        if A is None:
            A, charges = T[0], ch
        else:
            A = np.einsum("bOI,bcoi->cOoIi", A, T)
            s = A.shape
            A = A.reshape(s[0], s[1] * s[2], s[3] * s[4])
            charges = (charges[:, None, :] + ch[None, :, :]).reshape(-1, 2)
    assert A.shape[0] == 1
    return A[0], charges


@pytest.mark.parametrize("L,seed", [(4, 3), (5, 1)])
def test_mpo_spectrum_matches_fci(L, seed):
    h, V, e = synthetic_integrals(L, seed)
    m = MPO.qc(h, V)
    H, ch = dense_mpo(m.tensors())
    assert np.abs(H - H.T).max() < 1e-12
    for nu, nd in [(L // 2, L // 2), (1, 2), (L - 1, 1)]:
        sel = np.where((ch[:, 0] == nu) & (ch[:, 1] == nd))[0]
        ev = np.sort(np.linalg.eigvalsh(H[np.ix_(sel, sel)]))
        evf = np.sort(np.linalg.eigvalsh(FCI(h, V, e, nu, nd).dense()))
        assert len(ev) == len(evf)
        assert np.abs(ev - evf).max() < 1e-11


def test_twosite_mpo_spectrum():
    L = 4
    h, V, e = synthetic_integrals(L, 5)
    ts = MPO.qc(h, V).twosite().tensors()
    assert len(ts) == L - 1 and all(t["twosite"] for t in ts)
    H, ch = dense_mpo([ts[0], ts[2]])
    sel = np.where((ch[:, 0] == 2) & (ch[:, 1] == 2))[0]
    ev = np.sort(np.linalg.eigvalsh(H[np.ix_(sel, sel)]))
    evf = np.sort(np.linalg.eigvalsh(FCI(h, V, e, 2, 2).dense()))
    assert np.abs(ev - evf).max() < 1e-11


def test_blob_roundtrip():
    h, V, e = synthetic_integrals(6, 2)
    m = MPO.qc(h, V)
    b = m.blob()
    assert MPO.from_blob(b).blob() == b
    t2 = MPO.from_blob(m.twosite().blob())
    assert len(t2) == 5
    ts = parse_blob(b)
    assert ts[0]["rows"] == 1 and ts[-1]["cols"] == 1
    for a, c in zip(ts[:-1], ts[1:]):
        assert a["cols"] == c["rows"]


def test_fcidump_roundtrip(tmp_path):
    h, V, e = synthetic_integrals(5, 4)
    p = tmp_path / "FCIDUMP"
    write_fcidump(str(p), h, V, e, nelec=5)
    h2, V2, e2 = read_fcidump(str(p))
    assert np.abs(h - h2).max() < 1e-14
    assert np.abs(V - V2).max() < 1e-14


def test_synthetic_recipe_properties():
    h, V, e = synthetic_integrals(6, 0)
    assert np.allclose(h, h.T)
    # 8-fold symmetry and PSD Coulomb matrix
    assert np.allclose(V, V.transpose(1, 0, 2, 3))
    assert np.allclose(V, V.transpose(2, 3, 0, 1))
    w = np.linalg.eigvalsh(V.reshape(36, 36))
    assert w.min() > -1e-12
    assert e == 0.0


def _left_parts(ts, p):
    """E[b, out, in]: the operator of bond index b on sites 0..p (dense)."""
    A = None
    for t in ts[:p + 1]:
        n = sum(s[2] for s in t["phys"])
        T = np.zeros((t["rows"], t["cols"], n, n))
        for b1, b2, op, sc in zip(t["b1"], t["b2"], t["op"], t["scale"]):
            T[b1, b2] += sc * dense_operator(t, op)
        if A is None:
            A = T[0]
        else:
            A = np.einsum("bOI,bcoi->cOoIi", A, T)
            s = A.shape
            A = A.reshape(s[0], s[1] * s[2], s[3] * s[4])
    return A


def _right_parts(ts, p):
    """F[b, out, in]: the operator of bond index b (bond after site p) on sites p+1..L-1 (dense)."""
    A = None
    for t in reversed(ts[p + 1:]):
        n = sum(s[2] for s in t["phys"])
        T = np.zeros((t["rows"], t["cols"], n, n))
        for b1, b2, op, sc in zip(t["b1"], t["b2"], t["op"], t["scale"]):
            T[b1, b2] += sc * dense_operator(t, op)
        if A is None:
            A = T[:, 0]
        else:
            A = np.einsum("bcoi,cOI->boOiI", T, A)
            s = A.shape
            A = A.reshape(s[0], s[1] * s[2], s[3] * s[4])
    return A


@pytest.mark.parametrize("L,seed", [(4, 1), (5, 2)])
def test_mpo_hermitian_pairs(L, seed):
    """Every operator-carrying bond index has a registered partner (or is self-adjoint) whose bond
    operators, on either side of the bond, are its transposes times the pair's phase: the property
    complement_transpose relies on (tagged_mpo_maker_optim.hpp:292-307, boundary.h:161-191)."""
    h, V, e = synthetic_integrals(L, seed)
    m = MPO.qc(h, V)
    ts = m.tensors()
    for p in range(L - 1):
        herm, phase = ts[p]["herm_right"][:, 0], ts[p]["herm_right"][:, 1]
        hl, pl, hr, pr = m.hermitian(p + 1)
        assert (hl == herm).all() and (pl == phase).all()
        assert (herm[herm >= 0][:, None] >= 0).all()
        for b in np.where(herm >= 0)[0]:
            assert herm[herm[b]] == b and phase[herm[b]] == phase[b]
        E, F = _left_parts(ts, p), _right_parts(ts, p)
        paired = np.where(herm >= 0)[0]
        # only the two operator-free indices (nothing placed / term complete) stay unregistered
        assert len(paired) == ts[p]["cols"] - 2
        for b in paired:
            c = herm[b]
            assert np.abs(E[b].T - phase[b] * E[c]).max() < 1e-12 * max(1.0, np.abs(E[b]).max())
            assert np.abs(F[b].T - phase[b] * F[c]).max() < 1e-12 * max(1.0, np.abs(F[b]).max())
        # the pairs are not trivial: most indices have a partner other than themselves
        assert (herm[paired] != paired).sum() > len(paired) // 2


def test_mpo_from_terms_roundtrip_and_gauge():
    """qcm_mpo_create / qcm_mpo_set_tensor rebuild the MPO exactly; a sign gauge on the bond indices
    leaves the Hamiltonian unchanged and gives phase -1 pairs."""
    L = 5
    h, V, e = synthetic_integrals(L, 3)
    m = MPO.qc(h, V)
    b = m.blob()
    assert MPO.from_tensors(parse_blob(b)).blob() == b
    t2 = m.twosite()
    assert MPO.from_tensors(parse_blob(t2.blob()), twosite=True).blob() == t2.blob()
    g = gauge_signed(m.tensors(), 7)
    mg = MPO.from_tensors(g)
    assert any((t["herm_right"][:, 1] < 0).any() for t in mg.tensors())
    H0, _ = dense_mpo(m.tensors())
    Hg, _ = dense_mpo(mg.tensors())
    assert np.abs(H0 - Hg).max() < 1e-12
    tg = mg.tensors()
    for p in range(L - 1):
        herm, phase = tg[p]["herm_right"][:, 0], tg[p]["herm_right"][:, 1]
        E = _left_parts(tg, p)
        for bb in np.where(herm >= 0)[0]:
            assert np.abs(E[bb].T - phase[bb] * E[herm[bb]]).max() < 1e-12 * max(1.0, np.abs(E[bb]).max())


def test_mpo_from_terms_rejects_bad_input():
    from qcmaquis_b200._lib import QcmError
    h, V, e = synthetic_integrals(4, 0)
    ts = MPO.qc(h, V).tensors()
    bad = dict(ts[1])
    hl = bad["herm_left"].copy()
    i = int(np.where(hl[:, 0] >= 0)[0][0])
    hl[i, 0] = (hl[i, 0] + 1) % len(hl)
    bad["herm_left"] = hl
    with pytest.raises(QcmError, match="not symmetric|phase"):
        MPO.from_tensors([ts[0], bad, ts[2], ts[3]])
    bad = dict(ts[1])
    bad["b1"] = bad["b1"].copy()
    bad["b1"][0] = bad["rows"]
    with pytest.raises(QcmError, match="out of range"):
        MPO.from_tensors([ts[0], bad, ts[2], ts[3]])
    import ctypes
    from qcmaquis_b200._lib import lib
    out = ctypes.c_void_p()
    assert lib.qcm_mpo_create(4, 0, ctypes.byref(out)) == 0
    part = MPO(out)
    part.set_tensor(0, ts[0])
    with pytest.raises(QcmError, match="never set"):
        part.blob()
    nb = [dict(t) for t in ts]
    nb[2] = dict(ts[2])
    nb[2]["herm_left"] = None
    with pytest.raises(QcmError, match="disagree"):
        MPO.from_tensors(nb).blob()
