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


def test_tracked_mpo_provenance_and_dense_gradient():
    """The QC MPO with integral provenance: the records reproduce every entry's scale, zero integrals keep
    their entries, the Hamiltonian is the plain MPO's, and the entry gradients of the FCI ground state (dense
    contraction, c^T dH/d scale_e c) summed through the records give dE/dh = the FCI one-particle density
    matrix and sum h dh + sum V dV = E - ecore."""
    L = 4
    h, V, e = synthetic_integrals(L, 3)
    h[0, 3] = h[3, 0] = 0.0
    for (p, q, r, s) in ((0, 1, 2, 3), (1, 0, 2, 3), (0, 1, 3, 2), (1, 0, 3, 2),
                         (2, 3, 0, 1), (3, 2, 0, 1), (2, 3, 1, 0), (3, 2, 1, 0)):
        V[p, q, r, s] = 0.0
    m = MPO.qc_tracked(h, V)
    x = np.concatenate([h.ravel(), V.ravel()])
    ts = m.tensors()
    prov = [m.provenance(k) for k in range(L)]
    ids_seen = set()
    for k in range(L):
        ptr, ids, val = prov[k]
        sc = ts[k]["scale"]
        assert ptr.size == sc.size + 1 and ptr[0] == 0 and ptr[-1] == ids.size
        for j in range(sc.size):
            a, b = int(ptr[j]), int(ptr[j + 1])
            if a == b:
                assert sc[j] == 1.0  # pass-through entry
            else:
                assert abs(np.dot(val[a:b], x[ids[a:b]]) - sc[j]) < 1e-14
        ids_seen.update(int(i) for i in ids)
    assert 0 * L + 3 in ids_seen and L * L + ((0 * L + 1) * L + 2) * L + 3 in ids_seen
    H, ch = dense_mpo(ts)
    H0, ch0 = dense_mpo(MPO.qc(h, V).tensors())
    assert np.abs(H - H0).max() < 1e-12 and np.array_equal(ch, ch0)
    nu = nd = L // 2
    sel = np.where((ch[:, 0] == nu) & (ch[:, 1] == nd))[0]
    w, Z = np.linalg.eigh(H[np.ix_(sel, sel)])
    c = Z[:, 0]
    grads = []
    for k in range(L):
        g = np.zeros(ts[k]["scale"].size)
        for j in range(g.size):
            unit = [dict(t) for t in ts]
            s = np.zeros(g.size)
            s[j] = 1.0
            unit[k]["scale"] = s
            Hj, _ = dense_mpo(unit)
            g[j] = c @ Hj[np.ix_(sel, sel)] @ c
        grads.append(g)
    dx = np.zeros(x.size)
    for k in range(L):
        ptr, ids, val = prov[k]
        for j in range(grads[k].size):
            a, b = int(ptr[j]), int(ptr[j + 1])
            np.add.at(dx, ids[a:b].astype(np.int64), val[a:b] * grads[k][j])
    dh = dx[:L * L].reshape(L, L)
    dV = dx[L * L:].reshape((L,) * 4)
    f = FCI(h, V, e, nu, nd)
    wf, Zf = np.linalg.eigh(f.dense())
    cf = Zf[:, 0]
    g1 = np.array([[cf @ (f.E[p][q] @ cf) for q in range(L)] for p in range(L)])
    assert abs(w[0] + e - wf[0]) < 1e-11
    assert np.abs(dh - g1).max() < 1e-10, np.abs(dh - g1).max()
    assert abs(np.sum(h * dh) + np.sum(V * dV) - w[0]) < 1e-10
