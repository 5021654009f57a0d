"""QC MPO (input prep): exactness against FCI spectra by dense contraction."""
import numpy as np
import pytest

from qcmaquis_b200.fcidump import synthetic_integrals, write_fcidump, read_fcidump
from qcmaquis_b200.mpo import MPO, dense_operator, parse_blob
from oracle.fci import FCI


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
