"""Host-side MPO handle: build the QC MPO through the C-ABI and read the blob back.

The blob layout ("QMPO" v1) is documented in qcmaquis_b200/csrc/qc_mpo.cpp.
"""
from __future__ import annotations

import ctypes
import struct

import numpy as np

from . import _lib
from ._lib import lib, check


class MPO:
    def __init__(self, handle):
        self._h = ctypes.c_void_p(handle) if not isinstance(handle, ctypes.c_void_p) else handle

    @classmethod
    def qc(cls, h, V, cutoff: float = 1e-20) -> "MPO":
        h = np.ascontiguousarray(h, dtype=np.float64)
        V = np.ascontiguousarray(V, dtype=np.float64)
        L = h.shape[0]
        out = ctypes.c_void_p()
        check(lib.qcm_mpo_build_qc(L, _lib.dptr(h), _lib.dptr(V), cutoff, ctypes.byref(out)), "qcm_mpo_build_qc")
        return cls(out)

    @classmethod
    def from_blob(cls, blob: bytes) -> "MPO":
        out = ctypes.c_void_p()
        buf = ctypes.create_string_buffer(blob, len(blob))
        check(lib.qcm_mpo_deserialize(buf, len(blob), ctypes.byref(out)), "qcm_mpo_deserialize")
        return cls(out)

    @classmethod
    def from_tensors(cls, tensors, twosite: bool = False) -> "MPO":
        """MPO handed in tensor by tensor (qcm_mpo_create + qcm_mpo_set_tensor), from dicts in the
        layout parse_blob returns (herm_left / herm_right: (n, 2) arrays of partner and phase, or None)."""
        out = ctypes.c_void_p()
        check(lib.qcm_mpo_create(len(tensors), int(twosite), ctypes.byref(out)), "qcm_mpo_create")
        m = cls(out)
        for site, t in enumerate(tensors):
            m.set_tensor(site, t)
        return m

    def set_tensor(self, site: int, t) -> None:
        u32 = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
        i32 = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        keep = []

        def arr(x, dt):
            a = np.ascontiguousarray(x, dtype=dt)
            keep.append(a)
            return a
        b1, b2, op = arr(t["b1"], np.uint32), arr(t["b2"], np.uint32), arr(t["op"], np.uint32)
        sc = arr(t["scale"], np.float64)
        ops = t["ops"]
        ptr = arr(np.concatenate([[0], np.cumsum([len(o) for o in ops])]), np.uint64)
        oin = arr(np.concatenate([o["inp"] for o in ops]) if ops else [], np.uint32)
        oout = arr(np.concatenate([o["out"] for o in ops]) if ops else [], np.uint32)
        oval = arr(np.concatenate([o["val"] for o in ops]) if ops else [], np.float64)
        pc = arr([[a, b] for (a, b, _) in t["phys"]], np.int32)
        ps = arr([s for (_, _, s) in t["phys"]], np.uint32)
        d = _lib.MPOTensorDesc(rows=t["rows"], cols=t["cols"], n_terms=b1.size, b1=u32(b1), b2=u32(b2), op=u32(op),
                               scale=_lib.dptr(sc), n_ops=len(ops),
                               op_ptr=ptr.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), op_in=u32(oin),
                               op_out=u32(oout), op_val=_lib.dptr(oval), n_phys=len(t["phys"]),
                               phys_charge=i32(pc), phys_size=u32(ps))
        for side in ("left", "right"):
            h = t.get("herm_" + side)
            if h is not None:
                hh = arr(np.asarray(h)[:, 0], np.int32)
                ph = arr(np.asarray(h)[:, 1], np.int32)
                setattr(d, "herm_" + side, i32(hh))
                setattr(d, "phase_" + side, i32(ph))
        check(lib.qcm_mpo_set_tensor(self._h, site, ctypes.byref(d)), "qcm_mpo_set_tensor")

    def hermitian(self, site: int):
        """(herm_left, phase_left, herm_right, phase_right) of tensor `site` (qcm_mpo_tensor_hermitian)."""
        r, c = ctypes.c_uint32(), ctypes.c_uint32()
        check(lib.qcm_mpo_tensor_info(self._h, site, ctypes.byref(r), ctypes.byref(c), None, None), "qcm_mpo_tensor_info")
        out = [np.zeros(n, np.int32) for n in (r.value, r.value, c.value, c.value)]
        i32 = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        check(lib.qcm_mpo_tensor_hermitian(self._h, site, *[i32(a) for a in out]), "qcm_mpo_tensor_hermitian")
        return tuple(out)

    def twosite(self) -> "MPO":
        out = ctypes.c_void_p()
        check(lib.qcm_mpo_make_twosite(self._h, ctypes.byref(out)), "qcm_mpo_make_twosite")
        return MPO(out)

    @classmethod
    def qc_tracked(cls, h, V) -> "MPO":
        """The QC MPO with every term the spin structure allows and its integral provenance (provenance())."""
        h = np.ascontiguousarray(h, dtype=np.float64)
        V = np.ascontiguousarray(V, dtype=np.float64)
        L = h.shape[0]
        out = ctypes.c_void_p()
        check(lib.qcm_mpo_build_qc_tracked(L, _lib.dptr(h), _lib.dptr(V), ctypes.byref(out)), "qcm_mpo_build_qc_tracked")
        return cls(out)

    def provenance(self, site: int):
        """(ptr, id, val) of tensor `site`: scale[e] = sum(val[ptr[e]:ptr[e+1]] * x[id[ptr[e]:ptr[e+1]]]), x = (h, V)
        flattened row-major."""
        n = ctypes.c_uint64()
        check(lib.qcm_mpo_provenance(self._h, site, None, None, None, 0, ctypes.byref(n)), "qcm_mpo_provenance")
        ne = self.terms(site)["scale"].size
        ptr = np.zeros(ne + 1, dtype=np.uint64)
        ids = np.zeros(n.value, dtype=np.uint64)
        val = np.zeros(n.value)
        u64 = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
        check(lib.qcm_mpo_provenance(self._h, site, u64(ptr), u64(ids), _lib.dptr(val), n.value, ctypes.byref(n)),
              "qcm_mpo_provenance")
        return ptr, ids, val

    def __len__(self):
        return lib.qcm_mpo_length(self._h)

    @property
    def handle(self):
        return self._h

    def blob(self) -> bytes:
        n = ctypes.c_size_t()
        check(lib.qcm_mpo_serialize(self._h, None, 0, ctypes.byref(n)), "qcm_mpo_serialize")
        buf = ctypes.create_string_buffer(n.value)
        check(lib.qcm_mpo_serialize(self._h, buf, n.value, ctypes.byref(n)), "qcm_mpo_serialize")
        return buf.raw

    def tensors(self):
        return parse_blob(self.blob())

    def copy(self) -> "MPO":
        return MPO.from_blob(self.blob())

    def terms(self, site: int):
        """Entries of tensor `site` in entry order: dict of b1, b2, op (uint32) and scale (float64)."""
        n = ctypes.c_uint64()
        check(lib.qcm_mpo_tensor_terms(self._h, site, None, None, None, None, 0, ctypes.byref(n)), "qcm_mpo_tensor_terms")
        out = {k: np.zeros(n.value, dtype=np.uint32) for k in ("b1", "b2", "op")}
        out["scale"] = np.zeros(n.value)
        u32 = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
        check(lib.qcm_mpo_tensor_terms(self._h, site, u32(out["b1"]), u32(out["b2"]), u32(out["op"]),
                                       _lib.dptr(out["scale"]), n.value, ctypes.byref(n)), "qcm_mpo_tensor_terms")
        return out

    def set_scales(self, site: int, scale: np.ndarray):
        scale = np.ascontiguousarray(scale, dtype=np.float64)
        check(lib.qcm_mpo_set_scales(self._h, site, _lib.dptr(scale), scale.size), "qcm_mpo_set_scales")

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value:
            lib.qcm_mpo_free(self._h)
            self._h = ctypes.c_void_p()


def parse_blob(b: bytes):
    """Decode a QMPO blob into a list of dicts (phys, rows, cols, b1, b2, op, scale, herm, ops)."""
    off = 0

    def get(fmt):
        nonlocal off
        v = struct.unpack_from("<" + fmt, b, off)
        off += struct.calcsize("<" + fmt)
        return v

    magic, ver, nt, ts = get("IIII")
    assert magic == 0x4F504D51 and ver == 1
    out = []
    rec = np.dtype([("b1", "<u4"), ("b2", "<u4"), ("op", "<u4"), ("scale", "<f8")])
    orec = np.dtype([("inp", "<u4"), ("out", "<u4"), ("val", "<f8")])
    for _ in range(nt):
        (ns,) = get("I")
        phys = [get("iiI") for _ in range(ns)]
        rows, cols, nnz = get("IIQ")
        ent = np.frombuffer(b, dtype=rec, count=nnz, offset=off)
        off += rec.itemsize * nnz
        hl = np.frombuffer(b, dtype="<i4", count=2 * rows, offset=off).reshape(rows, 2)
        off += 8 * rows
        hr = np.frombuffer(b, dtype="<i4", count=2 * cols, offset=off).reshape(cols, 2)
        off += 8 * cols
        (nops,) = get("I")
        ops = []
        for _ in range(nops):
            (k,) = get("I")
            e = np.frombuffer(b, dtype=orec, count=k, offset=off)
            off += orec.itemsize * k
            ops.append(e)
        out.append(dict(phys=phys, rows=rows, cols=cols, b1=ent["b1"].copy(), b2=ent["b2"].copy(),
                        op=ent["op"].copy(), scale=ent["scale"].copy(), herm_left=hl.copy(),
                        herm_right=hr.copy(), ops=ops, twosite=bool(ts)))
    return out


def dense_operator(tensor, op_id):
    """Dense <out|O|in> matrix of one operator of an MPO tensor."""
    n = sum(s[2] for s in tensor["phys"])
    M = np.zeros((n, n))
    e = tensor["ops"][op_id]
    M[e["out"], e["inp"]] = e["val"]
    return M
