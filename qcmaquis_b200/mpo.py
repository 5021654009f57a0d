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

    def twosite(self) -> "MPO":
        out = ctypes.c_void_p()
        check(lib.qcm_mpo_make_twosite(self._h, ctypes.byref(out)), "qcm_mpo_make_twosite")
        return MPO(out)

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
