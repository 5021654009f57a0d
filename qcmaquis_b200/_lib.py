"""ctypes binding of libqcm_b200.so (the C-ABI declared in include/qcm_b200.h).

The library is built in-tree (qcmaquis_b200/libqcm_b200.so).  Importing this
module fails loudly if it is missing: there is no Python or CPU fallback for
the device path.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libqcm_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(f"qcmaquis_b200: native library missing at {LIB_PATH}; "
                      "build it with `make -C qcmaquis_b200/csrc` (or __graft_entry__.build())")

lib = ctypes.CDLL(LIB_PATH)

c_int, c_double, c_size_t, c_void_p = ctypes.c_int, ctypes.c_double, ctypes.c_size_t, ctypes.c_void_p
c_uint32, c_uint64 = ctypes.c_uint32, ctypes.c_uint64
P = ctypes.POINTER


class QcmError(RuntimeError):
    pass


def check(rc: int, what: str = "") -> None:
    if rc != 0:
        msg = lib.qcm_last_error().decode()
        raise QcmError(f"{what}: status {rc}: {msg}")


def _sig(name, restype, *argtypes):
    f = getattr(lib, name)
    f.restype = restype
    f.argtypes = list(argtypes)
    return f


_sig("qcm_last_error", ctypes.c_char_p)
_sig("qcm_version", ctypes.c_char_p)
_sig("qcm_mpo_build_qc", c_int, c_int, P(c_double), P(c_double), c_double, P(c_void_p))
_sig("qcm_mpo_build_qc_tracked", c_int, c_int, P(c_double), P(c_double), P(c_void_p))
_sig("qcm_mpo_provenance", c_int, c_void_p, c_int, P(ctypes.c_uint64), P(ctypes.c_uint64), P(c_double), c_uint64,
     P(c_uint64))
_sig("qcm_mpo_make_twosite", c_int, c_void_p, P(c_void_p))
_sig("qcm_mpo_length", c_int, c_void_p)
_sig("qcm_mpo_serialize", c_int, c_void_p, c_void_p, c_size_t, P(c_size_t))
_sig("qcm_mpo_deserialize", c_int, c_void_p, c_size_t, P(c_void_p))
_sig("qcm_mpo_free", None, c_void_p)
_sig("qcm_mpo_tensor_terms", c_int, c_void_p, c_int, P(ctypes.c_uint32), P(ctypes.c_uint32), P(ctypes.c_uint32),
     P(c_double), ctypes.c_uint64, P(ctypes.c_uint64))
_sig("qcm_mpo_set_scales", c_int, c_void_p, c_int, P(c_double), ctypes.c_uint64)


class MPOTensorDesc(ctypes.Structure):
    """qcm_mpo_tensor_desc"""
    _fields_ = [("rows", c_uint32), ("cols", c_uint32), ("n_terms", c_uint64),
                ("b1", P(c_uint32)), ("b2", P(c_uint32)), ("op", P(c_uint32)), ("scale", P(c_double)),
                ("n_ops", c_uint32), ("op_ptr", P(c_uint64)), ("op_in", P(c_uint32)), ("op_out", P(c_uint32)),
                ("op_val", P(c_double)), ("n_phys", c_uint32), ("phys_charge", P(ctypes.c_int32)),
                ("phys_size", P(c_uint32)), ("herm_left", P(ctypes.c_int32)), ("phase_left", P(ctypes.c_int32)),
                ("herm_right", P(ctypes.c_int32)), ("phase_right", P(ctypes.c_int32))]


_sig("qcm_mpo_create", c_int, c_int, c_int, P(c_void_p))
_sig("qcm_mpo_set_tensor", c_int, c_void_p, c_int, P(MPOTensorDesc))
_sig("qcm_mpo_tensor_info", c_int, c_void_p, c_int, P(c_uint32), P(c_uint32), P(c_uint32), P(c_uint32))
_sig("qcm_mpo_tensor_hermitian", c_int, c_void_p, c_int, P(ctypes.c_int32), P(ctypes.c_int32), P(ctypes.c_int32),
     P(ctypes.c_int32))


def dptr(a):
    """double* of a C-contiguous float64 numpy array."""
    return a.ctypes.data_as(P(c_double))
