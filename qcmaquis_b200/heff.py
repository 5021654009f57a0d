"""Host-side mirror of the reference's H_eff interface over the C-ABI.

Reference interface (framework/dmrg/solver/solver.h:38-68):
    BoundaryView{host_data, device_data}, SuperHamil{left, right, schedule},
    ietl::mult(SuperHamil, x, y)  ->  y = H_eff x   (ietl_interface_dv.h:112-118)
Here: Context (device + stream), Boundary (resident in HBM), HeffPlan (schedule
staged in HBM) with apply()/apply_device().

Frozen site problems use the "QSPB" v1 snapshot layout (the analogue of the
reference's left_/right_/initial_/tsmpo snapshots, optimize/ts_optimize.hpp:185-215):
    "QSPB" u32 ver; Index phys, left, right; u32 nblocks; per block
    (i32 a, i32 b, u32 rows, u32 cols, rows*cols f64 column-major);
    boundary L; boundary R -- each: Index bra, ket; u32 ncoh, aux; per cohort
    (u32 bra_pos, ket_pos; u8 tr; u32 lsz, rsz, nb; aux x i64 offset;
    aux x f64 cscale; u64 n; n x f64).
Index: u32 n; n x (i32 a, i32 b, u32 size).
"""
from __future__ import annotations

import ctypes
import struct

import numpy as np

from . import _lib
from ._lib import lib, check, P, c_int, c_void_p, c_uint32, c_uint64, c_double


class Sector(ctypes.Structure):
    _fields_ = [("a", ctypes.c_int32), ("b", ctypes.c_int32), ("size", ctypes.c_uint32)]


class BoundaryDesc(ctypes.Structure):
    _fields_ = [("n_bra", c_uint32), ("n_ket", c_uint32), ("bra", P(Sector)), ("ket", P(Sector)),
                ("n_cohorts", c_uint32), ("aux_dim", c_uint32), ("cohort_bra", P(c_uint32)),
                ("cohort_ket", P(c_uint32)), ("tr", P(ctypes.c_uint8)), ("n_blocks", P(c_uint32)),
                ("offsets", P(ctypes.c_int64)), ("cscale", P(c_double)), ("data_offset", P(c_uint64)),
                ("data", P(c_double))]


class MPSDesc(ctypes.Structure):
    _fields_ = [("n_phys", c_uint32), ("n_left", c_uint32), ("n_right", c_uint32), ("phys", P(Sector)),
                ("left", P(Sector)), ("right", P(Sector))]


class HeffInfo(ctypes.Structure):
    _fields_ = [("vec_len", c_uint64), ("t_len", c_uint64), ("s_len", c_uint64), ("n_tjobs", c_uint64),
                ("n_ttiles", c_uint64), ("n_gtasks", c_uint64), ("n_alpha", c_uint64), ("n_segs", c_uint64),
                ("n_outs", c_uint64), ("n_otiles", c_uint64), ("flops", c_double), ("flops_t", c_double),
                ("flops_ls", c_double), ("flops_s", c_double), ("g_elems", c_uint64), ("g_reads", c_uint64),
                ("l_len", c_uint64), ("r_len", c_uint64), ("n_kitems", c_uint64), ("flops_sdense", c_double), ("launches", c_uint64), ("w_len", c_uint64), ("flops_sexec", c_double),
                ("p_len", c_uint64)]


class BoundaryInfo(ctypes.Structure):
    _fields_ = [("n_bra", c_uint32), ("n_ket", c_uint32), ("n_cohorts", c_uint32), ("aux_dim", c_uint32),
                ("total", c_uint64), ("resident", c_uint32)]


_lib._sig("qcm_ctx_create", c_int, c_int, P(c_void_p))
_lib._sig("qcm_ctx_destroy", None, c_void_p)
_lib._sig("qcm_ctx_synchronize", c_int, c_void_p)
_lib._sig("qcm_boundary_upload", c_int, c_void_p, P(BoundaryDesc), P(c_void_p))
_lib._sig("qcm_boundary_index_create", c_int, P(BoundaryDesc), P(c_void_p))
_lib._sig("qcm_boundary_free", None, c_void_p)
_lib._sig("qcm_boundary_get_info", c_int, c_void_p, P(BoundaryInfo))
_lib._sig("qcm_boundary_download", c_int, c_void_p, P(Sector), P(Sector), P(c_uint32), P(c_uint32), P(ctypes.c_uint8),
          P(c_uint32), P(ctypes.c_int64), P(c_double), P(c_uint64), P(c_double))
_lib._sig("qcm_heff_plan_create", c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_int, P(MPSDesc), c_int, P(c_void_p))
_lib._sig("qcm_heff_get_info", c_int, c_void_p, P(HeffInfo))
_lib._sig("qcm_heff_apply", c_int, c_void_p, P(c_double), P(c_double))
_lib._sig("qcm_heff_stream_coefficients", c_int, c_void_p, c_uint64)
_lib._sig("qcm_heff_chunk_apply", c_int, c_void_p, c_uint64)
_lib._sig("qcm_heff_adjoint", c_int, c_void_p, P(c_double), P(c_double), P(c_double), P(c_double))
_lib._sig("qcm_heff_adjoint_terms", c_int, c_void_p, P(c_uint64))
_lib._sig("qcm_heff_apply_device", c_int, c_void_p, c_void_p, c_void_p)
_lib._sig("qcm_heff_bookkeeping", c_int, c_void_p, P(c_uint32), P(c_double), c_uint64, P(c_uint64))
_lib._sig("qcm_heff_profile", c_int, c_void_p, c_void_p, c_void_p, P(ctypes.c_float))
_lib._sig("qcm_heff_apply_device_noalloc", c_int, c_void_p, c_void_p, c_void_p)
_lib._sig("qcm_heff_apply_mode", c_int, c_void_p, P(c_double), P(c_double), c_int)
_lib._sig("qcm_heff_apply_device_mode", c_int, c_void_p, c_void_p, c_void_p, c_int)
_lib._sig("qcm_heff_profile_mode", c_int, c_void_p, c_void_p, c_void_p, P(ctypes.c_float), c_int)

# precision forms of H_eff . psi (QCM_PRECISION_*)
FP64, MIXED, MIXED_TC = 0, 1, 2


def precision_mode(precision) -> int:
    """"fp64" / "mixed" / "mixed_tc" (or 0 / 1 / 2) -> QCM_PRECISION_*."""
    m = {"fp64": FP64, "mixed": MIXED, "mixed_tc": MIXED_TC, FP64: FP64, MIXED: MIXED, MIXED_TC: MIXED_TC}
    if precision not in m:
        raise ValueError(f"unknown precision {precision!r}")
    return m[precision]
NOALLOC_SCRATCH_DOUBLES = 8 * 1024 * 1024
_lib._sig("qcm_heff_free", None, c_void_p)
_lib._sig("qcm_heff_group_create", c_int, c_void_p, P(c_void_p), c_int, P(c_void_p))
_lib._sig("qcm_heff_group_layout", c_int, c_void_p, P(c_uint64), P(c_uint64), P(c_uint64))
_lib._sig("qcm_heff_group_get_info", c_int, c_void_p, P(HeffInfo))
_lib._sig("qcm_heff_group_apply", c_int, c_void_p, P(c_double), P(c_double))
_lib._sig("qcm_heff_group_apply_device", c_int, c_void_p, c_void_p, c_void_p)
_lib._sig("qcm_jd_solve_batched", c_int, c_void_p, P(c_double), c_double, c_int, c_int, P(c_double), P(c_double),
          P(ctypes.c_int), P(ctypes.c_int))
_lib._sig("qcm_heff_group_free", None, c_void_p)
_lib._sig("qcm_probe_fp64_peaks", c_int, P(c_double), P(c_double))


def probe_fp64_peaks():
    """(DMMA TFLOP/s, DFMA TFLOP/s) measured on the current device."""
    a, b = c_double(), c_double()
    check(lib.qcm_probe_fp64_peaks(ctypes.byref(a), ctypes.byref(b)), "qcm_probe_fp64_peaks")
    return a.value, b.value

PLAN_BOOKKEEPING = 1
PLAN_HOST_ONLY = 2


# ---------------------------------------------------------------------------
# snapshot parsing

def _sectors(lst):
    arr = (Sector * max(1, len(lst)))()
    for i, (a, b, s) in enumerate(lst):
        arr[i].a, arr[i].b, arr[i].size = a, b, s
    return arr


class _Reader:
    """Little-endian reader of the QSPB / QBSP blobs."""

    def __init__(self, blob: bytes):
        self.blob, self.off = blob, 0

    def get(self, fmt):
        v = struct.unpack_from("<" + fmt, self.blob, self.off)
        self.off += struct.calcsize("<" + fmt)
        return v

    def idx(self):
        (n,) = self.get("I")
        return [self.get("iiI") for _ in range(n)]

    def arr(self, dtype, n):
        a = np.frombuffer(self.blob, dtype=dtype, count=n, offset=self.off).copy()
        self.off += np.dtype(dtype).itemsize * n
        return a

    def blocks(self):
        (nb,) = self.get("I")
        out = []
        for _ in range(nb):
            a, b, r, c = self.get("iiII")
            out.append(((a, b), self.arr("<f8", r * c).reshape(c, r).T))
        return out

    def bnd(self):
        bra, ket = self.idx(), self.idx()
        nc, aux = self.get("II")
        cb, ck, tr, ls, rs, nb = [], [], [], [], [], []
        offs, cs, data, doff = [], [], [], []
        pos = 0
        for _ in range(nc):
            b0, k0 = self.get("II")
            (t,) = self.get("B")
            l, r, n = self.get("III")
            cb.append(b0); ck.append(k0); tr.append(t); ls.append(l); rs.append(r); nb.append(n)
            offs.append(self.arr("<i8", aux))
            cs.append(self.arr("<f8", aux))
            (nd,) = self.get("Q")
            data.append(self.arr("<f8", nd))
            doff.append(pos)
            pos += nd
        return dict(bra=bra, ket=ket, aux=aux, cohort_bra=np.array(cb, np.uint32), cohort_ket=np.array(ck, np.uint32),
                    tr=np.array(tr, np.uint8), lsz=np.array(ls, np.uint32), rsz=np.array(rs, np.uint32),
                    n_blocks=np.array(nb, np.uint32),
                    offsets=np.concatenate(offs).astype(np.int64) if offs else np.zeros(0, np.int64),
                    cscale=np.concatenate(cs) if cs else np.zeros(0),
                    data=np.concatenate(data) if data else np.zeros(0),
                    data_offset=np.array(doff, np.uint64))


def parse_site_problem(blob: bytes):
    r = _Reader(blob)
    magic, ver = r.get("II")
    assert magic == 0x42505351 and ver == 1, "not a QSPB v1 site problem"
    phys, left, right = r.idx(), r.idx(), r.idx()
    blocks = r.blocks()
    L = r.bnd()
    R = r.bnd()
    return dict(phys=phys, left=left, right=right, blocks=blocks, L=L, R=R)


def parse_mps_tensor(blob: bytes):
    """"QMPS" v1: Index phys, left, right; right-paired blocks (ls x stripe) in left-sector order."""
    r = _Reader(blob)
    magic, ver = r.get("II")
    assert magic == 0x53504D51 and ver == 1, "not a QMPS v1 site tensor"
    phys, left, right = r.idx(), r.idx(), r.idx()
    return dict(phys=phys, left=left, right=right, blocks=r.blocks())


def parse_boundary_step(blob: bytes):
    """"QBSP" v1: u32 side (0 left, 1 right), u32 site; Index phys, left, right; the site
    tensor's right-paired blocks (as in QSPB); input boundary; output boundary."""
    r = _Reader(blob)
    magic, ver = r.get("II")
    assert magic == 0x50534251 and ver == 1, "not a QBSP v1 boundary step"
    side, site = r.get("II")
    phys, left, right = r.idx(), r.idx(), r.idx()
    blocks = r.blocks()
    bin_ = r.bnd()
    bout = r.bnd()
    return dict(side=side, site=site, phys=phys, left=left, right=right, blocks=blocks, B_in=bin_, B_out=bout)


def twin_vector(problem) -> np.ndarray:
    """Concatenated right-paired blocks in left-sector order (column-major)."""
    return np.concatenate([b.T.ravel() for (_, b) in problem["blocks"]])


# ---------------------------------------------------------------------------

class Context:
    def __init__(self, device: int = 0):
        h = c_void_p()
        check(lib.qcm_ctx_create(device, ctypes.byref(h)), "qcm_ctx_create")
        self.h = h

    def synchronize(self):
        check(lib.qcm_ctx_synchronize(self.h), "qcm_ctx_synchronize")

    def __del__(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib.qcm_ctx_destroy(self.h)
            self.h = c_void_p()


class Boundary:
    """Boundary resident in HBM (ctx given) or index-only on the host (ctx None)."""

    def __init__(self, ctx, b: dict):
        self.ctx = ctx
        self._keep = []
        k = self._keep.append
        bra, ket = _sectors(b["bra"]), _sectors(b["ket"])
        k(bra); k(ket)
        arrs = {}
        for name, dt in (("cohort_bra", np.uint32), ("cohort_ket", np.uint32), ("tr", np.uint8),
                         ("n_blocks", np.uint32), ("offsets", np.int64), ("cscale", np.float64),
                         ("data_offset", np.uint64), ("data", np.float64)):
            a = np.ascontiguousarray(b[name], dtype=dt)
            if a.size == 0:
                a = np.zeros(1, dtype=dt)
            arrs[name] = a
            k(a)
        d = BoundaryDesc()
        d.n_bra, d.n_ket, d.bra, d.ket = len(b["bra"]), len(b["ket"]), bra, ket
        d.n_cohorts, d.aux_dim = len(b["cohort_bra"]), b["aux"]
        d.cohort_bra = arrs["cohort_bra"].ctypes.data_as(P(c_uint32))
        d.cohort_ket = arrs["cohort_ket"].ctypes.data_as(P(c_uint32))
        d.tr = arrs["tr"].ctypes.data_as(P(ctypes.c_uint8))
        d.n_blocks = arrs["n_blocks"].ctypes.data_as(P(c_uint32))
        d.offsets = arrs["offsets"].ctypes.data_as(P(ctypes.c_int64))
        d.cscale = arrs["cscale"].ctypes.data_as(P(c_double))
        d.data_offset = arrs["data_offset"].ctypes.data_as(P(c_uint64))
        d.data = arrs["data"].ctypes.data_as(P(c_double))
        h = c_void_p()
        if ctx is None:
            check(lib.qcm_boundary_index_create(ctypes.byref(d), ctypes.byref(h)), "qcm_boundary_index_create")
        else:
            check(lib.qcm_boundary_upload(ctx.h, ctypes.byref(d), ctypes.byref(h)), "qcm_boundary_upload")
        self.h = h
        self._keep = None

    @classmethod
    def from_handle(cls, ctx, h):
        b = cls.__new__(cls)
        b.ctx, b.h, b._keep = ctx, h, None
        return b

    def info(self) -> dict:
        i = BoundaryInfo()
        check(lib.qcm_boundary_get_info(self.h, ctypes.byref(i)), "qcm_boundary_get_info")
        return {f: getattr(i, f) for f, _ in BoundaryInfo._fields_}

    def download(self) -> dict:
        """Index and data as a dict with the fields of the boundary description (data_offset per cohort)."""
        i = self.info()
        nc, aux, nb_, nk_ = i["n_cohorts"], i["aux_dim"], i["n_bra"], i["n_ket"]
        bra, ket = (Sector * max(1, nb_))(), (Sector * max(1, nk_))()
        out = dict(cohort_bra=np.zeros(max(nc, 1), np.uint32), cohort_ket=np.zeros(max(nc, 1), np.uint32),
                   tr=np.zeros(max(nc, 1), np.uint8), n_blocks=np.zeros(max(nc, 1), np.uint32),
                   offsets=np.zeros(max(nc * aux, 1), np.int64), cscale=np.zeros(max(nc * aux, 1)),
                   data_offset=np.zeros(max(nc, 1), np.uint64), data=np.zeros(max(i["total"], 1)))
        check(lib.qcm_boundary_download(self.h, bra, ket, out["cohort_bra"].ctypes.data_as(P(c_uint32)),
                                        out["cohort_ket"].ctypes.data_as(P(c_uint32)),
                                        out["tr"].ctypes.data_as(P(ctypes.c_uint8)),
                                        out["n_blocks"].ctypes.data_as(P(c_uint32)),
                                        out["offsets"].ctypes.data_as(P(ctypes.c_int64)), _lib.dptr(out["cscale"]),
                                        out["data_offset"].ctypes.data_as(P(c_uint64)),
                                        _lib.dptr(out["data"]) if i["resident"] else None), "qcm_boundary_download")
        for k in ("cohort_bra", "cohort_ket", "tr", "n_blocks", "data_offset"):
            out[k] = out[k][:nc]
        out["offsets"], out["cscale"] = out["offsets"][:nc * aux], out["cscale"][:nc * aux]
        out["data"] = out["data"][:i["total"]]
        out["bra"] = [(s.a, s.b, s.size) for s in bra[:nb_]]
        out["ket"] = [(s.a, s.b, s.size) for s in ket[:nk_]]
        out["aux"] = aux
        return out

    def __del__(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib.qcm_boundary_free(self.h)
            self.h = c_void_p()


class HeffPlan:
    """H_eff of one two-site problem; apply() is the Davidson H.psi callback."""

    def __init__(self, ctx, L: Boundary, R: Boundary, ts_mpo, site: int, phys, left, right,
                 bookkeeping: bool = False):
        self.ctx, self.L, self.R, self.mpo = ctx, L, R, ts_mpo
        ps, ls, rs = _sectors(phys), _sectors(left), _sectors(right)
        d = MPSDesc()
        d.n_phys, d.n_left, d.n_right = len(phys), len(left), len(right)
        d.phys, d.left, d.right = ps, ls, rs
        h = c_void_p()
        flags = (PLAN_BOOKKEEPING if bookkeeping else 0) | (PLAN_HOST_ONLY if ctx is None else 0)
        check(lib.qcm_heff_plan_create(ctx.h if ctx is not None else None, L.h, R.h, ts_mpo.handle, site,
                                       ctypes.byref(d), flags, ctypes.byref(h)), "qcm_heff_plan_create")
        self.h = h
        info = HeffInfo()
        check(lib.qcm_heff_get_info(h, ctypes.byref(info)), "qcm_heff_get_info")
        self.info = {f: getattr(info, f) for f, _ in HeffInfo._fields_}
        self.n = int(info.vec_len)

    @classmethod
    def from_handle(cls, ctx, h, owner=None):
        """Wrap a plan handle made by the library (owner keeps its boundaries alive)."""
        self = cls.__new__(cls)
        self.ctx, self.L, self.R, self.mpo, self.owner = ctx, None, None, None, owner
        self.h = h
        info = HeffInfo()
        check(lib.qcm_heff_get_info(h, ctypes.byref(info)), "qcm_heff_get_info")
        self.info = {f: getattr(info, f) for f, _ in HeffInfo._fields_}
        self.n = int(info.vec_len)
        return self

    def stream_coefficients(self, nbytes: int):
        """Keep at most nbytes of coefficient blocks on the device, generated chunk by chunk in every FP64
        apply (0: whole); the plan is staged again and its info refreshed."""
        check(lib.qcm_heff_stream_coefficients(self.h, int(nbytes)), "qcm_heff_stream_coefficients")
        info = HeffInfo()
        check(lib.qcm_heff_get_info(self.h, ctypes.byref(info)), "qcm_heff_get_info")
        self.info = {f: getattr(info, f) for f, _ in HeffInfo._fields_}

    def chunk_apply(self, nbytes: int):
        """Apply in ket-sector chunks of at most nbytes of T, S and coefficient blocks (0: whole); the plan
        is staged again and its info refreshed."""
        check(lib.qcm_heff_chunk_apply(self.h, int(nbytes)), "qcm_heff_chunk_apply")
        info = HeffInfo()
        check(lib.qcm_heff_get_info(self.h, ctypes.byref(info)), "qcm_heff_get_info")
        self.info = {f: getattr(info, f) for f, _ in HeffInfo._fields_}

    def apply(self, x: np.ndarray, precision="fp64") -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        assert x.size == self.n
        y = np.empty_like(x)
        mode = precision_mode(precision)
        if mode == FP64:
            check(lib.qcm_heff_apply(self.h, _lib.dptr(x), _lib.dptr(y)), "qcm_heff_apply")
        else:
            check(lib.qcm_heff_apply_mode(self.h, _lib.dptr(x), _lib.dptr(y), mode), "qcm_heff_apply_mode")
        return y

    def adjoint(self, x: np.ndarray, ybar: np.ndarray):
        """Adjoint of the apply for f = ybar . H_eff x: (psi_bar = H_eff^T ybar, coeff_bar = df/d scale per
        entry of the plan's two-site MPO tensor, in entry order)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        ybar = np.ascontiguousarray(ybar, dtype=np.float64)
        assert x.size == self.n and ybar.size == self.n
        nt = c_uint64()
        check(lib.qcm_heff_adjoint_terms(self.h, ctypes.byref(nt)), "qcm_heff_adjoint_terms")
        pb = np.empty_like(x)
        cb = np.empty(nt.value)
        check(lib.qcm_heff_adjoint(self.h, _lib.dptr(x), _lib.dptr(ybar), _lib.dptr(pb), _lib.dptr(cb)),
              "qcm_heff_adjoint")
        return pb, cb

    def apply_device(self, x_ptr: int, y_ptr: int, precision="fp64"):
        mode = precision_mode(precision)
        if mode == FP64:
            check(lib.qcm_heff_apply_device(self.h, c_void_p(x_ptr), c_void_p(y_ptr)), "qcm_heff_apply_device")
        else:
            check(lib.qcm_heff_apply_device_mode(self.h, c_void_p(x_ptr), c_void_p(y_ptr), mode),
                  "qcm_heff_apply_device_mode")

    def apply_device_noalloc(self, x_ptr: int, y_ptr: int):
        """apply_device without any device allocation: scratch in the library's fixed 64 MiB array
        (for hosts that cannot cudaMalloc here; overlapping calls on one GPU race)."""
        check(lib.qcm_heff_apply_device_noalloc(self.h, c_void_p(x_ptr), c_void_p(y_ptr)),
              "qcm_heff_apply_device_noalloc")

    def profile(self, x_ptr: int, y_ptr: int, precision="fp64"):
        """Per-phase device times (ms): T-GEMM, S gather, L.S GEMM, total."""
        ms = (ctypes.c_float * 4)()
        check(lib.qcm_heff_profile_mode(self.h, c_void_p(x_ptr), c_void_p(y_ptr), ms, precision_mode(precision)),
              "qcm_heff_profile_mode")
        return list(ms)

    def bookkeeping(self):
        n = c_uint64()
        check(lib.qcm_heff_bookkeeping(self.h, None, None, 0, ctypes.byref(n)), "qcm_heff_bookkeeping")
        ints = np.zeros(10 * n.value, dtype=np.uint32)
        al = np.zeros(n.value)
        check(lib.qcm_heff_bookkeeping(self.h, ints.ctypes.data_as(P(c_uint32)), _lib.dptr(al), n.value,
                                       ctypes.byref(n)), "qcm_heff_bookkeeping")
        return ints.reshape(-1, 10), al

    def __del__(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib.qcm_heff_free(self.h)
            self.h = c_void_p()


def plan_from_problem(ctx: Context, problem: dict, ts_mpo, site: int, bookkeeping: bool = False):
    L = Boundary(ctx, problem["L"])
    R = Boundary(ctx, problem["R"])
    return HeffPlan(ctx, L, R, ts_mpo, site, problem["phys"], problem["left"], problem["right"], bookkeeping)


class HeffGroup:
    """Independent plans of one context merged into one (qcm_heff_group): one apply or one lockstep
    Jacobi-Davidson for all of them.  Vectors are arenas of n doubles, member i's at offsets[i]."""

    def __init__(self, ctx, plans):
        self.ctx, self.plans = ctx, list(plans)
        arr = (c_void_p * len(self.plans))(*[p.h.value if isinstance(p.h, c_void_p) else p.h for p in self.plans])
        h = c_void_p()
        check(lib.qcm_heff_group_create(ctx.h, arr, len(self.plans), ctypes.byref(h)), "qcm_heff_group_create")
        self.h = h
        n = c_uint64()
        self.offsets = np.zeros(len(self.plans), np.uint64)
        self.lengths = np.zeros(len(self.plans), np.uint64)
        u64 = lambda a: a.ctypes.data_as(P(c_uint64))
        check(lib.qcm_heff_group_layout(h, ctypes.byref(n), u64(self.offsets), u64(self.lengths)), "qcm_heff_group_layout")
        self.n = int(n.value)
        info = HeffInfo()
        check(lib.qcm_heff_group_get_info(h, ctypes.byref(info)), "qcm_heff_group_get_info")
        self.info = {f: getattr(info, f) for f, _ in HeffInfo._fields_}

    def pack(self, xs) -> np.ndarray:
        out = np.zeros(self.n)
        for x, o, l in zip(xs, self.offsets, self.lengths):
            assert x.size == l
            out[int(o):int(o) + int(l)] = x
        return out

    def unpack(self, arena):
        return [arena[int(o):int(o) + int(l)].copy() for o, l in zip(self.offsets, self.lengths)]

    def apply(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        assert x.size == self.n
        y = np.empty_like(x)
        check(lib.qcm_heff_group_apply(self.h, _lib.dptr(x), _lib.dptr(y)), "qcm_heff_group_apply")
        return y

    def apply_device(self, x_ptr: int, y_ptr: int):
        check(lib.qcm_heff_group_apply_device(self.h, c_void_p(x_ptr), c_void_p(y_ptr)), "qcm_heff_group_apply_device")

    def jd_solve(self, x0: np.ndarray, tol: float = 1e-10, maxiter: int = 8, graphs: bool = True):
        """Lockstep Jacobi-Davidson of every member: (eigenvalues, eigenvector arena, iterations, group applies)."""
        x0 = np.ascontiguousarray(x0, dtype=np.float64)
        assert x0.size == self.n
        out = np.empty_like(x0)
        k = len(self.plans)
        ev = np.zeros(k)
        it = np.zeros(k, dtype=np.int32)
        na = ctypes.c_int()
        check(lib.qcm_jd_solve_batched(self.h, _lib.dptr(x0), tol, maxiter, 1 if graphs else 0, _lib.dptr(out),
                                       _lib.dptr(ev), it.ctypes.data_as(P(ctypes.c_int)), ctypes.byref(na)),
              "qcm_jd_solve_batched")
        return ev, out, it, na.value

    def __del__(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib.qcm_heff_group_free(self.h)
            self.h = c_void_p()
