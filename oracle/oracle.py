"""ctypes binding of the oracle (CPU restatement of the reference path).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / --impl reference legs of bench.py, never by the product package.
"""
from __future__ import annotations

import ctypes
import glob
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")

P = ctypes.POINTER
c_int, c_double, c_size_t, c_void_p = ctypes.c_int, ctypes.c_double, ctypes.c_size_t, ctypes.c_void_p


def build() -> None:
    subprocess.run(["make", "-C", _HERE], check=True, stdout=subprocess.DEVNULL)


def openblas_path() -> str:
    import scipy
    libs = glob.glob(os.path.join(os.path.dirname(scipy.__file__) + ".libs", "libscipy_openblas*.so"))
    if not libs:
        raise RuntimeError("scipy-bundled OpenBLAS not found")
    return libs[0]


_lib = None


def lib(nthreads: int = 0):
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.orc_last_error.restype = ctypes.c_char_p
        L.orc_init.argtypes = [ctypes.c_char_p, c_int]
        L.orc_max_threads.restype = c_int
        L.orc_free.argtypes = [c_void_p]
        L.orc_dmrg_create.argtypes = [c_void_p, c_size_t, c_int, c_int, c_size_t, c_size_t, c_double, c_double, c_int,
                                      c_double, P(c_void_p)]
        L.orc_dmrg_free.argtypes = [c_void_p]
        L.orc_dmrg_set_mmax.argtypes = [c_void_p, c_size_t]
        L.orc_dmrg_set_heev.argtypes = [c_void_p, c_int, c_double, c_double, c_double, c_int, c_int]
        L.orc_dmrg_sweep.argtypes = [c_void_p, c_int, P(c_double), P(c_double), P(c_double), P(ctypes.c_uint64), c_int,
                                     P(c_void_p), P(c_size_t)]
        L.orc_dmrg_stats.argtypes = [c_void_p, P(c_double)]
        L.orc_dmrg_boundary_export.argtypes = [c_void_p, c_int, c_int, P(c_void_p), P(c_size_t)]
        L.orc_dmrg_mps_export.argtypes = [c_void_p, c_int, P(c_void_p), P(c_size_t)]
        L.orc_mpo_build_qc.argtypes = [c_int, P(c_double), P(c_double), c_double, P(c_void_p), P(c_size_t)]
        L.orc_site_problem.argtypes = [c_void_p, c_size_t, c_int, P(c_void_p), P(c_size_t), c_int, P(c_void_p), P(c_size_t)]
        L.orc_heff_apply.argtypes = [c_void_p, c_size_t, c_void_p, c_size_t, c_int, P(c_double), P(c_double), c_size_t,
                                     c_int, P(c_double), P(c_double)]
        L.orc_schedule_export.argtypes = [c_void_p, c_size_t, c_void_p, c_size_t, c_int, P(c_void_p), P(c_size_t),
                                          P(c_double)]
        L.orc_jd_solve.argtypes = [c_void_p, c_size_t, c_void_p, c_size_t, c_int, P(c_double), c_size_t, P(c_double), c_int,
                                   c_int, c_double, c_int, P(c_double), P(c_double), P(c_int), P(c_int)]
        L.orc_dmrg_set_gmres.argtypes = [c_void_p, c_int]
        L.orc_dmrg_set_single_site.argtypes = [c_void_p, c_int]
        L.orc_dmrg_steps_per_sweep.argtypes = [c_void_p]
        L.orc_dmrg_set_ortho.argtypes = [c_void_p, c_int, P(c_void_p), P(c_size_t)]
        L.orc_heff_adjoint.argtypes = [c_void_p, c_size_t, c_void_p, c_size_t, c_int, P(c_double), P(c_double), c_size_t,
                                       P(c_double), P(c_double), c_size_t]
        U32 = P(ctypes.c_uint32)
        L.orc_truncate_svd.argtypes = [ctypes.c_uint32, U32, U32, P(c_double), ctypes.c_uint64, c_double, U32, P(c_double),
                                       P(c_double), P(c_double), P(c_double)]
        L.orc_truncate_heev.argtypes = [ctypes.c_uint32, U32, P(c_double), ctypes.c_uint64, c_double, U32, P(c_double),
                                        P(c_double), P(c_double)]
        _check(L, L.orc_init(openblas_path().encode(), nthreads))
        _lib = L
    return _lib


def _check(L, rc):
    if rc != 0:
        raise RuntimeError("oracle: " + L.orc_last_error().decode())


def _dp(a):
    return a.ctypes.data_as(P(c_double))


class OracleDMRG:
    """Two-site DMRG on the CPU restatement (ts_optimize semantics)."""

    def __init__(self, mpo_blob: bytes, L: int, nup: int, ndown: int, M: int, init_bond_dimension: int | None = None,
                 cutoff: float = 1e-16, tol: float = 1e-10, maxiter: int = 8, ecore: float = 0.0):
        self.lib = lib()
        self.L = L
        self._blob = ctypes.create_string_buffer(mpo_blob, len(mpo_blob))
        h = c_void_p()
        _check(self.lib, self.lib.orc_dmrg_create(self._blob, len(mpo_blob), nup, ndown, M,
                                                  init_bond_dimension or M, cutoff, tol, maxiter, ecore,
                                                  ctypes.byref(h)))
        self.h = h

    def set_single_site(self, on: bool = True):
        """optimization = singlesite (ss_optimize): 2L steps per sweep, each grown by the density-matrix
        prediction with the noise of set_heev's alphas."""
        _check(self.lib, self.lib.orc_dmrg_set_single_site(self.h, 1 if on else 0))

    def sweep(self, sweep: int = 0):
        n = self.lib.orc_dmrg_steps_per_sweep(self.h)
        E, tw, tf = np.zeros(n), np.zeros(n), np.zeros(n)
        bd = np.zeros(n, dtype=np.uint64)
        _check(self.lib, self.lib.orc_dmrg_sweep(self.h, sweep, _dp(E), _dp(tw), _dp(tf),
                                                 bd.ctypes.data_as(P(ctypes.c_uint64)), -1, None, None))
        return E, tw, tf, bd

    def snapshot(self, sweep: int, step: int) -> bytes:
        """Run the sweep up to `step` and return the frozen site problem of that step."""
        p, n = c_void_p(), c_size_t()
        _check(self.lib, self.lib.orc_dmrg_sweep(self.h, sweep, None, None, None, None, step, ctypes.byref(p),
                                                 ctypes.byref(n)))
        b = ctypes.string_at(p, n.value)
        self.lib.orc_free(p)
        return b

    def boundary_export(self, side: int, site: int) -> bytes:
        """Boundary step case ("QBSP" v1) from the current state: side 0 = left step of
        mps[site] from left_[site], side 1 = right step of mps[site] from right_[site + 1]."""
        p, n = c_void_p(), c_size_t()
        _check(self.lib, self.lib.orc_dmrg_boundary_export(self.h, side, site, ctypes.byref(p), ctypes.byref(n)))
        b = ctypes.string_at(p, n.value)
        self.lib.orc_free(p)
        return b

    def mps_export(self, site: int) -> bytes:
        """Current site tensor ("QMPS" v1, right-paired blocks)."""
        p, n = c_void_p(), c_size_t()
        _check(self.lib, self.lib.orc_dmrg_mps_export(self.h, site, ctypes.byref(p), ctypes.byref(n)))
        b = ctypes.string_at(p, n.value)
        self.lib.orc_free(p)
        return b

    def set_heev(self, heev: bool = True, alpha_initial: float = 1e-2, alpha_main: float = 1e-4,
                 alpha_final: float = 1e-8, ngrowsweeps: int = 0, nmainsweeps: int = 0):
        """twosite_truncation = heev (density matrix with noise) instead of svd."""
        self.lib.orc_dmrg_set_heev(self.h, 1 if heev else 0, alpha_initial, alpha_main, alpha_final, ngrowsweeps,
                                   nmainsweeps)

    def set_ortho(self, states):
        """Excited states: states = [[site blob ("QMPS", mps_export) for each site] per ortho state]; every
        solution is kept orthogonal to them.  Call at the start of a sweep."""
        blobs = [b for st in states for b in st]
        bufs = [ctypes.create_string_buffer(b, len(b)) for b in blobs]
        ptrs = (c_void_p * max(1, len(bufs)))(*[ctypes.cast(b, c_void_p) for b in bufs])
        lens = (c_size_t * max(1, len(bufs)))(*[len(b) for b in blobs])
        _check(self.lib, self.lib.orc_dmrg_set_ortho(self.h, len(states), ptrs, lens))

    def set_gmres(self, gmres: int):
        """ietl_jcd_gmres of the sweep's Jacobi-Davidson solves."""
        _check(self.lib, self.lib.orc_dmrg_set_gmres(self.h, gmres))

    def set_mmax(self, M: int):
        self.lib.orc_dmrg_set_mmax(self.h, M)

    def stats(self):
        out = np.zeros(7)
        self.lib.orc_dmrg_stats(self.h, _dp(out))
        keys = ["hpsi_count", "hpsi_time", "hpsi_flops", "jd_time", "schedule_time", "trunc_time", "boundary_time"]
        return dict(zip(keys, out.tolist()))

    def __del__(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.orc_dmrg_free(self.h)
            self.h = c_void_p()


def mpo_blob_qc(h: np.ndarray, V: np.ndarray, cutoff: float = 1e-20) -> bytes:
    """QC MPO blob ("QMPO") of the integrals, built inside the oracle library (no product library)."""
    L = lib()
    h = np.ascontiguousarray(h, dtype=np.float64)
    V = np.ascontiguousarray(V, dtype=np.float64)
    p, n = c_void_p(), c_size_t()
    _check(L, L.orc_mpo_build_qc(h.shape[0], _dp(h), _dp(V), cutoff, ctypes.byref(p), ctypes.byref(n)))
    b = ctypes.string_at(p, n.value)
    L.orc_free(p)
    return b


def site_problem(mpo_blob: bytes, site_blobs, site1: int) -> bytes:
    """Frozen two-site problem ("QSPB") at (site1, site1 + 1) of the MPS given as "QMPS" blobs: boundaries
    from init_left_right(mpo, site1) on that MPS, no optimisation."""
    L = lib()
    mb = ctypes.create_string_buffer(mpo_blob, len(mpo_blob))
    bufs = [ctypes.create_string_buffer(b, len(b)) for b in site_blobs]
    ptrs = (c_void_p * len(bufs))(*[ctypes.cast(b, c_void_p) for b in bufs])
    lens = (c_size_t * len(bufs))(*[len(b) for b in site_blobs])
    p, n = c_void_p(), c_size_t()
    _check(L, L.orc_site_problem(mb, len(mpo_blob), len(bufs), ptrs, lens, site1, ctypes.byref(p), ctypes.byref(n)))
    b = ctypes.string_at(p, n.value)
    L.orc_free(p)
    return b


def heff_apply(snap: bytes, mpo_blob: bytes, site1: int, x: np.ndarray, repeat: int = 1):
    """Oracle H_eff x on a frozen site problem; returns (y, flops_per_apply, seconds_per_apply)."""
    L = lib()
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros_like(x)
    fl, sec = c_double(), c_double()
    sb = ctypes.create_string_buffer(snap, len(snap))
    mb = ctypes.create_string_buffer(mpo_blob, len(mpo_blob))
    _check(L, L.orc_heff_apply(sb, len(snap), mb, len(mpo_blob), site1, _dp(x), _dp(y), x.size, repeat,
                               ctypes.byref(fl), ctypes.byref(sec)))
    return y, fl.value, sec.value


def jd_solve(snap: bytes, mpo_blob: bytes, site1: int, x0: np.ndarray, tol: float = 1e-10, maxiter: int = 8,
             ortho=(), gmres: int = 0):
    """Oracle Jacobi-Davidson on a frozen site problem: (eigenvalue, vector, iterations, H_eff applies)."""
    L = lib()
    x0 = np.ascontiguousarray(x0, dtype=np.float64)
    O = np.ascontiguousarray(np.array(ortho, dtype=np.float64).reshape(len(ortho), x0.size))
    out = np.zeros_like(x0)
    ev, it, na = c_double(), c_int(), c_int()
    sb = ctypes.create_string_buffer(snap, len(snap))
    mb = ctypes.create_string_buffer(mpo_blob, len(mpo_blob))
    _check(L, L.orc_jd_solve(sb, len(snap), mb, len(mpo_blob), site1, _dp(x0), x0.size, _dp(O) if len(ortho) else None,
                             len(ortho), gmres, tol, maxiter, _dp(out), ctypes.byref(ev), ctypes.byref(it),
                             ctypes.byref(na)))
    return ev.value, out, it.value, na.value


def heff_adjoint(snap: bytes, mpo_blob: bytes, site1: int, x: np.ndarray, ybar: np.ndarray, n_terms: int):
    """Oracle adjoint of H_eff x: (psi_bar = H ybar, d(ybar . H x)/d scale per two-site MPO entry)."""
    L = lib()
    x = np.ascontiguousarray(x, dtype=np.float64)
    ybar = np.ascontiguousarray(ybar, dtype=np.float64)
    pb = np.zeros_like(x)
    g = np.zeros(n_terms)
    sb = ctypes.create_string_buffer(snap, len(snap))
    mb = ctypes.create_string_buffer(mpo_blob, len(mpo_blob))
    _check(L, L.orc_heff_adjoint(sb, len(snap), mb, len(mpo_blob), site1, _dp(x), _dp(ybar), x.size, _dp(pb), _dp(g),
                                 n_terms))
    return pb, g


def schedule_export(snap: bytes, mpo_blob: bytes, site1: int):
    L = lib()
    p, n, fl = c_void_p(), c_size_t(), c_double()
    sb = ctypes.create_string_buffer(snap, len(snap))
    mb = ctypes.create_string_buffer(mpo_blob, len(mpo_blob))
    _check(L, L.orc_schedule_export(sb, len(snap), mb, len(mpo_blob), site1, ctypes.byref(p), ctypes.byref(n),
                                    ctypes.byref(fl)))
    b = ctypes.string_at(p, n.value)
    L.orc_free(p)
    return b, fl.value


def _u32(a):
    return a.ctypes.data_as(P(ctypes.c_uint32))


def truncate_svd(blocks, max_bond_dimension: int, cutoff: float):
    """svd_truncate (block_matrix_algorithms.h:185-240) of a list of 2-D blocks:
    ([(U, S, Vt) per block, kept columns only], dict(bond_dimension, truncated_weight,
    truncated_fraction, smallest_ev))."""
    L = lib()
    bl = [np.asarray(b, dtype=np.float64) for b in blocks]
    rows = np.array([b.shape[0] for b in bl], dtype=np.uint32)
    cols = np.array([b.shape[1] for b in bl], dtype=np.uint32)
    k = np.minimum(rows, cols).astype(np.int64)
    data = np.ascontiguousarray(np.concatenate([b.ravel(order="F") for b in bl]))
    U = np.zeros(max(1, int((rows * k).sum()))); S = np.zeros(max(1, int(k.sum()))); Vt = np.zeros(max(1, int((k * cols).sum())))
    keep = np.zeros(len(bl), dtype=np.uint32)
    res = np.zeros(4)
    _check(L, L.orc_truncate_svd(len(bl), _u32(rows), _u32(cols), _dp(data), max_bond_dimension, cutoff, _u32(keep), _dp(U),
                                 _dp(S), _dp(Vt), _dp(res)))
    return unpack_svd(rows, cols, keep, U, S, Vt), _result(res)


def truncate_heev(blocks, max_bond_dimension: int, cutoff: float):
    """heev_truncate (block_matrix_algorithms.h:299-355) of a list of symmetric blocks:
    ([(U, evals) per block, kept eigenpairs, descending], result dict)."""
    L = lib()
    bl = [np.asarray(b, dtype=np.float64) for b in blocks]
    dims = np.array([b.shape[0] for b in bl], dtype=np.uint32)
    data = np.ascontiguousarray(np.concatenate([b.ravel(order="F") for b in bl]))
    U = np.zeros(max(1, int((dims.astype(np.int64) ** 2).sum()))); ev = np.zeros(max(1, int(dims.sum())))
    keep = np.zeros(len(bl), dtype=np.uint32)
    res = np.zeros(4)
    _check(L, L.orc_truncate_heev(len(bl), _u32(dims), _dp(data), max_bond_dimension, cutoff, _u32(keep), _dp(U), _dp(ev),
                                  _dp(res)))
    return unpack_heev(dims, keep, U, ev), _result(res)


def _result(res):
    return {"bond_dimension": int(res[0]), "truncated_weight": res[1], "truncated_fraction": res[2], "smallest_ev": res[3]}


def unpack_svd(rows, cols, keep, U, S, Vt):
    """Per block (U rows x keep, S keep, Vt keep x cols) from the packed column-major arrays."""
    out, pu, ps, pv = [], 0, 0, 0
    for m, n, kp in zip(rows.tolist(), cols.tolist(), keep.tolist()):
        out.append((U[pu:pu + m * kp].reshape(kp, m).T.copy(), S[ps:ps + kp].copy(), Vt[pv:pv + kp * n].reshape(n, kp).T.copy()))
        pu += m * kp; ps += kp; pv += kp * n
    return out


def unpack_heev(dims, keep, U, ev):
    out, pu, pe = [], 0, 0
    for n, kp in zip(dims.tolist(), keep.tolist()):
        out.append((U[pu:pu + n * kp].reshape(kp, n).T.copy(), ev[pe:pe + kp].copy()))
        pu += n * kp; pe += kp
    return out
