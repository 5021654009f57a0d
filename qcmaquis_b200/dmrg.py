"""Two-site DMRG on the device: Jacobi-Davidson solve, boundary steps and the sweep.

Reference interface mirrored here:
    solve<double>(out, initial, SH, ortho, jcd_gmres, jcd_tol, jcd_max_iter)   (solver/solver.cpp:14-28)
    contraction::Engine::overlap_mpo_left_step / overlap_mpo_right_step       (contractions/engine.hpp:54-71)
    ts_optimize::sweep                                                         (optimize/ts_optimize.hpp:114-362)
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import lib, check, P, c_int, c_void_p, c_uint64, c_double
from .heff import Boundary, HeffPlan, MPSDesc, _sectors, precision_mode


class DMRGParams(ctypes.Structure):
    _fields_ = [("max_bond_dimension", c_uint64), ("init_bond_dimension", c_uint64), ("truncation_cutoff", c_double),
                ("jcd_tol", c_double), ("jcd_maxiter", ctypes.c_int32), ("ecore", c_double),
                ("twosite_truncation", ctypes.c_int32), ("alpha_initial", c_double), ("alpha_main", c_double),
                ("alpha_final", c_double), ("ngrowsweeps", ctypes.c_int32), ("nmainsweeps", ctypes.c_int32),
                ("hpsi_precision", ctypes.c_int32), ("jcd_gmres", ctypes.c_int32), ("optimization", ctypes.c_int32),
                ("mixed_residual_floor", c_double), ("mixed_fp64_refine", ctypes.c_int32)]


OPTIMIZATION = {"twosite": 0, "singlesite": 1}


def _params(M, init_bd, cutoff, tol, maxiter, ecore, heev, precision="fp64", gmres=0, optimization="twosite",
            mixed_floor=0.0, mixed_refine=0):
    """heev: None (svd truncation) or dict(alpha_initial, alpha_main, alpha_final, ngrowsweeps, nmainsweeps);
    precision: "fp64" or "mixed" (JD with the mixed H.psi, then the FP64 residual correction: the FP64
    Rayleigh quotient and up to mixed_refine FP64 correction steps; mixed_floor: 0 (the default) stops the
    mixed iterations by the FP64 rule, so the sweep follows the FP64 sweep's path; > 0 also stops them once
    the residual stalls below mixed_floor |theta|);
    gmres: ietl_jcd_gmres, GMRES iterations per JD correction;
    optimization: "twosite" (ts_optimize) or "singlesite" (ss_optimize: the alphas of heev, or its defaults,
    are the noise of every step's growth)."""
    if optimization not in OPTIMIZATION:
        raise ValueError(f"optimization must be one of {sorted(OPTIMIZATION)}")
    h = heev or {}
    return DMRGParams(M, init_bd, cutoff, tol, maxiter, ecore, 1 if heev else 0, h.get("alpha_initial", 1e-2),
                      h.get("alpha_main", 1e-4), h.get("alpha_final", 1e-8), h.get("ngrowsweeps", 0),
                      h.get("nmainsweeps", 0), precision_mode(precision), gmres, OPTIMIZATION[optimization],
                      mixed_floor, mixed_refine)


class TruncResult(ctypes.Structure):
    _fields_ = [("bond_dimension", c_uint64), ("truncated_weight", c_double), ("truncated_fraction", c_double),
                ("smallest_ev", c_double)]


class DMRGStats(ctypes.Structure):
    _fields_ = [("hpsi_count", c_uint64), ("hpsi_flops", c_double), ("plan_s", c_double), ("jd_s", c_double),
                ("trunc_s", c_double), ("boundary_s", c_double), ("total_s", c_double),
                ("hpsi_count_fp64", c_uint64), ("hpsi_flops_fp64", c_double), ("plans_built", c_uint64),
                ("plans_reused", c_uint64), ("bsteps_built", c_uint64), ("bsteps_reused", c_uint64),
                ("boundary_bytes_peak", c_uint64), ("boundaries_offloaded", c_uint64), ("boundaries_fetched", c_uint64)]


_lib._sig("qcm_jd_solve", c_int, c_void_p, P(c_double), c_double, c_int, P(c_double), P(c_double), P(c_int))
_lib._sig("qcm_jd_solve_mode", c_int, c_void_p, P(c_double), c_double, c_int, c_int, P(c_double), P(c_double), P(c_int))
_lib._sig("qcm_jd_solve_ex", c_int, c_void_p, P(c_double), P(P(c_double)), c_int, c_int, c_double, c_int, c_int,
          P(c_double), P(c_double), P(c_int), P(c_int))
_lib._sig("qcm_boundary_step_left", c_int, c_void_p, c_void_p, c_void_p, c_int, P(MPSDesc), P(c_double), c_int,
          P(c_void_p))
_lib._sig("qcm_boundary_step_right", c_int, c_void_p, c_void_p, c_void_p, c_int, P(MPSDesc), P(c_double), c_int,
          P(c_void_p))
_lib._sig("qcm_dmrg_create", c_int, c_void_p, c_void_p, c_int, c_int, P(DMRGParams), P(c_void_p))
_lib._sig("qcm_dmrg_create_from_mps", c_int, c_void_p, c_void_p, P(DMRGParams), P(MPSDesc), P(P(c_double)),
          P(c_void_p))
_lib._sig("qcm_dmrg_create_from_mps_at", c_int, c_void_p, c_void_p, P(DMRGParams), P(MPSDesc), P(P(c_double)), c_int,
          P(c_void_p))
_lib._sig("qcm_dmrg_length", c_int, c_void_p)
_lib._sig("qcm_dmrg_steps_per_sweep", c_int, c_void_p)
_lib._sig("qcm_dmrg_set_ortho", c_int, c_void_p, c_int, P(MPSDesc), P(P(c_double)))
_lib._sig("qcm_dmrg_export_site", c_int, c_void_p, c_int, c_void_p, ctypes.c_size_t, P(ctypes.c_size_t))
_lib._sig("qcm_dmrg_measure_1rdm", c_int, c_void_p, P(c_double))
_lib._sig("qcm_dmrg_measure_2rdm_grad", c_int, c_void_p, P(c_double))
_lib._sig("qcm_dmrg_mpo_gradient", c_int, c_void_p, c_void_p, P(P(c_double)))
_lib._sig("qcm_dmrg_integral_gradient", c_int, c_void_p, P(c_double), P(c_double), P(c_double), P(c_double))
_lib._sig("qcm_dmrg_run", c_int, c_void_p, c_int, P(c_double), P(TruncResult), P(c_int))
_lib._sig("qcm_dmrg_next_step", c_int, c_void_p)
_lib._sig("qcm_dmrg_pending_plan", c_int, c_void_p, P(c_double), c_uint64, P(c_void_p))
_lib._sig("qcm_dmrg_pending_twin", c_int, c_void_p, P(c_double), c_uint64, P(c_uint64))
_lib._sig("qcm_dmrg_pending_export", c_int, c_void_p, c_int, c_void_p, ctypes.c_size_t, P(ctypes.c_size_t))
_lib._sig("qcm_dmrg_sweep", c_int, c_void_p, P(c_double), P(TruncResult))
_lib._sig("qcm_dmrg_get_stats", c_int, c_void_p, P(DMRGStats))
_lib._sig("qcm_dmrg_group_sweep", c_int, P(c_void_p), c_int, P(c_double), P(TruncResult))
_lib._sig("qcm_dmrg_set_boundary_budget", c_int, c_void_p, c_uint64)
_lib._sig("qcm_dmrg_set_coefficient_budget", c_int, c_void_p, c_uint64)
_lib._sig("qcm_dmrg_set_apply_budget", c_int, c_void_p, c_uint64)
_lib._sig("qcm_dmrg_bond_dimensions", c_int, c_void_p, P(c_uint64))
_lib._sig("qcm_dmrg_free", None, c_void_p)
_U32 = P(ctypes.c_uint32)
_lib._sig("qcm_truncate_svd", c_int, c_void_p, ctypes.c_uint32, _U32, _U32, P(c_double), c_uint64, c_double, _U32,
          P(c_double), P(c_double), P(c_double), P(TruncResult))
_lib._sig("qcm_truncate_heev", c_int, c_void_p, ctypes.c_uint32, _U32, P(c_double), c_uint64, c_double, _U32, P(c_double),
          P(c_double), P(TruncResult))


def _u32(a: np.ndarray):
    return a.ctypes.data_as(_U32)


def truncate_svd(ctx, blocks, max_bond_dimension: int, cutoff: float = 1e-16):
    """svd_truncate of a block matrix (list of 2-D blocks) on the device: ([(U, S, Vt) per block,
    kept columns only], truncation result dict)."""
    bl = [np.asarray(b, dtype=np.float64) for b in blocks]
    rows = np.array([b.shape[0] for b in bl], dtype=np.uint32)
    cols = np.array([b.shape[1] for b in bl], dtype=np.uint32)
    k = np.minimum(rows, cols).astype(np.int64)
    data = np.ascontiguousarray(np.concatenate([b.ravel(order="F") for b in bl]))
    U = np.zeros(max(1, int((rows * k).sum())))
    S = np.zeros(max(1, int(k.sum())))
    Vt = np.zeros(max(1, int((k * cols).sum())))
    keep = np.zeros(len(bl), dtype=np.uint32)
    r = TruncResult()
    check(lib.qcm_truncate_svd(ctx.h, len(bl), _u32(rows), _u32(cols), _lib.dptr(data), max_bond_dimension, cutoff, _u32(keep),
                               _lib.dptr(U), _lib.dptr(S), _lib.dptr(Vt), ctypes.byref(r)), "qcm_truncate_svd")
    out, pu, ps, pv = [], 0, 0, 0
    for m, n, kp in zip(rows.tolist(), cols.tolist(), keep.tolist()):
        out.append((U[pu:pu + m * kp].reshape(kp, m).T.copy(), S[ps:ps + kp].copy(), Vt[pv:pv + kp * n].reshape(n, kp).T.copy()))
        pu += m * kp; ps += kp; pv += kp * n
    return out, {f: getattr(r, f) for f, _ in TruncResult._fields_}


_lib._sig("qcm_qr_blocks", c_int, c_void_p, ctypes.c_uint32, _U32, _U32, P(c_double), c_int, P(c_double), P(c_double))


def qr_blocks(ctx, blocks, lq: bool = False):
    """Thin QR (or LQ) of every block on the device, one launch: [(Q, R) per block] (LQ: [(L, Q)])."""
    bl = [np.asarray(b, dtype=np.float64) for b in blocks]
    rows = np.array([b.shape[0] for b in bl], dtype=np.uint32)
    cols = np.array([b.shape[1] for b in bl], dtype=np.uint32)
    k = np.minimum(rows, cols).astype(np.int64)
    data = np.ascontiguousarray(np.concatenate([b.ravel(order="F") for b in bl]))
    nq = int((k * (cols if lq else rows)).sum())
    nr = int((k * (rows if lq else cols)).sum())
    Q, R = np.zeros(max(1, nq)), np.zeros(max(1, nr))
    check(lib.qcm_qr_blocks(ctx.h, len(bl), _u32(rows), _u32(cols), _lib.dptr(data), 1 if lq else 0, _lib.dptr(Q),
                            _lib.dptr(R)), "qcm_qr_blocks")
    out, pq, pr = [], 0, 0
    for m, n, kk in zip(rows.tolist(), cols.tolist(), k.tolist()):
        if lq:
            Qb = Q[pq:pq + kk * n].reshape(n, kk).T.copy()
            Lb = R[pr:pr + m * kk].reshape(kk, m).T.copy()
            out.append((Lb, Qb))
        else:
            Qb = Q[pq:pq + m * kk].reshape(kk, m).T.copy()
            Rb = R[pr:pr + kk * n].reshape(n, kk).T.copy()
            out.append((Qb, Rb))
        pq += kk * (n if lq else m); pr += kk * (m if lq else n)
    return out


def truncate_heev(ctx, blocks, max_bond_dimension: int, cutoff: float = 1e-16):
    """heev_truncate of symmetric blocks on the device: ([(U, evals) per block, kept eigenpairs in
    descending order], truncation result dict; truncated_weight = truncated_fraction)."""
    bl = [np.asarray(b, dtype=np.float64) for b in blocks]
    dims = np.array([b.shape[0] for b in bl], dtype=np.uint32)
    data = np.ascontiguousarray(np.concatenate([b.ravel(order="F") for b in bl]))
    U = np.zeros(max(1, int((dims.astype(np.int64) ** 2).sum())))
    ev = np.zeros(max(1, int(dims.sum())))
    keep = np.zeros(len(bl), dtype=np.uint32)
    r = TruncResult()
    check(lib.qcm_truncate_heev(ctx.h, len(bl), _u32(dims), _lib.dptr(data), max_bond_dimension, cutoff, _u32(keep),
                                _lib.dptr(U), _lib.dptr(ev), ctypes.byref(r)), "qcm_truncate_heev")
    out, pu, pe = [], 0, 0
    for n, kp in zip(dims.tolist(), keep.tolist()):
        out.append((U[pu:pu + n * kp].reshape(kp, n).T.copy(), ev[pe:pe + kp].copy()))
        pu += n * kp; pe += kp
    return out, {f: getattr(r, f) for f, _ in TruncResult._fields_}


def jd_solve(plan, x0: np.ndarray, tol: float = 1e-10, maxiter: int = 8, precision="fp64", ortho=(), gmres: int = 0,
             return_applies: bool = False):
    """Lowest eigenpair of a plan's H_eff from start vector x0: (eigenvalue, eigenvector, iterations[, applies]).
    precision "mixed": iterations with the mixed H.psi, eigenvalue = FP64 Rayleigh quotient.
    ortho: states the solution is kept orthogonal to (excited states); gmres: GMRES iterations per
    correction equation (ietl_jcd_gmres)."""
    x0 = np.ascontiguousarray(x0, dtype=np.float64)
    assert x0.size == plan.n
    out = np.empty_like(x0)
    ev, it, na = c_double(), c_int(), c_int()
    if len(ortho) == 0 and gmres == 0 and not return_applies:
        check(lib.qcm_jd_solve_mode(plan.h, _lib.dptr(x0), tol, maxiter, precision_mode(precision), _lib.dptr(out),
                                    ctypes.byref(ev), ctypes.byref(it)), "qcm_jd_solve_mode")
        return ev.value, out, it.value
    keep = [np.ascontiguousarray(o, dtype=np.float64) for o in ortho]
    for o in keep:
        assert o.size == plan.n
    ptrs = (P(c_double) * max(1, len(keep)))(*[_lib.dptr(o) for o in keep])
    check(lib.qcm_jd_solve_ex(plan.h, _lib.dptr(x0), ptrs, len(keep), gmres, tol, maxiter, precision_mode(precision),
                              _lib.dptr(out), ctypes.byref(ev), ctypes.byref(it), ctypes.byref(na)), "qcm_jd_solve_ex")
    return (ev.value, out, it.value, na.value) if return_applies else (ev.value, out, it.value)


def boundary_step(ctx, B: Boundary, mpo, site: int, phys, left, right, data_rp: np.ndarray, side: str,
                  symmetric: bool = True) -> Boundary:
    """New boundary from site tensor `site` (right-paired blocks concatenated in left-sector order)
    and the previous boundary B: side "left" (L[site] -> L[site+1]) or "right" (R[site+1] -> R[site])."""
    ps, ls, rs = _sectors(phys), _sectors(left), _sectors(right)
    d = MPSDesc()
    d.n_phys, d.n_left, d.n_right = len(phys), len(left), len(right)
    d.phys, d.left, d.right = ps, ls, rs
    data_rp = np.ascontiguousarray(data_rp, dtype=np.float64)
    h = c_void_p()
    fn = lib.qcm_boundary_step_left if side == "left" else lib.qcm_boundary_step_right
    check(fn(ctx.h, B.h, mpo.handle, site, ctypes.byref(d), _lib.dptr(data_rp), 1 if symmetric else 0, ctypes.byref(h)),
          "qcm_boundary_step_" + side)
    return Boundary.from_handle(ctx, h)


def _pack_sites(sites):
    """MPS site tensors (dict(phys, left, right, blocks), right-paired blocks in left-sector order) as C-ABI
    descriptors and data pointers; keep holds the arrays the pointers refer to."""
    descs = (MPSDesc * len(sites))()
    keep, ptrs = [], (P(c_double) * len(sites))()
    for i, st in enumerate(sites):
        if [tuple(b[0]) for b in st["blocks"]] != [tuple(x[:2]) for x in st["left"]]:
            raise ValueError(f"site {i}: expected one right-paired block per left sector, in sector order")
        ps, ls, rs = _sectors(st["phys"]), _sectors(st["left"]), _sectors(st["right"])
        data = np.ascontiguousarray(np.concatenate([blk.T.ravel() for (_, blk) in st["blocks"]]))
        keep += [ps, ls, rs, data]
        descs[i].n_phys, descs[i].n_left, descs[i].n_right = len(st["phys"]), len(st["left"]), len(st["right"])
        descs[i].phys, descs[i].left, descs[i].right = ps, ls, rs
        ptrs[i] = _lib.dptr(data)
    return descs, ptrs, keep


class DMRG:
    """Ground-state DMRG (TwoU1, init_state = const) with every step on the device: two-site sweeps
    (ts_optimize) or single-site sweeps (ss_optimize, optimization="singlesite")."""

    def __init__(self, ctx, mpo, nup: int, ndown: int, max_bond_dimension: int, init_bond_dimension: int | None = None,
                 truncation_cutoff: float = 1e-16, jcd_tol: float = 1e-10, jcd_maxiter: int = 8, ecore: float = 0.0,
                 heev: dict | None = None, precision="fp64", jcd_gmres: int = 0, optimization: str = "twosite",
                 mixed_floor: float = 0.0, mixed_refine: int = 0):
        self.ctx, self.mpo = ctx, mpo
        p = _params(max_bond_dimension, init_bond_dimension or max_bond_dimension, truncation_cutoff, jcd_tol,
                    jcd_maxiter, ecore, heev, precision, jcd_gmres, optimization, mixed_floor, mixed_refine)
        h = c_void_p()
        check(lib.qcm_dmrg_create(ctx.h, mpo.handle, nup, ndown, ctypes.byref(p), ctypes.byref(h)), "qcm_dmrg_create")
        self.h = h
        self.L = lib.qcm_dmrg_length(h)
        self.steps = lib.qcm_dmrg_steps_per_sweep(h)

    @classmethod
    def from_mps(cls, ctx, mpo, sites, max_bond_dimension: int, truncation_cutoff: float = 1e-16,
                 jcd_tol: float = 1e-10, jcd_maxiter: int = 8, ecore: float = 0.0, heev: dict | None = None,
                 precision="fp64", jcd_gmres: int = 0, optimization: str = "twosite", initial_site: int = 0,
                 mixed_floor: float = 0.0, mixed_refine: int = 0):
        """Restart from a given MPS: sites = [dict(phys, left, right, blocks)] with right-paired blocks
        (one per left sector, in sector order), sites 1 .. L-1 right-normalised.  initial_site > 0 resumes
        the sweep at that site (boundaries built from the given MPS, qcm_dmrg_create_from_mps_at)."""
        self = cls.__new__(cls)
        self.ctx, self.mpo = ctx, mpo
        p = _params(max_bond_dimension, max_bond_dimension, truncation_cutoff, jcd_tol, jcd_maxiter, ecore, heev,
                    precision, jcd_gmres, optimization, mixed_floor, mixed_refine)
        descs, ptrs, keep = _pack_sites(sites)
        h = c_void_p()
        check(lib.qcm_dmrg_create_from_mps_at(ctx.h, mpo.handle, ctypes.byref(p), descs, ptrs, initial_site,
                                              ctypes.byref(h)), "qcm_dmrg_create_from_mps_at")
        self.h = h
        self.L = lib.qcm_dmrg_length(h)
        self.steps = lib.qcm_dmrg_steps_per_sweep(h)
        return self

    def sweep(self):
        """One sweep: (energies[steps], list of truncation dicts); steps = 2L - 2 (two-site) or 2L."""
        n = self.steps
        E = np.zeros(n)
        tr = (TruncResult * n)()
        check(lib.qcm_dmrg_sweep(self.h, _lib.dptr(E), tr), "qcm_dmrg_sweep")
        return E, [{f: getattr(t, f) for f, _ in TruncResult._fields_} for t in tr]

    @staticmethod
    def group_sweep(runs):
        """One sweep of independent two-site FP64 runs in lockstep (one merged plan group and one lockstep
        Jacobi-Davidson per step): (energies[len(runs), steps], per run a list of truncation dicts)."""
        runs = list(runs)
        n, steps = len(runs), runs[0].steps
        E = np.zeros((n, steps))
        tr = (TruncResult * (n * steps))()
        hs = (c_void_p * n)(*[r.h.value for r in runs])
        check(lib.qcm_dmrg_group_sweep(hs, n, _lib.dptr(E), tr), "qcm_dmrg_group_sweep")
        T = [{f: getattr(t, f) for f, _ in TruncResult._fields_} for t in tr]
        return E, [T[i * steps:(i + 1) * steps] for i in range(n)]

    def run(self, stop_step: int):
        """Run the current sweep up to (not including) step stop_step: (energies, truncation dicts)."""
        n = self.steps
        E = np.zeros(n)
        tr = (TruncResult * n)()
        k = c_int()
        check(lib.qcm_dmrg_run(self.h, stop_step, _lib.dptr(E), tr, ctypes.byref(k)), "qcm_dmrg_run")
        return E[:k.value], [{f: getattr(t, f) for f, _ in TruncResult._fields_} for t in tr[:k.value]]

    @property
    def next_step(self) -> int:
        return lib.qcm_dmrg_next_step(self.h)

    def pending_plan(self):
        """(H_eff plan, start vector) of the pending step; the plan is valid until the sweep continues."""
        h = c_void_p()
        check(lib.qcm_dmrg_pending_plan(self.h, None, 0, ctypes.byref(h)), "qcm_dmrg_pending_plan")
        plan = HeffPlan.from_handle(self.ctx, h, owner=self)
        n = c_uint64()
        check(lib.qcm_dmrg_pending_twin(self.h, None, 0, ctypes.byref(n)), "qcm_dmrg_pending_twin")
        x = np.zeros(n.value)
        check(lib.qcm_dmrg_pending_twin(self.h, _lib.dptr(x), x.size, ctypes.byref(n)), "qcm_dmrg_pending_twin")
        assert x.size == plan.n
        return plan, x

    def pending_export(self, index_only: bool = False) -> bytes:
        """The pending step's frozen site problem ("QSPB" v1); index_only: sectors and boundary indices only."""
        n = ctypes.c_size_t()
        fl = 1 if index_only else 0
        check(lib.qcm_dmrg_pending_export(self.h, fl, None, 0, ctypes.byref(n)), "qcm_dmrg_pending_export")
        buf = ctypes.create_string_buffer(n.value)
        check(lib.qcm_dmrg_pending_export(self.h, fl, buf, n.value, ctypes.byref(n)), "qcm_dmrg_pending_export")
        return buf.raw

    def export_mps(self):
        """The current MPS as "QMPS" site blobs (right-paired; heff.parse_mps_tensor reads them)."""
        out = []
        for i in range(self.L):
            n = ctypes.c_size_t()
            check(lib.qcm_dmrg_export_site(self.h, i, None, 0, ctypes.byref(n)), "qcm_dmrg_export_site")
            buf = ctypes.create_string_buffer(n.value)
            check(lib.qcm_dmrg_export_site(self.h, i, buf, n.value, ctypes.byref(n)), "qcm_dmrg_export_site")
            out.append(buf.raw)
        return out

    def measure_1rdm(self) -> np.ndarray:
        """Spin-summed one-particle density matrix (L x L) of the current MPS, between sweeps."""
        g = np.zeros((self.L, self.L))
        check(lib.qcm_dmrg_measure_1rdm(self.h, _lib.dptr(g)), "qcm_dmrg_measure_1rdm")
        return g  # symmetric: column-major and row-major agree

    def measure_2rdm_grad(self) -> np.ndarray:
        """dE/dV_pqrs (L^4, [p, q, r, s]) of the current MPS for 8-fold symmetric integrals, between sweeps."""
        G = np.zeros(self.L ** 4)
        check(lib.qcm_dmrg_measure_2rdm_grad(self.h, _lib.dptr(G)), "qcm_dmrg_measure_2rdm_grad")
        return G.reshape((self.L,) * 4, order="F")

    def mpo_gradient(self, W) -> list:
        """dE/d scale of every entry of every site tensor of the single-site MPO W (an MPO object of the
        state's physical basis), E = <Psi|W|Psi> / <Psi|Psi>, through the adjoint of the single-site
        apply at each site; one array per site in W's entry order.  Between sweeps."""
        grads = [np.zeros(W.terms(k)["scale"].size) for k in range(self.L)]
        ptrs = (P(c_double) * self.L)(*[_lib.dptr(g) for g in grads])
        check(lib.qcm_dmrg_mpo_gradient(self.h, W.handle, ptrs), "qcm_dmrg_mpo_gradient")
        return grads

    def integral_gradient(self, h, V, with_V: bool = True):
        """(dE/dh [p, q], dE/dV [p, q, r, s] or None) for the QC Hamiltonian of the integrals h (L x L) and V
        (L^4, chemist notation, row-major as for MPO.qc), every array element its own variable: dh is the
        spin-summed 1-RDM; dV averaged over the 8 permutations of real (pq|rs) is measure_2rdm_grad."""
        L = self.L
        h = np.ascontiguousarray(h, dtype=np.float64).reshape(L, L)
        V = np.ascontiguousarray(V, dtype=np.float64).reshape(L, L, L, L)
        dh = np.zeros((L, L))
        dV = np.zeros((L, L, L, L)) if with_V else None
        check(lib.qcm_dmrg_integral_gradient(self.h, _lib.dptr(h), _lib.dptr(V), _lib.dptr(dh),
                                             _lib.dptr(dV) if with_V else None), "qcm_dmrg_integral_gradient")
        return dh, dV

    def set_ortho(self, states):
        """Excited states: states = [[site dicts of an ortho state, as for from_mps]]; every step's solution
        is kept orthogonal to their projections (ts_optimize.hpp:217-223).  Call at the start of a sweep."""
        sites = [st for state in states for st in state]
        descs, ptrs, keep = _pack_sites(sites)
        check(lib.qcm_dmrg_set_ortho(self.h, len(states), descs, ptrs), "qcm_dmrg_set_ortho")

    def set_boundary_budget(self, nbytes: int):
        """Device bytes allowed for the sweep's boundaries (0: no limit); over it, boundaries move to
        pinned host memory and back (qcm_dmrg_set_boundary_budget)."""
        check(lib.qcm_dmrg_set_boundary_budget(self.h, int(nbytes)), "qcm_dmrg_set_boundary_budget")

    def set_coefficient_budget(self, nbytes: int):
        """Device bytes of coefficient blocks each H_eff plan built from here on keeps (0: no limit); larger
        plans generate them chunk by chunk in every apply (qcm_dmrg_set_coefficient_budget)."""
        check(lib.qcm_dmrg_set_coefficient_budget(self.h, int(nbytes)), "qcm_dmrg_set_coefficient_budget")

    def set_apply_budget(self, nbytes: int):
        """Device bytes of T, S and coefficient blocks one apply chunk of the plans built from here on may
        hold (0: whole applies; qcm_dmrg_set_apply_budget)."""
        check(lib.qcm_dmrg_set_apply_budget(self.h, int(nbytes)), "qcm_dmrg_set_apply_budget")

    def stats(self) -> dict:
        s = DMRGStats()
        check(lib.qcm_dmrg_get_stats(self.h, ctypes.byref(s)), "qcm_dmrg_get_stats")
        return {f: getattr(s, f) for f, _ in DMRGStats._fields_}

    def bond_dimensions(self) -> np.ndarray:
        d = np.zeros(self.L - 1, dtype=np.uint64)
        check(lib.qcm_dmrg_bond_dimensions(self.h, d.ctypes.data_as(P(c_uint64))), "qcm_dmrg_bond_dimensions")
        return d

    def __del__(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib.qcm_dmrg_free(self.h)
            self.h = c_void_p()
