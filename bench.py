#!/usr/bin/env python
"""Benchmark of the two-site DMRG effective-Hamiltonian hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--L 24] [--M 512] [--seed 0] [--sweeps 8]

Workload (both arms build it the same way, without running a sweep): the seeded
synthetic ab-initio Hamiltonian of the precision-form configuration (L = 24
orbitals, N = 24 electrons, TwoU1 Sz = 0, seed 0) and an MPS whose bond sectors
are those of a converged M = 512 two-site DMRG state of it (recorded in
tests/golden/bench_sectors_L24_M512.json by tests/golden/make_bench_sectors.py),
with site-tensor entries drawn from numpy.random.default_rng(seed).  The frozen
site problem is the two-site problem at the middle bond (sites L/2 - 1, L/2):
left boundaries over the sites before it and right boundaries over the sites
after it, built from that MPS with the MPO's Hermitian pairs (the reference's
init_left_right(mpo, site), optimize/optimize.h:158-195).

A step is one H_eff . psi (the Davidson callback, super_hamil_mv) on that frozen
problem.  `value` = reference work count (ScheduleNew::total_flops,
solver/tasks.cpp:388-398, 777-796) x steps / device time (CUDA events on the
plan stream, L2 flushed between steps), summed over ranks / max over ranks.
`e2e` is the same metric through qcm_heff_apply with pinned host buffers (H2D
of psi and D2H of H.psi inside the timed region).  The path does not shard
across GPUs here (one B200 per solve): N > 1 runs N independent replicas.

Reported beside the metric (not part of it): the mixed-precision forms of the
same step; the adjoint; `--sweeps` full two-site sweeps of the configuration
from the const initial state in the FP64 form and in the mixed form (per-sweep
time, energy, truncated weight and the mixed form's deviations); one
single-site sweep; the boundary storage with and without the Hermitian pairs;
the batching form (128 independent L=12, M=128 problems as one plan group:
grouped apply and lockstep Jacobi-Davidson against separate ones).

The reference arm (--impl reference) times the CPU restatement of the same
H.psi (the oracle: OpenMP over ket sectors, OpenBLAS dgemm, all host threads)
on the same frozen problem, which it builds itself (the oracle's boundary steps
over the same MPS); it loads no library of the device path.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import struct
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--L", type=int, default=24)
    ap.add_argument("--M", type=int, default=512)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--sweeps", type=int, default=8, help="sweeps of the FP64 / mixed sweep comparison (0: none)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed-sweep", action="store_true", help="skip the mixed-precision sweeps")
    ap.add_argument("--no-single-site-sweep", action="store_true", help="skip the single-site sweep")
    ap.add_argument("--no-extras", action="store_true", help="the metric only (no sweeps, forms, adjoint)")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-solve form")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# the frozen problem's inputs (numpy only: shared by both arms)

def _fcidump():
    """The integral recipe module, loaded from its file (importing the package would load the device library)."""
    spec = importlib.util.spec_from_file_location("qcm_fcidump", os.path.join(ROOT, "qcmaquis_b200", "fcidump.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def bond_sectors(a):
    path = os.path.join(ROOT, "tests", "golden", f"bench_sectors_L{a.L}_M{a.M}.json")
    with open(path) as f:
        d = json.load(f)
    if d["L"] != a.L or d["M"] != a.M:
        raise ValueError(f"{path}: sector fixture for another configuration")
    return [tuple(p) for p in d["phys"]], [[tuple(s) for s in b] for b in d["bonds"]], os.path.basename(path)


def synthetic_mps(phys, bonds, seed):
    """Site tensors (dict(phys, left, right, blocks)) over the given bond sectors, right-paired: one block per
    left sector (rows: its size; columns: the phys sectors in order, each with the right sector it leads to),
    entries N(0, 1) / sqrt(4 D_left), drawn site by site and block by block from default_rng(seed)."""
    rng = np.random.default_rng(seed)
    sites = []
    for i in range(len(bonds) - 1):
        left, right = bonds[i], bonds[i + 1]
        rsize = {(s[0], s[1]): s[2] for s in right}
        dleft = sum(s[2] for s in left)
        blocks = []
        for (qa, qb, ls) in left:
            stripe = sum(d * rsize.get((qa + pa, qb + pb), 0) for (pa, pb, d) in phys)
            if stripe == 0:
                raise ValueError(f"site {i}: left sector {(qa, qb)} reaches no right sector")
            blocks.append(((qa, qb), rng.standard_normal((ls, stripe)) / np.sqrt(4.0 * dleft)))
        sites.append(dict(phys=list(phys), left=list(left), right=list(right), blocks=blocks))
    return sites


def qmps_blob(site):
    """A site tensor as a "QMPS" v1 blob (right-paired blocks, column-major)."""
    out = [struct.pack("<II", 0x53504D51, 1)]
    for idx in (site["phys"], site["left"], site["right"]):
        out.append(struct.pack("<I", len(idx)))
        out += [struct.pack("<iiI", int(s[0]), int(s[1]), int(s[2])) for s in idx]
    out.append(struct.pack("<I", len(site["blocks"])))
    for (ch, blk) in site["blocks"]:
        out.append(struct.pack("<iiII", ch[0], ch[1], blk.shape[0], blk.shape[1]))
        out.append(np.ascontiguousarray(blk.T, dtype="<f8").tobytes())
    return b"".join(out)


def twin_of_problem(snap: bytes) -> np.ndarray:
    """The two-site tensor of a "QSPB" v1 site problem as the H_eff vector (its blocks, column-major, in order)."""
    off = 8
    for _ in range(3):
        (n,) = struct.unpack_from("<I", snap, off)
        off += 4 + 12 * n
    (nb,) = struct.unpack_from("<I", snap, off)
    off += 4
    parts = []
    for _ in range(nb):
        _, _, r, c = struct.unpack_from("<iiII", snap, off)
        off += 16
        parts.append(np.frombuffer(snap, dtype="<f8", count=r * c, offset=off))
        off += 8 * r * c
    return np.concatenate(parts)


def problem_inputs(a):
    fd = _fcidump()
    h, V, e = fd.synthetic_integrals(a.L, a.seed)
    phys, bonds, fixture = bond_sectors(a)
    sites = synthetic_mps(phys, bonds, a.seed)
    return h, V, sites, a.L // 2 - 1, fixture


def config_of(a, fixture, flops):
    return {"workload": (f"two-site H_eff.psi at the middle bond (sites {a.L // 2 - 1}, {a.L // 2}) of the synthetic "
                         f"ab-initio Hamiltonian L={a.L} N={a.L} TwoU1 Sz=0 seed {a.seed}; MPS with the bond sectors of "
                         f"a converged M={a.M} state ({fixture}), entries N(0,1) from default_rng({a.seed})"),
            "L": a.L, "N": a.L, "M": a.M, "seed": a.seed, "site": a.L // 2 - 1, "flops_per_step": float(flops),
            "boundaries": "Hermitian-paired MPO bonds (transposed partner cohorts)",
            "l2": "flushed between steps (256 MiB write)"}


def oracle_problem(h, V, sites, site1):
    """The frozen problem built by the oracle alone: (mpo blob, QSPB snapshot, twin vector)."""
    from oracle.oracle import mpo_blob_qc, site_problem
    blob = mpo_blob_qc(h, V)
    snap = site_problem(blob, [qmps_blob(s) for s in sites], site1)
    return blob, snap, twin_of_problem(snap)


# ---------------------------------------------------------------------------

class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        out, _ = self.p.communicate(timeout=10)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1])); mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(a):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1 and a.impl == "b200":
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(v, pg, dev):
    """The largest of every rank's v (a time): all ranks take part; with no process group, v."""
    if pg is None:
        return float(v)
    import torch
    t = torch.tensor([float(v)], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def measured_traffic(a):
    """DRAM bytes (read + written) of the S-GEMM phase per apply, from the ncu capture of this workload
    summarised in profiles/ (dram__bytes_read.sum + dram__bytes_write.sum), or (None, None)."""
    import re
    path = os.path.join(ROOT, "profiles", f"heff_launches_traffic_L{a.L}_M{a.M}.md")
    if a.seed != 0 or not os.path.exists(path):
        return None, None
    m = re.search(r"S-GEMM phase[^*]*\*\*([0-9.]+) GB\*\* per apply", open(path).read())
    return (float(m.group(1)) * 1e9, os.path.relpath(path, ROOT)) if m else (None, None)


def cpu_baseline(snap, blob, site, x, flops, budget_s=20.0):
    from oracle.oracle import heff_apply, lib as olib
    olib()
    y, _, sec = heff_apply(snap, blob, site, x, repeat=1)
    reps = max(1, min(50, int(budget_s / max(sec, 1e-3))))
    _, _, sec = heff_apply(snap, blob, site, x, repeat=reps)
    return {"value": flops / sec / 1e9, "unit": "GFLOP/s", "cores": olib().orc_max_threads(), "kind": "port",
            "sample": f"{reps} H_eff.psi applies of the same frozen problem (oracle, OpenMP over ket sectors, "
                      f"OpenBLAS dgemm), {sec * 1e3:.1f} ms each"}


def run_reference(a, world, rank):
    """The oracle's H.psi on the same frozen problem, with all host threads (rank 0 only)."""
    if rank != 0:
        return
    from oracle.oracle import heff_apply, lib as olib
    h, V, sites, site1, fixture = problem_inputs(a)
    blob, snap, x = oracle_problem(h, V, sites, site1)
    for _ in range(a.warmup):
        heff_apply(snap, blob, site1, x, repeat=1)
    t0 = time.perf_counter()
    _, flops, sec = heff_apply(snap, blob, site1, x, repeat=a.steps)
    wall = time.perf_counter() - t0
    val = flops / sec / 1e9
    cores = olib().orc_max_threads()
    line = {"impl": "reference", "metric": "H_eff.psi GFLOP/s (FP64 plain form)", "value": val, "unit": "GFLOP/s",
            "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup, "ms_per_step": sec * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_of(a, fixture, flops),
            "cpu_baseline": {"value": val, "unit": "GFLOP/s", "cores": cores, "kind": "port",
                             "sample": f"{a.steps} H_eff.psi applies ({wall:.1f} s) with all host threads"},
            "e2e": {"value": val, "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the oracle builds the frozen problem itself (its boundary steps over the same MPS, untimed)"}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# device arm

def device_problem(ctx, h, V, sites, site1, M, hermitian=True):
    """The frozen problem on the device: (dmrg, plan, x, mpo).  The device builds the boundaries from the
    same MPS (qcm_dmrg_create_from_mps_at); hermitian=False drops the MPO's Hermitian pairs."""
    from qcmaquis_b200.dmrg import DMRG
    from qcmaquis_b200.mpo import MPO
    m = MPO.qc(h, V)
    if not hermitian:
        ts = m.tensors()
        for t in ts:
            t["herm_left"], t["herm_right"] = None, None
        m = MPO.from_tensors(ts)
    d = DMRG.from_mps(ctx, m, sites, M, initial_site=site1)
    plan, x = d.pending_plan()
    return d, plan, x, m


def boundary_storage(d, plan):
    """Stored doubles and cohorts (transposed ones among them) of the pending step's two boundaries."""
    from qcmaquis_b200.heff import parse_site_problem
    p = parse_site_problem(d.pending_export(index_only=True))
    nc = sum(len(p[k]["tr"]) for k in ("L", "R"))
    ntr = sum(int(p[k]["tr"].sum()) for k in ("L", "R"))
    return {"doubles": int(plan.info["l_len"] + plan.info["r_len"]), "cohorts": nc, "transposed_cohorts": ntr,
            "stored_cohorts": nc - ntr, "flops_per_step": float(plan.info["flops"])}


def measure_mixed(a, plan, xd, yd, xp, yp, hb, flush, info, world, pg, dev, snap, blob, site, x_host, form="mixed"):
    """A mixed-precision form on the same frozen problem (S build 3xTF32 on the tensor cores, FP32
    accumulation; T-GEMM and L.S in FP64), same timing rules as the FP64 form."""
    import torch
    from qcmaquis_b200._lib import lib, check
    from qcmaquis_b200.heff import precision_mode
    mode = precision_mode(form)
    for _ in range(a.warmup):
        plan.apply_device(xd.data_ptr(), yd.data_ptr(), precision=form)
    torch.cuda.synchronize()
    times, phases = [], []
    torch.cuda.nvtx.range_push("timed_" + form)  # profilers select this form's timed launches by the range
    for _ in range(a.steps):
        flush.zero_()
        torch.cuda.synchronize()
        ms = plan.profile(xd.data_ptr(), yd.data_ptr(), precision=form)
        times.append(ms[3])
        phases.append(ms[:3])
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    total_ms = float(sum(times))
    e2e_t = []
    for _ in range(a.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        check(lib.qcm_heff_apply_mode(plan.h, xp, yp, mode), "qcm_heff_apply_mode")
        e2e_t.append(time.perf_counter() - t0)
    total_ms = max_over_ranks(total_ms, pg, dev)
    e2e_s = max_over_ranks(sum(e2e_t), pg, dev)
    ph = np.mean(np.array(phases), axis=0)
    y_mixed = hb["y"].numpy().copy()
    out = {"value": info["flops"] * a.steps * world / (total_ms * 1e-3) / 1e9, "unit": "GFLOP/s",
           "ms_per_step": total_ms / a.steps,
           "form": ("S build 3xTF32 (mma.sync m16n8k8, FP32 operands split at the fragment loads, FP32 accumulation), "
                    "T-GEMM and L.S FP64") if mode == 1 else
                   ("S build 3xTF32 from operands split in HBM: 16/32-line tiles on tcgen05 (accumulator in tensor memory), "
                    "others on mma.sync; T-GEMM and L.S FP64"),
           "e2e": {"value": info["flops"] * a.steps * world / e2e_s / 1e9, "unit": "GFLOP/s",
                   "h2d_bytes_per_step": 8 * plan.n, "d2h_bytes_per_step": 8 * plan.n},
           "phase_ms": {"k_tgemm": float(ph[0]), "k_sgemm_x3": float(ph[1]), "k_lspart+k_lsreduce": float(ph[2])},
           "s_build_tflops": info["flops_s"] / (ph[1] * 1e-3) / 1e12,
           "s_build_executed_tf32_tflops": 3 * info["flops_sexec"] / (ph[1] * 1e-3) / 1e12}
    if snap is not None:
        from oracle.oracle import heff_apply
        y_ref, _, _ = heff_apply(snap, blob, site, x_host)
        out["max_rel_err_vs_oracle"] = float(np.abs(y_mixed - y_ref).max() / np.abs(y_ref).max())
    return out


def measure_adjoint(a, plan, x_host, mpo, site):
    """The differentiation form on the same frozen problem: qcm_heff_adjoint with host buffers (x and
    ybar in, psi_bar and the gradient per two-site MPO entry out), wall time per call."""
    rng = np.random.default_rng(a.seed)
    ybar = rng.standard_normal(x_host.size)
    pb, g = plan.adjoint(x_host, ybar)  # first call: work lists and buffers
    reps = 3
    t0 = time.perf_counter()
    for _ in range(reps):
        pb, g = plan.adjoint(x_host, ybar)
    dt = (time.perf_counter() - t0) / reps
    # f = ybar . H x is linear in the scales: the gradient contracted with the scales gives f back
    terms = mpo.twosite().terms(site)["scale"]
    f = float(ybar @ plan.apply(x_host))
    return {"ms_per_call": dt * 1e3, "n_terms": int(g.size), "h2d_bytes": 16 * x_host.size,
            "d2h_bytes": 8 * (x_host.size + g.size),
            "euler_check_rel": abs(float(g @ terms) - f) / abs(f),
            "note": "psi_bar = H ybar and d(ybar.Hx)/d scale per entry; sum_e scale_e * grad_e = ybar.Hx (f is linear "
                    "in the scales) is the consistency check"}


def measure_streamed(a, plan, xd, yd, flush, info):
    """The same H.psi with its coefficient blocks streamed through a bounded scratch (generated chunk by
    chunk in every apply instead of kept, the form for problems whose blocks do not fit): per chunk size the
    time per apply and of its S phase (CUDA events, L2 flushed), and whether the result equals the kept
    form's to the bit."""
    import torch
    plan.apply_device(xd.data_ptr(), yd.data_ptr())
    torch.cuda.synchronize()
    y_kept = yd.clone()
    out = {"coefficient_block_bytes": 8 * int(info["w_len"]), "chunks": []}
    try:
        for mib in (512, 128):
            plan.stream_coefficients(mib * 2**20)
            for _ in range(3):
                plan.apply_device(xd.data_ptr(), yd.data_ptr())
            tot, sph = [], []
            for _ in range(10):
                flush.zero_()
                torch.cuda.synchronize()
                ms = plan.profile(xd.data_ptr(), yd.data_ptr())
                tot.append(ms[3])
                sph.append(ms[1])
            torch.cuda.synchronize()
            out["chunks"].append({"chunk_bytes": mib * 2**20, "launches_per_apply": int(plan.info["launches"]),
                                  "ms_per_apply": float(np.mean(tot)), "s_phase_ms": float(np.mean(sph)),
                                  "gflops": info["flops"] / (np.mean(tot) * 1e-3) / 1e9,
                                  "bitwise_equal_to_kept": bool(torch.equal(yd, y_kept))})
        # the apply cut by ket sector: T, coefficient blocks, S and split-K partials chunk by chunk
        out["sector_chunks"] = []
        whole = 8 * (int(info["t_len"]) + int(info["s_len"]) + int(info["w_len"]))
        ts_bytes, w_bytes = 8 * (int(info["t_len"]) + int(info["s_len"])), 8 * int(info["w_len"])
        # two budgets below the coefficient blocks' share (each chunk generates its own), and one that
        # keeps them whole (generated once) while T and S run in four chunks
        for budget in (whole // 4, whole // 16, max(2 * w_bytes, w_bytes + ts_bytes // 4)):
            plan.chunk_apply(budget)
            for _ in range(3):
                plan.apply_device(xd.data_ptr(), yd.data_ptr())
            tot = []
            for _ in range(10):
                flush.zero_()
                torch.cuda.synchronize()
                tot.append(plan.profile(xd.data_ptr(), yd.data_ptr())[3])
            torch.cuda.synchronize()
            out["sector_chunks"].append({"budget_bytes": budget, "launches_per_apply": int(plan.info["launches"]),
                                         "ms_per_apply": float(np.mean(tot)),
                                         "gflops": info["flops"] / (np.mean(tot) * 1e-3) / 1e9,
                                         "bitwise_equal_to_kept": bool(torch.equal(yd, y_kept))})
    finally:
        plan.chunk_apply(0)
        plan.stream_coefficients(0)
    return out


def sweep_record(d, E, tr, dt, st0, st1, s):
    tw = np.array([t["truncated_weight"] for t in tr])
    return {"sweep": s, "seconds": dt, "energy_min": float(E.min()), "truncated_weight_max": float(tw.max()),
            "truncated_weight_sum": float(tw.sum()),
            "max_bond_dimension": int(max(t["bond_dimension"] for t in tr)),
            "hpsi": int(st1["hpsi_count"] - st0["hpsi_count"]),
            "hpsi_fp64_rayleigh": int(st1["hpsi_count_fp64"] - st0["hpsi_count_fp64"]),
            "hpsi_gflop": (st1["hpsi_flops"] - st0["hpsi_flops"]) / 1e9,
            "plans_reused": int(st1["plans_reused"] - st0["plans_reused"]),
            "boundary_schedules_reused": int(st1["bsteps_reused"] - st0["bsteps_reused"]),
            "phase_s": {k: st1[k] - st0[k] for k in ("plan_s", "jd_s", "trunc_s", "boundary_s")}}


def run_sweeps(a, ctx, h, V, precision):
    """`a.sweeps` two-site sweeps of the configuration from the const initial state (init_bond_dimension 64)."""
    from qcmaquis_b200.dmrg import DMRG
    from qcmaquis_b200.mpo import MPO
    m = MPO.qc(h, V)
    d = DMRG(ctx, m, a.L // 2, a.L // 2, a.M, 64, precision=precision)
    out = []
    for s in range(a.sweeps):
        st0 = d.stats()
        t0 = time.perf_counter()
        E, tr = d.sweep()
        dt = time.perf_counter() - t0
        out.append(sweep_record(d, E, tr, dt, st0, d.stats(), s))
    return d, m, out


def single_site_sweep(a, ctx, m, d, e_ts):
    """One single-site sweep (optimization = singlesite: 2L steps, density-matrix growth with noise 1e-8)
    from the two-site sweeps' MPS at the same Mmax: its time, phases and H.psi work, and its lowest energy
    against the last two-site sweep's.  A failure is recorded, not raised."""
    from qcmaquis_b200.dmrg import DMRG
    from qcmaquis_b200.heff import parse_mps_tensor
    try:
        sites = [parse_mps_tensor(b) for b in d.export_mps()]
        noise = dict(alpha_initial=1e-8, alpha_main=1e-8, alpha_final=1e-8)
        s = DMRG.from_mps(ctx, m, sites, a.M, heev=noise, optimization="singlesite")
        del sites
        st0 = s.stats()
        t0 = time.perf_counter()
        E, tr = s.sweep()
        dt = time.perf_counter() - t0
        st1 = s.stats()
        out = {"steps": int(E.size), "seconds": dt, "energy_min": float(E.min()),
               "energy_dev_vs_twosite": float(E.min() - e_ts),
               "max_bond_dimension": int(max(t["bond_dimension"] for t in tr)),
               "hpsi": int(st1["hpsi_count"] - st0["hpsi_count"]),
               "hpsi_gflop": (st1["hpsi_flops"] - st0["hpsi_flops"]) / 1e9,
               "phase_s": {k: st1[k] - st0[k] for k in ("plan_s", "jd_s", "trunc_s", "boundary_s")}}
        del s
        return out
    except Exception as ex:  # reported beside the metric, never in place of it
        return {"error": f"{type(ex).__name__}: {ex}"}


def batched_solves(a, ctx, n=128, L=12, M=128):
    """The batching form on the batched-solve configuration: n independent problems (synthetic Hamiltonians
    of L orbitals, N = L, seeds 1 .. n; MPS over the bond sectors of a converged M state, seeded entries), the
    two-site problem at the middle bond of each.  Their plans merged into one group: one apply of all against
    n separate applies, and one lockstep Jacobi-Davidson (each iteration a CUDA graph) against n separate
    solves (tol 1e-10, maxiter 8), with the largest eigenvalue difference."""
    import torch
    from qcmaquis_b200 import heff
    from qcmaquis_b200.dmrg import jd_solve
    fd = _fcidump()
    phys, bonds, fixture = bond_sectors(argparse.Namespace(L=L, M=M))
    site1 = L // 2 - 1
    t0 = time.perf_counter()
    dmrgs, plans, xs = [], [], []
    for seed in range(1, n + 1):
        h, V, _ = fd.synthetic_integrals(L, seed)
        d, plan, x, _ = device_problem(ctx, h, V, synthetic_mps(phys, bonds, seed), site1, M)
        dmrgs.append(d); plans.append(plan); xs.append(x)
    g = heff.HeffGroup(ctx, plans)
    setup = time.perf_counter() - t0
    dev = torch.device("cuda", torch.cuda.current_device())
    X = torch.from_numpy(g.pack(xs)).to(dev)
    Y = torch.empty_like(X)
    xd = [torch.from_numpy(x).to(dev) for x in xs]
    yd = [torch.empty_like(x) for x in xd]
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, reps):
        for _ in range(3):
            fn()
        ctx.synchronize()
        torch.cuda.synchronize()
        t = time.perf_counter()
        for _ in range(reps):
            fn()
        ctx.synchronize()
        return (time.perf_counter() - t) / reps

    t_group = timed(lambda: g.apply_device(X.data_ptr(), Y.data_ptr()), 20)
    t_sep = timed(lambda: [p.apply_device(x.data_ptr(), y.data_ptr()) for p, x, y in zip(plans, xd, yd)], 5)
    x0 = g.pack(xs)
    t = time.perf_counter()
    evb, _, itb, napply = g.jd_solve(x0, 1e-10, 8, graphs=True)
    t_jd_group = time.perf_counter() - t
    t = time.perf_counter()
    ev_sep = [jd_solve(p, x, 1e-10, 8)[0] for p, x in zip(plans, xs)]
    t_jd_sep = time.perf_counter() - t
    flops = g.info["flops"]
    out = {"workload": (f"{n} independent two-site problems at the middle bond: synthetic Hamiltonians L={L} N={L} "
                        f"TwoU1 Sz=0 seeds 1..{n}, MPS over the bond sectors of a converged M={M} state ({fixture}), "
                        f"seeded entries"),
           "setup_s": setup, "flops_per_group_apply": flops, "launches_per_group_apply": int(g.info["launches"]),
           "group_apply_ms": t_group * 1e3, "separate_applies_ms": t_sep * 1e3,
           "group_apply_gflops": flops / t_group / 1e9, "separate_applies_gflops": flops / t_sep / 1e9,
           "group_jd_s": t_jd_group, "separate_jd_s": t_jd_sep, "group_jd_applies": napply,
           "jd_max_abs_eigenvalue_diff": float(np.max(np.abs(np.array(ev_sep) - evb))),
           "note": "wall times with host synchronisation; the group JD replays one CUDA graph per iteration"}
    del g, plans, dmrgs
    return out


def group_sweeps(a, ctx, n=16, L=12, M=128, sweeps=6):
    """Whole DMRG runs in lockstep: n independent two-site FP64 runs (synthetic Hamiltonians of L orbitals,
    N = L, seeds 1 .. n, const initial state with bond dimension 16, Mmax M) swept together by
    qcm_dmrg_group_sweep (one merged plan group and one lockstep JD per step) against the same runs swept one
    after the other; per-sweep wall times of both and the largest step-energy difference between them."""
    from qcmaquis_b200.dmrg import DMRG
    from qcmaquis_b200.mpo import MPO
    fd = _fcidump()
    mpos = []
    for seed in range(1, n + 1):
        h, V, _ = fd.synthetic_integrals(L, seed)
        mpos.append(MPO.qc(h, V))
    grp = [DMRG(ctx, m, L // 2, L // 2, M, 16) for m in mpos]
    sep = [DMRG(ctx, m, L // 2, L // 2, M, 16) for m in mpos]
    t_grp, t_sep, dE = [], [], []
    for s in range(sweeps):
        t = time.perf_counter()
        Eg, _ = DMRG.group_sweep(grp)
        t_grp.append(time.perf_counter() - t)
        t = time.perf_counter()
        Es = np.array([d.sweep()[0] for d in sep])
        t_sep.append(time.perf_counter() - t)
        dE.append(float(np.abs(Eg - Es).max()))
    st = [d.stats() for d in grp]
    out = {"workload": (f"{n} independent two-site DMRG runs: synthetic Hamiltonians L={L} N={L} TwoU1 Sz=0 seeds "
                        f"1..{n}, Mmax {M}, const initial state (bond dimension 16), jcd_tol 1e-10, maxiter 8"),
           "group_sweep_s": t_grp, "separate_sweeps_s": t_sep,
           "group_jd_s": sum(x["jd_s"] for x in st), "group_plan_s": sum(x["plan_s"] for x in st),
           "group_trunc_s": sum(x["trunc_s"] for x in st), "group_boundary_s": sum(x["boundary_s"] for x in st),
           "max_abs_step_energy_diff": dE,
           "note": "wall times; the group form batches the JD of every step, truncation and boundary steps run per run"}
    del grp, sep
    return out


def sweep_comparison(a, ctx, h, V):
    """FP64 and mixed-form sweeps from the same const state: per-sweep time, energy, truncated weight, and
    the mixed form's deviations from the FP64 sweeps (the FP64 device sweeps match the oracle's to 1e-10 Eh
    in the parity tests)."""
    d64, m, fp64 = run_sweeps(a, ctx, h, V, "fp64")
    out = {"sweeps": a.sweeps, "init_bond_dimension": 64, "fp64": fp64}
    if not a.no_single_site_sweep:
        out["single_site"] = single_site_sweep(a, ctx, m, d64, fp64[-1]["energy_min"])
    del d64
    if not a.no_mixed_sweep:
        dmx, _, mixed = run_sweeps(a, ctx, h, V, "mixed")
        del dmx
        for r, r64 in zip(mixed, fp64):
            r["energy_dev_vs_fp64"] = r["energy_min"] - r64["energy_min"]
            r["truncated_weight_sum_dev_vs_fp64"] = r["truncated_weight_sum"] - r64["truncated_weight_sum"]
        out["mixed"] = mixed
        out["max_abs_energy_dev"] = max(abs(r["energy_dev_vs_fp64"]) for r in mixed)
    return out


def run_b200(a, world, rank, local, pg):
    import ctypes
    import torch
    from qcmaquis_b200 import heff
    from qcmaquis_b200._lib import lib, check, P, c_double
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    h, V, sites, site1, fixture = problem_inputs(a)
    ctx = heff.Context(local)
    d, plan, x_host, mpo = device_problem(ctx, h, V, sites, site1, a.M)
    info = plan.info
    n = plan.n
    xd = torch.from_numpy(x_host).to(dev)
    yd = torch.empty_like(xd)
    flush = torch.empty(int(256 * 2**20 // 4), dtype=torch.float32, device=dev)  # 256 MiB > L2 (126 MB)
    dmma_peak, dfma_peak = heff.probe_fp64_peaks()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()  # sampled from the warm-up on, stopped after the timed region
    for _ in range(a.warmup):
        plan.apply_device(xd.data_ptr(), yd.data_ptr())
    ctx.synchronize()
    # timed region: per-step CUDA events on the plan's stream via qcm_heff_profile
    if pg is not None:
        pg.barrier()
    torch.cuda.synchronize()
    times, phases = [], []
    torch.cuda.nvtx.range_push("timed")  # profilers select the timed launches by this range
    for _ in range(a.steps):
        flush.zero_()
        torch.cuda.synchronize()
        ms = plan.profile(xd.data_ptr(), yd.data_ptr())
        times.append(ms[3])
        phases.append(ms[:3])
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    ck = clocks.stop()
    total_ms = max_over_ranks(sum(times), pg, dev)
    if pg is not None:
        pg.barrier()
    value = info["flops"] * a.steps * world / (total_ms * 1e-3) / 1e9
    # e2e through the C-ABI with pinned host buffers
    xh = torch.from_numpy(x_host).pin_memory()
    yh = torch.empty_like(xh).pin_memory()
    xp = ctypes.cast(xh.data_ptr(), P(c_double))
    yp = ctypes.cast(yh.data_ptr(), P(c_double))
    for _ in range(2):
        check(lib.qcm_heff_apply(plan.h, xp, yp), "qcm_heff_apply")
    e2e_t = []
    for _ in range(a.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        check(lib.qcm_heff_apply(plan.h, xp, yp), "qcm_heff_apply")
        e2e_t.append(time.perf_counter() - t0)
    e2e_s = max_over_ranks(sum(e2e_t), pg, dev)
    e2e_val = info["flops"] * a.steps * world / e2e_s / 1e9
    y_dev = yh.numpy().copy()
    # the checker: the oracle builds the same problem itself; the device result against it, and the
    # device's own twin against the oracle's
    snap = blob = None
    rel = twin_rel = None
    want_oracle = rank == 0 and not a.no_cpu_baseline
    if want_oracle:
        from oracle.oracle import heff_apply
        blob, snap, x_or = oracle_problem(h, V, sites, site1)
        twin_rel = float(np.abs(x_or - x_host).max() / np.abs(x_or).max())
        y_ref, flops_or, _ = heff_apply(snap, blob, site1, x_host)
        rel = float(np.abs(y_dev - y_ref).max() / np.abs(y_ref).max())
        if flops_or != info["flops"]:
            raise RuntimeError(f"device and oracle work counts differ: {info['flops']} vs {flops_or}")
    # roofline of the dominant kernel (phase): reference flop count of the phase / its device time
    ph = np.mean(np.array(phases), axis=0)
    names = ["k_tgemm", "k_sgemm", "k_lspart+k_lsreduce"]
    work = [info["flops_t"], info["flops_s"], info["flops_ls"]]
    dom = int(np.argmax(ph))
    ach = work[dom] / (ph[dom] * 1e-3) / 1e12
    traffic, tsrc = measured_traffic(a)
    roof = {"kernel": names[dom], "bound": "tensor", "achieved": ach, "peak": dmma_peak, "unit": "TFLOP/s",
            "frac": ach / dmma_peak, "traffic": traffic if dom == 1 else None, "traffic_source": tsrc,
            "traffic_min_bytes": 8.0 * (info["w_len"] + info["t_len"] + info["s_len"]),
            "algorithmic": "reference flop count of the phase (ScheduleNew::total_flops terms)",
            "peak_source": "FP64 DMMA probe qcm_probe_fp64_peaks (of measured)"}
    if dom == 1:
        roof["executed_tflops"] = info["flops_sexec"] / (ph[1] * 1e-3) / 1e12
        roof["executed_frac"] = roof["executed_tflops"] / dmma_peak
    roof["phase_ms"] = {k: float(v) for k, v in zip(names, ph)}
    extras = {}
    if not a.no_extras:
        hb = {"xh": xh, "y": yh}
        mixed = measure_mixed(a, plan, xd, yd, xp, yp, hb, flush, info, world, pg, dev, snap, blob, site1, x_host)
        mixed["tensor_memory_form"] = measure_mixed(a, plan, xd, yd, xp, yp, hb, flush, info, world, pg, dev, snap,
                                                    blob, site1, x_host, form="mixed_tc")
        extras["mixed"] = mixed
        extras["adjoint"] = measure_adjoint(a, plan, x_host, mpo, site1)
        extras["streamed_coefficients"] = measure_streamed(a, plan, xd, yd, flush, info)
        herm = boundary_storage(d, plan)
        del plan, d
        dn, pn, _, _ = device_problem(ctx, h, V, sites, site1, a.M, hermitian=False)
        extras["boundary_storage"] = {"hermitian_pairs": herm, "no_pairs": boundary_storage(dn, pn)}
        del pn, dn
        if a.sweeps > 0:
            extras["sweep"] = sweep_comparison(a, ctx, h, V)
        if not a.no_batched:
            try:
                extras["batched"] = batched_solves(a, ctx)
            except FileNotFoundError as ex:  # the sector fixture of the batched configuration is missing
                extras["batched"] = {"error": str(ex)}
            extras["group_sweeps"] = group_sweeps(a, ctx)
    cpu = None
    if want_oracle and world == 1:
        cpu = cpu_baseline(snap, blob, site1, x_host, info["flops"])
    if rank == 0:
        line = {"metric": "H_eff.psi GFLOP/s (FP64 plain form)", "value": value, "unit": "GFLOP/s", "n_gpus": world,
                "steps": a.steps, "warmup": a.warmup, "ms_per_step": total_ms / a.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": config_of(a, fixture, info["flops"]),
                "plan": {"vec_len": n, "coefficient_block_doubles": info["w_len"], "s_len": info["s_len"],
                         "t_len": info["t_len"], "p_len": info["p_len"], "l_len": info["l_len"], "r_len": info["r_len"],
                         "parallelism": f"replicas x{world}"},
                "e2e": {"value": e2e_val, "unit": "GFLOP/s", "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n},
                "gpu_launches": int(info["launches"]) * a.steps, "roofline": roof, "cpu_baseline": cpu, "clocks": ck,
                "fp64_peaks_tflops": {"dmma": dmma_peak, "dfma": dfma_peak},
                "max_rel_err_vs_oracle": rel, "twin_max_rel_diff_vs_oracle": twin_rel}
        line.update(extras)
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


def main():
    a = parse()
    world, rank, local, pg = dist_setup(a)
    if a.impl == "reference":
        run_reference(a, world, rank)
        return
    run_b200(a, world, rank, local, pg)


if __name__ == "__main__":
    main()
