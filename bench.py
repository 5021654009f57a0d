#!/usr/bin/env python
"""Benchmark of the two-site DMRG effective-Hamiltonian hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--L 24] [--M 512] [--init-bd 64] [--sweeps 2] [--seed 0]

Workload: the seeded synthetic ab-initio Hamiltonian of the precision-form
configuration (L = 24 orbitals, N = 24 electrons, TwoU1 Sz = 0, M = 512; FP64
plain form).  Setup (untimed): the device engine runs `--sweeps` full two-site
sweeps from the const initial state (each timed on its own and reported under
"sweep"), then continues the next sweep up to the middle bond (step L/2 - 1)
and freezes that site problem.

A step is one H_eff . psi (the Davidson callback, super_hamil_mv) on that
frozen problem.  `value` = reference work count (ScheduleNew::total_flops,
solver/tasks.cpp:388-398, 777-796) x steps / device time (CUDA events on the
plan stream, L2 flushed between steps), summed over ranks / max over ranks.
`e2e` is the same metric through qcm_heff_apply with pinned host buffers (H2D
of psi and D2H of H.psi inside the timed region).  The path does not shard
across GPUs here (one B200 per solve): N > 1 runs N independent replicas.

"mixed" reports the mixed-precision form of the same step (S build as 3xTF32 on
the tensor cores, T-GEMM and L.S in FP64) with the same timing rules, its
deviation from the oracle, and (unless --no-mixed-sweep) the same sweeps run
with every Jacobi-Davidson solve in the mixed form (FP64 Rayleigh quotient per
step): sweep times and the energy deviation from the FP64 sweeps.

The reference arm (--impl reference) times the CPU restatement of the same
H.psi (the oracle: OpenMP over ket sectors, OpenBLAS dgemm) on the same frozen
problem, exported by the device engine as a "QSPB" blob.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
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
    ap.add_argument("--init-bd", type=int, default=64)
    ap.add_argument("--sweeps", type=int, default=2)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed-sweep", action="store_true", help="skip the mixed-precision sweeps (bench of the apply only)")
    ap.add_argument("--no-single-site-sweep", action="store_true", help="skip the single-site sweep after the two-site ones")
    return ap.parse_args()


def workload_name(a):
    return (f"two-site H_eff.psi, synthetic ab-initio L={a.L} N={a.L} TwoU1 Sz=0 seed {a.seed}, M={a.M} "
            f"(init_bond_dimension {a.init_bd}), middle bond after {a.sweeps} sweeps")


def frozen_problem(a, device: int, export: bool):
    """Device sweeps, then the middle-bond site problem: (ctx, dmrg, plan, x, mpo_blob, snap, site, sweep_info)."""
    from qcmaquis_b200.fcidump import synthetic_integrals
    from qcmaquis_b200.mpo import MPO
    from qcmaquis_b200.heff import Context
    from qcmaquis_b200.dmrg import DMRG
    h, V, e = synthetic_integrals(a.L, a.seed)
    m = MPO.qc(h, V)
    ctx = Context(device)
    t0 = time.perf_counter()
    d = DMRG(ctx, m, a.L // 2, a.L // 2, a.M, a.init_bd)
    t_init = time.perf_counter() - t0
    sweeps = []
    for s in range(a.sweeps):
        st0 = d.stats()
        t0 = time.perf_counter()
        E, tr = d.sweep()
        dt = time.perf_counter() - t0
        st1 = d.stats()
        sweeps.append({"sweep": s, "seconds": dt, "energy_min": float(E.min()),
                       "max_bond_dimension": int(max(t["bond_dimension"] for t in tr)),
                       "hpsi": int(st1["hpsi_count"] - st0["hpsi_count"]),
                       "hpsi_gflop": (st1["hpsi_flops"] - st0["hpsi_flops"]) / 1e9,
                       "phase_s": {k: st1[k] - st0[k] for k in ("plan_s", "jd_s", "trunc_s", "boundary_s")}})
    if not a.no_single_site_sweep:
        sweeps_ss = single_site_sweep(a, ctx, m, d, sweeps[-1]["energy_min"])
    site = a.L // 2 - 1
    d.run(site)
    plan, x = d.pending_plan()
    snap = d.pending_export() if export else None
    info = {"init_s": t_init, "sweeps": sweeps, "site": site}
    if not a.no_single_site_sweep:
        info["single_site"] = sweeps_ss
    return ctx, d, plan, x, m.blob(), snap, site, info


def single_site_sweep(a, ctx, m, d, e_ts):
    """One single-site sweep (optimization = singlesite: 2L steps, density-matrix growth with noise 1e-8)
    from the two-site sweeps' MPS at the same Mmax: its time, phases and H.psi work, and its lowest energy
    against the last two-site sweep's.  Reported beside the metric; a failure is recorded, not raised."""
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
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl" if a.impl == "b200" else "gloo", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def cpu_baseline(snap, blob, site, x, flops, budget_s=20.0):
    from oracle.oracle import heff_apply, lib as olib
    olib()
    y, _, sec = heff_apply(snap, blob, site, x, repeat=1)
    reps = max(1, min(50, int(budget_s / max(sec, 1e-3))))
    _, _, sec = heff_apply(snap, blob, site, x, repeat=reps)
    return {"value": flops / sec / 1e9, "unit": "GFLOP/s", "cores": olib().orc_max_threads(), "kind": "port",
            "sample": f"{reps} H_eff.psi applies of the same frozen problem (oracle, OpenMP over ket sectors, "
                      f"OpenBLAS dgemm), {sec * 1e3:.1f} ms each"}


def run_reference(a, world, rank, pg):
    if rank != 0:
        return
    from oracle.oracle import heff_apply, lib as olib
    ctx, d, plan, x, blob, snap, site, sinfo = frozen_problem(a, 0, export=True)
    flops = plan.info["flops"]
    del plan, d
    for _ in range(a.warmup):
        heff_apply(snap, blob, site, x, repeat=1)
    t0 = time.perf_counter()
    _, flops_o, sec = heff_apply(snap, blob, site, x, repeat=a.steps)
    wall = time.perf_counter() - t0
    val = flops_o / sec / 1e9
    cores = olib().orc_max_threads()
    line = {"impl": "reference", "metric": "H_eff.psi GFLOP/s (FP64 plain form)", "value": val, "unit": "GFLOP/s",
            "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup, "ms_per_step": sec * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload_name(a), "L": a.L, "M": a.M, "init_bond_dimension": a.init_bd,
                       "seed": a.seed, "flops_per_step": flops_o},
            "cpu_baseline": {"value": val, "unit": "GFLOP/s", "cores": cores, "kind": "port",
                             "sample": f"{a.steps} H_eff.psi applies ({wall:.1f} s) with all host threads"},
            "e2e": {"value": val, "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "frozen problem produced by the device engine (untimed) and exported as a QSPB blob"}
    assert abs(flops_o - flops) <= 1e-9 * flops, "oracle and device work counts differ"
    print(json.dumps(line), flush=True)


def measure_mixed(a, plan, xd, yd, xp, yp, xh, yh, flush, info, world, pg, dev, snap, blob, site, x_host, form="mixed"):
    """A mixed-precision form on the same frozen problem: S build 3xTF32 on the tensor cores
    (FP32 accumulation), T-GEMM and L.S in FP64; same timing rules as the FP64 form."""
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
    e2e_s = float(sum(e2e_t))
    if pg is not None:
        t = torch.tensor([total_ms, e2e_s], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        total_ms, e2e_s = float(t[0].item()), float(t[1].item())
    ph = np.mean(np.array(phases), axis=0)
    y_mixed = yh.numpy().copy()
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


def measure_adjoint(a, plan, x_host, blob, site):
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
    from qcmaquis_b200.mpo import MPO
    terms = MPO.from_blob(blob).twosite().terms(site)["scale"]  # same builder: the plan's entry order
    f = float(ybar @ plan.apply(x_host))
    return {"ms_per_call": dt * 1e3, "n_terms": int(g.size), "h2d_bytes": 16 * x_host.size,
            "d2h_bytes": 8 * (x_host.size + g.size),
            "euler_check_rel": abs(float(g @ terms) - f) / abs(f),
            "note": "psi_bar = H ybar and d(ybar.Hx)/d scale per entry; sum_e scale_e * grad_e = ybar.Hx (f is linear "
                    "in the scales) is the consistency check"}


def mixed_sweeps(a, ctx, blob, sinfo):
    """The same sweeps with every JD in the mixed form (FP64 Rayleigh quotient per step): times and
    the per-sweep energy deviation from the FP64 device sweeps."""
    from qcmaquis_b200.mpo import MPO
    from qcmaquis_b200.dmrg import DMRG
    m = MPO.from_blob(blob)
    d = DMRG(ctx, m, a.L // 2, a.L // 2, a.M, a.init_bd, precision="mixed")
    out = []
    for s in range(a.sweeps):
        st0 = d.stats()
        t0 = time.perf_counter()
        E, tr = d.sweep()
        dt = time.perf_counter() - t0
        st1 = d.stats()
        e64 = sinfo["sweeps"][s]["energy_min"]
        out.append({"sweep": s, "seconds": dt, "energy_min": float(E.min()), "energy_dev_vs_fp64": float(E.min() - e64),
                    "max_bond_dimension": int(max(t["bond_dimension"] for t in tr)),
                    "hpsi_mixed": int(st1["hpsi_count"] - st0["hpsi_count"]),
                    "hpsi_fp64": int(st1["hpsi_count_fp64"] - st0["hpsi_count_fp64"]),
                    "phase_s": {k: st1[k] - st0[k] for k in ("plan_s", "jd_s", "trunc_s", "boundary_s")}})
    del d
    return out


def run_b200(a, world, rank, local, pg):
    import torch
    from qcmaquis_b200 import heff
    torch.cuda.set_device(local)
    want_cpu = rank == 0 and world == 1 and not a.no_cpu_baseline
    ctx, d, plan, x_host, blob, snap, site, sinfo = frozen_problem(a, local, export=want_cpu)
    info = plan.info
    n = plan.n
    dev = torch.device("cuda", local)
    xd = torch.from_numpy(x_host).to(dev)
    yd = torch.empty_like(xd)
    flush = torch.empty(int(256 * 2**20 // 4), dtype=torch.float32, device=dev)  # 256 MiB > L2 (126 MB)
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    dmma_peak, dfma_peak = heff.probe_fp64_peaks()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()  # sampled from the warm-up on, stopped after the timed region
    # warm-up (plan stream; the context stream is separate from torch's)
    for _ in range(a.warmup):
        plan.apply_device(xd.data_ptr(), yd.data_ptr())
    ctx.synchronize()
    prof = [plan.profile(xd.data_ptr(), yd.data_ptr()) for _ in range(3)]
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
    total_ms = float(sum(times))
    if pg is not None:
        t = torch.tensor([total_ms], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        total_ms = float(t.item())
        pg.barrier()
    value = info["flops"] * a.steps * world / (total_ms * 1e-3) / 1e9
    # e2e through the C-ABI with pinned host buffers
    xh = torch.from_numpy(x_host).pin_memory()
    yh = torch.empty_like(xh).pin_memory()
    import ctypes
    from qcmaquis_b200._lib import lib, check, P, c_double
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
    e2e_s = float(sum(e2e_t))
    if pg is not None:
        t = torch.tensor([e2e_s], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_val = info["flops"] * a.steps * world / e2e_s / 1e9
    # correctness guard on the timed problem: device result vs the oracle
    rel = None
    if snap is not None:
        from oracle.oracle import heff_apply
        y_ref, _, _ = heff_apply(snap, blob, site, x_host)
        rel = float(np.abs(yh.numpy() - y_ref).max() / np.abs(y_ref).max())
    # roofline of the dominant kernel (phase): reference flop count of the phase / its device time
    ph = np.mean(np.array(phases), axis=0)
    names = ["k_tgemm", "k_sgemm", "k_lspart+k_lsreduce"]
    work = [info["flops_t"], info["flops_s"], info["flops_ls"]]
    dom = int(np.argmax(ph))
    ach = work[dom] / (ph[dom] * 1e-3) / 1e12
    roof = {"kernel": names[dom], "bound": "tensor", "achieved": ach, "peak": dmma_peak, "unit": "TFLOP/s",
            "frac": ach / dmma_peak, "traffic": None,
            "algorithmic": "reference flop count of the phase (ScheduleNew::total_flops terms)",
            "peak_source": "FP64 DMMA probe qcm_probe_fp64_peaks (of measured)"}
    if dom == 1:
        # tensor work the S-GEMM tiles really issue (padding included) over the same time
        roof["executed_tflops"] = info["flops_sexec"] / (ph[1] * 1e-3) / 1e12
        roof["executed_frac"] = roof["executed_tflops"] / dmma_peak
    roof["phase_ms"] = {k: float(v) for k, v in zip(names, ph)}
    mixed = measure_mixed(a, plan, xd, yd, xp, yp, xh, yh, flush, info, world, pg, dev, snap, blob, site, x_host)
    mixed["tensor_memory_form"] = measure_mixed(a, plan, xd, yd, xp, yp, xh, yh, flush, info, world, pg, dev, snap, blob,
                                                site, x_host, form="mixed_tc")
    adjoint = measure_adjoint(a, plan, x_host, blob, site)
    if not a.no_mixed_sweep:
        mixed["sweep"] = mixed_sweeps(a, ctx, blob, sinfo)
    cpu = None
    if want_cpu:
        cpu = cpu_baseline(snap, blob, site, x_host, info["flops"])
    if rank == 0:
        line = {"metric": "H_eff.psi GFLOP/s (FP64 plain form)", "value": value, "unit": "GFLOP/s", "n_gpus": world,
                "steps": a.steps, "warmup": a.warmup, "ms_per_step": total_ms / a.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": workload_name(a), "L": a.L, "M": a.M, "init_bond_dimension": a.init_bd,
                           "seed": a.seed, "vec_len": n, "flops_per_step": info["flops"],
                           "coefficient_block_doubles": info["w_len"], "s_len": info["s_len"], "t_len": info["t_len"],
                           "l2": "flushed between steps (256 MiB write)", "parallelism": f"replicas x{world}"},
                "sweep": sinfo,
                "e2e": {"value": e2e_val, "unit": "GFLOP/s", "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n},
                "gpu_launches": int(info["launches"]) * a.steps, "roofline": roof, "cpu_baseline": cpu, "clocks": ck,
                "fp64_peaks_tflops": {"dmma": dmma_peak, "dfma": dfma_peak},
                "max_rel_err_vs_oracle": rel, "mixed": mixed, "adjoint": adjoint}
        print(json.dumps(line), flush=True)
    del plan, d
    if pg is not None:
        pg.destroy_process_group()


def main():
    a = parse()
    world, rank, local, pg = dist_setup(a)
    if a.impl == "reference":
        run_reference(a, world, rank, pg)
        if pg is not None:
            pg.destroy_process_group()
        return
    run_b200(a, world, rank, local, pg)


if __name__ == "__main__":
    main()
