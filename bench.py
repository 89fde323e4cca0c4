"""Benchmark: seconds per 256^3 KH 3D-RISM solve on one B200 (and N replicas).

Workload: the protein-scale synthetic solute (846 atoms, compact random
chain, Rg ~15 A, sigma 3.0-3.8 A, charges N(0, 0.3) shifted to net zero;
seed 2) on a 256^3 grid in a 128 A cubic cell, KH closure, AN2 (2 0.6 0.2),
convergence 1e-6, in the workloads' TIP3P water (298.15 K, 0.03334 /A^3;
tip3p_cfg_vv.xvk from the library's own 1D XRISM-KH solve).  One
step = one complete solve: potential grids, the iteration to convergence,
and the .xmu observables (mu_ex SC/SC_HNC/GF, PMV, pressure, SE).

  value  device time per solve, mixed precision (FP32 bulk + FP64 polish),
         solute already on the device, CUDA events on the solve stream
  e2e    the same through the C ABI from host arrays: rism3d_set_solute
         (host -> device) + rism3d_solve (result struct -> host), wall clock
  fp64   the plain FP64 solve (same algorithm as the reference) for the
         mixed-vs-FP64 speed-up and the |d mu_ex| check (<= 0.01 kcal/mol)

--impl reference runs the reference executable (built from its own sources
for sm_100a into oracle/_ref) on the same control file, whole-process wall
time as in the reference README; without that binary it falls back to the
CPU FP64 oracle.  Multi-GPU: one independent solve per rank (replicas, no
collective on the solve path); the step time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "3d-rism-cuda_b200"))
GOLDEN = os.path.join(ROOT, "tests", "golden")
WORKLOADS = {"protein846": "cfg2_protein846_kh", "globule300": "cfg1_globule300"}
WORKLOAD = WORKLOADS["protein846"]
METRIC = ("s per 256^3 KH solve, mixed vs FP64 at <=0.01 kcal/mol d(mu_ex); "
          "batch solves/s")
KCAL = 4184.0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-cli", action="store_true",
                   help="skip the whole-process timing of the drop-in executable")
    p.add_argument("--cli-reps", type=int, default=3)
    p.add_argument("--cpu-iters", type=int, default=2,
                   help="iterations in the CPU-oracle sample")
    p.add_argument("--batch-mols", type=int, default=256,
                   help="molecules in the batched-solve leg (0: skip)")
    p.add_argument("--workload", default="protein846", choices=sorted(WORKLOADS),
                   help="protein846: 256^3 (the metric's workload); globule300: the "
                        "128^3 case, used for profiler captures that must stay small")
    return p.parse_args()


# ----------------------------------------------------------------- clocks
class Clocks:
    """nvidia-smi sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu, self.rows, self.proc = gpu, [], None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        self.proc = subprocess.Popen(
            ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
             "--format=csv,noheader,nounits", "-lms", "200"],
            stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) > 8
                          for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


# -------------------------------------------------------------- workload
def workload():
    from oracle import formats as F
    ctrl, sol = F.read_control(os.path.join(GOLDEN, WORKLOAD + ".inp"))
    sv = F.read_xvk(os.path.join(GOLDEN, ctrl.fsolvent))
    return ctrl, sol, sv


def iter_bytes_per_point(V, s):
    """Algorithmic HBM bytes per grid point of each pass (V sites, element
    size s; complex site pairs; fk is FP64 complex on half the points)."""
    return {"pass_a": 9 * V * s, "pass_k": 2 * V * s + 8, "pass_r": 5 * V * s}


def fused_pipeline_bytes_per_iter(n, V, s, s_lr=None):
    """N (31 V s + 5 s_lr + 4): minimal fused pipeline of the per-site design;
    the long-range Coulomb grids (e, fr, fk) stay FP64 (s_lr = 8) in the
    mixed form."""
    s_lr = s if s_lr is None else s_lr
    return n * (31 * V * s + 5 * s_lr + 4)


def read_traffic(kernel):
    """Per-point DRAM traffic of `kernel` from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        f = line.split()
        if len(f) >= 2 and f[0] == kernel:
            try:
                return float(f[1])
            except ValueError:
                return None
    return None


# ------------------------------------------------------------- our arm
def run_ours(args, rank, world, dist):
    import numpy as np
    import torch
    import rism3d_b200 as R

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream()          # all solver work and the events
    ctrl, sol, sv = workload()
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)

    def make(prec):
        s = R.Solver(ctrl.grid, ctrl.box, closure=ctrl.closure, convergence=ctrl.conv,
                     maxstep=ctrl.maxstep, an2=(ctrl.count, ctrl.m, ctrl.mp),
                     precision=prec, device=dev, stream=stream.cuda_stream)
        s.set_solvent_obj(sv)
        s.set_solute(sol.sig, sol.eps, sol.q, sol.xyz)
        return s

    def barrier():
        if dist:
            import torch.distributed as D
            D.barrier()

    from rism3d_b200 import replicas as RP

    def max_over_ranks(x):
        return RP.max_over_ranks(x, "cuda") if dist else x

    mixed = make(R.MIXED)
    fp64 = make(R.FP64)
    # warm-up (plans, graphs, caches)
    for _ in range(args.warmup):
        mixed.refresh_potentials(); rm = mixed.solve()
    fp64.refresh_potentials(); r64 = fp64.solve()

    # ---- timed: device-resident solves, mixed precision
    clk = Clocks(dev)
    barrier(); torch.cuda.synchronize()
    l0 = mixed.kernel_launches()
    clk.start()
    e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("mixed_solve")     # profiler filter (ncu --nvtx-include)
    e0.record(stream)
    res = []
    for _ in range(args.steps):
        mixed.refresh_potentials()
        res.append(mixed.solve())
    e1.record(stream)
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    clocks = clk.stop()
    barrier()
    launches = mixed.kernel_launches() - l0
    ms_mixed = max_over_ranks(e0.elapsed_time(e1)) / args.steps
    rm = res[-1]

    # ---- FP64 plain solve (the reference algorithm), same protocol
    barrier(); torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("fp64_solve")
    e0.record(stream)
    res64 = []
    for _ in range(args.steps):
        fp64.refresh_potentials(); r64 = fp64.solve()
        res64.append(r64)
    e1.record(stream)
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    ms_fp64 = max_over_ranks(e0.elapsed_time(e1)) / args.steps

    # ---- opt-in depth-5 Anderson for the FP32 bulk (RISM3D_MDIIS=5), same
    # protocol, reported beside the AN2 form (not the headline)
    os.environ["RISM3D_MDIIS"] = "5"
    try:
        dm = make(R.MIXED)
    finally:
        del os.environ["RISM3D_MDIIS"]
    dm.refresh_potentials(); rdm = dm.solve()
    barrier(); torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        dm.refresh_potentials(); rdm = dm.solve()
    e1.record(stream)
    torch.cuda.synchronize()
    ms_dm = max_over_ranks(e0.elapsed_time(e1)) / args.steps
    dm.close()

    # ---- e2e through the C ABI from host buffers
    import ctypes
    h2d = 8 * 6 * len(sol.q)               # sig, eps, q, x, y, z per atom
    d2h = ctypes.sizeof(R.Result)          # the result struct
    barrier(); torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        mixed.set_solute(sol.sig, sol.eps, sol.q, sol.xyz)
        re2e = mixed.solve()
    torch.cuda.synchronize()
    s_e2e = max_over_ranks(time.perf_counter() - t0) / args.steps

    # ---- live roofline of the dominant streaming kernels (CUDA events on
    # the solve stream; run after the results were read)
    n = ctrl.grid[0] * ctrl.grid[1] * ctrl.grid[2]
    V = sv.natv
    bpp32 = iter_bytes_per_point(V, 4)
    bpp64 = iter_bytes_per_point(V, 8)
    kern = {}
    for name, kid, bpp in (("pass_a_fp32", 10, bpp32["pass_a"]), ("pass_k_fp32", 11, bpp32["pass_k"]),
                           ("pass_r_fp32", 12, bpp32["pass_r"])):
        ms = mixed.time_kernel(kid, 20)
        kern[name] = {"ms": ms, "gbs": bpp * n / ms / 1e6}
    # the FP32 iteration folds the x and y axes of its transforms into passes
    # A, K and R when the cell allows (256^3 here); cuFFT then transforms
    # along z only (kernel id 14, one strided C2C pass: 16 B/point read +
    # write of the packed site pair)
    fused = True
    try:
        ms = mixed.time_kernel(14, 20)
        kern["fft_z_fp32"] = {"ms": ms, "gbs": 2 * 8 * ((V + 1) // 2) * n / ms / 1e6}
    except R.RismError:
        fused = False
    for name, kid, bpp in (("pass_a_fp64", 0, bpp64["pass_a"]), ("pass_k_fp64", 1, bpp64["pass_k"]),
                           ("pass_r_fp64", 2, bpp64["pass_r"])):
        ms = fp64.time_kernel(kid, 20)
        kern[name] = {"ms": ms, "gbs": bpp * n / ms / 1e6}
    # the real-space potential grids (LJ per site, esr, fr): pair evaluations/s
    pairs = n * len(sol.q)
    for name, solver in (("potential_r_mixed", mixed), ("potential_r_fp64", fp64)):
        ms = solver.time_kernel(20, 3)
        kern[name] = {"ms": ms, "gpairs_per_s": pairs / ms / 1e6}
    # adjoint gradients of mu_ex (all charges, LJ parameters, positions) on
    # the converged mixed solve: the exact discrete adjoint
    torch.cuda.synchronize()
    mixed.set_solute(sol.sig, sol.eps, sol.q, sol.xyz)
    mixed.solve()
    mixed.grad()                                  # warm-up: allocates the adjoint's scratch
    t1 = time.perf_counter()
    mixed.grad()
    adjoint_s = time.perf_counter() - t1
    mixed.grad(precision=R.MIXED)                 # the FP32 adjoint variant (own scratch)
    t1 = time.perf_counter()
    mixed.grad(precision=R.MIXED)
    adjoint32_s = time.perf_counter() - t1
    mixed.close(); fp64.close()
    batch = run_batch(args, dev, stream, rank, world, dist) if args.batch_mols > 0 else None
    cli = None
    if rank == 0 and not args.no_cli:
        c64, i64, f64 = time_cli(args, 0, args.cli_reps)
        c32, i32, f32 = time_cli(args, 1, args.cli_reps)
        cli = {"cli_fp64_s": c64, "cli_mixed_s": c32, "iterations_fp64": i64,
               "iterations_mixed": i32, "sfe_sc_fp64": f64, "sfe_sc_mixed": f32,
               "reps": args.cli_reps,
               "what": "bin/rism3d-b200 on the same control file, whole-process wall time "
                       "(context, file reads, solve, .xmu), as the reference executable is timed"}
    dom = "pass_a_fp32"
    achieved = kern[dom]["gbs"]
    dom_kernel = ("k_pass_ax<float> (FP32 pass A with the x-axis DFTs: inverse x-DFT of the "
                  "last OZ result, AN2 update, closure, forward x-DFT)" if fused else
                  "k_pass_a<float> (FP32 pass A: AN2 update + closure + forward pack)")
    traffic_pp = read_traffic("k_pass_ax_fp32" if fused else "k_pass_a_fp32")
    dmu = abs(rm["sfe_sc"] - r64["sfe_sc"])
    out = {
        "metric": METRIC, "value": ms_mixed / 1e3 / world, "unit": "s/solve",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_mixed, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": ("protein-like solute, 846 atoms, 256^3 grid, 128 A cell, KH, "
                                "AN2 2/0.6/0.2, conv 1e-6, TIP3P water 298.15 K 0.03334/A^3 (tip3p_cfg_vv.xvk, "
                                "1D XRISM-KH)")
                   if WORKLOAD == WORKLOADS["protein846"] else
                   ("globular solute, 300 atoms, 128^3 grid, 64 A cell, KH, AN2 2/0.6/0.2, "
                    "conv 1e-6, TIP3P water (tip3p_cfg_vv.xvk, 1D XRISM-KH)"),
                   "grid": list(ctrl.grid), "box": list(ctrl.box), "natom": len(sol.q),
                   "natv": V, "precision": "FP32 bulk + FP64 polish",
                   "l2": "state ~5 GB per solve >> 126 MB L2 (no flush needed)",
                   "parallelism": "replicas" if world > 1 else "1 GPU"},
        "fp64": {"s_per_solve": ms_fp64 / 1e3 / world, "iterations": r64["iterations"],
                 "sfe_sc": r64["sfe_sc"],
                 "per_solve_ms": [[round(r[k], 2) for k in ("ms_setup", "ms_iterate", "ms_observe")]
                                  for r in res64]},
        "mixed": {"iterations": rm["iterations"], "iterations_fp32": rm["iterations_fp32"],
                  "sfe_sc": rm["sfe_sc"], "ms_setup": rm["ms_setup"],
                  "ms_iterate": rm["ms_iterate"], "ms_observe": rm["ms_observe"],
                  "per_solve_ms": [[round(r[k], 2) for k in ("ms_setup", "ms_iterate", "ms_observe")]
                                   for r in res]},
        "mixed_mdiis5": {"s_per_solve": ms_dm / 1e3 / world, "iterations": rdm["iterations"],
                         "iterations_fp32": rdm["iterations_fp32"],
                         "ms_iterate": rdm["ms_iterate"], "sfe_sc": rdm["sfe_sc"],
                         "what": "the mixed solve with the opt-in depth-5 Anderson FP32 bulk "
                                 "(RISM3D_MDIIS=5) in place of AN2; refinement and FP64 "
                                 "cycles unchanged"},
        "speedup_mixed_vs_fp64": ms_fp64 / ms_mixed,
        "dmu_mixed_vs_fp64_j_per_mol": dmu, "dmu_within_0.01kcal": dmu <= 0.01 * KCAL,
        "e2e": {"value": s_e2e / world, "unit": "s/solve", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "kernel": dom_kernel, "achieved": achieved, "peak": hbm_peak,
                     "unit": "GB/s", "frac": achieved / hbm_peak,
                     "traffic": None if traffic_pp is None else traffic_pp * n,
                     "algorithmic_bytes_per_launch": bpp32["pass_a"] * n,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback 6650"},
        "batch": batch,
        "cli": cli,
        "adjoint": {"s_per_gradient": adjoint_s, "s_per_gradient_fp32": adjoint32_s,
                    "timing": "second call (the first allocates scratch)",
                    "outputs": "d mu/d(q, sigma, eps, xyz) of all "
                    "%d atoms" % len(sol.q)},
        "kernels": kern,
        "bytes_per_iteration": {"fp64": sum(bpp64.values()) * n, "fp32": sum(bpp32.values()) * n,
                                "fused_pipeline_fp64": fused_pipeline_bytes_per_iter(n, V, 8),
                                "fused_pipeline_fp32": fused_pipeline_bytes_per_iter(n, V, 4, 8)},
        # whole-iteration rate under the per-site byte model N (31 V s + 5 s + 4)
        # (FP32 bulk: 31 V x 4 B, the long-range terms at 8 B): bytes x steps /
        # iteration time; above the copy peak means the fused passes move fewer
        # bytes than that model assumes
        "iteration_rate": {
            "fp64": {"ms_iterate": r64["ms_iterate"], "steps": r64["iterations"],
                     "model_gbs": fused_pipeline_bytes_per_iter(n, V, 8) * r64["iterations"]
                     / (r64["ms_iterate"] * 1e6)},
            "mixed": {"ms_iterate": rm["ms_iterate"], "steps": rm["iterations"],
                      "model_gbs": n * (31 * V * 4 + 5 * 8 + 4) * rm["iterations"]
                      / (rm["ms_iterate"] * 1e6)}},
        "clocks": clocks,
    }
    return out


# ------------------------------------------------------------ batch leg
def run_batch(args, dev, stream, rank=0, world=1, dist=False):
    """Batched small solutes (BASELINE config 3 shapes): 256 molecules of
    8-40 atoms on 48^3 / 64^3 / 96^3 grids at 0.5 A, FP32 bulk + FP64 polish,
    in the reference's 3-site water + 0.1 M NaCl table (4 site types; the
    5-site water of the config needs the project's 1D XRISM tables).  Reports
    solves/s of one rism3d_solve_batch call and of a per-solute loop that
    reuses one context per grid size (timed on every molecule).
    Under N ranks the molecules are split by estimated cost (grid points);
    solves/s is all ranks' molecules over the slowest rank's time."""
    import torch
    import rism3d_b200 as R
    from oracle import formats as F
    from rism3d_b200 import synth
    sv = F.read_xvk(os.path.join(GOLDEN, "naclaq_sub4_vv.xvk"))
    from rism3d_b200 import replicas as RP
    mols = []
    for m in synth.small_batch(seed=3, nmol=args.batch_mols):
        F.centre(m.xyz)
        mols.append((m.sig, m.eps, m.q, m.xyz, m.grid[0], m.box[0]))
    n_total = len(mols)
    mine = list(range(n_total))
    if dist:
        part = RP.partition_by_cost([RP.solve_cost(m[4] ** 3, len(m[2])) for m in mols], world)
        mine = part[rank]
        mols = [mols[i] for i in mine]
    parent = R.Solver((48, 48, 48), (24.0, 24.0, 24.0), precision=R.MIXED, device=dev,
                      stream=stream.cuda_stream)
    parent.set_solvent_obj(sv)
    parent.solve_batch(mols)                      # warm-up: children, plans, graphs
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    res = parent.solve_batch(mols)
    e1.record(stream)
    torch.cuda.synchronize()
    s_batch = e0.elapsed_time(e1) / 1e3
    parent.close()
    # per-solute loop over the same molecules, one context per grid size (warm)
    ctxs = {}
    for g in sorted({m[4] for m in mols}):
        L = [m[5] for m in mols if m[4] == g][0]
        c = R.Solver((g, g, g), (L, L, L), precision=R.MIXED, device=dev, stream=stream.cuda_stream)
        c.set_solvent_obj(sv)
        ctxs[g] = c
    sample = mols                                 # every molecule of the batch
    for m in sample[:3]:
        ctxs[m[4]].set_solute(*m[:4]); ctxs[m[4]].solve()
    torch.cuda.synchronize()
    e0.record(stream)
    for m in sample:
        c = ctxs[m[4]]
        c.set_solute(*m[:4])
        c.solve()
    e1.record(stream)
    torch.cuda.synchronize()
    s_loop = e0.elapsed_time(e1) / 1e3
    for c in ctxs.values():
        c.close()
    dev_name = "cuda" if dist else None
    # every rank's per-solute results, gathered into input order
    allres = RP.gather_results(res, mine, n_total, dev_name)
    ok = sum(1 for r in allres if r["status"] == 0)
    rate = RP.job_rate(len(mols), s_batch, dev_name)
    loop_rate = RP.job_rate(len(sample), s_loop, dev_name)
    s_batch = RP.max_over_ranks(s_batch, dev_name)
    return {"solves_per_s": rate, "n_mols": n_total, "converged": ok,
            "s_batch": s_batch, "loop_solves_per_s": loop_rate,
            "loop_sample": len(sample),
            "speedup_vs_loop": rate / loop_rate,
            "solvent": "naclaq_vv.xvk (3-site water + 0.1 M NaCl), every 4th k row",
            "precision": "FP32 bulk + FP64 polish"}


# ------------------------------------------------- whole-process drop-in
def time_cli(args, prec, reps):
    """Wall time of the drop-in executable (bin/rism3d-b200) as a whole
    process on the workload's control file: CUDA context, file reads, the
    solve and the .xmu output, the way the reference executable is timed
    (its README times whole runs).  prec 0: plain FP64; 1: -p 1 (FP32 bulk
    + FP64 polish).  Returns (mean seconds, iterations, SFE_SC)."""
    exe = os.path.join(ROOT, "3d-rism-cuda_b200", "bin", "rism3d-b200")
    work = tempfile.mkdtemp(prefix="rism_cli_")
    ctrl, _, _ = workload()
    shutil.copyfile(os.path.join(GOLDEN, WORKLOAD + ".inp"), os.path.join(work, WORKLOAD + ".inp"))
    shutil.copyfile(os.path.join(GOLDEN, ctrl.fsolvent), os.path.join(work, ctrl.fsolvent))
    dev = os.environ.get("LOCAL_RANK", "0")
    times, iters, sfe = [], None, None
    for i in range(1 + reps):                     # one untimed warm-up run
        t0 = time.perf_counter()
        p = subprocess.run([exe, "-d", dev, "-p", str(prec), WORKLOAD + ".inp"], cwd=work,
                           capture_output=True, text=True, timeout=600)
        dt = time.perf_counter() - t0
        if p.returncode != 0:
            raise RuntimeError("rism3d-b200 failed: " + p.stderr[-500:])
        if i > 0:
            times.append(dt)
        iters = len(re.findall(r"Step = \d+", p.stdout))
        out = open(os.path.join(work, WORKLOAD + ".xmu")).read()
        sfe = float(re.search(r"SFE_SC=\s*(\S+)", out).group(1))
    shutil.rmtree(work, ignore_errors=True)
    return sum(times) / len(times), iters, sfe


# ------------------------------------------------------------ CPU oracle
def cpu_baseline(args):
    """The CPU FP64 OpenMP oracle on a bounded sample of the same solve:
    full potential setup, `cpu_iters` iterations and the observables, then
    seconds per solve = setup + iterations_of_the_FP64_solve * per-iteration
    + observables."""
    from oracle import oracle as O
    ctrl, sol, sv = workload()
    case = O.Case(ctrl.grid, ctrl.box, sv, sol.sig, sol.eps, sol.q, sol.xyz,
                  ctrl.closure, ctrl.conv, args.cpu_iters, ctrl.count, ctrl.m, ctrl.mp)
    r = O.solve(case)
    ref_iters = json.load(open(os.path.join(GOLDEN, "ref_b200", "summary.json")))[WORKLOAD]["iterations"]
    per_it = r["t_iter"] / max(1, r["iterations"])
    value = r["t_setup"] + per_it * ref_iters + r["t_obs"]
    return {"value": value, "unit": "s/solve", "cores": O.lib().oracle_num_threads(),
            "kind": "port",
            "sample": "oracle: potentials + %d iterations + observables, extrapolated to the "
                      "%d iterations of the FP64 solve (%.2f s/iteration)"
                      % (r["iterations"], ref_iters, per_it)}


# -------------------------------------------------------- reference arm
def run_reference(args):
    binp = os.path.join(ROOT, "oracle", "_ref", "3drism-cuda")
    if not os.path.exists(binp):
        cb = cpu_baseline(args)
        return {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "s/solve",
                "n_gpus": 1, "steps": 1, "warmup": 0, "higher_is_better": False,
                "note": "reference executable not built; CPU FP64 oracle port instead",
                "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": "s/solve", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
    work = tempfile.mkdtemp(prefix="rism_ref_")
    shutil.copyfile(os.path.join(GOLDEN, WORKLOAD + ".inp"), os.path.join(work, WORKLOAD + ".inp"))
    ctrl, _, _ = workload()
    shutil.copyfile(os.path.join(GOLDEN, ctrl.fsolvent), os.path.join(work, ctrl.fsolvent))
    times, iters, out = [], None, ""
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        p = subprocess.run([binp, WORKLOAD + ".inp"], cwd=work, capture_output=True, text=True,
                           timeout=600)
        dt = time.perf_counter() - t0
        if p.returncode != 0:
            raise RuntimeError("reference run failed: " + p.stderr[-500:])
        iters = len(re.findall(r"Step = \d+", p.stdout))
        out = open(os.path.join(work, WORKLOAD + ".xmu")).read()
        if i >= args.warmup:
            times.append(dt)
    sfe = float(re.search(r"SFE_SC=\s*(\S+)", out).group(1))
    v = sum(times) / len(times)
    shutil.rmtree(work, ignore_errors=True)
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": "s/solve", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "same control file, reference 3drism-cuda (FP64, AN2) built "
                                   "from its own sources for sm_100a, whole-process wall time",
                       "iterations": iters, "sfe_sc": sfe},
            "reference_kind": "the reference's own CUDA executable on the same B200 (it has no "
                              "CPU implementation of the path)",
            "cpu_baseline": cpu_baseline(args),
            "e2e": {"value": v, "unit": "s/solve", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def main():
    global WORKLOAD
    args = parse()
    WORKLOAD = WORKLOADS[args.workload]
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = world > 1
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)))
        return 0
    if dist:
        import datetime
        import torch
        import torch.distributed as D
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        D.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    out = run_ours(args, rank, world, dist)
    if rank == 0:
        if not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(args)
        print(json.dumps(out))
    if dist:
        import torch.distributed as D
        D.barrier()
        D.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
