#!/usr/bin/env python
"""Benchmark: Poisson solve time to ||r||/||b|| <= 1e-8 on one B200.

Workload (default, --config 3): 512x256x256 cells (33.5M) as 4x2x2 blocks of
128^3, all-Neumann, seeded spectral right-hand side.  One step = one full
solve from p = 0 to the FP64 relative residual 1e-8 by the FP32-smoothing /
FP64-refined multigrid (`value`, ms per solve, lower is better).  The plain
FP64 GPU multigrid (the reference's arithmetic) is timed beside it on the
same resident inputs, and the solution error of the mixed solve against the
FP64 one is reported.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--config C]

With N > 1 (torchrun) every rank solves its own replica (the path does not
shard across GPUs in this build); the value is the whole job's ms per solve
(max-over-ranks device time / (N*K)).  `--impl reference` times the CPU
implementation of the same path (the oracle restatement of the reference
Fortran, OpenMP over all host cores): every timed step one complete
converged solve.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

TOL = 1e-8
# The mixed solver's cycle per workload: (pre-sweeps, post-sweeps, FP32
# V-cycles per FP64 refinement step) and its FP32 sweeps: (over-relaxation
# factor, rb_order: 1 = red-black order across block faces, 0 = the reference's
# per-block order); the fastest measured choice whose solution stays within the
# error of the V(2,1) x 4 Gauss-Seidel one.  Configuration 3: V(2,1) x 3 with
# omega 1.25 across blocks 5.1 ms, 6 cycles, error 9.2e-10, against V(2,1) x 4
# Gauss-Seidel per block 8.3 ms, 12 cycles, 1.4e-9 (omega 1.25 per block or
# across blocks alone: 12 cycles; omega 1.3: 9 cycles; V(1,1) x 3: 9 cycles,
# 6.0 ms); configuration 2: V(2,1) x 3, omega 1.25 across blocks 2.0 ms against
# V(2,1) x 5 2.8 ms; 5 (1000:1 density, one block: no order across blocks to
# take): V(2,1) x 4, omega 1.5 17.9 ms, 16 cycles, error 2.1e-8, against
# V(2,1) x 8 Gauss-Seidel 33.4 ms,
# 2.8e-7 (omega 1.35-1.6 also 16 cycles, 1.25 24 cycles, 1.7 20 cycles;
# V(2,2) x 3 with omega 1.6 16.8 ms but error 1.1e-7).  One block (1): omega 1.25 takes
# 6 cycles, not 8, but its error grows from 3.7e-8 to 9.5e-7; independent
# blocks (4) and refinement (6, whose expression-filled levels keep the
# per-block order): no fewer cycles.  6: V(2,2) x 6 12.3 ms against V(2,1) x 4
# 20.6 ms; 4: V(1,2) x 6 12.2 against V(2,1) x 2 13.2 ms.
MIXED_CYCLE = {1: (2, 1, 4), 2: (2, 1, 3), 3: (2, 1, 3), 4: (1, 2, 6), 5: (2, 1, 4), 6: (2, 2, 6)}
MIXED_SMOOTHER = {1: (1.0, 0), 2: (1.25, 1), 3: (1.25, 1), 4: (1.0, 0), 5: (1.5, 0), 6: (1.0, 0)}
# Sweeps of the FP64 coarsest level in the mixed solver: enough to converge
# that level (on the configuration-3 hierarchy 16 leave 14 V-cycles, 32 and 64
# both 12), so the V-cycle contracts every mode at the rate of its finer
# levels instead of the reference's 3 coarsest sweeps (54 V-cycles).
COARSE_SWEEPS = 32
# The mixed solver solves a small coarsest level (at most 512 cells) directly by
# its pseudo-inverse inside the coarse cluster instead of those sweeps.
COARSE_DIRECT = True
# Tolerance of the FP64 solve the mixed solution's error is measured against.
EXACT_TOL = 1e-12
# Cycle cap of the reference-algorithm FP64 solve on the variable-coefficient
# workload (it does not reach 1e-8 in any practical number of cycles).
FP64_CAP = 200
WORKLOADS = {
    1: "config1: 64^3 single block, walls, U(-1,1) divergence, 4 levels, V(2,1) RBGS",
    2: "config2: 192^3 as 2x2x2 blocks of 96^3, periodic x, 6 levels, warm start",
    3: "config3: 512x256x256 (33.5M cells) as 4x2x2 blocks of 128^3, all-Neumann, k^-5/3 spectral rhs, 7 levels",
    4: "config4: 27 independent all-Neumann blocks, axes from {32,48,64,96,128}, 4 levels",
    5: "config5: 256^3 two-phase 1000:1 density (L_LSM coefficients), 8 levels",
    6: "config6 (local mesh refinement): 4x2x2 blocks of 64^3 at h=1/128, the 8 blocks of x index 1-2 refined "
       "to 128^3 at h=1/256 (18.9M cells), walls, 7 levels, rhs = A p of a seeded smooth pressure",
}


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def max_over_ranks(x, world):
    """The largest x over all ranks (device-timed milliseconds: the slowest
    replica sets the job time); x itself on one rank."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as tdist
    t = torch.tensor([float(x)], dtype=torch.float64)
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    return float(t.item())


def job_ms_per_solve(total_ms_max, steps, world):
    """Whole-job time per solve of N replicas that each ran `steps` solves:
    the slowest replica's total over all solves of the job."""
    return total_ms_max / (steps * world)


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def wait_running(self, timeout=5.0):
        """Blocks until nvidia-smi has printed its first sample (the timed
        region then starts with the sampler already running)."""
        t0 = time.perf_counter()
        while self.proc and not self.lines and time.perf_counter() - t0 < timeout:
            time.sleep(0.01)
        self.mark = len(self.lines)

    def count(self):
        return len(self.lines) - getattr(self, "mark", 0)

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines[getattr(self, "mark", 0):]:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def oracle_resolve(ext, bc, h, ngrid):
    """Block neighbours found by the oracle's read_infodom restatement (the
    CPU arms build their blocks without the CUDA library)."""
    from oracle import oracle as O
    return O.topology(ext, bc, h, ngrid)


def make_problem(cfg, resolve=None, prev_solve=None, residual_of=None):
    """The workload of configuration `cfg`.  Configuration 2 starts from the
    converged pressure of its independent previous-seed problem:
    `prev_solve(problem)` solves that problem to 1e-8 (untimed set-up) and
    returns its block host fields.  Configuration 6's right-hand side is
    A p_exact by the arm's own operator: `residual_of(problem)` returns the
    function synth.manufacture calls."""
    from hydro3d_b200 import synth
    if cfg != 2:
        prob = synth.CONFIGS[cfg](resolve=resolve)
        if prob.b is None:
            synth.manufacture(prob, residual_of(prob))
        return prob
    prev = synth.config2(seed=1017, resolve=resolve)
    fields = prev_solve(prev)
    return synth.config2(p0=synth.gather(fields, prev.blocks), resolve=resolve)


def stop_rule(prob):
    """Independent blocks (configuration 4) are each solved to the tolerance:
    the per-block rule; otherwise the global relative residual."""
    return 2 if prob.name == "config4" else 0


def gpu_residual_of(prob):
    """b - A p with b = 0 on the GPU (the FP64 defect into the level-1 rhs)."""
    def residual(pex):
        from hydro3d_b200 import MultigridSolver, host_field
        s = MultigridSolver(prob.blocks, prob.ngrid, device=int(os.environ.get("LOCAL_RANK", 0)))
        s.coeff()
        s.zero_field("b")
        for ib in range(len(prob.blocks)):
            s.upload("p", ib, pex[ib])
        s.residual()
        out = [s.get_level(1, "rhs", ib) for ib in range(len(prob.blocks))]
        s.close()
        return out
    return residual


def oracle_residual_of(threads):
    """b - A p with b = 0 by the oracle (its level-1 exchangepp ghost fill)."""
    def make(prob):
        def residual(pex):
            from hydro3d_b200 import with_ghost
            o = OracleSolver(prob, threads, need_b=False)
            p = [np.ascontiguousarray(with_ghost(x, d)) for x, d in zip(pex, prob.blocks)]
            zeros = [np.zeros((d.n[2], d.n[1], d.n[0])) for d in prob.blocks]
            r, _, _, _ = o.orc.residual(p, zeros)
            o.close()
            return r
        return residual
    return make


def gpu_prev_solve(prob):
    s = build_solver_dev(prob, "fp64", int(os.environ.get("LOCAL_RANK", 0)))
    info = s.solve_resident(tol=TOL, maxcy=400)
    if not info["converged"]:
        raise RuntimeError("previous-seed solve did not converge")
    from hydro3d_b200 import host_field
    out = [host_field(d) for d in prob.blocks]
    for ib in range(len(prob.blocks)):
        s.download("p", ib, out[ib])
    s.close()
    return out


class OracleSolver:
    """The oracle (C restatement of the reference multigrid, OpenMP over the
    planes of each block) set up on one workload."""

    def __init__(self, prob, threads, need_b=True):
        from oracle import oracle as O
        import ctypes as C
        from hydro3d_b200 import interior, with_ghost
        od = (O.BlockDesc * len(prob.blocks))()
        C.memmove(od, (type(prob.blocks[0]) * len(prob.blocks))(*prob.blocks), C.sizeof(od))
        self.orc = O.Oracle(list(od), prob.ngrid, 3, 2, 1, lsm=prob.var_coef, threads=threads)
        if prob.var_coef:
            for ib, (d, x) in enumerate(zip(prob.blocks, prob.dens)):
                self.orc.set_density(ib, np.ascontiguousarray(interior(x, d)))
        self.orc.coeff()
        if not need_b:
            return
        self.b = [np.ascontiguousarray(interior(x, d)) for x, d in zip(prob.b, prob.blocks)]
        self.p0 = [np.ascontiguousarray(with_ghost(x, d)) for x, d in zip(prob.p0, prob.blocks)]

    def solve(self, maxcy=400, tol=TOL):
        """One defect-correction solve from p0; returns (ms, result)."""
        t0 = time.perf_counter()
        res = self.orc.solve(self.p0, self.b, tol=tol, maxcy=maxcy)
        return (time.perf_counter() - t0) * 1e3, res

    def close(self):
        self.orc.close()


def oracle_prev_solve(threads):
    def solve(prob):
        from hydro3d_b200 import host_field, interior
        o = OracleSolver(prob, threads)
        _, res = o.solve()
        o.close()
        if res["status"] != 0:
            raise RuntimeError("previous-seed oracle solve did not converge")
        out = [host_field(d) for d in prob.blocks]
        for x, d, pr in zip(out, prob.blocks, res["p"]):
            interior(x, d)[...] = pr[1:-1, 1:-1, 1:-1]
        return out
    return solve


def timed_solves(s, prob, steps, warmup, profile=False, barrier=None, maxcy=400, require=True):
    """Returns per-step device ms and the last info (inputs resident in HBM).
    require=False accepts a solve that ends at maxcy (its time and residual
    are reported as they are)."""
    def one():
        if not any(np.any(p) for p in prob.p0):
            s.zero_field("p")
        else:
            for ib in range(len(prob.blocks)):
                s.upload("p", ib, prob.p0[ib])
        return s.solve_resident(tol=TOL, maxcy=maxcy, stop_rule=stop_rule(prob), raise_diverged=require)
    for _ in range(warmup):
        info = one()
    s.set_profiling(profile)
    if barrier:
        barrier()
    ms, infos = [], []
    for _ in range(steps):
        info = one()
        if require and not info["converged"]:
            raise RuntimeError(f"solve did not converge: {info}")
        ms.append(info["device_ms"])
        infos.append(info)
    s.set_profiling(False)
    return ms, infos


def e2e_solves(s, prob, steps):
    """newsolv_mg through the public API from pinned host buffers (H2D and D2H
    inside the timed region)."""
    import torch
    pin_b = [torch.from_numpy(x).pin_memory().numpy() for x in prob.b]
    pin_p = [torch.from_numpy(x).pin_memory().numpy() for x in prob.p0]
    work = [torch.empty(x.shape, dtype=torch.float64).pin_memory().numpy() for x in prob.p0]
    times = []
    for _ in range(steps):
        for w, p in zip(work, pin_p):
            w[...] = p
        t0 = time.perf_counter()
        info = s.newsolv_mg(work, pin_b, tol=TOL, maxcy=400, stop_rule=stop_rule(prob))
        times.append((time.perf_counter() - t0) * 1e3)
        if not info["converged"]:
            raise RuntimeError("e2e solve did not converge")
    h2d = sum(x.nbytes for x in prob.b) + sum(x.nbytes for x in prob.p0)
    d2h = sum(x.nbytes for x in prob.p0)
    return times, h2d, d2h


def mean_removed_error(a_list, b_list, blocks, per_block=False):
    """Relative L2 difference after removing the mean (of every block when
    the blocks are independent problems, each with its own constant)."""
    from hydro3d_b200 import interior
    a = [interior(x, d).ravel() for x, d in zip(a_list, blocks)]
    b = [interior(x, d).ravel() for x, d in zip(b_list, blocks)]
    if per_block:
        a = [x - x.mean() for x in a]
        b = [x - x.mean() for x in b]
    a = np.concatenate(a)
    b = np.concatenate(b)
    a = a - a.mean()
    b = b - b.mean()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def cpu_full_solve(prob, threads):
    """One complete FP64 solve of the workload by the oracle to 1e-8 (the
    reference algorithm, measured, not projected).  On the variable-density
    workload the reference's coarse operator diverges: the solve stops at
    FP64_CAP cycles and the result says so (res["status"] != 0)."""
    o = OracleSolver(prob, threads)
    ms, res = o.solve(maxcy=FP64_CAP if prob.var_coef else 400)
    o.close()
    if res["status"] != 0 and not prob.var_coef:
        raise RuntimeError(f"oracle solve did not converge ({res['cycles']} cycles)")
    return ms, res


def run_reference(args):
    """The reference's CPU algorithm (the oracle: a C restatement of the
    reference multigrid, no Fortran toolchain exists to build the reference
    itself) on the box's host cores.  Every timed step is one complete
    converged FP64 solve of the workload; every warm-up step one V-cycle.
    Neither the problem set-up nor the solve loads the CUDA library."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    from oracle import oracle as O
    O.lib()
    prob = make_problem(args.config, resolve=oracle_resolve, prev_solve=oracle_prev_solve(threads),
                        residual_of=oracle_residual_of(threads))
    o = OracleSolver(prob, threads)
    for _ in range(args.warmup):
        o.solve(maxcy=1, tol=0.0)
    ms, cycles = [], []
    for _ in range(args.steps):
        t, res = o.solve()
        if res["status"] != 0:
            raise RuntimeError(f"oracle solve did not converge ({res['cycles']} cycles)")
        ms.append(t)
        cycles.append(res["cycles"])
    o.close()
    value = sum(ms) / len(ms)
    line = {
        "impl": "reference", "metric": "poisson_solve_ms_to_1e-8", "value": round(value, 3), "unit": "ms",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(value, 3),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_of(args.config, prob),
        "cycles": cycles[-1], "relres": res["relres"],
        "cpu_baseline": {"value": round(value, 3), "unit": "ms", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} complete FP64 solves of the full workload to 1e-8 "
                                   f"({cycles[-1]} V(2,1) cycles each, measured); warm-up steps one V-cycle"},
        "e2e": {"value": round(value, 3), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def config_of(cfg, prob):
    return {"workload": WORKLOADS[cfg], "tol": TOL, "cells": prob.cells,
            "l2": "inputs larger than L2 (one level-1 FP64 field is %.0f MB)" % (prob.cells * 8 / 1e6)
            if prob.cells * 8 > 126e6 else "inputs smaller than L2 (no flush between solves)"}


def mcell_updates(prob, cycles, sweeps=3):
    """Cell updates of `cycles` V-cycles of `sweeps` sweeps a level (V(2,1):
    two before and one after the coarse correction)."""
    per = 0
    for d in prob.blocks:
        for g in range(1, prob.ngrid + 1):
            s = 2 ** (min(g, d.ngrid) - 1)  # level clamp of a block past its last level
            per += (d.n[0] // s) * (d.n[1] // s) * (d.n[2] // s) * sweeps
    return per * cycles


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--ncu-region", action="store_true",
                    help="profiling driver: mixed solver only, warm-up solves, then one solve inside "
                         "cudaProfilerStart/Stop (use with ncu --profile-from-start off)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)

    rank, world, local = dist_env()
    dist = world > 1
    barrier = None
    if dist:
        import torch.distributed as tdist
        from datetime import timedelta
        tdist.init_process_group("gloo", timeout=timedelta(seconds=600))
        barrier = tdist.barrier
    import hydro3d_b200  # noqa: F401  (loads libh3dmg.so; raises if missing)
    os.environ.setdefault("CUDA_DEVICE_ORDER", "PCI_BUS_ID")
    device = local
    prob = make_problem(args.config, prev_solve=gpu_prev_solve, residual_of=gpu_residual_of)
    peak, peak_kind = load_peaks()
    if args.ncu_region:
        import torch
        s = build_solver_dev(prob, "mixed", device)
        for _ in range(args.warmup):
            s.zero_field("p")
            s.solve_resident(tol=TOL, maxcy=400)
        s.zero_field("p")
        torch.cuda.profiler.start()
        info = s.solve_resident(tol=TOL, maxcy=400)
        torch.cuda.profiler.stop()
        print(json.dumps({"ncu_region": True, "cycles": info["cycles"], "device_ms": info["device_ms"],
                          "kernel_launches": info["kernel_launches"]}), flush=True)
        return

    mixed = build_solver_dev(prob, "mixed", device)
    fp64 = build_solver_dev(prob, "fp64", device)
    # the FP64 solution to EXACT_TOL (FP64 V-cycles with the converged
    # coarsest level): what "error against the FP64 solution" is measured on
    exact = build_solver_dev(prob, "fp64", device, coarse_sweeps=COARSE_SWEEPS,
                             coarse_op=1 if prob.var_coef else 0, same_cycle=True)
    # the FP64 counterpart of the mixed solver (the same V-cycle in FP64) to
    # the benchmark tolerance, then to EXACT_TOL
    ms_fp64c, infos_fp64c = timed_solves(exact, prob, max(1, min(args.steps, 3)), 1, barrier=barrier)
    ex_info = exact.solve_resident(tol=EXACT_TOL, maxcy=400, stop_rule=stop_rule(prob))
    if not ex_info["converged"]:
        raise RuntimeError(f"FP64 solve to {EXACT_TOL} did not converge: {ex_info}")

    clocks = ClockSampler(device)
    clocks.start()
    clocks.wait_running()
    ms_mixed, infos_mixed = timed_solves(mixed, prob, args.steps, args.warmup, barrier=barrier)
    # a timed region of a few tens of ms can fall between two samples: the
    # same solves continue (untimed) until the sampler has three from the
    # window that began with the timed region
    t_extra = time.perf_counter()
    while clocks.count() < 3 and time.perf_counter() - t_extra < 3.0:
        timed_solves(mixed, prob, 1, 0)
    clk = clocks.stop()
    clk["window"] = "the timed region and the same solves after it until three samples (50 ms interval)"
    # the smoother roofline: the same solves again with every level-1 sweep
    # bracketed by CUDA events on the solve stream (outside the timed region,
    # whose graphs carry no event nodes)
    _, infos_prof = timed_solves(mixed, prob, args.steps, 1, profile=True)
    # the reference's FP64 algorithm; on the 1000:1 two-phase workload its
    # coarse levels (coefficients from the averaged density) do not converge
    # (it diverges at 128^3 and 256^3): it is run for at most FP64_CAP cycles
    # and reported as it ends
    fp64_cap = FP64_CAP if prob.var_coef else 400
    ms_fp64, infos_fp64 = timed_solves(fp64, prob, max(1, min(args.steps, 3)), min(args.warmup, 3) if prob.var_coef
                                       else args.warmup, barrier=barrier, maxcy=fp64_cap,
                                       require=not prob.var_coef)

    total_ms = max_over_ranks(sum(ms_mixed), world)
    value = job_ms_per_solve(total_ms, args.steps, world)

    # solution errors against the FP64 solution (same inputs, solved to EXACT_TOL)
    from hydro3d_b200 import host_field
    pm = [host_field(d) for d in prob.blocks]
    pf = [host_field(d) for d in prob.blocks]
    px = [host_field(d) for d in prob.blocks]
    for ib in range(len(prob.blocks)):
        mixed.download("p", ib, pm[ib])
        fp64.download("p", ib, pf[ib])
        exact.download("p", ib, px[ib])
    indep = stop_rule(prob) == 2
    err = mean_removed_error(pm, px, prob.blocks, indep)
    err_plain = mean_removed_error(pf, px, prob.blocks, indep)
    exact.close()

    # roofline of the dominant kernel (level-1 FP32 smoother)
    info = infos_mixed[-1]
    sm_ms = sum(i["smoother_ms"] for i in infos_prof)
    sm_n = sum(i["smoother_launches"] for i in infos_prof)
    sm_bytes = sum(i["smoother_bytes"] for i in infos_prof)  # full sweeps: 12 B a cell (iterate, rhs, new iterate)
    bytes_launch = sm_bytes / max(sm_n, 1)
    avg_launch_ms = sm_ms / max(sm_n, 1)
    achieved = sm_bytes / (sm_ms * 1e-3) / 1e9 if sm_n else None
    traffic = read_profile_traffic(args.config, mixed.get_smoother(1)[0])

    e2e = None
    if not args.no_e2e:
        et, h2d, d2h = e2e_solves(mixed, prob, max(1, min(args.steps, 3)))
        e2e = {"value": round(statistics.median(et), 3), "unit": "ms", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        v, res = cpu_full_solve(prob, threads)
        what = ("one complete FP64 solve of the full workload to 1e-8 by the oracle" if res["status"] == 0 else
                "the oracle's FP64 solve of the full workload stopped unconverged (the reference algorithm "
                f"diverges here, relres {res['relres']:.3g})")
        cpu = {"value": round(v, 1), "unit": "ms", "cores": threads, "kind": "port",
               "sample": f"{what} ({res['cycles']} V(2,1) cycles, measured)", "cycles": res["cycles"],
               "converged": res["status"] == 0}

    if rank == 0:
        fp64_ms = statistics.median(ms_fp64)
        line = {
            "metric": "poisson_solve_ms_to_1e-8", "value": round(value, 3), "unit": "ms", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(value, 3),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic (seeded; no dataset)",
            "config": dict(config_of(args.config, prob),
                           precision="FP32 V(%d,%d) RBGS inside FP64 refinement" % MIXED_CYCLE[args.config][:2],
                           inner_cycles=MIXED_CYCLE[args.config][2],
                           fp32_sweeps="over-relaxation %.2f, %s" % (
                               MIXED_SMOOTHER[args.config][0],
                               "red-black order across block faces" if MIXED_SMOOTHER[args.config][1]
                               else "the reference's per-block red-black order"),
                           coarse="FP64 coarsest level: solved by its pseudo-inverse when it has at most "
                                  "%d cells, else %d RBGS sweeps" % (8 * COARSE_SWEEPS, COARSE_SWEEPS)
                           + ("; coarse coefficients by face sums" if prob.var_coef else ""),
                           parallelism="replicas" if world > 1 else "single GPU"),
            "fp64_ms": round(fp64_ms, 3), "speedup_vs_fp64": round(fp64_ms / (total_ms / (args.steps * world) * world), 3)
            if world == 1 and infos_fp64[-1]["converged"] else None,
            "fp64_status": "converged" if infos_fp64[-1]["converged"] else
            ("diverged" if infos_fp64[-1]["status"] == -4 else "not converged") +
            f" after {infos_fp64[-1]['cycles']} cycles",
            "fp64_same_cycle_ms": round(statistics.median(ms_fp64c), 3),
            "speedup_vs_fp64_same_cycle": round(statistics.median(ms_fp64c) / value, 3) if world == 1 else None,
            "cycles_fp64_same_cycle": infos_fp64c[-1]["cycles"],
            "cycles_mixed": info["cycles"], "outer_mixed": info["outer"], "cycles_fp64": infos_fp64[-1]["cycles"],
            "relres_mixed": info["relres"], "relres_fp64": infos_fp64[-1]["relres"], "error_vs_fp64": err,
            "error_note": f"relative L2 (means removed) against the FP64 solution solved to {EXACT_TOL}; "
                          f"the plain FP64 solve to {TOL} is {err_plain:.2e} from it",
            "error_plain_fp64": err_plain,
            "mcell_updates_per_s": round(mcell_updates(prob, info["cycles"], sum(MIXED_CYCLE[args.config][:2]))
                                         / (value * 1e-3) / 1e6, 1),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1) if achieved else None, "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4) if achieved else None,
                         "traffic": traffic, "kernel": "level-1 FP32 full red-black sweep (autotuned variant %d)"
                         % mixed.get_smoother(1)[0],
                         "bytes_per_launch": bytes_launch, "avg_launch_ms": round(avg_launch_ms, 5),
                         "peak_source": peak_kind},
            "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": int(sum(i["kernel_launches"] for i in infos_mixed)),
            "smoother_level1": list(mixed.get_smoother(1)[:2]),
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    if dist:
        import torch.distributed as tdist
        tdist.barrier()
        tdist.destroy_process_group()


def read_profile_traffic(cfg, variant):
    """DRAM bytes (read + write) per level-1 smoother launch from the committed
    ncu summary of this workload (lines `traffic_bytes_per_launch[variant] =
    bytes`), when it holds a capture of the variant the autotuner chose in this
    run; None otherwise."""
    p = os.path.join(ROOT, "profiles", "k_rbgs_win_fp32_config3.md")
    if cfg != 3 or not os.path.exists(p):
        return None
    key = "traffic_bytes_per_launch[%d]" % variant
    for ln in open(p):
        if "=" in ln and ln.split("=")[0].strip() == key:
            try:
                return float(ln.split("=", 1)[1].strip())
            except ValueError:
                return None
    return None


def prob_config(prob):
    """Configuration number of a workload built by synth (config1 .. config5)."""
    return int(prob.name[-1]) if prob.name.startswith("config") else 0


def build_solver_dev(prob, precision, device, coarse_sweeps=None, coarse_op=None, same_cycle=None):
    """A solver on `device` with the workload's b and p0 resident.  The mixed
    solver runs the workload's cycle (MIXED_CYCLE), converges its FP64
    coarsest level (directly or by COARSE_SWEEPS sweeps) and, for variable
    coefficients, builds its coarse levels by face sums; the FP64 solver keeps
    the reference's V(2,1), 3 coarsest sweeps and coarse coefficients unless
    told otherwise (same_cycle: the mixed solver's cycle shape and coarse
    solve, in FP64)."""
    from hydro3d_b200 import MultigridSolver
    mixed = precision == "mixed"
    same = mixed if same_cycle is None else same_cycle
    if coarse_sweeps is None:
        coarse_sweeps = COARSE_SWEEPS if mixed else 0
    if coarse_op is None:
        coarse_op = 1 if (mixed and prob.var_coef) else 0
    ir, ip, inner = MIXED_CYCLE[prob_config(prob)]
    om, rbo = MIXED_SMOOTHER[prob_config(prob)] if mixed else (0.0, 0)
    s = MultigridSolver(prob.blocks, prob.ngrid, precision=precision, var_coef=prob.var_coef, maxcy=400,
                        device=device, coarse_sweeps=coarse_sweeps, coarse_op=coarse_op,
                        coarse_direct=COARSE_DIRECT and same,
                        irestr=ir if same else 2, iproln=ip if same else 1, inner_cycles=inner if mixed else 0,
                        omega=om, rb_order=rbo)
    if prob.var_coef:
        for ib, d in enumerate(prob.dens):
            s.set_density(ib, d)
    s.coeff()
    for ib in range(len(prob.blocks)):
        s.upload("b", ib, prob.b[ib])
        s.upload("p", ib, prob.p0[ib])
    return s


if __name__ == "__main__":
    main()
