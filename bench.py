#!/usr/bin/env python
"""Benchmark: time to relative residual 1e-10 on one B200.

Workload (the configuration the headline metric is quoted on): 3D 7-point
Poisson on a 128^3 grid (n = 2,097,152, nnz = 14,581,760), FP64, stored as
ELL (width 7) — CSR with --format csr — b ~ U(-1,1) from seed 0, x0 = 0,
BiCGSTAB + ILU(0), rtol 1e-10.  One step = one complete solve of that system
by the mixed-precision refinement (FP64 outer residual/update, one FP32
BiCGSTAB carried across the refinement steps, BF16 ILU(0) factors, ILU(0)
applied by 3 Jacobi sweeps per triangle — the reference GPU path's
approximate triangular solve).  The FP64 GPU path with the same sweeps, and
FP64 and mixed with the exact triangular solves, are timed alongside under
`variants`; `speedup_vs_fp64_same_trsv` divides FP64 by mixed for each
triangular-solve mode.

  value   device time per solve (ms), inputs resident in HBM, CUDA events on
          the solver's stream, max over ranks
  e2e     the same solve through the C ABI with host buffers: xs_mat_update
          (values H2D + numeric ILU(0) on the device) + xs_solve (b, x0 H2D;
          x D2H), all inside the timed region
  roofline  the dominant kernel of the timed solve (ILU(0) apply by 3 Jacobi
          sweeps, BF16 factors / FP32 vectors) timed live: algorithmic
          bytes / CUDA-event duration
  cpu_baseline  the reference algorithm on the host (restated BiCGSTAB +
          ILU(0) with the reference's own compiled ilu0_simple arithmetic,
          exact triangular solves), one whole solve timed; SpMV and vector
          operations on all host threads, the factorisation and the
          triangular solves sequential as in the reference

Multi-GPU (--gpus N under torchrun): replicas — every rank solves its own
copy of the system; no data-path collective exists in a single solve.
`--impl reference` times whole solves of the reference CPU implementation of
the same workload on the host (rank 0 only).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time-to-1e-10 residual (FP64 vs mixed-refined, 1 B200); SpMV/SpTRSV HBM GB/s"
# one string for both arms: the problem, and the triangular-solve mode each arm times
WORKLOAD = ("3D 7-point Poisson 128^3 (n=2097152, nnz=14581760), b~U(-1,1) seed 0, x0=0, BiCGSTAB + ILU(0) to "
            "relative residual 1e-10; GPU arm: mixed-precision refinement, ILU(0) applied by 3 Jacobi sweeps per "
            "triangle; reference arm: FP64, exact ILU(0) triangular solves")


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) > 8:
                for k, nm in enumerate(names):
                    if r[5 + k].lower() == "active":
                        reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def profile_traffic(name: str):
    """DRAM bytes (read + write) summed over the launches of an ncu summary
    committed under profiles/ (one capture of the kernel's launches on this
    workload), or None when the summary is absent."""
    path = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(path):
        return None
    scale = {"byte": 1.0, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9}
    total = 0.0
    for line in open(path):
        for what in ("| DRAM read (", "| DRAM write ("):
            if line.startswith(what):
                unit = line[len(what):].split(")")[0]
                vals = [c.strip() for c in line.split("|")[2:-1]]
                total += sum(float(v) for v in vals) * scale[unit]
    return total or None


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def shard(items, ws, rank):
    """Replica assignment: item i belongs to rank i % ws."""
    return [x for i, x in enumerate(items) if i % ws == rank]


def max_over_ranks(value, ws, device=None):
    if ws == 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()


def make_problem():
    from xsolver_b200 import stencils as st

    A = st.poisson3d_7pt(128)
    b = st.rhs_uniform(A.n, 0)
    return A, b


def cpu_threads():
    """Host threads this process may run on."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_reference_solve(A, b):
    """One whole solve of the reference algorithm on the host: ILU(0)
    factorisation (sequential, as the reference's ilu0_simple), then the
    reference BiCGSTAB with its SpMV and vector operations on all host
    threads and the exact ILU(0) triangular solves sequential, as the
    reference's CPU path runs them, to relative residual 1e-10.  Returns
    (setup s, solve s, iterations, true relative residual, threads)."""
    import oracle

    T = cpu_threads()
    t0 = time.perf_counter()
    F = oracle.ilu0(A)
    t_setup = time.perf_counter() - t0
    t0 = time.perf_counter()
    x, it, _ = oracle.bicgstab_threads(A, b, F, tol=1e-10, maxiter=1000, threads=T)
    t_solve = time.perf_counter() - t0
    rel = float(np.linalg.norm(b - A.to_scipy() @ x) / np.linalg.norm(b))
    return t_setup, t_solve, it, rel, T


def cpu_reference_warmup(A, b):
    """Untimed warm-up: ILU(0) plus two iterations (pages the matrix and the
    libraries in without the cost of a whole solve)."""
    import oracle

    F = oracle.ilu0(A)
    oracle.bicgstab_threads(A, b, F, tol=1e-300, maxiter=2, threads=cpu_threads())


def run_reference(args):
    ws, rank, local = _dist()
    if rank != 0:
        return 0
    A, b = make_problem()
    for _ in range(args.warmup):
        cpu_reference_warmup(A, b)
    setup, solve, iters, rels = [], [], [], []
    threads = cpu_threads()
    for _ in range(args.steps):
        ts, tv, it, rel, threads = cpu_reference_solve(A, b)
        setup.append(ts * 1e3)
        solve.append(tv * 1e3)
        iters.append(it)
        rels.append(rel)
    tot = [a + c for a, c in zip(setup, solve)]
    v = float(np.median(tot))
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "ms", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": v, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded stencil system)",
        "config": {"workload": WORKLOAD, "format": "csr",
                   "solver": "reference CPU path: ILU(0) factorisation + FP64 BiCGSTAB with exact ILU(0) "
                             "triangular solves; SpMV and vector operations on all host threads, the "
                             "factorisation and the triangular solves sequential"},
        "cpu_baseline": {"value": v, "unit": "ms", "cores": threads, "kind": "port",
                         "sample": "one whole solve per step: ILU(0) factorisation (the reference's ilu0_simple "
                                   "arithmetic) + restated BiCGSTAB to relative residual 1e-10 with its SpMV and "
                                   "vector operations on all host threads; warm-up steps run the factorisation "
                                   "and 2 iterations",
                         "host_threads_available": os.cpu_count()},
        "setup_ms": float(np.median(setup)), "solve_ms": float(np.median(solve)),
        "steps_ms": [round(t, 1) for t in tot], "iterations": int(np.median(iters)),
        "true_relres": float(max(rels)), "statistic": "median of the timed steps",
        "e2e": {"value": v, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch

    ws, rank, local = _dist()
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    from xsolver_b200.api import Plan, Solver

    A, b = make_problem()
    n = A.n
    fmt = args.format

    def make_solver(mixed: bool, trsv: int):
        S = Solver(A, fmt=fmt).ksp_settype("bicgstab").ksp_setoption(1e-10, 3000).pc_settype("ilu0")
        S.pc_set_trsv(trsv)
        if mixed:
            # one FP32 BiCGSTAB carried across the refinement steps, the true
            # residual replaced every two decades (the best interval of those
            # measured over six right-hand sides)
            S.set_precision("fp64", "fp32", "bf16").set_inner(1e-2, 300).set_refinement_mode(True)
        return S

    # headline: mixed-precision refinement with BF16 ILU(0) factors and the
    # Jacobi-sweep triangular solve in the inner FP32 solve; the FP64 GPU path
    # (exact sync-free SpTRSV) and the two cross-over variants are timed too
    variants = {
        "mixed_sweeps": make_solver(True, args.sweeps),
        "fp64_exact": make_solver(False, 0),
        "fp64_sweeps": make_solver(False, args.sweeps),
        "mixed_exact": make_solver(True, 0),
    }
    db = torch.from_numpy(b).to(dev)
    x = torch.zeros(n, dtype=torch.float64, device=dev)

    # pinned host buffers for the end-to-end measurement
    h_vals = torch.from_numpy(A.val).pin_memory().numpy()
    h_b = torch.from_numpy(b).pin_memory().numpy()
    h_x = torch.zeros(n, dtype=torch.float64).pin_memory().numpy()

    def timed(S, steps, mode="device"):
        """mode 'device': inputs resident, one solve per step.  'e2e': every
        step uploads the matrix values (xs_mat_update: H2D + numeric ILU(0)
        refactorisation on the device) and solves through xs_solve with host
        b / x0 / x (H2D of b and x0, D2H of x), all from pinned memory.
        'e2e_solve': xs_solve alone (factors kept from the previous step)."""
        stream = torch.cuda.ExternalStream(S.stream_ptr(), device=dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        barrier(ws)
        torch.cuda.synchronize()
        e0.record(stream)
        launches = 0
        for _ in range(steps):
            if mode == "device":
                x.zero_()
                torch.cuda.synchronize()
                S.solve_device(db, x)
            else:
                if mode == "e2e":
                    S.mat_update(h_vals)
                h_x[:] = 0.0
                S.solve(h_b, out=h_x)
            launches += S.launches()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(ws)
        ms = e0.elapsed_time(e1) / steps
        return max_over_ranks(ms, ws, dev), launches

    # warm-up (includes factorisation and graph capture)
    for _ in range(max(args.warmup, 3)):
        for S in variants.values():
            x.zero_()
            S.solve_device(db, x)
    clocks = Clocks(local)
    clocks.start()
    res = {}
    for name, S in variants.items():
        steps = args.steps if name in ("mixed_sweeps", "fp64_exact") else max(1, args.steps // 2)
        ms, launches = timed(S, steps)
        t = S.timing()
        res[name] = {"ms": ms, "iterations": t["iterations"], "outer_steps": S.outer_steps(),
                     "launches_per_solve": launches // steps, "setup_ms": t["setup_ms"]}
    clk = clocks.stop()
    Asp = A.to_scipy()
    for name, S in variants.items():
        x.zero_()
        S.solve_device(db, x)
        xs = x.cpu().numpy()
        res[name]["true_relres"] = float(np.linalg.norm(b - Asp @ xs) / np.linalg.norm(b))
    S_mix = variants["mixed_sweeps"]
    ms_mix = res["mixed_sweeps"]["ms"]
    # e2e through the public API with pinned host buffers: one untimed step,
    # then every step timed on its own (the host issues these calls, so a
    # busy host shows up as GPU idle time); the median step is reported
    def timed_steps(S, steps, mode):
        timed(S, 1, mode)
        per = [timed(S, 1, mode)[0] for _ in range(steps)]
        return float(np.median(per)), per

    e2e_ms, e2e_per = timed_steps(S_mix, max(5, args.steps), "e2e")
    e2e_solve_ms, _ = timed_steps(S_mix, max(5, args.steps), "e2e_solve")
    # numeric refactorisation after a value update: median of 5 (one sample
    # can catch a host stall between the launches it times)
    refactor = []
    for _ in range(5):
        S_mix.mat_update(h_vals)
        x.zero_()
        S_mix.solve_device(db, x)
        refactor.append(S_mix.timing()["setup_ms"])
    refactor_ms = float(np.median(refactor))

    # kernel roofline, timed live with CUDA events (L2 flushed between reps)
    peak, peak_kind = _peaks()
    P = Plan(A).factor("ilu0")
    P.build_ell()
    kern = {}

    def tk(label, op, prec, trsv):
        P.set_factor_precision(prec)
        P.set_trsv(trsv)
        t = P.time_op(op, reps=10, flush_l2=True)
        by = P.op_bytes(op)
        kern[label] = {"ms": t, "bytes": by, "GBs": by / t / 1e6, "frac": by / t / 1e6 / peak}

    tk("spmv_csr_fp64", "csr64", "fp64", 0)
    tk("spmv_ell_fp64", "ell64", "fp64", 0)
    tk("spmv_csr_fp32", "csr32", "fp64", 0)
    tk("spmv_ell_fp32", "ell32", "fp64", 0)
    tk("sptrsv_L_fp64_exact", "lsolve", "fp64", 0)
    tk("sptrsv_U_fp64_exact", "usolve", "fp64", 0)
    tk("sptrsv_LU_bf16_exact", "lusolve", "bf16", 0)
    tk(f"lu_bf16_sweeps{args.sweeps}", "lusolve", "bf16", args.sweeps)
    tk(f"lu_fp64_sweeps{args.sweeps}", "lusolve", "fp64", args.sweeps)
    levels = P.levels()
    dom = kern[f"lu_bf16_sweeps{args.sweeps}"]
    lines = {
        "metric": METRIC, "value": ms_mix, "unit": "ms", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_mix, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 (outer) / f32 (inner) / bf16 (factors)",
        "data": "synthetic (seeded stencil system, inputs larger than L2)",
        "config": {"workload": WORKLOAD, "format": fmt,
                   "solver": f"mixed-precision refinement: FP64 outer residual/update, one FP32 BiCGSTAB carried "
                             f"across the steps (residual replaced by the FP64 residual every 1e-2 drop), "
                             f"BF16 ILU(0) factors, triangular solves by {args.sweeps} Jacobi sweeps",
                   "parallelism": f"replicas x{ws}", "l2": "inputs (175 MB matrix) larger than L2; kernels timed "
                                                           "with an L2 flush (384 MB written, then 384 MB read) "
                                                           "between repetitions"},
        "speedup_vs_fp64_same_trsv": {"sweeps": res["fp64_sweeps"]["ms"] / ms_mix,
                                      "exact": res["fp64_exact"]["ms"] / res["mixed_exact"]["ms"]},
        "variants": res, "levels": {"L": levels[0], "U": levels[1]},
        "e2e": {"value": e2e_ms, "unit": "ms", "h2d_bytes_per_step": A.nnz * 8 + 2 * n * 8,
                "d2h_bytes_per_step": n * 8,
                "includes": "xs_mat_update (matrix values H2D + numeric ILU(0) on the device) + xs_solve "
                            "(b, x0 H2D; x D2H), pinned host buffers",
                "solve_only_ms": e2e_solve_ms, "steps_ms": [round(v, 3) for v in e2e_per],
                "statistic": "median of the timed steps"},
        "setup_ms": {"first": res["mixed_sweeps"]["setup_ms"], "numeric_refactor": refactor_ms},
        "gpu_launches": int(res["mixed_sweeps"]["launches_per_solve"] * args.steps),
        "roofline": {"bound": "hbm", "kernel": f"ILU(0) apply, BF16 factors, FP32 vectors, {args.sweeps} Jacobi sweeps",
                     "achieved": dom["GBs"], "peak": peak, "unit": "GB/s", "frac": dom["frac"],
                     "peak_kind": peak_kind,
                     "traffic": profile_traffic("sweep_bf16_diagonal_ell_128cubed.md"),
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum over the 4 launches of one "
                                       "apply, profiles/sweep_bf16_diagonal_ell_128cubed.md (writes land in L2)",
                     "algorithmic_bytes": dom["bytes"]},
        "kernels": kern,
        "clocks": clk,
    }
    if rank == 0 and not args.no_cpu and ws == 1:
        t_setup, t_solve, it_cpu, rel_cpu, thr = cpu_reference_solve(A, b)
        lines["cpu_baseline"] = {"value": (t_setup + t_solve) * 1e3, "unit": "ms", "cores": thr, "kind": "port",
                                 "sample": "one whole solve: ILU(0) factorisation (the reference's ilu0_simple "
                                           "arithmetic) + restated BiCGSTAB with exact ILU(0) triangular solves to "
                                           "relative residual 1e-10 (FP64); SpMV and vector operations on all "
                                           "host threads, factorisation and triangular solves sequential",
                                 "setup_ms": t_setup * 1e3, "solve_ms": t_solve * 1e3, "iterations": it_cpu,
                                 "true_relres": rel_cpu, "host_threads_available": os.cpu_count()}
    if rank == 0:
        print(json.dumps(lines), flush=True)
    if ws > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--format", default="ell", choices=["csr", "ell"])
    ap.add_argument("--sweeps", type=int, default=3)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
