#!/usr/bin/env python
"""Benchmark: time to a relative residual of 1e-8, mixed-precision vs FP64 MG-PCG, on the
3D Q1 Poisson problem of 16,974,593 DOFs (unit cube, 256^3 cells, per-element coefficient
k = exp(g), g ~ N(0,1) i.i.d., f = 1, homogeneous Dirichlet), one B200 per rank.

One "step" is one complete solve from a zero initial guess to ||r|| <= 1e-8 ||r0|| with the
hierarchy resident in HBM (every finest-level operator application streams more than L2 holds).
  value  = mixed-precision solve time (FP64 outer PCG, FP32 V-cycle, matrix-free Q1 operator)
  e2e    = the same solve through fb_mg_solve_host with pinned host rhs/solution buffers
  fp64   = the plain FP64 GPU MG-PCG (the drop-in, assembled SELL matrices) on the same problem;
           fp64_stencil / fp64_matfree: the FP64 solve on the other storage forms
  cpu_baseline = the oracle (this project's threaded restatement of the reference solver) solving
           the same problem at full size on the host cores; its solution gives err_vs_oracle
--impl reference: the reference's own CPU solver (FEAT3 built from its sources, serial) on the
  same full-size problem, as many complete timed solves as fit the time budget
Multi-GPU: replicas only (each rank solves its own copy; no collective on the data path).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--level L] [--impl reference]
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

METRIC = "time-to-rel-1e-8 (mixed vs FP64 MG-PCG, 1 B200); SpMV HBM GB/s vs 8 TB/s"
# headline form: FP64 outer PCG around an FP32 V-cycle on the matrix-free operator
HEAD_PREC, HEAD_FMT = "f32", "matfree"
HEAD_KERNEL = "matfree_jacobi_f32"
HEAD_KERNEL_NAME = ("k_mf_q1_stream12<float, EpiJacobiK<float,0,0>> finest level (matrix-free Q1, streaming slabs of "
                    "three planes, bulk-copy ring, two rows per thread, inverse diagonal from the cell coefficients, "
                    "packed FP32 pairs)")


# DRAM bytes per launch of the dominant kernel (dram__bytes_read.sum + dram__bytes_write.sum) from
# one ncu capture of that kernel alone; the capture and its scaling to the 257^3 lattice are
# stated with the figure's command in the design notes. It is a capture figure, not a live
# measurement of this run.
HEAD_KERNEL_DRAM_BYTES = 292.9e6


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--level", type=int, default=8, help="refinement level (N = 2^level cells per side)")
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--seed", type=int, default=2026)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-budget-s", type=float, default=240.0,
                    help="reference arm: seconds of timed full solves (no solve starts that would end past it; at least one)")
    ap.add_argument("--only", default=None,
                    help="profiling aid, e.g. f16, f64-sell, f16-stencil: run just this form's timed solves")
    return ap.parse_args()


def workload(level):
    n = (2 ** level + 1) ** 3
    return {"workload": f"3D Q1 Poisson, unit cube, {2 ** level}^3 cells ({n:,} DOFs), k=exp(N(0,1)) per element, "
                        f"f=1, Dirichlet 0; PCG + MG V(2,2) Richardson-Jacobi(0.5), levels 1..{level}, direct coarse",
            "dofs": n, "level": level,
            "l2": "inputs larger than L2 (126 MB): a finest-level matrix-free FP32 smoothing step streams 273 MB "
                  "(x, k, rhs, result) at level 8; the assembled FP64 matrix is 5.5 GB"}


def bench_config(args, world):
    """the workload both arms report, identically"""
    return {**workload(args.level), "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "seed": args.seed}


def coefficient(level, seed):
    rng = np.random.default_rng(seed)
    return np.exp(rng.standard_normal((2 ** level) ** 3))


# ------------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons every 50 ms while the headline form runs: start()
    returns once the sampler has printed its first line (at most 5 s), and only the samples read
    after that point count, so they all fall in the form's warm-up and timed solves."""
    def __init__(self, index):
        self.index, self.samples, self.proc, self.t_begin = index, [], None, 0.0

    def start(self):
        q = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
            "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            t0 = time.time()
            while not self.samples and time.time() - t0 < 5.0 and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        self.t_begin = time.time()

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append((time.time(), [s.strip() for s in line.split(",")]))

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        run = [f for t, f in self.samples if t >= self.t_begin]
        sm = [float(s[0]) for s in run if len(s) >= 8 and s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in run if len(s) >= 8 and s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in run if len(s) >= 8 for i in range(4) if s[4 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(run)}


# ------------------------------------------------------------------------------- CPU reference
def run_reference_cpu(args):
    """The reference's own FP64 MG-PCG (oracle/_ref/feat_ref: FEAT3 compiled from its sources, the
    same composition) on the full-size problem with the same coefficient field, serial (the
    reference's lafem CPU kernels have no threading). One process: assembly once (untimed), up to
    min(W, 1) warm-up solves capped at one iteration, then complete solves from a zero initial
    guess, TimeStamp around Solver::solve only, until K are done or the next would end past the
    time budget (at least one)."""
    from oracle import pyoracle as po
    k = coefficient(args.level, args.seed)
    R = po.run_ref(3, 1, args.level, 1, rhs="one", k=k, solver="pcg", nu=2, omega_jac=0.5, coarse="direct",
                   tol=1e-8, repeat=max(1, args.steps), warmup=min(args.warmup, 1), budget_s=args.ref_budget_s,
                   outputs=False)
    info = R["info"]
    import shutil
    shutil.rmtree(R["workdir"], ignore_errors=True)
    times = [float(t) for t in np.atleast_1d(info["solve_times"])]
    return {"times": times, "iters": int(info["iters"]), "status": int(info["status"]),
            "setup_s": float(info["setup_time"]), "warmup_solves": int(info.get("warmup_solves", 0)),
            "final_rel_residual": float(info["def_final"]) / float(info["def_init"])}


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    from oracle import pyoracle as po
    if not po.have_ref():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/feat_ref was not built (reference sources absent at build time)"}))
        return 0
    ref = run_reference_cpu(args)
    t = float(np.median(ref["times"]))
    n = (2 ** args.level + 1) ** 3
    sample = (f"reference FEAT3 CPU MG-PCG (oracle/_ref/feat_ref, 1 thread: the reference's lafem CPU path is "
              f"serial) on the full problem ({n:,} DOFs): {len(ref['times'])} complete timed solve(s) of "
              f"{ref['iters']} iterations each (as many as fit in {args.ref_budget_s:.0f} s of timed solving, at "
              f"least one; {args.steps} requested), median {t:.1f} s; assembly {ref['setup_s']:.1f} s untimed; "
              f"{ref['warmup_solves']} warm-up solve(s) of one iteration")
    line = {"metric": METRIC, "impl": "reference", "value": t, "unit": "s", "n_gpus": world,
            "steps": len(ref["times"]), "steps_requested": args.steps, "warmup": args.warmup,
            "warmup_run": f"{ref['warmup_solves']} one-iteration solve(s)", "ms_per_step": 1e3 * t,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": bench_config(args, world),
            "cpu_baseline": {"value": t, "unit": "s", "cores": 1, "kind": "reference", "sample": sample,
                             "solve_times_s": ref["times"], "iters": ref["iters"], "setup_s": ref["setup_s"],
                             "dof_it_per_s": n * ref["iters"] / t, "host_cores_available": os.cpu_count()},
            "iters": ref["iters"], "status": ref["status"], "final_rel_residual": ref["final_rel_residual"],
            "e2e": {"value": t, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def oracle_baseline(args, k, n):
    """cpu_baseline leg of the native arm: the oracle (the threaded restatement of the reference
    solver, pinned to the reference's own full-size solve) on the same full-size problem. Returns
    the cpu_baseline entry and the oracle's FP64 solution, against which the GPU forms' errors are
    reported."""
    import time as _t
    from oracle import pyoracle as po
    t0 = _t.perf_counter()
    H = po.Hierarchy(3, 1, args.level, 1, k)
    b = H.rhs("one")
    t1 = _t.perf_counter()
    ref = H.solve(b, solver="pcg", nu=2, omega_jac=0.5, coarse="direct", tol=1e-8)
    t2 = _t.perf_counter()
    del H
    cb = {"value": t2 - t1, "unit": "s", "cores": po.threads(), "kind": "port",
          "sample": f"the oracle (this project's restatement of the reference's FP64 MG-PCG, independent loops on "
                    f"{po.threads()} OpenMP threads, reductions sequential) on the full problem ({n:,} DOFs): one "
                    f"complete solve of {ref['iters']} iterations; assembly {t1 - t0:.1f} s untimed",
          "iters": ref["iters"], "dof_it_per_s": n * ref["iters"] / (t2 - t1), "host_cores_available": os.cpu_count()}
    return cb, ref


def reference_run_samples(args):
    """the reference's own 257^3 solution at every 997th DOF (tests/golden/ref_c5_full_q1_3d_L8.npz,
    made by tests/golden/gen_golden.py from oracle/_ref/feat_ref) when this run solves that problem"""
    fn = os.path.join(ROOT, "tests", "golden", "ref_c5_full_q1_3d_L8.npz")
    if args.level != 8 or args.seed != 2026 or not os.path.exists(fn):
        return None
    d = np.load(fn)
    return int(d["u_stride"]), d["u_sample"], int(d["iters"])


# ------------------------------------------------------------------------------- ranks
class Ranks:
    """One process per GPU under torchrun (RANK / WORLD_SIZE / MASTER_* from the environment).
    Replicas only: every rank solves its own copy of the problem; the process group carries the
    barriers around the timed region and the max over ranks of each measured time, nothing of
    the data path. backend/device: "nccl"/"cuda" for the bench, "gloo"/"cpu" in the tests."""

    def __init__(self, backend="nccl", device="cuda", timeout_s=600):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.device = device
        self.dist = None
        if self.world > 1:
            import datetime
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()
        if self.device == "cuda":
            import torch
            torch.cuda.synchronize()

    def max(self, v):
        """the job's time of a per-rank time: the slowest rank"""
        if self.dist is None:
            return v
        import torch
        t = torch.tensor([v], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


# ------------------------------------------------------------------------------- native arm
def native_arm(args):
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    ranks = Ranks("nccl", "cuda")
    rank, world = ranks.rank, ranks.world

    from feat3_b200.solver import MultiGrid
    from feat3_b200 import _lib
    import ctypes as C

    level = args.level
    k = coefficient(level, args.seed + rank)
    t0 = time.time()
    mg = MultiGrid.structured(3, 1, level, 1, k)
    setup_s = time.time() - t0
    n = mg.ndofs()
    rhs = mg.assemble_rhs("one")
    common = dict(outer="pcg", nu=2, omega_jac=0.5, coarse="direct", tol=1e-8)

    barrier = ranks.barrier
    max_over_ranks = ranks.max

    def run_form(prec, steps, warmup, host=False, fmt="stencil"):
        mg.configure(precision=prec, format=fmt, **common)
        hb = torch.empty(n, dtype=torch.float64).pin_memory().numpy()
        hx = torch.zeros(n, dtype=torch.float64).pin_memory().numpy()
        hb[:] = rhs.cpu().numpy()
        res = None
        for _ in range(warmup):
            res = mg.solve_host(hb, hx, zero_init=True) if host else mg.solve(rhs)
        barrier()
        times, launches, iters = [], 0, []
        t_wall = time.time()
        for _ in range(steps):
            if host:
                # the user's call: rhs in pinned host memory, solve from zero, solution back to host
                res = mg.solve_host(hb, hx, zero_init=True)
            else:
                res = mg.solve(rhs)
            times.append(res["solve_ms"] / 1e3)
            launches += res["kernel_launches"]
            iters.append(res["iters"])
        barrier()
        wall = time.time() - t_wall
        return res, times, launches, iters, wall

    if args.only:
        prec, _, fmt = args.only.partition("-")
        r, t, l, it, _ = run_form(prec, args.steps, args.warmup, fmt=fmt or "stencil")
        if rank == 0:
            print(json.dumps({"form": args.only, "time_s": float(np.median(t)), "iters": it[-1], "launches": l,
                              "dofs": n, "level": level}))
        ranks.close()
        mg.close()
        return 0
    # --- FP64 forms: the drop-in (SELL-C-sigma, CSR transfers), the stencil storage, matrix-free
    r64, t64, _, it64, _ = run_form("f64", args.steps, args.warmup, fmt="sell")
    u64 = r64["u"].clone()
    r64s, t64s, _, it64s, _ = run_form("f64", args.steps, args.warmup, fmt="stencil")
    r64m, t64m, _, it64m, _ = run_form("f64", args.steps, args.warmup, fmt=HEAD_FMT)
    # --- mixed forms: FP16 stencil storage, and the headline (matrix-free FP32 V-cycle)
    rmxs, tmxs, _, itmxs, _ = run_form("f16", args.steps, args.warmup, fmt="stencil")
    err_s = float(torch.linalg.norm(rmxs["u"] - u64) / torch.linalg.norm(u64))
    # the reference's own mixed composition: FP64 Richardson around ConvertPrecond(FP32 MG)
    common_r = dict(common, outer="richardson")
    mg.configure(precision=HEAD_PREC, format=HEAD_FMT, **common_r)
    rmr = None
    for _ in range(max(1, args.warmup)):
        rmr = mg.solve(rhs)
    barrier()
    tmr = []
    for _ in range(max(1, args.steps // 2)):
        rmr = mg.solve(rhs)
        tmr.append(rmr["solve_ms"] / 1e3)
    err_r = float(torch.linalg.norm(rmr["u"] - u64) / torch.linalg.norm(u64))
    clk = ClockSampler(local)
    clk.start()
    rmx, tmx, lmx, itmx, wall = run_form(HEAD_PREC, args.steps, args.warmup, fmt=HEAD_FMT)
    clocks = clk.stop()
    umx = rmx["u"]
    err = float(torch.linalg.norm(umx - u64) / torch.linalg.norm(u64))
    # --- one adjoint gradient solve on the same hierarchy (transposed MG-PCG + element gradient):
    # J = 1/2 ||u - u_t||^2 with u_t = u + N(0, (1e-2 max|u|)^2) noise (seed 23)
    u_host = umx.cpu().numpy()
    noise = np.random.default_rng(23).standard_normal(n)
    u_target = torch.tensor(u_host + 1e-2 * np.abs(u_host).max() * noise, device="cuda")
    adj = {}
    for prec in (HEAD_PREC, "f64"):
        mg.configure(precision=prec, format=HEAD_FMT, **common)
        mg.adjoint_grad(umx, u_target)  # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        lam, grad, ainfo = mg.adjoint_grad(umx, u_target)
        torch.cuda.synchronize()
        adj[prec] = {"time_s": time.perf_counter() - t0, "solve_s": ainfo["solve_ms"] / 1e3, "iters": ainfo["iters"],
                     "status": ainfo["status"], "grad_norm": float(torch.linalg.norm(grad))}
        adj[prec + "_grad"] = grad
    adj_err = float(torch.linalg.norm(adj[HEAD_PREC + "_grad"] - adj["f64_grad"]) / torch.linalg.norm(adj["f64_grad"]))
    adjoint = {"mixed": adj[HEAD_PREC], "fp64": adj["f64"], "grad_rel_diff_mixed_vs_fp64": adj_err,
               "objective": "J = 1/2 ||u - u_t||^2, u_t = u + N(0, (1e-2 max|u|)^2) noise"}
    # --- end to end through the host-buffer entry point
    re2e, te2e, _, _, _ = run_form(HEAD_PREC, max(2, args.steps // 2), 1, host=True, fmt=HEAD_FMT)

    # --- roofline of the finest-level operator kernels (CUDA events on the solver stream)
    nnz = mg.nnz(0)
    ne = (2 ** level) ** 3
    rf = {}
    for name, prec, fmt, which in (
            ("matfree_jacobi_f32", "f32", "matfree", 0), ("matfree_pcgq_f64", "f64", "matfree", 2),
            ("matfree_pcgq_p32", "f32", "matfree", 3),
            ("stencil_jacobi_f16", "f16", "stencil", 0), ("stencil_jacobi_f64", "f64", "stencil", 0),
            ("stencil_pcgq_f64", "f64", "stencil", 2), ("sell_jacobi_f64", "f64", "sell", 0),
            ("sell_pcgq_f64", "f64", "sell", 2), ("sell_jacobi_f16", "f16", "sell", 0)):
        mg.configure(precision=prec, format=fmt, **common)
        ms = C.c_double(0.0)
        _lib.call("fb_mg_time_spmv", mg.h, 0, which, {"f64": 0, "f32": 1, "f16": 2}[prec], 20, C.byref(ms))
        sx = 8 if prec == "f64" else 4                    # vector element size
        vec = n * sx * (3 if which == 0 else 1)           # Jacobi: rhs, invd, out; PCG q: q (p is the input)
        if which == 0 and fmt == "matfree" and prec == "f32":
            vec = n * sx * 2                              # the FP32 tiled step forms invd from the coefficients
        if which == 3:                                    # FP32 direction in, FP64 q out, FP64 coefficients
            vec = n * 8
        if fmt == "matfree":
            mat = ne * (8 if which == 3 else sx)          # per-cell coefficient instead of a matrix
        else:
            sv = {"f64": 8, "f32": 4, "f16": 2}[prec]
            mat = nnz * (sv + (4 if fmt == "sell" else 0))  # values (+ 32-bit column indices)
        alg = mat + n * sx + vec + n / 8                  # + the input vector once + the filter mask
        rf[name] = {"ms": ms.value, "bytes": alg, "GBps": alg / (ms.value * 1e-3) / 1e9}
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    dom = rf[HEAD_KERNEL]

    t_mixed = max_over_ranks(float(np.median(tmx)))
    t_mixed_s = max_over_ranks(float(np.median(tmxs)))
    t_mixed_r = max_over_ranks(float(np.median(tmr)))
    t_fp64 = max_over_ranks(float(np.median(t64)))
    t_fp64s = max_over_ranks(float(np.median(t64s)))
    t_fp64m = max_over_ranks(float(np.median(t64m)))
    t_e2e = max_over_ranks(float(np.median(te2e)))
    cpu, oracle_err, refrun_err = None, None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, oref = oracle_baseline(args, k, n)
        uo = oref["u"]
        forms = {"mixed": umx, "fp64": u64, "fp64_matfree": r64m["u"], "mixed_f16_stencil": rmxs["u"],
                 "mixed_richardson": rmr["u"]}
        host = {name: u.cpu().numpy() for name, u in forms.items()}
        oracle_err = {name: float(np.linalg.norm(u - uo) / np.linalg.norm(uo)) for name, u in host.items()}
        oracle_err["oracle_iters"] = oref["iters"]
        samples = reference_run_samples(args)
        if samples is not None:
            stride, us, ref_iters = samples
            refrun_err = {name: float(np.linalg.norm(host[name][::stride] - us) / np.linalg.norm(us))
                          for name in ("mixed", "fp64", "fp64_matfree")}
            refrun_err["oracle"] = float(np.linalg.norm(uo[::stride] - us) / np.linalg.norm(us))
            refrun_err["reference_iters"] = ref_iters
            refrun_err["what"] = (f"relative error at every {stride}th DOF against the reference's own 257^3 solve "
                                  "(tests/golden/ref_c5_full_q1_3d_L8.npz, oracle/_ref/feat_ref)")
    if rank == 0:
        line = {
            "metric": METRIC, "value": t_mixed, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_mixed, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 outer PCG / f32 V-cycle (matrix-free operator)", "data": "synthetic",
            "config": bench_config(args, world),
            "err_vs_oracle": oracle_err,
            "err_vs_reference_run": refrun_err,
            "mixed": {"time_s": t_mixed, "iters": itmx[-1], "err_vs_fp64": err,
                      "dof_it_per_s": n * itmx[-1] / t_mixed, "final_rel_residual": rmx["hist"][-1] / rmx["hist"][0],
                      "storage": "matrix-free Q1 operator from per-cell coefficients + matrix-free Q1 transfers"},
            "mixed_richardson": {"time_s": t_mixed_r, "iters": rmr["iters"],
                                 "err_vs_fp64": err_r, "status": rmr["status"],
                                 "outer": "FP64 Richardson around ConvertPrecond(FP32 matrix-free MG)"},
            "mixed_f16_stencil": {"time_s": t_mixed_s, "iters": itmxs[-1], "err_vs_fp64": err_s,
                                  "storage": "FP16 stencil values (SELL-32, implicit columns) + matrix-free transfers"},
            "fp64": {"time_s": t_fp64, "iters": it64[-1], "dof_it_per_s": n * it64[-1] / t_fp64,
                     "final_rel_residual": r64["hist"][-1] / r64["hist"][0],
                     "storage": "SELL-C-sigma (C=32, 32-bit column indices) + CSR transfers (drop-in form)"},
            "fp64_stencil": {"time_s": t_fp64s, "iters": it64s[-1], "dof_it_per_s": n * it64s[-1] / t_fp64s,
                             "storage": "SELL-32 with implicit stencil columns + matrix-free Q1 transfers"},
            "fp64_matfree": {"time_s": t_fp64m, "iters": it64m[-1], "dof_it_per_s": n * it64m[-1] / t_fp64m,
                             "storage": "matrix-free Q1 operator + matrix-free Q1 transfers"},
            "speedup_mixed_vs_fp64": t_fp64 / t_mixed,
            "speedup_mixed_vs_fp64_same_storage": t_fp64m / t_mixed,
            "roofline": {"bound": "hbm", "achieved": dom["GBps"], "peak": peak, "unit": "GB/s",
                         "frac": dom["GBps"] / peak, "traffic": HEAD_KERNEL_DRAM_BYTES,
                         "traffic_source": "ncu capture of the kernel alone (design notes: measurement)",
                         "kernel": HEAD_KERNEL_NAME, "kernels": rf,
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (burst copy)" if peaks else "fallback 6650"},
            "adjoint": adjoint,
            "cpu_baseline": cpu,
            "e2e": {"value": t_e2e, "unit": "s", "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n,
                    "entry_point": "fb_mg_solve_host_zero (pinned host rhs in, solution out, zero initial guess)"},
            "gpu_launches": lmx,
            "gpu_launches_per_step": lmx // max(1, args.steps),
            "clocks": clocks, "setup_s": setup_s,
            "wall_s_mixed_steps": wall,
        }
        print(json.dumps(line))
    ranks.close()
    mg.close()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    return native_arm(args)


if __name__ == "__main__":
    sys.exit(main())
