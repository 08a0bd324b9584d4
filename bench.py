#!/usr/bin/env python
"""Benchmark of the matrix-free p = 2 B-spline elasticity PCG on B200.

Workload (default): the SIMP cantilever on 128 x 64 x 64 elements (1,698,840 DOF), box
[0,2]x[0,1]x[0,1], densities i.i.d. U[0.01,1] smoothed by a 3x3x3 box filter (seeded PCG64),
E0 = 1, E_min = 1e-9, nu = 0.3, SIMP penalty 3, x = 0 clamped, unit downward traction on x = 2.
One step = one Jacobi-PCG solve to relative residual 1e-8 from x = 0, in the mixed-precision form
(tensor-core split-TF32 FP32 iterations with FP64 residual replacement) by default; the plain FP64
solve of the same system is timed beside it (config.vs_fp64).  --mode fp64 times the plain solve only.

value    = DOF * iterations / device seconds of the solve, inputs resident in HBM (CUDA events on
           the solver's stream, L2 flushed between steps), summed over ranks (replicas).
e2e      = the same metric through the host-pointer C ABI call (icc_op_update_scale +
           icc_pcg_solve): H2D of the step's scale and load, D2H of the solution, inside the timing.
roofline = the dominant kernel: for the mixed form the tensor-core brick apply, algorithmic
           2*81*81 flops per element (the three split-TF32 products are credited once) over its
           mean CUDA-event duration against this run's cuBLAS TF32 GEMM (the MMA work it executes,
           three products padded to 96 x 96, is reported beside it as executed_flops); for
           --mode fp64 the FP64 DMMA brick apply, 2*81*81 flops per element against this run's
           cuBLAS DGEMM.  roofline.iteration: the whole PCG iteration against HBM bandwidth,
           algorithmic bytes per iteration over ms_per_step / iterations.
cpu_baseline / --impl reference = the oracle (C restatement of the reference's CPU path:
           element-loop operator with OpenMP, serial PCG vector loops) on the host cores, a
           bounded number of PCG iterations of the same workload.
"""
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

METRIC = "PCG time-to-1e-8 & DOF·iter/s, mixed vs FP64 on 1 B200; err vs FP64 oracle"
UNIT = "DOF*iter/s"
TOL = 1e-8
SEED = 2026
WORKLOADS = {
    "cantilever128": dict(nel=(128, 64, 64), smooth=True),
    "cantilever24": dict(nel=(24, 16, 12), smooth=False),
    "cantilever256": dict(nel=(256, 128, 128), smooth=True),
    # the immersed case: unit cube minus three r = 0.25 cylinders, 96^3 cells, Jacobi clamp 1e-6
    "cylinders96": dict(kind="cylinders", n=96),
    # 64 cantilever designs 2k x k x k, k ~ U{8..48} from the seed, each with its own densities:
    # one batched mixed-precision call against 64 sequential FP64 solves
    "batched64": dict(kind="batched", count=64, kmin=8, kmax=48),
    # multi-RHS topology loop: 256 x 128 x 128 on [0,2]x[0,1]x[0,1], 4 tip load cases, SIMP p = 3,
    # volfrac 0.3, filter radius 1.5 cells, warm starts; --steps design iterations, mixed vs FP64
    "topopt256": dict(kind="topopt", nel=(256, 128, 128)),
}


def make_problem(W, wl, seed):
    if wl.get("kind") == "cylinders":
        return W.cylinders(wl["n"])
    return W.cantilever(wl["nel"], smooth=wl["smooth"], seed=seed)


def workload_label(prob, wl):
    """The workload name both arms print (the same inputs: make_problem with the same seed)."""
    if wl.get("kind") == "cylinders":
        return f"{prob.name} immersed cube minus three cylinders"
    return f"{prob.name} SIMP cantilever, " + ("smoothed densities" if wl.get("smooth") else "i.i.d. densities")


def hbm_peak():
    """HBM bandwidth denominator (GB/s): MEASURED_PEAKS.json's copy bandwidth when present, else the
    pool's earlier measurement (6,650 GB/s)."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        for k in ("hbm_gbs", "hbm_GBs", "hbm"):
            if k in d and float(d[k]) > 0:
                return float(d[k]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        pass
    return 6650.0, "fallback 6,650 GB/s (MEASURED_PEAKS.json absent)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cantilever128", choices=sorted(WORKLOADS))
    ap.add_argument("--mode", default="mixed", choices=["fp64", "mixed"],
                    help="mixed: the tensor-core solve, timed beside the plain FP64 solve; fp64: the plain solve only")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU baseline sample budget")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-ref-solution", action="store_true", help="skip the tight FP64 error reference")
    ap.add_argument("--solves-only", action="store_true",
                    help="only run the warmup + timed solves of the chosen mode (for profiler launch lists)")
    ap.add_argument("--kernel-only", action="store_true",
                    help="only run warmup + steps operator applies (for profiler captures)")
    ap.add_argument("--delta", type=float, default=0.0,
                    help="mixed form: FP64 residual replacement when the FP32 residual fell by this factor")
    ap.add_argument("--check-every", type=int, default=32, help="PCG iterations per device batch")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def gemm_peak(torch, dev, dtype, tf32=False):
    """Measured tensor-core peak of this GPU for one GEMM type: cuBLAS through torch.matmul, 8192^3,
    best of 5 (TFLOP/s).  float64 -> DGEMM; float32 with tf32=True -> TF32 tensor cores."""
    n = 8192
    old = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = tf32
    a = torch.randn(n, n, dtype=dtype, device=dev)
    b = torch.randn(n, n, dtype=dtype, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    torch.backends.cuda.matmul.allow_tf32 = old
    del a, b
    torch.cuda.empty_cache()
    return best


def cpu_sample_csr(problem, oracle_mod):
    """The reference's own CPU path, restated in C by the oracle: AssemblyPattern CSR assembly
    (rust/src/sparse.rs:128-175), then Jacobi-PCG to 1e-8 with the row-parallel CSR SpMV
    (rust/src/sparse.rs:60-68) inside the masked closure (rust/src/topopt_iga.rs:151-159)."""
    O = oracle_mod
    osp = O.Space(problem.bounds, problem.nel, 2)
    lam, mu = O.lame(1.0, 0.3)
    types, tid, _ = osp.element_matrices(lam, mu)
    b = np.where(problem.free_mask > 0, problem.force, 0.0)
    t0 = time.perf_counter()
    k = O.Csr.assemble(osp, types, tid, problem.scale)
    t_asm = time.perf_counter() - t0
    diag = np.maximum(k.diagonal(), 1e-12)
    t0 = time.perf_counter()
    x, it, res = k.pcg(b, diag, 20 * problem.ndof, TOL, problem.free_mask, 1)
    dt = time.perf_counter() - t0
    return {"value": problem.ndof * it / dt, "unit": UNIT, "cores": O.num_threads(), "kind": "port",
            "sample": f"full solve of {problem.name} ({problem.ndof} DOF) to {TOL:g}: CSR assembly "
                      f"{t_asm * 1e3:.1f} ms (not in value), Jacobi-PCG {it} iterations {dt * 1e3:.1f} ms with the "
                      f"row-parallel CSR SpMV (OpenMP) and serial vector loops",
            "seconds": dt, "assembly_ms": t_asm * 1e3, "iterations": it}


def cpu_sample(problem, seconds, oracle_mod):
    """Oracle (reference CPU path restated in C) PCG iterations on the host for ~seconds.  The small
    cantilever (19,656 DOF) runs the reference's assembled path to convergence; larger problems, whose
    CSR does not fit in host memory, run a bounded number of iterations of the matrix-free element loop."""
    O = oracle_mod
    if problem.ndof <= 200000:
        return cpu_sample_csr(problem, O)
    osp = O.Space(problem.bounds, problem.nel, 2)
    lam, mu = O.lame(1.0, 0.3)
    types, tid, _ = osp.element_matrices(lam, mu)
    b = np.where(problem.free_mask > 0, problem.force, 0.0)
    diag = np.maximum(O.mf_diagonal(osp, types, tid, problem.scale), 1e-12)
    t0 = time.perf_counter()
    O.pcg_mf(osp, types, tid, problem.scale, b, diag, 1, 0.0, problem.free_mask, 1)
    t_one = time.perf_counter() - t0
    iters = int(max(2, min(500, seconds / max(t_one, 1e-6))))
    t0 = time.perf_counter()
    x, it, res = O.pcg_mf(osp, types, tid, problem.scale, b, diag, iters, 0.0, problem.free_mask, 1)
    dt = time.perf_counter() - t0
    return {"value": problem.ndof * it / dt, "unit": UNIT, "cores": O.num_threads(), "kind": "port",
            "sample": f"{it} Jacobi-PCG iterations of {problem.name} ({problem.ndof} DOF) with the oracle's "
                      f"matrix-free element-loop operator (OpenMP) and serial vector loops, {dt:.1f} s",
            "seconds": dt}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from immersed_catmull_clark_b200 import workloads as W
    from oracle import oracle as O
    O.build()
    wl = WORKLOADS[args.workload]
    prob = make_problem(W, wl, SEED)
    per_step = max(2.0, min(10.0, args.cpu_seconds))
    vals = []
    for i in range(args.warmup + args.steps):
        s = cpu_sample(prob, per_step, O)
        if i >= args.warmup:
            vals.append(s)
    value = float(np.mean([s["value"] for s in vals]))
    ms = float(np.mean([s["seconds"] for s in vals]) * 1e3)
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
           "config": {"workload": workload_label(prob, wl), "ndof": prob.ndof, "tol": TOL, "seed": SEED},
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": vals[0]["cores"], "kind": "port",
                            "sample": vals[0]["sample"]},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def run_batched(args, wl):
    """The batched-designs configuration: host-timed (the batched call is synchronous and spans many
    streams), inputs and outputs in host memory, so the number is end to end."""
    import torch
    import immersed_catmull_clark_b200 as icc
    from immersed_catmull_clark_b200 import workloads as W

    ks, probs = W.batched_designs(wl["count"], wl["kmin"], wl["kmax"], SEED)
    lam, mu = icc.lame(W.E0, W.NU)
    ops, bs, ndofs = [], [], []
    for p in probs:
        sp = icc.SpaceBox(p.bounds, p.nel, 2)
        em = icc.elasticity_element_matrices(sp, lam, mu)
        ops.append(icc.MatrixFreeOperator(sp, em, p.scale, p.free_mask, icc.MASK_ZERO))
        bs.append(W.rhs_masked(p))
        ndofs.append(sp.ndof)
    ndofs = np.array(ndofs)

    def timed(fn, steps):
        ts, out = [], None
        for _ in range(steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = fn()
            torch.cuda.synchronize()
            ts.append((time.perf_counter() - t0) * 1e3)
        return ts, out

    batched = lambda: icc.solve_batched(ops, bs, tol=TOL, max_iter=100000, precision=icc.MIXED)
    for _ in range(args.warmup):
        batched()
    with ClockSampler(torch.cuda.current_device()) as clk:
        ms, (xs, its, res, st) = timed(batched, args.steps)
    work = float(np.sum(ndofs * its))
    value = work / (np.mean(ms) * 1e-3)

    def sequential(precision):
        out = []
        for op, b, n in zip(ops, bs, ndofs):
            x, it, r = icc.PcgSolver(100000, TOL, precision=precision).solve(int(n), b, None, op)
            out.append((x, it))
        return out
    sequential(icc.FP64)
    ms64, seq = timed(lambda: sequential(icc.FP64), 1)
    err = max(float(np.linalg.norm(x - xr) / np.linalg.norm(xr)) for x, (xr, _) in zip(xs, seq))
    # controls that separate the gain of batching from the gain of precision: the same 64 mixed
    # solves one after another, and the 64 FP64 solves as one batched call
    sequential(icc.MIXED)
    ms_seq_mixed, _ = timed(lambda: sequential(icc.MIXED), 1)
    batched64 = lambda: icc.solve_batched(ops, bs, tol=TOL, max_iter=100000, precision=icc.FP64)
    batched64()
    ms_bat64, (_, _, _, st64) = timed(batched64, 1)
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": float(np.mean(ms)), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "tf32x3+f32+f64", "data": "synthetic",
           "config": {"workload": f"{wl['count']} cantilever designs 2k x k x k, k ~ U{{{wl['kmin']}..{wl['kmax']}}}",
                      "total_ndof": int(ndofs.sum()), "ks": [int(k) for k in ks], "tol": TOL, "seed": SEED,
                      "mode": "batched mixed", "iterations_total": int(np.sum(its)),
                      "all_converged": bool(np.all(st == icc.ICC_OK)), "time_to_tol_ms": ms,
                      "vs_sequential_fp64": {"sequential_fp64_ms": ms64[0],
                                             "speedup": ms64[0] / float(np.mean(ms)),
                                             "max_disp_rel_l2_vs_fp64_1e-8": err},
                      "controls": {"sequential_mixed_ms": ms_seq_mixed[0],
                                   "batching_gain_mixed": ms_seq_mixed[0] / float(np.mean(ms)),
                                   "batched_fp64_ms": ms_bat64[0],
                                   "batched_fp64_all_converged": bool(np.all(st64 == icc.ICC_OK)),
                                   "precision_gain_batched": ms_bat64[0] / float(np.mean(ms))}},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": int(8 * ndofs.sum()),
                   "d2h_bytes_per_step": int(8 * ndofs.sum())},
           "clocks": clk.summary()}
    print(json.dumps(out), flush=True)


def run_topopt(args, wl):
    """The multi-RHS topology-optimisation configuration: --steps design iterations of the device
    SIMP loop with the four tip load cases, mixed-precision state solves against FP64 ones."""
    import torch
    import immersed_catmull_clark_b200 as icc
    from immersed_catmull_clark_b200 import workloads as W

    nel = wl["nel"]
    loads = W.tip_load_cases(nel, size=(2.0, 1.0, 1.0))
    ndof = loads.shape[1]
    res = {}
    with ClockSampler(torch.cuda.current_device()) as clk:
        for name, prec in (("mixed", icc.MIXED), ("fp64", icc.FP64)):
            t = icc.CantileverTopOpt(nel, size=(2.0, 1.0, 1.0), volfrac=0.3, penal=3.0, rmin=1.5, emin=1e-9,
                                     pcg_tol=TOL, precision=prec)
            t.set_loads(loads)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            h = t.run(args.steps)
            torch.cuda.synchronize()
            res[name] = (time.perf_counter() - t0, h)
            del t
    tm, hm = res["mixed"]
    tf, hf = res["fp64"]
    drift = (np.abs(hm.compliance - hf.compliance) / hf.compliance).tolist()
    work = float(ndof * np.sum(hm.pcg_iterations))
    out = {"metric": METRIC, "value": work / tm, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": 0,
           "ms_per_step": tm / args.steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "tf32x3+f32+f64", "data": "synthetic",
           "config": {"workload": f"SIMP cantilever {nel[0]}x{nel[1]}x{nel[2]}, 4 tip load cases, warm starts",
                      "ndof": ndof, "design_iterations": args.steps, "tol": TOL,
                      "mixed": {"s_per_design_iteration": tm / args.steps, "compliance": hm.compliance.tolist(),
                                "pcg_iterations": hm.pcg_iterations.tolist()},
                      "fp64": {"s_per_design_iteration": tf / args.steps, "compliance": hf.compliance.tolist(),
                               "pcg_iterations": hf.pcg_iterations.tolist()},
                      "compliance_drift_mixed_vs_fp64": drift,
                      "density_max_diff": float(np.abs(hm.density - hf.density).max()),
                      "speedup_per_design_iteration": tf / tm,
                      "timing": "host clock around each synchronous run (state solves, energies, filter, OC)"},
           "e2e": {"value": work / tm, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "clocks": clk.summary()}
    print(json.dumps(out), flush=True)


def aggregate_replicas(dist, torch, device, t_ms, work, e2e_value):
    """Replicas on N GPUs: the job's time is the slowest rank's (max over ranks), its throughput
    the work of all ranks over that time; e2e throughputs add.  Returns (t_ms, value, e2e)."""
    t = torch.tensor([t_ms, work, e2e_value], dtype=torch.float64, device=device)
    mx = t.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    sm = t.clone()
    dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    t_all = float(mx[0])
    return t_all, float(sm[1]) / (t_all * 1e-3), float(sm[2])


def run_ours(args):
    import torch
    import torch.distributed as dist

    rank, world, local = dist_env()
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if WORKLOADS[args.workload].get("kind") in ("batched", "topopt"):
        if rank == 0:
            kind = WORKLOADS[args.workload]["kind"]
            (run_batched if kind == "batched" else run_topopt)(args, WORKLOADS[args.workload])
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return

    import immersed_catmull_clark_b200 as icc
    from immersed_catmull_clark_b200 import workloads as W

    wl = WORKLOADS[args.workload]
    prob = make_problem(W, wl, SEED + rank)
    sp = icc.SpaceBox(prob.bounds, prob.nel, 2)
    lam, mu = icc.lame(W.E0, W.NU)
    em = icc.elasticity_element_matrices(sp, lam, mu)
    op = icc.MatrixFreeOperator(sp, em, prob.scale, prob.free_mask, icc.MASK_ZERO)
    n = sp.ndof
    stream = torch.cuda.ExternalStream(op.stream, device=dev)
    b_host = W.rhs_masked(prob)
    b_dev = torch.from_numpy(b_host).to(dev)
    # Jacobi diagonal: the operator's own (0) for the cantilever; clamped at 1e-6 for the immersed
    # case as the reference does (rust/src/immersed.rs:555)
    diag_host, diag_ptr = None, 0
    if wl.get("kind") == "cylinders":
        diag_host = np.maximum(op.diagonal(), 1e-6)
        diag_t = torch.from_numpy(diag_host).to(dev)
        diag_ptr = diag_t.data_ptr()
    x_dev = torch.zeros(n, dtype=torch.float64, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2
    precision = icc.MIXED if args.mode == "mixed" else icc.FP64
    # iteration cap: 20 n as the reference's solve_state, but at most 100k for the benchmark
    solver = icc.PcgSolver(min(20 * n, 100000), TOL, precision=precision, check_every=args.check_every,
                           inner_tol=args.delta)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    if args.kernel_only:
        vdt = torch.float32 if args.mode == "mixed" else torch.float64
        apply = op.matvec_f32_dev if args.mode == "mixed" else op.matvec_dev
        y_dev = torch.empty(n, dtype=vdt, device=dev)
        p_dev = torch.from_numpy(np.random.default_rng(1).standard_normal(n)).to(dev).to(vdt)
        for _ in range(args.warmup):
            apply(p_dev.data_ptr(), y_dev.data_ptr())
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
        for _ in range(args.steps):
            apply(p_dev.data_ptr(), y_dev.data_ptr())
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        if rank == 0:
            print(json.dumps({"kernel_only": True, "workload": prob.name, "ndof": n,
                              "ms_per_apply": e0.elapsed_time(e1) / args.steps}), flush=True)
        return

    def timed_solves(slv, steps, warmup, x_out):
        for _ in range(warmup):
            slv.solve_dev(n, b_dev.data_ptr(), diag_ptr, x_out.data_ptr(), op)
        barrier()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        iters, launches = [], 0
        for i in range(steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                ev[i][0].record(stream)
            it, res = slv.solve_dev(n, b_dev.data_ptr(), diag_ptr, x_out.data_ptr(), op)
            with torch.cuda.stream(stream):
                ev[i][1].record(stream)
            iters.append(int(it))
            launches += op.last_solve_info().kernel_launches
        barrier()
        return [a_.elapsed_time(b_) for a_, b_ in ev], iters, launches, op.last_solve_info()

    with ClockSampler(torch.cuda.current_device()) as clk:
        ms_steps, iters, launches, info = timed_solves(solver, args.steps, args.warmup, x_dev)
    if args.solves_only:
        if rank == 0:
            print(json.dumps({"solves_only": True, "workload": prob.name, "mode": args.mode, "iterations": iters,
                              "time_to_tol_ms": ms_steps}), flush=True)
        return
    t_ms = float(np.sum(ms_steps))
    local_value = n * float(np.sum(iters)) / (t_ms * 1e-3)

    # the plain FP64 solve of the same system, timed the same way, for the mixed/FP64 comparison
    cmp = None
    if precision == icc.MIXED:
        x64_dev = torch.zeros_like(x_dev)
        s64 = icc.PcgSolver(min(20 * n, 100000), TOL, precision=icc.FP64, check_every=args.check_every)
        k64 = max(1, min(args.steps, 2))
        ms64, it64, _, _ = timed_solves(s64, k64, 1, x64_dev)
        t_mixed, t_fp64 = float(np.mean(ms_steps)), float(np.mean(ms64))
        cmp = {"fp64_time_to_tol_ms": t_fp64, "fp64_iterations": it64, "mixed_time_to_tol_ms": t_mixed,
               "mixed_iterations": iters, "speedup_time_to_tol": t_fp64 / t_mixed}

    # roofline of the dominant kernel, timed on the solver's stream
    flops_el = 2.0 * 81 * 81
    nbricks = int(np.prod([-(-d // b) for d, b in zip(sp.nel_dir, (8, 4, 4))]))
    executed = None
    if precision == icc.MIXED:
        y32 = torch.empty(n, dtype=torch.float32, device=dev)
        p32 = torch.from_numpy(np.random.default_rng(1).standard_normal(n)).to(dev).to(torch.float32)
        contract_ms, gather_ms = op.profile_apply_f32(p32.data_ptr(), y32.data_ptr(), 20)
        flops = flops_el * sp.nel   # algorithmic: one 81 x 81 product per element
        # executed MMA work: three split products of 128 x 96 x 96 per brick of 8 x 4 x 4 elements
        executed = 3 * 2.0 * 128 * 96 * 96 * nbricks
        peak = gemm_peak(torch, dev, torch.float32, tf32=True)
        kname, tkey = "apply_tc_kernel (tcgen05 kind::tf32, 3-term split)", "apply_tc_kernel"
        peak_src = ("measured in this run: cuBLAS TF32 GEMM (torch.matmul float32 with TF32 tensor cores, 8192^3); "
                    "MEASURED_PEAKS.json has no TF32 figure")
    else:
        y_dev = torch.empty_like(x_dev)
        p_dev = torch.from_numpy(np.random.default_rng(1).standard_normal(n)).to(dev)
        contract_ms, gather_ms = op.profile_apply(p_dev.data_ptr(), y_dev.data_ptr(), 20)
        flops = flops_el * sp.nel
        executed = 2.0 * 88 * 84 * sp.nel   # DMMA tiles: 81 padded to 84 (trial) x 88 (test)
        peak = gemm_peak(torch, dev, torch.float64)
        kname, tkey = "apply_f64_kernel (FP64 DMMA)", "apply_f64_kernel"
        peak_src = ("measured in this run: cuBLAS DGEMM (torch.matmul float64 8192^3); "
                    "MEASURED_PEAKS.json has no FP64 figure")
    achieved = flops / (contract_ms * 1e-3) / 1e12
    traffic, traffic_src = None, None
    tpath = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tpath):
        try:
            t = json.load(open(tpath)).get(tkey, {}).get(args.workload)
            traffic = None if t is None else float(t)
            traffic_src = ("dram__bytes_read.sum + dram__bytes_write.sum of one launch from an earlier ncu capture "
                           "of the same kernel and workload, recorded in profiles/ncu_traffic.json (not this run)")
        except Exception:
            traffic = None
    # the whole iteration against HBM: the apply reads p and s_e and writes Ap, the vector step
    # reads x, r, p, Ap, D^-1 and writes x, r, p (FP32 for the mixed form, FP64 for the plain one)
    vb = 4 if precision == icc.MIXED else 8
    iter_bytes = 5 * vb * n + vb * sp.nel + 3 * vb * n
    ms_per_iter = float(np.sum(ms_steps)) / max(1, int(np.sum(iters)))
    hbm, hbm_src = hbm_peak()
    iter_gbs = iter_bytes / (ms_per_iter * 1e-3) / 1e9

    # end to end through the host-pointer C ABI call (pinned host buffers)
    b_pin = torch.from_numpy(b_host).pin_memory()
    s_pin = torch.from_numpy(prob.scale.copy()).pin_memory()
    x_pin = torch.empty(n, dtype=torch.float64).pin_memory()
    e2e_steps = max(1, min(args.steps, 2))
    barrier()
    e2e_ms, e2e_it = 0.0, 0
    for _ in range(e2e_steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            flush.zero_()
            e0.record(stream)
        op.update_scale(s_pin.numpy())
        it, res = solver.solve_host_ptr(n, b_pin.numpy(), diag_host, x_pin.numpy(), op)
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        e2e_ms += e0.elapsed_time(e1)
        e2e_it += it
    e2e_local = n * e2e_it / (e2e_ms * 1e-3)

    # accuracy against a tight FP64 solution (FP64 device PCG at 1e-12)
    err = {}
    if not args.no_ref_solution:
        x_ref = torch.zeros_like(x_dev)
        ref_solver = icc.PcgSolver(40 * n, 1e-12, precision=icc.FP64)
        it_ref, res_ref = ref_solver.solve_dev(n, b_dev.data_ptr(), diag_ptr, x_ref.data_ptr(), op)
        xr, xs = x_ref.cpu().numpy(), x_dev.cpu().numpy()
        c_ref, c = float(prob.force @ xr), float(prob.force @ xs)
        err = {"disp_rel_l2": float(np.linalg.norm(xs - xr) / np.linalg.norm(xr)),
               "compliance_rel": abs(c - c_ref) / abs(c_ref), "ref": f"FP64 device PCG to {res_ref:.1e} ({it_ref} it)"}

    # max over ranks of time, sum of throughput
    if world > 1:
        t_ms_all, value, e2e_value = aggregate_replicas(dist, torch, dev, t_ms, n * float(np.sum(iters)), e2e_local)
    else:
        t_ms_all, value, e2e_value = t_ms, local_value, e2e_local

    cpu = None
    if rank == 0 and not args.no_cpu:
        from oracle import oracle as O
        O.build()
        cpu = cpu_sample(prob, args.cpu_seconds, O)
        cpu.pop("seconds", None)

    if rank == 0:
        cfg = {"workload": workload_label(prob, wl),
               "ndof": n, "nel": sp.nel, "tol": TOL, "seed": SEED, "mode": args.mode,
               "iterations": iters, "time_to_tol_ms": ms_steps,
               "l2": "flushed between steps (256 MB write)", "parallelism": f"replicas x{world}"}
        if cmp:
            cfg["vs_fp64"] = cmp
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": t_ms_all / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f64" if precision == icc.FP64 else "tf32x3+f32+f64",
               "data": "synthetic", "config": cfg,
               "roofline": {"bound": "tensor", "kernel": kname, "achieved": achieved, "peak": peak,
                            "unit": "TFLOP/s", "frac": achieved / peak, "frac_of": "measured", "traffic": traffic,
                            "traffic_source": traffic_src,
                            "algorithmic_flops_per_launch": flops, "executed_flops_per_launch": executed,
                            "executed_tflops": executed / (contract_ms * 1e-3) / 1e12,
                            "launch_ms": contract_ms, "node_sum_kernel_ms": gather_ms, "peak_source": peak_src,
                            "iteration": {"bound": "hbm", "algorithmic_bytes": iter_bytes, "ms": ms_per_iter,
                                          "achieved_gbs": iter_gbs, "peak_gbs": hbm, "frac": iter_gbs / hbm,
                                          "peak_source": hbm_src}},
               "cpu_baseline": cpu,
               "e2e": {"value": e2e_value, "unit": UNIT,
                       "h2d_bytes_per_step": 8 * n + 8 * sp.nel + (8 * n if diag_host is not None else 0),
                       "d2h_bytes_per_step": 8 * n},
               "gpu_launches": int(launches),
               "clocks": clk.summary(),
               "accuracy": err,
               "solve_info": {"rel_res": info.rel_res, "device_ms": info.device_ms,
                              "iterations": int(info.iterations), "residual_replacements": int(info.outer_iterations),
                              "fp64_applies": int(info.fp64_applies), "tc_applies": int(info.mixed_applies)}}
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
