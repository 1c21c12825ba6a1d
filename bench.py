"""Benchmark of the AMG-preconditioned PCG solve path on B200.

Workload: 3D linear elasticity, trilinear hex (Q1) elements on the unit cube,
ne^3 elements (default 80^3: 1,574,640 DOF, ~81 nnz/row), E = 1, nu = 0.3,
clamped at z = 0; BAMG prolongation with the six rigid-body modes as test
space, adaptive FSAI smoother, V(1,1); right-hand side = unit body force plus
seeded N(0, 0.01) noise; x0 = 0; PCG_CJ to relative residual 1e-8.

One step = one full PCG solve to 1e-8 on inputs resident in HBM.  `value` is
the FP32-hierarchy solve time (FP64 outer PCG), lower is better; the all-FP64
GPU path is timed in the same run (`fp64_ms`).  `e2e` is the same solve through
the public C ABI call with host buffers (host->device copy of b and x0 and the
device->host copy of x inside the timed region).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl product|reference]

Multi-GPU: a single solve does not shard (dependent SpMVs and global dot
products), so N GPUs run N independent replicas (different right-hand-side
seeds), weak scaling; `value` is the slowest rank's time per solve.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "PCG time-to-1e-8 rel-res, FP32-hierarchy vs FP64 GPU; V-cycle HBM GB/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["product", "reference"], default="product")
    ap.add_argument("--ne", type=int, default=80, help="elements per cube edge")
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--itmax", type=int, default=1000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=["c1", "c2", "c3", "c4", "c5", "emin"], default="c2",
                    help="c2: elasticity (default, the headline); c1: Poisson 32^3; c3: "
                         "diffusion 128^3 with a block of 16 right-hand sides; c4: 64 batched "
                         "problems; c5: adjoint gradient on log-normal diffusion 64^3; emin: the "
                         "energy-minimised prolongation of the elasticity's first level "
                         "(pattern + minimisation) against the reference's EMIN C++")
    ap.add_argument("--profile-solve", choices=["fp32", "fp64"], default=None,
                    help="for ncu --profile-from-start off: build one hierarchy, warm up, "
                         "then bracket exactly one solve with the profiler range and exit")
    return ap.parse_args()


def run_profile_solve(args):
    import torch
    import chronoslab_b200 as cb
    if args.workload == "c3":
        return run_profile_block(args)
    if args.workload == "c4":
        return run_profile_batch(args)
    A, TV, b = build_problem(args.ne, seed=0)
    prec = cb.CHRONOS_FP32 if args.profile_solve == "fp32" else cb.CHRONOS_FP64
    # ncu cannot profile the kernel nodes of a graph holding a conditional
    # node: the profiled solve runs the same per-iteration graph from a host
    # loop (use_graph = 0), kernel for kernel the same work
    h = cb.Hierarchy(A, TV, cb.params(precision=prec, use_graph=0))
    dev = torch.device("cuda", 0)
    bd = torch.from_numpy(b).to(dev)
    x = torch.zeros(A.shape[0], dtype=torch.float64, device=dev)
    h.pcg_dev(bd.data_ptr(), x.data_ptr(), args.itmax, args.tol)
    x.zero_()
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    it, flag, sec = h.pcg_dev(bd.data_ptr(), x.data_ptr(), args.itmax, args.tol)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print(json.dumps({"profile_solve": args.profile_solve, "ne": args.ne, "iterations": it,
                      "flag": flag, "ms": sec * 1e3, "levels": [h.level_info(l)
                                                                for l in range(h.nlevels)]}))
    h.close()
    return 0


def run_profile_block(args):
    """One block solve of the c3 workload (16 right-hand sides) bracketed by
    the profiler range, its iterations launched from a host loop."""
    import numpy as np
    import torch
    import chronoslab_b200 as cb
    from chronoslab_b200 import problems as PB
    ne = 128 if args.ne == 80 else args.ne
    A, _ = PB.diffusion7(ne, sigma=2.0, corr_len=8.0, zaniso=0.01, seed=0)
    B = PB.uniform_rhs(A.shape[0], seed=1, ncols=16)
    prec = cb.CHRONOS_FP32 if args.profile_solve == "fp32" else cb.CHRONOS_FP64
    with cb.Hierarchy(A, np.ones(A.shape[0]), cb.params(precision=prec, ntv=1, use_graph=0)) as h:
        h.pcg_block(B, itmax=args.itmax, tol=args.tol)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        X, its, fl, sec = h.pcg_block(B, itmax=args.itmax, tol=args.tol)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        print(json.dumps({"profile_solve": args.profile_solve, "workload": "c3", "ne": ne,
                          "iterations": its.tolist(), "ms": sec * 1e3,
                          "levels": [h.level_info(l) for l in range(h.nlevels)]}))
    return 0


def c4_problems():
    """64 problems: edge drawn uniformly in [16, 64] from the seed, even ones
    Poisson, odd ones log-normal diffusion."""
    import numpy as np
    from chronoslab_b200 import problems as PB
    rng = np.random.default_rng(0)
    edges = rng.integers(16, 65, 64)
    As, bs = [], []
    for p, e in enumerate(edges):
        if p % 2 == 0:
            A = PB.poisson7(int(e))
        else:
            A, _ = PB.diffusion7(int(e), sigma=2.0, corr_len=8.0, zaniso=0.01, seed=p)
        As.append(A)
        bs.append(PB.uniform_rhs(A.shape[0], seed=1000 + p))
    return As, bs


def run_profile_batch(args):
    """One grouped batch solve of the c4 workload bracketed by the profiler
    range, its iterations launched from a host loop."""
    import torch
    import chronoslab_b200 as cb
    As, bs = c4_problems()
    prec = cb.CHRONOS_FP32 if args.profile_solve == "fp32" else cb.CHRONOS_FP64
    with cb.Batch(As, cb.params(precision=prec, ntv=1, nstep=15, step_size=4,
                                use_graph=0)) as Bt:
        Bt.solve(bs, itmax=args.itmax, tol=args.tol)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        xs, its, fl, sec = Bt.solve(bs, itmax=args.itmax, tol=args.tol)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        print(json.dumps({"profile_solve": args.profile_solve, "workload": "c4",
                          "iterations": [int(its.min()), int(its.max())], "ms": sec * 1e3}))
    return 0


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi during a region."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax = max(smax, float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def traffic_from_profiles(name):
    """Per-launch DRAM bytes of a kernel from the committed ncu summary."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f).get(name)
    except (OSError, ValueError):
        return None


def build_problem(ne, seed):
    from chronoslab_b200 import problems as PB
    A, X = PB.elasticity_q1(ne, return_coords=True)
    TV = PB.rbm_test_space(X)
    b = PB.elasticity_rhs(A, X, seed=seed)
    return A, TV, b


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ---------------------------------------------------------------------------
# reference arm: the reference's CPU implementation of the path
# ---------------------------------------------------------------------------

def run_reference(args, world, rank):
    if rank != 0:
        return 0
    import numpy as np
    from oracle import amg_oracle as O
    from oracle import c_oracle as CO
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref (the reference's FSAI/BAMG C++) was not built"}))
        return 0
    A, TV, b = build_problem(args.ne, seed=0)
    threads = cpu_threads()
    prm = O.default_params(threads)
    t0 = time.perf_counter()
    H = CO.reference_hierarchy(A, TV, prm)
    setup_s = time.perf_counter() - t0
    CH = CO.CHierarchy(H, threads=threads)
    for _ in range(args.warmup):
        CH.pcg(b, itmax=args.itmax, tol=args.tol)
    times, its = [], []
    x = None
    for _ in range(args.steps):
        t = time.perf_counter()
        x, it, rv, flag = CH.pcg(b, itmax=args.itmax, tol=args.tol)
        times.append((time.perf_counter() - t) * 1e3)
        its.append(it)
    ms = sum(times) / len(times)
    relres = float(np.linalg.norm(b - A @ x) / np.linalg.norm(b))
    out = {
        "impl": "reference", "metric": METRIC, "value": ms, "unit": "ms",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Q1 elasticity, body force + N(0,0.01) noise)",
        "config": {"workload": f"Q1 elasticity {args.ne}^3 elements, {A.shape[0]} DOF, "
                               f"{A.nnz} nnz, PCG_CJ + AMG V(1,1) to {args.tol}",
                   "solver": "FP64 PCG_CJ + V-cycle, C/OpenMP restatement of the MATLAB path; "
                             "hierarchy from the reference's own FSAI and BAMG C++"},
        "iterations": its[-1], "true_relres": relres, "setup_s": setup_s,
        "cpu_baseline": {"value": ms, "unit": "ms", "cores": threads, "kind": "reference",
                         "sample": "one full PCG_CJ solve to 1e-8 per step"},
        "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))
    return 0


# ---------------------------------------------------------------------------
# product arm
# ---------------------------------------------------------------------------

def run_product(args, world, rank, local):
    import numpy as np
    import torch
    import chronoslab_b200 as cb

    dist = None
    if world > 1:
        import torch.distributed as tdist
        from datetime import timedelta
        tdist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                 device_id=torch.device("cuda", 0))
        dist = tdist
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)

    A, TV, b = build_problem(args.ne, seed=rank)
    n = A.shape[0]
    h32 = cb.Hierarchy(A, TV, cb.params(precision=cb.CHRONOS_FP32))
    h64 = cb.Hierarchy(A, TV, cb.params(precision=cb.CHRONOS_FP64))
    # the FP32 hierarchy with the FP64 operator in the outer PCG (exact PCG_CJ arithmetic)
    h32x = cb.Hierarchy(A, TV, cb.params(precision=cb.CHRONOS_FP32, exact_outer=1))
    setup32, setup64 = h32.setup_times(), h64.setup_times()

    bd = torch.from_numpy(b).to(dev)
    x32 = torch.zeros(n, dtype=torch.float64, device=dev)
    x64 = torch.zeros(n, dtype=torch.float64, device=dev)

    def solve(h, x):
        x.zero_()
        torch.cuda.synchronize()
        return h.pcg_dev(bd.data_ptr(), x.data_ptr(), args.itmax, args.tol)

    x32x = torch.zeros(n, dtype=torch.float64, device=dev)
    for _ in range(args.warmup):
        solve(h32, x32)
        solve(h64, x64)
        solve(h32x, x32x)

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    clocks = Clocks(local)
    barrier()
    with clocks:
        t32, t64, it32, it64 = [], [], [], []
        for _ in range(args.steps):
            it, flag, sec = solve(h32, x32)
            assert flag == 0, "FP32-hierarchy PCG did not converge"
            t32.append(sec * 1e3)
            it32.append(it)
        for _ in range(args.steps):
            it, flag, sec = solve(h64, x64)
            assert flag == 0, "FP64 PCG did not converge"
            t64.append(sec * 1e3)
            it64.append(it)
        t32x, it32x = [], []
        for _ in range(args.steps):
            it, flag, sec = solve(h32x, x32x)
            assert flag == 0, "FP32-hierarchy PCG (exact outer) did not converge"
            t32x.append(sec * 1e3)
            it32x.append(it)
    barrier()
    ms32 = sum(t32) / len(t32)
    ms64 = sum(t64) / len(t64)
    ms32x = sum(t32x) / len(t32x)
    if dist:
        tt = torch.tensor([ms32, ms64, ms32x], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms32, ms64, ms32x = tt.tolist()

    # end to end through the public call with host buffers: b and x0 in pinned
    # host memory, copied to the device and the solution back inside the call
    e2e = []
    bh = torch.empty(n, dtype=torch.float64).pin_memory().numpy()
    xh = torch.empty(n, dtype=torch.float64).pin_memory().numpy()
    bh[:] = b
    xh[:] = 0.0
    h32.pcg_host(bh, xh, args.itmax, args.tol)       # untimed: the staging buffers
    barrier()
    for _ in range(args.steps):
        xh[:] = 0.0                                   # x0 = 0, set before the clock starts
        t = time.perf_counter()
        it, flag, _ = h32.pcg_host(bh, xh, args.itmax, args.tol)
        e2e.append((time.perf_counter() - t) * 1e3)
        assert flag == 0, "host-buffer PCG did not converge"
    e2e_ms = sum(e2e) / len(e2e)
    if dist:
        tt = torch.tensor([e2e_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_ms = tt.item()

    x32h = x32.cpu().numpy()
    x64h = x64.cpu().numpy()
    x32xh = x32x.cpu().numpy()
    bn = np.linalg.norm(b)
    relres32 = float(np.linalg.norm(b - A @ x32h) / bn)
    relres64 = float(np.linalg.norm(b - A @ x64h) / bn)
    relres32x = float(np.linalg.norm(b - A @ x32xh) / bn)
    h32x.close()

    prof = h32.profile(reps=20)
    prof64 = h64.profile(reps=20)
    peak, peak_kind = peaks()
    achieved = prof["top_apply_bytes"] / (prof["top_apply_ms"] * 1e-3) / 1e9
    vgbs32 = prof["vcycle_bytes"] / (prof["vcycle_ms"] * 1e-3) / 1e9
    vgbs64 = prof64["vcycle_bytes"] / (prof64["vcycle_ms"] * 1e-3) / 1e9
    it_gbs = prof["iteration_bytes"] * it32[-1] / (ms32 * 1e-3) / 1e9

    levels = [h32.level_info(l) for l in range(h32.nlevels)]
    amg = h32.amg_info()[0]

    cpu = None
    rel_err_oracle = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import amg_oracle as O
        from oracle import c_oracle as CO
        parts = []
        for l in range(h64.nlevels):
            p = {"A": h64.export(l, "A")}
            if l < h64.nlevels - 1:
                p.update(G=h64.export(l, "G"), P=h64.export(l, "P"),
                         omega=h64.level_info(l)["omega"])
            parts.append(p)
        threads = cpu_threads()
        CH = CO.CHierarchy(O.hierarchy_from_parts(parts), threads=threads)
        t = time.perf_counter()
        xo, ito, _, flo = CH.pcg(b, itmax=args.itmax, tol=args.tol)
        cpu_ms = (time.perf_counter() - t) * 1e3
        rel_err_oracle = float(np.linalg.norm(x32h - xo) / np.linalg.norm(xo))
        cpu = {"value": cpu_ms, "unit": "ms", "cores": threads, "kind": "port",
               "sample": f"one full FP64 PCG_CJ solve to {args.tol} of the same system "
                         f"({ito} iterations) with the oracle's C/OpenMP V-cycle on the "
                         f"GPU hierarchy's FP64 level matrices"}
        # one host thread: a bounded sample of k iterations, scaled to the full count
        k1 = min(8, max(ito, 1))
        CH1 = CO.CHierarchy(O.hierarchy_from_parts(parts), threads=1)
        t = time.perf_counter()
        CH1.pcg(b, itmax=k1, tol=0.0)
        one_ms = (time.perf_counter() - t) * 1e3 * ito / k1
        cpu["one_core"] = {"value": one_ms, "unit": "ms", "cores": 1,
                           "sample": f"{k1} PCG_CJ iterations on one thread, scaled to {ito}"}
        # Iteration parity on the reference's own prolongation (a check, not
        # timed): the CPU path built with the reference's FSAI/BAMG C++, and
        # the GPU hierarchy built on that path's P level by level, beside the
        # GPU hierarchy on this library's own coarsening and BAMG.
        if O.ref_available():
            H = CO.reference_hierarchy(A, TV, O.default_params())
            _, itr, _, flr = CO.CHierarchy(H, threads=threads).pcg(b, itmax=args.itmax,
                                                                   tol=args.tol)
            Ps = [lv.P for lv in H.levels[:-1]]
            on_ref = {}
            for prec, name in ((cb.CHRONOS_FP64, "fp64"), (cb.CHRONOS_FP32, "fp32")):
                with cb.Hierarchy.with_prolongation(A, Ps, cb.params(precision=prec)) as hp:
                    _, itp, _, flp, _ = hp.pcg(b, itmax=args.itmax, tol=args.tol)
                on_ref[name] = itp if flp == 0 else None
            cpu["iteration_parity"] = {
                "reference_path": itr if flr == 0 else None,
                "gpu_on_reference_prolongation": on_ref,
                "gpu_own_coarsening_and_bamg": {"fp32": it32[-1], "fp64": it64[-1]},
                "levels_reference_path": [lv.A.shape[0] for lv in H.levels]}

    launches = (prof["kernels_per_iteration"] * it32[-1] + prof["kernels_per_solve"]) * args.steps \
        + (prof64["kernels_per_iteration"] * it64[-1] + prof64["kernels_per_solve"]) * args.steps \
        + (prof64["kernels_per_iteration"] * it32x[-1] + prof64["kernels_per_solve"]) * args.steps

    out = {
        "metric": METRIC, "value": ms32, "unit": "ms", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms32, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 hierarchy / f64 outer",
        "data": "synthetic (seeded Q1 elasticity, body force + N(0,0.01) noise)",
        "config": {
            "workload": f"Q1 elasticity {args.ne}^3 elements, {n} DOF, {A.nnz} nnz, "
                        f"BAMG + aFSAI V(1,1), PCG_CJ to {args.tol}",
            "levels": [L["n"] for L in levels],
            "grid_complexity": amg["grid_comp"], "operator_complexity": amg["oper_comp"],
            "l2": "inputs larger than L2 (level-1 operator alone is "
                  f"{A.nnz * 12 / 1e9:.2f} GB in FP64)",
            "parallelism": f"{world} independent replica(s), one per GPU",
        },
        "fp64_ms": ms64,
        "speedup_fp32_vs_fp64": ms64 / ms32,
        "fp32_exact_outer_ms": ms32x,
        "iterations": {"fp32": it32[-1], "fp64": it64[-1], "fp32_exact_outer": it32x[-1]},
        "true_relres": {"fp32": relres32, "fp64": relres64, "fp32_exact_outer": relres32x},
        "outer": "FP32-hierarchy solve: outer A p from the stored FP32 level-1 values with FP64 "
                 "accumulation, FP64 vectors/dots, FP64 true-residual replacement (ratio 0.01 "
                 "and before stopping); fp32_exact_outer_ms: the same hierarchy with the FP64 "
                 "outer operator",
        "rel_err_vs_fp64_oracle": rel_err_oracle,
        "vcycle_hbm_gbs": {"fp32": vgbs32, "fp64": vgbs64},
        "outer_spmv": {"fp32": {"ms": prof["outer_spmv_ms"],
                                "gbs": prof["outer_spmv_bytes"] / (prof["outer_spmv_ms"] * 1e-3) / 1e9},
                       "fp64": {"ms": prof64["outer_spmv_ms"],
                                "gbs": prof64["outer_spmv_bytes"] / (prof64["outer_spmv_ms"] * 1e-3) / 1e9}},
        "pcg_iteration_hbm_gbs": it_gbs,
        "setup_s": {"fp32": setup32["total"], "fp64": setup64["total"]},
        "setup_breakdown_s": {"fp32": {k: round(v, 3) for k, v in setup32.items()}},
        "roofline": {"bound": "hbm", "kernel": "level-1 residual r = b - A x (FP32 sliced 3x3 block form)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": traffic_from_profiles("top_apply"),
                     "algorithmic_bytes": prof["top_apply_bytes"],
                     "launch_ms": prof["top_apply_ms"]},
        "clocks": clocks.summary(),
        "e2e": {"value": e2e_ms, "unit": "ms", "h2d_bytes_per_step": 2 * n * 8,
                "d2h_bytes_per_step": n * 8},
        "gpu_launches": launches,
    }
    if cpu:
        out["cpu_baseline"] = cpu
    if rank == 0:
        print(json.dumps(out))
    h32.close()
    h64.close()
    if dist:
        dist.destroy_process_group()
    return 0


def run_block_or_batch(args, world=1, rank=0):
    """C3 (block of 16 right-hand sides, SpMM V-cycles) or C4 (64 independent
    problems of uneven sizes, queued together); FP32 hierarchy vs FP64.  With
    N ranks (one per GPU) the units are split with no collective on the data
    path: C4's problems largest-first by stored entries, C3's columns in
    contiguous ranges (every rank holds the operator's hierarchy); each step
    is timed on the device by every rank for its share, and the step's time
    is the slowest rank's (NCCL max), the total work staying 64 problems /
    16 columns (strong scaling).  The per-unit iterations and flags are
    gathered once at the end."""
    import numpy as np
    import torch
    import chronoslab_b200 as cb
    from chronoslab_b200 import problems as PB
    from chronoslab_b200.sharding import ShardedBatch, ShardedBlock
    dist = None
    if world > 1:
        import torch.distributed as tdist
        from datetime import timedelta
        torch.cuda.set_device(0)
        tdist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                 device_id=torch.device("cuda", 0))
        dist = tdist
    out = {"metric": METRIC, "unit": "ms", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "higher_is_better": False,
           "scaling": "strong" if world > 1 else "weak",
           "vs_baseline": None, "dtype": "f32 hierarchy / f64 outer",
           "data": "synthetic (seeded)"}

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def slowest(ms):
        if not dist:
            return ms
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return t.item()

    res = {}
    if args.workload == "c3":
        ne = 128 if args.ne == 80 else args.ne
        A, _ = PB.diffusion7(ne, sigma=2.0, corr_len=8.0, zaniso=0.01, seed=0)
        B = PB.uniform_rhs(A.shape[0], seed=1, ncols=16)
        for prec, name in ((cb.CHRONOS_FP32, "fp32"), (cb.CHRONOS_FP64, "fp64")):
            sh = ShardedBlock(A, 16, world, rank, dist, prm=cb.params(precision=prec, ntv=1))
            for _ in range(args.warmup):
                sh.solve_local(B, itmax=args.itmax, tol=args.tol)
            barrier()
            ts = []
            for _ in range(args.steps):
                X, its, fl, sec = sh.solve_local(B, itmax=args.itmax, tol=args.tol)
                assert np.all(np.asarray(fl) == 0)
                ts.append(sec * 1e3)
            barrier()
            relres = max((np.linalg.norm(B[:, j] - A @ X[:, k]) / np.linalg.norm(B[:, j])
                          for k, j in enumerate(range(sh.lo, sh.hi))), default=0.0)
            one = []
            if sh.local is not None:
                for _ in range(2):
                    _, _, _, _, sec1 = sh.local.pcg(B[:, sh.lo], itmax=args.itmax, tol=args.tol)
                    one.append(sec1 * 1e3)
            units, _ = sh.solve(B, itmax=args.itmax, tol=args.tol, gather_x=False)
            res[name] = {"ms": slowest(sum(ts) / len(ts)),
                         "iters": [units[j]["iters"] for j in range(16)],
                         "single_rhs_ms": min(one) if one else None,
                         "true_relres_max": float(slowest(relres)),
                         "levels": ([sh.local.level_info(l)["n"] for l in range(sh.local.nlevels)]
                                    if sh.local is not None else None)}
            sh.close()
        out["config"] = {"workload": f"log-normal diffusion {ne}^3 ({A.shape[0]} rows, {A.nnz} "
                                     "nnz), block of 16 RHS, SpMM V-cycles, PCG_CJ to "
                                     f"{args.tol} per column",
                         "parallelism": f"columns split over {world} rank(s)" if world > 1
                         else "one GPU"}
    else:
        As, bs = c4_problems()
        for prec, name in ((cb.CHRONOS_FP32, "fp32"), (cb.CHRONOS_FP64, "fp64")):
            t0 = time.perf_counter()
            sh = ShardedBatch(As, world, rank, dist,
                              prm=cb.params(precision=prec, ntv=1, nstep=15, step_size=4))
            setup = time.perf_counter() - t0
            for _ in range(args.warmup):
                sh.solve_local(bs, itmax=args.itmax, tol=args.tol)
            barrier()
            ts = []
            for _ in range(args.steps):
                xs, its, fl, sec = sh.solve_local(bs, itmax=args.itmax, tol=args.tol)
                assert np.all(np.asarray(fl) == 0)
                ts.append(sec * 1e3)
            barrier()
            units, _ = sh.solve(bs, itmax=args.itmax, tol=args.tol, gather_x=False)
            its_all = [units[p]["iters"] for p in range(len(As))]
            phases = (sh.local.setup_times() if sh.local is not None else {})
            walls = (sh.local.setup_wall() if sh.local is not None else {})
            res[name] = {"ms": slowest(sum(ts) / len(ts)), "setup_s": slowest(setup),
                         "setup_wall_s": {k: round(v, 3) for k, v in walls.items()},
                         "setup_thread_s": {k: round(v, 3) for k, v in phases.items()},
                         "iters_min_max": [int(min(its_all)), int(max(its_all))],
                         "problems_per_rank": [len(p) for p in sh.parts]}
            sh.close()
        out["config"] = {"workload": "64 independent problems (Poisson / log-normal diffusion, "
                                     f"edge U[16,64]: {min(A.shape[0] for A in As)} to "
                                     f"{max(A.shape[0] for A in As)} rows), FSAI 15 steps x 4, "
                                     "batch solve, PCG_CJ to 1e-8 each",
                         "parallelism": f"problems split largest-first over {world} rank(s)"
                         if world > 1 else "one GPU"}
    out["value"] = res["fp32"]["ms"]
    out["ms_per_step"] = res["fp32"]["ms"]
    out["fp64_ms"] = res["fp64"]["ms"]
    out["speedup_fp32_vs_fp64"] = res["fp64"]["ms"] / res["fp32"]["ms"]
    out["detail"] = res
    if rank == 0:
        print(json.dumps(out))
    if dist:
        dist.destroy_process_group()
    return 0


def run_c1_or_c5(args):
    """C1 (7-point Poisson 32^3, Dirichlet eliminated, constant test vector,
    PCG_CJ to tol from x0 = 0) or C5 (log-normal diffusion 64^3, sigma = 1:
    gradient of J = 1/2 ||u - u*||^2 on A's pattern by a forward solve and
    the adjoint solve on the same hierarchy); FP32 hierarchy vs FP64, solve
    times by CUDA events inside the library, setup excluded."""
    import numpy as np
    import chronoslab_b200 as cb
    from chronoslab_b200 import problems as PB
    out = {"metric": METRIC, "unit": "ms", "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "higher_is_better": False, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32 hierarchy / f64 outer", "data": "synthetic (seeded)"}
    res = {}
    if args.workload == "c1":
        A = PB.poisson7(32)
        b = PB.uniform_rhs(A.shape[0], seed=0)
        for prec, name in ((cb.CHRONOS_FP32, "fp32"), (cb.CHRONOS_FP64, "fp64")):
            with cb.Hierarchy(A, np.ones((A.shape[0], 1)), cb.params(precision=prec, ntv=1)) as h:
                for _ in range(args.warmup):
                    h.pcg(b, itmax=args.itmax, tol=args.tol)
                ts = []
                for _ in range(args.steps):
                    x, it, _, flag, sec = h.pcg(b, itmax=args.itmax, tol=args.tol)
                    assert flag == 0
                    ts.append(sec * 1e3)
                res[name] = {"ms": sum(ts) / len(ts), "iters": it,
                             "true_relres": float(np.linalg.norm(b - A @ x) / np.linalg.norm(b)),
                             "levels": [h.level_info(l)["n"] for l in range(h.nlevels)]}
        out["config"] = {"workload": f"7-point Poisson 32^3 ({A.shape[0]} rows, {A.nnz} nnz), "
                                     f"DOM 0.01 + BAMG + aFSAI V(1,1), PCG_CJ to {args.tol}"}
    else:
        shape = (64, 64, 64)
        logk = PB.gaussian_field(shape, 8.0, seed=5)
        A = PB.diffusion_from_logk(logk, 0.01)
        rng = np.random.default_rng(11)
        b = rng.uniform(-1, 1, A.shape[0])
        ustar = rng.uniform(-1, 1, A.shape[0]) * 0.01
        grads = {}
        for prec, name in ((cb.CHRONOS_FP32, "fp32"), (cb.CHRONOS_FP64, "fp64")):
            with cb.Hierarchy(A, np.ones((A.shape[0], 1)), cb.params(precision=prec, ntv=1)) as h:
                ts = []
                for k in range(args.warmup + args.steps):
                    u, it, _, flag, s1 = h.pcg(b, itmax=args.itmax, tol=1e-12)
                    t0 = time.perf_counter()
                    lam, g, it2 = h.adjoint_grad(u, u - ustar, itmax=args.itmax, tol=1e-12)
                    s2 = time.perf_counter() - t0
                    assert flag == 0
                    if k >= args.warmup:
                        ts.append((s1 + s2) * 1e3)
                grads[name] = g
                res[name] = {"ms": sum(ts) / len(ts), "iters_forward": it, "iters_adjoint": it2}
        res["grad_rel_diff_fp32_vs_fp64"] = float(np.linalg.norm(grads["fp32"] - grads["fp64"]) /
                                                  np.linalg.norm(grads["fp64"]))
        out["config"] = {"workload": f"log-normal diffusion 64^3 ({A.shape[0]} rows, {A.nnz} "
                                     "nnz), sigma 1, correlation 8 cells, z-faces x 0.01: "
                                     "forward solve + adjoint solve + dJ/dA scatter, tol 1e-12 "
                                     "(forward: device time; adjoint: host clock around the call)"}
    out["value"] = res["fp32"]["ms"]
    out["ms_per_step"] = res["fp32"]["ms"]
    out["fp64_ms"] = res["fp64"]["ms"]
    out["speedup_fp32_vs_fp64"] = res["fp64"]["ms"] / res["fp32"]["ms"]
    out["detail"] = res
    print(json.dumps(out))
    return 0


def run_emin(args):
    """prolong.m:207-235 on the first level of the C2 elasticity (--ne): the
    pattern (chronos_emin_pattern) and the energy minimisation (chronos_emin)
    of the library's own BAMG prolongation, timed end to end through the C
    ABI with host arrays (value), with the device phases of the minimisation
    from its info array; the reference's MEX_cptProlPatt and EMIN_ImpProl
    (oracle/_ref, all host threads) on the same inputs as cpu_baseline, and
    the parity of the two (pattern bit for bit, P's largest difference)."""
    import numpy as np
    import scipy.sparse as sp
    import chronoslab_b200 as cb
    A, TV0, _ = build_problem(args.ne, seed=0)
    A = sp.csr_matrix(A)
    A.sort_indices()
    n = A.shape[0]
    prm = cb.params()
    fc, nc, S = cb.coarsen(A, prm, 0)
    S = sp.csr_matrix(S)
    S.sort_indices()
    d = A.diagonal()
    rows = np.repeat(np.arange(n), np.diff(S.indptr))
    a = np.asarray(A[rows, S.indices]).ravel()
    S = sp.csr_matrix((np.abs(a) / np.sqrt(d[rows] * d[S.indices]), S.indices, S.indptr),
                      shape=(n, n))                     # cpt_SoC_dom.m:26-47 values
    TV, _ = np.linalg.qr(TV0)
    P, _ = cb.bamg(S, fc, TV, prm)
    ntv = TV.shape[1]

    def step():
        t0 = time.perf_counter()
        patt, host_rows = cb.emin_pattern(S, P, fc, kpow=prm.patt_pow, nnzr_max=prm.nnzr_max,
                                          nnzr_min=ntv)
        t1 = time.perf_counter()
        Pe, info = cb.emin(A, P, patt, fc, TV, prm)
        t2 = time.perf_counter()
        return patt, Pe, info, host_rows, (t1 - t0) * 1e3, (t2 - t1) * 1e3

    for _ in range(args.warmup):
        step()
    rec = [step() for _ in range(args.steps)]
    patt, Pe, info, host_rows = rec[-1][:4]
    t_patt = sum(r[4] for r in rec) / len(rec)
    t_emin = sum(r[5] for r in rec) / len(rec)
    iters = int(info[7])
    out = {"metric": "EMIN prolongation time (pattern + energy minimisation), level 1",
           "value": t_patt + t_emin, "unit": "ms", "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": t_patt + t_emin, "higher_is_better": False,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded Q1 elasticity, rigid-body test space)",
           "config": {"workload": f"Q1 elasticity {args.ne}^3 elements, {n} DOF, level-1 EMIN "
                                  f"(patt_pow {prm.patt_pow}, nnzr_max {prm.nnzr_max}, "
                                  f"itmax_emin {prm.itmax_emin}, Jacobi) of this library's BAMG P "
                                  f"({nc} coarse nodes)",
                      "pattern_entries": int(patt.nnz), "cg_steps": iters,
                      "host_rows": int(host_rows)},
           "e2e": {"value": t_patt + t_emin, "unit": "ms",
                   "h2d_bytes_per_step": int(2 * (A.data.nbytes + A.indices.nbytes + A.indptr.nbytes)
                                             + S.data.nbytes + S.indices.nbytes + 2 * P.data.nbytes),
                   "d2h_bytes_per_step": int(12 * patt.nnz + 12 * Pe.nnz)},
           "detail": {"pattern_ms": t_patt, "minimisation_ms": t_emin,
                      "device_constraints_ms": info[2] * 1e3, "device_cg_ms": info[3] * 1e3,
                      "device_total_ms": info[5] * 1e3, "svd_rows": int(info[6])},
           "gpu_launches": args.steps * (1 + 3 + (iters + 1) + (2 * iters + 1) + 2 * iters + 1)}
    if not args.no_cpu_baseline:
        sys.path.insert(0, ROOT)
        from oracle import amg_oracle as O
        nth = cpu_threads()
        pro = O.default_params(nth)["prolong"]
        t0 = time.perf_counter()
        R = O.ref_emin_pattern(prm.patt_pow, S, P, fc, prm.nnzr_max, ntv, nth)
        t1 = time.perf_counter()
        Pr, rinfo = O.ref_emin(pro, A, R, P, TV, fc)
        t2 = time.perf_counter()
        out["cpu_baseline"] = {
            "value": (t2 - t0) * 1e3, "unit": "ms", "cores": nth, "kind": "reference",
            "sample": "one call each of the reference's MEX_cptProlPatt and EMIN_ImpProl "
                      "(oracle/_ref) on the same inputs",
            "pattern_ms": (t1 - t0) * 1e3, "minimisation_ms": (t2 - t1) * 1e3,
            "cg_steps": int(rinfo[7]),
            "parity": {"pattern_bit_identical": bool(np.array_equal(R.indptr, patt.indptr) and
                                                     np.array_equal(R.indices, patt.indices) and
                                                     np.array_equal(R.data, patt.data)),
                       "P_max_diff_over_max": float(abs(Pe - Pr).max() / abs(Pr).max())}}
    print(json.dumps(out))
    return 0


def main():
    args = parse()
    world, rank, local = dist_env()
    if world > 1:
        # one device per rank: both CUDA runtimes in the process (torch's and
        # the library's) then see the same single device
        os.environ["CUDA_VISIBLE_DEVICES"] = str(local)
    if args.impl == "reference":
        return run_reference(args, world, rank)
    if args.profile_solve:
        return run_profile_solve(args)
    if args.workload in ("c1", "c5"):
        return run_c1_or_c5(args)
    if args.workload == "emin":
        return run_emin(args)
    if args.workload != "c2":
        return run_block_or_batch(args, world, rank)
    return run_product(args, world, rank, local)


if __name__ == "__main__":
    sys.exit(main())
