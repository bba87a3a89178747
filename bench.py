"""Benchmark of the geometric-multigrid Poisson solve path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Default workload (the configuration the headline metric is quoted on): 2D Poisson, Q1 on the unit
square, level 10 (1,050,625 DOFs, 9,443,329 nnz), right-hand side a sum of 8 seeded Gaussians,
PCG preconditioned by one V(2,2) cycle (Richardson + Jacobi omega 0.7, exact coarse solve on level
1) run in FP32 inside FP64 PCG (iterative refinement), relative residual 1e-8.  The problem is
numbered lexicographically and solved in that order (--ordering native), so its system matrices
are held as diagonals; --ordering rcm gives the sliced-ELL form.

One step = one complete solve from a zero initial guess with the matrices resident in HBM.  Each
step is timed with CUDA events on the stream of the call; the L2 is overwritten between steps
(outside the timed interval).  `value` is milliseconds per solve for the whole job (max over ranks
of the per-rank time / solves of all ranks); every GPU solves its own replica ("replicas only":
a single solve does not shard).  rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "feat3.doxytest_b200"))

METRIC = "solve ms to 1e-8 residual vs plain FP64 GPU multigrid; SpMV HBM GB/s"
FALLBACK_HBM_GBS = 6650.0

WORKLOADS = {
    # name: (dim, level, rhs, precision, description)
    "poisson2d_l10_mixed": (2, 10, "gauss", "f32",
                            "2D Poisson Q1 unit square L10 (1,050,625 DOFs), 8-Gaussian RHS seed 1, "
                            "PCG + FP32 V(2,2) Jacobi(0.7) multigrid in FP64 refinement, tol_rel 1e-8"),
    "poisson2d_l10_bf16": (2, 10, "gauss", "f32_bf16",
                           "as poisson2d_l10_mixed with BF16 matrix values in the V-cycle"),
    "poisson2d_l10_fp64": (2, 10, "gauss", "f64", "plain FP64 PCG + V(2,2) multigrid, L10, 8-Gaussian RHS"),
    "poisson2d_l7_fp64": (2, 7, "sine", "f64", "2D Poisson Q1 L7 (16,641 DOFs), sine-bubble RHS, plain FP64"),
    "poisson3d_l6_rhs64_mixed": (3, 6, "gauss64", "f32",
                                 "3D Poisson Q1 unit cube L6 (274,625 DOFs, 27-point), 64 right-hand sides of 8 "
                                 "Gaussians each (seeds 100..163), solved together, FP32 V(2,2) in FP64 PCG"),
    "poisson2d_l9_warmstart": (2, 9, "family", "f32",
                               "-div(kappa grad u)=f family at L9 (263,169 DOFs; kappa = exp(16x16-mode field), "
                               "8-Gaussian f): U-Net on the 129^2 L7 grid trained on FP64-multigrid solutions, "
                               "prediction prolongated as the PCG initial guess (zero-guess fallback), FP32 V(2,2) "
                               "in FP64 PCG, stop at ||d|| <= 1e-8 ||b||; evaluated on unseen seeds"),
    "poisson2d_batch256_mixed": (2, 9, "batch", "f32",
                                 "256 independent -div(kappa grad u)=f instances, levels uniform in 5..9 (seed 7), "
                                 "kappa = exp(16x16-mode random field), 8-Gaussian RHS, one launch per V-cycle phase, "
                                 "FP32 V(2,2) in FP64 PCG, tol 1e-8 per instance"),
}
DEFAULT_WORKLOAD = "poisson2d_l10_mixed"

# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one launch, from an ncu capture of
# the kernel as built from the current sources: (workload, ordering, kernel) -> bytes
MEASURED_TRAFFIC = {("poisson2d_l10_mixed", "native", "pcg_spmv"): 85.150720e6 + 3.981824e6}


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def csr_alg_bytes(nnz, rows, cols, s_v, s_i, s_x, row_vectors=0):
    """Algorithmic bytes of a CSR SpMV y = A x: values and column indices, the row pointer, x
    once, y written, plus `row_vectors` further row-wise vectors read (b of a defect)."""
    return nnz * (s_v + s_i) + (rows + 1) * s_i + cols * s_x + rows * s_x + row_vectors * rows * s_x


def read_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""
    FIELDS = "timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.out = None

    def start(self):
        try:
            self.out = tempfile.TemporaryFile(mode="w+")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self, t0=None, t1=None):
        """Samples taken between wall-clock times t0 and t1 (the timed region), or all."""
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.seek(0)
        import datetime
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out.read().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                mhz, mx = float(parts[2]), float(parts[3])
            except ValueError:
                continue
            if t0 is not None and not (t0 - 0.25 <= ts <= t1 + 0.25):
                continue
            sm.append(mhz)
            smax.append(mx)
            try:
                power.append(float(parts[4]))
            except ValueError:
                pass
            for n, v in zip(names, parts[6:10]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm),
                "power_w_median": float(np.median(power)) if power else None}


def build_problem(dim, level, rhs_kind):
    from featb200 import assembly as AS
    gauss = AS.gauss_params(1, dim, width=(0.02, 0.1) if dim == 2 else (0.03, 0.12)) if rhs_kind == "gauss" else None
    levels, b = AS.poisson_hierarchy(level, dim, rhs=rhs_kind, gauss=gauss)
    return levels, b, gauss


def batch_levels(count=256):
    from featb200 import assembly as AS
    return AS.batch_family_levels(count)


def _batch_instance(args):
    sys.path.insert(0, os.path.join(ROOT, "feat3.doxytest_b200"))
    from featb200 import assembly as AS
    level, k = args
    return AS.batch_instance(level, k)


def start_batch_build(count=256):
    """Config-4 family assembled on a spawn-started process pool (host set-up, no CUDA in the
    workers); returns (levels, pool, async result)."""
    import multiprocessing as mp
    levels = batch_levels(count)
    pool = mp.get_context("spawn").Pool(min(32, os.cpu_count() or 1))
    res = pool.map_async(_batch_instance, [(L, k) for k, L in enumerate(levels)])
    return levels, pool, res


def finish_batch_build(started):
    levels, pool, res = started
    inst = res.get()
    pool.close()
    pool.join()
    return levels, inst


def build_batch_problem(count=256):
    return finish_batch_build(start_batch_build(count))


def build_rhs64_problem():
    from featb200 import assembly as AS
    return AS.rhs64_family(6, 3, 64)


class L2Flush:
    """Untimed cache flush between timed solves: overwrite a 256 MiB buffer, then read another
    256 MiB buffer, so that the L2 (126 MB) holds none of the solver's data and no dirty lines whose
    write-back would land inside the timed interval."""
    DESC = "flushed before every timed solve (256 MiB write, then 256 MiB read of another buffer)"

    def __init__(self, torch):
        self.w = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
        self.r = torch.zeros(64 << 20, dtype=torch.int32, device="cuda")

    def __call__(self):
        self.w.fill_(1)
        self.r.sum()


def run_warmstart(args):
    """Learned warm start (value = mean device ms per solve of the unseen instances, network
    inference, prolongation and the fallback test included; assembly excluded).  Training data:
    args.ws_train instances solved by the FP64 multigrid; evaluation: args.ws_eval unseen instances,
    each solved from zero and from the network's start by the same mixed-precision solver."""
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    import featb200 as fb
    from featb200.warmstart import ParametricFamily, WarmStart
    dim, level, rhs_kind, precision, desc = WORKLOADS[args.workload]
    t0 = time.time()
    gen = ParametricFamily(level=9, net_level=7, precision="f64")
    X, Y, its_train = gen.generate(range(0, args.ws_train))
    t_gen = time.time() - t0
    ws = WarmStart(gen, max_batch=32, seed=0)
    t0 = time.time()
    hist = ws.fit(X, Y, epochs=args.ws_epochs, batch=32, lr=3e-3)
    torch.cuda.synchronize()
    t_fit = time.time() - t0
    del X, Y
    fam = ParametricFamily(level=9, net_level=7, precision=precision)
    ws.family = fam
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    stream = torch.cuda.current_stream()

    def timed(fn):
        torch.cuda.synchronize()
        ev0.record(stream)
        out = fn()
        ev1.record(stream)
        ev1.synchronize()
        return out, ev0.elapsed_time(ev1)

    ev = range(50_000, 50_000 + args.ws_eval)
    # warm-up (untimed)
    for k in range(40_000, 40_000 + args.warmup):
        fam.setup(k)
        fam.solve(torch.zeros(fam.n, dtype=torch.float64, device="cuda"))
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    wall0 = time.time()
    l0 = fb.launch_count()
    rows = []
    for k in ev:
        fam.setup(k)
        x = torch.zeros(fam.n, dtype=torch.float64, device="cuda")
        (st0, it0), ms0 = timed(lambda: fam.solve(x))

        def warm():
            x0, used, ratio = ws.initial_guess(k)
            st, it = fam.solve(x0)
            return x0, used, ratio, st, it
        (x0, used, ratio, st1, it1), ms1 = timed(warm)
        rows.append((it0, it1, ms0, ms1, used, float((x0 - x).norm() / x.norm()),
                     st0 == fb.Status.success and st1 == fb.Status.success))
    launches = fb.launch_count() - l0
    wall1 = time.time()
    time.sleep(0.3)
    clk = clocks.stop(wall0, wall1)
    a = np.array([r[:6] for r in rows], dtype=np.float64)
    ms_warm = float(a[:, 3].mean())
    print(json.dumps({"metric": METRIC, "value": ms_warm, "unit": "ms", "n_gpus": world, "steps": len(rows),
                      "warmup": args.warmup, "ms_per_step": ms_warm, "higher_is_better": False, "scaling": "weak",
                      "vs_baseline": None, "dtype": "f32+f64 (network bf16/f32)", "data": "synthetic",
                      "config": {"workload": args.workload + ": " + desc, "dofs": fam.n, "train_instances": args.ws_train,
                                 "epochs": args.ws_epochs, "eval_instances": len(rows), "network_grid": "129x129",
                                 "l2": "not flushed (each step reassembles the instance first)"},
                      "ms_zero_guess": float(a[:, 2].mean()), "iterations_zero": float(a[:, 0].mean()),
                      "iterations_warm": float(a[:, 1].mean()), "network_used": float(a[:, 4].mean()),
                      "max_rel_diff_warm_vs_zero": float(a[:, 5].max()), "all_success": all(r[6] for r in rows),
                      "train_loss_last": float(hist[-1]), "generate_s": t_gen, "train_s": t_fit,
                      "train_iterations_fp64": float(np.mean(its_train)),
                      "gpu_launches": int(launches), "clocks": clk}))
    return 0


def run_multi(args, kind):
    """Secondary workloads: the 64-RHS 3D solve and the 256-instance batch (value = ms per solve of
    the whole set).  With N ranks the batch's instances are sharded by a longest-processing-time
    assignment on DOF count (no collective on the data path; total work fixed: strong scaling);
    the 64-RHS set is solved as a replica on every rank (weak scaling)."""
    pre = build_batch_problem(args.batch_count) if kind == "batch" else None
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
        pg = dist
    import featb200 as fb
    from featb200 import sharding
    dim, level, rhs_kind, precision, desc = WORKLOADS[args.workload]
    mine = None
    if kind == "batch":
        levels, inst = pre
        mine = sharding.shard([b.size for _, b in inst], rank, world)
        inst = [inst[i] for i in mine]
        hs = [fb.build_hierarchy(lv) for lv, _ in inst]
        solver = fb.BatchPCG(hs, precision=precision, ordering=args.ordering, use_graph=not args.profile_solves)
        rhs = np.concatenate([b for _, b in inst])
        units, dofs = len(inst), int(rhs.size)
    else:
        lv, B = build_rhs64_problem()
        solver = fb.MultiRhsPCG(fb.build_hierarchy(lv), 64, precision=precision, ordering=args.ordering,
                                use_graph=not args.profile_solves)
        rhs = B.ravel()
        units, dofs = 64, int(B.shape[0])
    stream = torch.cuda.current_stream()
    rhs_d = torch.tensor(rhs, device="cuda")
    sol_d = torch.zeros_like(rhs_d)
    flush = L2Flush(torch)
    for _ in range(args.warmup):
        sol_d.zero_()
        solver.solve_device(sol_d, rhs_d, stream)
    torch.cuda.synchronize()
    if args.profile_solves:
        for _ in range(args.profile_solves):
            sol_d.zero_()
            solver.solve_device(sol_d, rhs_d, stream)
        torch.cuda.synchronize()
        print(json.dumps({"profile_solves": args.profile_solves, "iterations_max": int(max(solver.iterations()))}))
        return 0
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    wall0 = time.time()
    l0 = fb.launch_count()
    times = []
    for _ in range(args.steps):
        flush()
        sol_d.zero_()
        ev0.record(stream)
        solver.solve_device(sol_d, rhs_d, stream)
        ev1.record(stream)
        ev1.synchronize()
        times.append(ev0.elapsed_time(ev1))
    launches = fb.launch_count() - l0
    wall1 = time.time()
    time.sleep(0.3)
    clk = clocks.stop(wall0, wall1)
    st = solver.statuses()
    its = solver.iterations()
    total = float(np.sum(times))
    if pg:
        t = torch.tensor([total], device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        total = float(t.item())
    if kind == "batch":
        n_all = len(pre[1])
        its = sharding.gather_results(pg, rank, world, mine, its, n_all)
        st = sharding.gather_results(pg, rank, world, mine, [float(x) for x in st], n_all)
        units = n_all
    ms = total / args.steps
    # per-step time of the whole job: the batch's shards run concurrently (max over ranks); the 64-RHS
    # replicas solve world x 64 right-hand sides in that time
    value = ms if kind == "batch" else ms / world
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    if rank == 0:
        print(json.dumps({"metric": METRIC, "value": value, "unit": "ms", "n_gpus": world, "steps": args.steps,
                          "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
                          "scaling": "strong" if kind == "batch" else "weak",
                          "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
                          "config": {"workload": args.workload + ": " + desc, "solves_per_step": units,
                                     "dofs_per_step": dofs, "ordering": args.ordering,
                                     "iterations_max": int(max(its)), "iterations_min": int(min(its)),
                                     "all_success": all(int(x) == int(fb.Status.success) for x in st),
                                     "parallelism": (f"instances sharded x{world} (LPT on DOFs)" if kind == "batch"
                                                     else f"replicas x{world}"),
                                     "l2": L2Flush.DESC},
                          "solves_per_s": units * world ** (kind != "batch") * 1e3 / ms,
                          "gpu_launches": int(launches), "clocks": clk}))
    return 0


def cpu_reference_times(dim, level, rhs_kind, gauss, reps, timeout=900, field=None, backend=None):
    """The reference's own CPU solver (oracle/_ref/feat_oracle, built from the reference's sources)
    on the same problem; returns its JSON summary with per-solve times (1 warm-up + reps).
    backend="cuda": the reference's own GPU backend instead (oracle/_ref/feat_cuda)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not (O.feat_cuda_available() if backend == "cuda" else O.feat_available()):
        return None
    from featb200 import assembly as AS
    with tempfile.TemporaryDirectory() as d:
        params = kappa = None
        if gauss is not None:
            params = os.path.join(d, "gauss.txt")
            AS.write_params(params, gauss=gauss)
        if field is not None:
            kappa = os.path.join(d, "kappa.txt")
            AS.write_params(kappa, field=field)
        return O.feat_solve(d, dim=dim, level=level, rhs=rhs_kind, params=params, kappa=kappa, dump=False,
                            time_reps=reps, timeout=timeout, b200=backend)


def reference_sample(args):
    """(ms per step, iterations, dofs, nnz, sample description) of the reference's CPU solver for
    the workload, from a bounded sample (a few minutes at most)."""
    dim, level, rhs_kind, precision, desc = WORKLOADS[args.workload]
    from featb200 import assembly as AS
    if rhs_kind in ("sine", "gauss"):
        reps = max(1, min(args.warmup + args.steps, 40))
        gauss = AS.gauss_params(1, dim) if rhs_kind == "gauss" else None
        res = cpu_reference_times(dim, level, rhs_kind, gauss, reps)
        if res is None:
            return None
        t = res["times_ms"]
        return (float(np.mean(t)), res["iters"], res["dofs"], res["nnz"],
                f"{len(t)} FP64 solves of the workload (after 1 warm-up) by the reference's generic "
                "(single-threaded) backend, solve only")
    if rhs_kind == "gauss64":
        g = AS.gauss_params(100, 3, width=(0.03, 0.12))
        res = cpu_reference_times(3, level, "gauss", g, 3)
        if res is None:
            return None
        t = float(np.mean(res["times_ms"]))
        return (64.0 * t, res["iters"], res["dofs"], res["nnz"],
                "3 FP64 single right-hand-side solves of the 3D L6 problem (right-hand side 0 of the 64) by the "
                "reference's generic backend, times 64 (the reference solves the columns one after the other)")
    if rhs_kind == "batch":
        levels = batch_levels(256)
        per_level = {}
        for L in sorted(set(levels)):
            k = levels.index(L)
            res = cpu_reference_times(2, L, "gauss", AS.gauss_params(10_000 + 2 * k, 2), 1,
                                      field=AS.field_params(10_001 + 2 * k))
            if res is None:
                return None
            per_level[L] = (float(res["times_ms"][-1]), res["iters"])
        ms = float(sum(per_level[L][0] for L in levels))
        return (ms, max(v[1] for v in per_level.values()), None, None,
                "one instance per level 5..9 of the 256-instance batch solved by the reference's generic backend "
                "(FP64, single-threaded, solve only); value = sum over the 256 instances of their level's time")
    if rhs_kind == "family":
        from featb200.warmstart import SEED_BASE
        ts, its = [], []
        for k in range(50_000, 50_004):
            s0 = SEED_BASE + 2 * k
            res = cpu_reference_times(2, level, "gauss", AS.gauss_params(s0, 2), 1, field=AS.field_params(s0 + 1))
            if res is None:
                return None
            ts.append(float(res["times_ms"][-1]))
            its.append(res["iters"])
        return (float(np.mean(ts)), float(np.mean(its)), res["dofs"], res["nnz"],
                "4 of the unseen instances solved from a zero guess by the reference's generic backend (FP64, "
                "single-threaded, solve only; the reference has no learned start)")
    return None


def run_reference_gpu(args):
    """The reference's own GPU backend (FEAT built with its CUDA sources: cuSPARSE SpMV, cuBLAS
    vector ops, managed memory, one synchronised launch per LAFEM op) on the default workload, FP64:
    a timing column beside the library, not the default reference arm (the generic CPU path)."""
    dim, level, rhs_kind, precision, desc = WORKLOADS[args.workload]
    from featb200 import assembly as AS
    if rhs_kind not in ("sine", "gauss"):
        print(json.dumps({"impl": "reference", "reference_backend": "cuda",
                          "unavailable": "timed for the single-system workloads only"}))
        return 0
    gauss = AS.gauss_params(1, dim) if rhs_kind == "gauss" else None
    try:
        res = cpu_reference_times(dim, level, rhs_kind, gauss, max(1, min(args.warmup + args.steps, 20)),
                                  backend="cuda")
    except (subprocess.CalledProcessError, subprocess.TimeoutExpired) as e:
        print(json.dumps({"impl": "reference", "reference_backend": "cuda",
                          "unavailable": f"the reference's CUDA build did not run here ({type(e).__name__}; "
                                         "it needs a GPU)"}))
        return 0
    if res is None:
        print(json.dumps({"impl": "reference", "reference_backend": "cuda",
                          "unavailable": "oracle/_ref/feat_cuda is missing; build it with `make -C oracle cuda`"}))
        return 0
    t = res["times_ms"]
    ms = float(np.mean(t))
    print(json.dumps({"impl": "reference", "reference_backend": "cuda", "metric": METRIC, "value": ms, "unit": "ms",
                      "n_gpus": 1, "steps": len(t), "warmup": 1, "ms_per_step": ms, "higher_is_better": False,
                      "dtype": "f64", "data": "synthetic", "times_ms": t, "status": res["status"],
                      "config": {"workload": args.workload + ": " + desc + " (the reference's GPU path is FP64)",
                                 "dofs": res["dofs"], "nnz": res["nnz"], "iterations": res["iters"]},
                      "timing": "host wall clock around Solver::solve (every op synchronises), after 1 warm-up solve"}))
    return 0


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    if args.reference_backend == "cuda":
        return run_reference_gpu(args)
    dim, level, rhs_kind, precision, desc = WORKLOADS[args.workload]
    res = reference_sample(args)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/feat_oracle (the reference built from "
                          "its sources) is missing; build it with `make -C oracle ref`"}))
        return 0
    ms, iters, dofs, nnz, sample = res
    line = {"impl": "reference", "metric": METRIC, "value": ms, "unit": "ms", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload + ": " + desc + " (the reference's CPU path is FP64 only)",
                       "dofs": dofs, "nnz": nnz, "iterations": iters},
            "cpu_baseline": {"value": ms, "unit": "ms", "cores": 1, "kind": "reference", "sample": sample},
            "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


PASS_KERNELS = {
    "pcg_spmv": "k_tma_pass<OpPcgQ>: FP64 q = F(A p) and q.p (PCG)",
    "mg_smooth": "k_tma_pass<OpSmooth>: pre-smoothing step 2",
    "mg_defect": "k_tma_pass<OpDefect>: defect d = F(b - A x) before restriction",
    "mg_restrict": "k_tma_pass<OpRestrict>: b_c = F(R d), sol1_c = F(D_c b_c)",
    "mg_prolong": "k_tma_pass<OpProlong>: x += F(P x_c)",
    "mg_post1": "k_tma_pass<OpPost1>: post-smoothing step 1 (defect, Jacobi correction, norm)",
    "mg_post2": "k_tma_pass<OpPost2>: post-smoothing step 2 with the PCG's z and r.z",
    "mg_down": "k_fz_down: fused pre-smoothing step 2 + defect + restriction (structured 2D level)",
    "mg_up": "k_fz_up: fused prolongation + post-smoothing with the PCG's z and r.z (structured 2D level)",
    "mg_sdown": "k_fs_down: the fused down pass streamed through bands of coarse rows (structured 2D level)",
    "mg_sup": "k_fs_up: the fused up pass streamed through bands of coarse rows (structured 2D level)",
}
FUSED_PASSES = ("mg_down", "mg_up")
STREAM_PASSES = ("mg_sdown", "mg_sup")


def pass_table(solver, levels, precision, reps=20):
    """Each finest-level pass of a solve timed alone (cold L2) with its CSR-algorithmic bytes
    (nnz * (value + 4 B index) + (rows + 1) * 4 B + the vectors it reads and writes: the bytes a CSR
    pass over the reference's containers must move) and the bytes it moves as stored on the device
    (solver's count)."""
    sv = {"f64": 8, "f32": 4, "f32_bf16": 2}[precision]
    sx = 8 if precision == "f64" else 4
    A = levels[0]["matrix"]
    n = int(A.rows())
    nnz = int(A.used_elements())
    tr = levels[0]["transfer"]
    nc = int(tr.rest.rows())
    nnz_r, nnz_p = int(tr.rest.used_elements()), int(tr.prol.used_elements())

    def csr(nz, rows, sval):
        return nz * (sval + 4) + (rows + 1) * 4

    alg = {
        "pcg_spmv": (csr(nnz, n, 8) + 2 * n * 8, "CSR FP64: nnz*(8+4) + (n+1)*4 + n*8 gathered p + n*8 q written"),
        "mg_smooth": (csr(nnz, n, sv) + n * sx * 4, "CSR: nnz*(s_v+4) + (n+1)*4 + x gathered, x' written, b and D read"),
        "mg_defect": (csr(nnz, n, sv) + n * sx * 3, "CSR: nnz*(s_v+4) + (n+1)*4 + x gathered, d written, b read"),
        "mg_post1": (csr(nnz, n, sv) + n * sx * 5, "CSR: nnz*(s_v+4) + (n+1)*4 + x gathered, b and D read, d and c written"),
        "mg_post2": (csr(nnz, n, sv) + n * sx * 4 + n * 16,
                     "CSR: nnz*(s_v+4) + (n+1)*4 + c gathered, d, D, x read (s_x), r read and z written (FP64)"),
        "mg_restrict": (csr(nnz_r, nc, sv) + n * sx + nc * sx * 3,
                        "CSR of R: nnz_R*(s_v+4) + (n_c+1)*4 + d gathered, b_c and sol1_c written, D_c read"),
        "mg_prolong": (csr(nnz_p, n, sv) + nc * sx + 2 * n * sx,
                       "CSR of P: nnz_P*(s_v+4) + (n+1)*4 + x_c gathered, x read and written"),
        "mg_down": (csr(nnz, n, sv) + n * sx * 4 + csr(nnz_r, nc, sv) + nc * sx * 3,
                    "CSR of A once + x read, x2 written, b and D read + CSR of R + b_c, sol1_c written, D_c read"),
        "mg_up": (csr(nnz, n, sv) + csr(nnz_p, n, sv) + nc * sx + n * sx * 3 + n * 16,
                  "CSR of A once + CSR of P + x_c gathered + x2, b, D read (s_x) + r read and z written (FP64)"),
    }
    alg["mg_sdown"] = alg["mg_down"]
    alg["mg_sup"] = alg["mg_up"]
    out = {}
    fused = True
    for k, (by, definition) in alg.items():
        try:
            ms, stored = solver.time_kernel(k, reps=reps, flush_l2=True)
        except Exception:
            if k in FUSED_PASSES or k in STREAM_PASSES:   # the finest level is not a structured grid
                fused = False
                continue
            raise
        out[k] = {"kernel": PASS_KERNELS[k], "us": ms * 1e3, "csr_bytes": by, "csr_definition": definition,
                  "csr_gbs": by / (ms * 1e-3) / 1e9, "stored_bytes": stored, "stored_gbs": stored / (ms * 1e-3) / 1e9}
    # which of them the solve launches on the finest level
    tiled = fused and solver.cfg.fused >= n
    streamed = fused and not tiled and 0 < solver.cfg.streamed <= n
    for k in out:
        kind = "tiled" if k in FUSED_PASSES else ("streamed" if k in STREAM_PASSES else "unfused")
        out[k]["in_solve"] = k == "pcg_spmv" or kind == ("tiled" if tiled else ("streamed" if streamed else "unfused"))
    return out


def run_target(args, batch, flush, torch, fb, stream):
    """The method's target measured on the uneven-instance family (256 instances, levels 5..9,
    kappa fields): arm A = the plain FP64 drop-in solver on every instance one after the other (a
    solver per instance, each solve timed alone on the device with a cold L2); arm B = the same
    instances in one FP32-in-FP64 batched solve.  Both stop at 1e-8 relative residual per instance.
    Returns the comparison (ms per set, ratio, largest error of arm B against arm A's FP64
    solution)."""
    levels, inst = batch
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    xs_a, t_a, it_a, ok_a = [], [], [], True
    for lv, b in inst:
        s = fb.build_pcg_multigrid(lv, precision="f64", ordering="native")
        rhs = torch.tensor(b, device="cuda")
        x = torch.zeros_like(rhs)
        s.correct_device(x, rhs, stream)                  # warm-up (untimed)
        flush()
        x.zero_()
        ev0.record(stream)
        st = s.correct_device(x, rhs, stream)
        ev1.record(stream)
        ev1.synchronize()
        t_a.append(ev0.elapsed_time(ev1))
        it_a.append(s.get_num_iter())
        ok_a = ok_a and st == fb.Status.success
        xs_a.append(x.cpu().numpy())
        s.done()
    hs = [fb.build_hierarchy(lv) for lv, _ in inst]
    bat = fb.BatchPCG(hs, precision="f32", ordering="native")
    rhs = torch.tensor(np.concatenate([b for _, b in inst]), device="cuda")
    sol = torch.zeros_like(rhs)
    for _ in range(args.warmup):
        sol.zero_()
        bat.solve_device(sol, rhs, stream)
    t_b = []
    for _ in range(max(3, min(args.steps, 10))):
        flush()
        sol.zero_()
        ev0.record(stream)
        bat.solve_device(sol, rhs, stream)
        ev1.record(stream)
        ev1.synchronize()
        t_b.append(ev0.elapsed_time(ev1))
    xb = bat.split(sol.cpu().numpy())
    err = max(float(np.linalg.norm(xb[k] - xs_a[k]) / np.linalg.norm(xs_a[k])) for k in range(len(inst)))
    its_b = bat.iterations()
    ok_b = all(st == fb.Status.success for st in bat.statuses())
    bat.done()
    ms_a, ms_b = float(np.sum(t_a)), float(np.mean(t_b))
    return {"family": f"{len(inst)} -div(kappa grad u)=f instances, levels uniform in 5..9 (seed 7), kappa = "
                      "exp(16x16-mode field), 8-Gaussian f; stop at 1e-8 relative residual per instance",
            "instances": len(inst), "dofs": int(sum(b.size for _, b in inst)),
            "plain_fp64_ms": ms_a, "plain_fp64_definition": "sum over the instances of one FP64 PCG-multigrid solve "
                                                            "each (device time, cold L2, solver set-up excluded)",
            "batched_mixed_ms": ms_b, "batched_mixed_definition": "one FP32-in-FP64 batched solve of all instances "
                                                                  "(device time, cold L2, mean of the timed repeats)",
            "ratio": ms_a / ms_b, "plain_solves_per_s": len(inst) * 1e3 / ms_a,
            "batched_solves_per_s": len(inst) * 1e3 / ms_b,
            "max_rel_err_vs_fp64": err, "error_reference": "arm A's FP64 solutions (the plain path, pinned to the "
                                                           "FP64 oracle within 1e-12 by the tests)",
            "iterations_plain": [int(min(it_a)), int(max(it_a))], "iterations_batched": [int(min(its_b)), int(max(its_b))],
            "all_success": bool(ok_a and ok_b), "warm_start": "not used (it does not pay at this accuracy)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default=DEFAULT_WORKLOAD)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 comparison solve")
    ap.add_argument("--profile-solves", type=int, default=0,
                    help="only run warm-up + this many solves (for a profiler's launch list), print nothing else")
    ap.add_argument("--profile-kernel", default=None, choices=sorted(PASS_KERNELS) + ["mg_tail"],
                    help="only launch this finest-level pass a few times alone (for a profiler), print nothing else")
    ap.add_argument("--tail-rows", type=int, default=None)
    ap.add_argument("--tma-rows", type=int, default=None,
                    help="levels with at least this many rows use the TMA-staged passes")
    ap.add_argument("--cluster-rows", type=int, default=None,
                    help="levels with at most this many rows run in the cluster tail kernel (0 = off)")
    ap.add_argument("--tma-window", type=int, choices=[0, 1, 2], default=0,
                    help="gathered-vector window of a TMA chunk: 2 prefetch into L2, 1 stage in shared memory, 0 none")
    ap.add_argument("--diagonal", type=int, choices=[0, 1], default=1,
                    help="diagonal storage of system matrices on at most 27 diagonals (1) or sliced ELL (0)")
    ap.add_argument("--fused-rows", type=int, default=None,
                    help="structured 2D levels with at most this many rows run fused V(2,2) passes "
                         "(default: the library's threshold; 0 = one pass per step everywhere)")
    ap.add_argument("--streamed-rows", type=int, default=None,
                    help="structured 2D levels above the fused threshold with at least this many rows run "
                         "the streamed fused passes (default: the library's threshold; 0 = never)")
    ap.add_argument("--pdl", type=int, choices=[0, 1], default=1,
                    help="programmatic dependent launch of the solve's kernels (1) or plain stream order (0)")
    ap.add_argument("--cycle", choices=["V", "F", "W"], default="V",
                    help="multigrid cycle of the preconditioner (the reference's MultiGridCycle)")
    ap.add_argument("--ordering", choices=["native", "rcm"], default="native",
                    help="device DOF ordering (the generated problems are numbered lexicographically)")
    ap.add_argument("--ws-train", type=int, default=20000, help="training instances (learned warm start)")
    ap.add_argument("--ws-epochs", type=int, default=20)
    ap.add_argument("--ws-eval", type=int, default=1000, help="unseen evaluation instances")
    ap.add_argument("--no-target", action="store_true",
                    help="skip the plain-FP64 vs batched-mixed comparison on the uneven-instance family")
    ap.add_argument("--target-count", type=int, default=256, help="instances of that comparison")
    ap.add_argument("--batch-count", type=int, default=256, help="instances of the batch workload")
    ap.add_argument("--reference-backend", choices=["generic", "cuda"], default="generic",
                    help="with --impl reference: the reference's generic CPU backend (default) or its own CUDA "
                         "backend (cuSPARSE / cuBLAS, built by `make -C oracle cuda`)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "poisson2d_l9_warmstart":
        return run_warmstart(args)
    if args.workload in ("poisson2d_batch256_mixed", "poisson3d_l6_rhs64_mixed"):
        return run_multi(args, "batch" if "batch" in args.workload else "rhs64")

    # the target comparison's instances are assembled on host worker processes while the main
    # workload's problem is assembled (single-GPU runs of the default workload only)
    started = None
    if (not args.no_target and not args.profile_solves and not args.profile_kernel and dist_env()[1] == 1
            and args.workload == DEFAULT_WORKLOAD):
        started = start_batch_build(args.target_count)

    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
        pg = dist
    import featb200 as fb

    dim, level, rhs_kind, precision, desc = WORKLOADS[args.workload]
    levels, b, gauss = build_problem(dim, level, rhs_kind)
    n = b.size
    # every timed region runs with idle host cores: the instance build finishes first
    batch = finish_batch_build(started) if started is not None else None
    # a profiler cannot see the kernels of a graph with a device-side loop: profile runs launch per kernel
    solver = fb.build_pcg_multigrid(levels, precision=precision, ordering=args.ordering, tail_rows=args.tail_rows,
                                    use_graph=not args.profile_solves, tma_window=args.tma_window,
                                    cluster_rows=args.cluster_rows, tma_rows=args.tma_rows, cycle=args.cycle,
                                    diagonal=args.diagonal, pdl=args.pdl, fused=args.fused_rows,
                                    streamed=args.streamed_rows)
    info_lv = solver.level_info()
    if args.profile_kernel:
        ms_k, by_k = solver.time_kernel(args.profile_kernel, reps=3, flush_l2=True)
        print(json.dumps({"profile_kernel": args.profile_kernel, "us": ms_k * 1e3, "stored_bytes": by_k}))
        return 0

    stream = torch.cuda.current_stream()
    rhs_d = torch.tensor(b, device="cuda")
    sol_d = torch.zeros_like(rhs_d)
    flush = L2Flush(torch)

    def one_step():
        sol_d.zero_()
        st = solver.correct_device(sol_d, rhs_d, stream)
        return st

    clocks = ClockSampler(local)
    if not args.profile_solves:
        clocks.start()
    for _ in range(args.warmup):
        st = one_step()
    torch.cuda.synchronize()
    if args.profile_solves:
        for _ in range(args.profile_solves):
            one_step()
        torch.cuda.synchronize()
        print(json.dumps({"profile_solves": args.profile_solves, "iterations": solver.get_num_iter()}))
        return 0
    if pg:
        pg.barrier()
    time.sleep(0.3)
    wall0 = time.time()
    launches0 = fb.launch_count()
    times = []
    iters = []
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    for _ in range(args.steps):
        flush()                                          # cold, clean L2 for every solve (not timed)
        ev0.record(stream)
        st = one_step()
        ev1.record(stream)
        ev1.synchronize()
        times.append(ev0.elapsed_time(ev1))
        iters.append(solver.get_num_iter())
        if st != fb.Status.success:
            raise SystemExit(f"solve failed: {st}")
    torch.cuda.synchronize()
    launches = fb.launch_count() - launches0
    wall1 = time.time()
    time.sleep(0.3)
    clk = clocks.stop(wall0, wall1)
    total_ms = float(np.sum(times))
    if pg:
        t = torch.tensor([total_ms], device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        total_ms = float(t.item())
        pg.barrier()
    ms_per_step = total_ms / args.steps
    value = ms_per_step / world

    # accuracy against the residual and the FP64 solution
    x = sol_d.cpu().numpy()
    A = levels[0]["matrix"].to_scipy()
    r = b - A @ x
    r[levels[0]["filter"].indices.astype(np.int64)] = 0.0
    rel_res = float(np.linalg.norm(r) / np.linalg.norm(b))

    extra = {}
    if not args.no_plain and precision != "f64":
        plain = fb.build_pcg_multigrid(levels, precision="f64", ordering=args.ordering, tma_window=args.tma_window,
                                       diagonal=args.diagonal, pdl=args.pdl, fused=args.fused_rows,
                                    streamed=args.streamed_rows)
        pt = []
        for k in range(args.warmup + max(3, args.steps // 2)):
            flush()
            sol2 = torch.zeros_like(rhs_d)
            ev0.record(stream)
            plain.correct_device(sol2, rhs_d, stream)
            ev1.record(stream)
            ev1.synchronize()
            if k >= args.warmup:
                pt.append(ev0.elapsed_time(ev1))
        x64 = sol2.cpu().numpy()
        extra["plain_fp64_ms"] = float(np.mean(pt))
        extra["plain_fp64_iterations"] = plain.get_num_iter()
        extra["speedup_vs_plain_fp64"] = extra["plain_fp64_ms"] / ms_per_step
        extra["error_vs_fp64"] = float(np.abs(x - x64).max() / np.abs(x64).max())
        plain.done()

    # every finest-level pass timed alone on the solver's stream with a cold L2: the roofline kernel
    # is the one with the largest time per solve (each runs once per V-cycle / PCG iteration)
    peak, peak_kind = read_peaks()
    passes = pass_table(solver, levels, precision)
    dom = max((k for k in passes if passes[k]["in_solve"]), key=lambda k: passes[k]["us"])
    dp = passes[dom]
    traffic = MEASURED_TRAFFIC.get((args.workload, args.ordering, dom))
    spmv_gbs = {"pcg_spmv_f64": passes["pcg_spmv"]["csr_gbs"],
                "mg_defect_" + precision: passes["mg_defect"]["csr_gbs"]}
    # where a preconditioner application goes: one whole cycle, and its coarse-level tail kernel
    breakdown = {"mg_cycle_us": solver.time_kernel("mg_cycle", reps=20, flush_l2=False)[0] * 1e3}
    if args.tail_rows != 0 and args.cluster_rows in (None, 0):
        breakdown["mg_tail_us"] = solver.time_kernel("mg_tail", reps=20, flush_l2=False)[0] * 1e3
        breakdown["mg_tail_us_cold_l2"] = solver.time_kernel("mg_tail", reps=20, flush_l2=True)[0] * 1e3
    # the whole solve: bytes the launched kernels move as stored (solver's own count) / device time
    solve_bytes = float(solver.info.bytes_moved)
    solve_gbs = solve_bytes / (ms_per_step * 1e-3) / 1e9
    whole_solve = {"bytes_stored": solve_bytes, "ms": ms_per_step, "gbs": solve_gbs, "frac": solve_gbs / peak,
                   "definition": "sum over the solve's launches of the matrix bytes as stored + gathered vector + "
                                 "row-wise vectors + masks, divided by the device time of the solve"}

    # end to end through the C ABI with host buffers (copies inside the timed region)
    pin_rhs = torch.tensor(b).pin_memory()
    pin_sol = torch.zeros(n, dtype=torch.float64).pin_memory()
    e2e_t = []
    for k in range(args.warmup + args.steps):
        flush()
        torch.cuda.synchronize()
        pin_sol.zero_()
        t0 = time.perf_counter()
        xs = fb.DenseVector(pin_sol.numpy())
        solver.correct(xs, fb.DenseVector(pin_rhs.numpy()))
        t1 = time.perf_counter()
        if k >= args.warmup:
            e2e_t.append((t1 - t0) * 1e3)
    e2e_ms = float(np.mean(e2e_t))

    target = run_target(args, batch, flush, torch, fb, stream) if batch is not None else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        res = cpu_reference_times(dim, level, rhs_kind, gauss, 5)
        if res is not None:
            cpu = {"value": float(np.median(res["times_ms"][1:] or res["times_ms"])), "unit": "ms", "cores": 1,
                   "kind": "reference",
                   "sample": f"{len(res['times_ms']) - 1} FP64 solves (after 1 warm-up) of the same problem by the "
                             f"reference's generic backend, single-threaded, solve only; {res['iters']} iterations"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "ms", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32+f64" if precision != "f64" else "f64", "data": "synthetic",
                "config": {"workload": args.workload + ": " + desc, "dofs": int(n),
                           "nnz": int(levels[0]["matrix"].used_elements()), "nnz_stored": int(info_lv[0][1]),
                           "levels": int(info_lv.shape[0]), "ordering": args.ordering, "precision": precision,
                           "cycle": args.cycle, "parallelism": f"replicas x{world}", "l2": L2Flush.DESC,
                           "iterations": int(np.median(iters))},
                "spmv_gbs": spmv_gbs, "rel_residual": rel_res, "breakdown": breakdown,
                "roofline": {"bound": "hbm", "kernel": dom, "kernel_name": dp["kernel"],
                             "achieved": dp["csr_gbs"], "peak": peak, "unit": "GB/s",
                             "frac": dp["csr_gbs"] / peak, "traffic": traffic,
                             "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch of this "
                                                "kernel at this workload, same kernel source" if traffic else None),
                             "traffic_frac": (traffic / (dp["us"] * 1e-6) / 1e9 / peak if traffic else None),
                             "peak_source": f"{peak_kind} hbm_gbs", "launch_us": dp["us"],
                             "bytes_per_launch": dp["csr_bytes"], "bytes_definition": dp["csr_definition"],
                             "stored_bytes_per_launch": dp["stored_bytes"],
                             "stored_frac": dp["stored_gbs"] / peak},
                "passes": passes, "whole_solve": whole_solve,
                "e2e": {"value": e2e_ms, "unit": "ms", "h2d_bytes_per_step": int(2 * 8 * n),
                        "d2h_bytes_per_step": int(8 * n)},
                "gpu_launches": int(launches), "clocks": clk}
        line.update(extra)
        if target is not None:
            line["target"] = target
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line))
    solver.done()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
