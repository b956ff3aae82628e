"""Benchmark: factor + solve of the 3D P1 elasticity system (40^3 hexes x 6 Kuhn tets, 201,720 DOFs, x = 0 clamped,
nested-dissection ordering) on one B200, FP64 and mixed precision + FP64 refinement, to relative residual <= 1e-12.

One step = one numeric factorization + the solve of the system's right-hand sides (with refinement) of the seeded
system; the symbolic analysis is per pattern and is reported separately (symbolic_ms), as the reference reuses it
across factorizations.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--precision fp64|mixed|both]
                  [--workload elastic3d|heat3d_p2|maxwell3d|heat2d_batch] [--size S]

Workloads (right-hand sides per step as the benchmark configurations state them): elastic3d 40^3 (1), heat3d_p2 48^3
(16), maxwell3d 32^3 LDL^T (64), heat2d_batch 256 problems (1-64 each).

With --gpus N > 1 (launched by torch.distributed.run) every rank solves its own replica of a single system ("replicas
only": one factorization does not shard), while the batched heat set is split over the ranks (each rank factors and
solves its share of the 256 independent problems; no data-path collective). Rank 0 prints the whole-job throughput.

--impl reference times the reference's algorithm on the host cores: the oracle (a C restatement of the reference,
with an SSE2 restatement of its WASM SIMD front and solve kernels), single-threaded as the reference is, ordering and
analysis by the oracle itself, each step one complete factorization + solve of the same system, as many steps as
fit a wall-clock budget.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "applied-multiphysics_b200"))

METRIC = "factor+solve TFLOP/s to rel. residual <= 1e-12 ({title}, 1 x B200)"
UNIT = "TFLOP/s"
RESIDUAL = 1e-12
# the benchmark systems: elasticity (the headline), P2 heat, Nedelec Maxwell (indefinite, LDL^T) and the batch
SYSTEMS = {
    "elastic3d": {"size": 40, "q": 1, "title": "3D P1 elasticity {N}^3", "kind": "chol",
                  "desc": "elastic3d-{N}: 3D P1 linear elasticity, {N}^3 hexes x 6 tets, E=1 nu=0.3, x=0 clamped, "
                          "nd3Order, 1 RHS"},
    "heat3d_p2": {"size": 48, "q": 16, "title": "3D P2 heat {N}^3, 16 RHS", "kind": "chol",
                  "desc": "heat3d-p2-{N}: 3D P2 (tet10) heat, {N}^3 hexes x 6 tets, k=100 in 64 seeded spheres "
                          "(r=0.05) else 1, Dirichlet x=0 and x=1, nd3Order, 16 RHS"},
    "heat2d_batch": {"size": 256, "q": None, "title": "batched 2D P1 heat, {N} problems", "kind": "batch",
                     "desc": "heat2d-batch-{N}: {N} P1 heat problems on unit squares, N ~ U{{16..128}} cells per side, "
                             "lognormal(0,1) conductivity, Dirichlet, 1-64 RHS each; AMD per matrix, one "
                             "block-diagonal factorization per GPU"},
    "maxwell3d": {"size": 32, "q": 64, "title": "3D Nedelec Maxwell {N}^3 LDL^T, 64 RHS", "kind": "ldlt",
                  "desc": "maxwell3d-{N}: lowest-order Nedelec curl-curl - k^2 eps_r mass, {N}^3 hexes x 6 tets, "
                          "eps_r=12 in 8 seeded boxes, PEC, k^2 between the 10th and 11th eigenvalues, nd3Order on "
                          "edge midpoints, 64 RHS"},
}
ORACLE_FULL_FLOPS = 1.2e12  # the oracle runs a complete factorization up to this size (about 2 min on one core)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0, "fallback": True}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = max(mx, float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


class _Batch:
    """The batched heat set (or one rank's share of it) as one block-diagonal system: pattern, values, max q_i RHS
    (zeros where a matrix has fewer), per-matrix AMD orders."""

    def __init__(self, count: int, rank: int = 0, world: int = 1, amd=None):
        import workloads as wl
        import batch
        import replicas
        ws = wl.heat2d_batch(count)
        # every rank computes the same split without communicating; cost ~ n^1.5 (2D nested-dissection flops)
        part = replicas.shard_batch([float(w.n) ** 1.5 for w in ws], world)[rank]
        ws = [ws[i] for i in part]
        self.count_all, self.count = count, len(ws)
        self.pat, offs, _ = batch.block_diagonal([w.pat for w in ws])
        self.values = np.concatenate([w.values for w in ws])
        q = max(w.rhs.shape[0] for w in ws)
        self.rhs = np.zeros((q, self.pat.n))
        for i, w in enumerate(ws):
            self.rhs[: w.rhs.shape[0], offs[i]: offs[i + 1]] = w.rhs
        if amd is None:
            import ampsolve as amp
            amd = amp.amdOrder
        self.perm = np.concatenate([amd(w.pat) + offs[i] for i, w in enumerate(ws)]).astype(np.int32)
        self.offs, self.q = offs, [w.rhs.shape[0] for w in ws]
        self.n = self.pat.n
        self.x = self.y = self.z = None


def make_system(name: str = "elastic3d", size: int = 40, rank: int = 0, world: int = 1, amd=None):
    import workloads as wl
    if name == "heat2d_batch":
        return _Batch(size, rank, world, amd)
    if name == "heat3d_p2":
        return wl.heat3d_p2(size, q=SYSTEMS[name]["q"])
    if name == "maxwell3d":
        return wl.maxwell3d(size, q=SYSTEMS[name]["q"])
    return wl.elastic3d(size, seed=2, q=1)


def solve_flops(colcount: np.ndarray, w) -> float:
    """4 nnzL per right-hand side (forward + backward); in the batch matrix i solves its own q_i vectors."""
    cc = colcount.astype(np.float64)
    if isinstance(w, _Batch):
        return float(sum(4.0 * cc[w.offs[i]: w.offs[i + 1]].sum() * qi for i, qi in enumerate(w.q)))
    return 4.0 * float(cc.sum()) * w.rhs.shape[0]


def measure_gemm(torch, dtype):
    """cuBLAS GEMM 8192^3 (DGEMM: the FP64 tensor-core denominator; SGEMM with TF32 off: the FP32 CUDA-core one)."""
    torch.backends.cuda.matmul.allow_tf32 = False
    a = torch.randn(8192, 8192, dtype=dtype, device="cuda")
    b = torch.randn_like(a)
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(5):
        a @ b
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / 5
    del a, b
    torch.cuda.empty_cache()
    return 2 * 8192 ** 3 / ms / 1e9


def _pin_one_core():
    try:
        keep = os.sched_getaffinity(0)
        os.sched_setaffinity(0, {min(keep)})
        return keep
    except (AttributeError, OSError):
        return None


def oracle_step(orc, so, w, kind: str):
    """The reference's numeric phase restated by the oracle: factor (SSE2 WASM front kernel), solve every right-hand
    side (SSE2 WASM solve kernels; LDL^T: all vectors in one solveMany sweep), then the reference's solveRefined for
    any vector above the tolerance. Returns (seconds, X (q, n), worst relative residual)."""
    B = w.rhs
    q, n = B.shape
    t0 = time.perf_counter()
    ok, Lx, D, _, _ = orc.factor(so, w.values, kind=kind, simd=True)
    if not ok:
        raise RuntimeError("oracle factorization failed")
    if kind == "ldlt":
        X = orc.solve_ldlt(so, Lx, D, np.ascontiguousarray(B).reshape(-1), q=q, simd=True).reshape(q, n).copy()
    else:
        X = np.stack([orc.solve_chol(so, Lx, B[k], simd=True) for k in range(q)])
    worst = 0.0
    for k in range(q):
        bn = float(np.linalg.norm(B[k])) or 1.0
        rr = float(np.linalg.norm(orc.matvec(w.pat, w.values, X[k]) - B[k])) / bn
        if rr >= RESIDUAL:
            X[k], rr, _ = orc.solve_refined(so, w.pat, w.values, Lx, D, B[k], kind=kind, max_steps=3, tol=RESIDUAL)
        worst = max(worst, rr)
    return time.perf_counter() - t0, X, worst


def _subtree_flops(so) -> np.ndarray:
    cc2 = so.colCount.astype(np.float64) ** 2
    sub = np.add.reduceat(cc2, so.superStart[:-1]) if so.nsuper else np.zeros(0)
    for s in range(so.nsuper):
        p = so.superParent[s]
        if p >= 0:
            sub[p] += sub[s]
    return sub


def _small_subtree(so, target: float = 2e8) -> int:
    sub = _subtree_flops(so)
    order = np.argsort(sub)
    return int(order[np.searchsorted(sub[order], target)]) if np.any(sub >= target) else int(order[-1])


def oracle_sample(orc, so, w, kind: str, budget_s: float = 20.0):
    """A bounded CPU sample for systems too large to factor whole on one core: the factorization of the largest
    complete subtree whose estimated time fits the budget. Returns (TFLOP/s, description)."""
    sub = _subtree_flops(so)
    small = _small_subtree(so)
    t = time.perf_counter()
    orc.factor_subtree(so, w.values, small, kind=kind, simd=True)
    rate = sub[small] / max(time.perf_counter() - t, 1e-6)
    cand = np.where(sub <= rate * budget_s)[0]
    root = int(cand[np.argmax(sub[cand])]) if cand.size else small
    t = time.perf_counter()
    _, fl = orc.factor_subtree(so, w.values, root, kind=kind, simd=True)
    dt = time.perf_counter() - t
    return fl / dt / 1e12, (f"factor of the subtree of supernode {root} ({fl:.3e} of {so.flops:.3e} flops, {dt:.1f} s; "
                            f"the whole system is too large for one core within the run)")


def oracle_analysis(orc, w):
    """The oracle's own ordering (nd3Order, or AMD per matrix for the batch) and analysis."""
    if isinstance(w, _Batch):
        return orc.analyze(w.pat, perm=w.perm)
    return orc.analyze(w.pat, perm=orc.nd3_order(w.pat, w.x, w.y, w.z))


def run_reference(args, rank):
    """The reference arm: complete oracle steps (factor + solve) on one pinned core until the budget is spent."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    w = make_system(args.workload, args.size, amd=orc.amd_order)
    kind = "ldlt" if args.ldlt else "chol"
    so = oracle_analysis(orc, w)
    work = so.flops + solve_flops(so.colCount, w)
    keep = _pin_one_core()
    # warm-up: W factorizations of a small subtree (the library's code and allocator paths; a complete step of the
    # benchmark system takes a minute or more on one core, so the complete steps below are all timed)
    small = _small_subtree(so)
    for _ in range(args.warmup):
        orc.factor_subtree(so, w.values, small, kind=kind, simd=True)
    times = []
    t_all = time.perf_counter()
    if so.flops <= ORACLE_FULL_FLOPS:
        while len(times) < args.steps:
            dt, _, worst = oracle_step(orc, so, w, kind)
            times.append(dt)
            elapsed = time.perf_counter() - t_all
            if elapsed + dt > args.ref_budget:  # the next step would not fit the budget
                break
        ms = 1e3 * float(np.mean(times))
        value = work / (ms * 1e-3) / 1e12
        sample = (f"{len(times)} complete factor + solve steps of the whole system ({so.flops:.3e} factor flops, "
                  f"{w.rhs.shape[0]} RHS, worst rel. residual {worst:.1e}); oracle ordering and analysis; SSE2 "
                  f"restatement of the reference's WASM kernels, 1 pinned thread")
    else:
        value, sample = oracle_sample(orc, so, w, kind)
        ms, times = None, []
    if keep:
        os.sched_setaffinity(0, keep)
    line = {"impl": "reference", "metric": args.metric, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": len(times), "steps_requested": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": args.desc, "n": w.n, "nnz": w.pat.nnz, "flops_factor": so.flops,
                       "rhs": int(w.rhs.shape[0]), "sample": sample,
                       "warmup": "factorizations of a small subtree", "budget_s": args.ref_budget,
                       # every timed step is a complete factor + solve of the whole system, all inside this run
                       "fits_in_driver_run": bool(times)},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# DRAM bytes per launch of the roofline kernel (dram__bytes_read.sum + dram__bytes_write.sum from one ncu capture;
# profiles/ names the command). Keyed by (workload, size, precision, kernel class).
# DRAM bytes per launch of the dominant kernel: the largest tcgen05 update launch of an elastic3d-32 mixed factor moves
# 169.3 MB for 26.2 GFLOP (ncu dram__bytes_read.sum + dram__bytes_write.sum), scaled by the flops of an average cfg2
# update launch (764.6 GFLOP over 183 launches)
TRAFFIC = {
    ("elastic3d", 40, "mixed", "update_syrk"): 169.3e6 / 26.2e9 * 764.6e9 / 183,
    # the group panel: its longest elastic3d-32 launch moves 22.9 MB for 0.602 GFLOP, scaled by the flops of an average
    # cfg2 group-panel launch (26.8 GFLOP over 157 launches)
    ("elastic3d", 40, "mixed", "group_panel"): 22.9e6 / 0.602e9 * 26.8e9 / 157,
}


def schedule_kw(args) -> dict:
    """analyze options of --schedule G,S,D (pivot blocks per group, largest whole front, deferral of part B)"""
    if not args.schedule:
        return {}
    g, sf, d = (int(v) for v in args.schedule.split(","))
    return {"groupBlocks": g, "smallFront": sf, "deferUpdates": d}


def one_factor(args, w, amp, local):
    if isinstance(w, _Batch):
        sym = amp.analyze(w.pat, perm=w.perm, device=local, **schedule_kw(args))
    else:
        sym = amp.analyze(w.pat, ordering="nd3", x=w.x, y=w.y, z=w.z, device=local, **schedule_kw(args))
    prec = amp.FP64 if args.precision == "fp64" else amp.MIXED
    num = amp.NumericFactor(sym, amp.LDLT if args.ldlt else amp.CHOLESKY, prec)
    num.profile(True)  # direct launches, each bracketed by events, in stream order
    ok = num.factor(w.values)
    k, ms, fl = num.profile_launches()
    out = {"workload": args.desc, "ok": ok}
    for name, kind in (("group_panel", 1), ("update", 2), ("assemble", 0)):
        idx = np.where(k == kind)[0]
        if idx.size:
            j = int(np.argmax(ms[idx]))
            out[name] = {"launches": int(idx.size), "longest_index": j, "longest_ms": float(ms[idx][j]),
                         "longest_tflops": float(fl[idx][j] / ms[idx][j] / 1e9), "total_ms": float(ms[idx].sum())}
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="both", choices=["fp64", "fp64-bk", "mixed", "both"],
                    help="both: fp64 and mixed, and for an LDL^T workload also fp64-bk (FP64 LDL^T with Bunch-Kaufman "
                         "pivots inside each pivot block)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="elastic3d", choices=sorted(SYSTEMS))
    ap.add_argument("--size", type=int, default=0, help="hexes per side, or problems of the batch (0 = benchmark size)")
    ap.add_argument("--ref-budget", type=float, default=240.0, help="wall seconds of the reference arm's steps")
    ap.add_argument("--no-autotune", action="store_true", help="the default schedule instead of the autotuned one")
    ap.add_argument("--schedule", default="",
                    help="G,S,D: a given schedule for every precision instead of the autotuned one (pivot blocks per "
                         "group panel, largest whole front, part-B deferral), e.g. 2,128,4")
    ap.add_argument("--one-factor", action="store_true",
                    help="profiling case: one factorization of the workload (first precision of --precision) with "
                         "direct launches in stream order; prints the per-class launch index of the longest group "
                         "panel and update (the -s of an ncu capture)")
    args = ap.parse_args()
    sysinfo = SYSTEMS[args.workload]
    args.size = args.size or sysinfo["size"]
    args.metric = METRIC.format(title=sysinfo["title"].format(N=args.size))
    args.desc = sysinfo["desc"].format(N=args.size)
    args.ldlt = sysinfo["kind"] == "ldlt"
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    import torch
    import torch.distributed as dist

    import ampsolve as amp

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    w = make_system(args.workload, args.size, rank, world)
    if args.one_factor:
        one_factor(args, w, amp, local)
        return
    n = w.n
    nq = w.rhs.shape[0]
    t0 = time.perf_counter()
    if isinstance(w, _Batch):
        sym = amp.analyze(w.pat, perm=w.perm, device=local)
    else:
        sym = amp.analyze(w.pat, ordering="nd3", x=w.x, y=w.y, z=w.z, device=local)
    symbolic_ms = (time.perf_counter() - t0) * 1e3
    flops_factor = sym.flops
    work = flops_factor + solve_flops(sym.colCount, w)  # the same algorithmic work for both precisions

    precisions = (["fp64", "fp64-bk", "mixed"] if args.ldlt else ["fp64", "mixed"]) if args.precision == "both" \
        else [args.precision]
    results = {}
    dev = torch.device("cuda", local)
    vals_d = torch.from_numpy(w.values).to(dev)
    b_d = torch.from_numpy(np.ascontiguousarray(w.rhs).reshape(-1)).to(dev)
    x_d = torch.empty_like(b_d)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2
    tuning = {}
    for prec in precisions:
        kind, precision = amp.LDLT if args.ldlt else amp.CHOLESKY, amp.MIXED if prec == "mixed" else amp.FP64
        if prec == "fp64-bk":
            kind = amp.LDLT_BK
        psym = sym
        # the schedule per precision, chosen by timing candidates (per pattern, not timed)
        if args.schedule:
            if isinstance(w, _Batch):
                psym = amp.analyze(w.pat, perm=w.perm, device=local, **schedule_kw(args))
            else:
                psym = amp.analyze(w.pat, ordering="nd3", x=w.x, y=w.y, z=w.z, device=local, **schedule_kw(args))
        elif not args.no_autotune:
            if isinstance(w, _Batch):
                psym = amp.analyze(w.pat, perm=w.perm, device=local)
            else:
                psym = amp.analyze(w.pat, ordering="nd3", x=w.x, y=w.y, z=w.z, device=local)
            tuning[prec] = amp.autotune(psym, w.values, kind, precision)
        num = amp.NumericFactor(psym, kind, precision)
        if isinstance(w, _Batch):
            num.set_row_groups(w.offs)  # the residual is measured per matrix

        # mixed precision, one right-hand side: GMRES-IR (the mixed factor as right preconditioner, FP64 Arnoldi and
        # residuals on the device): fewer solves than plain refinement to reach 1e-12, and it converges for
        # indefinite systems, where plain refinement need not. Several right-hand sides use plain refinement with
        # all vectors in each sweep.
        gmres = prec == "mixed" and nq == 1

        def solve(bp, xp, on_device):
            if gmres:
                rr, its, _ = num.solve_gmres_ptr(bp, xp, on_device, tol=RESIDUAL, restart=40, maxIter=300)
                return rr, its
            if on_device:
                return num.solve_refined_device(bp, xp, nq, maxSteps=10, tol=RESIDUAL)
            return num.solve_refined_host_pinned(bp, xp, nq, 10, RESIDUAL)

        def step():
            ok = num.factor((vals_d.data_ptr(), vals_d.numel()), on_device=True)
            relres, steps = solve(b_d.data_ptr(), x_d.data_ptr(), True)
            return ok, relres, steps

        for _ in range(args.warmup):
            ok, relres, irs = step()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        with ClockSampler(local) as clk:
            for k in range(args.steps):
                flush.zero_()
                torch.cuda.synchronize()
                ev[k][0].record()
                ok, relres, irs = step()  # synchronous library calls on the factor's own stream
                ev[k][1].record()
                torch.cuda.synchronize()
        ms = float(np.mean([a.elapsed_time(b) for a, b in ev]))
        if world > 1:
            t = torch.tensor([ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        # end to end through the C ABI with host buffers (pinned): H2D values + b, D2H x, every step
        vals_h = torch.from_numpy(w.values).pin_memory()
        b_h = torch.from_numpy(np.ascontiguousarray(w.rhs).reshape(-1)).pin_memory()
        x_h = torch.empty_like(b_h).pin_memory()
        e2e = []
        for k in range(max(2, args.steps)):
            flush.zero_()
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            num.factor(vals_h.numpy())  # H2D of the values inside the call
            rr, ss = solve(b_h.data_ptr(), x_h.data_ptr(), False)  # H2D b, D2H x inside the call
            b.record()
            torch.cuda.synchronize()
            e2e.append(a.elapsed_time(b))
        e2e_ms = float(np.mean(e2e[1:])) if len(e2e) > 1 else e2e[0]
        if world > 1:
            t = torch.tensor([e2e_ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_ms = float(t.item())
        # profile pass: per-kernel device time with CUDA events on the factor's stream
        num.profile(True)
        num.factor((vals_d.data_ptr(), vals_d.numel()), on_device=True)
        solve(b_d.data_ptr(), x_d.data_ptr(), True)
        prof = num.profile_read()
        num.profile(False)
        xsol = x_d.cpu().numpy().reshape(nq, n)
        results[prec] = {"ok": ok, "ms": ms, "relres": relres, "ir_steps": irs, "clk": clk.summary(),
                         "converged": bool(ok and relres <= RESIDUAL),
                         "refinement": "gmres-ir (iterations)" if gmres else "ir (steps)",
                         "prof": prof, "e2e_ms": e2e_ms, "factor_ms": num.ms, "x": xsol}
        del num, psym
    # units processed by all ranks: a replica each, or each rank's share of the batch
    total_work = work
    if world > 1:
        t = torch.tensor([work], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        total_work = float(t.item())
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    # the headline is the faster of the paths that reached the residual bar (both are in the line)
    valid = [p for p in results if results[p]["converged"]] or list(results)
    head = min(valid, key=lambda p: results[p]["ms"])
    R = results[head]
    pk = peaks()
    dom = max(R["prof"], key=lambda k: k["ms"])
    fp64_peak = measure_gemm(torch, torch.float64)
    fp32_peak = measure_gemm(torch, torch.float32)
    if dom["flops"] > 0 and dom["name"] == "update_syrk" and head == "mixed":
        peak, bound, punit, note = pk.get("bf16_tflops_sustained", 1400.0), "tensor", "TFLOP/s", \
            ("MEASURED_PEAKS.json bf16_tflops_sustained" if "fallback" not in pk else "fallback 1400") + \
            " (BF16 tensor; 3 products per FP32 update counted once)"
    elif dom["flops"] > 0 and head == "mixed":
        peak, bound, punit, note = fp32_peak, "fp32", "TFLOP/s", "measured cuBLAS SGEMM 8192^3 (no TF32) in this run"
    elif dom["flops"] > 0:
        peak, bound, punit, note = fp64_peak, "tensor", "TFLOP/s", "measured cuBLAS DGEMM 8192^3 in this run"
    if dom["flops"] > 0:
        achieved = dom["flops"] / (dom["ms"] * 1e-3) / 1e12
    else:
        achieved, bound, punit, peak, note = dom["bytes"] / (dom["ms"] * 1e-3) / 1e9, "hbm", "GB/s", pk["hbm_gbs"], \
            "MEASURED_PEAKS.json hbm_gbs" if "fallback" not in pk else "fallback 6650 GB/s"
    launches = sum(k["launches"] for k in R["prof"])
    line = {
        "metric": args.metric, "value": total_work / (R["ms"] * 1e-3) / 1e12, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": R["ms"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+bf16x3 (f64 refinement)" if head == "mixed" else "f64", "data": "synthetic",
        "config": {"workload": args.desc, "n": n, "nnz": w.pat.nnz, "nnzL": sym.nnzL, "rhs": int(nq),
                   "flops_factor": flops_factor, "flops_step": work,
                   "maxFront": sym.maxFront, "nsuper": sym.nsuper, "levels": sym.nlevels, "precision": head,
                   "l2": "flushed between timed steps (256 MB write)",
                   "parallelism": ("batch split over ranks" if isinstance(w, _Batch) else "replicas")
                   if world > 1 else "1 gpu",
                   "symbolic_ms": symbolic_ms,
                   "schedule": {p: {"group_blocks": t["groupBlocks"], "small_front": t["smallFront"],
                                    "defer_updates": t["deferUpdates"],
                                    "factor_ms_tuned": t["msBest"], "factor_ms_default": t["msDefault"]}
                                for p, t in tuning.items()} or (f"given (--schedule {args.schedule})" if args.schedule
                                                                else "default (group 4 x 64 columns, whole fronts <= 128)")},
        "relres": R["relres"], "ir_steps": R["ir_steps"], "factor_ms": R["factor_ms"],
        "e2e": {"value": total_work / (R["e2e_ms"] * 1e-3) / 1e12, "unit": UNIT,
                "h2d_bytes_per_step": int(8 * w.pat.nnz + 8 * n * nq), "d2h_bytes_per_step": int(8 * n * nq),
                "ms_per_step": R["e2e_ms"]},
        "gpu_launches": int(launches * args.steps),
        "clocks": R["clk"],
        "roofline": {"bound": bound, "kernel": dom["name"], "achieved": achieved, "peak": peak, "unit": punit,
                     "frac": achieved / peak, "traffic": TRAFFIC.get((args.workload, args.size, head, dom["name"])),
                     "peak_source": note},
        "kernels": R["prof"],
        "fp64_dgemm_tflops": fp64_peak,
        "fp32_sgemm_tflops": fp32_peak,
    }
    import scipy.sparse as sp
    A = sp.csr_matrix((w.values, w.pat.colidx, w.pat.rowptr), shape=(n, n))
    anorm = float(np.sqrt(np.sum(w.values * w.values)))
    for p, r in results.items():
        X = r["x"]
        be = max(float(np.linalg.norm(w.rhs[k] - A @ X[k]) / (anorm * np.linalg.norm(X[k]) + np.linalg.norm(w.rhs[k])))
                 for k in range(nq))
        line[p] = {"ms_per_step": r["ms"], "value": total_work / (r["ms"] * 1e-3) / 1e12, "relres": r["relres"],
                   "ir_steps": r["ir_steps"], "refinement": r["refinement"], "factor_ms": r["factor_ms"],
                   "ok": r["ok"], "converged": r["converged"], "backward_error": be}
    if world == 1 and not args.no_cpu_baseline:
        # the CPU baseline (the oracle, 1 pinned core): a complete factor + solve when it fits the run, which also
        # gives the FP64 reference solution for the forward errors; else a bounded subtree sample
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as orc
        kind = "ldlt" if args.ldlt else "chol"
        so = orc.analyze(w.pat, perm=sym.perm)
        keep = _pin_one_core()
        if so.flops <= ORACLE_FULL_FLOPS:
            dt, Xo, worst = oracle_step(orc, so, w, kind)
            cb_value = work / dt / 1e12
            sample = (f"one complete factor + solve of the whole system ({dt:.1f} s, {nq} RHS, worst rel. residual "
                      f"{worst:.1e}); SSE2 restatement of the reference's WASM kernels, 1 pinned thread")
            for p, r in results.items():
                line[p]["forward_error_vs_oracle"] = max(
                    float(np.linalg.norm(r["x"][k] - Xo[k]) / max(np.linalg.norm(Xo[k]), 1e-300)) for k in range(nq))
        else:
            cb_value, sample = oracle_sample(orc, so, w, kind)
        if keep:
            os.sched_setaffinity(0, keep)
        line["cpu_baseline"] = {"value": cb_value, "unit": UNIT, "cores": 1, "kind": "port", "sample": sample}
    if "fp64" in results and "mixed" in results:
        Xm, Xd = results["mixed"]["x"], results["fp64"]["x"]
        line["mixed"]["forward_error_vs_fp64"] = max(
            float(np.linalg.norm(Xm[k] - Xd[k]) / max(np.linalg.norm(Xd[k]), 1e-300)) for k in range(nq))
        line["mixed_vs_fp64_speedup"] = results["fp64"]["ms"] / results["mixed"]["ms"]
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
