"""Benchmark: factor + solve of the 3D P1 elasticity system (40^3 hexes x 6 Kuhn tets, 201,720 DOFs, x = 0 clamped,
nested-dissection ordering) on one B200, FP64 and mixed precision + FP64 refinement, to relative residual <= 1e-12.

One step = one numeric factorization + one solve (with refinement) of the seeded system; the symbolic analysis is
per pattern and is reported separately (symbolic_ms), as the reference reuses it across factorizations.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--precision fp64|mixed|both]

With --gpus N > 1 (launched by torch.distributed.run) every rank solves its own replica of the system (the path does
not shard; "replicas only") and rank 0 prints the whole-job throughput. --impl reference times the reference's
algorithm on the host cores: the oracle (a C restatement of the reference, including an SSE2 restatement of its WASM
SIMD front kernel) on a bounded sample (one complete subtree of the same factorization), single-threaded because the
reference is single-threaded by design.
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
# the benchmark systems: elasticity (the headline), P2 heat and Nedelec Maxwell (indefinite, LDL^T)
SYSTEMS = {
    "elastic3d": {"size": 40, "title": "3D P1 elasticity {N}^3", "kind": "chol",
                  "desc": "elastic3d-{N}: 3D P1 linear elasticity, {N}^3 hexes x 6 tets, E=1 nu=0.3, x=0 clamped, "
                          "nd3Order"},
    "heat3d_p2": {"size": 48, "title": "3D P2 heat {N}^3", "kind": "chol",
                  "desc": "heat3d-p2-{N}: 3D P2 (tet10) heat, {N}^3 hexes x 6 tets, k=100 in 64 seeded spheres "
                          "(r=0.05) else 1, Dirichlet x=0 and x=1, nd3Order"},
    "heat2d_batch": {"size": 256, "title": "batched 2D P1 heat, {N} problems", "kind": "batch",
                     "desc": "heat2d-batch-{N}: {N} P1 heat problems on unit squares, N ~ U{{16..128}} cells per side, "
                             "lognormal(0,1) conductivity, Dirichlet, 1-64 RHS each; AMD per matrix, one "
                             "block-diagonal factorization"},
    "maxwell3d": {"size": 32, "title": "3D Nedelec Maxwell {N}^3, LDL^T", "kind": "ldlt",
                  "desc": "maxwell3d-{N}: lowest-order Nedelec curl-curl - k^2 eps_r mass, {N}^3 hexes x 6 tets, "
                          "eps_r=12 in 8 seeded boxes, PEC, k^2 between the 10th and 11th eigenvalues, nd3Order on "
                          "edge midpoints"},
}


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
    """The batched heat set as one block-diagonal system (pattern, values, q_max RHS) with per-matrix AMD orders."""

    def __init__(self, count: int):
        import workloads as wl
        import ampsolve as amp
        import batch
        ws = wl.heat2d_batch(count)
        self.pat, offs, _ = batch.block_diagonal([w.pat for w in ws])
        self.values = np.concatenate([w.values for w in ws])
        q = max(w.rhs.shape[0] for w in ws)
        self.rhs = np.zeros((q, self.pat.n))
        for i, w in enumerate(ws):
            self.rhs[: w.rhs.shape[0], offs[i]: offs[i + 1]] = w.rhs
        self.perm = np.concatenate([amp.amdOrder(w.pat) + offs[i] for i, w in enumerate(ws)]).astype(np.int32)
        self.offs, self.q = offs, [w.rhs.shape[0] for w in ws]
        self.n = self.pat.n
        self.x = self.y = self.z = None


def make_system(name: str = "elastic3d", size: int = 40):
    import workloads as wl
    if name == "heat2d_batch":
        return _Batch(size)
    if name == "heat3d_p2":
        return wl.heat3d_p2(size, q=1)
    if name == "maxwell3d":
        return wl.maxwell3d(size, q=1)
    return wl.elastic3d(size, seed=2, q=1)


def measure_dgemm(torch):
    """cuBLAS DGEMM 8192^3 (the FP64 roofline denominator; no FP64 figure is in MEASURED_PEAKS.json)."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
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


def measure_sgemm(torch):
    """cuBLAS SGEMM 8192^3 with TF32 off: the FP32 CUDA-core denominator for the FP32 panel kernel."""
    torch.backends.cuda.matmul.allow_tf32 = False
    a = torch.randn(8192, 8192, dtype=torch.float32, device="cuda")
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


def cpu_baseline_sample(w, perm, budget_s: float = 15.0, kind: str = "chol"):
    """Oracle (SSE2 restatement of the reference's WASM front kernel) on one complete subtree of the factorization,
    pinned to one core (the reference's solver is single-threaded)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    try:
        keep = os.sched_getaffinity(0)
        os.sched_setaffinity(0, {min(keep)})
    except (AttributeError, OSError):
        keep = None
    so = orc.analyze(w.pat, perm=perm)
    # subtree flops
    ns = so.nsuper
    sub = np.zeros(ns)
    cc2 = so.colCount.astype(np.float64) ** 2
    own = np.add.reduceat(cc2, so.superStart[:-1]) if ns else np.zeros(0)
    sub[:] = own
    for s in range(ns):
        p = so.superParent[s]
        if p >= 0:
            sub[p] += sub[s]
    # calibrate on a small subtree, then pick the largest subtree that fits the budget
    order = np.argsort(sub)
    small = int(order[np.searchsorted(sub[order], 2e8)]) if np.any(sub >= 2e8) else int(order[-1])
    t = time.perf_counter()
    orc.factor_subtree(so, w.values, small, kind=kind, simd=True)
    rate = sub[small] / max(time.perf_counter() - t, 1e-6)
    target = rate * budget_s
    cand = np.where(sub <= target)[0]
    root = int(cand[np.argmax(sub[cand])]) if cand.size else small
    t = time.perf_counter()
    ok, fl = orc.factor_subtree(so, w.values, root, kind=kind, simd=True)
    dt = time.perf_counter() - t
    if keep:
        os.sched_setaffinity(0, keep)
    return {"value": fl / dt / 1e12, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"factor of the subtree of supernode {root} ({fl:.3e} of {so.flops:.3e} flops, "
                      f"{dt:.1f} s, SSE2 restatement of the reference's WASM front kernel, 1 pinned thread); "
                      f"extrapolated full factor {so.flops / (fl / dt):.0f} s",
            "full_factor_s_est": so.flops / (fl / dt)}


# DRAM bytes per launch of the roofline kernel (dram__bytes_read.sum + dram__bytes_write.sum, one ncu capture: the
# launch list of `bench.py --precision mixed --steps 1 --warmup 1 --no-cpu-baseline`, every launch of the kernel class,
# total / launches). Keyed by (workload, size, precision, kernel class).
TRAFFIC = {
    ("elastic3d", 40, "mixed", "update_syrk"): 50.229e9 / 2485,
}


def solution_errors(w, results):
    """Per precision: the normwise backward error max_k ||b_k - A x_k|| / (||A||_F ||x_k|| + ||b_k||) (2-norms, FP64
    on the host), and for the mixed path the forward error max_k ||x_k - x_k(FP64)|| / ||x_k(FP64)|| against the FP64
    GPU solution (the FP64 path itself matches the oracle to 1e-12 in the parity tests)."""
    import scipy.sparse as sp

    A = sp.csr_matrix((w.values, w.pat.colidx, w.pat.rowptr), shape=(w.n, w.n))
    anorm = float(np.sqrt(np.sum(w.values * w.values)))
    B = np.ascontiguousarray(w.rhs[: next(iter(results.values()))["x"].shape[0]])
    out = {}
    for p, r in results.items():
        X = r["x"]
        be = 0.0
        for k in range(X.shape[0]):
            rk = B[k] - A @ X[k]
            be = max(be, float(np.linalg.norm(rk) / (anorm * np.linalg.norm(X[k]) + np.linalg.norm(B[k]))))
        out[p] = {"backward_error": be}
    if "fp64" in results and "mixed" in results:
        X, Xr = results["mixed"]["x"], results["fp64"]["x"]
        fe = max(float(np.linalg.norm(X[k] - Xr[k]) / max(np.linalg.norm(Xr[k]), 1e-300)) for k in range(X.shape[0]))
        out["mixed"]["forward_error_vs_fp64"] = fe
    return out


def run_reference(args, rank):
    if rank != 0:
        return
    import workloads as wl  # noqa: F401
    w = make_system(args.workload, args.size)
    import ampsolve as amp
    try:
        perm = w.perm if isinstance(w, _Batch) else amp.nd3Order(w.pat, w.x, w.y, w.z)
    except Exception:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as orc
        perm = orc.nd3_order(w.pat, w.x, w.y, w.z)
    times, vals = [], []
    for it in range(args.warmup + args.steps):
        cb = cpu_baseline_sample(w, perm, budget_s=max(5.0, 60.0 / max(1, args.warmup + args.steps)),
                                 kind="ldlt" if args.ldlt else "chol")
        if it >= args.warmup:
            vals.append(cb["value"])
            times.append(0)
    v = float(np.median(vals))
    # the step time this rate implies for the whole factorization (the sample is a subtree of it)
    ms_est = 1e3 * cb["full_factor_s_est"] * cb["value"] / v if v > 0 else None
    line = {"impl": "reference", "metric": args.metric, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_est, "ms_per_step_kind": "extrapolated from the sample's rate",
            "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.desc, "n": w.n, "nnz": w.pat.nnz, "sample": cb["sample"]},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "port", "sample": cb["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="both", choices=["fp64", "mixed", "both"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="elastic3d", choices=sorted(SYSTEMS))
    ap.add_argument("--size", type=int, default=0, help="hexes per side (0 = the system's benchmark size)")
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
    w = make_system(args.workload, args.size)
    n = w.n
    t0 = time.perf_counter()
    if isinstance(w, _Batch):
        sym = amp.analyze(w.pat, perm=w.perm, device=local)
    else:
        sym = amp.analyze(w.pat, ordering="nd3", x=w.x, y=w.y, z=w.z, device=local)
    symbolic_ms = (time.perf_counter() - t0) * 1e3
    flops_factor = sym.flops
    flops_solve = 4.0 * sym.nnzL  # per right-hand side (forward + backward)
    nq = 1
    if isinstance(w, _Batch):  # every matrix solves its own q_i vectors: 4 nnzL_i q_i
        cc = sym.colCount.astype(np.float64)
        flops_solve = sum(4.0 * cc[w.offs[i]: w.offs[i + 1]].sum() * qi for i, qi in enumerate(w.q))
        nq = w.rhs.shape[0]

    precisions = ["fp64", "mixed"] if args.precision == "both" else [args.precision]
    results = {}
    dev = torch.device("cuda", local)
    vals_d = torch.from_numpy(w.values).to(dev)
    b_d = torch.from_numpy(np.ascontiguousarray(w.rhs[:nq]).reshape(-1)).to(dev)
    x_d = torch.empty_like(b_d)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2
    for prec in precisions:
        num = amp.NumericFactor(sym, amp.LDLT if args.ldlt else amp.CHOLESKY, amp.FP64 if prec == "fp64" else amp.MIXED)
        if isinstance(w, _Batch):
            num.set_row_groups(w.offs)  # the residual is measured per matrix

        # mixed precision, one right-hand side: GMRES-IR (the mixed factor as right preconditioner, FP64 Arnoldi and
        # residuals on the device). It needs fewer solves than plain refinement to reach 1e-12 (elasticity 40^3: 4
        # against 5) and converges for indefinite systems, where plain refinement need not. Several right-hand sides
        # (the batch) use plain refinement, all vectors in each sweep.
        gmres = prec == "mixed" and nq == 1

        def solve(bp, xp, on_device):
            if gmres:
                rr, its, _ = num.solve_gmres_ptr(bp, xp, on_device, tol=1e-12, restart=40, maxIter=300)
                return rr, its
            if on_device:
                return num.solve_refined_device(bp, xp, nq, maxSteps=10, tol=1e-12)
            return num.solve_refined_host_pinned(bp, xp, nq, 10, 1e-12)

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
        b_h = torch.from_numpy(np.ascontiguousarray(w.rhs[:nq]).reshape(-1)).pin_memory()
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
        work = flops_factor + flops_solve  # the same algorithmic work for both precisions: factor + one solve
        results[prec] = {"ok": ok, "ms": ms, "relres": relres, "ir_steps": irs, "work": work, "clk": clk.summary(),
                         "refinement": "gmres-ir (iterations)" if gmres else ("ir (steps)" if prec == "mixed" else "ir"),
                         "prof": prof, "e2e_ms": e2e_ms, "factor_ms": num.ms, "x": xsol}
        del num
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    # the headline is the faster of the measured paths (both are in the line): mixed + refinement where it wins (the
    # SPD systems), FP64 where the mixed factor needs too many Krylov iterations (the indefinite Maxwell system)
    head = min(results, key=lambda p: results[p]["ms"])
    R = results[head]
    pk = peaks()
    dom = max(R["prof"], key=lambda k: k["ms"])
    fp64_peak = measure_dgemm(torch)
    fp32_peak = measure_sgemm(torch)
    if dom["flops"] > 0 and dom["name"] == "update_syrk" and head == "mixed":
        peak, bound, punit, note = pk.get("bf16_tflops_sustained", 1400.0), "tensor", "TFLOP/s", \
            "MEASURED_PEAKS.json bf16_tflops_sustained (BF16 tensor; 3 products per FP32 update counted once)"
    elif dom["flops"] > 0 and head == "mixed":
        peak, bound, punit, note = fp32_peak, "tensor", "TFLOP/s", "measured cuBLAS SGEMM 8192^3 (no TF32) in this run"
    elif dom["flops"] > 0:
        peak, bound, punit, note = fp64_peak, "tensor", "TFLOP/s", "measured cuBLAS DGEMM 8192^3 in this run"
    if dom["flops"] > 0:
        achieved = dom["flops"] / (dom["ms"] * 1e-3) / 1e12
    else:
        achieved, bound, punit, peak, note = dom["bytes"] / (dom["ms"] * 1e-3) / 1e9, "hbm", "GB/s", pk["hbm_gbs"], \
            "MEASURED_PEAKS.json hbm_gbs"
    launches = sum(k["launches"] for k in R["prof"])
    value = world * R["work"] / (R["ms"] * 1e-3) / 1e12
    line = {
        "metric": args.metric, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": R["ms"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if head == "fp64" else "f32+bf16x3 (f64 refinement)", "data": "synthetic",
        "config": {"workload": args.desc, "n": n, "nnz": w.pat.nnz, "nnzL": sym.nnzL,
                   "flops_factor": flops_factor,
                   "maxFront": sym.maxFront, "nsuper": sym.nsuper, "levels": sym.nlevels, "precision": head,
                   "l2": "flushed between timed steps (256 MB write)", "parallelism": "replicas" if world > 1 else "1 gpu",
                   "symbolic_ms": symbolic_ms},
        "relres": R["relres"], "ir_steps": R["ir_steps"], "factor_ms": R["factor_ms"],
        "e2e": {"value": world * R["work"] / (R["e2e_ms"] * 1e-3) / 1e12, "unit": UNIT,
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
    errs = solution_errors(w, results)
    for p, r in results.items():
        line[p] = {"ms_per_step": r["ms"], "value": world * r["work"] / (r["ms"] * 1e-3) / 1e12, "relres": r["relres"],
                   "ir_steps": r["ir_steps"], "refinement": r["refinement"], "factor_ms": r["factor_ms"], "ok": r["ok"],
                   **errs.get(p, {})}
    if world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline_sample(w, sym.perm, kind="ldlt" if args.ldlt else "chol")
        line["cpu_baseline"] = {k: v for k, v in cb.items() if k != "full_factor_s_est"}
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
