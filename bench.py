"""Benchmark: time-to-solution of the 100^3 7-point Laplacian (n = 10^6) to
backward error 1e-12 on one B200, FP32 factorization + FP64 GPU CG refinement
against the plain FP64 factorization + solve (+ refinement check).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One step = numerical factorization + solve + refinement of one system (the
hot path; the analysis is done once, outside the timed region).  `value` is
the device-timed seconds per step with the matrix values and the right-hand
side already in HBM; `e2e` is the same step through the C ABI with host
buffers (pastix_task_numfact + pastix_task_solve + pastix_task_refine), the
host<->device copies inside the timed region.  Multi-GPU runs are independent
replicas (one system per GPU, no collective on the data path); the time is the
max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOADS = {
    # name: (grid, factorization, refinement, rhs seed)
    "lap100": ((100, 100, 100), "POTRF", "CG", 1),
}
BERR_TARGET = 1e-12


def backward_error(A, x, b) -> float:
    import scipy.sparse.linalg as spla
    r = b - A @ x
    return float(np.linalg.norm(r) / (spla.norm(A) * np.linalg.norm(x) + np.linalg.norm(b)))


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        load = [s for s in sm if smax and s > 0.3 * smax] or sm
        return {"sm_mhz": float(np.median(load)) if load else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def max_over_ranks(t: float, ws: int, device: str = "cuda") -> float:
    """The slowest rank's time (replicas: the whole job ends when the last
    rank does); every rank takes part and receives it."""
    if ws <= 1:
        return t
    import torch
    import torch.distributed as dist
    tt = torch.tensor([t], device=device, dtype=torch.float64)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def fp64_peak_tflops(torch) -> float:
    """cuBLAS DGEMM throughput measured in this run (the FP64 roofline denominator)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def update_flops(info) -> float:
    """Algorithmic flops of the update GEMMs (the update term of the reference's
    sum1d for LL^T: N*M*(M+1) per cblk, symbol/symbol_cost.c:53-88)."""
    N = (info["cb_lcol"] - info["cb_fcol"] + 1).astype(np.float64)
    M = (info["cb_stride"] - N).astype(np.float64)
    return float((N * M * (M + 1)).sum())


def solve_bytes(info) -> float:
    """Algorithmic bytes of one FP64 LL^T solve: the factor read twice (forward and backward)."""
    return 2.0 * 8.0 * float(info["coefnbr"])


def time_solves(pd, n, info, mode, S) -> dict:
    """Device time of one solve (1 and 16 right-hand sides, pgpu_solve_device)
    and of one residual SpMV (pgpu_spmv_device) with the resident factors, and
    their algorithmic HBM bytes: per sweep the factor panels once
    (sizeof(T) * coefnbr) plus the right-hand sides read and written; the SpMV
    reads the permuted CSR (8-byte values, 4-byte column indices, 4-byte row
    pointers), x, and reads and writes y."""
    import torch
    from pastix_b200 import pastix as px
    fs = 4 if mode == "mixed" else 8
    out = {}
    g = torch.Generator(device="cuda").manual_seed(9)
    for nrhs in (1, 16):
        B0 = torch.rand(n, nrhs, dtype=torch.float64, device="cuda", generator=g).t().contiguous().t()
        B = B0.clone()
        ts = []
        for rep in range(8):
            B.copy_(B0)  # in-place solves: start every repetition from the same right-hand sides
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            px.solve_device(pd, B if nrhs > 1 else B[:, 0])
            e1.record()
            torch.cuda.synchronize()
            if rep >= 2:
                ts.append(e0.elapsed_time(e1))
        ms = float(np.median(ts))
        # two sweeps; the FP32 path also casts the FP64 right-hand sides in and out
        byts = 2.0 * (fs * info["coefnbr"] + 2.0 * n * nrhs * fs) + 2.0 * n * nrhs * 8 * 2
        out[f"nrhs{nrhs}_ms"] = ms
        out[f"nrhs{nrhs}_gbs"] = byts / (ms / 1e3) / 1e9
    if mode == "fp64":
        # the SpMV kernel's own device time (library events around its launch),
        # L2 flushed before every call: its 111 MB would otherwise stay in the
        # 126 MB L2 from one call to the next
        x = torch.rand(n, dtype=torch.float64, device="cuda", generator=g)
        y = torch.zeros_like(x)
        flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
        nnz = int(S.full().nnz)
        for _ in range(3):
            px.spmv_device(pd, 1.0, x, 0.0, y)
        torch.cuda.synchronize()
        reps = 20
        px.profile(pd, True)
        for _ in range(reps):
            flush.zero_()
            px.spmv_device(pd, 1.0, x, 0.0, y)
        torch.cuda.synchronize()
        prof = px.profile_get(pd)
        px.profile(pd, False)
        ms = prof["spmv"][0] / max(prof["spmv"][1], 1)
        byts = nnz * (8 + 4) + 4 * (n + 1) + 16 * n  # CSR, x read, y written (beta = 0)
        out["spmv_ms"] = ms
        out["spmv_gbs"] = byts / (ms / 1e3) / 1e9
    return out


def run_b200(args, ws, rank, local):
    import torch
    from pastix_b200 import gen
    from pastix_b200 import pastix as px
    from pastix_b200.spm import mtxtype, spmatrix

    torch.cuda.set_device(local)
    grid, fact, refine, seed = WORKLOADS[args.workload]
    A = gen.laplacian7(*grid)
    n = A.shape[0]
    S = spmatrix(A, mtxtype.Symmetric)
    Af = S.full()
    xt = gen.rhs_uniform(n, 1, seed)[:, 0]
    b_h = np.ascontiguousarray(Af @ xt)
    vals = torch.from_numpy(S.values).cuda()
    b = torch.from_numpy(b_h).cuda()

    results = {}
    for mode in ("mixed", "fp64"):
        ip, dp = px.initParam()
        ip[px.iparm.factorization] = px.factotype.POTRF
        ip[px.iparm.mixed] = 1 if mode == "mixed" else 0
        ip[px.iparm.refinement] = px.refine.CG
        dp[px.dparm.epsilon_refinement] = BERR_TARGET
        pd = px.init(ip, dp)
        t0 = time.time()
        px.analyze_grid(pd, S, *grid)
        t_an = time.time() - t0
        # one-time setup outside the timed region: bucket boundaries of the update tiles
        t0 = time.time()
        tuning = px.autotune(pd, vals)
        t_tune = time.time() - t0
        info = px.solver_info(pd)
        x = torch.zeros_like(b)
        stream = torch.cuda.ExternalStream(px.stream_ptr(pd))

        def step():
            px.numfact_device(pd, vals)
            px.solve_refine_device(pd, b, x)

        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        if ws > 1:
            torch.distributed.barrier()
        sampler = ClockSampler(local) if mode == "mixed" else None
        if sampler:
            sampler.start()
        px.profile(pd, False)  # count launches, no per-launch events
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3 / args.steps
        launches = sum(v[1] for v in px.profile_get(pd).values())
        clocks = sampler.stop() if sampler else None
        t = max_over_ranks(t, ws)
        xh = x.cpu().numpy()
        berr = backward_error(Af, xh, b_h)
        results[mode] = dict(t=t, berr=berr, fwd=float(np.linalg.norm(xh - xt) / np.linalg.norm(xt)),
                             fact_time=float(dp[px.dparm.fact_time]), iters=int(ip[px.iparm.nbiter]),
                             npiv=int(ip[px.iparm.static_pivoting]), launches=launches / args.steps,
                             analyze_s=t_an, clocks=clocks, thflops=info["thflops"],
                             tuning={"dmma_min_rows": tuning[0], "dmma_min_width": tuning[1],
                                     "tcgen05_min_width": tuning[2], "autotune_s": t_tune})
        # profiled pass (per-class device times) for the roofline of the dominant kernel
        px.profile(pd, True)
        step()
        prof = px.profile_get(pd)
        px.profile(pd, False)
        results[mode]["profile"] = prof
        results[mode]["info"] = {k: info[k] for k in ("cb_lcol", "cb_fcol", "cb_stride", "coefnbr")}
        results[mode]["solve"] = time_solves(pd, n, info, mode, S)
        # 16 right-hand sides (b = A x_true, x_true ~ U[-1,1] seed 1): time to backward error 1e-12 of all
        xt16 = gen.rhs_uniform(n, 16, seed)
        b16h = np.asfortranarray(Af @ xt16)
        B16 = torch.from_numpy(np.ascontiguousarray(b16h.T)).cuda().t()
        X16 = torch.zeros(16, n, dtype=torch.float64, device="cuda").t()
        t16 = []
        for rep in range(4):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            px.numfact_device(pd, vals)
            px.solve_refine_device(pd, B16, X16)
            e1.record(stream)
            torch.cuda.synchronize()
            if rep:
                t16.append(e0.elapsed_time(e1) / 1e3)
        X16h = X16.cpu().numpy()
        results[mode]["rhs16"] = {"s": float(np.median(t16)), "iters": int(ip[px.iparm.nbiter]),
                                  "berr_max": max(backward_error(Af, X16h[:, j], b16h[:, j]) for j in range(16))}
        if mode == "mixed":
            # e2e through the C ABI with host buffers
            # (each step timed on its own; the median over the steps is reported, the
            # host side of these calls shares the machine's cores with other jobs)
            xe = np.asfortranarray(b_h.copy())
            px.task_numfact(pd, S)  # warm
            torch.cuda.synchronize()
            te = []
            for _ in range(max(3, args.steps)):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                px.task_numfact(pd, S)
                xe[:] = b_h
                px.task_solve(pd, S, xe)
                px.task_refine(pd, S, b_h, xe)
                e1.record(stream)
                torch.cuda.synchronize()
                te.append(e0.elapsed_time(e1) / 1e3)
            results[mode]["e2e"] = float(np.median(te))
            results[mode]["e2e_steps"] = te
            results[mode]["e2e_berr"] = backward_error(Af, xe, b_h)
            results[mode]["h2d"] = 8 * S.nnz + 8 * n + 2 * 8 * n
            results[mode]["d2h"] = 8 * n + 8 * n
        px.finalize(pd)
    return results, n


def run_reference(args, modes=("mixed", "fp64"), nsteps: int = 1, warmup: int = 0) -> dict:
    """The reference PaStiX itself (oracle/_ref: its own sources compiled here,
    with OpenBLAS) on the same workload: its analysis once (grid nested
    dissection, pastixOrderGrid as example/ordering_grid.c), then per step
    pastix_task_numfact + pastix_task_solve + pastix_task_refine (CG, 1e-12)
    with the static scheduler (IPARM_SCHEDULER = 1) on every host core.  Each
    mode: FP64 factors, or FP32 factors (IPARM_MIXED = 1) refined in FP64.
    Nothing of the product is loaded."""
    from oracle import ref
    from pastix_b200 import gen
    grid, fact, refine, seed = WORKLOADS[args.workload]
    if args.cpu_sample_grid < grid[0]:
        grid = tuple(min(g, args.cpu_sample_grid) for g in grid)
    A = gen.laplacian7(*grid)
    n = A.shape[0]
    xt = gen.rhs_uniform(n, 1, seed)[:, 0]
    b = A @ xt
    threads = os.cpu_count() or 1
    out = {"grid": grid, "threads": threads, "modes": {}}
    for mode in modes:
        r = ref.RefPastix(A, fact, nthreads=threads, scheduler="static", mixed=(mode == "mixed"))
        r.iparm[ref.IPARM_REFINEMENT] = 1  # PastixRefineCG
        r.dparm[ref.DPARM_EPSILON_REFINEMENT] = BERR_TARGET
        t0 = time.perf_counter()
        r.analyze(grid=grid)
        t_an = time.perf_counter() - t0
        steps = []
        for it in range(warmup + nsteps):
            t0 = time.perf_counter()
            r.numfact()
            x = r.solve(b)
            x = r.refine(b, x)
            if it >= warmup:
                steps.append(time.perf_counter() - t0)
        out["modes"][mode] = {
            "t": float(np.median(steps)), "steps_s": steps, "analysis_s": t_an,
            "berr": backward_error(A, x[:, 0], b),
            "fact_s": float(r.dparm[ref.DPARM_FACT_TIME]), "solve_s": float(r.dparm[ref.DPARM_SOLV_TIME]),
            "refine_s": float(r.dparm[ref.DPARM_REFINE_TIME]), "refine_iters": int(r.iparm[ref.IPARM_NBITER]),
            "thflops": float(r.dparm[ref.DPARM_FACT_THFLOPS])}
        r.close()
    ok = {m: v for m, v in out["modes"].items() if v["berr"] <= BERR_TARGET}
    best = min(ok or out["modes"], key=lambda m: (ok or out["modes"])[m]["t"])
    out["best"] = best
    out["t"] = out["modes"][best]["t"]
    return out


def reference_sample(r: dict, full_grid) -> str:
    modes = ", ".join(f"{m} {v['t']:.2f} s (factor {v['fact_s']:.2f} s, {v['refine_iters']} CG iters, "
                      f"berr {v['berr']:.1e})" for m, v in r["modes"].items())
    size = "full workload" if tuple(r["grid"]) == tuple(full_grid) else f"reduced grid {r['grid']}"
    return (f"{size}: reference PaStiX built from its sources (oracle/_ref), static scheduler, "
            f"{r['threads']} threads, OpenBLAS; numfact + solve + refine per step; {modes}; best {r['best']}")


def run_adjoint(reps: int = 20, ndir: int = 20) -> dict:
    """Adjoint of the solve on the variable-coefficient 2D diffusion (512x512,
    k = exp(GRF), seed 2): loss 0.5||x - x_obs||^2 with x_obs the solution for an
    independent field (seed 12) plus 1% Gaussian noise.  Times one forward solve
    against one backward pass (transposed solve + sampled outer product over the
    pattern) with CUDA events, and checks the gradient against central finite
    differences along `ndir` random directions of (values, b)."""
    import torch
    from pastix_b200 import gen
    from pastix_b200 import pastix as px
    from pastix_b200.autograd import SparseSolver, solve

    A, grid, fact = gen.workload("grf512")
    s = grid[0]
    solver = SparseSolver(A, fact, grid=grid)
    n = A.shape[0]
    rng = np.random.default_rng(2)
    vals = torch.tensor(solver.spm.values, device="cuda")
    b = torch.tensor(rng.standard_normal(n), device="cuda")
    # observations: the solution for an independent field, plus 1% noise
    A_obs = gen.diffusion5_grf(s, s, np.exp(gen.grf_2d(s, s, 16.0, 1.0, 12)))
    obs = SparseSolver(A_obs, fact, grid=grid)
    obs.factorize(torch.tensor(obs.spm.values, device="cuda"))
    x_obs = obs.solve(b)
    x_obs = x_obs + 0.01 * x_obs.abs().mean() * torch.tensor(rng.standard_normal(n), device="cuda")
    px.finalize(obs.pd)

    solver.factorize(vals)
    x = solver.solve(b)
    g = x - x_obs
    st = torch.cuda.current_stream()

    def timed(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(reps):
            fn()
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    t_fwd = timed(lambda: solver.solve(b))
    t_bwd = timed(lambda: solver.sampled_outer(solver.solve(g, transposed=True), x))

    def fwd_total():
        solver.factorize(vals)
        solver.solve(b)
    t_fact_solve = timed(fwd_total)

    # gradient through torch.autograd, then central differences
    v = vals.clone().requires_grad_(True)
    bb = b.clone().requires_grad_(True)
    xs = solve(v, bb, solver)
    loss = 0.5 * ((xs - x_obs) ** 2).sum()
    loss.backward()
    gv, gb = v.grad, bb.grad
    drng = np.random.default_rng(20)

    def central(h, dv, db):
        # (f(+h) - f(-h)) / 2h with the loss difference written as a product, so
        # that the large loss does not cancel: 0.5 (x+ - x-) . (x+ + x- - 2 x_obs)
        with torch.no_grad():
            xp = solve(vals + h * dv, b + h * db, solver)
            xm = solve(vals - h * dv, b - h * db, solver)
            return (0.5 * ((xp - xm) * (xp + xm - 2 * x_obs)).sum()).item() / (2 * h)

    worst = 0.0
    for _ in range(ndir):
        dv = torch.tensor(drng.standard_normal(vals.numel()), device="cuda") * vals.abs()
        db = torch.tensor(drng.standard_normal(n), device="cuda")
        # Richardson extrapolation of the central difference (h, h/2) cancels the
        # h^2 term, which dominates at this contrast of k = exp(GRF)
        h = 1e-6
        fd = (4.0 * central(h / 2, dv, db) - central(h, dv, db)) / 3.0
        an = (gv * dv).sum().item() + (gb * db).sum().item()
        worst = max(worst, abs(fd - an) / max(abs(an), 1e-300))
    px.finalize(solver.pd)
    return {"workload": "grf512: 2D 5-point diffusion 512x512 (n=262144), k=exp(GRF l=16 var=1 seed 2), LL^T",
            "forward_solve_ms": t_fwd, "adjoint_ms": t_bwd, "adjoint_over_solve": t_bwd / t_fwd,
            "factor_plus_solve_ms": t_fact_solve, "fd_directions": ndir, "fd_max_rel_err": worst,
            "fd_rule": "central differences h=1e-6 and 5e-7, Richardson-extrapolated"}


# The other configurations at full size (one JSON line each with --workload):
# FP32 factorization + FP64 refinement against the plain FP64 path, every
# right-hand side to backward error 1e-12.
CONFIGS = {
    "grf512": dict(desc="2D 5-point variable-coefficient diffusion 512x512 (n=262144), k=exp(GRF, l=16 cells, "
                        "var 1, seed 2), Dirichlet, LL^T, CG; 1 RHS b=A x_true, x_true~U[-1,1] seed 2",
                   refine="CG", nrhs=1, rhs="xtrue", seed=2),
    "cd64": dict(desc="27-point upwind convection-diffusion 64^3 (n=262144), velocity U[-50,50]^3 per cell seed 3, "
                      "diagonal dominance 0.95, LU with static pivoting, GMRES(30); 4 RHS b=A x_true, "
                      "x_true~U[-1,1] seed 3", refine="GMRES", nrhs=4, rhs="xtrue", seed=3),
    "el48": dict(desc="3-dof 27-point elasticity block stencil 48^3 nodes (n=331776), Wishart(3, 6 dof) coupling "
                      "blocks seed 4, shifted by -sigma I at the 5th percentile of a Lanczos spectrum estimate, "
                      "LDL^T, GMRES(30); 256 RHS ~ N(0,1)", refine="GMRES", nrhs=256, rhs="normal", seed=4),
}


def run_config(args) -> int:
    """Full-size run of one configuration: analysis and autotuning once, then
    `steps` timed passes of factorization + solve + refinement of all
    right-hand sides (device-resident values and right-hand sides), for the
    FP32 path and the FP64 path; rank 0 prints one JSON line."""
    import torch
    from pastix_b200 import gen
    from pastix_b200 import pastix as px
    from pastix_b200.spm import mtxtype, spmatrix
    cfg = CONFIGS[args.workload]
    A, grid, fact = gen.workload(args.workload)
    S = spmatrix(A, mtxtype.General if fact == "GETRF" else mtxtype.Symmetric)
    Af = S.full()
    n = A.shape[0]
    nrhs = cfg["nrhs"]
    if cfg["rhs"] == "xtrue":
        xt = gen.rhs_uniform(n, nrhs, cfg["seed"])
        bh = np.asfortranarray(Af @ xt)
    else:
        xt = None
        bh = np.asfortranarray(np.random.default_rng(cfg["seed"]).standard_normal((n, nrhs)))
    vals = torch.from_numpy(S.values).cuda()
    B = torch.from_numpy(np.ascontiguousarray(bh.T)).cuda().t()  # column major, ld = n
    import scipy.sparse.linalg as spla
    anorm = spla.norm(Af)
    out = {}
    for mode in ("mixed", "fp64"):
        ip, dp = px.initParam()
        ip[px.iparm.factorization] = {"POTRF": 0, "SYTRF": 1, "GETRF": 2}[fact]
        ip[px.iparm.mixed] = 1 if mode == "mixed" else 0
        ip[px.iparm.refinement] = px.refine.CG if cfg["refine"] == "CG" else px.refine.GMRES
        ip[px.iparm.gmres_im] = 30
        dp[px.dparm.epsilon_refinement] = BERR_TARGET
        pd = px.init(ip, dp)
        t0 = time.time()
        px.analyze_grid(pd, S, *grid)
        t_an = time.time() - t0
        t0 = time.time()
        tuning = px.autotune(pd, vals)
        t_tune = time.time() - t0
        info = px.solver_info(pd)
        X = torch.zeros(nrhs, n, dtype=torch.float64, device="cuda").t()  # column major, ld = n
        stream = torch.cuda.ExternalStream(px.stream_ptr(pd))

        def step():
            px.numfact_device(pd, vals)
            px.solve_refine_device(pd, B, X)

        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fts = []
        for _ in range(args.steps):
            step()
            fts.append(dp[px.dparm.fact_time])
        e1.record(stream)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3 / args.steps
        Xh = X.cpu().numpy()
        R = bh - Af @ Xh
        berr = float(max(np.linalg.norm(R[:, j]) / (anorm * np.linalg.norm(Xh[:, j]) + np.linalg.norm(bh[:, j]))
                         for j in range(nrhs)))
        res = {"s": t, "factor_s": float(np.median(fts)), "berr_max": berr,
               "factor_tflops": info["thflops"] / float(np.median(fts)) / 1e12,
               "refine_iters_last_rhs": int(ip[px.iparm.nbiter]), "static_pivots": int(ip[px.iparm.static_pivoting]),
               "analyze_s": t_an, "autotune_s": t_tune, "tuning": list(tuning)}
        if xt is not None:
            res["fwd_err"] = float(np.linalg.norm(Xh - xt) / np.linalg.norm(xt))
        out[mode] = res
        px.finalize(pd)
    best = "mixed" if (out["mixed"]["berr_max"] <= BERR_TARGET and out["mixed"]["s"] <= out["fp64"]["s"]) else "fp64"
    line = {"metric": "time-to-solution at backward error 1e-12 (factor + solve + refine, all RHS)",
            "value": out[best]["s"], "unit": "s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": out[best]["s"] * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64" if best == "mixed" else "f64", "data": "synthetic",
            "config": {"workload": f"{args.workload}: {cfg['desc']}", "global_batch": nrhs, "seq_len": None,
                       "parallelism": "replicas1", "l2": "factor larger than L2"},
            "path": best, "fp32_refine": out["mixed"], "fp64": out["fp64"], "thflops": info["thflops"]}
    print(json.dumps(line))
    return 0


def run_probe(s: int, mixed: bool = False) -> int:
    import torch
    from pastix_b200 import gen
    from pastix_b200 import pastix as px
    from pastix_b200.spm import mtxtype, spmatrix
    A = gen.laplacian7(s, s, s)
    ip, dp = px.initParam()
    ip[px.iparm.factorization] = px.factotype.POTRF
    ip[px.iparm.refinement] = px.refine.CG
    ip[px.iparm.mixed] = 1 if mixed else 0
    pd = px.init(ip, dp)
    S = spmatrix(A, mtxtype.Symmetric)
    px.analyze_grid(pd, S, s, s, s)
    vals = torch.from_numpy(S.values).cuda()
    b = torch.ones(A.shape[0], dtype=torch.float64, device="cuda")
    x = torch.zeros_like(b)
    for _ in range(2):
        px.numfact_device(pd, vals)
        px.solve_refine_device(pd, b, x)
    torch.cuda.synchronize()
    print("probe ok")
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="lap100", choices=list(WORKLOADS) + list(CONFIGS),
                    help="lap100 (the headline line, default) or one of the other configurations at full size")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-grid", type=int, default=100)
    ap.add_argument("--probe", type=int, default=0,
                    help="profiling case: analysis of an N^3 Laplacian then two LL^T FP64 "
                         "factor + solve + CG passes, no timing (used for ncu captures)")
    ap.add_argument("--probe-mixed", action="store_true", help="the --probe case with FP32 factors")
    args = ap.parse_args()
    if args.probe:
        return run_probe(args.probe, args.probe_mixed)
    args.warmup = max(args.warmup, 3)
    if args.workload in CONFIGS:
        if args.impl == "reference" or int(os.environ.get("RANK", "0")) != 0:
            return 0
        return run_config(args)

    ws, rank, local = (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
                       int(os.environ.get("LOCAL_RANK", "0")))
    grid = WORKLOADS[args.workload][0]
    config = {"workload": f"{args.workload}: 3D 7-point Laplacian {grid[0]}x{grid[1]}x{grid[2]} (n=10^6), LL^T, "
                          "1 RHS x_true~U[-1,1] seed 1, grid nested dissection",
              "global_batch": ws, "seq_len": None, "parallelism": f"replicas{ws}",
              "l2": "inputs larger than L2 (factor 8.5 GB FP64)"}
    metric = "time-to-solution at backward error 1e-12 (factor + solve + refine)"

    if args.impl == "reference":
        if rank != 0:
            return 0
        # a full-workload step takes tens of seconds on the host cores: at most
        # two per mode, so that the whole run stays within a few minutes
        r = run_reference(args, nsteps=max(1, min(args.steps, 2)), warmup=1)
        v = r["t"]
        line = {"metric": metric, "value": v, "unit": "s", "n_gpus": 0, "steps": len(r["modes"][r["best"]]["steps_s"]),
                "warmup": 1, "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64" if r["best"] == "fp64" else "f32 factor + f64 refine",
                "data": "synthetic", "config": config, "impl": "reference",
                "cpu_baseline": {"value": v, "unit": "s", "cores": r["threads"], "kind": "reference",
                                 "sample": reference_sample(r, WORKLOADS[args.workload][0])},
                "reference_modes": r["modes"],
                "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    import torch
    ws, rank, local = dist_setup()
    res, n = run_b200(args, ws, rank, local)
    mixed, fp64 = res["mixed"], res["fp64"]
    best = "mixed" if (mixed["berr"] <= BERR_TARGET and mixed["t"] <= fp64["t"]) else "fp64"
    value = res[best]["t"]
    prof = fp64["profile"]
    uflops = update_flops(fp64["info"])
    # FP64 path: DMMA update GEMMs against the cuBLAS DGEMM rate measured here
    upd_ms = prof["update"][0] + prof["update_big"][0]
    upd_launch = prof["update"][1] + prof["update_big"][1]
    peak64 = fp64_peak_tflops(torch) if rank == 0 else None
    ach64 = uflops / (upd_ms / 1e3) / 1e12 if upd_ms > 0 else None
    # FP32 path (the headline when it wins): tcgen05 update GEMMs, six BF16 products per FP32 product
    prof32 = mixed["profile"]
    tc_ms, tc_launch = prof32["update_big"]
    peaks = {}
    pfile = ROOT / "MEASURED_PEAKS.json"
    if pfile.exists():
        try:
            peaks = json.loads(pfile.read_text())
        except Exception:
            peaks = {}
    bf16 = peaks.get("bf16_tflops")
    peak32 = bf16 / 6.0 if bf16 else 1590.0 / 6.0
    ach32 = uflops / (tc_ms / 1e3) / 1e12 if tc_ms > 0 else None
    traffic = None
    tfile = ROOT / "profiles" / "traffic.json"
    if tfile.exists():
        try:
            traffic = json.loads(tfile.read_text()).get("k_update_tc_lap100")
        except Exception:
            traffic = None
    if best == "mixed":
        roof = {"kernel": "k_update_tcp (FP32 supernode update GEMMs on tcgen05, split BF16 terms, scatter-add)",
                "bound": "tensor", "achieved": ach32, "peak": peak32, "unit": "TFLOP/s",
                "frac": (ach32 / peak32) if ach32 else None, "traffic": traffic,
                "peak_source": ("measured dense bf16 %s TFLOP/s (MEASURED_PEAKS.json, burst) / 6 BF16 products per "
                                "FP32 product" % bf16) if bf16 else "fallback 1590 TFLOP/s bf16 / 6",
                "launches": tc_launch, "ms_total": tc_ms, "algorithmic_flops": uflops}
    else:
        roof = {"kernel": "k_update_dmma + k_update (FP64 supernode update GEMMs + scatter-add)", "bound": "tensor",
                "achieved": ach64, "peak": peak64, "unit": "TFLOP/s",
                "frac": (ach64 / peak64) if (ach64 and peak64) else None, "traffic": None,
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run", "launches": upd_launch,
                "ms_total": upd_ms, "algorithmic_flops": uflops}
    line = {
        "metric": metric, "value": value, "unit": "s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64" if best == "mixed" else "f64", "data": "synthetic", "config": config,
        "path": best,
        "fp32_refine": {"s": mixed["t"], "berr": mixed["berr"], "fwd_err": mixed["fwd"], "cg_iters": mixed["iters"],
                        "factor_s": mixed["fact_time"], "tuning": mixed["tuning"]},
        "fp64": {"s": fp64["t"], "berr": fp64["berr"], "fwd_err": fp64["fwd"], "refine_iters": fp64["iters"],
                 "factor_s": fp64["fact_time"], "factor_tflops": fp64["thflops"] / fp64["fact_time"] / 1e12,
                 "tuning": fp64["tuning"]},
        "factor_tflops_fp32": mixed["thflops"] / mixed["fact_time"] / 1e12,
        "rhs16": {"fp32_refine": mixed["rhs16"], "fp64": fp64["rhs16"],
                  "note": "factor + solve + refinement of 16 right-hand sides (block CG) to backward error 1e-12"},
        "static_pivots": fp64["npiv"],
        "roofline": roof,
        "roofline_fp64": {"kernel": "k_update_dmma + k_update", "achieved": ach64, "peak": peak64,
                          "unit": "TFLOP/s", "frac": (ach64 / peak64) if (ach64 and peak64) else None,
                          "peak_source": "cuBLAS DGEMM 8192^3 measured in this run"},
        "profile_ms": {k: v[0] for k, v in prof.items() if v[1]},
        "profile_ms_fp32": {k: v[0] for k, v in mixed["profile"].items() if v[1]},
        "clocks": mixed["clocks"],
        "gpu_launches": int(res[best]["launches"]),
        "e2e": {"value": mixed["e2e"], "unit": "s", "h2d_bytes_per_step": mixed["h2d"],
                "d2h_bytes_per_step": mixed["d2h"], "berr": mixed["e2e_berr"], "statistic": "median",
                "steps_s": mixed["e2e_steps"]},
    }
    hbm = peaks.get("hbm_gbs") or 6650.0
    hbm_src = "measured copy (MEASURED_PEAKS.json)" if peaks.get("hbm_gbs") else "fallback 6650 GB/s"
    line["solve"] = {"fp32_factor": mixed["solve"], "fp64_factor": {k: v for k, v in fp64["solve"].items()
                                                                   if not k.startswith("spmv")},
                     "peak_gbs": hbm, "peak_source": hbm_src,
                     "frac_nrhs1_fp32": mixed["solve"]["nrhs1_gbs"] / hbm,
                     "frac_nrhs16_fp64": fp64["solve"]["nrhs16_gbs"] / hbm}
    line["spmv"] = {"ms": fp64["solve"]["spmv_ms"], "gbs": fp64["solve"]["spmv_gbs"], "peak_gbs": hbm,
                    "frac": fp64["solve"]["spmv_gbs"] / hbm}
    if rank == 0 and ws == 1:
        line["adjoint"] = run_adjoint()
    if rank == 0 and not args.no_cpu_baseline and ws == 1:
        # one step of the reference's faster mode (FP32 factors + FP64 CG) on the full workload
        cb = run_reference(args, modes=("mixed",), nsteps=1)
        line["cpu_baseline"] = {"value": cb["t"], "unit": "s", "cores": cb["threads"], "kind": "reference",
                                "sample": reference_sample(cb, WORKLOADS[args.workload][0])}
    if rank == 0:
        print(json.dumps(line))
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
