"""Solve-phase benchmark: time to a 1e-10 relative residual on one B200 per rank.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl prism|reference]
                    [--precond amsed|ic] [--grid G] [--config 1..5] [--no-secondary]

Headline workload: 3D Poisson 7-point Laplacian 128^3 (n = 2,097,152,
nnz = 14,581,760; generateLaplacianCSR), b ~ N(0,1) from a fixed seed, x0 = 0,
flexible CG + AMSED/MSLR (3 HID levels, natural order inside each domain
(MatrixReorderNo), ILDLT(1e-3) blocks, ICT(1e-3) on the last level, low-rank
correction of rank <= 32 per level from 64 classic generalized Lanczos steps,
MSLR correction H = lambda/(1-lambda)), relative tolerance 1e-10, max 1000
iterations.  `--precond ic` runs FCG + ICT(1e-3) on the same system instead.
The preconditioner is set up once on the host (outside the timed region); one
step is one complete device-resident solve.  The headline is the
mixed-precision solve: FP32 factor values and FP32 arithmetic inside the
streamed triangular sweeps (PRISM_FP32_APPLY), FP64 Krylov vectors, scalars,
SpMV and true residual.  Beside it: the reference's own <float,double>
instantiation (FP32 values, FP64 arithmetic: PRISM_FP32), the solve with FP64
factor values, and the forward error of both against the reference's own FP64
solution of the same system.

The default run (N = 1) also measures the other benchmark configurations as
extra keys of the same line ("configs"), each with the reference's CPU solver
timed beside it: 2D Poisson 64^2 FCG + ICT; 3D convection-diffusion 100^3
FGMRES(50) + GMSLR; batched solves (64 right-hand sides on 2D Poisson 512^2,
256 uneven 2D systems); the differentiable 64^3 variable-coefficient solve.
`--config N` prints configuration N alone.

Multi-GPU: replicas only (one independent system per rank, no collective on the
data path); the process group is used for the barrier and the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import platform
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time-to-1e-10 rel. residual, mixed FP32-factor / FP64-Krylov, 1 B200"
# MatrixReorderNo inside each HID domain: the domains keep the grid's natural
# order, which gives their incomplete factors about half the dependency
# wavefronts of the RCM order at the same iteration count.
AMSED = dict(levels=3, lanczos_steps=64, low_rank=32, eig_bound=0.8, lowrank_type=0, lanczos_type=0, reorder=0)
SEED = 2024
# DRAM bytes / algorithmic bytes of the streamed sweep kernel's level-0 lower sweep (one ncu capture on the
# 96^3 case, profiles/k_sweep_stream_fp32apply_level0_lower_96cube.md), applied to each launch's algorithmic bytes
TRAFFIC_RATIO = {"level-order": 181.2 / 183.6, "stream": 256.4 / 183.6}
TRAFFIC_SOURCE = ("ncu capture of the level-0 lower sweep at 96^3 (183.6 MB algorithmic): DRAM read + write "
                  "bytes / algorithmic bytes, scaled to this launch")
# the reference library's timing build (oracle/Makefile FAST_FLAGS)
REF_BUILD = "g++ -O3 -ffast-math -march=x86-64-v3 (AVX2, FMA) -fopenmp, 4 OpenMP threads (THREAD_NUM)"


def workload(grid: int, tol: float, precond: str) -> str:
    n = grid ** 3
    nnz = 7 * n - 6 * grid * grid
    pc = ("AMSED/MSLR (3 levels, natural local order, rank<=32, 64 Lanczos steps)" if precond == "amsed" else "ICT(1e-3)")
    return f"3D Poisson 7-pt {grid}^3 (n={n}, nnz={nnz}), FCG + {pc}, tol {tol:g}, b~N(0,1) seed {SEED}"


def build_precond(PB, A, precond: str, precision: int):
    """Host setup of the preconditioner (timed separately, outside the solve)."""
    if precond == "amsed":
        return PB.HostAmsed(A, precision=precision, **AMSED)
    return PB.HostFactor(A, PB.PRECOND_IC, tol=1e-3, precision=precision)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="prism", choices=["prism", "reference"])
    p.add_argument("--grid", type=int, default=128)
    p.add_argument("--precond", default="amsed", choices=["amsed", "ic"])
    p.add_argument("--tol", type=float, default=1e-10)
    p.add_argument("--no-fp64", action="store_true", help="skip the FP64-factor comparison solve")
    p.add_argument("--no-cpu-baseline", action="store_true", help="skip every reference CPU measurement")
    p.add_argument("--no-secondary", action="store_true", help="headline line without the other configurations")
    p.add_argument("--only-sweep", default=None, choices=["global", "stream"],
                   help="profiling aid: set up the workload with this sweep layout forced, run the level-0 "
                        "lower sweep of the preconditioner four times and the SpMV twice, and exit (no JSON line)")
    p.add_argument("--config", type=int, default=2, choices=[1, 2, 3, 4, 5],
                   help="2: the headline (3D Poisson, FCG + AMSED); 1: 2D Poisson 64^2, FCG + ICT; 3: 3D "
                        "convection-diffusion 100^3, FGMRES(50) + GMSLR; 4: batched solves (64 RHS on 2D 512^2 "
                        "+ 256 uneven 2D systems); 5: differentiable 64^3 variable-coefficient diffusion")
    p.add_argument("--full-batch-reference", action="store_true",
                   help="config 4: time the reference on all 64 right-hand sides instead of 16")
    return p.parse_args()


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_gbs():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def host_cpu() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return f"{line.split(':', 1)[1].strip()}, nproc {os.cpu_count()}"
    except Exception:
        pass
    return f"{platform.processor() or 'unknown CPU'}, nproc {os.cpu_count()}"


# ---------------------------------------------------------------------------
# reference CPU solver (oracle/_ref timing build, else the oracle port)
# ---------------------------------------------------------------------------
class CpuReference:
    """The reference's CG<double> + AMSEDPrecondition<float,double> (or
    IncompleteCholesky<float,double>) on the host cores (oracle/_ref, built from
    the reference's sources with its Release flags; 4 OpenMP threads as
    THREAD_NUM hard-wires), else the oracle port.  Setup runs once in the
    constructor (so the solve's own setup() is a no-op, AMSEDPrecondition.cpp:
    1952) and is excluded from the timings."""

    def __init__(self, grid: int, tol: float, precond: str = "amsed"):
        from oracle import ref
        self.tol = tol
        self.b = np.random.default_rng(SEED).standard_normal(grid ** 3)
        t0 = time.perf_counter()
        if ref.available(fast=True):
            self.A = ref.RefCSR.laplacian(grid, grid, grid, fast=True)
            if precond == "amsed":
                a = AMSED
                self.P = ref.RefAmsed(self.A, a["levels"], a["lanczos_steps"], a["low_rank"], a["eig_bound"],
                                      a["reorder"], a["lowrank_type"], a["lanczos_type"], True)
            else:
                self.P = ref.RefPrecond(self.A, ref.KIND_IC, True, 1e-3)
            self.P.setup()
            self.cores, self.kind = 4, "reference"
            self._solve = lambda: ref.cg_solve(self.A, self.P, self.b, tol=tol, maxit=1000, flexible=True)[1]
        else:
            import prispack_b200 as PB
            from oracle import oracle as orc
            A = PB.CSRMatrix.laplacian(grid, grid, grid)
            F = build_precond(PB, A, precond, PB.PRISM_FP32)
            if precond == "amsed":
                self._keep = orc.Amsed(F)
                OP = self._keep.precond()
            else:
                rp, ci, v, _ = F.arrays(0)
                OP = orc.Precond(1, A.n, (rp, ci, v))
            self.cores, self.kind = 1, "port"
            self._solve = lambda: orc.cg(A.rowptr, A.col, A.val, self.b, OP, tol=tol, maxit=1000)[1]
        self.setup_s = time.perf_counter() - t0

    def full(self) -> dict:
        """One complete solve to the tolerance, timed unscaled."""
        t = time.perf_counter()
        it = self._solve()
        s = time.perf_counter() - t
        build = REF_BUILD if self.kind == "reference" else "the oracle's C port, 1 thread"
        return {"value": s * 1e3, "unit": "ms", "cores": self.cores, "kind": self.kind, "iters": it,
                "sample": f"one full FCG solve to {self.tol:g} ({it} iterations, {s:.2f} s) of the same system; host "
                          f"setup {self.setup_s:.1f} s excluded; {build}; host {host_cpu()}"}


def reference_fp64_solution(grid: int, tol: float, precond: str):
    """The reference's own FP64 solve of the headline system (parity build: no fast-math),
    untimed: (x, iterations), or None where the reference build is absent."""
    from oracle import ref
    if not ref.available():
        return None
    A = ref.RefCSR.laplacian(grid, grid, grid)
    if precond == "amsed":
        a = AMSED
        P = ref.RefAmsed(A, a["levels"], a["lanczos_steps"], a["low_rank"], a["eig_bound"], a["reorder"],
                         a["lowrank_type"], a["lanczos_type"], False)
    else:
        P = ref.RefPrecond(A, ref.KIND_IC, False, 1e-3)
    P.setup()
    b = np.random.default_rng(SEED).standard_normal(grid ** 3)
    x, it, _, conv = ref.cg_solve(A, P, b, tol=tol, maxit=1000, flexible=True)
    return (x, it) if conv else None


# ---------------------------------------------------------------------------
# secondary configurations (one GPU; rank 0 only)
# ---------------------------------------------------------------------------
CONVDIFF = dict(grid=100, pe=50.0, levels=4, low_rank=24, restart=50)


def _device_ms(stream, fn, steps, warm):
    import torch
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    out = [fn() for _ in range(steps)]
    ev1.record(stream)
    torch.cuda.synchronize()
    return ev0.elapsed_time(ev1) / steps, out


def _ref_ready(args):
    if args.no_cpu_baseline:
        return None
    from oracle import ref
    return ref if ref.available(fast=True) else None


def bench_config1(args, local):
    """2D Poisson 64^2 (n = 4096), FCG + ICT(1e-3), b ~ U[-1,1] seeded, tol 1e-8, max
    1000 iterations: the reference's own CPU case.  L2-resident: a latency figure."""
    import torch
    import prispack_b200 as PB
    A = PB.CSRMatrix.laplacian(64, 64, 1)
    b_host = np.random.default_rng(SEED).uniform(-1.0, 1.0, A.n)
    S = PB.DeviceSystem(A, device=local)
    stream = torch.cuda.current_stream()
    S.set_stream(stream.cuda_stream)
    S.set_precond(PB.PRECOND_IC, tol=1e-3)
    b = torch.tensor(b_host, device="cuda")
    x = torch.zeros_like(b)

    def one():
        x.zero_()
        return S.solve(b, x, tol=1e-8, max_iter=1000)[1]

    ms, sts = _device_ms(stream, one, max(args.steps, 5) * 4, 3)
    out = {"workload": "2D Poisson 5-pt 64^2 (n=4096, nnz=20224), FCG + ICT(1e-3), tol 1e-8, b~U[-1,1] "
                       f"seed {SEED}, FP64", "ms": round(ms, 4), "iterations": sts[-1].num_iter,
           "true_rel_residual": sts[-1].true_rel_residual}
    ref = _ref_ready(args)
    if ref is not None:
        RA = ref.RefCSR.laplacian(64, 64, 1, fast=True)
        RP = ref.RefPrecond(RA, ref.KIND_IC, False, 1e-3)
        RP.setup()
        reps, t = 20, time.perf_counter()
        for _ in range(reps):
            xr, itr, _, _ = ref.cg_solve(RA, RP, b_host, tol=1e-8, maxit=1000, flexible=True)
        cpu_ms = (time.perf_counter() - t) * 1e3 / reps
        _, st = S.solve(b_host, tol=1e-8, max_iter=1000, x_ref=xr)
        out.update({"cpu_baseline": {"value": round(cpu_ms, 3), "unit": "ms", "cores": 4, "kind": "reference",
                                     "iters": itr, "sample": f"mean of {reps} full reference FCG + "
                                     f"IncompleteCholesky<double,double> solves; {REF_BUILD}"},
                    "forward_error_vs_reference": st.forward_error, "iteration_diff": sts[-1].num_iter - itr})
    return out


def bench_convdiff(args, local):
    """3D convection-diffusion 100^3 (central diffusion + first-order upwind
    convection, v = (1, 0.5, 0.25) * Pe, Pe = 50), FGMRES(50) + GMSLR (4 levels,
    rank 24, ILUT(20, 1e-2) blocks), FP32 factor values / FP64 Arnoldi, tol 1e-10;
    the same solve with FP64 factors beside it, and the reference's own FGMRES +
    GMSLR on the host cores."""
    import torch
    import prispack_b200 as PB
    c = CONVDIFF
    g, pe = c["grid"], c["pe"]
    torch.cuda.set_device(local)
    A = PB.CSRMatrix.convection_diffusion(g, g, g, pe, 0.5 * pe, 0.25 * pe)
    b_host = np.random.default_rng(SEED).standard_normal(A.n)
    stream = torch.cuda.current_stream()
    res = {}
    for name, prec in (("fp32", PB.PRISM_FP32_APPLY), ("fp64", PB.PRISM_FP64)):
        t0 = time.perf_counter()
        G = PB.HostGmslr(A, levels=c["levels"], low_rank=c["low_rank"], precision=prec)
        setup_s = time.perf_counter() - t0
        S = PB.DeviceSystem(A, device=local)
        S.set_stream(stream.cuda_stream)
        S.attach(G)
        b = torch.tensor(b_host, device="cuda")
        x = torch.zeros(A.n, dtype=torch.float64, device="cuda")

        def one():
            x.zero_()
            return S.solve(b, x, solver=PB.SOLVER_FGMRES, tol=args.tol, max_iter=1000, restart=c["restart"])[1]

        ms, sts = _device_ms(stream, one, max(1, args.steps // 2), 1)
        st = sts[-1]
        res[name] = {"ms": ms, "iters": st.num_iter, "true_rel_residual": st.true_rel_residual,
                     "converged": bool(st.converged), "host_setup_s": round(setup_s, 2), "info": G.info(),
                     "S": S, "G": G, "host_syncs": st.host_syncs, "graph_nodes": st.graph_nodes}
    S32 = res["fp32"]["S"]

    def plain_one():
        x.zero_()
        return S32.solve(b, x, solver=PB.SOLVER_FGMRES, tol=args.tol, max_iter=1000, restart=c["restart"],
                         launch_mode=PB.LAUNCH_STREAM)[1]

    plain_ms, plain_sts = _device_ms(stream, plain_one, max(1, args.steps // 2), 1)
    pin_b = torch.from_numpy(b_host).pin_memory()
    pin_x = torch.zeros(A.n, dtype=torch.float64).pin_memory()
    bnp, xnp = pin_b.numpy(), pin_x.numpy()

    def host_one():
        xnp[:] = 0.0
        return S32.solve(bnp, xnp, solver=PB.SOLVER_FGMRES, tol=args.tol, max_iter=1000, restart=c["restart"])[1]

    e2e_ms, _ = _device_ms(stream, host_one, 1, 1)
    cpu, fwd = None, {}
    ref = _ref_ready(args)
    if ref is not None:
        RA = ref.RefCSR.from_arrays(A.rowptr, A.col, A.val, fast=True)
        RG = ref.RefGmslr(RA, c["levels"], 20, c["low_rank"], low_precision=True)
        RG.setup()
        t = time.perf_counter()
        xr, it, err, conv = ref.gmres_solve(RA, RG, b_host, tol=args.tol, restart=c["restart"], flexible=True)
        cpu = {"value": round((time.perf_counter() - t) * 1e3, 1), "unit": "ms", "cores": 4, "kind": "reference",
               "iters": it, "sample": f"one full reference FGMRES({c['restart']}) + GMSLR<float,double> solve: {it} "
                                      f"iterations, error {err:.2e}, converged {conv}; host setup excluded; {REF_BUILD}"}
        for name in ("fp32", "fp64"):
            _, st = res[name]["S"].solve(b_host, solver=PB.SOLVER_FGMRES, tol=args.tol, max_iter=1000,
                                         restart=c["restart"], x_ref=xr)
            fwd[name] = st.forward_error
    r32, r64 = res["fp32"], res["fp64"]
    info = r32["info"]
    return {"workload": f"3D convection-diffusion {g}^3 (n={A.n}, nnz={A.nnz}), central diffusion + first-order "
                        f"upwind convection, v=(1,0.5,0.25)*{pe:g}, FGMRES({c['restart']}) + GMSLR ({c['levels']} "
                        f"levels, rank {c['low_rank']}), tol {args.tol:g}, b~N(0,1) seed {SEED}",
            "ms": round(r32["ms"], 3), "precision": "PRISM_FP32_APPLY", "iterations": r32["iters"],
            "true_rel_residual": r32["true_rel_residual"], "converged": r32["converged"],
            "host_setup_s": r32["host_setup_s"],
            "gmslr": {"nlev": info["nlev"], "lev_ptr": info["lev_ptr"].tolist(), "ranks": info["ranks"].tolist(),
                      "mnnz": info["mnnz"]},
            "e2e": {"value": round(e2e_ms, 3), "unit": "ms", "h2d_bytes_per_step": 16 * A.n,
                    "d2h_bytes_per_step": 8 * A.n},
            "fp64_factor": {"ms": round(r64["ms"], 3), "iters": r64["iters"],
                            "true_rel_residual": r64["true_rel_residual"], "mixed_speedup": r64["ms"] / r32["ms"]},
            "launches": {"cycle_graph": {"ms": round(r32["ms"], 3), "host_syncs": r32["host_syncs"],
                                         "graph_nodes_per_arnoldi_step": r32["graph_nodes"]},
                         "plain": {"ms": round(plain_ms, 3), "host_syncs": plain_sts[-1].host_syncs,
                                   "iters": plain_sts[-1].num_iter}},
            "forward_error_vs_reference": fwd or None, "cpu_baseline": cpu}


def bench_adjoint(args, local):
    """Differentiable solve: 3D variable-coefficient diffusion 64^3, kappa =
    exp(g), g a Gaussian random field (sigma 1, correlation length 8 cells);
    loss ||x - x*||^2; forward FCG + IC solve and hand-written adjoint (one
    solve with the same preconditioner + the sampled outer product), timed
    together; gradient wrt kappa checked against central differences
    (h = 1e-6) on 64 random cells."""
    import torch
    import prispack_b200 as PB
    from prispack_b200.autograd import DiffusionPattern, SolveSpec, gaussian_random_field, solve
    torch.cuda.set_device(local)
    D = DiffusionPattern(64, 64, 64)
    kappa = np.exp(gaussian_random_field(D.shape, 1.0, 8.0, seed=SEED))
    rng = np.random.default_rng(SEED + 1)
    b_host, xs_host = rng.standard_normal(D.n), rng.standard_normal(D.n)
    S = PB.DeviceSystem(D.matrix(kappa), device=local)
    stream = torch.cuda.current_stream()
    S.set_stream(stream.cuda_stream)
    S.set_precond(PB.PRECOND_IC, tol=1e-3)  # factored once: every step runs with the same kappa
    spec = SolveSpec(tol=1e-13, max_iter=5000, refactor=False)
    b = torch.tensor(b_host, device="cuda")
    xs = torch.tensor(xs_host, device="cuda")

    def step():
        kap = torch.tensor(kappa, device="cuda", requires_grad=True)
        x = solve(S, D.values(kap), b, spec)
        loss = ((x - xs) ** 2).sum()
        loss.backward()
        return kap.grad

    ms, grads = _device_ms(stream, step, max(1, args.steps // 2), 1)
    grad = grads[-1].cpu().numpy()
    # the same step with the IC factor recomputed on the device at every forward call
    spec_rf = SolveSpec(tol=1e-13, max_iter=5000, refactor="device")

    def step_rf():
        kap = torch.tensor(kappa, device="cuda", requires_grad=True)
        x = solve(S, D.values(kap), b, spec_rf)
        loss = ((x - xs) ** 2).sum()
        loss.backward()
        return kap.grad

    ms_rf, grads_rf = _device_ms(stream, step_rf, max(1, args.steps // 2), 1)
    # host factorisation (what a new setup repeats) against the device refactorisation
    t0 = time.perf_counter()
    PB.HostFactor(D.matrix(kappa), PB.PRECOND_IC, tol=1e-3)
    host_factor_ms = (time.perf_counter() - t0) * 1e3
    rf_ms, _ = _device_ms(stream, S.refactor, 3, 1)
    # central differences without cancellation: L+ - L- = d . (2 x- + d - 2 x*), d = x+ - x-
    cells = rng.choice(D.n, 64, replace=False)
    rows = np.repeat(np.arange(D.n), np.diff(D.A0.rowptr.astype(np.int64)))
    h = 1e-6
    fd = []
    for m in cells:
        kp, km = kappa.copy(), kappa.copy()
        kp[m] += h
        km[m] -= h
        vp = D.values(torch.from_numpy(kp)).numpy()
        vm = D.values(torch.from_numpy(km)).numpy()
        S.update_values(vm)  # the factor of the unperturbed kappa stays: the solves stay exact
        xm, _ = S.solve(b_host, tol=1e-13, max_iter=5000)
        r = np.zeros(D.n)
        np.add.at(r, rows, (vp - vm) * xm[D.A0.col])
        S.update_values(vp)
        d, _ = S.solve(-r, tol=1e-13, max_iter=5000)
        fd.append(float(d @ (2 * xm + d - 2 * xs_host)) / (2 * h))
    fd = np.array(fd)
    err = np.abs(fd - grad[cells]) / np.maximum(np.abs(grad[cells]), 1e-12 * np.abs(grad).max())
    return {"workload": "3D variable-coefficient diffusion 64^3 (n=262144), kappa=exp(g), g Gaussian random field "
                        "(sigma 1, correlation length 8 cells), loss ||x - x*||^2, FCG + IC (factored once), tol "
                        "1e-13; grad wrt kappa and b by the adjoint",
            "ms": round(ms, 3), "unit": "ms forward + adjoint",
            "refactor_each_step": {"ms": round(ms_rf, 3),
                                   "grad_rel_diff_to_factored_once": float(
                                       np.abs(grads_rf[-1].cpu().numpy() - grad).max() / np.abs(grad).max())},
            "refactor": {"what": "IC(1e-3) factor of the 64^3 operator",
                         "host_factorisation_ms": round(host_factor_ms, 1), "device_refactorisation_ms": round(rf_ms, 3),
                         "speedup": round(host_factor_ms / rf_ms, 1)},
            "fd_check": {"cells": 64, "h": h, "max_rel_err": float(err.max()), "median_rel_err": float(np.median(err)),
                         "within_1e-6": int((err <= 1e-6).sum())},
            "cpu_baseline": None, "note": "the reference has no adjoint or gradient path"}


def bench_batched(args, local):
    """Batched solves, FCG + ICT(1e-3) with FP32 factor values, tol 1e-10:
    (a) 2D Poisson 512^2 with a block of 64 random-normal right-hand sides,
    one block solve (prism_solve_batched) against 64 solves one after another,
    and the same block with AMSED / MSLR (FP32 factor values; block sweeps per
    level; the low-rank block products on the tensor cores in BF16 with FP32
    accumulation);
    (b) 256 independent 2D Poisson systems on grids with sides drawn uniformly
    from 32..256, assembled on the diagonal of one CSR and solved together
    (prism_solve_segments).  The reference solves one right-hand side and one
    system per call: it is timed on 16 of the 64 right-hand sides (all 64 with
    --full-batch-reference) and on all 256 systems."""
    import torch
    import prispack_b200 as PB
    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    rng = np.random.default_rng(SEED)
    tol = args.tol
    # ---- (a) block of 64 right-hand sides
    A = PB.CSRMatrix.laplacian(512, 512, 1)
    k = 64
    S = PB.DeviceSystem(A, device=local)
    S.set_stream(stream.cuda_stream)
    S.set_precond(PB.PRECOND_IC, tol=1e-3, precision=PB.PRISM_FP32)
    B_host = rng.standard_normal((k, A.n))
    B = torch.tensor(B_host, device="cuda")

    def block():
        return S.solve_batched(B, tol=tol, max_iter=1000)[1]

    block_ms, bst = _device_ms(stream, block, max(1, args.steps // 2), 1)
    bst = bst[-1]
    x0 = torch.zeros(A.n, dtype=torch.float64, device="cuda")

    def single():
        x0.zero_()
        return S.solve(B[0], x0, tol=tol, max_iter=1000)[1]

    single_ms, _ = _device_ms(stream, single, max(1, args.steps), 1)
    # ---- (a') the same block with AMSED / MSLR, FP32 factor values: block sweeps per level and
    # the low-rank block products on the tensor cores (BF16 operands, FP32 accumulation)
    t0 = time.perf_counter()
    HA = PB.HostAmsed(A, precision=PB.PRISM_FP32, **AMSED)
    amsed_setup_s = time.perf_counter() - t0
    SA = PB.DeviceSystem(A, device=local)
    SA.set_stream(stream.cuda_stream)
    SA.attach(HA)

    def block_amsed():
        return SA.solve_batched(B, tol=tol, max_iter=1000)[1]

    am_ms, amst = _device_ms(stream, block_amsed, max(1, args.steps // 2), 1)
    amst = amst[-1]
    # ---- (b) 256 uneven systems
    sides = rng.integers(32, 257, size=256)
    blocks = [PB.CSRMatrix.laplacian(int(q), int(q), 1) for q in sides]
    Ab, seg = PB.CSRMatrix.block_diagonal(blocks)
    t0 = time.perf_counter()
    Sb = PB.DeviceSystem(Ab, device=local)
    Sb.set_stream(stream.cuda_stream)
    Sb.set_precond(PB.PRECOND_IC, tol=1e-3, precision=PB.PRISM_FP32)
    setup_s = time.perf_counter() - t0
    bb_host = rng.standard_normal(Ab.n)
    bb = torch.tensor(bb_host, device="cuda")
    xb = torch.zeros_like(bb)

    def segs():
        xb.zero_()
        return Sb.solve_segments(seg, bb, xb, tol=tol, max_iter=1000)[1]

    seg_ms, segst = _device_ms(stream, segs, max(1, args.steps // 2), 1)
    segst = segst[-1]
    cpu = None
    cpu_amsed = None
    ref = _ref_ready(args)
    if ref is not None:
        RA = ref.RefCSR.laplacian(512, 512, 1, fast=True)
        RP = ref.RefPrecond(RA, ref.KIND_IC, True, 1e-3)
        RP.setup()
        kk = k if args.full_batch_reference else 16
        t = time.perf_counter()
        for c in range(kk):
            ref.cg_solve(RA, RP, B_host[c], tol=tol, maxit=1000, flexible=True)
        rhs_s = time.perf_counter() - t
        a = AMSED
        RM = ref.RefAmsed(RA, a["levels"], a["lanczos_steps"], a["low_rank"], a["eig_bound"], a["reorder"],
                          a["lowrank_type"], a["lanczos_type"], True)
        RM.setup()
        t = time.perf_counter()
        for c in range(kk):
            ref.cg_solve(RA, RM, B_host[c], tol=tol, maxit=1000, flexible=True)
        am_rhs_s = time.perf_counter() - t
        cpu_amsed = {"value": round(am_rhs_s * k / kk * 1e3, 1), "unit": "ms", "cores": 4, "kind": "reference",
                     "sample": f"reference FCG + AMSEDPrecondition<float,double> solves timed one by one: {kk} of "
                               f"the 64 right-hand sides ({am_rhs_s:.2f} s; the total counts {k}/{kk} times that); "
                               f"setup excluded; {REF_BUILD}"}
        sys_s = 0.0
        for q, Bq in enumerate(blocks):
            Rq = ref.RefCSR.from_arrays(Bq.rowptr, Bq.col, Bq.val, fast=True)
            Pq = ref.RefPrecond(Rq, ref.KIND_IC, True, 1e-3)
            Pq.setup()
            t = time.perf_counter()
            ref.cg_solve(Rq, Pq, bb_host[seg[q]:seg[q + 1]], tol=tol, maxit=1000, flexible=True)
            sys_s += time.perf_counter() - t
        cpu = {"value": round((rhs_s * k / kk + sys_s) * 1e3, 1), "unit": "ms", "cores": 4, "kind": "reference",
               "block_rhs_measured": kk, "block_rhs_ms_measured": round(rhs_s * 1e3, 1),
               "uneven_systems_ms_measured": round(sys_s * 1e3, 1),
               "sample": f"reference FCG + IncompleteCholesky<float,double> solves timed one by one: {kk} of the 64 "
                         f"right-hand sides ({rhs_s:.2f} s; the total counts {k}/{kk} times that) and all 256 uneven "
                         f"systems ({sys_s:.2f} s); setups excluded; {REF_BUILD}"}
    its = [q.num_iter for q in segst]
    return {"workload": "FCG + ICT(1e-3), FP32 factor values, tol 1e-10; (a) 2D Poisson 512^2 (n=262144) with 64 "
                        f"N(0,1) right-hand sides; (b) 256 2D Poisson systems, sides U{{32..256}} seed {SEED} "
                        f"(total n={Ab.n}, nnz={Ab.nnz})",
            "ms": round(block_ms + seg_ms, 3),
            "block_of_64": {"ms": round(block_ms, 3), "iters_first4": [q.num_iter for q in bst][:4],
                            "all_converged": all(q.converged for q in bst), "one_rhs_alone_ms": round(single_ms, 3),
                            "speedup_vs_64_single": round(64 * single_ms / block_ms, 2)},
            "block_of_64_amsed": {"ms": round(am_ms, 3), "iters_first4": [q.num_iter for q in amst][:4],
                                  "all_converged": all(q.converged for q in amst),
                                  "max_true_rel_residual": max(q.true_rel_residual for q in amst),
                                  "precond": "AMSED/MSLR (3 levels, natural local order), FP32 factor values, block "
                                             "sweeps per level, low-rank W (H o (W^T X)) on the tensor cores "
                                             "(mma.sync m16n8k16, BF16 operands, FP32 accumulation)",
                                  "ranks": HA.info()["ranks"].tolist(), "host_setup_s": round(amsed_setup_s, 2),
                                  "cpu_baseline": cpu_amsed},
            "uneven_256": {"ms": round(seg_ms, 3), "iters_min_max": [min(its), max(its)],
                           "all_converged": all(q.converged for q in segst),
                           "max_true_rel_residual": max(q.true_rel_residual for q in segst),
                           "host_setup_s": round(setup_s, 1)},
            "cpu_baseline": cpu}


SECONDARY = {1: bench_config1, 3: bench_convdiff, 4: bench_batched, 5: bench_adjoint}


# ---------------------------------------------------------------------------
_JSON_OUT = None


def quiet_stdout():
    """The reference library prints its setup progress to stdout; route fd 1 to
    stderr for the whole run so that stdout carries the JSON line alone."""
    global _JSON_OUT
    sys.stdout.flush()
    _JSON_OUT = os.fdopen(os.dup(1), "w")
    os.dup2(2, 1)


def emit(obj):
    out = _JSON_OUT if _JSON_OUT is not None else sys.stdout
    out.write(json.dumps(obj) + "\n")
    out.flush()


def standalone_line(n: int, r: dict, args) -> dict:
    """A secondary configuration as its own JSON line (--config N)."""
    metric = {1: "time-to-1e-8 rel. residual, FCG + ICT, 2D Poisson 64^2, 1 B200",
              3: "time-to-1e-10 rel. residual, FGMRES(50) + GMSLR, mixed FP32-factor / FP64-Arnoldi, 1 B200",
              4: "batched time-to-1e-10: 64 RHS on 2D Poisson 512^2 + 256 uneven 2D Poisson systems, 1 B200",
              5: "forward + adjoint solve time, variable-coefficient diffusion, 1 B200"}[n]
    line = {"metric": metric, "value": r["ms"], "unit": "ms", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["ms"], "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if n in (1, 5) else "f64 (Krylov) / f32 (factor values)",
            "data": "synthetic", "config": {k: v for k, v in r.items() if k not in ("ms", "cpu_baseline", "e2e")},
            "cpu_baseline": r.get("cpu_baseline")}
    if "e2e" in r:
        line["e2e"] = r["e2e"]
    return line


def main():
    args = parse()
    quiet_stdout()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.config != 2:
        if rank != 0 or args.impl == "reference":
            if args.impl == "reference" and rank == 0:
                emit({"impl": "reference", "unavailable": "secondary configs carry their reference "
                      "timing in the prism line's cpu_baseline"})
            return
        import torch
        torch.cuda.set_device(local)
        return emit(standalone_line(args.config, SECONDARY[args.config](args, local), args))

    if args.impl == "reference":
        return reference_arm(args, rank, world)

    import torch
    import prispack_b200 as PB

    if args.only_sweep:
        os.environ["PRISM_SWEEP_KERNEL"] = args.only_sweep
        torch.cuda.set_device(local)
        A = PB.CSRMatrix.laplacian(args.grid, args.grid, args.grid)
        S = PB.DeviceSystem(A, device=local)
        S.set_stream(torch.cuda.current_stream().cuda_stream)
        prec = PB.PRISM_FP32_APPLY if args.only_sweep == "stream" else PB.PRISM_FP32
        S.attach(build_precond(PB, A, args.precond, prec))
        info = S.sweep_info(0)
        vin = torch.tensor(np.random.default_rng(SEED).standard_normal(info["n"]), device="cuda")
        vout = torch.empty_like(vin)
        for _ in range(4):
            S.sweep_device(0, vin, vout, 1)
        x = torch.tensor(np.random.default_rng(SEED).standard_normal(A.n), device="cuda")
        y = torch.empty_like(x)
        for _ in range(2):
            S.spmv_into(x, y)
        torch.cuda.synchronize()
        print(f"sweep 0: {info}", file=sys.stderr)
        return

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    g = args.grid
    A = PB.CSRMatrix.laplacian(g, g, g)
    n = A.n
    b_host = np.random.default_rng(SEED).standard_normal(n)
    t0 = time.perf_counter()
    F32 = build_precond(PB, A, args.precond, PB.PRISM_FP32_APPLY)
    setup32_s = time.perf_counter() - t0
    S = PB.DeviceSystem(A, device=local)
    stream = torch.cuda.current_stream()
    S.set_stream(stream.cuda_stream)
    S.attach(F32)
    b = torch.tensor(b_host, device="cuda")
    x = torch.zeros(n, dtype=torch.float64, device="cuda")

    def barrier():
        if dist is not None:
            dist.barrier()

    def timed_solves(steps, warm):
        for _ in range(warm):
            x.zero_()
            S.solve(b, x, tol=args.tol, max_iter=1000)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        launches0 = PB.kernel_launch_count()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        stats = []
        for _ in range(steps):
            x.zero_()
            _, st = S.solve(b, x, tol=args.tol, max_iter=1000)
            stats.append((st.num_iter, st.true_rel_residual, st.converged, st.device_ms))
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1) / steps
        return ms, stats, PB.kernel_launch_count() - launches0

    clocks = ClockSampler(local)
    clocks.start()
    ms32, stats32, launches = timed_solves(args.steps, args.warmup)
    clk = clocks.stop()
    iters = stats32[-1][0]

    # ---- e2e through the host-buffer C-ABI call (H2D b, x0; D2H x inside the timed region)
    pin_b = torch.from_numpy(b_host).pin_memory()
    pin_x = torch.zeros(n, dtype=torch.float64).pin_memory()
    bnp, xnp = pin_b.numpy(), pin_x.numpy()
    S.solve(bnp, xnp, tol=args.tol, max_iter=1000)  # warm
    torch.cuda.synchronize()
    barrier()
    e2e = []
    for _ in range(max(1, args.steps)):
        xnp[:] = 0.0
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        xs, st = S.solve(bnp, xnp, tol=args.tol, max_iter=1000)
        e1.record(stream)
        torch.cuda.synchronize()
        e2e.append(e0.elapsed_time(e1))
    e2e_ms = statistics.mean(e2e)

    # ---- dominant kernel: the triangular sweeps, each timed alone with CUDA events.  For AMSED
    # these are the lower/upper sweeps of the level-0 block-diagonal factor (every subdomain in
    # one launch, the largest sweeps of the apply); for ICT the whole-matrix factor's sweeps.
    reps = 10
    sweep_ms, sweep_infos = [], []
    for sw in (0, 1):
        info = S.sweep_info(sw)
        sweep_infos.append(info)
        vin = torch.randn(info["n"], dtype=torch.float64, device="cuda")
        vout = torch.empty_like(vin)
        S.sweep_device(sw, vin, vout, 1)
        torch.cuda.synchronize()
        tot = 0.0
        for _ in range(reps):
            s0 = torch.cuda.Event(enable_timing=True)
            s1 = torch.cuda.Event(enable_timing=True)
            s0.record(stream)
            # the whole sweep as the apply runs it: marking the output pending (and, for the
            # streamed layout, staging the right-hand side into its round records), then the sweep
            S.sweep_device(sw, vin, vout, 1)
            s1.record(stream)
            torch.cuda.synchronize()
            tot += s0.elapsed_time(s1)
        sweep_ms.append(tot / reps)
    # algorithmic bytes of one sweep launch: per stored entry a column index (4 B) and a value
    # (4 B FP32); per row its offset (4 B), position->row map (4 B), diagonal (8 B), right-hand
    # side read (8 B) and result write (8 B)
    sweep_bytes = [i["nnz"] * (4 + i["value_bytes"]) + i["n"] * 32 + 4 for i in sweep_infos]
    achieved = statistics.mean(b_ / (t * 1e-3) / 1e9 for b_, t in zip(sweep_bytes, sweep_ms))
    peak, peak_src = measured_peak_gbs()
    vin = torch.randn(n, dtype=torch.float64, device="cuda")
    vout = torch.empty_like(vin)

    # ---- SpMV alone (the other bandwidth kernel), for reference
    spmv_ms = []
    for _ in range(reps):
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        S.spmv_into(vin, vout)
        s1.record(stream)
        torch.cuda.synchronize()
        spmv_ms.append(s0.elapsed_time(s1))
    spmv_bytes = 12 * A.nnz + 20 * n + 4
    spmv_gbs = spmv_bytes / (statistics.median(spmv_ms) * 1e-3) / 1e9

    # ---- the reference's own FP64 solution of the same system (untimed): forward errors
    xref = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            xref = reference_fp64_solution(g, args.tol, args.precond)
        except Exception as e:  # reported, not fatal
            print(f"reference FP64 solve failed: {e}", file=sys.stderr)
    parity = None
    if xref is not None:
        xr_d = torch.tensor(xref[0], device="cuda")
        x.zero_()
        _, stp = S.solve(b, x, tol=args.tol, max_iter=1000, x_ref=xr_d)
        parity = {"reference_fp64_iters": xref[1], "mixed": {"forward_error": stp.forward_error,
                                                              "iteration_diff": stp.num_iter - xref[1]}}

    # ---- FP64-factor solve beside it
    fp64 = None
    fp32_storage = None
    if not args.no_fp64:
        t0 = time.perf_counter()
        F64 = build_precond(PB, A, args.precond, PB.PRISM_FP64)
        setup64_s = time.perf_counter() - t0
        S.attach(F64)
        ms64, stats64, _ = timed_solves(max(1, args.steps // 2), 1)
        fp64 = {"ms": ms64, "iters": stats64[-1][0], "true_rel_residual": stats64[-1][1],
                "mixed_speedup": ms64 / ms32, "host_setup_s": setup64_s}
        if xref is not None:
            x.zero_()
            _, stp = S.solve(b, x, tol=args.tol, max_iter=1000, x_ref=xr_d)
            parity["fp64"] = {"forward_error": stp.forward_error, "iteration_diff": stp.num_iter - xref[1]}
        # the reference's <float,double> instantiation: float values, double arithmetic
        FS = build_precond(PB, A, args.precond, PB.PRISM_FP32)
        S.attach(FS)
        msS, statsS, _ = timed_solves(max(1, args.steps // 2), 1)
        fp32_storage = {"ms": round(msS, 3), "iters": statsS[-1][0], "true_rel_residual": statsS[-1][1],
                        "converged": bool(statsS[-1][2]), "speedup_over_fp64": ms64 / msS,
                        "sweeps": "float factor values, double arithmetic (the reference's <float,double>)"}
        del FS
        S.attach(F32)

    # ---- max over ranks
    ms32, e2e_ms = max_over_ranks([ms32, e2e_ms], dist, "cuda")

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = CpuReference(g, args.tol, args.precond).full()
            cpu.pop("iters", None)
        except Exception as e:  # reported, not fatal
            cpu = {"value": None, "unit": "ms", "cores": 0, "kind": "unavailable", "sample": str(e)[:200]}

    configs = None
    if rank == 0 and world == 1 and not args.no_secondary:
        configs = {}
        for k, fn in SECONDARY.items():
            try:
                configs[str(k)] = fn(args, local)
            except Exception as e:  # reported, not fatal
                configs[str(k)] = {"error": f"{type(e).__name__}: {e}"[:300]}

    if rank == 0:
        amsed_info = None
        if args.precond == "amsed":
            amsed_info = {k: (v.tolist() if hasattr(v, "tolist") else v) for k, v in F32.info().items()}
            amsed_info["note"] = ("ranks: the MSLR correction keeps the eigenpairs above the bound; rank 32 is a cap "
                                  "that this operator does not reach")
        line = {
            "metric": METRIC,
            "value": round(ms32, 4),
            "unit": "ms",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(ms32, 4),
            "higher_is_better": False,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64 (Krylov, SpMV, residual) / f32 (factor values and sweep arithmetic)",
            "data": "synthetic",
            "config": {"workload": workload(g, args.tol, args.precond), "n": n, "nnz": A.nnz,
                       "precond_nnz": F32.info()["mnnz"], "precision": "PRISM_FP32_APPLY", "amsed": amsed_info,
                       "iterations": iters, "true_rel_residual": stats32[-1][1],
                       "converged": bool(stats32[-1][2]), "host_setup_s": round(setup32_s, 2),
                       "l2": "inputs larger than L2 (A 216 MB + factor > 600 MB per solve)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "spmv_per_iter": 1},
            "e2e": {"value": round(e2e_ms, 4), "unit": "ms", "h2d_bytes_per_step": 2 * 8 * n,
                    "d2h_bytes_per_step": 8 * n},
            "roofline": {"bound": "hbm",
                         "kernel": ("level-0 block-diagonal sweeps" if args.precond == "amsed" else "ICT sweeps")
                                   + ", FP32 values and arithmetic (lower/upper average)",
                         "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_source": peak_src,
                         "bytes_per_launch": sweep_bytes, "launch_ms": [round(t, 4) for t in sweep_ms],
                         "rows": [i["n"] for i in sweep_infos], "wavefronts": [i["levels"] for i in sweep_infos],
                         "us_per_wavefront": [round(t * 1e3 / max(i["levels"], 1), 4)
                                              for t, i in zip(sweep_ms, sweep_infos)],
                         "kernels": [i["kernel"] for i in sweep_infos],
                         "traffic": round(statistics.mean(TRAFFIC_RATIO.get(i["kernel"], 1.0) * b_
                                                          for i, b_ in zip(sweep_infos, sweep_bytes))),
                         "traffic_source": TRAFFIC_SOURCE},
            "spmv": {"ms": round(statistics.median(spmv_ms), 4), "bytes": spmv_bytes, "GB/s": round(spmv_gbs, 1),
                     "frac": round(spmv_gbs / peak, 4), "shape": list(S.spmv_shape())},
            "fp64_factor": fp64,
            "fp32_storage": fp32_storage,
            "parity_vs_reference_fp64": parity,
            "cpu_baseline": cpu,
            "gpu_launches": int(launches / max(args.steps, 1)) * args.steps,
            "clocks": clk,
            "configs": configs,
        }
        emit(line)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def max_over_ranks(values, dist=None, device="cpu"):
    """Replicas run concurrently, so a job's time is its slowest rank's: the
    element-wise max of `values` over the process group (identity without one).
    Every rank takes this step, in the same order."""
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def reference_arm(args, rank, world):
    """The reference's own CPU solver on the host cores (rank 0 only): each step
    one complete solve to the tolerance, timed unscaled."""
    if rank != 0:
        return
    from oracle import ref
    R = CpuReference(args.grid, args.tol, args.precond)
    first = R.full()  # untimed warm-up; also sizes the run
    # every step is one full solve; at most about 150 s of them, so that the arm ends in minutes
    steps = max(1, min(args.steps, int(150e3 / max(first["value"], 1.0))))
    runs = [R.full() for _ in range(steps)]
    v = statistics.mean(r["value"] for r in runs)
    desc = runs[-1]
    if steps < args.steps:
        desc["sample"] += f"; mean of {steps} timed solves (of {args.steps} steps asked, to bound the run)"
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "ms", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(v, 3), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64 (Krylov) / f32 (factor values)",
            "data": "synthetic", "config": {"workload": workload(args.grid, args.tol, args.precond)},
            "cpu_baseline": {"value": round(v, 3), "unit": "ms", "cores": desc["cores"], "kind": desc["kind"],
                             "sample": desc["sample"]},
            "e2e": {"value": round(v, 3), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if not ref.available(fast=True):
        line["note"] = "reference build absent on this host: the oracle port was timed"
    emit(line)


if __name__ == "__main__":
    main()
