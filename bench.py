#!/usr/bin/env python
"""Benchmark: batched SQP solves/s on one B200 (replicas on N GPUs).

Workload (one "step" = one batched solve): iiwa14, N=32 knots, dt=0.01 s,
batch 1024 problems per GPU, seeded figure-8 end-effector goals, warm-started
from a perturbed converged solution (XU and lambda), 5 SQP iterations, PCG
max 173 iterations at tol 1e-5, FP32, cost weights at the reference interface
defaults.  Each timed step starts from the same warm start (the solver's
persistent lambda / rho are restored between steps, outside the timed region),
and L2 is flushed between steps.

  value     solves/s of the fused CUDA-graph form, inputs resident in HBM
  e2e       solves/s through gato_solve_host (host buffers; H2D of XU, x0,
            goals and D2H of XU inside the timed region)
  plain     solves/s of the plain per-kernel form, same workload
  by_precision  fused and plain solves/s in FP32, mixed (FP64 reductions)
            and FP64, the fused form's solves/s through the host API
            (e2e_value), and each form's device time per kernel group
  roofline  FP32 CUDA-core roofline of the kernel with the largest share of
            device time (the persistent PCG, k_pcg_rows_stream)
  cpu_baseline  the FP64 oracle of the same SQP on the host cores, bounded
            sample of the same workload
  accuracy_vs_fp64_oracle  every precision's trajectory error against the
            oracle, the oracle's own FP32-storage floor, and a converged
            (30-iteration) solve
  at_1e-4   the fastest precision whose trajectories all meet 1e-4 against
            the oracle (the largest error), with its fused/plain ratio

`--impl reference` times the reference's algorithm on the host CPU (the FP64
oracle port: the reference's solver has no CPU implementation and its CUDA
kernels do not compile for the host) on a bounded sample per step.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PLANT, N, DT = "iiwa14", 32, 0.01
# DRAM bytes (read + write) per launch from one ncu capture of the first SQP
# iteration of this workload (profiles/k_fused_kkt_schur_iiwa14_N32_B1024.md,
# profiles/k_pcg_rows_stream_iiwa14_N32_B1024.md); the KKT + Schur group is
# both of its kernels
TRAFFIC_PER_LAUNCH = {"fused_iter": 391_866_000, "pcg": 238_080_000}
KERNEL_NAMES = {"fused_iter": "k_fused_kkt + k_fused_schur", "pcg": "k_pcg_rows_stream",
                "line_search": "k_merit_ls", "merit": "k_merit_ls (one step size)"}
# kernels per timed group of gato_profile_solve (the KKT + Schur group is two)
KERNELS_PER_GROUP = {"fused_iter": 2}
SQP_ITERS, PCG_MAX, PCG_TOL = 5, 173, 1e-5
METRIC = "SQP solves/s (iiwa14 N=32, batch 1024, 5 SQP iters, PCG tol 1e-5)"
WORKLOAD = ("iiwa14 N=32 dt=0.01, batch 1024 per GPU, seeded figure-8 goals, perturbed "
            "converged warm start, 5 SQP iters, PCG max 173 tol 1e-5, interface-default costs")


def solver_kwargs():
    # BSQP interface defaults (python/bsqp/interface.py:13-26) with the
    # workload's iteration limits
    return dict(max_sqp_iters=SQP_ITERS, max_pcg_iters=PCG_MAX, pcg_tol=PCG_TOL, kkt_tol=1e-4,
                solve_ratio=1.0, mu=1.0, q_cost=2.0, qd_cost=1e-4, u_cost=1e-6, N_cost=50.0,
                q_lim_cost=1e-3, vel_lim_cost=0.0, ctrl_lim_cost=0.0, rho=0.0)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=1024)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "mixed", "fp64"],
                    help="headline solver arithmetic (fp64: profile workload only)")
    ap.add_argument("--cpu-sample", type=int, default=0,
                    help="problems in the CPU baseline sample (0: sized to ~10 s)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--workload", default="single",
                    choices=["single", "mixed", "mpc", "sweep", "profile"],
                    help="single: the headline iiwa14 N=32 batch; mixed: 4096 problems of "
                         "both plants and four horizons in one solve; profile: one solve per "
                         "form, untimed, as the target of an ncu capture")
    ap.add_argument("--horizon", type=int, default=N, help="knots (profile workload only)")
    ap.add_argument("--plant", default=PLANT, help="robot (profile workload only)")
    ap.add_argument("--sqp-iters", type=int, default=2, help="SQP iterations (profile workload only)")
    return ap.parse_args()


# --------------------------------------------------------------------------
# The workload, built the same way by both arms from the arm's own robot
# tables and forward kinematics: seeded problems (the formulas of
# gato_b200/workloads.py: q ~ U(0.8 x limits), qd ~ N(0, 0.1^2), figure-8
# end-effector goals in the shape of python/bsqp/common.py:27-45), solved in
# FP64 from the default warm start (30 SQP iterations, PCG tol 1e-6), then
# perturbed by seeded noise.  Both FP64 solves reproduce each other to about
# 1e-10, so after rounding to FP32 the two arms start from the same XU and
# lambda.
WARM_KW = dict(max_sqp_iters=30, pcg_tol=1e-6, max_pcg_iters=400)


def seeded_problems(nq, q_limit, fk, B, seed):
    """xs [B, 2nq], goal [B, 6N] (float32), the default warm start [B, traj]
    and the generator state."""
    rng = np.random.default_rng(seed)
    lim = np.array([q_limit[i] for i in range(nq)])
    xs = np.concatenate([rng.uniform(-0.8, 0.8, (B, nq)) * lim, rng.normal(0.0, 0.1, (B, nq))],
                        axis=1)
    p0 = fk(xs[:, :nq])
    centre = p0 + rng.normal(0.0, 0.02, (B, 3))
    amp, period = rng.uniform(0.1, 0.3, B), rng.uniform(2.0, 6.0, B)
    phase = rng.uniform(0.0, 2 * np.pi, B)
    th = np.pi / 4
    Rz = np.array([[np.cos(th), -np.sin(th), 0.0], [np.sin(th), np.cos(th), 0.0], [0, 0, 1.0]])
    tau = 2 * np.pi * np.arange(N)[None, :] * DT / period[:, None] + phase[:, None]
    local = np.stack([amp[:, None] * np.sin(tau), np.zeros_like(tau),
                      amp[:, None] * np.sin(2 * tau) / 2], axis=-1)
    goal = np.zeros((B, N, 6))
    goal[:, :, :3] = centre[:, None, :] + local @ Rz.T
    nx, nu = 2 * nq, nq
    xu = np.zeros((B, N, nx + nu))
    xu[:, :, :nx] = xs[:, None, :]
    xu = xu.reshape(B, -1)[:, : N * (nx + nu) - nu]
    return (xs.astype(np.float32), goal.reshape(B, 6 * N).astype(np.float32),
            xu.astype(np.float32), rng)


def perturbed_warm_start(xu_conv, lam, xs, nq, rng):
    """q, qd + N(0, 0.01^2) and u + N(0, 0.1^2) on every knot but x_0."""
    B = xu_conv.shape[0]
    nx, nu = 2 * nq, nq
    full = np.zeros((B, N * (nx + nu)))
    full[:, : xu_conv.shape[1]] = xu_conv
    full = full.reshape(B, N, nx + nu)
    full[:, 1:, :nx] += rng.normal(0.0, 0.01, (B, N - 1, nx))
    full[:, :, nx:] += rng.normal(0.0, 0.1, (B, N, nu))
    xu0 = full.reshape(B, -1)[:, : xu_conv.shape[1]].astype(np.float32)
    xu0[:, :nx] = xs
    return dict(xs=xs, xu=xu0, lam=np.asarray(lam).astype(np.float32))


def make_workload(batch, seed):
    """This arm's copy: the library's robot tables and kinematics, warm
    start from its FP64 solver."""
    import gato_b200
    from gato_b200.kinematics import ee_position
    model = gato_b200.builtin_model(PLANT)
    xs, goal, xu, rng = seeded_problems(model.nq, model.q_limit,
                                        lambda q: ee_position(model, q), batch, seed)
    s = gato_b200.BSQP(batch_size=batch, N=N, dt=DT, plant_type=PLANT, form="fused",
                       precision="fp64", **dict(solver_kwargs(), **WARM_KW))
    res = s.solve_raw(xu.astype(np.float64), DT, xs.astype(np.float64), goal.astype(np.float64))
    lam = s.get_lambda()
    s.close()
    return dict(perturbed_warm_start(res["XU"], lam, xs, model.nq, rng), goal=goal)


# Per-knot FLOPs of the reference's own device functions for iiwa14, counted
# by running them with an operation-counting scalar type
# (oracle/ref_shim/flop_count.cpp, built by oracle/build_ref.py; the CPU
# tests re-derive these numbers when that counter is built).
REF_KNOT_FLOPS = {"kkt_dynamics": 45716, "kkt_cost": 13165, "merit_cost": 1006,
                  "merit_defect": 12882}


def schur_flops(nx=14, nu=7):
    """Schur complement, preconditioner and gamma of one problem
    (schur_linsys.cuh:54-260 restated): per knot two n x n and one m x m
    Gauss-Jordan inverses (2k^2(k+1) flops each), the theta / phi products
    and the preconditioner's off-diagonal product."""
    gj = lambda n: 2 * n * n * (n + 1)
    return (N - 1) * (2 * gj(nx) + gj(nu) + 2 * (nx ** 3) * 2 + 2 * nx * nu * nu
                      + 2 * nx * nx * nu + 4 * nx * nx + 4 * nx ** 3)


def dz_flops(nx=14, nu=7):
    """Step recovery of one problem (schur_linsys.cuh:312-431)."""
    return N * (2 * nx * nx * 2 + 2 * nx * nu * 2 + 2 * nu * nu)


def pcg_iter_flops(nx=14):
    """One PCG iteration of one problem: two block-tridiagonal matvecs
    (N block rows of n x 3n multiply-adds each) plus the dot products and
    vector updates (about 10 flops per padded entry)."""
    return 2 * (2 * N * nx * 3 * nx) + 10 * (N + 2) * nx


def kernel_flops(B, pcg_iters, launches):
    """Algorithmic FLOPs of each fused-form kernel over one solve:
    fused_iter  KKT blocks of every knot (dynamics, derivatives, cost) and
                the Schur system, per SQP iteration
    pcg         the PCG iterations actually run, plus step recovery
    line_search 8 step sizes x N knots of cost + integrator defect
    merit       the initial and final merits (one step size)"""
    F = REF_KNOT_FLOPS
    knot_kkt = F["kkt_dynamics"] + F["kkt_cost"]
    knot_merit = F["merit_cost"] + F["merit_defect"]
    return {
        "fused_iter": launches["fused_iter"] * B * (N * knot_kkt + schur_flops()),
        "pcg": float(np.sum(pcg_iters)) * pcg_iter_flops() + launches["pcg"] * B * dz_flops(),
        "line_search": launches["line_search"] * B * 8 * N * knot_merit,
        "merit": launches["merit"] * B * N * knot_merit,
    }


class ClockSampler:
    """Samples nvidia-smi SM clocks and throttle reasons during the timed
    region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax = float(parts[2])
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


HBM_FALLBACK_GBS = 6650.0  # B200 copy bandwidth measured earlier, used when no measured-peaks file is present


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


def fp32_peak_tflops(torch, dev):
    """Measured FP32 CUDA-core throughput: cuBLAS SGEMM 8192^3 with TF32
    disabled, best of 5 (the same kind of measurement as the driver's bf16
    GEMM peak)."""
    torch.backends.cuda.matmul.allow_tf32 = False
    torch.backends.cudnn.allow_tf32 = False
    n = 8192
    a = torch.randn(n, n, device=dev, dtype=torch.float32)
    b = torch.randn(n, n, device=dev, dtype=torch.float32)
    c = torch.empty(n, n, device=dev, dtype=torch.float32)
    for _ in range(2):
        torch.matmul(a, b, out=c)
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b, out=c)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b, c
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


# --------------------------------------------------------------------------
def cpu_baseline(wl, sample, threads, with_result=False):
    """The FP64 oracle of the same SQP on `sample` problems of the workload,
    `threads` host threads; returns (solves/s, seconds) and, with_result,
    the oracle's trajectories and statistics (the checker of the GPU
    solution of the same problems)."""
    from oracle import oracle as O
    kw = solver_kwargs()
    P = O.make_params(dt=DT, **kw)
    S = O.Solver(PLANT, N, sample, P, threads=threads)
    S.set_lambda(wl["lam"][:sample].astype(np.float64))
    t0 = time.perf_counter()
    xo, so = S.solve(wl["xu"][:sample].astype(np.float64), DT,
                     wl["xs"][:sample].astype(np.float64), wl["goal"][:sample].astype(np.float64))
    dt = time.perf_counter() - t0
    if with_result:
        so = dict(so, lam=S.get_lambda())
        return sample / dt, dt, xo, so
    return sample / dt, dt


def kkt_measures(xu, lam, xs, goal):
    """Per problem, at trajectory xu with multipliers lam (padded [(N+2) nx]),
    from the FP64 oracle's KKT blocks: the dynamics defect max|c| (c_0 =
    x_0 - x_s, c_{k+1} the integrator defect) and the KKT stationarity
    max|grad L|, the residuals of the reference's step recovery
    (schur_linsys.cuh:312-431): q_k - lam_k + A_k^T lam_{k+1} and
    r_k + B_k^T lam_{k+1}."""
    from oracle import oracle as O
    P = O.make_params(dt=DT, **solver_kwargs())
    model = O.Model(PLANT)
    n = 2 * model.nq
    defect, stat = [], []
    for b in range(xu.shape[0]):
        kb = model.setup_kkt(N, P, DT, xu[b], xs[b], goal[b])
        lk = lam[b].reshape(N + 2, n)[1:N + 1]
        res = [kb["q"][k] - lk[k] + (kb["A"][k] @ lk[k + 1] if k < N - 1 else 0.0)
               for k in range(N)]
        res += [kb["r"][k] + kb["B"][k] @ lk[k + 1] for k in range(N - 1)]
        defect.append(float(np.abs(kb["c"]).max()))
        stat.append(float(max(np.abs(v).max() for v in res)))
    return np.array(defect), np.array(stat)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    sample = args.cpu_sample or max(threads, min(args.batch, 8 * threads))
    wl = make_reference_workload(args.batch, replica_seed(0), threads)
    for _ in range(args.warmup):
        cpu_baseline(wl, min(sample, threads), threads)
    times = []
    for _ in range(args.steps):
        v, dt = cpu_baseline(wl, sample, threads)
        times.append(dt)
    value = args.steps * sample / float(np.sum(times))
    ref_gpu = reference_gpu_leg(args, wl)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * float(np.mean(times)), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "global_batch": args.batch, "seq_len": N,
                   "parallelism": f"{threads} host threads",
                   "warm_start": "FP64 oracle, 30 SQP iterations, then the seeded perturbation "
                                 "(the same XU and lambda as the other arm to FP32 rounding)"},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": "port",
                         "sample": f"{sample} problems of the workload per step (FP64 oracle "
                                   f"port of the reference SQP; the reference's solver has "
                                   f"no CPU implementation)"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "reference_gpu": ref_gpu,
    }
    print(json.dumps(line))
    return 0


_REF_MODULE = {}


def reference_gpu_leg(args, wl):
    """The reference's own CUDA solver (python/bindings.cu compiled unmodified
    for sm_100a into oracle/_ref by oracle/build_ref_gpu.py) on the same
    workload `wl` (make_reference_workload), through its own solve(): host
    arrays in, host arrays out, as its Python interface calls it.  Reported
    beside the CPU arm; absent module or GPU gives an "unavailable" entry.
    Its lambda lives inside the module with no setter: it starts at zero and
    carries from call to call, the one input that differs from the other
    arm."""
    import glob
    import importlib.util
    paths = glob.glob(os.path.join(ROOT, "oracle", "_ref", f"bsqpN{N}_{PLANT}*.so"))
    if not paths:
        return {"unavailable": "reference CUDA module not built (oracle/build_ref_gpu.py)"}
    try:
        import torch
        if not torch.cuda.is_available():
            return {"unavailable": "no GPU"}
        torch.cuda.init()
    except ImportError:
        return {"unavailable": "torch missing"}
    name = f"bsqpN{N}_{PLANT}"
    if name not in _REF_MODULE:  # a pybind11 module loads once per process
        spec = importlib.util.spec_from_file_location(name, paths[0])
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        _REF_MODULE[name] = mod
    mod = _REF_MODULE[name]
    B = wl["xu"].shape[0]
    cls = getattr(mod, f"BSQP_{B}_float", None)
    if cls is None:
        return {"unavailable": f"the reference module has no batch-{B} class"}
    kw = solver_kwargs()
    solver = cls(DT, kw["max_sqp_iters"], kw["kkt_tol"], kw["max_pcg_iters"], kw["pcg_tol"],
                 kw["solve_ratio"], kw["mu"], kw["q_cost"], kw["qd_cost"], kw["u_cost"],
                 kw["N_cost"], kw["q_lim_cost"], kw["vel_lim_cost"], kw["ctrl_lim_cost"],
                 kw["rho"])
    f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)
    xs, goal = f32(wl["xs"]), f32(wl["goal"])
    wall, own = [], []
    for i in range(args.warmup + args.steps):
        solver.reset_rho()
        xin = f32(wl["xu"]).copy()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = solver.solve(xin, DT, xs, goal)
        t1 = time.perf_counter()
        if i >= args.warmup:
            wall.append(t1 - t0)
            own.append(float(out["sqp_time_us"]) * 1e-6)
    pcg = np.array(out["pcg_iters"])
    return {"value": B / float(np.mean(wall)), "unit": "solves/s",
            "own_timer_value": B / float(np.mean(own)),
            "ms_per_step": 1e3 * float(np.mean(wall)),
            "p50_ms": 1e3 * float(np.median(wall)), "p99_ms": 1e3 * float(np.percentile(wall, 99)),
            "kind": "reference CUDA build, FP32 -use_fast_math, sm_100a",
            "note": "solve() with host arrays (its own H2D/D2H inside); the same XU warm "
                    "start as the other arm; lambda internal to the module (zero at the "
                    "first call, then carried between calls); rho reset before each call",
            "pcg_iters_mean": float(pcg.mean()) if pcg.size else None}


def make_reference_workload(batch, seed, threads):
    """The reference arm's copy of the workload: the oracle's robot tables and
    forward kinematics, warm start from the FP64 oracle.  Nothing of this
    library is imported on this arm."""
    from oracle import oracle as O
    model = O.builtin_model(PLANT)
    m = O.Model(PLANT)
    fk = lambda q: np.stack([m.ee_pos(qq) for qq in np.asarray(q, np.float64)])
    xs, goal, xu, rng = seeded_problems(model.nq, model.q_limit, fk, batch, seed)
    S = O.Solver(PLANT, N, batch, O.make_params(dt=DT, **dict(solver_kwargs(), **WARM_KW)),
                 threads=threads)
    xc, _ = S.solve(xu.astype(np.float64), DT, xs.astype(np.float64), goal.astype(np.float64))
    return dict(perturbed_warm_start(xc, S.get_lambda(), xs, model.nq, rng), goal=goal)


# --------------------------------------------------------------------------
def replica_seed(rank):
    """Seed of the problems a rank solves: every GPU runs an independent
    replica batch (problems do not interact, so the batch shards with no
    data-path collective)."""
    return 2026 + rank


def max_over_ranks(x, dist=None, device=None):
    """The slowest rank's value of a per-rank time (all ranks take part)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_solves_per_s(world, batch, ms_per_step):
    """Whole-job throughput: every rank's batch over the slowest rank's time."""
    return world * batch / (ms_per_step * 1e-3)


def time_device_steps(torch, solver, bufs, wl, steps, warmup, flush, stream):
    """Per-step CUDA-event times of solver.solve_device (fused graph or plain
    driver) with warm-start state restored and L2 flushed between steps."""
    import gato_b200._lib as L
    d_xu, d_xs, d_goal, d_xu0 = bufs
    times = []
    for i in range(warmup + steps):
        d_xu.copy_(d_xu0)
        solver.set_lambda(wl["lam"])
        solver.reset_rho()
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            fn = L.load().gato_solve_f64 if solver.precision == "fp64" else L.load().gato_solve
            L.check(fn(solver._h, stream.cuda_stream, L.vptr(d_xu), L.vptr(d_xs),
                       L.vptr(d_goal), None))
            e1.record(stream)
        torch.cuda.synchronize()
        if i >= warmup:
            times.append(e0.elapsed_time(e1))
    return np.array(times)


PRECISIONS = ("fp32", "mixed", "fp64", "fp64-p32")


def new_solver(prec, B, **kw):
    """A fused- or plain-form solver of the workload's plant and horizon in
    precision `prec`: "fp32", "mixed", "fp64", or "fp64-p32" (FP64 with the
    preconditioner applied in FP32, gato_set_fp32_preconditioner)."""
    import gato_b200
    s = gato_b200.BSQP(batch_size=B, N=N, dt=DT, plant_type=PLANT,
                       precision="fp64" if prec.startswith("fp64") else prec, **kw)
    if prec == "fp64-p32":
        s.set_fp32_preconditioner(True)
    return s


def profile_kernels(solver, wl, bufs, stream):
    """Device time per kernel group of one solve from the warm start
    (gato_profile_solve: CUDA events around every launch, the fused form
    without its graph): {group: {"ms", "launches"}}."""
    import ctypes
    import gato_b200._lib as L
    d_xu, d_xs, d_goal, d_xu0 = bufs
    d_xu.copy_(d_xu0)
    solver.set_lambda(wl["lam"])
    solver.reset_rho()
    msk = (ctypes.c_double * len(L.KERNELS))()
    nk = (ctypes.c_int32 * len(L.KERNELS))()
    fn = L.load().gato_profile_solve_f64 if solver.precision == "fp64" else \
        L.load().gato_profile_solve
    L.check(fn(solver._h, ctypes.c_void_p(stream.cuda_stream), L.vptr(d_xu), L.vptr(d_xs),
               L.vptr(d_goal), msk, nk))
    return {L.KERNELS[i]: {"ms": msk[i], "launches": nk[i]} for i in range(len(L.KERNELS))}


def precision_times(torch, dev, B, prec, wl, args, flush, stream):
    """Mean ms per solve of the fused and the plain form in precision
    `prec` on the workload (inputs resident, timed like the headline), and
    each form's device time per kernel group ({"fused": ..., "plain": ...})."""
    import gato_b200
    dt = torch.float64 if prec.startswith("fp64") else torch.float32
    T = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=dt, device=dev)
    d_xu0, d_xs, d_goal = T(wl["xu"]), T(wl["xs"]), T(wl["goal"])
    bufs = (d_xu0.clone(), d_xs, d_goal, d_xu0)
    out = []
    kern = {}
    for form in ("fused", "plain"):
        s = new_solver(prec, B, form=form, **solver_kwargs())
        steps = args.steps if form == "fused" else max(3, args.steps // 2)
        out.append(float(np.mean(time_device_steps(torch, s, bufs, wl, steps, max(1, args.warmup),
                                                   flush, stream))))
        kern[form] = profile_kernels(s, wl, bufs, stream)
        if form == "fused":
            kern["e2e_s"] = host_api_times(torch, s, wl, steps, max(1, args.warmup), flush)
        s.close()
    return out[0], out[1], kern


def host_api_times(torch, solver, wl, steps, warmup, flush):
    """Seconds per solve through the host API (gato_solve_host, or its _f64
    form), pinned host buffers, H2D of XU, x0, goals and D2H of XU inside
    the timed region; warm start restored and L2 flushed between solves."""
    import gato_b200._lib as L
    f64 = solver.precision == "fp64"
    dt = torch.float64 if f64 else torch.float32
    h_xu = torch.empty(tuple(wl["xu"].shape), dtype=dt).pin_memory()
    h_xs = torch.tensor(wl["xs"], dtype=dt).pin_memory()
    h_goal = torch.tensor(wl["goal"], dtype=dt).pin_memory()
    fn = L.load().gato_solve_host_f64 if f64 else L.load().gato_solve_host
    ptr = L.dptr if f64 else L.fptr
    out = []
    for i in range(warmup + steps):
        h_xu.copy_(torch.from_numpy(wl["xu"]))
        solver.set_lambda(wl["lam"])
        solver.reset_rho()
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        L.check(fn(solver._h, ptr(h_xu), DT, ptr(h_xs), ptr(h_goal), None))
        if i >= warmup:
            out.append(time.perf_counter() - t0)
    return float(np.mean(out))


def trajectory_errors(xg, xo):
    """Per problem max |XU - XU_oracle| / max(1, max |XU_oracle|)."""
    return np.abs(xg - xo).max(axis=1) / np.maximum(1.0, np.abs(xo).max(axis=1))


def compare_with_oracle(xg, pcg_g, step_g, xo, pcg_o, step_o):
    """Trajectory error statistics, PCG-count agreement and the problems
    whose line-search decision differs from the oracle's, each with the
    first SQP iteration at which it differs."""
    e = trajectory_errors(xg, xo)
    rows = min(step_g.shape[0], step_o.shape[0])
    diff = step_g[:rows] != np.asarray(step_o[:rows], np.float32)
    div = np.nonzero(diff.any(axis=0))[0]
    agree = np.ones(e.shape[0], bool)
    agree[div] = False
    out = {"xu_rel_err_median": float(np.median(e)), "xu_rel_err_p90": float(np.percentile(e, 90)),
           "xu_rel_err_max": float(e.max()), "frac_within_1e-4": float(np.mean(e <= 1e-4)),
           "pcg_iters_equal_frac": float(np.mean(pcg_g[:rows] == pcg_o[:rows])),
           "ls_diverged_problems": int(div.size),
           "ls_first_divergent_iteration": {int(b): int(diff[:, b].argmax()) for b in div},
           "xu_rel_err_median_where_ls_agrees": float(np.median(e[agree])) if agree.any()
           else None}
    return out


def accuracy_block(wl, sample, threads, xo, so):
    """Each precision's fused solve of the first `sample` problems against
    the FP64 oracle of the same SQP from the same XU, lambda and rho:
      per precision   trajectory error, PCG counts, line-search divergences
      fp32_storage_floor  the oracle itself with every stored stage output
                      (KKT blocks, Schur system, lambda, XU) rounded to FP32
                      and all arithmetic in FP64: the error an ideal FP32
                      solver would show
      converged       30 SQP iterations at PCG tol 1e-6 (sample of 256):
                      trajectory error and the dynamics defect / KKT
                      stationarity (FP64 KKT blocks) of each result beside
                      the oracle's"""
    import gato_b200
    from oracle import oracle as O
    out = {"sample": sample}
    xs, goal = wl["xs"][:sample], wl["goal"][:sample]

    def gpu(prec, kwx=None, n=sample):
        s = new_solver(prec, n, form="fused", **dict(solver_kwargs(), **(kwx or {})))
        f = np.float64 if prec.startswith("fp64") else np.float32
        s.set_lambda(wl["lam"][:n].astype(f))
        s.reset_rho()
        g = s.solve_raw(wl["xu"][:n].astype(f), DT, xs[:n].astype(f), goal[:n].astype(f))
        lam = s.get_lambda().astype(np.float64)
        s.close()
        return g, lam

    for prec in PRECISIONS:
        g, _ = gpu(prec)
        out[prec] = compare_with_oracle(np.asarray(g["XU"], np.float64), g["pcg_iters"],
                                        g["ls_step_size"], xo, so["pcg_iters"], so["ls_step_size"])
    S = O.Solver(PLANT, N, sample, O.make_params(dt=DT, **solver_kwargs()), threads=threads)
    S.set_round_f32(S.ROUND_ALL)
    S.set_lambda(wl["lam"][:sample].astype(np.float64))
    xf, sf = S.solve(wl["xu"][:sample].astype(np.float64), DT, xs.astype(np.float64),
                     goal.astype(np.float64))
    out["fp32_storage_floor"] = compare_with_oracle(xf, sf["pcg_iters"], sf["ls_step_size"], xo,
                                                    so["pcg_iters"], so["ls_step_size"])
    # converged workload
    kc = min(sample, 256)
    S = O.Solver(PLANT, N, kc, O.make_params(dt=DT, **dict(solver_kwargs(), **WARM_KW)),
                 threads=threads)
    S.set_lambda(wl["lam"][:kc].astype(np.float64))
    xc, sc = S.solve(wl["xu"][:kc].astype(np.float64), DT, xs[:kc].astype(np.float64),
                     goal[:kc].astype(np.float64))
    ks = min(kc, 64)
    xs64, goal64 = xs[:ks].astype(np.float64), goal[:ks].astype(np.float64)
    do, so_ = kkt_measures(xc[:ks], S.get_lambda()[:ks], xs64, goal64)
    conv = {"problems": kc, "sqp_iters": WARM_KW["max_sqp_iters"], "pcg_tol": WARM_KW["pcg_tol"],
            "oracle": {"defect_median": float(np.median(do)), "stationarity_median":
                       float(np.median(so_)), "stationarity_max": float(so_.max())}}
    for prec in PRECISIONS:
        g, lam = gpu(prec, WARM_KW, kc)
        xg = np.asarray(g["XU"], np.float64)
        dg, sg = kkt_measures(xg[:ks], lam[:ks], xs64, goal64)
        e = trajectory_errors(xg, xc)
        conv[prec] = {"xu_rel_err_median": float(np.median(e)), "xu_rel_err_max": float(e.max()),
                      "defect_median": float(np.median(dg)),
                      "stationarity_median": float(np.median(sg)),
                      "stationarity_abs_diff_max": float(np.abs(sg - so_).max()),
                      "defect_abs_diff_max": float(np.abs(dg - do).max())}
    out["converged"] = conv
    out["note"] = ("fused solves vs the FP64 oracle of the same SQP, same inputs; defect and "
                   "stationarity evaluated with FP64 KKT blocks at each solver's own result")
    return out


# --------------------------------------------------------------------------
# Differentiable solve (iiwa14 N=32, batch 256): loss |XU* - XU_target|^2
# with XU_target = warm start + N(0, 0.1^2), gradients with respect to x0,
# the goal trajectory and the Q/R diagonals, log-parameterised with
# log w ~ U[-2, 2]; checked against the dense FP64 KKT gradient
# (oracle/adjoint_ref.py) on every problem and FP64 central differences
# (h = 1e-6) of the same QP map through the device's own QP step on 16.
ADJ_B, ADJ_FD, ADJ_H = 256, 16, 1e-6
ADJ_TOL = {"fp32": 1e-8, "mixed": 1e-8, "fp64": 1e-20}


def _rel_err(a, b):
    return float(np.abs(np.asarray(a) - b).max() / max(1e-12, np.abs(b).max()))


def adjoint_config4(torch, dev, threads, precisions=("fp32", "mixed", "fp64"), B=ADJ_B,
                    fd_problems=ADJ_FD):
    """Per precision: device times of the forward solve and the adjoint, and
    each gradient's relative error (max |g - g_dense| / max |g_dense| per
    problem; median and max over problems) against the dense FP64 gradient
    at that precision's own solution; for FP64, central differences through
    gato_qp_step_f64 against the dense gradient as well."""
    import gato_b200
    import gato_b200._lib as L
    from oracle import adjoint_ref as AR
    from oracle import oracle as O
    wl = make_workload(B, seed=2032)
    rng = np.random.default_rng(2033)
    nq, nx, nu = 7, 14, 7
    logw = rng.uniform(-2.0, 2.0, (B, nx + nu))
    target = wl["xu"].astype(np.float64) + rng.normal(0.0, 0.1, wl["xu"].shape)
    m = O.Model(PLANT)
    P = O.make_params(dt=DT, **solver_kwargs())
    out = {"batch": B, "loss": "|XU* - XU_target|^2, XU_target = warm start + N(0, 0.1^2)",
           "weights": "Q/R diagonals exp(u), u ~ U[-2, 2]", "what": "relative error "
           "max|g - g_ref| / max|g_ref| per problem, median and max over problems"}
    for prec in precisions:
        dt_ = torch.float64 if prec == "fp64" else torch.float32
        f = np.float64 if prec == "fp64" else np.float32
        T = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=dt_, device=dev)
        s = gato_b200.BSQP(batch_size=B, N=N, dt=DT, plant_type=PLANT, precision=prec,
                           **solver_kwargs())
        w = np.exp(logw)
        s.set_cost_diag_batch(w[:, :nx], w[:, nx:])
        w_held = s._wdiag.astype(np.float64)
        d_xs, d_goal, d_xu0 = T(wl["xs"]), T(wl["goal"]), T(wl["xu"])
        times = {"forward": [], "adjoint": []}
        for i in range(4):
            d_xu = d_xu0.clone()
            s.set_lambda(wl["lam"].astype(f))
            s.reset_rho()
            torch.cuda.synchronize()
            e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            cs = torch.cuda.current_stream().cuda_stream
            e[0].record()
            s.solve_device(d_xu, d_xs, d_goal, with_stats=False, stream=cs)
            e[1].record()
            dl = (2.0 * (d_xu.double() - T(target).double())).to(dt_).contiguous()
            e[2].record()
            res = s.adjoint_device(d_xu, d_xs, d_goal, dl, tol=ADJ_TOL[prec],
                                   with_iters=(i == 0), stream=cs)
            e[3].record()
            if i == 0:
                its = res[3]
            g_xs, g_goal, g_w = res[:3]
            torch.cuda.synchronize()
            if i:
                times["forward"].append(e[0].elapsed_time(e[1]))
                times["adjoint"].append(e[2].elapsed_time(e[3]))
        xu = d_xu.double().cpu().numpy()
        rho = s.get_rho().astype(np.float64)
        lam = s.get_lambda().astype(np.float64)
        dln = dl.double().cpu().numpy()
        g = [t.double().cpu().numpy() for t in (g_xs, g_goal, g_w)]
        errs = {"x0": [], "goal": [], "log_qr": []}
        dense = []
        for b in range(B):
            r = AR.adjoint_grad(m, N, P, DT, xu[b], wl["xs"][b].astype(np.float64),
                                wl["goal"][b].astype(np.float64), w_held[b], float(rho[b]), dln[b])
            dense.append(r)
            gi = np.zeros(6 * N, bool)
            gi[np.arange(6 * N) % 6 < 3] = True
            errs["x0"].append(_rel_err(g[0][b], r["g_xs"]))
            errs["goal"].append(_rel_err(g[1][b][gi], r["g_goal"][gi]))
            errs["log_qr"].append(_rel_err(g[2][b] * w_held[b], r["g_wdiag"] * w_held[b]))
        res = {"forward_ms": float(np.mean(times["forward"])),
               "adjoint_ms": float(np.mean(times["adjoint"])),
               "adjoint_pcg_tol": ADJ_TOL[prec],
               "pcg_iters_mean": {"forward_qp_step": float(its[0].mean()),
                                  "adjoint": float(its[1].mean())},
               "pcg_iters_max": {"forward_qp_step": int(its[0].max()),
                                 "adjoint": int(its[1].max())},
               "vs_dense_fp64": {k: {"median": float(np.median(v)), "max": float(np.max(v))}
                                 for k, v in errs.items()}}
        res["backward_vs_forward"] = res["adjoint_ms"] / res["forward_ms"]
        if prec == "fp64" and fd_problems:
            # h = 1e-6 as specified; its error is rounding noise of the QP
            # solve divided by h (cond(KKT) ~ 1e5-1e6 here), so h = 1e-4, whose
            # truncation error is below that noise, is reported beside it
            res["fd_device_vs_dense"] = _device_fd(torch, dev, xu, wl, w_held, rho, lam, dln,
                                                   dense, fd_problems, ADJ_H)
            res["fd_device_vs_dense_h1e-4"] = _device_fd(torch, dev, xu, wl, w_held, rho, lam,
                                                         dln, dense, fd_problems, 1e-4)
        s.close()
        out[prec] = res
    return out


def _device_fd(torch, dev, xu, wl, w_held, rho, lam, dl, dense, K, h):
    """Central differences (step h, on x0, the goal positions and the log
    weights) of l(theta) = dl . (xu + dz(theta)), dz the QP step at the fixed
    xu computed by the device in FP64 (gato_qp_step_f64, 1500 PCG iterations
    for every evaluation, no tolerance stop), for the first K problems: all
    perturbed problems form one batch."""
    import gato_b200
    import gato_b200._lib as L
    nx, nu = 14, 7
    gi = [6 * j + a for j in range(N) for a in range(3)]
    params = [("x0", i) for i in range(nx)] + [("goal", i) for i in gi] + \
             [("w", i) for i in range(nx + nu)]
    rows = []
    for b in range(K):
        for kind, i in params:
            for sgn in (1.0, -1.0):
                rows.append((b, kind, i, sgn))
    M = len(rows)
    xs = np.zeros((M, nx))
    goal = np.zeros((M, 6 * N))
    wd = np.zeros((M, nx + nu))
    xum = np.zeros((M, xu.shape[1]))
    for r, (b, kind, i, sgn) in enumerate(rows):
        xs[r], goal[r], wd[r], xum[r] = wl["xs"][b], wl["goal"][b], w_held[b], xu[b]
        if kind == "x0":
            xs[r, i] += sgn * h
        elif kind == "goal":
            goal[r, i] += sgn * h
        else:
            wd[r, i] *= np.exp(sgn * h)
    f = gato_b200.BSQP(batch_size=M, N=N, dt=DT, plant_type=PLANT, precision="fp64",
                       **solver_kwargs())
    f.set_cost_diag_batch(wd[:, :nx], wd[:, nx:])
    f.set_rho_penalty_batch(np.array([rho[b] for b, *_ in rows]), True)
    f.set_lambda(np.stack([lam[b] for b, *_ in rows]))
    T = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    d_xu, d_xs, d_goal = T(xum), T(xs), T(goal)
    d_dz = torch.empty_like(d_xu)
    L.check(L.load().gato_qp_step_f64(f._h, None, L.vptr(d_xu), L.vptr(d_xs), L.vptr(d_goal),
                                      L.vptr(d_dz), 0.0, 1500, None))
    torch.cuda.synchronize()
    f.close()
    dz = d_dz.cpu().numpy()
    loss = np.array([dl[b] @ (xu[b] + dz[r]) for r, (b, *_) in enumerate(rows)])
    errs = {"x0": [], "goal": [], "log_qr": []}
    r = 0
    for b in range(K):
        fd = {"x0": [], "goal": [], "w": []}
        for kind, i in params:
            fd[kind].append((loss[r] - loss[r + 1]) / (2 * h))
            r += 2
        d = dense[b]
        errs["x0"].append(_rel_err(fd["x0"], d["g_xs"]))
        errs["goal"].append(_rel_err(fd["goal"], d["g_goal"][gi]))
        errs["log_qr"].append(_rel_err(fd["w"], d["g_wdiag"] * w_held[b]))
    return {"problems": K, "h": h, "pcg_iters": 1500,
            "rel_err": {k: {"median": float(np.median(v)), "max": float(np.max(v))}
                        for k, v in errs.items()}}


def run_ours(args):
    if args.precision == "fp64":
        raise SystemExit("--precision fp64 applies to --workload profile only (the headline "
                         "line reports FP64 under by_precision)")
    import torch
    import gato_b200
    import gato_b200._lib as L

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=dev)
    B = args.batch
    wl = make_workload(B, seed=replica_seed(rank))
    kw = solver_kwargs()
    fused = gato_b200.BSQP(batch_size=B, N=N, dt=DT, plant_type=PLANT, form="fused",
                           precision=args.precision, **kw)
    plain = gato_b200.BSQP(batch_size=B, N=N, dt=DT, plant_type=PLANT, form="plain",
                           precision=args.precision, **kw)
    T = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device=dev)
    d_xu0, d_xs, d_goal = T(wl["xu"]), T(wl["xs"]), T(wl["goal"])
    d_xu = d_xu0.clone()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.Stream(device=dev)
    bufs = (d_xu, d_xs, d_goal, d_xu0)

    # untimed: statistics of one solve (iteration counts for the FLOP count)
    d_xu.copy_(d_xu0)
    fused.set_lambda(wl["lam"])
    fused.reset_rho()
    st = fused.solve_device(d_xu, d_xs, d_goal, stream=stream.cuda_stream)
    pcg_total = int(np.sum(st["pcg_iters"]))
    # per-kernel device times of the same solve (events around each launch)
    kern = profile_kernels(fused, wl, bufs, stream)
    total_prof = sum(v["ms"] for v in kern.values())

    peaks = measured_peaks()
    fp32_peak = fp32_peak_tflops(torch, dev)

    # timed: fused form (headline), clocks sampled during it
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    t_fused = time_device_steps(torch, fused, bufs, wl, args.steps, args.warmup, flush, stream)
    clk = clocks.stop()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    # plain form on the same workload
    t_plain = time_device_steps(torch, plain, bufs, wl, max(3, args.steps // 2), 1, flush, stream)

    # e2e through the host API (pinned host buffers)
    h_xu = torch.empty((B, wl["xu"].shape[1]), dtype=torch.float32).pin_memory()
    h_xs = torch.tensor(wl["xs"]).pin_memory()
    h_goal = torch.tensor(wl["goal"]).pin_memory()
    e2e_times = []
    for i in range(args.warmup + args.steps):
        h_xu.copy_(torch.from_numpy(wl["xu"]))
        fused.set_lambda(wl["lam"])
        fused.reset_rho()
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        L.check(L.load().gato_solve_host(fused._h, L.fptr(h_xu), DT, L.fptr(h_xs),
                                         L.fptr(h_goal), None))
        t1 = time.perf_counter()
        if i >= args.warmup:
            e2e_times.append(t1 - t0)
    e2e_times = np.array(e2e_times)

    # adjoint (gato_adjoint) of the fused solve's returned trajectory, timed
    # like the forward step: CUDA events on the stream, L2 flushed between
    # calls; the loss gradient is a seeded dense vector
    d_xu.copy_(d_xu0)
    fused.set_lambda(wl["lam"])
    fused.reset_rho()
    fused.solve_device(d_xu, d_xs, d_goal, stream=stream.cuda_stream, with_stats=False)
    d_dl = torch.tensor(np.random.default_rng(7).normal(0, 1, tuple(d_xu.shape)),
                        dtype=torch.float32, device=dev)
    adj_ms, adj_its = [], None
    with torch.cuda.stream(stream):
        for i in range(args.warmup + max(3, args.steps // 5)):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            out = fused.adjoint_device(d_xu, d_xs, d_goal, d_dl, stream=stream.cuda_stream,
                                       with_iters=(i == 0))
            e1.record(stream)
            torch.cuda.synchronize()
            if i == 0:
                adj_its = out[3]
            if i >= args.warmup:
                adj_ms.append(e0.elapsed_time(e1))
    ms_adj = max_over_ranks(float(np.mean(adj_ms)), dist, dev)

    ms_fused = max_over_ranks(float(np.mean(t_fused)), dist, dev)
    ms_plain = max_over_ranks(float(np.mean(t_plain)), dist, dev)
    s_e2e = max_over_ranks(float(np.mean(e2e_times)), dist, dev)
    p50 = max_over_ranks(float(np.median(t_fused)), dist, dev)
    p99 = max_over_ranks(float(np.percentile(t_fused, 99)), dist, dev)

    # the other precisions' throughput on the same workload (fused and plain)
    by_prec = {args.precision: {"value": B / (float(np.mean(t_fused)) * 1e-3),
                                "plain_value": B / (float(np.mean(t_plain)) * 1e-3),
                                "fused_vs_plain": float(np.mean(t_plain) / np.mean(t_fused)),
                                "e2e_value": B / float(np.mean(e2e_times))}}
    kern_by_prec = {args.precision: {k: round(v["ms"], 4) for k, v in kern.items()
                                     if v["launches"]}}
    plain_kern_by_prec = {args.precision: None}
    for prec in PRECISIONS:
        if prec in by_prec:
            continue
        tf, tp, kp = precision_times(torch, dev, B, prec, wl, args, flush, stream)
        by_prec[prec] = {"value": B / (tf * 1e-3), "plain_value": B / (tp * 1e-3),
                         "fused_vs_plain": tp / tf, "e2e_value": B / kp.pop("e2e_s")}
        kern_by_prec[prec] = {k: round(v["ms"], 4) for k, v in kp["fused"].items()
                              if v["launches"]}
        plain_kern_by_prec[prec] = {k: round(v["ms"], 4) for k, v in kp["plain"].items()
                                    if v["launches"]}
    by_prec = {k: {kk: max_over_ranks(vv, dist, dev) for kk, vv in v.items()}
               for k, v in by_prec.items()}
    for k in by_prec:
        by_prec[k]["kernels_ms"] = kern_by_prec[k]
        if plain_kern_by_prec.get(k):
            by_prec[k]["plain_kernels_ms"] = plain_kern_by_prec[k]

    # CPU baseline (rank 0, N=1 only)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        sample = args.cpu_sample or int(min(B, max(threads, 64 * threads)))
        v, secs, xo, so = cpu_baseline(wl, sample, threads, with_result=True)
        cpu = {"value": v, "unit": "solves/s", "cores": threads, "kind": "port",
               "sample": f"{sample} problems of the workload, one solve, {secs:.1f} s wall "
                         f"(FP64 oracle port of the reference SQP)"}
        accuracy = accuracy_block(wl, sample, threads, xo, so)
        adj4 = adjoint_config4(torch, dev, threads)
    if dist:
        dist.destroy_process_group()
    if rank != 0:
        return 0

    traj = wl["xu"].shape[1]
    solves = world * B
    launches = {k: v["launches"] for k, v in kern.items()}
    flops = kernel_flops(B, st["pcg_iters"], launches)
    roof = {}
    for k, f in flops.items():
        if kern[k]["launches"]:
            ms = kern[k]["ms"] / kern[k]["launches"]
            tf = f / kern[k]["launches"] / (ms * 1e-3) / 1e12
            roof[k] = {"ms_per_launch": ms, "tflops": tf, "frac": tf / fp32_peak}
    top = max(roof, key=lambda k: kern[k]["ms"])
    line = {
        "metric": METRIC,
        "value": aggregate_solves_per_s(world, B, ms_fused),
        "unit": "solves/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_fused,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32" if args.precision == "fp32" else "f32+f64-reductions",
        "data": "synthetic (seeded figure-8 goals, perturbed converged warm start)",
        "config": {"workload": WORKLOAD + ", form=fused (CUDA graph)",
                   "global_batch": solves, "seq_len": N, "parallelism": f"replicas x{world}",
                   "l2": "flushed between steps (256 MB write)"},
        "p50_latency_ms": p50,
        "p99_latency_ms": p99,
        "sqp_iters_per_s": solves * SQP_ITERS / (ms_fused * 1e-3),
        "plain_form": {"value": solves / (ms_plain * 1e-3), "unit": "solves/s",
                       "ms_per_step": ms_plain},
        "fused_vs_plain": ms_plain / ms_fused,
        "by_precision": by_prec,
        "adjoint": {"ms_per_call": ms_adj, "vs_forward_solve": ms_adj / ms_fused,
                    "pcg_iters_mean": {"forward_qp_step": float(adj_its[0].mean()),
                                       "adjoint": float(adj_its[1].mean())},
                    "pcg_iters_max": {"forward_qp_step": int(adj_its[0].max()),
                                      "adjoint": int(adj_its[1].max())},
                    "what": "gradients for x0, goals, Q/R diagonals of a dense loss "
                            "gradient (FP32, relative PCG tol 1e-12)"},
        "e2e": {"value": solves / s_e2e, "unit": "solves/s",
                "h2d_bytes_per_step": int(4 * B * (traj + 14 + 6 * N)),
                "d2h_bytes_per_step": int(4 * B * traj)},
        "gpu_launches": int(sum(v["launches"] * KERNELS_PER_GROUP.get(k, 1)
                                for k, v in kern.items())) * args.steps,
        "kernels_ms": {k: round(v["ms"], 4) for k, v in kern.items() if v["launches"]},
        "pcg_iters_mean": float(np.mean(st["pcg_iters"])),
        "roofline": {"bound": "fp32", "achieved": roof[top]["tflops"], "peak": fp32_peak,
                     "unit": "TFLOP/s", "frac": roof[top]["frac"],
                     "traffic": TRAFFIC_PER_LAUNCH.get(top),
                     "kernel": KERNEL_NAMES[top],
                     "peak_source": "measured FP32 SGEMM on this GPU (TF32 off)",
                     "flops_source": "reference device functions run with a counting scalar",
                     "hbm_peak_gbs": peaks.get("hbm_gbs", HBM_FALLBACK_GBS),
                     "hbm_peak_source": "MEASURED_PEAKS.json" if "hbm_gbs" in peaks
                     else "fallback (earlier measurement on this pool)"},
        "roofline_by_kernel": {KERNEL_NAMES[k]: {kk: round(vv, 4) for kk, vv in v.items()}
                               for k, v in roof.items()},
        "clocks": clk,
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
        line["accuracy_vs_fp64_oracle"] = accuracy
        line["adjoint_config4"] = adj4
        # the fastest form whose trajectories meet the 1e-4 bound against the
        # oracle on this workload, every problem (the largest error)
        ok = [p for p in PRECISIONS if accuracy[p]["xu_rel_err_max"] <= 1e-4]
        if ok:
            best = max(ok, key=lambda p: by_prec[p]["value"])
            line["at_1e-4"] = {"precision": best, "form": "fused (CUDA graph)",
                               "value": by_prec[best]["value"], "unit": "solves/s",
                               "e2e_value": by_prec[best]["e2e_value"],
                               "plain_value": by_prec[best]["plain_value"],
                               "fused_vs_plain": by_prec[best]["fused_vs_plain"],
                               "xu_rel_err_median": accuracy[best]["xu_rel_err_median"],
                               "xu_rel_err_max": accuracy[best]["xu_rel_err_max"],
                               "pcg_iters_equal_frac": accuracy[best]["pcg_iters_equal_frac"],
                               "ls_diverged_problems": accuracy[best]["ls_diverged_problems"]}
    print(json.dumps(line))
    return 0


# --------------------------------------------------------------------------
# mixed workload: 4096 problems, plant 50/50 indy7 / iiwa14, horizon drawn
# from {8, 32, 64, 128}, figure-8 goals, default warm start, per-problem rho
# ~ logU[1e-2, 1e2], FP32 arithmetic with FP64 PCG inner products and merit
# sums, 5 SQP iterations, PCG max 173 at tol 1e-5
MIXED_TOTAL, MIXED_HORIZONS, MIXED_PLANTS = 4096, (8, 32, 64, 128), ("indy7", "iiwa14")


def mixed_classes(seed=2027):
    """(plant, N, count) of the seeded draw, longest first, and per-class
    seeds for the problem data."""
    rng = np.random.default_rng(seed)
    plants = rng.integers(0, 2, MIXED_TOTAL)
    hor = rng.integers(0, 4, MIXED_TOTAL)
    out = []
    for h in reversed(range(4)):
        for p in (1, 0):
            c = int(np.sum((plants == p) & (hor == h)))
            if c:
                out.append((MIXED_PLANTS[p], MIXED_HORIZONS[h], c))
    return out


def mixed_data(classes, seed=2027):
    from gato_b200 import workloads as W
    rng = np.random.default_rng(seed + 1)
    data = []
    for i, (plant, n, c) in enumerate(classes):
        pr = W.make_problem(plant, n, c, seed=seed + 10 + i, goals="figure8", dt=DT)
        pr["rho"] = np.exp(rng.uniform(np.log(1e-2), np.log(1e2), c)).astype(np.float32)
        data.append(pr)
    return data


def mixed_kwargs():
    kw = solver_kwargs()
    return kw


def run_mixed(args):
    import torch
    import gato_b200
    from gato_b200.mixed import MixedBSQP
    torch.cuda.set_device(0)
    dev = torch.device("cuda")
    classes = mixed_classes()
    data = mixed_data(classes)
    kw = mixed_kwargs()
    T = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device=dev)
    xs = [T(d["xs"]) for d in data]
    goal = [T(d["goal"]) for d in data]
    xu0 = [T(d["xu"]) for d in data]
    xu = [x.clone() for x in xu0]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.Stream(device=dev)
    mx = MixedBSQP(classes, dt=DT, precision="mixed", **kw)

    def reset(solvers, ds=None):
        for s, d in zip(solvers, ds or data):
            s.set_rho_penalty_batch(d["rho"], True)
            s.reset_dual()
            s.reset_rho()

    reset(mx.cls)
    with torch.cuda.stream(stream):
        shapes = mx.tune(xu, xs, goal, stream=stream.cuda_stream)
    torch.cuda.synchronize()
    times = []
    for i in range(args.warmup + args.steps):
        for a, b in zip(xu, xu0):
            a.copy_(b)
        reset(mx.cls)
        flush.zero_()
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            mx.solve_device(xu, xs, goal, stream=stream.cuda_stream)
        torch.cuda.synchronize()
        if i >= args.warmup:
            times.append(mx.elapsed_ms())
    stats = [mx.stats(c) for c in range(len(classes))]
    mx.close()
    # each class alone in its own fused solver (graph), one after another:
    # how a caller of per-(plant, N) solvers runs this workload
    alone = []
    for (plant, n, c), d, x0, xsc, gc in zip(classes, data, xu0, xs, goal):
        s = gato_b200.BSQP(batch_size=c, N=n, dt=DT, plant_type=plant, precision="mixed",
                           form="fused", **kw)
        x = x0.clone()
        ts = []
        for i in range(args.warmup + max(3, args.steps // 2)):
            x.copy_(x0)
            reset([s], [d])
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                e0.record(stream)
                s.solve_device(x, xsc, gc, stream=stream.cuda_stream, with_stats=False)
                e1.record(stream)
            torch.cuda.synchronize()
            if i >= args.warmup:
                ts.append(e0.elapsed_time(e1))
        s.close()
        alone.append((float(np.median(ts)), float(np.percentile(ts, 99))))
    ms = float(np.mean(times))
    line = {
        "metric": "mixed-batch SQP solves/s (4096 problems: indy7/iiwa14 x N 8/32/64/128)",
        "value": MIXED_TOTAL / (ms * 1e-3), "unit": "solves/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "p50_ms": float(np.median(times)), "p99_ms": float(np.percentile(times, 99)),
        "higher_is_better": True, "dtype": "f32+f64-reductions",
        "data": "synthetic (seeded draw of plants/horizons, figure-8 goals, rho ~ logU[1e-2,1e2])",
        "config": {"workload": "mixed 4096", "classes": classes, "sqp_iters": SQP_ITERS,
                   "l2": "flushed between steps"},
        "tuner_ms": {f"lanes{k[0]}_ppb{k[1]}_ctas{k[2]}": v for k, v in shapes.items()},
        "per_class": [{"plant": p, "N": n, "count": c,
                       "p50_ms_in_mixed_launch": float(np.median(times)),
                       "p99_ms_in_mixed_launch": float(np.percentile(times, 99)),
                       "p50_ms_alone": a[0], "p99_ms_alone": a[1],
                       "pcg_iters_mean": float(np.mean(st["pcg_iters"]))}
                      for (p, n, c), a, st in zip(classes, alone, stats)],
        "latency_note": "in the mixed launch every problem's result is ready when the launch "
                        "ends (the SQP stages run as one launch per stage over all classes), so "
                        "each class's latency is the launch's; alone = the class's own fused "
                        "solve",
        "sequential_alone_ms": float(sum(a[0] for a in alone)),
        "mixed_vs_sequential": float(sum(a[0] for a in alone)) / ms,
    }
    print(json.dumps(line))
    return 0


def run_reference_mixed(args):
    """The reference's mixed-workload arm: its modules (one per plant and
    horizon, one solve() per class) are not run.  The FP32 module
    bsqpN128_indy7 ended its process with cudaErrorIllegalAddress on this
    workload (484 problems padded to its batch-512 class), so the arm reports
    no number."""
    print(json.dumps({"impl": "reference", "unavailable":
                      "the reference's bsqpN128_indy7 module raised an illegal-address fault "
                      "(exit 188) on this workload; not run again"}))
    return 0


# --------------------------------------------------------------------------
# closed-loop workload: per plant, N=128, batch 512, 50 receding-horizon steps
# of 10 ms with seeded torque noise N(0, 0.05^2), figure-8 goals; forward
# rollout (one graph) and its reverse pass into x0, goals and the Q/R
# diagonals for a tracking loss; precision sweep against FP64
MPC_N, MPC_B, MPC_STEPS, MPC_SQP_ITERS = 128, 512, 50, 3


def run_mpc(args):
    """Per plant and precision: forward rollout and reverse pass times (CUDA
    events), the closed-loop state error against the FP64 rollout after 1, 10
    and 50 steps, and the gradient error of the reverse pass run on the FP64
    rollout's own trajectory and checkpoints (cast to the precision)."""
    import ctypes
    import torch
    import gato_b200
    import gato_b200._lib as L
    from gato_b200 import mpc
    from gato_b200 import workloads as W
    torch.cuda.set_device(0)
    dev = torch.device("cuda")
    steps = MPC_STEPS
    # the reference's MPC settings (python/bsqp/config.py:36-51, PCG max 200
    # at 1e-4) with three SQP iterations per control step instead of its one:
    # with one, the FP64 oracle's own closed loop leaves the joint velocity
    # limits (max |qd| 19.9 rad/s after 50 steps on iiwa14), with three it
    # tracks (1.25 rad/s, end-effector error 0.15 -> 0.05 m)
    kw = dict(max_sqp_iters=MPC_SQP_ITERS, kkt_tol=1e-3, max_pcg_iters=200, pcg_tol=1e-4,
              solve_ratio=1.0, mu=10.0, q_cost=2.0, qd_cost=1e-2, u_cost=2e-6, N_cost=50.0,
              q_lim_cost=0.01, vel_lim_cost=0.0, ctrl_lim_cost=0.0, rho=0.01)
    out = {"metric": "closed-loop MPC rollout (N=128, batch 512, 50 steps of 10 ms), ms",
           "solver": "reference MPC settings, three SQP iterations per step",
           "unit": "ms", "higher_is_better": False,
           "loss": "sum over steps of |x_t - x_0|^2 (states of the closed loop)",
           "plants": {}}

    def backward(s, o, dt, gt):
        B, nx = s.batch_size, s.nx
        dl = (2 * (o["x"] - o["x"][0])).to(dt).contiguous()
        dl[0] = 0
        g_x0 = torch.empty((B, nx), dtype=dt, device=dev)
        g_goal = torch.empty_like(gt)
        g_w = torch.empty((B, nx + s.nu), dtype=dt, device=dev)
        L.check(L.load().gato_rollout_backward(
            s._h, None, steps, L.vptr(gt), L.vptr(o["x"]), L.vptr(o["u"]), L.vptr(o["ckpt_xu"]),
            L.vptr(o["ckpt_rho"]), L.vptr(dl), L.vptr(g_x0), L.vptr(g_goal), L.vptr(g_w),
            0.0, 0))
        return g_w

    for plant in ("indy7", "iiwa14"):
        pr = W.make_problem(plant, MPC_N, MPC_B, seed=2028, goals="figure8", dt=DT)
        rng = np.random.default_rng(2029)
        nq = pr["model"].nq
        gt_np = W.figure8_goals(pr["model"], pr["xs"], MPC_N + steps, DT, rng)
        noise = rng.normal(0, 0.05, (steps, MPC_B, nq))
        res, ref = {}, None
        for prec in ("fp64", "mixed", "fp32"):
            dt = torch.float64 if prec == "fp64" else torch.float32
            T = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=dt, device=dev)
            s = gato_b200.BSQP(batch_size=MPC_B, N=MPC_N, dt=DT, plant_type=plant,
                               precision=prec, **kw)
            qd, rd = s.default_cost_diag()
            s.set_cost_diag_batch(qd, rd)
            x0, gt, nz = T(pr["xs"]), T(gt_np), T(noise)
            fw, bw = [], []
            for i in range(1 + max(1, args.steps // 25)):
                s.reset_dual()
                s.reset_rho()
                torch.cuda.synchronize()
                e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
                e[0].record()
                o = mpc.rollout(s, x0, gt, steps, nz)
                e[1].record()
                g_w = backward(s, o, dt, o["goal_traj"])
                e[2].record()
                torch.cuda.synchronize()
                if i >= 1:
                    fw.append(e[0].elapsed_time(e[1]))
                    bw.append(e[1].elapsed_time(e[2]))
            r = dict(forward_ms=float(np.mean(fw)), backward_ms=float(np.mean(bw)),
                     x=o["x"].double().cpu().numpy(),
                     nonfinite_x=int((~torch.isfinite(o["x"])).sum()),
                     nonfinite_grad=int((~torch.isfinite(g_w)).sum()),
                     max_abs_x=float(o["x"].abs().max()),
                     max_abs_qd=float(o["x"][..., nq:].abs().max()))
            if prec == "fp64":
                ref = dict(o=o, g_w=g_w.cpu().numpy(), gt=o["goal_traj"])
            else:
                # the reverse pass of this precision on the FP64 trajectory
                o64 = {k: (v.to(dt) if torch.is_tensor(v) else v) for k, v in ref["o"].items()}
                s.set_rho_penalty_batch(s.get_rho(), False)
                gw = backward(s, o64, dt, o64["goal_traj"].contiguous()).double().cpu().numpy()
                ok = np.isfinite(gw).all(axis=1) & np.isfinite(ref["g_w"]).all(axis=1)
                r["grad_w_err_vs_fp64"] = float(np.abs(gw[ok] - ref["g_w"][ok]).max()
                                                / np.abs(ref["g_w"][ok]).max())
                r["grad_nonfinite_problems_on_fp64_traj"] = int((~ok).sum())
                # the FP64 gradient's size where this precision's is not finite,
                # beside its median size over all problems
                gmax = np.abs(ref["g_w"]).max(axis=1)
                r["fp64_grad_absmax_median"] = float(np.median(gmax))
                r["fp64_grad_absmax_where_nonfinite"] = (
                    [float(v) for v in gmax[~ok]] if (~ok).any() else [])
            res[prec] = r
            s.close()
        x64 = res["fp64"]["x"]
        scale = max(1.0, float(np.abs(x64).max()))
        out["plants"][plant] = {
            p: {k: v for k, v in r.items() if k != "x"} | {
                f"x_err_vs_fp64_step{t}": float(np.abs(r["x"][t] - x64[t]).max() / scale)
                for t in (1, 10, steps)}
            for p, r in res.items()}
    print(json.dumps(out))
    return 0


# --------------------------------------------------------------------------
# batch-size sweep of the headline workload (iiwa14 N=32, 5 SQP iterations)
SWEEP_BATCHES = (1, 32, 128, 512, 1024)
# this library's arm also runs batches past the headline's, to the sizes an
# HBM-resident batch reaches (16384 problems: about 13 GB of solver buffers)
SWEEP_BATCHES_OURS = SWEEP_BATCHES + (4096, 16384)


def run_sweep(args):
    import torch
    import gato_b200
    import gato_b200._lib as L
    torch.cuda.set_device(0)
    dev = torch.device("cuda")
    kw = solver_kwargs()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.Stream(device=dev)
    rows = []
    for B in SWEEP_BATCHES_OURS:
        wl = make_workload(B, seed=2026)
        s = gato_b200.BSQP(batch_size=B, N=N, dt=DT, plant_type=PLANT, form="fused", **kw)
        T = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device=dev)
        d_xu0, d_xs, d_goal = T(wl["xu"]), T(wl["xs"]), T(wl["goal"])
        d_xu = d_xu0.clone()
        t = time_device_steps(torch, s, (d_xu, d_xs, d_goal, d_xu0), wl, args.steps,
                              args.warmup, flush, stream)
        h_xu = torch.empty(tuple(d_xu.shape), dtype=torch.float32).pin_memory()
        h_xs, h_goal = torch.tensor(wl["xs"]).pin_memory(), torch.tensor(wl["goal"]).pin_memory()
        e2e = []
        for i in range(args.warmup + args.steps):
            h_xu.copy_(torch.from_numpy(wl["xu"]))
            s.set_lambda(wl["lam"])
            s.reset_rho()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            L.check(L.load().gato_solve_host(s._h, L.fptr(h_xu), DT, L.fptr(h_xs),
                                             L.fptr(h_goal), None))
            if i >= args.warmup:
                e2e.append(1e3 * (time.perf_counter() - t0))
        s.close()
        rows.append({"batch": B, "solves_per_s": B / (float(np.mean(t)) * 1e-3),
                     "p50_ms": float(np.median(t)), "p99_ms": float(np.percentile(t, 99)),
                     "e2e_solves_per_s": B / (float(np.mean(e2e)) * 1e-3),
                     "e2e_p50_ms": float(np.median(e2e)), "e2e_p99_ms": float(np.percentile(e2e, 99))})
    print(json.dumps({"metric": "SQP solves/s and latency vs batch size (iiwa14 N=32, 5 SQP iters)",
                      "unit": "solves/s", "rows": rows}))
    return 0


def run_reference_sweep(args):
    rows = []
    threads = os.cpu_count() or 1
    for B in SWEEP_BATCHES:
        r = reference_gpu_leg(args, make_reference_workload(B, 2026, threads))
        r["batch"] = B
        rows.append(r)
    print(json.dumps({"impl": "reference", "metric": "SQP solves/s and latency vs batch size "
                      "(iiwa14 N=32, 5 SQP iters)", "unit": "solves/s", "rows": rows}))
    return 0


def run_profile(args):
    """One batched solve in each form, for ncu: a plain-form solve (k_merit,
    k_merit_sum, then per SQP iteration k_kkt, k_schur_inv, k_schur,
    k_schur_off, k_pcg, k_dz, k_merit, k_line_search), then a fused-form solve
    without its CUDA graph (per SQP iteration k_fused_kkt and k_fused_schur or the knot-parallel
    KKT and Schur kernels, the PCG kernel, k_check, k_merit_ls).  Default
    warm start perturbed by seeded noise; prints the per-kernel event times."""
    import ctypes
    import torch
    import gato_b200
    import gato_b200._lib as L
    from gato_b200 import workloads as W
    torch.cuda.set_device(0)
    pr = W.make_problem(args.plant, args.horizon, args.batch, seed=5)
    nq = pr["model"].nq
    xu = W.perturb(pr["xu"], nq, args.horizon, pr["rng"]).astype(np.float32)
    xu[:, :2 * nq] = pr["xs"]
    kw = dict(max_sqp_iters=args.sqp_iters, pcg_tol=PCG_TOL, max_pcg_iters=PCG_MAX)
    dev = torch.device("cuda")
    f64 = args.precision == "fp64"
    dt_ = torch.float64 if f64 else torch.float32
    T = lambda x: torch.tensor(np.ascontiguousarray(x), dtype=dt_, device=dev)
    d_xs, d_goal = T(pr["xs"]), T(pr["goal"])
    for form in ("plain", "fused"):
        s = gato_b200.BSQP(batch_size=args.batch, N=args.horizon, dt=DT, plant_type=args.plant,
                           form=form, precision=args.precision, **kw)
        d_xu = T(xu)
        ms = (ctypes.c_double * len(L.KERNELS))()
        n = (ctypes.c_int32 * len(L.KERNELS))()
        fn = L.load().gato_profile_solve_f64 if f64 else L.load().gato_profile_solve
        L.check(fn(s._h, None, L.vptr(d_xu), L.vptr(d_xs), L.vptr(d_goal), ms, n))
        print(form, {L.KERNELS[i]: round(ms[i], 3) for i in range(len(L.KERNELS)) if n[i]})
        s.close()
    return 0


def main():
    args = parse()
    if args.workload == "profile":
        return run_profile(args)
    if args.workload == "sweep":
        return run_reference_sweep(args) if args.impl == "reference" else run_sweep(args)
    if args.workload == "mpc":
        return run_mpc(args)
    if args.workload == "mixed":
        return run_reference_mixed(args) if args.impl == "reference" else run_mixed(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
