"""Closed-loop receding-horizon MPC on the batched solver (no counterpart in
the reference's solver: its loop is Python around one solve per step,
python/bsqp/mpc_controller.py).

    out = rollout(solver, x0, goal_traj, steps, noise)      # one CUDA graph
    xs = rollout_differentiable(solver, x0, goal_traj, steps, q_diag, r_diag,
                                noise)                        # torch autograd
    loss(xs).backward()   # gradients for x0, goal_traj, q_diag, r_diag

Every step solves from the current state with the goal window of that step,
applies the first control plus noise to the same dynamics for one dt, and
shifts the warm start by one knot (gato_rollout).  The reverse pass
(gato_rollout_backward) chains the simulator's step Jacobians with the
adjoint of each step's QP from per-step checkpoints of the solution and rho,
recomputing the dynamics derivatives.
"""
import ctypes

import numpy as np
import torch

from . import _lib as L
from .interface import BSQP


def _dtype(solver):
    return torch.float64 if solver.precision == "fp64" else torch.float32


def default_warm_start(solver, x0):
    B, nx, nu, N = solver.batch_size, solver.nx, solver.nu, solver.N
    xu = torch.zeros((B, solver.traj_size), dtype=x0.dtype, device=x0.device)
    for k in range(N):
        xu[:, k * (nx + nu):k * (nx + nu) + nx] = x0
    return xu


def rollout(solver: BSQP, x0, goal_traj, steps, noise=None, xu_init=None, checkpoints=True,
            stream=None):
    """Runs `steps` receding-horizon steps.  x0 [B, nx], goal_traj
    [B, 6 (N + steps)], noise [steps, B, nu] or None (torch CUDA tensors of
    the solver's dtype).  Returns dict(x [steps+1, B, nx], u [steps, B, nu]
    (applied), xu (final warm start), ckpt_xu, ckpt_rho)."""
    dt = _dtype(solver)
    dev = x0.device
    B, nx, nu = solver.batch_size, solver.nx, solver.nu
    x = torch.empty((steps + 1, B, nx), dtype=dt, device=dev)
    x[0] = x0.detach().to(dt)
    u = torch.empty((steps, B, nu), dtype=dt, device=dev)
    xu = (xu_init.detach().to(dt).clone() if xu_init is not None
          else default_warm_start(solver, x[0]))
    gt = goal_traj.detach().to(dt).contiguous()
    nz = noise.detach().to(dt).contiguous() if noise is not None else None
    ck_xu = torch.empty((steps, B, solver.traj_size), dtype=dt, device=dev) if checkpoints else None
    ck_rho = torch.empty((steps, B), dtype=dt, device=dev) if checkpoints else None
    st = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
    L.check(L.load().gato_rollout(solver._h, ctypes.c_void_p(int(st)), int(steps), L.vptr(gt),
                                  L.vptr(xu), L.vptr(nz), L.vptr(x), L.vptr(u), L.vptr(ck_xu),
                                  L.vptr(ck_rho)))
    return dict(x=x, u=u, xu=xu, ckpt_xu=ck_xu, ckpt_rho=ck_rho, goal_traj=gt)


class RolloutFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x0, goal_traj, q_diag, r_diag, solver, steps, noise, xu_init):
        dt = _dtype(solver)
        qd, rd = q_diag.detach().to(dt), r_diag.detach().to(dt)
        solver.set_cost_diag_batch(qd.cpu().numpy(), rd.cpu().numpy())
        out = rollout(solver, x0, goal_traj, steps, noise, xu_init)
        ctx.solver, ctx.steps = solver, steps
        ctx.save_for_backward(out["x"], out["u"], out["ckpt_xu"], out["ckpt_rho"],
                              out["goal_traj"], qd, rd)
        ctx.in_dtypes = (x0.dtype, goal_traj.dtype, q_diag.dtype, r_diag.dtype)
        return out["x"].clone()

    @staticmethod
    def backward(ctx, g_x):
        x, u, ck_xu, ck_rho, gt, qd, rd = ctx.saved_tensors
        solver, steps = ctx.solver, ctx.steps
        solver.set_cost_diag_batch(qd.cpu().numpy(), rd.cpu().numpy())
        B, nx = solver.batch_size, solver.nx
        dl = g_x.detach().to(x.dtype).contiguous()
        g_x0 = torch.empty((B, nx), dtype=x.dtype, device=x.device)
        g_goal = torch.empty_like(gt)
        g_w = torch.empty((B, nx + solver.nu), dtype=x.dtype, device=x.device)
        st = torch.cuda.current_stream(x.device).cuda_stream
        L.check(L.load().gato_rollout_backward(
            solver._h, ctypes.c_void_p(int(st)), int(steps), L.vptr(gt), L.vptr(x), L.vptr(u),
            L.vptr(ck_xu), L.vptr(ck_rho), L.vptr(dl), L.vptr(g_x0), L.vptr(g_goal),
            L.vptr(g_w), 0.0, 0))
        d = ctx.in_dtypes
        return (g_x0.to(d[0]), g_goal.to(d[1]), g_w[:, :nx].to(d[2]), g_w[:, nx:].to(d[3]),
                None, None, None, None)


def rollout_differentiable(solver: BSQP, x0, goal_traj, steps, q_diag=None, r_diag=None,
                           noise=None, xu_init=None):
    """States [steps+1, B, nx] of the closed loop, differentiable with
    respect to x0, goal_traj and the diagonal cost weights (default: the
    solver's scalar weights)."""
    dev = x0.device
    if q_diag is None or r_diag is None:
        dq, dr = solver.default_cost_diag()
        q_diag = torch.tensor(dq, device=dev) if q_diag is None else q_diag
        r_diag = torch.tensor(dr, device=dev) if r_diag is None else r_diag
    return RolloutFunction.apply(x0, goal_traj, q_diag, r_diag, solver, int(steps), noise,
                                 xu_init)


def goal_trajectory(solver, model, xs, steps, rng, dt=0.01):
    """Figure-8 goals long enough for `steps` receding-horizon steps
    (gato_b200.workloads.figure8_goals over N + steps knots)."""
    from . import workloads as W
    return W.figure8_goals(model, np.asarray(xs), solver.N + steps, dt, rng)


# ---------------------------------------------------------------- hypotheses
def select_hypothesis(solver: BSQP, x_last, u_last, x_curr, dt, xu=None, stream=None):
    """Batch-hypothesis selection on the device (gato_select_hypothesis;
    python/bsqp/mpc_controller.py:295-309 and 241-242): every problem
    simulates (x_last, u_last) for dt under its own wrench hypothesis (the
    solver's f_ext batch); returns (best index (int), errors [B] tensor) and,
    when xu [B, traj] is given, overwrites every row with row `best`.
    x_last [nx], u_last [nu], x_curr [nx]: CUDA tensors of the solver's
    dtype."""
    dt_ = _dtype(solver)
    dev = x_curr.device
    B = solver.batch_size
    err = torch.empty(B, dtype=dt_, device=dev)
    best = torch.empty(1, dtype=torch.int32, device=dev)
    xl, ul, xc = (t.detach().to(dt_).contiguous() for t in (x_last, u_last, x_curr))
    st = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
    L.check(L.load().gato_select_hypothesis(solver._h, ctypes.c_void_p(int(st)), L.vptr(xl),
                                            L.vptr(ul), L.vptr(xc), float(dt), L.vptr(xu),
                                            L.vptr(err), L.vptr(best)))
    return int(best.item()), err


class ForceEstimator:
    """Host-side wrench-hypothesis generator and update rule of the
    reference's batch MPC (examples/force_estimator.py:4-137, with the
    settings of python/bsqp/mpc_controller.py:123-134): problem 0 takes the
    smoothed estimate, 1 no wrench, 2 the estimate pushed along its momentum,
    and the rest probe a sphere of the current radius around the estimate
    (Fibonacci-spiral directions, randomly rotated after every update).  A
    winner among the first three shrinks the radius, an exploring winner
    grows it.  The rotation draws from `rng` (numpy.random.Generator) instead
    of numpy's global state."""

    def __init__(self, batch_size, initial_radius=5.0, min_radius=2.0, max_radius=20.0,
                 smoothing_factor=0.5, rng=None):
        if batch_size <= 3:
            raise ValueError("the hypothesis batch needs more than 3 problems")
        self.B = batch_size
        self.radius0 = initial_radius
        self.min_radius, self.max_radius = min_radius, max_radius
        self.smoothing = smoothing_factor
        self.rng = rng if rng is not None else np.random.default_rng()
        n = batch_size - 3
        i = np.arange(n)
        y = 1.0 - 2.0 * i / (n - 1) if n > 1 else np.zeros(n)
        r = np.sqrt(np.maximum(0.0, 1.0 - y * y))
        th = 2.0 * np.pi * i / ((1.0 + np.sqrt(5.0)) / 2.0)
        self.dirs = np.stack([r * np.cos(th), y, r * np.sin(th)], axis=1).astype(np.float32)
        self.reset()

    def reset(self):
        self.estimate = np.zeros(6, np.float32)
        self.momentum = np.zeros(6, np.float32)
        self.smoothed = np.zeros(6, np.float32)
        self.radius = self.radius0
        self.confidence = 0.0
        self.errors = []
        self.rotation = np.eye(3, dtype=np.float32)

    def generate_batch(self):
        """[B, 6] wrench hypotheses (force xyz, torque xyz)."""
        out = np.zeros((self.B, 6), np.float32)
        out[0] = self.smoothed
        out[2] = self.smoothed + 0.5 * self.momentum
        centre = 0.7 * self.smoothed[:3] + 0.3 * self.estimate[:3]
        out[3:, :3] = centre + self.radius * (self.dirs @ self.rotation.T)
        out[3:, 3:] = self.smoothed[3:]
        return out

    def _rotation(self):
        u1, u2, u3 = self.rng.random(3)
        a, b = np.sqrt(1.0 - u1), np.sqrt(u1)
        x, y = a * np.sin(2 * np.pi * u2), a * np.cos(2 * np.pi * u2)
        z, w = b * np.sin(2 * np.pi * u3), b * np.cos(2 * np.pi * u3)
        return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                         [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                         [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]],
                        np.float32)

    def update(self, best, errors, alpha=0.6, beta=0.5):
        """Moves the estimate toward the winning hypothesis (the weights of
        mpc_controller.py:306) and adapts the search radius."""
        errors = np.asarray(errors, np.float64)
        self.errors.append(float(np.min(errors)))
        win = self.generate_batch()[best]
        self.momentum = beta * self.momentum + (1 - beta) * (win - self.estimate)
        raw = alpha * win + (1 - alpha) * self.estimate
        self.estimate = 0.8 * self.estimate + 0.2 * (raw + 0.5 * self.momentum)
        self.smoothed = (1 - self.smoothing) * self.smoothed + self.smoothing * self.estimate
        if best < 3:
            self.radius *= 0.95
            self.confidence = min(1.0, self.confidence + 0.05)
        else:
            self.radius *= 1.05
            self.confidence = max(0.0, self.confidence - 0.1)
        self.radius = float(np.clip(self.radius, self.min_radius, self.max_radius))
        if len(self.errors) > 5:
            recent = np.array(self.errors[-5:])
            if np.std(recent) < 0.01:
                self.radius *= 0.9
            elif recent[-1] > 1.5 * np.mean(recent[:-1]):
                self.radius *= 1.3
                self.confidence *= 0.5
            self.radius = float(np.clip(self.radius, self.min_radius, self.max_radius))
        self.rotation = self._rotation()


def hypothesis_step(solver: BSQP, estimator: ForceEstimator, x_last, u_last, x_curr, dt,
                    goals, xu, stream=None):
    """One control step of the batch-hypothesis MPC loop
    (mpc_controller.py:225-243): score the current hypotheses against the
    state just measured (device), update the estimator (host), install the
    next hypotheses, broadcast the winning trajectory as every problem's warm
    start and solve from x_curr.  xu [B, traj] holds the previous solve's
    trajectories and is updated in place; returns (best, errors, stats)."""
    best, err = select_hypothesis(solver, x_last, u_last, x_curr, dt, xu=xu, stream=stream)
    estimator.update(best, err.double().cpu().numpy())
    solver.set_f_ext_B(estimator.generate_batch())
    xu[:, :solver.nx] = x_curr
    xs = x_curr.expand(solver.batch_size, -1).contiguous()
    stats = solver.solve_device(xu, xs, goals,
                                stream=stream if stream is not None else
                                torch.cuda.current_stream(x_curr.device).cuda_stream)
    return best, err, stats
