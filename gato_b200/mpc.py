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
