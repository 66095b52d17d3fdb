"""Differentiable batched solve: torch.autograd.Function over gato_solve and
gato_adjoint (no counterpart in the reference).

    XU = solve_differentiable(solver, x0, goals, q_diag, r_diag, xu_init)
    loss(XU).backward()   # gradients for x0, goals, q_diag, r_diag

The forward pass is the solver's batched SQP (XU[:, :nx] = x0 as in
bsqp.interface.BSQP.solve).  The backward pass differentiates the QP of the
returned trajectory implicitly (gato_adjoint): one KKT formation at XU with
recomputed dynamics derivatives, the Schur system, and two PCG solves (the
forward QP step and the transposed KKT system), no stored tape.  The
gradient is exact for the QP map XU + dz(theta) and for a converged solve;
the solver's lambda and rho are not changed by the backward pass, and the
cost weights are re-applied from the saved inputs, so other solves may run
between forward and backward (rho is taken at backward time).
"""
import torch

from .interface import BSQP


class DifferentiableSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x0, goals, q_diag, r_diag, solver, xu_init):
        nx = solver.nx
        dt = torch.float64 if solver.precision == "fp64" else torch.float32
        x0c = x0.detach().to(dt).contiguous()
        gc = goals.detach().to(dt).contiguous()
        qd = q_diag.detach().to(dt)
        rd = r_diag.detach().to(dt)
        solver.set_cost_diag_batch(qd.cpu().numpy(), rd.cpu().numpy())
        xu = xu_init.detach().to(dt).clone().contiguous()
        xu[:, :nx] = x0c
        stream = torch.cuda.current_stream(xu.device).cuda_stream
        solver.solve_device(xu, x0c, gc, stream=stream, with_stats=False)
        ctx.solver = solver
        ctx.save_for_backward(xu, x0c, gc, qd, rd)
        ctx.in_dtypes = (x0.dtype, goals.dtype, q_diag.dtype, r_diag.dtype)
        return xu.clone()

    @staticmethod
    def backward(ctx, g_xu):
        xu, x0c, gc, qd, rd = ctx.saved_tensors
        solver = ctx.solver
        solver.set_cost_diag_batch(qd.cpu().numpy(), rd.cpu().numpy())
        stream = torch.cuda.current_stream(xu.device).cuda_stream
        dl = g_xu.detach().to(xu.dtype).contiguous()
        g_xs, g_goal, g_w = solver.adjoint_device(xu, x0c, gc, dl, stream=stream)
        nx = solver.nx
        d = ctx.in_dtypes
        return (g_xs.to(d[0]), g_goal.to(d[1]), g_w[:, :nx].to(d[2]), g_w[:, nx:].to(d[3]),
                None, None)


def solve_differentiable(solver: BSQP, x0, goals, q_diag=None, r_diag=None, xu_init=None):
    """XU [B, traj] of the batched solve, differentiable with respect to x0
    [B, nx], goals [B, 6N] and the diagonal cost weights q_diag [B, nx],
    r_diag [B, nu] (default: the solver's scalar weights, [0, qd_cost] and
    u_cost).  xu_init defaults to x0 repeated with zero controls (the
    reference's default warm start)."""
    B, nx, nu, N = solver.batch_size, solver.nx, solver.nu, solver.N
    dev = x0.device
    if q_diag is None or r_diag is None:
        dq, dr = solver.default_cost_diag()
        if q_diag is None:
            q_diag = torch.tensor(dq, device=dev)
        if r_diag is None:
            r_diag = torch.tensor(dr, device=dev)
    if xu_init is None:
        xu_init = torch.zeros((B, solver.traj_size), dtype=x0.dtype, device=dev)
        for k in range(N):
            xu_init[:, k * (nx + nu):k * (nx + nu) + nx] = x0.detach()
    return DifferentiableSolve.apply(x0, goals, q_diag, r_diag, solver, xu_init)
