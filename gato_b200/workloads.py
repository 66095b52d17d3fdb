"""Seeded synthetic workloads with the shapes and value distributions of the
benchmark configurations (no dataset exists for this path; the reference's own
figure-8 generator, python/bsqp/common.py:10-46, sets the goal shape).

All arrays are float32 in the C ABI layouts:
  xs    [B, nx]      initial states
  goal  [B, 6N]      end-effector goals, [px py pz 0 0 0] per knot
  xu    [B, traj]    warm start [x_0 u_0 ... x_{N-1}]
"""
import numpy as np

from . import _lib as L
from .kinematics import ee_position


def limits(model):
    nq = model.nq
    return np.array([model.q_limit[i] for i in range(nq)])


def initial_states(model, B, rng):
    """q ~ U(0.8 x joint limits), qd ~ N(0, 0.1^2)."""
    lim = limits(model)
    q = rng.uniform(-0.8, 0.8, (B, model.nq)) * lim
    qd = rng.normal(0.0, 0.1, (B, model.nq))
    return np.concatenate([q, qd], axis=1)


def constant_goals(model, xs, N, rng, sigma=0.05):
    """A constant end-effector goal FK(q0) + N(0, sigma^2) per problem."""
    B = xs.shape[0]
    p0 = ee_position(model, xs[:, : model.nq])
    goal = np.zeros((B, N, 6))
    goal[:, :, :3] = (p0 + rng.normal(0.0, sigma, (B, 3)))[:, None, :]
    return goal.reshape(B, 6 * N)


def figure8_goals(model, xs, N, dt, rng):
    """Lemniscate goals in the shape of common.py:figure8: x = A sin(tau),
    z = A sin(2 tau)/2, rotated pi/4 about z; centre FK(q0) + N(0, 0.02^2),
    A ~ U[0.1, 0.3] m, period ~ U[2, 6] s, phase ~ U[0, 2 pi)."""
    B = xs.shape[0]
    p0 = ee_position(model, xs[:, : model.nq])
    centre = p0 + rng.normal(0.0, 0.02, (B, 3))
    A = rng.uniform(0.1, 0.3, B)
    period = rng.uniform(2.0, 6.0, B)
    phase = rng.uniform(0.0, 2 * np.pi, B)
    th = np.pi / 4
    Rz = np.array([[np.cos(th), -np.sin(th), 0.0], [np.sin(th), np.cos(th), 0.0], [0, 0, 1.0]])
    k = np.arange(N)
    tau = 2 * np.pi * k[None, :] * dt / period[:, None] + phase[:, None]
    local = np.stack([A[:, None] * np.sin(tau), np.zeros_like(tau),
                      A[:, None] * np.sin(2 * tau) / 2], axis=-1)
    pts = centre[:, None, :] + local @ Rz.T
    goal = np.zeros((B, N, 6))
    goal[:, :, :3] = pts
    return goal.reshape(B, 6 * N)


def default_warm_start(xs, N, nu):
    """x0 repeated at every knot, zero controls (common.py:93-99)."""
    B, nx = xs.shape
    xu = np.zeros((B, N, nx + nu))
    xu[:, :, :nx] = xs[:, None, :]
    return xu.reshape(B, -1)[:, : N * (nx + nu) - nu].copy()


def perturb(xu, nq, N, rng, sigma_x=0.01, sigma_u=0.1):
    """q, qd ~ +N(0, sigma_x^2), u ~ +N(0, sigma_u^2) on every knot but x_0."""
    B = xu.shape[0]
    nx, nu = 2 * nq, nq
    full = np.zeros((B, N * (nx + nu)))
    full[:, : xu.shape[1]] = xu
    full = full.reshape(B, N, nx + nu)
    full[:, 1:, :nx] += rng.normal(0.0, sigma_x, (B, N - 1, nx))
    full[:, :, nx:] += rng.normal(0.0, sigma_u, (B, N, nu))
    return full.reshape(B, -1)[:, : xu.shape[1]].copy()


def make_problem(plant, N, B, seed, goals="figure8", dt=0.01, model=None):
    """Returns dict(model, xs, goal, xu) as float32 arrays (`model`, a
    gato_model_t, replaces the built-in plant)."""
    model = model if model is not None else L.builtin_model(plant)
    rng = np.random.default_rng(seed)
    xs = initial_states(model, B, rng)
    if goals == "figure8":
        goal = figure8_goals(model, xs, N, dt, rng)
    else:
        goal = constant_goals(model, xs, N, rng)
    xu = default_warm_start(xs, N, model.nq)
    return dict(model=model, xs=xs.astype(np.float32), goal=goal.astype(np.float32),
                xu=xu.astype(np.float32), rng=rng)
