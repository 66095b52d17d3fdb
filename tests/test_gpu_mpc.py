"""Closed-loop rollout (gato_rollout) and its reverse pass
(gato_rollout_backward) in FP64:
  * the forward loop equals the same loop run with the FP64 oracle (solve,
    apply u_0 + noise to the oracle's dynamics, shift the warm start);
  * the reverse pass equals the composition, step by step, of gato_adjoint
    (checked against the dense FP64 reference elsewhere) and the simulator
    Jacobians of the oracle (checked against finite differences here)."""
import numpy as np
import pytest

from helpers import PARAMS_CFG2, nerr

pytestmark = pytest.mark.gpu

PLANT, N, B, STEPS = "iiwa14", 16, 2, 3
PARAMS = dict(PARAMS_CFG2, max_sqp_iters=4)


def _setup(seed):
    import torch
    import gato_b200
    from gato_b200 import mpc
    from gato_b200 import workloads as W
    torch.cuda.set_device(0)
    pr = W.make_problem(PLANT, N, B, seed=seed)
    rng = np.random.default_rng(seed)
    s = gato_b200.BSQP(batch_size=B, N=N, dt=0.01, plant_type=PLANT, precision="fp64", **PARAMS)
    gt = mpc.goal_trajectory(s, pr["model"], pr["xs"], STEPS, rng)
    noise = rng.normal(0, 0.05, (STEPS, B, s.nu))
    return s, pr, gt, noise


def _shift(xu, x_next, nx, nu):
    out = xu.copy()
    nxu = nx + nu
    Nk = (xu.shape[1] + nu) // nxu
    for k in range(Nk - 1):
        lo = k * nxu
        hi = lo + (nxu if k < Nk - 2 else nx)
        out[:, lo:hi] = xu[:, lo + nxu:hi + nxu]
    out[:, :nx] = x_next
    return out


def _sim(O, m, x, u, dt=0.01):
    nq = m.nq
    qdd = m.fd(x[:nq], x[nq:], u)
    return np.concatenate([x[:nq] + dt * x[nq:] + 0.5 * qdd * dt * dt, x[nq:] + dt * qdd])


def test_rollout_matches_oracle_loop(oracle_mod):
    import torch
    from gato_b200 import mpc
    O = oracle_mod
    s, pr, gt, noise = _setup(70)
    dev = torch.device("cuda")
    T = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    out = mpc.rollout(s, T(pr["xs"]), T(gt), STEPS, T(noise))
    xg = out["x"].cpu().numpy()
    m = O.Model(PLANT)
    ref = O.Solver(PLANT, N, B, O.make_params(dt=0.01, **PARAMS))
    nx, nu = 2 * m.nq, m.nq
    x = pr["xs"].astype(np.float64)
    xu = np.zeros((B, (nx + nu) * N - nu))
    for k in range(N):
        xu[:, k * (nx + nu):k * (nx + nu) + nx] = x
    for t in range(STEPS):
        xu[:, :nx] = x
        xu, _ = ref.solve(xu, 0.01, x, gt[:, 6 * t:6 * t + 6 * N])
        u = xu[:, nx:nx + nu] + noise[t]
        xn = np.stack([_sim(O, m, x[b], u[b]) for b in range(B)])
        assert nerr(xg[t + 1], xn) < 1e-8, t
        xu = _shift(xu, xn, nx, nu)
        x = xn
    s.close()


def test_rollout_backward_is_the_composition_of_step_adjoints(oracle_mod):
    import torch
    from gato_b200 import mpc
    O = oracle_mod
    s, pr, gt, noise = _setup(71)
    dev = torch.device("cuda")
    T = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    rng = np.random.default_rng(5)
    w = np.exp(rng.uniform(-1, 1, (B, 3 * s.nq)))
    s.set_cost_diag_batch(w[:, :s.nx], w[:, s.nx:])
    out = mpc.rollout(s, T(pr["xs"]), T(gt), STEPS, T(noise))
    dl = rng.normal(0, 1, (STEPS + 1, B, s.nx))
    g_x0, g_goal, g_w = (torch.empty((B, s.nx), dtype=torch.float64, device=dev),
                         torch.empty_like(out["goal_traj"]),
                         torch.empty((B, s.nx + s.nu), dtype=torch.float64, device=dev))
    import ctypes
    import gato_b200._lib as L
    rho_after = s.get_rho().copy()
    d_dl = T(dl)  # held in a name for the duration of the call
    L.check(L.load().gato_rollout_backward(
        s._h, None, STEPS, L.vptr(out["goal_traj"]), L.vptr(out["x"]), L.vptr(out["u"]),
        L.vptr(out["ckpt_xu"]), L.vptr(out["ckpt_rho"]), L.vptr(d_dl), L.vptr(g_x0),
        L.vptr(g_goal), L.vptr(g_w), 0.0, 0))
    torch.cuda.synchronize()
    np.testing.assert_allclose(s.get_rho(), rho_after, rtol=0, atol=0)
    # the same chain, step by step, from gato_adjoint and the oracle's Jacobians
    m = O.Model(PLANT)
    nx, nu = s.nx, s.nu
    x, u = out["x"].cpu().numpy(), out["u"].cpu().numpy()
    ck_xu, ck_rho = out["ckpt_xu"], out["ckpt_rho"].cpu().numpy()
    gx = dl[STEPS].copy()
    gw = np.zeros((B, nx + nu))
    gg = np.zeros_like(gt)
    h2, dt = 0.5 * 0.01 ** 2, 0.01
    for t in range(STEPS - 1, -1, -1):
        ga, gu = np.zeros((B, nx)), np.zeros((B, nu))
        for b in range(B):
            _, df = m.fd_grad(x[t, b, :7], x[t, b, 7:], u[t, b])
            dqdd_dx, minv = df[:, :nx], df[:, nx:]
            A = np.eye(nx)
            A[:7, 7:] += dt * np.eye(7)
            A[:7] += h2 * dqdd_dx
            A[7:] += dt * dqdd_dx
            Bm = np.vstack([h2 * minv, dt * minv])
            ga[b], gu[b] = A.T @ gx[b], Bm.T @ gx[b]
        dlxu = np.zeros((B, s.traj_size))
        dlxu[:, nx:nx + nu] = gu
        s.set_rho_penalty_batch(ck_rho[t], False)
        g_xs, g_goal_t, g_wt = s.adjoint_device(ck_xu[t].contiguous(), T(x[t]),
                                                T(gt[:, 6 * t:6 * t + 6 * N]), T(dlxu))
        gx = dl[t] + ga + g_xs.cpu().numpy()
        gw += g_wt.cpu().numpy()
        gg[:, 6 * t:6 * t + 6 * N] += g_goal_t.cpu().numpy()
    assert nerr(g_x0.cpu().numpy(), gx) < 1e-9
    assert nerr(g_w.cpu().numpy(), gw) < 1e-9
    assert nerr(g_goal.cpu().numpy(), gg) < 1e-9
    s.close()


def test_simulator_jacobians_match_finite_differences(oracle_mod):
    """The simulator Jacobians used above (trapezoidal step of the oracle's
    forward dynamics) against central differences."""
    O = oracle_mod
    m = O.Model(PLANT)
    rng = np.random.default_rng(3)
    x, u = np.concatenate([rng.uniform(-1, 1, 7), rng.normal(0, 0.2, 7)]), rng.normal(0, 3, 7)
    _, df = m.fd_grad(x[:7], x[7:], u)
    dt, h2 = 0.01, 0.5e-4
    A = np.eye(14)
    A[:7, 7:] += dt * np.eye(7)
    A[:7] += h2 * df[:, :14]
    A[7:] += dt * df[:, :14]
    h = 1e-6
    for j in range(14):
        e = np.zeros(14)
        e[j] = h
        num = (_sim(O, m, x + e, u) - _sim(O, m, x - e, u)) / (2 * h)
        np.testing.assert_allclose(A[:, j], num, rtol=1e-6, atol=1e-9)


def test_rollout_autograd_reaches_the_weights():
    import torch
    from gato_b200 import mpc
    s, pr, gt, noise = _setup(72)
    dev = torch.device("cuda")
    T = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    logq = torch.zeros((B, s.nx), dtype=torch.float64, device=dev, requires_grad=True)
    logr = torch.full((B, s.nu), -2.0, dtype=torch.float64, device=dev, requires_grad=True)
    x0 = T(pr["xs"]).requires_grad_(True)
    xs = mpc.rollout_differentiable(s, x0, T(gt), STEPS, logq.exp(), logr.exp(), T(noise))
    loss = (xs[1:] ** 2).sum()
    loss.backward()
    for t in (x0, logq, logr):
        assert t.grad is not None and torch.isfinite(t.grad).all()
    assert float(logr.grad.abs().sum()) > 0
    s.close()


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_hypothesis_selection_matches_oracle_simulator(oracle_mod, precision):
    """Batch-hypothesis selection (gato_select_hypothesis,
    mpc_controller.py:295-309): each problem's one-step simulation under its
    own wrench hypothesis is scored against a measured state made by the
    oracle's simulator under hypothesis 5; errors match the oracle's, the
    argmin is 5, and the winner's trajectory is broadcast to every row."""
    import torch
    import gato_b200
    from gato_b200 import mpc
    torch.cuda.set_device(0)
    O = oracle_mod
    plant, Bh, Nh, dt = "iiwa14", 16, 8, 0.01
    rng = np.random.default_rng(67)
    s = gato_b200.BSQP(batch_size=Bh, N=Nh, dt=dt, plant_type=plant, precision=precision)
    f = rng.normal(0, 5, (Bh, 6))
    s.set_f_ext_B(f)
    x_last = np.concatenate([rng.uniform(-1, 1, 7), rng.normal(0, 0.3, 7)])
    u_last = rng.normal(0, 5, 7)
    m = O.Model(plant)

    def sim(b):
        qdd = m.fd(x_last[:7], x_last[7:], u_last, f[b].astype(np.float32).astype(np.float64))
        return np.concatenate([x_last[:7] + dt * x_last[7:] + 0.5 * qdd * dt * dt,
                               x_last[7:] + dt * qdd])

    x_curr = sim(5) + rng.normal(0, 1e-7, 14)
    ref_err = np.array([np.linalg.norm(sim(b) - x_curr) for b in range(Bh)])
    dtt = torch.float64 if precision == "fp64" else torch.float32
    T = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=dtt, device="cuda")
    xu = T(rng.normal(0, 1, (Bh, s.traj_size)))
    row5 = xu[5].clone()
    x_l, u_l, x_c = T(x_last), T(u_last), T(x_curr)
    best, err = mpc.select_hypothesis(s, x_l, u_l, x_c, dt, xu=xu)
    torch.cuda.synchronize()
    s.close()
    assert best == 5
    tol = 1e-12 if precision == "fp64" else 2e-5
    np.testing.assert_allclose(err.double().cpu().numpy(), ref_err, rtol=0, atol=tol)
    assert torch.equal(xu, row5.expand(Bh, -1))
