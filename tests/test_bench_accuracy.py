"""The bench's accuracy measures (dynamics defect and KKT stationarity from the
FP64 oracle's KKT blocks, `bench.kkt_measures`) on trajectories whose values
are known: an exact rollout of the integrator has zero defect, a velocity
kick of size d at one knot shows as a defect of about d, and multipliers
built by the backward recursion lambda_k = q_k + A_k^T lambda_{k+1} zero the
state part of the stationarity, leaving the control part r_k + B_k^T
lambda_{k+1}."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rollout(m, N, dt, rng):
    """x_{k+1} = f(x_k, u_k) with the reference's integrator
    (q+ = q + dt qd + dt^2/2 qdd, qd+ = qd + dt qdd)."""
    n, nu = 14, 7
    xs = np.concatenate([rng.uniform(-0.5, 0.5, 7), rng.normal(0, 0.1, 7)])
    xu = np.zeros((n + nu) * N - nu)
    x = xs.copy()
    for k in range(N):
        xu[k * (n + nu):k * (n + nu) + n] = x
        if k < N - 1:
            u = rng.normal(0, 1, nu)
            xu[k * (n + nu) + n:(k + 1) * (n + nu)] = u
            qdd = m.fd(x[:7], x[7:], u)
            x = np.concatenate([x[:7] + dt * x[7:] + 0.5 * dt * dt * qdd, x[7:] + dt * qdd])
    return xs, xu


def test_defect_and_stationarity_measures():
    sys.path.insert(0, ROOT)
    import bench
    from oracle import oracle as O
    N, dt, n, nu = bench.N, bench.DT, 14, 7
    m = O.Model(bench.PLANT)
    rng = np.random.default_rng(11)
    xs, xu = _rollout(m, N, dt, rng)
    goal = rng.normal(0, 0.3, 6 * N)
    zero = np.zeros((N + 2) * n)
    d, _ = bench.kkt_measures(xu[None], zero[None], xs[None], goal[None])
    assert d[0] < 1e-12, d

    kick = 1e-3
    xk = xu.copy()
    xk[5 * (n + nu) + 9] += kick
    d, _ = bench.kkt_measures(xk[None], zero[None], xs[None], goal[None])
    assert 0.999 * kick <= d[0] < 1.1 * kick, d

    P = O.make_params(dt=dt, **bench.solver_kwargs())
    kb = m.setup_kkt(N, P, dt, xu, xs, goal)
    lam = np.zeros((N + 2, n))
    lam[N] = kb["q"][N - 1]
    for k in range(N - 2, -1, -1):
        lam[k + 1] = kb["q"][k] + kb["A"][k] @ lam[k + 2]
    u_part = max(np.abs(kb["r"][k] + kb["B"][k] @ lam[k + 2]).max() for k in range(N - 1))
    _, s = bench.kkt_measures(xu[None], lam.reshape(1, -1), xs[None], goal[None])
    assert abs(s[0] - u_part) <= 1e-12 * max(1.0, u_part), (s, u_part)
    # and with lambda = 0 the measure is the largest cost-gradient entry
    _, s0 = bench.kkt_measures(xu[None], zero[None], xs[None], goal[None])
    assert abs(s0[0] - max(np.abs(kb["q"]).max(), np.abs(kb["r"][:N - 1]).max())) < 1e-12
