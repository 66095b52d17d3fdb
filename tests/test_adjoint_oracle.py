"""The dense FP64 adjoint reference (oracle/adjoint_ref.py) against central
finite differences of the same QP map, on the CPU: this pins the gradient
formulas that gato_adjoint implements."""
import numpy as np
import pytest

from helpers import problem


@pytest.mark.parametrize("plant,with_wdiag", [("iiwa14", True), ("indy7", False),
                                              ("iiwa14", False)])
def test_dense_adjoint_matches_finite_differences(oracle_mod, plant, with_wdiag):
    from oracle import adjoint_ref as AR
    O = oracle_mod
    N = 6
    pr = problem(plant, N, 1, seed=7)
    m = O.Model(plant)
    nq = m.nq
    n, mm = 2 * nq, nq
    P = O.make_params(dt=0.01, q_cost=1.5, qd_cost=1e-2, u_cost=1e-3, q_lim_cost=1e-3)
    rng = np.random.default_rng(3)
    wdiag = np.exp(rng.uniform(-2, 2, n + mm)) if with_wdiag else None
    xu = pr["xu"][0].astype(np.float64)
    xs = pr["xs"][0].astype(np.float64) + rng.normal(0, 1e-3, n)
    goal = pr["goal"][0].astype(np.float64)
    dl = rng.normal(0, 1, xu.size)
    rho = 1e-3
    a = AR.adjoint_grad(m, N, P, 0.01, xu, xs, goal, wdiag, rho, dl)
    f = AR.fd_grad(m, N, P, 0.01, xu, xs, goal, wdiag, rho, dl)
    for k in ("g_xs", "g_goal", "g_wdiag"):
        scale = max(1.0, np.abs(f[k]).max())
        assert np.abs(a[k] - f[k]).max() / scale < 2e-6, (k, a[k], f[k])
    # the forward step solves the QP: stationarity and dynamics rows
    dz, lam, asm = AR.qp_step(m, N, P, 0.01, xu, xs, goal, wdiag, rho)
    assert np.abs(asm["G"] @ dz + asm["g"] + asm["H"].T @ lam).max() < 1e-8
    assert np.abs(asm["H"] @ dz - asm["c"]).max() < 1e-10


def test_dense_system_is_the_solvers_schur_system(oracle_mod):
    """The dense KKT system is the one the reference's Schur complement and
    step recovery solve (restated in the oracle): solving S lambda = gamma
    densely from its block rows gives the same lambda and step."""
    from oracle import adjoint_ref as AR
    O = oracle_mod
    N, plant = 5, "iiwa14"
    pr = problem(plant, N, 1, seed=9)
    m = O.Model(plant)
    nq = m.nq
    n = 2 * nq
    P = O.make_params(dt=0.01, q_cost=1.0, qd_cost=1e-2, u_cost=1e-3)
    xu, xs, goal = (pr[k][0].astype(np.float64) for k in ("xu", "xs", "goal"))
    rho = 1e-2
    dz, lam, asm = AR.qp_step(m, N, P, 0.01, xu, xs, goal, None, rho)
    kkt = asm["kkt"]
    sch = O.form_schur(nq, N, rho, kkt)
    Sd = np.zeros((N * n, N * n))
    for k in range(N):
        blk = sch["S"][k]
        for j, col in ((-1, 0), (0, 1), (1, 2)):
            if 0 <= k + j < N:
                Sd[k * n:(k + 1) * n, (k + j) * n:(k + j + 1) * n] = blk[:, col * n:(col + 1) * n]
    lp = np.zeros((N + 2) * n)
    lp[n:(N + 1) * n] = np.linalg.solve(Sd, sch["gamma"][n:(N + 1) * n])
    dz2, _, _ = O.compute_dz(nq, N, lp, sch["Qinv"], sch["Rinv"], kkt["q"], kkt["r"], kkt["A"],
                             kkt["B"])
    assert np.abs(lp[n:(N + 1) * n] - lam).max() / max(1, np.abs(lam).max()) < 1e-7
    assert np.abs(dz2 - dz).max() / max(1, np.abs(dz).max()) < 1e-7
