"""Generates the golden fixtures in this directory by running the reference's
own dynamics, plant cost and integrator code, compiled for the host in FP64
(oracle/_ref/libgrid_ref_<plant>.so, built by oracle/build_ref.py from the
reference sources).

The fixtures pin the FP64 oracle to the reference: tests/test_oracle_golden.py
checks the oracle against them on machines where the reference tree is absent.

Usage: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))

from oracle import oracle as O  # noqa: E402

LIMITS = {  # |q| limits (iiwa14_plant.cuh:37-46, indy7_plant.cuh:66-74)
    "iiwa14": np.array([2.96706, 2.09440, 2.96706, 2.09440, 2.96706, 2.09440, 3.05433]),
    "indy7": np.array([3.0543, 3.0543, 3.0543, 3.0543, 3.0543, 3.7520]),
}


def cases(plant, count, seed):
    rng = np.random.default_rng(seed)
    ref = O.RefDynamics(plant)
    nq = ref.nq
    nx, nu = 2 * nq, nq
    dt = 0.01
    out = {k: [] for k in [
        "q", "qd", "u", "fext", "has_fext", "weights", "goal", "goal1", "xnext",
        "qdd", "df_du", "ee_pose", "ee_grad", "cost", "cost_terminal", "Q", "qv", "R", "rv",
        "A", "B", "c", "int_err"]}
    for t in range(count):
        q = rng.uniform(-0.9, 0.9, nq) * LIMITS[plant]
        qd = rng.normal(0, 0.5, nq)
        u = rng.normal(0, 5, nq)
        has_f = t % 3 == 2
        fext = rng.normal(0, 3, 6) if has_f else np.zeros(6)
        w = np.array([rng.uniform(0.5, 3), 10 ** rng.uniform(-4, -1), 10 ** rng.uniform(-7, -3),
                      rng.uniform(5, 60), 10 ** rng.uniform(-4, -1), 10 ** rng.uniform(-4, -1),
                      10 ** rng.uniform(-6, -3)])
        goal = np.concatenate([rng.normal([0.3, 0.2, 0.6], 0.2), np.zeros(3)])
        goal1 = np.concatenate([rng.normal([0.3, 0.2, 0.6], 0.2), np.zeros(3)])
        xnext = np.concatenate([q + rng.normal(0, 0.01, nq), qd + rng.normal(0, 0.05, nq)])
        f = fext if has_f else None
        qdd, df = ref.fd_grad(q, qd, u, f)
        pose, grad = ref.ee(q)
        P = O.make_params(q_cost=w[0], qd_cost=w[1], u_cost=w[2], N_cost=w[3], q_lim_cost=w[4],
                          vel_lim_cost=w[5], ctrl_lim_cost=w[6])
        xu = np.concatenate([q, qd, u])
        cost = ref.tracking_cost(P, xu, goal, terminal=False)
        cost_t = ref.tracking_cost(P, xu[:nx], goal, terminal=True)
        Q, qv, R, rv = ref.cost_grad_hess(P, xu, goal)
        xux = np.concatenate([q, qd, u, xnext])
        A, B, c = ref.linearized_dynamics(xux, dt, f)
        ie = ref.integrator_error(xux, dt, f)
        for k, v in dict(q=q, qd=qd, u=u, fext=fext, has_fext=has_f, weights=w, goal=goal,
                         goal1=goal1, xnext=xnext, qdd=qdd, df_du=df, ee_pose=pose,
                         ee_grad=grad, cost=cost, cost_terminal=cost_t, Q=Q, qv=qv, R=R, rv=rv,
                         A=A, B=B, c=c, int_err=ie).items():
            out[k].append(v)
    return {k: np.array(v) for k, v in out.items()}


def main():
    for i, plant in enumerate(["iiwa14", "indy7"]):
        data = cases(plant, 24, 1234 + i)
        path = os.path.join(HERE, f"ref_dynamics_{plant}.npz")
        np.savez_compressed(path, dt=0.01, **data)
        print(path)


if __name__ == "__main__":
    main()
