"""The oracle's per-problem status word (the checker of the GPU solver's
GATO_STATUS_* bits) on host-made faults: a NaN input flags only its problem,
zero iteration limits give the reference's semantics (zero SQP iterations:
not converged; zero PCG iterations: converged), a singular KKT system is
flagged non-finite, and no fault stops the solve."""
import numpy as np

CONVERGED, MAX_ITER, LS_FAIL, NONFINITE, PCG_MAX = 1, 2, 4, 8, 16


def _problem(plant, N, B, seed):
    from gato_b200 import workloads as W
    pr = W.make_problem(plant, N, B, seed=seed)
    pr["xu"] = W.perturb(pr["xu"], pr["model"].nq, N, pr["rng"])
    pr["xu"][:, : 2 * pr["model"].nq] = pr["xs"]
    return {k: (np.asarray(v, np.float64) if k in ("xu", "xs", "goal") else v)
            for k, v in pr.items()}


def _solve(O, plant, N, B, pr, **kw):
    P = O.make_params(**dict(dict(dt=0.01, max_sqp_iters=5, pcg_tol=1e-5, max_pcg_iters=173,
                                  rho=1e-3, mu=10.0, q_cost=1.0, u_cost=1e-4, N_cost=10.0), **kw))
    S = O.Solver(plant, N, B, P, threads=2)
    return S.solve(pr["xu"], 0.01, pr["xs"], pr["goal"])


def test_nan_input_flags_only_its_problem(oracle_mod):
    O = oracle_mod
    pr = _problem("iiwa14", 16, 4, 71)
    x_clean, s_clean = _solve(O, "iiwa14", 16, 4, pr)
    assert np.all(s_clean["status"] & NONFINITE == 0)
    assert np.all((s_clean["status"] & CONVERGED != 0) == (s_clean["kkt_converged"] != 0))
    pr["xs"][1, 0] = np.nan
    pr["xu"][1, 0] = np.nan
    x, s = _solve(O, "iiwa14", 16, 4, pr)
    assert s["status"][1] & NONFINITE and s["status"][1] & MAX_ITER
    others = [0, 2, 3]
    assert np.all(s["status"][others] & NONFINITE == 0)
    np.testing.assert_array_equal(x[others], x_clean[others])


def test_iteration_limits_zero(oracle_mod):
    O = oracle_mod
    pr = _problem("indy7", 8, 3, 73)
    x, s = _solve(O, "indy7", 8, 3, pr, max_sqp_iters=0)
    np.testing.assert_array_equal(x, pr["xu"])
    np.testing.assert_array_equal(s["status"], [MAX_ITER] * 3)
    _, s = _solve(O, "indy7", 8, 3, pr, max_pcg_iters=0)
    np.testing.assert_array_equal(s["status"], [CONVERGED | PCG_MAX] * 3)


def test_singular_kkt_is_flagged(oracle_mod):
    O = oracle_mod
    pr = _problem("indy7", 8, 3, 79)
    P = O.make_params(dt=0.01, max_sqp_iters=3, pcg_tol=1e-5, max_pcg_iters=50, q_cost=0.0,
                      qd_cost=0.0, u_cost=0.0, N_cost=0.0, q_lim_cost=0.0, rho=0.0)
    S = O.Solver("indy7", 8, 3, P, threads=2)
    _, s = S.solve(pr["xu"], 0.01, pr["xs"], pr["goal"])
    assert np.all(s["status"] & NONFINITE), s["status"]
