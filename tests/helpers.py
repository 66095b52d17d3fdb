"""Shared helpers of the GPU parity tests."""
import ctypes

import numpy as np

PARAMS_CFG1 = dict(max_sqp_iters=1, pcg_tol=1e-5, max_pcg_iters=173, q_cost=1.0, u_cost=1e-4,
                   N_cost=10.0)
PARAMS_CFG2 = dict(max_sqp_iters=5, pcg_tol=1e-5, max_pcg_iters=173, rho=1e-3, mu=10.0,
                   q_cost=1.0, u_cost=1e-4, N_cost=10.0)


def nerr(a, b):
    """max |a - b| / max(1, max |b|)."""
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.max(np.abs(a - b)) / max(1.0, np.max(np.abs(b))))


def oracle_params(O, **kw):
    return O.make_params(dt=0.01, **kw)


def gpu_solver(plant, N, B, form="fused", precision="fp32", **kw):
    import gato_b200
    return gato_b200.BSQP(batch_size=B, N=N, dt=0.01, plant_type=plant, form=form,
                          precision=precision, **kw)


def create_raw(L, plant, N, B, params, form=0, precision=0):
    m = L.builtin_model(plant)
    gp = L.GatoParams(**params)
    h = ctypes.c_void_p()
    L.check(L.load().gato_create(ctypes.byref(m), N, B, ctypes.byref(gp), form, precision,
                                 ctypes.byref(h)))
    return h


def problem(plant, N, B, seed, perturbed=True, goals="figure8"):
    from gato_b200 import workloads as W
    pr = W.make_problem(plant, N, B, seed=seed, goals=goals)
    if perturbed:
        pr["xu"] = W.perturb(pr["xu"], pr["model"].nq, N, pr["rng"]).astype(np.float32)
        pr["xu"][:, : 2 * pr["model"].nq] = pr["xs"]
    return pr
