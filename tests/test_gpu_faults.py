"""Failure detection through the C ABI: the per-problem status word and
bounded device waits.  No GPU is faulted: every fault is made on the host
(non-finite inputs, zero cost weights that make the KKT blocks singular,
zero iteration limits) or is a device wait told to give up at once, whose
bulk copies still land before the kernel ends.  The reference flags only
kkt_converged, step_size = -1 and its rho reset
(gato/bsqp/kernels/line_search.cuh:75-81); the status bits of the FP64
solver equal the FP64 oracle's, fault cases included."""
import numpy as np
import pytest

from helpers import PARAMS_CFG2, gpu_solver, oracle_params, problem

pytestmark = pytest.mark.gpu

CONVERGED, MAX_ITER, LS_FAIL, NONFINITE, PCG_MAX = 1, 2, 4, 8, 16


@pytest.fixture(scope="module", autouse=True)
def cuda():
    import torch
    assert torch.cuda.is_available()
    torch.cuda.set_device(0)


def solve_both(O, plant, N, B, params, pr, precision="fp64", form="fused", lam=None):
    s = gpu_solver(plant, N, B, form=form, precision=precision, **params)
    ref = O.Solver(plant, N, B, oracle_params(O, **params), threads=4)
    if lam is not None:
        s.set_lambda(lam)
        ref.set_lambda(lam)
    f = np.float64 if precision == "fp64" else np.float32
    g = s.solve_raw(pr["xu"].astype(f), 0.01, pr["xs"].astype(f), pr["goal"].astype(f))
    s.close()
    xo, so = ref.solve(pr["xu"].astype(np.float64), 0.01, pr["xs"].astype(np.float64),
                       pr["goal"].astype(np.float64))
    return g, so


@pytest.mark.parametrize("form", ["fused", "plain"])
def test_status_equals_oracle(oracle_mod, form):
    pr = problem("iiwa14", 16, 6, seed=41)
    g, so = solve_both(oracle_mod, "iiwa14", 16, 6, PARAMS_CFG2, pr, form=form)
    np.testing.assert_array_equal(g["status"], so["status"])
    conv = g["kkt_converged"] != 0
    assert np.all((g["status"] & CONVERGED != 0) == conv)
    assert np.all((g["status"] & MAX_ITER != 0) == ~conv)


@pytest.mark.parametrize("field,form,precision", [("xs", "fused", "fp32"), ("xs", "plain", "fp32"),
                                                  ("goal", "fused", "fp32"),
                                                  ("xs", "fused", "fp64")])
def test_nonfinite_input_flags_only_its_problem(oracle_mod, field, form, precision):
    """A NaN in one problem's initial state or goals: the solve returns, that
    problem is flagged non-finite, and every other problem's result is the
    clean solve's, bit for bit."""
    plant, N, B, bad = "iiwa14", 32, 8, 3
    pr = problem(plant, N, B, seed=43)
    clean, _ = solve_both(oracle_mod, plant, N, B, PARAMS_CFG2, pr, precision, form)
    pr[field] = pr[field].copy()
    pr[field][bad, 2] = np.nan
    if field == "xs":
        pr["xu"] = pr["xu"].copy()
        pr["xu"][bad, 2] = np.nan
    g, so = solve_both(oracle_mod, plant, N, B, PARAMS_CFG2, pr, precision, form)
    assert g["status"][bad] & NONFINITE, g["status"]
    assert so["status"][bad] & NONFINITE, so["status"]
    others = np.arange(B) != bad
    assert np.all(g["status"][others] & NONFINITE == 0)
    if g["ls_num_iters"] == clean["ls_num_iters"]:
        np.testing.assert_array_equal(g["XU"][others], clean["XU"][others])
    if precision == "fp64":
        np.testing.assert_array_equal(g["status"], so["status"])


def test_zero_costs_singular_kkt(oracle_mod):
    """All cost weights zero: Q and R are zero, their inverses are not
    finite; the solve returns and flags every problem as the oracle does."""
    params = dict(PARAMS_CFG2, q_cost=0.0, qd_cost=0.0, u_cost=0.0, N_cost=0.0,
                  q_lim_cost=0.0, rho=0.0)
    pr = problem("indy7", 8, 4, seed=47)
    g, so = solve_both(oracle_mod, "indy7", 8, 4, params, pr)
    np.testing.assert_array_equal(g["status"], so["status"])
    assert np.all(g["status"] & NONFINITE)
    g32, _ = solve_both(oracle_mod, "indy7", 8, 4, params, pr, precision="fp32")
    assert np.all(g32["status"] & NONFINITE)


def test_zero_sqp_iterations(oracle_mod):
    """max_sqp_iters = 0: no SQP iteration runs, XU is returned unchanged and
    every problem ends not converged."""
    params = dict(PARAMS_CFG2, max_sqp_iters=0)
    pr = problem("iiwa14", 8, 3, seed=53)
    for form in ("fused", "plain"):
        g, so = solve_both(oracle_mod, "iiwa14", 8, 3, params, pr, form=form)
        assert g["ls_num_iters"] == 0
        np.testing.assert_array_equal(g["XU"], pr["xu"].astype(np.float64))
        np.testing.assert_array_equal(g["status"], np.full(3, MAX_ITER))
        np.testing.assert_array_equal(g["status"], so["status"])


def test_zero_pcg_iterations(oracle_mod):
    """max_pcg_iters = 0: every PCG returns after zero iterations, which the
    reference counts as converged (bsqp.cuh:153-156)."""
    params = dict(PARAMS_CFG2, max_pcg_iters=0)
    pr = problem("iiwa14", 8, 3, seed=59)
    g, so = solve_both(oracle_mod, "iiwa14", 8, 3, params, pr)
    np.testing.assert_array_equal(g["status"], so["status"])
    assert np.all(g["status"] & CONVERGED)


@pytest.mark.parametrize("limits", [(0, -1), (-1, 0)])
def test_expired_copy_wait_reports_timeout(limits):
    """The persistent FP32 PCG told to give up at once on its S / P^-1 copy
    (0, -1) or on its step-recovery copy (-1, 0): the solve reports
    GATO_ERR_TIMEOUT, the kernel leaves no copy in flight, and after the
    default bounds are restored the same handle solves exactly as before."""
    import gato_b200
    plant, N, B = "iiwa14", 32, 300
    pr = problem(plant, N, B, seed=61)
    s = gpu_solver(plant, N, B, form="fused", precision="fp32", **PARAMS_CFG2)
    lam0 = s.get_lambda()

    def run():
        s.set_lambda(lam0)
        s.reset_rho()
        return s.solve_raw(pr["xu"], 0.01, pr["xs"], pr["goal"])

    clean = run()
    s.set_wait_limits(*limits)
    with pytest.raises(gato_b200.GatoError, match="error -5"):
        run()
    s.set_wait_limits(-1, -1)
    again = run()
    s.close()
    np.testing.assert_array_equal(again["XU"], clean["XU"])
    np.testing.assert_array_equal(again["pcg_iters"], clean["pcg_iters"])


def test_expired_copy_wait_reports_timeout_fp64():
    """The FP64 PCG (S and P^-1 brought into shared memory by bulk copy) told
    to give up at once on its copy wait: the solve reports GATO_ERR_TIMEOUT,
    the kernel lets the copy land before the CTA ends, and after the default
    bound is restored the same handle solves exactly as before."""
    import gato_b200
    plant, N, B = "iiwa14", 32, 300
    pr = problem(plant, N, B, seed=67)
    s = gpu_solver(plant, N, B, form="fused", precision="fp64", **PARAMS_CFG2)
    lam0 = s.get_lambda()

    def run():
        s.set_lambda(lam0)
        s.reset_rho()
        return s.solve_raw(pr["xu"].astype(np.float64), 0.01, pr["xs"].astype(np.float64),
                           pr["goal"].astype(np.float64))

    clean = run()
    s.set_wait_limits(0, -1)
    with pytest.raises(gato_b200.GatoError, match="error -5"):
        run()
    s.set_wait_limits(-1, -1)
    again = run()
    s.close()
    np.testing.assert_array_equal(again["XU"], clean["XU"])
    np.testing.assert_array_equal(again["pcg_iters"], clean["pcg_iters"])
