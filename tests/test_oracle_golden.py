"""The FP64 oracle against golden fixtures produced by the reference's own
dynamics, plant cost and integrator code (tests/golden/make_golden.py runs
oracle/_ref/libgrid_ref_<plant>.so, the reference compiled for the host)."""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def load(plant):
    return np.load(os.path.join(GOLD, f"ref_dynamics_{plant}.npz"))


@pytest.mark.parametrize("plant", ["iiwa14", "indy7"])
def test_dynamics_match_reference(oracle_mod, plant):
    O = oracle_mod
    g = load(plant)
    m = O.Model(plant)
    for i in range(len(g["q"])):
        f = g["fext"][i] if g["has_fext"][i] else None
        qdd, df = m.fd_grad(g["q"][i], g["qd"][i], g["u"][i], f)
        np.testing.assert_allclose(qdd, g["qdd"][i], rtol=1e-8, atol=1e-8)
        np.testing.assert_allclose(df, g["df_du"][i], rtol=1e-7, atol=1e-7)
        np.testing.assert_allclose(m.fd(g["q"][i], g["qd"][i], g["u"][i], f), g["qdd"][i],
                                   rtol=1e-8, atol=1e-8)
        p, J = m.ee_pos(g["q"][i], jac=True)
        np.testing.assert_allclose(p, g["ee_pose"][i][:3], atol=1e-12)
        np.testing.assert_allclose(J, g["ee_grad"][i][:3], atol=1e-12)


@pytest.mark.parametrize("plant", ["iiwa14", "indy7"])
def test_cost_and_integrator_match_reference(oracle_mod, plant):
    O = oracle_mod
    g = load(plant)
    m = O.Model(plant)
    nq = m.nq
    nx = 2 * nq
    dt = float(g["dt"])
    for i in range(len(g["q"])):
        w = g["weights"][i]
        P = O.make_params(q_cost=w[0], qd_cost=w[1], u_cost=w[2], N_cost=w[3], q_lim_cost=w[4],
                          vel_lim_cost=w[5], ctrl_lim_cost=w[6])
        xu = np.concatenate([g["q"][i], g["qd"][i], g["u"][i]])
        f = g["fext"][i] if g["has_fext"][i] else None
        assert m.tracking_cost(P, xu, g["goal"][i], True, False) == pytest.approx(
            g["cost"][i], rel=1e-10, abs=1e-12)
        assert m.tracking_cost(P, xu[:nx], g["goal"][i], False, True) == pytest.approx(
            g["cost_terminal"][i], rel=1e-10, abs=1e-12)
        # a 2-knot KKT setup evaluates knot 0's cost blocks and linearisation
        xu2 = np.concatenate([xu, g["xnext"][i]])
        goal2 = np.concatenate([g["goal"][i], g["goal1"][i]])
        kkt = m.setup_kkt(2, P, dt, xu2, np.zeros(nx), goal2, f)
        np.testing.assert_allclose(kkt["Q"][0].T, g["Q"][i], rtol=1e-9, atol=1e-9)
        np.testing.assert_allclose(kkt["q"][0], g["qv"][i], rtol=1e-9, atol=1e-9)
        np.testing.assert_allclose(kkt["R"][0].T, g["R"][i], rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(kkt["r"][0], g["rv"][i], rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(kkt["A"][0].T, g["A"][i], rtol=1e-8, atol=1e-9)
        np.testing.assert_allclose(kkt["B"][0].T, g["B"][i], rtol=1e-8, atol=1e-9)
        np.testing.assert_allclose(kkt["c"][1], g["c"][i], rtol=1e-8, atol=1e-9)
        assert m.integrator_error(xu2, dt, f) == pytest.approx(g["int_err"][i], rel=1e-8)


def test_reference_build_matches_fixtures_when_present(oracle_mod):
    """Where oracle/_ref was built (the reference tree was present), the
    fixtures reproduce from it exactly."""
    O = oracle_mod
    for plant in ["iiwa14", "indy7"]:
        try:
            ref = O.RefDynamics(plant)
        except FileNotFoundError:
            pytest.skip("oracle/_ref not built here")
        g = load(plant)
        qdd, df = ref.fd_grad(g["q"][0], g["qd"][0], g["u"][0])
        if not g["has_fext"][0]:
            np.testing.assert_array_equal(qdd, g["qdd"][0])


def test_fp32_storage_floor_option(oracle_mod):
    """orc_solver_set_round_f32: with no flags the solve is the exact FP64
    solve, bit for bit; with every flag the stored stage outputs are FP32
    values and the result moves by a small, nonzero amount.  The Schur
    system's rounding dominates the floor (XU rounding alone moves far
    less)."""
    O = oracle_mod
    from gato_b200 import workloads as W
    N, B = 32, 8
    pr = W.make_problem("iiwa14", N, B, seed=19)
    xu = W.perturb(pr["xu"], 7, N, pr["rng"]).astype(np.float64)
    xu[:, :14] = pr["xs"]
    P = O.make_params(dt=0.01, max_sqp_iters=5, pcg_tol=1e-5, max_pcg_iters=173)
    outs = {}
    for name, flags in (("exact", None), ("zero", 0), ("all", O.Solver.ROUND_ALL),
                        ("xu", O.Solver.ROUND_XU)):
        S = O.Solver("iiwa14", N, B, P, threads=2)
        if flags is not None:
            S.set_round_f32(flags)
        outs[name] = S.solve(xu, 0.01, pr["xs"], pr["goal"])[0]
    np.testing.assert_array_equal(outs["exact"], outs["zero"])
    err = lambda a: np.abs(a - outs["exact"]).max(1) / np.maximum(1, np.abs(outs["exact"]).max(1))
    e_all, e_xu = err(outs["all"]), err(outs["xu"])
    assert np.all(e_all > 0) and np.median(e_all) < 1e-2, e_all
    assert np.median(e_xu) < np.median(e_all), (e_xu, e_all)
    # every XU value of the all-rounded solve is a float32 value
    np.testing.assert_array_equal(outs["all"], outs["all"].astype(np.float32).astype(np.float64))
