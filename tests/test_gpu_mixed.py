"""Mixed batches (gato_mixed_*): every class of a mixed solve gives the same
result as the same class solved alone by the fused form, in FP64 (where the
fused form reproduces the oracle) and in FP32 for every launch shape of the
autotuner."""
import numpy as np
import pytest

from helpers import PARAMS_CFG2, nerr, problem

pytestmark = pytest.mark.gpu

CLASSES = [("iiwa14", 8, 3), ("indy7", 32, 4), ("iiwa14", 64, 2), ("indy7", 16, 5)]


def _inputs(torch, dt, seed):
    data = []
    for i, (plant, N, B) in enumerate(CLASSES):
        pr = problem(plant, N, B, seed=seed + i)
        data.append(pr)
    T = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")
    return data, T


def _alone(plant, N, B, pr, precision, T):
    import gato_b200
    s = gato_b200.BSQP(batch_size=B, N=N, dt=0.01, plant_type=plant, precision=precision,
                       form="fused", **PARAMS_CFG2)
    xu = T(pr["xu"])
    st = s.solve_device(xu, T(pr["xs"]), T(pr["goal"]))
    out = xu.cpu().numpy(), st["pcg_iters"], s.get_lambda()
    s.close()
    return out


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_mixed_solve_matches_classes_solved_alone(precision):
    import torch
    from gato_b200.mixed import MixedBSQP
    torch.cuda.set_device(0)
    dt = torch.float64 if precision == "fp64" else torch.float32
    data, T = _inputs(torch, dt, 50)
    mx = MixedBSQP(CLASSES, precision=precision, **PARAMS_CFG2)
    from gato_b200.mixed import SHAPES
    shapes = [(16, 1, 2)] if precision == "fp64" else list(SHAPES)
    for kg, ppb, occ in shapes:
        for c in mx.cls:
            c.reset_dual()
            c.reset_rho()
        mx.config(kg, ppb, occ)
        xu = [T(pr["xu"]) for pr in data]
        xs, goal = [T(pr["xs"]) for pr in data], [T(pr["goal"]) for pr in data]
        mx.solve_device(xu, xs, goal)
        torch.cuda.synchronize()
        for c, ((plant, N, B), pr) in enumerate(zip(CLASSES, data)):
            ref_xu, ref_pcg, ref_lam = _alone(plant, N, B, pr, precision, T)
            st = mx.stats(c)
            if precision == "fp64":
                np.testing.assert_array_equal(st["pcg_iters"], ref_pcg)
                assert nerr(xu[c].cpu().numpy(), ref_xu) < 1e-10
            else:
                # the same kernels on the same data; KG=32 evaluates the KKT
                # with one knot per warp, which rounds alike but not bitwise
                assert np.mean(st["pcg_iters"] == ref_pcg) >= 0.75, (kg, ppb, c)
                assert nerr(xu[c].cpu().numpy(), ref_xu) < 5e-3, (kg, ppb, c)
    mx.close()


def test_mixed_tuner_picks_a_shape_and_restores_state():
    import torch
    from gato_b200.mixed import MixedBSQP, SHAPES
    torch.cuda.set_device(0)
    data, T = _inputs(torch, torch.float32, 60)
    mx = MixedBSQP(CLASSES, precision="fp32", **PARAMS_CFG2)
    xu = [T(pr["xu"]) for pr in data]
    xs = [T(pr["xs"]) for pr in data]
    goal = [T(pr["goal"]) for pr in data]
    before = [x.clone() for x in xu]
    lam0 = [c.get_lambda().copy() for c in mx.cls]
    times = mx.tune(xu, xs, goal)
    assert set(times) == set(SHAPES) and all(t > 0 for t in times.values())
    for a, b in zip(xu, before):
        assert torch.equal(a, b)
    for c, l in zip(mx.cls, lam0):
        np.testing.assert_array_equal(c.get_lambda(), l)
    mx.solve_device(xu, xs, goal)
    assert mx.elapsed_ms() > 0
    mx.close()


ORACLE_CLASSES = [("indy7", 128, 3), ("iiwa14", 64, 2), ("iiwa14", 32, 3), ("indy7", 8, 4)]


def test_fp64_mixed_solve_reproduces_oracle(oracle_mod):
    """One FP64 mixed solve over four classes, the N = 128 class (cluster
    PCG on a parallel graph branch) among them: every class reproduces the
    FP64 oracle run on the same problems (iteration counts, line-search
    steps, status, trajectories to 1e-8; 1e-5 for the cluster class)."""
    import torch
    from gato_b200.mixed import MixedBSQP
    torch.cuda.set_device(0)
    O = oracle_mod
    T = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    data = [problem(plant, N, B, seed=80 + i) for i, (plant, N, B) in enumerate(ORACLE_CLASSES)]
    mx = MixedBSQP(ORACLE_CLASSES, precision="fp64", **PARAMS_CFG2)
    xu = [T(pr["xu"]) for pr in data]
    xs, goal = [T(pr["xs"]) for pr in data], [T(pr["goal"]) for pr in data]
    mx.solve_device(xu, xs, goal)
    torch.cuda.synchronize()
    for c, ((plant, N, B), pr) in enumerate(zip(ORACLE_CLASSES, data)):
        ref = O.Solver(plant, N, B, O.make_params(dt=0.01, **PARAMS_CFG2), threads=4)
        xo, so = ref.solve(pr["xu"].astype(np.float64), 0.01, pr["xs"], pr["goal"])
        st = mx.stats(c)
        np.testing.assert_array_equal(st["pcg_iters"], so["pcg_iters"])
        np.testing.assert_array_equal(st["ls_step_size"], so["ls_step_size"].astype(np.float32))
        np.testing.assert_array_equal(st["status"], so["status"])
        # the N = 128 class sums its PCG inner products per CTA of the
        # cluster, then across CTAs: with equal iteration counts and steps,
        # that summation order alone moves its trajectories by ~1e-6, and the
        # class solved alone by the fused form (the same cluster PCG) gives
        # the mixed solve's result bit for bit
        assert nerr(xu[c].cpu().numpy(), xo) < (1e-5 if N > 64 else 1e-8), (plant, N)
        if N > 64:
            xa, pa, _ = _alone(plant, N, B, pr, "fp64", T)
            np.testing.assert_array_equal(xa, xu[c].cpu().numpy())
            np.testing.assert_array_equal(pa, st["pcg_iters"])
    mx.close()
