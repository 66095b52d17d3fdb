"""Solves of generic robots (seeded serial chains, gato_b200.models) on the
GPU reproduce the FP64 oracle built from the same description."""
import numpy as np
import pytest

from helpers import PARAMS_CFG2, nerr

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nq,seed,N", [(7, 11, 16), (6, 12, 32)])
def test_fp64_seeded_chain_solve_reproduces_oracle(oracle_mod, nq, seed, N):
    import torch
    import gato_b200
    from gato_b200 import models
    from gato_b200 import workloads as W
    O = oracle_mod
    torch.cuda.set_device(0)
    m = models.seeded_chain(nq, seed)
    B = 3
    pr = W.make_problem(None, N, B, seed=seed, model=m)
    xu = W.perturb(pr["xu"], nq, N, pr["rng"])
    xu[:, :2 * nq] = pr["xs"]
    s = gato_b200.BSQP(batch_size=B, N=N, dt=0.01, precision="fp64", model=m, **PARAMS_CFG2)
    g = s.solve_raw(xu.astype(np.float64), 0.01, pr["xs"].astype(np.float64),
                    pr["goal"].astype(np.float64))
    s.close()
    om = O.GatoModel.from_buffer_copy(bytes(m))
    ref = O.Solver(om, N, B, O.make_params(dt=0.01, **PARAMS_CFG2))
    xo, so = ref.solve(xu.astype(np.float64), 0.01, pr["xs"], pr["goal"])
    np.testing.assert_array_equal(g["pcg_iters"], so["pcg_iters"])
    assert nerr(g["XU"], xo) < 1e-8
