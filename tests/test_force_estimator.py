"""gato_b200.mpc.ForceEstimator (the host-side update rule of the
batch-hypothesis MPC loop) replays the reference's own estimator
(tests/golden/force_estimator.npz, made by make_force_estimator_golden.py
from examples/force_estimator.py) on the same winners, errors and random
rotations."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


class _GlobalDraws:
    """The draws numpy's global generator gives after numpy.random.seed(s)."""

    def __init__(self, seed):
        self.rs = np.random.RandomState(seed)

    def random(self, n):
        return self.rs.rand(n)


def test_estimator_replays_reference_sequence():
    pytest.importorskip("torch")
    from gato_b200.mpc import ForceEstimator
    g = np.load(os.path.join(HERE, "golden", "force_estimator.npz"))
    est = ForceEstimator(int(g["batch"]), initial_radius=5.0, min_radius=2.0, max_radius=20.0,
                         smoothing_factor=0.5, rng=_GlobalDraws(int(g["seed"])))
    np.testing.assert_allclose(est.generate_batch(), g["batches"][0], rtol=0, atol=1e-6)
    for t in range(len(g["best"])):
        est.update(int(g["best"][t]), g["errors"][t], alpha=0.6, beta=0.5)
        np.testing.assert_allclose(est.radius, g["radius"][t], rtol=1e-6)
        np.testing.assert_allclose(est.generate_batch(), g["batches"][t + 1], rtol=1e-5,
                                   atol=1e-5)
