"""Generates tests/golden/force_estimator.npz by running the reference's own
force estimator (examples/force_estimator.py, imported from the reference
tree, unmodified) with the settings of python/bsqp/mpc_controller.py:123-134
on a seeded sequence of winners and prediction errors.  Its random rotations
draw from numpy's global generator, seeded here; the fixture records that
seed so that gato_b200.mpc.ForceEstimator can replay the same draws.

Usage: python tests/golden/make_force_estimator_golden.py
"""
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
from build_ref import reference_root  # noqa: E402

B, STEPS, SEED = 12, 40, 7


def main():
    root = reference_root()
    if root is None:
        raise SystemExit("reference tree not found (set GATO_REF)")
    spec = importlib.util.spec_from_file_location(
        "force_estimator", os.path.join(root, "examples", "force_estimator.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    est = mod.ForceEstimator(batch_size=B, initial_radius=5.0, min_radius=2.0, max_radius=20.0,
                             smoothing_factor=0.5)
    rng = np.random.default_rng(2031)
    best = rng.integers(0, B, STEPS)
    errors = rng.uniform(0.01, 1.0, (STEPS, B))
    np.random.seed(SEED)
    batches = [est.generate_batch()]
    radius = []
    for t in range(STEPS):
        est.update(int(best[t]), errors[t], alpha=0.6, beta=0.5)
        batches.append(est.generate_batch())
        radius.append(est.radius)
    np.savez(os.path.join(HERE, "force_estimator.npz"), best=best, errors=errors,
             batches=np.array(batches), radius=np.array(radius), seed=SEED, batch=B)


if __name__ == "__main__":
    main()
