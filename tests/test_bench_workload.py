"""The bench builds its workload the same way on both arms from that arm's
own robot tables and kinematics: the formulas equal gato_b200.workloads, the
oracle's forward kinematics equals the library's, and the reference arm's
copy is built without importing this library."""
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def test_seeded_problems_match_library_generator():
    import bench
    import gato_b200
    from gato_b200 import workloads as W
    from gato_b200.kinematics import ee_position
    model = gato_b200.builtin_model(bench.PLANT)
    xs, goal, xu, _ = bench.seeded_problems(model.nq, model.q_limit,
                                            lambda q: ee_position(model, q), 6, 2026)
    pr = W.make_problem(bench.PLANT, bench.N, 6, seed=2026, goals="figure8", dt=bench.DT)
    np.testing.assert_array_equal(xs, pr["xs"])
    np.testing.assert_array_equal(goal, pr["goal"])
    np.testing.assert_array_equal(xu, pr["xu"])


def test_oracle_kinematics_match_library():
    import gato_b200
    from gato_b200.kinematics import ee_position
    from oracle import oracle as O
    rng = np.random.default_rng(3)
    for plant in ("iiwa14", "indy7"):
        model = gato_b200.builtin_model(plant)
        m = O.Model(plant)
        q = rng.uniform(-2, 2, (8, model.nq))
        ref = np.stack([m.ee_pos(qq) for qq in q])
        np.testing.assert_allclose(ee_position(model, q), ref, rtol=0, atol=1e-12)


def test_reference_workload_imports_no_library_code():
    code = ("import sys; sys.path.insert(0, %r); import bench; "
            "wl = bench.make_reference_workload(4, 2026, 2); "
            "assert wl['xu'].shape == (4, 665) and wl['lam'].shape == (4, 476); "
            "bad = [m for m in sys.modules if m.startswith('gato_b200')]; "
            "assert not bad, bad; print('ok')" % ROOT)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0 and "ok" in out.stdout, out.stderr[-2000:]
