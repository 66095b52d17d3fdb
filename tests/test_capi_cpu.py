"""CPU-only checks of the C ABI library and the host-side code: the library
loads and exports every entry point include/gato_b200.h declares, argument
errors are reported without touching a GPU, and the host helpers agree with
the oracle."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import have_gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gato_b200.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gato_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    import gato_b200._lib as L
    lib = L.load()
    names = header_functions()
    assert len(names) >= 25
    for name in names:
        assert hasattr(lib, name), name
        assert name in L.SIGNATURES, f"{name} missing from the ctypes signature table"


def test_version_and_builtin_models():
    import gato_b200._lib as L
    lib = L.load()
    assert b"sm_100a" in lib.gato_version()
    m = L.builtin_model("iiwa14")
    assert m.nq == 7 and m.barrier_style == 0
    assert m.link_inertial[6][1][0] == pytest.approx(0.057)
    m = L.builtin_model("indy7")
    assert m.nq == 6 and m.barrier_style == 1
    with pytest.raises(ValueError):
        L.builtin_model("ur5")


def test_argument_errors_need_no_gpu():
    import gato_b200
    for kw in [dict(N=1), dict(N=300), dict(batch_size=0), dict(dt=-1.0),
               dict(precision="fp16"), dict(form="other")]:
        args = dict(batch_size=2, N=8, dt=0.01, plant_type="iiwa14")
        args.update(kw)
        with pytest.raises(ValueError):
            gato_b200.BSQP(**args)


def test_extension_entry_points_validate_before_touching_the_gpu():
    """Argument errors of the entry points without a reference counterpart
    come back as GATO_ERR_ARG with a message, before any CUDA call."""
    import ctypes
    import gato_b200._lib as L
    lib = L.load()
    h = ctypes.c_void_p()
    P = L.GatoParams(dt=0.01, max_sqp_iters=1, max_pcg_iters=10, pcg_tol=1e-5, solve_ratio=1.0)
    assert lib.gato_mixed_create(None, 0, ctypes.byref(P), 0, ctypes.byref(h)) == -1
    cls = (L.GatoClass * 9)(*[L.GatoClass(0, 8, 1) for _ in range(9)])
    assert lib.gato_mixed_create(cls, 9, ctypes.byref(P), 0, ctypes.byref(h)) == -1
    assert b"classes" in lib.gato_last_error()
    assert lib.gato_mixed_solve(None, None, None, None, None) == -1
    assert lib.gato_adjoint(None, None, None, None, None, None, None, None, None, 0.0, 0,
                            None) == -1
    assert lib.gato_rollout(None, None, 1, None, None, None, None, None, None, None) == -1
    assert lib.gato_rollout_backward(None, None, 1, None, None, None, None, None, None, None,
                                     None, None, 0.0, 0) == -1
    assert lib.gato_set_cost_diag_batch(None, None) == -1
    buf = ctypes.c_void_p(16)
    assert lib.gato_pcg_static(None, 7, 32, 0, 1e-5, 10, buf, buf, buf, buf, buf) == -1
    assert lib.gato_pcg_static(None, 5, 32, 4, 1e-5, 10, buf, buf, buf, buf, buf) == -3
    assert lib.gato_pcg_static(None, 7, 32, 4, 1e-5, 10, None, buf, buf, buf, buf) == -1


def test_unsupported_joint_count():
    import gato_b200
    import gato_b200._lib as L
    m = L.builtin_model("iiwa14")
    m.nq = 5
    with pytest.raises(ValueError, match="nq=5"):
        gato_b200.BSQP(batch_size=1, N=8, model=m)


@pytest.mark.skipif(have_gpu(), reason="checks the no-GPU failure path")
def test_solver_fails_loudly_without_gpu():
    import gato_b200
    with pytest.raises(ValueError, match="(?i)cuda"):
        gato_b200.BSQP(batch_size=2, N=8, plant_type="iiwa14")


def test_missing_library_fails_loudly(tmp_path):
    import gato_b200._lib as L
    saved = L._lib
    try:
        L._lib = None
        with pytest.raises(OSError, match="no CPU fallback"):
            L.load(str(tmp_path / "missing.so"))
    finally:
        L._lib = saved


def test_kinematics_matches_oracle(oracle_mod):
    from gato_b200 import _lib as L
    from gato_b200.kinematics import ee_position
    rng = np.random.default_rng(0)
    for plant in ["iiwa14", "indy7"]:
        m = L.builtin_model(plant)
        om = oracle_mod.Model(plant)
        for _ in range(5):
            q = rng.uniform(-2, 2, m.nq)
            np.testing.assert_allclose(ee_position(m, q), om.ee_pos(q), atol=1e-12)


def test_workloads_are_seeded_and_shaped():
    from gato_b200 import workloads as W
    a = W.make_problem("iiwa14", 32, 5, seed=3)
    b = W.make_problem("iiwa14", 32, 5, seed=3)
    assert a["xs"].shape == (5, 14) and a["goal"].shape == (5, 192)
    assert a["xu"].shape == (5, 21 * 32 - 7)
    np.testing.assert_array_equal(a["goal"], b["goal"])
    lim = W.limits(a["model"])
    assert np.all(np.abs(a["xs"][:, :7]) <= 0.8 * lim + 1e-6)
    # figure-8 goals stay within the amplitude bound of their centre
    g = a["goal"].reshape(5, 32, 6)
    assert np.all(np.ptp(g[:, :, :3], axis=1) <= 0.6 + 1e-6)
    assert np.all(g[:, :, 3:] == 0)


def test_oracle_solver_batch_semantics(oracle_mod):
    """Host logic of the reference driver, on the oracle: sqp_iters counts
    converged problems too, and a batch stops when every problem converged."""
    O = oracle_mod
    from gato_b200 import workloads as W
    pr = W.make_problem("iiwa14", 8, 3, seed=21, goals="constant")
    P = O.make_params(max_sqp_iters=6, pcg_tol=1e-5, max_pcg_iters=173, q_cost=1.0,
                      u_cost=1e-4, N_cost=10.0, rho=1e-3, mu=10.0)
    S = O.Solver("iiwa14", 8, 3, P, threads=2)
    xu, st = S.solve(pr["xu"].astype(np.float64), 0.01, pr["xs"], pr["goal"])
    assert st["ls_num_iters"] <= 6
    assert np.all(st["sqp_iters"] >= st["ls_num_iters"])
    assert np.all(st["final_merit"] <= st["initial_merit"] + 1e-9)
