"""gato_b200.compat: stand-ins for the reference's pybind modules
bsqpN{N}_{plant} (python/bindings.cu), imported the way the reference's
interface imports them (python/bsqp/interface.py:43-60)."""
import importlib
import sys
import types

import numpy as np
import pytest

from helpers import problem


def test_module_attributes():
    from gato_b200 import compat
    m = compat.module(32, "iiwa14")
    assert m.KNOT_POINTS == 32
    for k in range(11):
        cls = getattr(m, f"BSQP_{2 ** k}_float")
        assert cls.__name__ == f"BSQP_{2 ** k}_float"
        for meth in ("solve", "set_f_ext_batch", "set_rho_penalty_batch", "set_drho_batch",
                     "set_mu_batch", "set_pcg_tol_batch", "sim_forward", "reset_dual",
                     "reset_rho", "set_rho_adaptation"):
            assert callable(getattr(cls, meth))
    assert not hasattr(m, "BSQP_2048_float")
    with pytest.raises(ValueError):
        compat.module(32, "ur5")


def test_install_resolves_reference_import_path():
    from gato_b200 import compat
    pkg = types.ModuleType("bsqp_ci_pkg")
    pkg.__path__ = []
    sys.modules["bsqp_ci_pkg"] = pkg
    try:
        compat.install(package="bsqp_ci_pkg", knots=(16, 32), plants=("indy7",))
        m = importlib.import_module("bsqp_ci_pkg.bsqpN32_indy7")
        assert m.KNOT_POINTS == 32 and hasattr(m, "BSQP_64_float")
        assert pkg.bsqpN16_indy7.KNOT_POINTS == 16
    finally:
        for k in [k for k in sys.modules if k.startswith("bsqp_ci_pkg")]:
            del sys.modules[k]


@pytest.mark.gpu
def test_compat_solve_matches_interface():
    """The stand-in class with the reference's positional parameters gives
    the same solve as gato_b200.BSQP with the same keyword parameters."""
    import gato_b200
    from gato_b200 import compat
    params = (0.01, 3, 1e-4, 100, 1e-5, 1.0, 10.0, 1.0, 1e-4, 1e-4, 10.0, 1e-3, 0.0, 0.0, 1e-3)
    B, N = 4, 16
    pr = problem("iiwa14", N, B, seed=21)
    m = compat.module(N, "iiwa14")
    a = m.BSQP_4_float(*params).solve(pr["xu"], 0.01, pr["xs"], pr["goal"])
    s = gato_b200.BSQP(batch_size=B, N=N, plant_type="iiwa14",
                       **dict(zip(compat.PARAM_NAMES, params)))
    b = s.solve_raw(pr["xu"], 0.01, pr["xs"], pr["goal"])
    s.close()
    assert set(a) == set(b)
    np.testing.assert_array_equal(a["pcg_iters"], b["pcg_iters"])
    np.testing.assert_array_equal(a["XU"], b["XU"])
    d = m.BSQP_1_float()  # the reference's no-argument constructor defaults
    assert d._s.params.mu == 10.0 and d._s.params.max_sqp_iters == 5
