"""Stand-ins for the reference's compiled pybind11 modules.

The reference's Python layer (python/bsqp/interface.py:43-60) imports a
module `bsqp.bsqpN{N}_{plant}` per horizon and plant (python/bindings.cu:
PYBIND11_MODULE) and instantiates its class `BSQP_{B}_float` per power-of-two
batch size with the 15 positional solver parameters.  `module(N, plant)`
builds a Python module with the same attributes (`KNOT_POINTS`,
`BSQP_{1..1024}_float`) whose classes run on gato_b200's C ABI, and
`install()` registers such modules under the reference's package name, so
that the reference's unmodified interface imports them.

The classes keep the pybind classes' methods, argument order and results
(python/bindings.cu:68-237): `solve(xu, dt, x_s, ref) -> dict`,
`set_f_ext_batch`, `set_rho_penalty_batch(rho, set_as_reset_default=True)`,
`set_drho_batch`, `set_mu_batch`, `set_pcg_tol_batch`,
`sim_forward(xk, uk, dt)`, `reset_dual`, `reset_rho`,
`set_rho_adaptation`.
"""
import sys
import types

from .interface import BSQP

# BSQP<T,B>() defaults (gato/bsqp/bsqp.cuh:25-27), used by the pybind
# classes' no-argument constructor
DEFAULT_PARAMS = (0.01, 5, 1e-4, 100, 1e-5, 1.0, 10.0, 1.0, 1e-3, 1e-6, 50.0, 1e-3, 0.0, 0.0,
                  1e-3)
PARAM_NAMES = ("dt", "max_sqp_iters", "kkt_tol", "max_pcg_iters", "pcg_tol", "solve_ratio", "mu",
               "q_cost", "qd_cost", "u_cost", "N_cost", "q_lim_cost", "vel_lim_cost",
               "ctrl_lim_cost", "rho")
BATCH_SIZES = tuple(2 ** k for k in range(11))  # 1 ... 1024, as the reference registers
KNOTS = (8, 16, 32, 64, 128)
PLANTS = ("indy7", "iiwa14")


def _solver_class(N, plant, B, form, precision):
    class Solver:
        """PyBSQP<float, B> of bsqpN{N}_{plant} on gato_b200."""

        def __init__(self, *params):
            if params and len(params) != len(PARAM_NAMES):
                raise TypeError(f"expected 0 or {len(PARAM_NAMES)} arguments, got {len(params)}")
            kw = dict(zip(PARAM_NAMES, params or DEFAULT_PARAMS))
            kw["max_sqp_iters"] = int(kw["max_sqp_iters"])
            kw["max_pcg_iters"] = int(kw["max_pcg_iters"])
            self._s = BSQP(batch_size=B, N=N, plant_type=plant, form=form, precision=precision,
                           **kw)

        def solve(self, xu_traj_batch, timestep, x_s_batch, reference_traj_batch):
            return self._s.solve_raw(xu_traj_batch, timestep, x_s_batch, reference_traj_batch)

        def set_f_ext_batch(self, f_ext_batch):
            self._s.set_f_ext_batch(f_ext_batch)

        def set_rho_penalty_batch(self, rho_batch, set_as_reset_default=True):
            self._s.set_rho_penalty_batch(rho_batch, set_as_reset_default)

        def set_drho_batch(self, drho_batch, set_as_reset_default=True):
            self._s.set_drho_batch(drho_batch, set_as_reset_default)

        def set_mu_batch(self, mu_batch):
            self._s.set_mu_batch(mu_batch)

        def set_pcg_tol_batch(self, eps_batch):
            self._s.set_pcg_tol_batch(eps_batch)

        def sim_forward(self, xk, uk, dt):
            return self._s.sim_forward(xk, uk, dt)

        def reset_dual(self):
            self._s.reset_dual()

        def reset_rho(self):
            self._s.reset_rho()

        def set_rho_adaptation(self, enabled):
            self._s.set_rho_adaptation(enabled)

    Solver.__name__ = Solver.__qualname__ = f"BSQP_{B}_float"
    return Solver


def module(N, plant, name=None, form="fused", precision="fp32"):
    """A module with the attributes of the reference's bsqpN{N}_{plant}."""
    if plant not in PLANTS:
        raise ValueError(f"unknown plant {plant!r}")
    m = types.ModuleType(name or f"bsqpN{N}_{plant}")
    m.KNOT_POINTS = int(N)
    for B in BATCH_SIZES:
        setattr(m, f"BSQP_{B}_float", _solver_class(int(N), plant, B, form, precision))
    return m


def install(package="bsqp", knots=KNOTS, plants=PLANTS, form="fused", precision="fp32"):
    """Registers `{package}.bsqpN{N}_{plant}` for every horizon and plant in
    sys.modules (and as attributes of the package when it is imported), so
    that `importlib.import_module(f"{package}.bsqpN{N}_{plant}")` returns the
    gato_b200-backed module."""
    pkg = sys.modules.get(package)
    for plant in plants:
        for N in knots:
            full = f"{package}.bsqpN{N}_{plant}"
            m = module(N, plant, full, form, precision)
            sys.modules[full] = m
            if pkg is not None:
                setattr(pkg, f"bsqpN{N}_{plant}", m)
