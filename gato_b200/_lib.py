"""ctypes binding of libgato_b200.so (include/gato_b200.h).

The CUDA library is the only implementation of the solver: if it cannot be
loaded, importing the solver fails loudly.  There is no CPU fallback.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgato_b200.so")
GATO_MAX_NQ = 8

PLANTS = {"iiwa14": 0, "indy7": 1}
FORMS = {"plain": 0, "fused": 1}
PRECISIONS = {"fp32": 0, "mixed": 1, "fp64": 2}
# per-problem status bits (GATO_STATUS_*)
STATUS = {"converged": 1, "max_iter": 2, "ls_fail": 4, "nonfinite": 8, "pcg_max_iter": 16}
KERNELS = ["kkt", "schur", "pcg", "dz", "merit", "line_search", "fused_iter", "check",
           "merit_sum"]

_fp = ctypes.POINTER(ctypes.c_float)
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)
_vp = ctypes.c_void_p


class GatoError(RuntimeError):
    """A C-ABI call returned an error status."""


class GatoModel(ctypes.Structure):
    _fields_ = [
        ("nq", ctypes.c_int),
        ("joint_xyz", ctypes.c_double * 3 * GATO_MAX_NQ),
        ("joint_rpy", ctypes.c_double * 3 * GATO_MAX_NQ),
        ("link_inertial", ctypes.c_double * 10 * 2 * GATO_MAX_NQ),
        ("q_limit", ctypes.c_double * GATO_MAX_NQ),
        ("qd_limit", ctypes.c_double * GATO_MAX_NQ),
        ("u_limit", ctypes.c_double * GATO_MAX_NQ),
        ("limit_margin", ctypes.c_double),
        ("gravity", ctypes.c_double),
        ("barrier_style", ctypes.c_int),
    ]


class GatoParams(ctypes.Structure):
    _fields_ = [
        ("dt", ctypes.c_double),
        ("max_sqp_iters", ctypes.c_int),
        ("kkt_tol", ctypes.c_double),
        ("max_pcg_iters", ctypes.c_int),
        ("pcg_tol", ctypes.c_double),
        ("solve_ratio", ctypes.c_double),
        ("mu", ctypes.c_double),
        ("q_cost", ctypes.c_double),
        ("qd_cost", ctypes.c_double),
        ("u_cost", ctypes.c_double),
        ("N_cost", ctypes.c_double),
        ("q_lim_cost", ctypes.c_double),
        ("vel_lim_cost", ctypes.c_double),
        ("ctrl_lim_cost", ctypes.c_double),
        ("rho", ctypes.c_double),
    ]


class GatoClass(ctypes.Structure):
    _fields_ = [("plant", ctypes.c_int), ("N", ctypes.c_int), ("count", ctypes.c_int)]


class GatoStats(ctypes.Structure):
    _fields_ = [
        ("sqp_time_us", ctypes.c_double),
        ("ls_num_iters", ctypes.c_int),
        ("sqp_iters", _ip),
        ("kkt_converged", _ip),
        ("final_merit", _fp),
        ("initial_merit", _fp),
        ("pcg_iters", _ip),
        ("ls_min_merit", _fp),
        ("ls_step_size", _fp),
        ("status", _ip),
    ]


# every symbol the header declares, with its signature
SIGNATURES = {
    "gato_last_error": (ctypes.c_char_p, []),
    "gato_version": (ctypes.c_char_p, []),
    "gato_builtin_model": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(GatoModel)]),
    "gato_create": (ctypes.c_int, [ctypes.POINTER(GatoModel), ctypes.c_int, ctypes.c_int,
                                   ctypes.POINTER(GatoParams), ctypes.c_int, ctypes.c_int,
                                   ctypes.POINTER(_vp)]),
    "gato_destroy": (None, [_vp]),
    "gato_sizes": (ctypes.c_int, [_vp, _ip, _ip, _ip, _ip, _ip]),
    "gato_solve": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, ctypes.POINTER(GatoStats)]),
    "gato_solve_host": (ctypes.c_int, [_vp, _fp, ctypes.c_float, _fp, _fp,
                                       ctypes.POINTER(GatoStats)]),
    "gato_solve_f64": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, ctypes.POINTER(GatoStats)]),
    "gato_solve_host_f64": (ctypes.c_int, [_vp, _dp, ctypes.c_double, _dp, _dp,
                                           ctypes.POINTER(GatoStats)]),
    "gato_set_f_ext_batch": (ctypes.c_int, [_vp, _fp]),
    "gato_set_rho_penalty_batch": (ctypes.c_int, [_vp, _fp, ctypes.c_int]),
    "gato_set_drho_batch": (ctypes.c_int, [_vp, _fp, ctypes.c_int]),
    "gato_set_mu_batch": (ctypes.c_int, [_vp, _fp]),
    "gato_set_pcg_tol_batch": (ctypes.c_int, [_vp, _fp]),
    "gato_set_dt": (ctypes.c_int, [_vp, ctypes.c_float]),
    "gato_set_wait_limits": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int]),
    "gato_reset_dual": (ctypes.c_int, [_vp]),
    "gato_reset_rho": (ctypes.c_int, [_vp]),
    "gato_set_rho_adaptation": (ctypes.c_int, [_vp, ctypes.c_int]),
    "gato_get_lambda": (ctypes.c_int, [_vp, _fp]),
    "gato_set_lambda": (ctypes.c_int, [_vp, _fp]),
    "gato_get_lambda_f64": (ctypes.c_int, [_vp, _dp]),
    "gato_set_lambda_f64": (ctypes.c_int, [_vp, _dp]),
    "gato_get_rho": (ctypes.c_int, [_vp, _fp]),
    "gato_sim_forward": (ctypes.c_int, [_vp, _fp, _fp, ctypes.c_float, _fp]),
    "gato_profile_solve": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp,
                                          ctypes.POINTER(ctypes.c_double), _ip]),
    "gato_profile_solve_f64": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp,
                                              ctypes.POINTER(ctypes.c_double), _ip]),
    "gato_stage_setup_kkt": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp] + [_vp] * 7),
    "gato_stage_form_schur": (ctypes.c_int, [_vp, _vp] + [_vp] * 10),
    "gato_stage_pcg": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "gato_set_cost_diag_batch": (ctypes.c_int, [_vp, _vp]),
    "gato_set_cost_diag_batch_f64": (ctypes.c_int, [_vp, _vp]),
    "gato_set_fp32_preconditioner": (ctypes.c_int, [_vp, ctypes.c_int]),
    "gato_rollout": (ctypes.c_int, [_vp, _vp, ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "gato_rollout_backward": (ctypes.c_int, [_vp, _vp, ctypes.c_int, _vp, _vp, _vp, _vp, _vp,
                                             _vp, _vp, _vp, _vp, ctypes.c_double,
                                             ctypes.c_int]),
    "gato_mixed_create": (ctypes.c_int, [ctypes.POINTER(GatoClass), ctypes.c_int,
                                         ctypes.POINTER(GatoParams), ctypes.c_int,
                                         ctypes.POINTER(_vp)]),
    "gato_mixed_destroy": (ctypes.c_int, [_vp]),
    "gato_mixed_class": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(_vp)]),
    "gato_mixed_solve": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp),
                                        ctypes.POINTER(_vp)]),
    "gato_mixed_stats": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(GatoStats)]),
    "gato_mixed_elapsed_ms": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_float)]),
    "gato_mixed_config": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "gato_mixed_tune": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp),
                                       ctypes.POINTER(_vp), ctypes.POINTER(ctypes.c_float)]),
    "gato_adjoint": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                    ctypes.c_double, ctypes.c_int, _vp]),
    "gato_adjoint_f64": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                        ctypes.c_double, ctypes.c_int, _vp]),
    "gato_qp_step": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_double,
                                    ctypes.c_int, _vp]),
    "gato_qp_step_f64": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_double,
                                        ctypes.c_int, _vp]),
    "gato_select_hypothesis": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, ctypes.c_double, _vp,
                                              _vp, _vp]),
    "gato_pcg_static": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_float, ctypes.c_int, _vp, _vp, _vp, _vp, _vp]),
}

_lib = None


def load(path=None):
    """Loads the CUDA library (raises OSError if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise OSError(
            f"{path} not found: build it with `python -m gato_b200.build` "
            "(the solver has no CPU fallback)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc):
    if rc != 0:
        msg = load().gato_last_error().decode(errors="replace")
        raise GatoError(f"gato error {rc}: {msg}")
    return rc


def builtin_model(plant):
    if plant not in PLANTS:
        raise ValueError(f"unknown plant {plant!r}; choose from {sorted(PLANTS)}")
    m = GatoModel()
    check(load().gato_builtin_model(PLANTS[plant], ctypes.byref(m)))
    return m


def fptr(a):
    """float* of a contiguous float32 numpy array or torch tensor."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return ctypes.cast(ctypes.c_void_p(a.data_ptr()), _fp)
    return a.ctypes.data_as(_fp)


def dptr(a):
    """double* of a contiguous float64 numpy array."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return ctypes.cast(ctypes.c_void_p(a.data_ptr()), _dp)
    return a.ctypes.data_as(_dp)


def iptr(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return ctypes.cast(ctypes.c_void_p(a.data_ptr()), _ip)
    return a.ctypes.data_as(_ip)


def vptr(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return ctypes.c_void_p(a.ctypes.data)
