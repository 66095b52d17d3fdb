"""ctypes wrappers of the FP64 oracle (liboracle.so) and of the reference's
own dynamics compiled for the host (oracle/_ref/libgrid_ref_<plant>.so).

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py.  The product package (gato_b200) never imports
this module.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
GATO_MAX_NQ = 8

PLANTS = {"iiwa14": 0, "indy7": 1}


class GatoModel(ctypes.Structure):
    """Mirror of gato_model_t (include/gato_b200.h)."""
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
    """Mirror of gato_params_t (include/gato_b200.h)."""
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


PARAM_NAMES = [f[0] for f in GatoParams._fields_]


def make_params(**kw):
    """gato_params_t with the BSQP constructor defaults
    (python/bsqp/interface.py:13-26) unless overridden."""
    d = dict(dt=0.01, max_sqp_iters=10, kkt_tol=1e-4, max_pcg_iters=100, pcg_tol=1e-4,
             solve_ratio=1.0, mu=1.0, q_cost=2.0, qd_cost=1e-4, u_cost=1e-6, N_cost=50.0,
             q_lim_cost=1e-3, vel_lim_cost=0.0, ctrl_lim_cost=0.0, rho=0.0)
    d.update(kw)
    return GatoParams(**d)


def build():
    """Compiles liboracle.so (and oracle/_ref when the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    import sys
    sys.path.insert(0, HERE)
    from build_ref import reference_root
    if reference_root():
        subprocess.run(["python", os.path.join(HERE, "build_ref.py")], check=True,
                       stdout=subprocess.DEVNULL)


def _load():
    if not os.path.exists(LIB):
        build()
    lib = ctypes.CDLL(LIB)
    vp = ctypes.c_void_p
    sig = {
        "orc_builtin_model": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(GatoModel)]),
        "orc_model_create": (vp, [ctypes.POINTER(GatoModel)]),
        "orc_model_destroy": (None, [vp]),
        "orc_rnea": (None, [vp, _dp, _dp, _dp, _dp, _dp]),
        "orc_mass_matrix": (None, [vp, _dp, _dp]),
        "orc_fd": (None, [vp, _dp, _dp, _dp, _dp, _dp]),
        "orc_fd_grad": (None, [vp, _dp, _dp, _dp, _dp, _dp, _dp]),
        "orc_rnea_grad": (None, [vp, _dp, _dp, _dp, _dp, _dp, _dp]),
        "orc_ee_pos": (None, [vp, _dp, _dp, _dp]),
        "orc_tracking_cost": (ctypes.c_double,
                              [vp, ctypes.POINTER(GatoParams), _dp, ctypes.c_int, _dp,
                               ctypes.c_int, _dp]),
        "orc_setup_kkt": (None, [vp, ctypes.c_int, ctypes.POINTER(GatoParams), ctypes.c_double,
                                 _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
        "orc_form_schur": (None, [ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp, _dp, _dp,
                                  _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
        "orc_pcg": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp,
                                   ctypes.c_double, ctypes.c_int]),
        "orc_compute_dz": (None, [ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp, _dp, _dp,
                                  _dp, _dp]),
        "orc_merit": (ctypes.c_double, [vp, ctypes.c_int, ctypes.POINTER(GatoParams),
                                        ctypes.c_double, ctypes.c_double, _dp, _dp,
                                        ctypes.c_double, _dp, _dp, _dp, _dp]),
        "orc_integrate": (None, [ctypes.c_int, _dp, _dp, ctypes.c_double, _dp]),
        "orc_integrator_error": (ctypes.c_double, [vp, _dp, _dp, ctypes.c_double]),
        "orc_set_snap": (None, [ctypes.c_double]),
        "orc_solver_create": (vp, [ctypes.POINTER(GatoModel), ctypes.c_int, ctypes.c_int,
                                   ctypes.POINTER(GatoParams)]),
        "orc_solver_destroy": (None, [vp]),
        "orc_solver_set_threads": (None, [vp, ctypes.c_int]),
        "orc_solver_set_rho": (None, [vp, _dp, ctypes.c_int]),
        "orc_solver_set_drho": (None, [vp, _dp, ctypes.c_int]),
        "orc_solver_set_mu": (None, [vp, _dp]),
        "orc_solver_set_tol": (None, [vp, _dp]),
        "orc_solver_set_fext": (None, [vp, _dp]),
        "orc_solver_set_cost_diag": (None, [vp, _dp]),
        "orc_solver_set_adapt": (None, [vp, ctypes.c_int]),
        "orc_solver_set_round_f32": (None, [vp, ctypes.c_int]),
        "orc_solver_reset_dual": (None, [vp]),
        "orc_solver_reset_rho": (None, [vp]),
        "orc_solver_get_lambda": (None, [vp, _dp]),
        "orc_solver_set_lambda": (None, [vp, _dp]),
        "orc_solver_get_rho": (None, [vp, _dp]),
        "orc_solver_solve": (ctypes.c_int, [vp, ctypes.c_double, _dp, _dp, _dp, _ip, _ip, _dp,
                                            _dp, _ip, _dp, _dp, _dp, _ip]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def _p(a):
    """double* of a C-contiguous float64 array (or NULL for None)."""
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def _ip_(a):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_ip)


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def builtin_model(plant):
    m = GatoModel()
    if lib().orc_builtin_model(PLANTS[plant], ctypes.byref(m)) != 0:
        raise ValueError(plant)
    return m


class Model:
    """FP64 dynamics of one robot (textbook spatial algebra)."""

    def __init__(self, model):
        if isinstance(model, str):
            model = builtin_model(model)
        self.desc = model
        self.nq = model.nq
        self.h = lib().orc_model_create(ctypes.byref(model))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_model_destroy(self.h)
            self.h = None

    def rnea(self, q, qd, qdd=None, fext=None):
        tau = np.zeros(self.nq)
        lib().orc_rnea(self.h, _p(_f64(q)), _p(_f64(qd)), _p(_f64(qdd)), _p(_f64(fext)), _p(tau))
        return tau

    def mass_matrix(self, q):
        M = np.zeros((self.nq, self.nq))
        lib().orc_mass_matrix(self.h, _p(_f64(q)), _p(M))
        return M

    def fd(self, q, qd, u, fext=None):
        qdd = np.zeros(self.nq)
        lib().orc_fd(self.h, _p(_f64(q)), _p(_f64(qd)), _p(_f64(u)), _p(_f64(fext)), _p(qdd))
        return qdd

    def fd_grad(self, q, qd, u, fext=None):
        """(qdd, df_du) with df_du nq x 3nq = [dqdd/dq | dqdd/dqd | Minv]."""
        n = self.nq
        qdd = np.zeros(n)
        df = np.zeros(3 * n * n)
        lib().orc_fd_grad(self.h, _p(_f64(q)), _p(_f64(qd)), _p(_f64(u)), _p(_f64(fext)),
                          _p(qdd), _p(df))
        return qdd, df.reshape(3 * n, n).T.copy()

    def rnea_grad(self, q, qd, qdd, fext=None):
        n = self.nq
        dq = np.zeros((n, n))
        dqd = np.zeros((n, n))
        lib().orc_rnea_grad(self.h, _p(_f64(q)), _p(_f64(qd)), _p(_f64(qdd)), _p(_f64(fext)),
                            _p(dq), _p(dqd))
        return dq, dqd

    def ee_pos(self, q, jac=False):
        p = np.zeros(3)
        J = np.zeros(3 * self.nq) if jac else None
        lib().orc_ee_pos(self.h, _p(_f64(q)), _p(p), _p(J))
        if jac:
            return p, J.reshape(self.nq, 3).T.copy()
        return p

    def tracking_cost(self, params, xu, goal, has_u=True, terminal=False, wdiag=None):
        return lib().orc_tracking_cost(self.h, ctypes.byref(params), _p(_f64(xu)), int(has_u),
                                       _p(_f64(goal)), int(terminal), _p(_f64(wdiag)))

    def setup_kkt(self, N, params, dt, xu, xs, goal, fext=None, wdiag=None):
        """KKT blocks of one problem in the reference's memory layout: square
        and rectangular blocks are column-major, so out["A"][k, c, r] is
        A_k[r, c] (and likewise Q, R, B)."""
        n, m = 2 * self.nq, self.nq
        out = dict(Q=np.zeros((N, n, n)), R=np.zeros((N, m, m)), q=np.zeros((N, n)),
                   r=np.zeros((N, m)), A=np.zeros((N, n, n)), B=np.zeros((N, m, n)),
                   c=np.zeros((N, n)))
        lib().orc_setup_kkt(self.h, N, ctypes.byref(params), dt, _p(_f64(xu)), _p(_f64(xs)),
                            _p(_f64(goal)), _p(_f64(fext)), *[_p(out[k]) for k in "QRqrABc"],
                            _p(_f64(wdiag)))
        return out

    def integrator_error(self, xux, dt, fext=None):
        return lib().orc_integrator_error(self.h, _p(_f64(xux)), _p(_f64(fext)), dt)

    def merit(self, N, params, dt, mu, xu, dz, alpha, xs, goal, fext=None, wdiag=None):
        return lib().orc_merit(self.h, N, ctypes.byref(params), dt, mu, _p(_f64(xu)),
                               _p(_f64(dz)), alpha, _p(_f64(xs)), _p(_f64(goal)), _p(_f64(fext)),
                               _p(_f64(wdiag)))


def form_schur(nq, N, rho, kkt):
    """Returns dict with S, Pinv (N x nx x 3nx row-major), gamma ((N+2)*nx),
    Qinv, Rinv.  kkt arrays as returned by Model.setup_kkt (not modified)."""
    n = 2 * nq
    Q = kkt["Q"].copy()
    R = kkt["R"].copy()
    S = np.zeros((N, n, 3 * n))
    P = np.zeros((N, n, 3 * n))
    g = np.zeros((N + 2) * n)
    lib().orc_form_schur(nq, N, rho, _p(Q), _p(R), _p(_f64(kkt["q"])), _p(_f64(kkt["r"])),
                         _p(_f64(kkt["A"])), _p(_f64(kkt["B"])), _p(_f64(kkt["c"])), _p(S),
                         _p(P), _p(g))
    return dict(S=S, Pinv=P, gamma=g, Qinv=Q, Rinv=R)


def pcg(nq, N, S, Pinv, gamma, lam, eps, max_iters):
    lam = np.ascontiguousarray(lam, dtype=np.float64).copy()
    it = lib().orc_pcg(nq, N, _p(_f64(S)), _p(_f64(Pinv)), _p(_f64(gamma)), _p(lam), eps,
                       max_iters)
    return lam, it


def compute_dz(nq, N, lam, Qinv, Rinv, q, r, A, B):
    n, m = 2 * nq, nq
    qq = np.ascontiguousarray(q, dtype=np.float64).copy()
    rr = np.ascontiguousarray(r, dtype=np.float64).copy()
    dz = np.zeros((n + m) * N - m)
    lib().orc_compute_dz(nq, N, _p(_f64(lam)), _p(_f64(Qinv)), _p(_f64(Rinv)), _p(qq), _p(rr),
                         _p(_f64(A)), _p(_f64(B)), _p(dz))
    return dz, qq, rr


class Solver:
    """Batched FP64 SQP solver with the reference driver's semantics."""

    def __init__(self, model, N, batch, params, threads=1):
        if isinstance(model, str):
            model = builtin_model(model)
        self.nq = model.nq
        self.nx, self.nu = 2 * model.nq, model.nq
        self.N, self.B = N, batch
        self.params = params
        self.traj = (self.nx + self.nu) * N - self.nu
        self.h = lib().orc_solver_create(ctypes.byref(model), N, batch, ctypes.byref(params))
        lib().orc_solver_set_threads(self.h, threads)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_solver_destroy(self.h)
            self.h = None

    def set_threads(self, n):
        lib().orc_solver_set_threads(self.h, int(n))

    def set_rho_penalty_batch(self, rho, set_as_reset_default=True):
        lib().orc_solver_set_rho(self.h, _p(_f64(rho)), int(set_as_reset_default))

    def set_drho_batch(self, v, set_as_reset_default=True):
        lib().orc_solver_set_drho(self.h, _p(_f64(v)), int(set_as_reset_default))

    def set_mu_batch(self, v):
        lib().orc_solver_set_mu(self.h, _p(_f64(v)))

    def set_pcg_tol_batch(self, v):
        lib().orc_solver_set_tol(self.h, _p(_f64(v)))

    def set_f_ext_batch(self, v):
        lib().orc_solver_set_fext(self.h, _p(_f64(np.reshape(v, -1))))

    def set_cost_diag_batch(self, wdiag):
        """Per-problem diagonal weights [B][nx+nu] (None: the scalar weights)."""
        lib().orc_solver_set_cost_diag(
            self.h, None if wdiag is None else _p(_f64(np.reshape(wdiag, -1))))

    def set_rho_adaptation(self, on):
        lib().orc_solver_set_adapt(self.h, int(bool(on)))

    # orc_solver_set_round_f32 flags
    ROUND_KKT, ROUND_SCHUR, ROUND_LAMBDA, ROUND_XU = 1, 2, 4, 8
    ROUND_ALL = 15

    def set_round_f32(self, flags):
        """Rounds the stored stage outputs named by `flags` to FP32 with all
        arithmetic in FP64: the accuracy floor of an ideal FP32 solver
        (0 restores exact FP64)."""
        lib().orc_solver_set_round_f32(self.h, int(flags))

    def reset_dual(self):
        lib().orc_solver_reset_dual(self.h)

    def reset_rho(self):
        lib().orc_solver_reset_rho(self.h)

    def get_lambda(self):
        out = np.zeros((self.B, (self.N + 2) * self.nx))
        lib().orc_solver_get_lambda(self.h, _p(out))
        return out

    def set_lambda(self, lam):
        lib().orc_solver_set_lambda(self.h, _p(_f64(lam)))

    def get_rho(self):
        out = np.zeros(self.B)
        lib().orc_solver_get_rho(self.h, _p(out))
        return out

    def solve(self, xu, dt, xs, goal):
        """Returns (XU float64 [B, traj], stats dict)."""
        B, it = self.B, self.params.max_sqp_iters
        xu = np.ascontiguousarray(xu, dtype=np.float64).reshape(B, self.traj).copy()
        xs = _f64(np.reshape(xs, (B, self.nx)))
        goal = _f64(np.reshape(goal, (B, 6 * self.N)))
        sqp = np.zeros(B, np.int32)
        conv = np.zeros(B, np.int32)
        fm = np.zeros(B)
        im = np.zeros(B)
        pcg_it = np.zeros(max(it, 1) * B, np.int32)
        lsm = np.zeros(max(it, 1) * B)
        lss = np.zeros(max(it, 1) * B)
        secs = ctypes.c_double(0)
        status = np.zeros(B, np.int32)
        n = lib().orc_solver_solve(self.h, dt, _p(xu), _p(xs), _p(goal), _ip_(sqp), _ip_(conv),
                                   _p(fm), _p(im), _ip_(pcg_it), _p(lsm), _p(lss),
                                   ctypes.byref(secs), _ip_(status))
        stats = dict(sqp_iters=sqp, kkt_converged=conv, final_merit=fm, initial_merit=im,
                     ls_num_iters=n, pcg_iters=pcg_it[: n * B].reshape(n, B),
                     ls_min_merit=lsm[: n * B].reshape(n, B),
                     ls_step_size=lss[: n * B].reshape(n, B), seconds=secs.value,
                     status=status)
        return xu, stats


class RefDynamics:
    """The reference's own GRiD dynamics / plant cost / integrator, compiled
    for the host in FP64 (oracle/_ref).  Available only where the build ran."""

    def __init__(self, plant):
        path = os.path.join(REF_DIR, f"libgrid_ref_{plant}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.ref_nq.restype = ctypes.c_int
        L.ref_knot_points.restype = ctypes.c_int
        L.ref_fd.argtypes = [_dp] * 5
        L.ref_fd_grad.argtypes = [_dp] * 6
        L.ref_ee.argtypes = [_dp] * 3
        L.ref_tracking_cost.restype = ctypes.c_double
        L.ref_tracking_cost.argtypes = [_dp, _dp, ctypes.c_int] + [ctypes.c_double] * 7
        L.ref_cost_grad_hess.argtypes = [_dp, _dp] + [ctypes.c_double] * 7 + [_dp] * 4
        L.ref_linearized_dynamics.argtypes = [_dp, _dp, ctypes.c_double, _dp, _dp, _dp]
        L.ref_integrator_error.restype = ctypes.c_double
        L.ref_integrator_error.argtypes = [_dp, _dp, ctypes.c_double]
        self.nq = L.ref_nq()

    def fd(self, q, qd, u, fext=None):
        out = np.zeros(self.nq)
        self.lib.ref_fd(_p(_f64(q)), _p(_f64(qd)), _p(_f64(u)), _p(_f64(fext)), _p(out))
        return out

    def fd_grad(self, q, qd, u, fext=None):
        n = self.nq
        qdd = np.zeros(n)
        df = np.zeros(3 * n * n)
        self.lib.ref_fd_grad(_p(_f64(q)), _p(_f64(qd)), _p(_f64(u)), _p(_f64(fext)), _p(qdd),
                             _p(df))
        return qdd, df.reshape(3 * n, n).T.copy()

    def ee(self, q):
        pose = np.zeros(6)
        grad = np.zeros(6 * self.nq)
        self.lib.ref_ee(_p(_f64(q)), _p(pose), _p(grad))
        return pose, grad.reshape(self.nq, 6).T.copy()

    def tracking_cost(self, params, xu, goal, terminal=False):
        P = params
        return self.lib.ref_tracking_cost(_p(_f64(xu)), _p(_f64(goal)), int(terminal), P.q_cost,
                                          P.qd_cost, P.u_cost, P.N_cost, P.q_lim_cost,
                                          P.vel_lim_cost, P.ctrl_lim_cost)

    def cost_grad_hess(self, params, xu, goal):
        n, m = 2 * self.nq, self.nq
        Q = np.zeros(n * n)
        qv = np.zeros(n)
        R = np.zeros(m * m)
        rv = np.zeros(m)
        P = params
        self.lib.ref_cost_grad_hess(_p(_f64(xu)), _p(_f64(goal)), P.q_cost, P.qd_cost, P.u_cost,
                                    P.N_cost, P.q_lim_cost, P.vel_lim_cost, P.ctrl_lim_cost,
                                    _p(Q), _p(qv), _p(R), _p(rv))
        return Q.reshape(n, n), qv, R.reshape(m, m), rv

    def linearized_dynamics(self, xux, dt, fext=None):
        n, m = 2 * self.nq, self.nq
        A = np.zeros(n * n)
        B = np.zeros(n * m)
        c = np.zeros(n)
        self.lib.ref_linearized_dynamics(_p(_f64(xux)), _p(_f64(fext)), dt, _p(A), _p(B), _p(c))
        return A.reshape(n, n).T.copy(), B.reshape(m, n).T.copy(), c

    def integrator_error(self, xux, dt, fext=None):
        return self.lib.ref_integrator_error(_p(_f64(xux)), _p(_f64(fext)), dt)
