"""Drop-in replacement of the reference's Python solver class
(python/bsqp/interface.py:6-237) over the B200 C ABI.

Differences a caller may notice:
  * N and batch_size are runtime values (the reference imports one compiled
    module per N and one class per power-of-two batch size).
  * pinocchio is not needed: nq/nv come from the built-in robot tables
    (`plant_type`), and `ee_pos` evaluates the same forward kinematics the
    solver uses.  `model_path` is accepted for signature compatibility and, if
    given without `plant_type`, only used to pick the plant by name as the
    reference does (interface.py:37-41).
  * `form` ("fused" or "plain") and `precision` ("fp32", "mixed" or "fp64")
    select the B200 execution form; all follow the same SQP method.  "fp64"
    corresponds to the reference's USE_DOUBLES build (double arrays in/out).
"""
import ctypes

import numpy as np

from . import _lib as L


class BSQP:
    def __init__(
        self,
        model_path=None,
        batch_size=1,
        N=32,
        dt=0.01,
        max_sqp_iters=10,
        kkt_tol=1e-4,
        max_pcg_iters=100,
        pcg_tol=1e-4,
        solve_ratio=1.0,
        mu=1.0,
        q_cost=2.0,
        qd_cost=1e-4,
        u_cost=1e-6,
        N_cost=50.0,
        q_lim_cost=1e-3,
        vel_lim_cost=0.0,
        ctrl_lim_cost=0.0,
        rho=0.0,
        rho_batch=None,
        mu_batch=None,
        pcg_tol_batch=None,
        adapt_rho=True,
        plant_type="indy7",
        form="fused",
        precision="fp32",
        model=None,
        _handle=None,
    ):
        if plant_type is None:
            plant_type = "iiwa14" if (model_path and "iiwa" in model_path.lower()) else "indy7"
        lib = L.load()
        self.plant_type = plant_type
        self._model = model if model is not None else L.builtin_model(plant_type)
        self.params = L.GatoParams(
            dt=dt, max_sqp_iters=max_sqp_iters, kkt_tol=kkt_tol, max_pcg_iters=max_pcg_iters,
            pcg_tol=pcg_tol, solve_ratio=solve_ratio, mu=mu, q_cost=q_cost, qd_cost=qd_cost,
            u_cost=u_cost, N_cost=N_cost, q_lim_cost=q_lim_cost, vel_lim_cost=vel_lim_cost,
            ctrl_lim_cost=ctrl_lim_cost, rho=rho)
        if form not in L.FORMS:
            raise ValueError(f"unknown form {form!r}")
        if precision not in L.PRECISIONS:
            raise ValueError(f"unknown precision {precision!r}")
        h = ctypes.c_void_p()
        self._owned = _handle is None
        if _handle is not None:  # a solver owned by a mixed batch (gato_mixed_class)
            h = _handle
        else:
            try:
                L.check(lib.gato_create(ctypes.byref(self._model), int(N), int(batch_size),
                                        ctypes.byref(self.params), L.FORMS[form],
                                        L.PRECISIONS[precision], ctypes.byref(h)))
            except L.GatoError as e:
                raise ValueError(str(e)) from e
        self._h = h
        self.batch_size = int(batch_size)
        self.N = int(N)
        self.dt = dt
        self.form = form
        self.precision = precision
        self.nq = self._model.nq
        self.nv = self.nq
        self.nx = 2 * self.nq
        self.nu = self.nq
        self.traj_size = self.N * (self.nx + self.nu) - self.nu
        self.f_ext_B = np.zeros((self.batch_size, 6), dtype=np.float32)
        self.set_f_ext_B(self.f_ext_B)
        self.XU_B = np.zeros((self.batch_size, self.traj_size), dtype=np.float32)
        self.stats = {
            "sqp_time_us": np.array([]),
            "sqp_iters": np.array([]),
            "kkt_converged": np.array([]),
            "pcg_iters": np.array([]),
            "pcg_times_us": np.array([]),
            "min_merit": np.array([]),
            "step_size": np.array([]),
            "initial_merit": np.array([]),
            "best_initial_merit": np.array([]),
        }
        if rho_batch is not None:
            self.set_rho_penalty_batch(rho_batch, True)
        self.set_rho_adaptation(bool(adapt_rho))
        if mu_batch is not None:
            self.set_mu_batch(mu_batch)
        if pcg_tol_batch is not None:
            self.set_pcg_tol_batch(pcg_tol_batch)

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            if getattr(self, "_owned", True):
                L.load().gato_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- solve --------------------------------------------------------------
    def _stats_struct(self):
        B, it = self.batch_size, max(1, self.params.max_sqp_iters)
        bufs = dict(
            sqp_iters=np.zeros(B, np.int32), kkt_converged=np.zeros(B, np.int32),
            final_merit=np.zeros(B, np.float32), initial_merit=np.zeros(B, np.float32),
            pcg_iters=np.zeros(it * B, np.int32), ls_min_merit=np.zeros(it * B, np.float32),
            ls_step_size=np.zeros(it * B, np.float32), status=np.zeros(B, np.int32))
        st = L.GatoStats(
            0.0, 0, L.iptr(bufs["sqp_iters"]), L.iptr(bufs["kkt_converged"]),
            L.fptr(bufs["final_merit"]), L.fptr(bufs["initial_merit"]),
            L.iptr(bufs["pcg_iters"]), L.fptr(bufs["ls_min_merit"]),
            L.fptr(bufs["ls_step_size"]), L.iptr(bufs["status"]))
        return st, bufs

    def solve_raw(self, xu, dt, x_s, reference_traj):
        """PyBSQP::solve (python/bindings.cu:68-148): host arrays in (float32,
        or float64 for precision="fp64"), the reference's result dict out."""
        B = self.batch_size
        f64 = self.precision == "fp64"
        dt_ = np.float64 if f64 else np.float32
        xu = np.ascontiguousarray(xu, dtype=dt_).reshape(B, self.traj_size).copy()
        x_s = np.ascontiguousarray(x_s, dtype=dt_).reshape(B, self.nx)
        ref = np.ascontiguousarray(reference_traj, dtype=dt_).reshape(B, 6 * self.N)
        st, bufs = self._stats_struct()
        if f64:
            L.check(L.load().gato_solve_host_f64(self._h, L.dptr(xu), float(dt), L.dptr(x_s),
                                                 L.dptr(ref), ctypes.byref(st)))
        else:
            L.check(L.load().gato_solve_host(self._h, L.fptr(xu), float(dt), L.fptr(x_s),
                                             L.fptr(ref), ctypes.byref(st)))
        n = int(st.ls_num_iters)
        return {
            "XU": xu,
            "sqp_time_us": float(st.sqp_time_us),
            "sqp_iters": bufs["sqp_iters"],
            "kkt_converged": bufs["kkt_converged"],
            "final_merit": bufs["final_merit"],
            "initial_merit": bufs["initial_merit"],
            "ls_num_iters": n,
            "pcg_times_us": np.zeros(n, np.float32),
            "pcg_iters": bufs["pcg_iters"][: n * B].reshape(n, B),
            "ls_min_merit": bufs["ls_min_merit"][: n * B].reshape(n, B),
            "ls_step_size": bufs["ls_step_size"][: n * B].reshape(n, B),
            "status": bufs["status"],
        }

    def solve(self, xcur_B, eepos_goals_B, XU_B=None):
        """interface.BSQP.solve (python/bsqp/interface.py:122-210)."""
        dt_ = np.float64 if self.precision == "fp64" else np.float32
        xcur_B = np.asarray(xcur_B, dtype=dt_)
        eepos_goals_B = np.asarray(eepos_goals_B, dtype=dt_)
        if XU_B is None:
            XU_B = self.XU_B.astype(dt_)
        else:
            XU_B = np.array(XU_B, dtype=dt_)
        XU_B = XU_B.reshape(self.batch_size, self.traj_size)
        XU_B[:, : self.nx] = xcur_B
        result = self.solve_raw(XU_B, self.dt, xcur_B, eepos_goals_B)
        self.XU_B = np.asarray(result["XU"], dtype=dt_)
        s = self.stats
        s["sqp_time_us"] = int(result["sqp_time_us"])
        s["sqp_iters"] = result["sqp_iters"].reshape(self.batch_size)
        s["kkt_converged"] = result["kkt_converged"].reshape(self.batch_size)
        s["final_merit"] = result["final_merit"].reshape(self.batch_size)
        s["initial_merit"] = result["initial_merit"].reshape(self.batch_size)
        s["best_initial_merit"] = float(np.min(s["initial_merit"])) if s["initial_merit"].size \
            else np.array([], dtype=np.float32)
        s["ls_num_iters"] = int(result["ls_num_iters"])
        s["pcg_iters"] = result["pcg_iters"]
        s["pcg_times_us"] = result["pcg_times_us"]
        s["min_merit"] = result["ls_min_merit"]
        s["step_size"] = result["ls_step_size"]
        s["status"] = result["status"]
        mm = s["min_merit"]
        if mm.size and mm.ndim == 2:
            best = np.min(mm.astype(np.float32), axis=1)
            s["best_merit_per_iter"] = best
            s["best_merit_iter1"] = float(best[0]) if best.size else float("nan")
        else:
            s["best_merit_per_iter"] = np.array([], dtype=np.float32)
            s["best_merit_iter1"] = float("nan")
        denom = s["best_initial_merit"]
        if np.size(denom) and denom and s["best_merit_per_iter"].size:
            s["best_merit_per_iter_normalized"] = s["best_merit_per_iter"] / float(denom)
        else:
            s["best_merit_per_iter_normalized"] = s["best_merit_per_iter"]
        return self.XU_B, result["sqp_time_us"]

    def solve_device(self, d_xu, d_xs, d_goal, stream=0, with_stats=True):
        """Solves on device buffers (torch CUDA tensors or raw pointers),
        stream-ordered; returns the stats dict (or None)."""
        st, bufs = self._stats_struct() if with_stats else (None, None)
        fn = L.load().gato_solve_f64 if self.precision == "fp64" else L.load().gato_solve
        L.check(fn(self._h, ctypes.c_void_p(int(stream)), L.vptr(d_xu), L.vptr(d_xs),
                   L.vptr(d_goal), ctypes.byref(st) if st is not None else None))
        if st is None:
            return None
        n, B = int(st.ls_num_iters), self.batch_size
        return {
            "sqp_time_us": float(st.sqp_time_us), "ls_num_iters": n,
            "sqp_iters": bufs["sqp_iters"], "kkt_converged": bufs["kkt_converged"],
            "final_merit": bufs["final_merit"], "initial_merit": bufs["initial_merit"],
            "pcg_iters": bufs["pcg_iters"][: n * B].reshape(n, B),
            "ls_min_merit": bufs["ls_min_merit"][: n * B].reshape(n, B),
            "ls_step_size": bufs["ls_step_size"][: n * B].reshape(n, B),
            "status": bufs["status"],
        }

    def adjoint_device(self, d_xu, d_xs, d_goal, d_dl, stream=0, tol=0.0, max_iters=0,
                       with_iters=False):
        """Gradients of a loss of the returned trajectory d_xu (torch CUDA
        tensors of the solver's dtype) through the QP at d_xu:
        (g_xs [B, nx], g_goal [B, 6N], g_wdiag [B, nx+nu]) from dl/dXU
        [B, traj] (gato_adjoint).  with_iters also returns the PCG iteration
        counts [2, B] (forward QP step, adjoint)."""
        import torch
        B, dev = self.batch_size, d_xu.device
        dt = torch.float64 if self.precision == "fp64" else torch.float32
        g_xs = torch.empty((B, self.nx), dtype=dt, device=dev)
        g_goal = torch.empty((B, 6 * self.N), dtype=dt, device=dev)
        g_w = torch.empty((B, self.nx + self.nu), dtype=dt, device=dev)
        its = np.zeros((2, B), np.int32) if with_iters else None
        fn = L.load().gato_adjoint_f64 if self.precision == "fp64" else L.load().gato_adjoint
        L.check(fn(self._h, ctypes.c_void_p(int(stream)), L.vptr(d_xu), L.vptr(d_xs),
                   L.vptr(d_goal), L.vptr(d_dl), L.vptr(g_xs), L.vptr(g_goal), L.vptr(g_w),
                   float(tol), int(max_iters), L.vptr(its)))
        if with_iters:
            return g_xs, g_goal, g_w, its
        return g_xs, g_goal, g_w

    # -- reference helpers -----------------------------------------------
    def ee_pos(self, q):
        """End-effector position of the last link frame (the quantity the
        tracking cost uses; interface.py:212-214 computes it with pinocchio)."""
        from .kinematics import ee_position
        return ee_position(self._model, np.asarray(q, dtype=np.float64))

    def reset(self):
        self.reset_dual()
        self.set_f_ext_B(np.zeros((self.batch_size, 6)))
        self.XU_B = np.zeros((self.batch_size, self.traj_size), dtype=np.float32)

    def sim_forward(self, xk, uk, sim_dt):
        xk = np.ascontiguousarray(xk, dtype=np.float32).reshape(self.nx)
        uk = np.ascontiguousarray(uk, dtype=np.float32).reshape(self.nu)
        out = np.zeros((self.batch_size, self.nx), dtype=np.float32)
        L.check(L.load().gato_sim_forward(self._h, L.fptr(xk), L.fptr(uk), float(sim_dt),
                                          L.fptr(out)))
        return out

    def set_f_ext_B(self, f_ext_B):
        self.f_ext_B = np.ascontiguousarray(f_ext_B, dtype=np.float32).reshape(self.batch_size, 6)
        L.check(L.load().gato_set_f_ext_batch(self._h, L.fptr(self.f_ext_B)))

    set_f_ext_batch = set_f_ext_B

    def _batch_arr(self, v):
        return np.ascontiguousarray(v, dtype=np.float32).reshape(self.batch_size)

    def set_rho_penalty_batch(self, rho_batch, set_as_reset_default=True):
        a = self._batch_arr(rho_batch)
        L.check(L.load().gato_set_rho_penalty_batch(self._h, L.fptr(a), int(set_as_reset_default)))

    def set_drho_batch(self, drho_batch, set_as_reset_default=True):
        a = self._batch_arr(drho_batch)
        L.check(L.load().gato_set_drho_batch(self._h, L.fptr(a), int(set_as_reset_default)))

    def set_mu_batch(self, mu_batch):
        a = self._batch_arr(mu_batch)
        L.check(L.load().gato_set_mu_batch(self._h, L.fptr(a)))

    def set_pcg_tol_batch(self, tol_batch):
        a = self._batch_arr(tol_batch)
        L.check(L.load().gato_set_pcg_tol_batch(self._h, L.fptr(a)))

    def set_cost_diag_batch(self, q_diag=None, r_diag=None):
        """Per-problem diagonal weights: q_diag [B, nx] on the state, r_diag
        [B, nu] on the control (the stage cost gains 1/2 Qd_i x_i^2 and
        1/2 Rd_i u_i^2 in place of the scalar qd_cost and u_cost terms).
        Both None returns to the scalar weights.  FP64 solvers keep them in
        FP64, the others round them to float.  No counterpart in the
        reference; these are the Q/R diagonals the adjoint differentiates."""
        if q_diag is None and r_diag is None:
            self._wdiag = None
            L.check(L.load().gato_set_cost_diag_batch(self._h, None))
            return
        B = self.batch_size
        f = np.float64 if self.precision == "fp64" else np.float32
        qd = np.broadcast_to(np.asarray(q_diag, f), (B, self.nx))
        rd = np.broadcast_to(np.asarray(r_diag, f), (B, self.nu))
        self._wdiag = np.ascontiguousarray(np.concatenate([qd, rd], axis=1), dtype=f)
        if f is np.float64:
            L.check(L.load().gato_set_cost_diag_batch_f64(self._h, L.dptr(self._wdiag)))
        else:
            L.check(L.load().gato_set_cost_diag_batch(self._h, L.fptr(self._wdiag)))

    def default_cost_diag(self):
        """(q_diag, r_diag) equal to the scalar weights: [0, qd_cost] and
        u_cost."""
        B, nq = self.batch_size, self.nq
        qd = np.zeros((B, self.nx), np.float32)
        qd[:, nq:] = self.params.qd_cost
        rd = np.full((B, self.nu), self.params.u_cost, np.float32)
        return qd, rd

    def set_fp32_preconditioner(self, enabled=True):
        """FP64 solvers: apply P^-1 in FP32 inside the FP64 PCG
        (gato_set_fp32_preconditioner); S, residuals, inner products and the
        recurrence stay FP64."""
        L.check(L.load().gato_set_fp32_preconditioner(self._h, int(bool(enabled))))

    def set_wait_limits(self, copy_tries=-1, step_copy_tries=-1):
        """Bounds of the persistent PCG's device waits for its bulk copies
        (gato_set_wait_limits): -1 restores the default, 0 gives up at once
        (the next solve then raises GatoError with GATO_ERR_TIMEOUT)."""
        L.check(L.load().gato_set_wait_limits(self._h, int(copy_tries), int(step_copy_tries)))

    def set_rho_adaptation(self, enabled):
        L.check(L.load().gato_set_rho_adaptation(self._h, int(bool(enabled))))

    def reset_rho(self):
        L.check(L.load().gato_reset_rho(self._h))

    def reset_dual(self):
        L.check(L.load().gato_reset_dual(self._h))

    def get_lambda(self):
        """The persistent dual warm start [B, (N+2)*nx] (float64 for fp64)."""
        shape = (self.batch_size, (self.N + 2) * self.nx)
        if self.precision == "fp64":
            out = np.zeros(shape, dtype=np.float64)
            L.check(L.load().gato_get_lambda_f64(self._h, L.dptr(out)))
            return out
        out = np.zeros(shape, dtype=np.float32)
        L.check(L.load().gato_get_lambda(self._h, L.fptr(out)))
        return out

    def set_lambda(self, lam):
        if self.precision == "fp64":
            a = np.ascontiguousarray(lam, dtype=np.float64).reshape(self.batch_size, -1)
            L.check(L.load().gato_set_lambda_f64(self._h, L.dptr(a)))
            return
        a = np.ascontiguousarray(lam, dtype=np.float32).reshape(self.batch_size, -1)
        L.check(L.load().gato_set_lambda(self._h, L.fptr(a)))

    def get_rho(self):
        out = np.zeros(self.batch_size, dtype=np.float32)
        L.check(L.load().gato_get_rho(self._h, L.fptr(out)))
        return out

    def get_stats(self):
        return self.stats
