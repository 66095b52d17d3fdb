"""Mixed batches: problems of several plants and horizons in one solve
(gato_mixed_* in include/gato_b200.h; no counterpart in the reference, which
needs one module call per plant and horizon).

    mx = MixedBSQP([("iiwa14", 32, 512), ("indy7", 128, 256), ...], dt=0.01,
                   precision="mixed", max_sqp_iters=5, ...)
    mx.cls[c].set_rho_penalty_batch(rho)       # per-class setters (a BSQP)
    mx.tune(xu, xs, goal)                      # autotuner (optional)
    mx.solve_device(xu, xs, goal)              # lists of per-class tensors
    mx.stats(c)                                # per-class statistics

Every stage of each SQP iteration is one persistent launch over all classes
fed from a device work queue, and the whole solve is one CUDA graph.
"""
import ctypes

import numpy as np

from . import _lib as L
from .interface import BSQP

PARAM_KEYS = ("max_sqp_iters", "kkt_tol", "max_pcg_iters", "pcg_tol", "solve_ratio", "mu",
              "q_cost", "qd_cost", "u_cost", "N_cost", "q_lim_cost", "vel_lim_cost",
              "ctrl_lim_cost", "rho")
DEFAULTS = dict(max_sqp_iters=10, kkt_tol=1e-4, max_pcg_iters=100, pcg_tol=1e-4,
                solve_ratio=1.0, mu=1.0, q_cost=2.0, qd_cost=1e-4, u_cost=1e-6, N_cost=50.0,
                q_lim_cost=1e-3, vel_lim_cost=0.0, ctrl_lim_cost=0.0, rho=0.0)
# (lanes per knot, problems per CTA, CTAs per SM)
SHAPES = ((16, 1, 2), (16, 1, 4), (16, 2, 2), (16, 2, 4), (32, 1, 2), (32, 1, 4), (32, 2, 2),
          (32, 2, 4))


class MixedBSQP:
    def __init__(self, classes, dt=0.01, precision="mixed", adapt_rho=True, **params):
        kw = dict(DEFAULTS)
        kw.update(params)
        self.params = L.GatoParams(dt=dt, **{k: kw[k] for k in PARAM_KEYS})
        self.classes = [(p, int(n), int(c)) for p, n, c in classes]
        self.precision = precision
        arr = (L.GatoClass * len(self.classes))(
            *[L.GatoClass(L.PLANTS[p], n, c) for p, n, c in self.classes])
        h = ctypes.c_void_p()
        L.check(L.load().gato_mixed_create(arr, len(self.classes), ctypes.byref(self.params),
                                           L.PRECISIONS[precision], ctypes.byref(h)))
        self._h = h
        self.cls = []
        for i, (p, n, c) in enumerate(self.classes):
            ch = ctypes.c_void_p()
            L.check(L.load().gato_mixed_class(h, i, ctypes.byref(ch)))
            self.cls.append(BSQP(batch_size=c, N=n, dt=dt, plant_type=p, precision=precision,
                                 form="fused", adapt_rho=adapt_rho, _handle=ch,
                                 **{k: kw[k] for k in PARAM_KEYS}))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            for s in self.cls:
                s._h = ctypes.c_void_p()
            L.load().gato_mixed_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ptrs(self, ts):
        arr = (ctypes.c_void_p * len(ts))(*[L.vptr(t).value for t in ts])
        return ctypes.cast(arr, ctypes.POINTER(ctypes.c_void_p)), arr

    def solve_device(self, xu, xs, goal, stream=0):
        """Solve in place: xu, xs, goal are lists (one per class) of device
        tensors of the class's shapes and the solver dtype."""
        pa, ka = self._ptrs(xu)
        pb, kb = self._ptrs(xs)
        pc, kc = self._ptrs(goal)
        L.check(L.load().gato_mixed_solve(self._h, ctypes.c_void_p(int(stream)), pa, pb, pc))

    def elapsed_ms(self):
        ms = ctypes.c_float()
        L.check(L.load().gato_mixed_elapsed_ms(self._h, ctypes.byref(ms)))
        return float(ms.value)

    def stats(self, c):
        s = self.cls[c]
        st, bufs = s._stats_struct()
        L.check(L.load().gato_mixed_stats(self._h, c, ctypes.byref(st)))
        n, B = int(st.ls_num_iters), s.batch_size
        return {"sqp_iters": bufs["sqp_iters"], "kkt_converged": bufs["kkt_converged"],
                "pcg_iters": bufs["pcg_iters"][: n * B].reshape(n, B), "ls_num_iters": n,
                "final_merit": bufs["final_merit"], "initial_merit": bufs["initial_merit"],
                "ls_step_size": bufs["ls_step_size"][: n * B].reshape(n, B),
                "status": bufs["status"]}

    def config(self, lanes_per_knot=16, problems_per_block=1, ctas_per_sm=2):
        L.check(L.load().gato_mixed_config(self._h, int(lanes_per_knot), int(problems_per_block),
                                           int(ctas_per_sm)))

    def tune(self, xu, xs, goal, stream=0):
        """Autotuner: times each launch shape on these inputs (state restored
        after every trial), keeps the fastest; returns {shape: ms}."""
        pa, ka = self._ptrs(xu)
        pb, kb = self._ptrs(xs)
        pc, kc = self._ptrs(goal)
        ms = (ctypes.c_float * len(SHAPES))()
        L.check(L.load().gato_mixed_tune(self._h, ctypes.c_void_p(int(stream)), pa, pb, pc, ms))
        return {SHAPES[i]: float(ms[i]) for i in range(len(SHAPES))}
