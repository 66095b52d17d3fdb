"""One batched solve of the benchmark workload shape in each form, as the
target of `ncu` captures (python -m gato_b200.profile_case --batch 1024).

Launch order: a plain-form solve (k_merit, k_merit_sum, then per SQP
iteration k_kkt, k_schur_inv, k_schur, k_schur_off, k_pcg, k_dz, k_merit,
k_line_search, ...), then a fused-form solve without its CUDA graph
(k_fused_iter, k_check, k_merit, k_line_search per iteration)."""
import argparse

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--batch", type=int, default=1024)
    ap.add_argument("--N", type=int, default=32)
    ap.add_argument("--plant", default="iiwa14")
    ap.add_argument("--iters", type=int, default=2)
    ap.add_argument("--precision", default="fp32")
    a = ap.parse_args()
    import ctypes
    import torch
    import gato_b200
    import gato_b200._lib as L
    from gato_b200 import workloads as W
    torch.cuda.set_device(0)
    pr = W.make_problem(a.plant, a.N, a.batch, seed=5)
    nq = pr["model"].nq
    xu = W.perturb(pr["xu"], nq, a.N, pr["rng"]).astype(np.float32)
    kw = dict(max_sqp_iters=a.iters, pcg_tol=1e-5, max_pcg_iters=173)
    dev = torch.device("cuda")
    T = lambda x: torch.tensor(np.ascontiguousarray(x), dtype=torch.float32, device=dev)
    d_xs, d_goal = T(pr["xs"]), T(pr["goal"])
    for form in ("plain", "fused"):
        s = gato_b200.BSQP(batch_size=a.batch, N=a.N, dt=0.01, plant_type=a.plant, form=form,
                           precision=a.precision, **kw)
        d_xu = T(xu)
        ms = (ctypes.c_double * len(L.KERNELS))()
        n = (ctypes.c_int32 * len(L.KERNELS))()
        L.check(L.load().gato_profile_solve(s._h, None, L.vptr(d_xu), L.vptr(d_xs),
                                            L.vptr(d_goal), ms, n))
        print(form, {L.KERNELS[i]: round(ms[i], 3) for i in range(len(L.KERNELS)) if n[i]})
        s.close()


if __name__ == "__main__":
    main()
