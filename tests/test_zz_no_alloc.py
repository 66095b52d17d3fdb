"""gato_pcg_static (the PCG stage with its scratch in a static device array,
no solver handle, no allocation) against gato_stage_pcg on the same Schur
systems.  Named to be collected last, so it also runs after every other test
in the same process."""
import numpy as np
import pytest

from helpers import create_raw, problem

PARAMS = dict(dt=0.01, max_sqp_iters=1, kkt_tol=1e-4, max_pcg_iters=173, pcg_tol=1e-5,
              solve_ratio=1.0, mu=10.0, q_cost=1.0, qd_cost=1e-4, u_cost=1e-4, N_cost=10.0,
              q_lim_cost=1e-3, vel_lim_cost=1e-4, ctrl_lim_cost=1e-6, rho=1e-3)


def _schur_system(torch, L, h, pr, nq, N, B):
    """S, Pinv, gamma of the perturbed problem batch from the solver's own
    KKT and Schur stages."""
    nx, nu = 2 * nq, nq
    dev = torch.device("cuda")
    t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device=dev)
    V = L.vptr
    z = lambda *shape: torch.zeros(*shape, device=dev)
    Q, R, q, r = z(B, N, nx * nx), z(B, N, nu * nu), z(B, N, nx), z(B, N, nu)
    A, Bm, c = z(B, N, nx * nx), z(B, N, nx * nu), z(B, N, nx)
    S, Pi = z(B, N, 3 * nx * nx), z(B, N, 3 * nx * nx)
    gam = z(B, (N + 2) * nx)
    lib = L.load()
    # inputs held in names: a temporary freed inside the argument list could
    # hand its memory to the next input before the kernel reads it
    d_xu, d_xs, d_goal = t(pr["xu"]), t(pr["xs"]), t(pr["goal"])
    L.check(lib.gato_stage_setup_kkt(h, None, V(d_xu), V(d_xs), V(d_goal),
                                     V(Q), V(R), V(q), V(r), V(A), V(Bm), V(c)))
    torch.cuda.synchronize()
    L.check(lib.gato_stage_form_schur(h, None, V(Q), V(R), V(q), V(r), V(A), V(Bm), V(c),
                                      V(S), V(Pi), V(gam)))
    return S, Pi, gam


@pytest.mark.gpu
@pytest.mark.parametrize("plant,N,B", [("iiwa14", 32, 64), ("indy7", 16, 5)])
def test_pcg_static_matches_stage_pcg(plant, N, B):
    import torch
    import gato_b200._lib as L
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    torch.cuda.set_device(0)
    pr = problem(plant, N, B, seed=11)
    nq = pr["model"].nq
    nx = 2 * nq
    V = L.vptr
    lib = L.load()
    h = create_raw(L, plant, N, B, PARAMS)
    try:
        S, Pi, gam = _schur_system(torch, L, h, pr, nq, N, B)
        lam_ref = torch.zeros(B, (N + 2) * nx, device="cuda")
        its_ref = torch.zeros(B, dtype=torch.int32, device="cuda")
        L.check(lib.gato_stage_pcg(h, None, V(S), V(Pi), V(gam), V(lam_ref), V(its_ref)))
        torch.cuda.synchronize()
    finally:
        lib.gato_destroy(h)
    assert int(its_ref.max()) > 0
    for call in range(2):
        lam = torch.zeros(B, (N + 2) * nx, device="cuda")
        its = torch.full((B,), -1, dtype=torch.int32, device="cuda")
        L.check(lib.gato_pcg_static(None, nq, N, B, PARAMS["pcg_tol"], PARAMS["max_pcg_iters"],
                                    V(S), V(Pi), V(gam), V(lam), V(its)))
        torch.cuda.synchronize()
        # the same kernel on the same data: iteration counts equal, solutions
        # equal to FP32 rounding
        assert torch.equal(its, its_ref), (call, its.tolist(), its_ref.tolist())
        err = float((lam - lam_ref).abs().max()) / max(1.0, float(lam_ref.abs().max()))
        assert err < 1e-6, (call, err)


@pytest.mark.gpu
def test_pcg_static_rejects_oversized_batch():
    import torch
    import gato_b200._lib as L
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    torch.cuda.set_device(0)
    lib = L.load()
    buf = torch.zeros(16, device="cuda")
    rc = lib.gato_pcg_static(None, 7, 32, 8193, 1e-5, 10, L.vptr(buf), L.vptr(buf),
                             L.vptr(buf), L.vptr(buf), L.vptr(buf))
    assert rc == -1
    assert b"static scratch" in lib.gato_last_error()
