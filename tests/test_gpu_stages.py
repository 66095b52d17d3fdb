"""Stage-level parity of the CUDA kernels with the FP64 oracle, through the
C ABI stage entry points (FP32 device arithmetic)."""
import numpy as np
import pytest

from helpers import create_raw, nerr, problem

pytestmark = pytest.mark.gpu

PARAMS = dict(dt=0.01, max_sqp_iters=5, kkt_tol=1e-4, max_pcg_iters=173, pcg_tol=1e-5,
              solve_ratio=1.0, mu=10.0, q_cost=1.0, qd_cost=1e-4, u_cost=1e-4, N_cost=10.0,
              q_lim_cost=1e-3, vel_lim_cost=1e-4, ctrl_lim_cost=1e-6, rho=1e-3)


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available()
    torch.cuda.set_device(0)
    return torch


def _kkt_gpu(torch, L, h, xu, xs, goal, nq, N, B):
    dev = torch.device("cuda")
    t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device=dev)
    nx, nu = 2 * nq, nq
    out = dict(Q=torch.zeros(B, N, nx * nx, device=dev), R=torch.zeros(B, N, nu * nu, device=dev),
               q=torch.zeros(B, N, nx, device=dev), r=torch.zeros(B, N, nu, device=dev),
               A=torch.zeros(B, N, nx * nx, device=dev), B=torch.zeros(B, N, nx * nu, device=dev),
               c=torch.zeros(B, N, nx, device=dev))
    V = L.vptr
    dxu, dxs, dg = t(xu), t(xs), t(goal)
    L.check(L.load().gato_stage_setup_kkt(h, None, V(dxu), V(dxs), V(dg),
                                          *[V(out[k]) for k in "QRqrABc"]))
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in out.items()}


@pytest.mark.parametrize("plant,fext_on", [("iiwa14", False), ("iiwa14", True),
                                           ("indy7", False), ("indy7", True)])
def test_kkt_blocks_match_oracle(torch_cuda, oracle_mod, plant, fext_on):
    import gato_b200._lib as L
    O = oracle_mod
    N, B = 16, 3
    pr = problem(plant, N, B, seed=3)
    nq = pr["model"].nq
    h = create_raw(L, plant, N, B, PARAMS)
    try:
        rng = np.random.default_rng(5)
        fext = (rng.normal(0, 2, (B, 6)) if fext_on else np.zeros((B, 6))).astype(np.float32)
        L.check(L.load().gato_set_f_ext_batch(h, L.fptr(fext)))
        g = _kkt_gpu(torch_cuda, L, h, pr["xu"], pr["xs"], pr["goal"], nq, N, B)
    finally:
        L.load().gato_destroy(h)
    m = O.Model(plant)
    P = O.make_params(**PARAMS)
    for b in range(B):
        o = m.setup_kkt(N, P, 0.01, pr["xu"][b], pr["xs"][b], pr["goal"][b],
                        fext[b] if fext_on else None)
        for k in "QqAc":
            assert nerr(g[k][b], o[k].reshape(g[k][b].shape)) < 2e-5, k
        for k in "RrB":  # blocks of knots 0..N-2 only
            assert nerr(g[k][b][: N - 1], o[k].reshape(g[k][b].shape)[: N - 1]) < 2e-5, k


@pytest.mark.parametrize("plant,N", [("iiwa14", 8), ("iiwa14", 32), ("indy7", 32)])
def test_schur_and_pcg_match_oracle(torch_cuda, oracle_mod, plant, N):
    import gato_b200._lib as L
    O = oracle_mod
    torch = torch_cuda
    B = 3
    pr = problem(plant, N, B, seed=4)
    nq = pr["model"].nq
    nx, nu = 2 * nq, nq
    m = O.Model(plant)
    P = O.make_params(**PARAMS)
    kkts = [m.setup_kkt(N, P, 0.01, pr["xu"][b], pr["xs"][b], pr["goal"][b]) for b in range(B)]
    dev = torch.device("cuda")
    t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device=dev)
    Q, R, q, r, A, Bm, c = [t(np.stack([k[n] for k in kkts])) for n in "QRqrABc"]
    S = torch.zeros(B, N, 3 * nx * nx, device=dev)
    Pi = torch.zeros_like(S)
    gam = torch.zeros(B, (N + 2) * nx, device=dev)
    lam = torch.zeros(B, (N + 2) * nx, device=dev)
    its = torch.zeros(B, dtype=torch.int32, device=dev)
    V = L.vptr
    h = create_raw(L, plant, N, B, PARAMS)
    try:
        L.check(L.load().gato_stage_form_schur(h, None, V(Q), V(R), V(q), V(r), V(A), V(Bm),
                                               V(c), V(S), V(Pi), V(gam)))
        torch.cuda.synchronize()
        sch = [O.form_schur(nq, N, PARAMS["rho"], k) for k in kkts]
        for b in range(B):
            assert nerr(S[b].cpu().numpy(), sch[b]["S"]) < 1e-5
            assert nerr(Pi[b].cpu().numpy(), sch[b]["Pinv"]) < 1e-5
            assert nerr(gam[b].cpu().numpy(), sch[b]["gamma"]) < 1e-5
            assert nerr(Q[b].cpu().numpy(), sch[b]["Qinv"]) < 1e-5
        # PCG on the oracle's own FP64 Schur system rounded to FP32
        So, Po, go = [t(np.stack([s[n] for s in sch])) for n in ("S", "Pinv", "gamma")]
        L.check(L.load().gato_stage_pcg(h, None, V(So), V(Po), V(go), V(lam), V(its)))
        torch.cuda.synchronize()
    finally:
        L.load().gato_destroy(h)
    for b in range(B):
        lo, io = O.pcg(nq, N, sch[b]["S"], sch[b]["Pinv"], sch[b]["gamma"],
                       np.zeros((N + 2) * nx), 1e-5, 173)
        assert abs(int(its[b]) - io) <= max(2, io // 20), (int(its[b]), io)
        assert nerr(lam[b].cpu().numpy(), lo) < 1e-3


def test_sim_forward_matches_oracle(torch_cuda, oracle_mod):
    import gato_b200
    O = oracle_mod
    B = 4
    rng = np.random.default_rng(7)
    s = gato_b200.BSQP(batch_size=B, N=8, dt=0.01, plant_type="iiwa14")
    fext = rng.normal(0, 3, (B, 6)).astype(np.float32)
    s.set_f_ext_B(fext)
    xk = rng.uniform(-1, 1, 14).astype(np.float32)
    uk = rng.normal(0, 5, 7).astype(np.float32)
    out = s.sim_forward(xk, uk, 0.01)
    s.close()
    m = O.Model("iiwa14")
    for b in range(B):
        qdd = m.fd(xk[:7], xk[7:], uk, fext[b])
        xn = np.concatenate([xk[:7] + 0.01 * xk[7:] + 0.5 * qdd * 1e-4, xk[7:] + 0.01 * qdd])
        assert nerr(out[b], xn) < 1e-5
