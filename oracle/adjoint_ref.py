"""Dense FP64 reference of the adjoint of the converged subproblem.

TEST INFRASTRUCTURE ONLY: the checker of gato_adjoint, never part of the
product path.

At a trajectory z the solver's QP (the reference's KKT, setup_kkt.cuh:52-107,
with rho on the q half of Q, linalg.cuh:84-96) is assembled here as a dense
KKT system and solved directly:

    [G  H'] [dz    ]   [-g]          G = blkdiag(Qt_0, R_0, ..., Qt_{N-1})
    [H  0 ] [lambda] = [ c]          H dz = c:  -dx_0 = c_0,
                                                A_k dx_k + B_k du_k - dx_{k+1} = c_{k+1}

(this is the system whose Schur complement S lambda = gamma the PCG solves,
schur_linsys.cuh:54-260).  The differentiated map is theta -> z + dz(theta)
with z fixed; theta = (x_s, goal positions, diagonal weights Qd, Rd).
`adjoint_grad` is the implicit-function gradient by a dense solve of the
transposed system, `fd_grad` central finite differences of the same map.
"""
import numpy as np


def assemble(model, N, params, dt, xu, xs, goal, wdiag, rho):
    """Dense G, g, H, c and the KKT blocks of the QP formed at xu."""
    nq = model.nq
    n, m = 2 * nq, nq
    kkt = model.setup_kkt(N, params, dt, xu, xs, goal, wdiag=wdiag)
    T = (n + m) * N - m
    G = np.zeros((T, T))
    g = np.zeros(T)
    H = np.zeros((N * n, T))
    c = np.zeros(N * n)
    for k in range(N):
        ox = k * (n + m)
        Qk = kkt["Q"][k].T.copy()
        Qk[np.arange(nq), np.arange(nq)] += rho
        G[ox:ox + n, ox:ox + n] = Qk
        g[ox:ox + n] = kkt["q"][k]
        if k < N - 1:
            G[ox + n:ox + n + m, ox + n:ox + n + m] = kkt["R"][k].T
            g[ox + n:ox + n + m] = kkt["r"][k]
    H[0:n, 0:n] = -np.eye(n)
    c[0:n] = kkt["c"][0]
    for k in range(N - 1):
        ox, rr = k * (n + m), (k + 1) * n
        H[rr:rr + n, ox:ox + n] = kkt["A"][k].T
        H[rr:rr + n, ox + n:ox + n + m] = kkt["B"][k].T
        H[rr:rr + n, ox + n + m:ox + 2 * n + m] = -np.eye(n)
        c[rr:rr + n] = kkt["c"][k + 1]
    return dict(G=G, g=g, H=H, c=c, kkt=kkt)


def kkt_matrix(a):
    T, M = a["G"].shape[0], a["H"].shape[0]
    K = np.zeros((T + M, T + M))
    K[:T, :T] = a["G"]
    K[:T, T:] = a["H"].T
    K[T:, :T] = a["H"]
    return K


def qp_step(model, N, params, dt, xu, xs, goal, wdiag, rho):
    """(dz, lambda) of the QP at xu by a dense solve."""
    a = assemble(model, N, params, dt, xu, xs, goal, wdiag, rho)
    T = a["G"].shape[0]
    sol = np.linalg.solve(kkt_matrix(a), np.concatenate([-a["g"], a["c"]]))
    return sol[:T], sol[T:], a


def default_wdiag(nq, params):
    w = np.zeros(3 * nq)
    w[nq:2 * nq] = params.qd_cost
    w[2 * nq:] = params.u_cost
    return w


def adjoint_grad(model, N, params, dt, xu, xs, goal, wdiag, rho, dl):
    """Gradient of l(xu + dz) with dl/dz = dl (a vector of the trajectory
    size) with respect to x_s [n], goal [6N] (rpy zero) and the diagonal
    weights [n + m], by the implicit function theorem with dense solves."""
    nq = model.nq
    n, m = 2 * nq, nq
    if wdiag is None:
        wdiag = default_wdiag(nq, params)
    dz, _, a = qp_step(model, N, params, dt, xu, xs, goal, wdiag, rho)
    T = a["G"].shape[0]
    sol = np.linalg.solve(kkt_matrix(a), np.concatenate([dl, np.zeros(a["H"].shape[0])]))
    v, mu = sol[:T], sol[T:]
    w = params.q_cost
    g_goal = np.zeros(6 * N)
    g_w = np.zeros(n + m)
    for j in range(N):
        kx = j if j < N - 1 else N - 2
        xh = xu[kx * (n + m):kx * (n + m) + n]
        p, J = model.ee_pos(xh[:nq], jac=True)
        ge = J.T @ (p - goal[6 * j:6 * j + 3])
        ox = j * (n + m)
        vq, dq = v[ox:ox + nq], dz[ox:ox + nq]
        Jv, Jd = J @ vq, J @ dq
        g_goal[6 * j:6 * j + 3] = w * (Jv + Jv * (ge @ dq) + (vq @ ge) * Jd)
        g_w[:n] -= v[ox:ox + n] * (xh + dz[ox:ox + n])
        if j < N - 1:
            g_w[n:] -= v[ox + n:ox + n + m] * (xu[ox + n:ox + n + m] + dz[ox + n:ox + n + m])
    return dict(g_xs=-mu[:n], g_goal=g_goal, g_wdiag=g_w, v=v, mu=mu, dz=dz)


def fd_grad(model, N, params, dt, xu, xs, goal, wdiag, rho, dl, h=1e-6):
    """Central finite differences of l(xu + dz(theta)) = dl . (xu + dz(theta))
    with respect to the same parameters."""
    nq = model.nq
    if wdiag is None:
        wdiag = default_wdiag(nq, params)

    def loss(xs_, goal_, w_):
        dz, _, _ = qp_step(model, N, params, dt, xu, xs_, goal_, w_, rho)
        return float(dl @ (xu + dz))

    def central(f, x0):
        out = np.zeros_like(x0)
        for i in range(x0.size):
            e = np.zeros_like(x0)
            e[i] = h
            out[i] = (f(x0 + e) - f(x0 - e)) / (2 * h)
        return out

    g_xs = central(lambda t: loss(t, goal, wdiag), np.array(xs, dtype=np.float64))
    gp = np.array(goal, dtype=np.float64)
    g_goal = np.zeros(6 * N)
    for j in range(N):
        for a_ in range(3):
            e = np.zeros_like(gp)
            e[6 * j + a_] = h
            g_goal[6 * j + a_] = (loss(xs, gp + e, wdiag) - loss(xs, gp - e, wdiag)) / (2 * h)
    g_w = central(lambda t: loss(xs, goal, t), np.array(wdiag, dtype=np.float64))
    return dict(g_xs=g_xs, g_goal=g_goal, g_wdiag=g_w)
