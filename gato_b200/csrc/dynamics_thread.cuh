// Forward dynamics and forward kinematics evaluated by one thread, for the
// sample-parallel kernels (the merit evaluation of every knot at every
// line-search step, sim_forward): 32 samples per warp, no cross-lane work.
//
//   bias      c = RNEA(q, qd, qdd = 0) with gravity and f_ext
//   inertia   M by the composite-rigid-body algorithm; the composite inertia
//             of a subtree is carried as its 10 inertial parameters
//             (mass, first moment h, rotational inertia about the link
//             origin) and moved to the parent frame in closed form
//   solve     qdd = M^-1 (u - c) by Cholesky
// Same quantities as the warp-level code in dynamics.cuh (and the reference's
// forward_dynamics_inner, gato/dynamics/iiwa14/iiwa14_fext.cuh:502-507).
#pragma once

#include "common.cuh"
#include "dynamics.cuh"

namespace gato {

// E = Rz(q)^T E0 and C = Rz(q)^T C0 (row-major) of joint i
template <int NQ, typename T>
__device__ __forceinline__ void thread_joint_ec(const DevModel<NQ, T>& M, int i, T sn, T cs, T* E,
                                                T* C)
{
    const T* E0 = M.E0[i];
    const T* C0 = M.C0[i];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        E[c] = cs * E0[c] + sn * E0[3 + c];
        E[3 + c] = -sn * E0[c] + cs * E0[3 + c];
        E[6 + c] = E0[6 + c];
        C[c] = cs * C0[c] + sn * C0[3 + c];
        C[3 + c] = -sn * C0[c] + cs * C0[3 + c];
        C[6 + c] = C0[6 + c];
    }
}

// qdd = FD(q, qd, u, f_ext) for one sample in one thread.
template <int NQ, typename T>
__device__ __forceinline__ void fd_thread(const DevModel<NQ, T>& M, const T* sn, const T* cs,
                                          const T* qd, const T* u, const T* fext, T* qdd)
{
    // --- RNEA bias forces
    T f[NQ][6];
    {
        T v[6] = {0, 0, 0, 0, 0, 0};
        T a[6] = {0, 0, 0, 0, 0, M.gravity};
#pragma unroll
        for (int i = 0; i < NQ; ++i) {
            T E[9], C[9], vn[6], an[6], t[6];
            thread_joint_ec<NQ, T>(M, i, sn[i], cs[i], E, C);
            x_mul(E, C, v, vn);
            vn[2] += qd[i];
            x_mul(E, C, a, an);
            add_cz(an, vn, qd[i]);
            i_mul(M, i, an, f[i]);
            i_mul(M, i, vn, t);
            add_crf(f[i], vn, t);
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                v[k] = vn[k];
                a[k] = an[k];
            }
        }
        if (fext != nullptr) {
#pragma unroll
            for (int k = 0; k < 6; ++k) f[NQ - 1][k] -= fext[k];
        }
    }
    T rhs[NQ];
#pragma unroll
    for (int i = NQ - 1; i >= 0; --i) {
        rhs[i] = u[i] - f[i][2];
        if (i > 0) {
            T E[9], C[9], t[6];
            thread_joint_ec<NQ, T>(M, i, sn[i], cs[i], E, C);
            xt_mul(E, C, f[i], t);
#pragma unroll
            for (int k = 0; k < 6; ++k) f[i - 1][k] += t[k];
        }
    }
    // --- joint-space inertia by composite rigid bodies (lower triangle)
    T Mm[NQ][NQ];
    T Ib[6], h[3], m;  // composite of the subtree rooted at link i, link-i frame
#pragma unroll
    for (int k = 0; k < 6; ++k) Ib[k] = M.Ibar[NQ - 1][k];
#pragma unroll
    for (int k = 0; k < 3; ++k) h[k] = M.h[NQ - 1][k];
    m = M.mass[NQ - 1];
#pragma unroll
    for (int i = NQ - 1; i >= 0; --i) {
        // F = Ic_i S, S = e_z angular: [Ib col z; -h x e_z]
        T F[6] = {Ib[2], Ib[4], Ib[5], -h[1], h[0], T(0)};
        Mm[i][i] = F[2];
#pragma unroll
        for (int j = i; j > 0; --j) {
            T E[9], C[9], t[6];
            thread_joint_ec<NQ, T>(M, j, sn[j], cs[j], E, C);
            xt_mul(E, C, F, t);
#pragma unroll
            for (int k = 0; k < 6; ++k) F[k] = t[k];
            Mm[i][j - 1] = F[2];
        }
        if (i > 0) {
            // move the composite to the parent frame: R = E^T, p = joint origin
            T E[9], C[9];
            thread_joint_ec<NQ, T>(M, i, sn[i], cs[i], E, C);
            const T* p = M.P[i];
            // Rh = R h = E^T h
            T Rh[3];
#pragma unroll
            for (int r = 0; r < 3; ++r) Rh[r] = E[r] * h[0] + E[3 + r] * h[1] + E[6 + r] * h[2];
            // R Ib R^T with Ib symmetric (xx xy xz yy yz zz)
            const T I3[9] = {Ib[0], Ib[1], Ib[2], Ib[1], Ib[3], Ib[4], Ib[2], Ib[4], Ib[5]};
            T IRt[9];  // Ib * R^T = Ib * E (row-major)
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    IRt[3 * r + c] = I3[3 * r] * E[c] + I3[3 * r + 1] * E[3 + c] + I3[3 * r + 2] * E[6 + c];
            T RIR[9];  // E^T * IRt
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    RIR[3 * r + c] = E[r] * IRt[c] + E[3 + r] * IRt[3 + c] + E[6 + r] * IRt[6 + c];
            // Ī' = R Ī R^T - (Rh)x px - px (Rh)x - m px px ; entries of a x b x:
            // (a x)(b x) = b a^T - (a.b) 1
            const T ab = Rh[0] * p[0] + Rh[1] * p[1] + Rh[2] * p[2];
            const T pp = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
            T Inew[9];
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const T dg = (r == c) ? T(1) : T(0);
                    const T hp = p[r] * Rh[c] - ab * dg;  // (Rh x)(p x)
                    const T ph = Rh[r] * p[c] - ab * dg;  // (p x)(Rh x)
                    const T pq = p[r] * p[c] - pp * dg;   // (p x)(p x)
                    Inew[3 * r + c] = RIR[3 * r + c] - hp - ph - m * pq;
                }
            const int pi = i - 1;
            Ib[0] = Inew[0] + M.Ibar[pi][0];
            Ib[1] = Inew[1] + M.Ibar[pi][1];
            Ib[2] = Inew[2] + M.Ibar[pi][2];
            Ib[3] = Inew[4] + M.Ibar[pi][3];
            Ib[4] = Inew[5] + M.Ibar[pi][4];
            Ib[5] = Inew[8] + M.Ibar[pi][5];
#pragma unroll
            for (int k = 0; k < 3; ++k) h[k] = Rh[k] + m * p[k] + M.h[pi][k];
            m += M.mass[pi];
        }
    }
    // --- Cholesky M = L L^T (in place, lower triangle) and solve
#pragma unroll
    for (int j = 0; j < NQ; ++j) {
        T d = Mm[j][j];
#pragma unroll
        for (int k = 0; k < j; ++k) d -= Mm[j][k] * Mm[j][k];
        const T ljj = sqrt(d);
        const T inv = T(1) / ljj;
        Mm[j][j] = ljj;
#pragma unroll
        for (int i = j + 1; i < NQ; ++i) {
            T t = Mm[i][j];
#pragma unroll
            for (int k = 0; k < j; ++k) t -= Mm[i][k] * Mm[j][k];
            Mm[i][j] = t * inv;
        }
    }
    T y[NQ];
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        T t = rhs[i];
#pragma unroll
        for (int k = 0; k < i; ++k) t -= Mm[i][k] * y[k];
        y[i] = t / Mm[i][i];
    }
#pragma unroll
    for (int i = NQ - 1; i >= 0; --i) {
        T t = y[i];
#pragma unroll
        for (int k = i + 1; k < NQ; ++k) t -= Mm[k][i] * qdd[k];
        qdd[i] = t / Mm[i][i];
    }
}

// End-effector position (origin of the last link frame) in one thread.
template <int NQ, typename T>
__device__ __forceinline__ void fk_thread(const DevModel<NQ, T>& M, const T* sn, const T* cs, T* p)
{
    T R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    T o[3] = {0, 0, 0};
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        const T* R0 = M.R0[i];
        const T* P = M.P[i];
#pragma unroll
        for (int r = 0; r < 3; ++r) o[r] += R[3 * r] * P[0] + R[3 * r + 1] * P[1] + R[3 * r + 2] * P[2];
        if (i == NQ - 1) break;
        T Rj[9];
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            Rj[3 * r] = cs[i] * R0[3 * r] + sn[i] * R0[3 * r + 1];
            Rj[3 * r + 1] = -sn[i] * R0[3 * r] + cs[i] * R0[3 * r + 1];
            Rj[3 * r + 2] = R0[3 * r + 2];
        }
        T Rn[9];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c)
                Rn[3 * r + c] = R[3 * r] * Rj[c] + R[3 * r + 1] * Rj[3 + c] + R[3 * r + 2] * Rj[6 + c];
#pragma unroll
        for (int k = 0; k < 9; ++k) R[k] = Rn[k];
    }
    p[0] = o[0];
    p[1] = o[1];
    p[2] = o[2];
}

// Merit contribution of one knot at one step size, one thread
// (computeMeritBatchedKernel, gato/bsqp/kernels/merit.cuh:34-91):
// tracking cost (iiwa14_plant.cuh:275-327, N_cost at the last knot) plus
// mu times the L1 integrator defect (or |x_0 - x_s|_1 at the last knot).
template <int NQ, typename T>
__device__ __forceinline__ T merit_thread(const DevModel<NQ, T>& M, const CostParams<T>& cp, int N,
                                          int k, T alpha, T mu, const T* __restrict__ xu,
                                          const T* __restrict__ dz, const T* __restrict__ xs,
                                          const T* __restrict__ goal, const T* fext)
{
    constexpr int nx = 2 * NQ, nu = NQ, nxu = nx + nu;
    const bool last = (k == N - 1);
    const T* xk = xu + k * nxu;
    const T* dk = dz ? dz + k * nxu : nullptr;
    T q[NQ], qd[NQ], u[NQ], sn[NQ], cs[NQ];
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        q[i] = xk[i] + (dk ? alpha * dk[i] : T(0));
        qd[i] = xk[NQ + i] + (dk ? alpha * dk[NQ + i] : T(0));
        u[i] = last ? T(0) : xk[nx + i] + (dk ? alpha * dk[nx + i] : T(0));
        gsincos(q[i], &sn[i], &cs[i]);
    }
    T cost = T(0);
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
        cost += T(0.5) * (cp.wdiag ? cp.wdiag[NQ + i] : cp.qd_cost) * qd[i] * qd[i];
        if (cp.wdiag) cost += T(0.5) * cp.wdiag[i] * q[i] * q[i];
        cost += cp.q_lim_cost * barrier(q[i], M.qlo[i], M.qhi[i]);
        cost += cp.vel_lim_cost * barrier(qd[i], M.vlo[i], M.vhi[i]);
        if (!last) {
            cost += T(0.5) * (cp.wdiag ? cp.wdiag[nx + i] : cp.u_cost) * u[i] * u[i];
            cost += cp.ctrl_lim_cost * barrier(u[i], M.ulo[i], M.uhi[i]);
        }
    }
    T p[3];
    fk_thread<NQ, T>(M, sn, cs, p);
    const T w = last ? cp.N_cost : cp.q_cost;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const T e = p[r] - goal[6 * k + r];
        cost += T(0.5) * w * e * e;
    }
    T defect = T(0);
    if (!last) {
        T qdd[NQ];
        fd_thread<NQ, T>(M, sn, cs, qd, u, fext, qdd);
        const T dt = cp.dt;
        const T* xk1 = xk + nxu;
        const T* dk1 = dk ? dk + nxu : nullptr;
#pragma unroll
        for (int i = 0; i < NQ; ++i) {
            const T qn = q[i] + dt * qd[i] + T(0.5) * qdd[i] * dt * dt;
            const T vn = qd[i] + dt * qdd[i];
            const T q1 = xk1[i] + (dk1 ? alpha * dk1[i] : T(0));
            const T v1 = xk1[NQ + i] + (dk1 ? alpha * dk1[NQ + i] : T(0));
            defect += gabs(q1 - qn) + gabs(v1 - vn);
        }
    } else {
#pragma unroll
        for (int i = 0; i < nx; ++i) defect += gabs(xu[i] + (dz ? alpha * dz[i] : T(0)) - xs[i]);
    }
    return cost + mu * defect;
}

}  // namespace gato
