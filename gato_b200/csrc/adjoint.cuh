// Adjoint of the converged SQP subproblem (no counterpart in the reference).
//
// At a returned trajectory z the solver's QP is
//     min  sum_k 1/2 dx_k' Qt_k dx_k + q_k' dx_k + 1/2 du_k' R_k du_k + r_k' du_k
//     s.t. dx_0 = -c_0,  dx_{k+1} = A_k dx_k + B_k du_k - c_{k+1}
// i.e. K [dz; lambda] = [-g; c] with K = [[G, H'], [H, 0]] symmetric (the
// Schur complement, PCG and step recovery of the forward solve are this
// system, schur_linsys.cuh / pcg.cuh).  For a loss l(z + dz(theta)) the
// adjoint [v; mu] solves K [v; mu] = [dl/dz; 0], which is the forward system
// with q, r replaced by -dl/dx, -dl/du and c by 0, so it runs through the same
// Schur matrices and PCG.  Then
//     dl/dtheta = v' d(-g)/dtheta + mu' dc/dtheta - v' (dG/dtheta) dz.
// Parameters: x_s (c_0 = x_0 - x_s), the goal positions (tracking gradient
// w J'(p - p_goal) and its Hessian w ge ge', ge = J'(p - p_goal)) and the
// diagonal cost weights Qd, Rd (gradient Qd_i x_i, Hessian Qd_i).
#pragma once

#include "kernels.cuh"

namespace gato {

// RHS of the adjoint system, one CTA per problem: q~ = -s dl/dx,
// r~ = -s dl/du with s = 1 / max|dl/dz| (a unit-scaled system), and the
// Schur vector
//     gamma~_0 = -Qi_0 q~_0,
//     gamma~_{k+1} = -Qi_{k+1} q~_{k+1} + A_k Qi_k q~_k + B_k Ri_k r~_k
// (the forward gamma of schur_linsys.cuh:54-210 with c = 0), into
// bt.q, bt.r, bt.gamma.  Shared memory: N*(nx+nu) T.
template <int NQ, typename T>
__global__ void k_adj_rhs(Batch<NQ, T> bt, const T* __restrict__ dl, T* __restrict__ scale)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int nx = Dims<NQ>::nx, nu = Dims<NQ>::nu, nxu = nx + nu;
    const int b = blockIdx.x, N = bt.N, tid = threadIdx.x, nt = blockDim.x;
    const Dims<NQ> d{N};
    T* a = reinterpret_cast<T*>(smem_raw);  // Qi_k q~_k  [N][nx]
    T* bb = a + N * nx;                     // Ri_k r~_k  [N][nu]
    __shared__ T red[32];
    const T* g = dl + (size_t)b * d.traj();
    T mx = T(0);
    for (int i = tid; i < d.traj(); i += nt) mx = gmax(mx, gabs(g[i]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = gmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane_id() == 0) red[warp_id()] = mx;
    __syncthreads();
    if (tid == 0) {
        T m = T(0);
        for (int w = 0; w < nt / WARP; ++w) m = gmax(m, red[w]);
        red[0] = m > T(0) ? T(1) / m : T(1);
        scale[b] = red[0];
    }
    __syncthreads();
    const T sc = red[0];
    T* qt = bt.q + (size_t)b * N * nx;
    T* rt = bt.r + (size_t)b * N * nu;
    for (int i = tid; i < N * nx; i += nt) qt[i] = -sc * g[(i / nx) * nxu + i % nx];
    for (int i = tid; i < N * nu; i += nt) {
        const int k = i / nu;
        rt[i] = k < N - 1 ? -sc * g[k * nxu + nx + i % nu] : T(0);
    }
    __syncthreads();
    const T* Qi = bt.Qi + (size_t)b * N * nx * nx;
    const T* Ri = bt.Ri + (size_t)b * N * nu * nu;
    for (int i = tid; i < N * nx; i += nt) {
        const int k = i / nx, r = i % nx;
        const T* Qk = Qi + (size_t)k * nx * nx;
        T s = T(0);
#pragma unroll
        for (int t = 0; t < nx; ++t) s += Qk[t * nx + r] * qt[k * nx + t];
        a[i] = s;
    }
    for (int i = tid; i < N * nu; i += nt) {
        const int k = i / nu, r = i % nu;
        T s = T(0);
        if (k < N - 1) {
            const T* Rk = Ri + (size_t)k * nu * nu;
#pragma unroll
            for (int t = 0; t < nu; ++t) s += Rk[t * nu + r] * rt[k * nu + t];
        }
        bb[i] = s;
    }
    __syncthreads();
    T* gam = bt.gamma + (size_t)b * d.vecp();
    const T* A = bt.A + (size_t)b * N * nx * nx;
    const T* Bm = bt.Bm + (size_t)b * N * nx * nu;
    for (int i = tid; i < d.vecp(); i += nt) {
        const int blk = i / nx, r = i % nx;
        T v = T(0);
        if (blk >= 1 && blk <= N) {
            const int j = blk - 1;
            v = -a[j * nx + r];
            if (j > 0) {
                const int k = j - 1;
                const T* Ak = A + (size_t)k * nx * nx;
                const T* Bk = Bm + (size_t)k * nx * nu;
#pragma unroll
                for (int t = 0; t < nx; ++t) v += Ak[t * nx + r] * a[k * nx + t];
#pragma unroll
                for (int t = 0; t < nu; ++t) v += Bk[t * nx + r] * bb[k * nu + t];
            }
        }
        gam[i] = v;
    }
}

// Parameter gradients from the adjoint (v, mu) and the forward QP step dz at
// the returned trajectory, one CTA per problem, one warp per KKT block.
// Block j's cost terms are evaluated at x_j (j <= N-2) and, for the terminal
// block j = N-1, at x_{N-2} against goal N-1 (the KKT's terminal-block rule).
// Outputs per problem: g_xs [nx], g_goal [6N] (rpy entries zero),
// g_wdiag [nx+nu] (Qd then Rd).  Shared memory:
// warps * (DynSmem + nx) T + warps * (nx+nu) T.
template <int NQ, typename T>
__global__ void k_adj_grad(Batch<NQ, T> bt, DevModel<NQ, T> M, const T* __restrict__ scale,
                           const T* __restrict__ v, const T* __restrict__ mu,
                           T* __restrict__ g_xs, T* __restrict__ g_goal,
                           T* __restrict__ g_wdiag)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int nx = Dims<NQ>::nx, nu = Dims<NQ>::nu, nxu = nx + nu;
    constexpr int WS = DynSmem<NQ>::SIZE + nx;
    const int b = blockIdx.x, N = bt.N, l = lane_id(), w = warp_id();
    const int nw = blockDim.x / WARP;
    const Dims<NQ> d{N};
    T* ws = reinterpret_cast<T*>(smem_raw) + w * WS;
    T* acc = reinterpret_cast<T*>(smem_raw) + nw * WS;  // [nw][nxu]
    const T inv = T(1) / scale[b];
    const T* xu = bt.xu + (size_t)b * d.traj();
    const T* vb = v + (size_t)b * d.traj();
    const T* dz = bt.dz + (size_t)b * d.traj();
    const T* goal = bt.goal + (size_t)b * d.goal();
    T* gg = g_goal + (size_t)b * d.goal();
    const T wq = bt.cp.q_cost;
    T aw = T(0);  // this lane's share of the diagonal-weight gradient
    for (int j = w; j < N; j += nw) {
        const int kx = j < N - 1 ? j : N - 2;  // knot the block's cost is evaluated at
        const T* xh = xu + kx * nxu;
        T* qs = ws + DynSmem<NQ>::SIZE;
        if (l < nx) qs[l] = xh[l];
        __syncwarp();
        dyn_load_transforms<NQ, T>(M, qs, ws);
        __syncwarp();
        T p[3], J[3] = {T(0), T(0), T(0)};
        fk_lane<NQ, T>(M, ws, p, J);
        const T* gj = goal + 6 * j;
        const T e0 = p[0] - gj[0], e1 = p[1] - gj[1], e2 = p[2] - gj[2];
        T vq = T(0), dq = T(0), ge = T(0);
        if (l < NQ) {
            vq = vb[j * nxu + l];
            dq = dz[j * nxu + l];
            ge = J[0] * e0 + J[1] * e1 + J[2] * e2;
        }
        const T vg = warp_sum(vq * ge);
        const T dg = warp_sum(dq * ge);
        T Jv[3], Jd[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            Jv[a] = warp_sum(l < NQ ? J[a] * vq : T(0));
            Jd[a] = warp_sum(l < NQ ? J[a] * dq : T(0));
        }
        if (l < 6) {
            T gv = T(0);
            if (l < 3) gv = wq * (Jv[l] + Jv[l] * dg + vg * Jd[l]) * inv;
            gg[6 * j + l] = gv;
        }
        // diagonal weights: -v_i (xhat_i + dz_i) on the state, -v_u (u + du) on the control
        if (l < nx) aw -= vb[j * nxu + l] * (xh[l] + dz[j * nxu + l]);
        if (l >= nx && l < nxu && j < N - 1)
            aw -= vb[j * nxu + l] * (xu[j * nxu + l] + dz[j * nxu + l]);
        __syncwarp();
    }
    if (l < nxu) acc[w * nxu + l] = aw;
    __syncthreads();
    if (threadIdx.x < nxu) {
        T s = T(0);
        for (int i = 0; i < nw; ++i) s += acc[i * nxu + threadIdx.x];
        g_wdiag[(size_t)b * nxu + threadIdx.x] = s * inv;
    }
    if (threadIdx.x < nx)
        g_xs[(size_t)b * nx + threadIdx.x] = -mu[(size_t)b * d.vecp() + nx + threadIdx.x] * inv;
}

}  // namespace gato
