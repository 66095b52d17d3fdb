// Closed-loop receding-horizon rollout (no counterpart in the reference's
// solver; its MPC loop is Python around one solve per step,
// python/bsqp/mpc_controller.py) and its reverse pass.  Every step: solve
// from the current state with the goal window of that step, apply the first
// control plus noise to the same dynamics (the integrator of
// gato/dynamics/integrator.cuh:20-45, as sim_forward), shift the warm start
// by one knot.  The reverse pass chains the step Jacobians of the simulator
// with the adjoint of each step's solve (adjoint.cuh).
#pragma once

#include "kernels.cuh"

namespace gato {

// goal window of step t: goal[b][0, 6N) = goal_traj[b][6t, 6t + 6N)
template <typename T>
__global__ void k_goal_window(const T* __restrict__ goal_traj, int stride, int t, int N, int B,
                              T* __restrict__ goal)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B * 6 * N) return;
    const int b = i / (6 * N), j = i % (6 * N);
    goal[i] = goal_traj[(size_t)b * stride + 6 * t + j];
}

// first state of the warm start := the current state (bsqp.interface.BSQP.solve)
template <typename T>
__global__ void k_set_x0(T* __restrict__ xu, const T* __restrict__ x, int B, int traj, int nx)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B * nx) return;
    xu[(size_t)(i / nx) * traj + i % nx] = x[i];
}

// one simulator step per problem (one warp): u = u_0 + noise,
// x' = trapezoidal step of the forward dynamics
template <int NQ, typename T>
__global__ void k_sim_step(DevModel<NQ, T> M, int B, T dt, const T* __restrict__ x,
                           const T* __restrict__ xu, int traj, const T* __restrict__ noise,
                           const T* fext, int use_fext, T* __restrict__ x_next,
                           T* __restrict__ u_out)
{
    constexpr int nx = 2 * NQ;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);
    const int b = blockIdx.x * (blockDim.x / WARP) + warp_id();
    if (b >= B) return;
    T* s = smem + warp_id() * (DynSmem<NQ>::SIZE + 3 * NQ);
    T* sx = s + DynSmem<NQ>::SIZE;  // q qd u
    const int l = lane_id();
    if (l < nx) sx[l] = x[(size_t)b * nx + l];
    if (l < NQ) {
        const T u = xu[(size_t)b * traj + nx + l] + (noise ? noise[(size_t)b * NQ + l] : T(0));
        sx[nx + l] = u;
        u_out[(size_t)b * NQ + l] = u;
    }
    __syncwarp();
    dyn_load_transforms<NQ, T>(M, sx, s);
    __syncwarp();
    T mc[NQ];
    dyn_forward<NQ, T>(M, s, sx, sx + NQ, sx + nx, use_fext ? fext + 6 * b : nullptr, false, mc);
    if (l < nx) {
        const T* q = sx;
        const T* qd = sx + NQ;
        const T* qdd = s + DynSmem<NQ>::QDD;
        x_next[(size_t)b * nx + l] = l < NQ ? q[l] + dt * qd[l] + T(0.5) * qdd[l] * dt * dt
                                            : qd[l - NQ] + dt * qdd[l - NQ];
    }
}

// warm start shifted by one knot: x_k <- x_{k+1}, u_k <- u_{k+1}, the last
// control and state repeated; then x_0 := the new state.  One CTA per problem.
template <typename T>
__global__ void k_shift(T* __restrict__ xu, const T* __restrict__ x_next, int N, int nx, int nu)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* s = reinterpret_cast<T*>(smem_raw);
    const int b = blockIdx.x, nxu = nx + nu, traj = nxu * N - nu;
    T* p = xu + (size_t)b * traj;
    for (int i = threadIdx.x; i < traj; i += blockDim.x) s[i] = p[i];
    __syncthreads();
    for (int i = threadIdx.x; i < traj; i += blockDim.x) {
        const int k = i / nxu, j = i % nxu;
        T v;
        if (k == 0 && j < nx)
            v = x_next[(size_t)b * nx + j];
        else if (k < N - 2 || (k == N - 2 && j < nx))
            v = s[i + nxu];  // knot k+1
        else
            v = s[i];  // u_{N-2} and x_{N-1} repeat
        p[i] = v;
    }
}

// reverse of one simulator step (one warp per problem): for g = dl/dx',
// gx = A' g and gu = B' g with A = dx'/dx, B = dx'/du at (x, u) (the
// integrator gradient of kkt_knot, integrator.cuh:143-184)
template <int NQ, typename T>
__global__ void k_sim_vjp(DevModel<NQ, T> M, int B, T dt, const T* __restrict__ x,
                          const T* __restrict__ u, const T* __restrict__ g, const T* fext,
                          int use_fext, T* __restrict__ gx, T* __restrict__ gu)
{
    constexpr int nx = 2 * NQ;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);
    const int b = blockIdx.x * (blockDim.x / WARP) + warp_id();
    if (b >= B) return;
    T* s = smem + warp_id() * (DynSmem<NQ>::SIZE + 3 * NQ + nx);
    T* sx = s + DynSmem<NQ>::SIZE;  // q qd u
    T* sg = sx + 3 * NQ;            // g
    const int l = lane_id();
    if (l < nx) {
        sx[l] = x[(size_t)b * nx + l];
        sg[l] = g[(size_t)b * nx + l];
    }
    if (l < NQ) sx[nx + l] = u[(size_t)b * NQ + l];
    __syncwarp();
    const T* q = sx;
    const T* qd = sx + NQ;
    const T* fe = use_fext ? fext + 6 * b : nullptr;
    dyn_load_transforms<NQ, T>(M, q, s);
    __syncwarp();
    T minv_col[NQ];
    dyn_forward<NQ, T>(M, s, q, qd, sx + nx, fe, true, minv_col);
    T qdd[NQ];
#pragma unroll
    for (int i = 0; i < NQ; ++i) qdd[i] = s[DynSmem<NQ>::QDD + i];
    T dtau[NQ];
    rnea_derivative_lane<NQ, T>(M, s, qd, qdd, fe, dtau);
    const T h2 = T(0.5) * dt * dt;
    if (l < nx) {
        // column l of A against g
        T acc = sg[l];
        if (l >= NQ) acc += dt * sg[l - NQ];
#pragma unroll
        for (int r = 0; r < NQ; ++r) {
            T dq = T(0);
#pragma unroll
            for (int t = 0; t < NQ; ++t) dq -= s[DynSmem<NQ>::MINV + t * NQ + r] * dtau[t];
            acc += (h2 * sg[r] + dt * sg[NQ + r]) * dq;
        }
        gx[(size_t)b * nx + l] = acc;
    }
    if (l >= NQ && l < nx) {
        T acc = T(0);
#pragma unroll
        for (int r = 0; r < NQ; ++r) acc += (h2 * sg[r] + dt * sg[NQ + r]) * minv_col[r];
        gu[(size_t)b * NQ + (l - NQ)] = acc;
    }
}

// dl/dXU of the step's solve: the control slot u_0 gets gu, the rest zero
template <typename T>
__global__ void k_scatter_u0(T* __restrict__ dl, const T* __restrict__ gu, int B, int traj,
                             int nx, int nu)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B * traj) return;
    const int b = i / traj, j = i % traj;
    dl[i] = (j >= nx && j < nx + nu) ? gu[(size_t)b * nu + j - nx] : T(0);
}

// gx := gx + a + c (state gradient of the previous step); acc += w
template <typename T>
__global__ void k_add3(T* __restrict__ gx, const T* __restrict__ a, const T* __restrict__ c,
                       int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) gx[i] = gx[i] + a[i] + c[i];
}
template <typename T>
__global__ void k_accum(T* __restrict__ acc, const T* __restrict__ w, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) acc[i] += w[i];
}
// goal-trajectory gradient: window t of problem b += g
template <typename T>
__global__ void k_goal_accum(T* __restrict__ g_traj, const T* __restrict__ g, int stride, int t,
                             int N, int B)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B * 6 * N) return;
    const int b = i / (6 * N), j = i % (6 * N);
    g_traj[(size_t)b * stride + 6 * t + j] += g[i];
}

// ------------------------------------------------------------------ hypotheses
// Batch-hypothesis selection of the reference's MPC loop
// (python/bsqp/mpc_controller.py:295-309 evaluate_best_trajectory, 241-242):
// problem b simulates (x_last, u_last) for one dt under its own wrench
// hypothesis f_ext[b] and scores err[b] = |x_b - x_curr|_2; the smallest
// error wins and its trajectory becomes every problem's warm start.
// One warp per problem; the squared differences are summed in FP64.
template <int NQ, typename T>
__global__ void k_hyp_error(DevModel<NQ, T> M, int B, T dt, const T* __restrict__ x_last,
                            const T* __restrict__ u_last, const T* __restrict__ x_curr,
                            const T* fext, int use_fext, T* __restrict__ err)
{
    constexpr int nx = 2 * NQ;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);
    const int b = blockIdx.x * (blockDim.x / WARP) + warp_id();
    if (b >= B) return;
    T* s = smem + warp_id() * DynSmem<NQ>::SIZE;
    const T* q = x_last;
    const T* qd = x_last + NQ;
    dyn_load_transforms<NQ, T>(M, q, s);
    __syncwarp();
    T mc[NQ];
    dyn_forward<NQ, T>(M, s, q, qd, u_last, use_fext ? fext + 6 * b : nullptr, false, mc);
    const int l = lane_id();
    double d2 = 0.0;
    if (l < nx) {
        T v;
        if (l < NQ)
            v = q[l] + dt * qd[l] + T(0.5) * s[DynSmem<NQ>::QDD + l] * dt * dt;
        else
            v = qd[l - NQ] + dt * s[DynSmem<NQ>::QDD + l - NQ];
        const double d = (double)v - (double)x_curr[l];
        d2 = d * d;
    }
    d2 = warp_sum(d2);
    if (l == 0) err[b] = (T)sqrt(d2);
}

// numpy.argmin order: a NaN counts as the smallest value, ties go to the
// lower index
template <typename T>
__device__ __forceinline__ bool hyp_before(T a, int ia, T b, int ib)
{
    const bool na = isnan((double)a), nb = isnan((double)b);
    if (na != nb) return na;
    if (!na && a != b) return a < b;
    return ia < ib;
}

// one block: best[0] = argmin_b err[b]
template <typename T>
__global__ void k_hyp_argmin(int B, const T* __restrict__ err, int* __restrict__ best)
{
    __shared__ T sv[1024];
    __shared__ int si[1024];
    const int t = threadIdx.x;
    T v = T(0);
    int iv = -1;
    for (int b = t; b < B; b += blockDim.x)
        if (iv < 0 || hyp_before(err[b], b, v, iv)) {
            v = err[b];
            iv = b;
        }
    sv[t] = v;
    si[t] = iv;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (t < w && si[t + w] >= 0 && (si[t] < 0 || hyp_before(sv[t + w], si[t + w], sv[t], si[t]))) {
            sv[t] = sv[t + w];
            si[t] = si[t + w];
        }
        __syncthreads();
    }
    if (t == 0) best[0] = si[0];
}

// every row of xu [B][traj] := row best[0] (the chosen trajectory as the
// warm start of all hypotheses)
template <typename T>
__global__ void k_hyp_broadcast(int B, int traj, const int* __restrict__ best, T* xu)
{
    const int src = best[0];
    const size_t n = (size_t)B * traj;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const int b = (int)(i / traj);
        if (b != src) xu[i] = xu[(size_t)src * traj + i % traj];
    }
}

}  // namespace gato
