// Batched kernels of the SQP solve.
//
// Plain form: one launch per stage with the reference's data flow through
// global memory (gato/bsqp/kernels/*.cuh).  Fused form: one block per problem
// runs KKT set-up -> Schur -> PCG -> step recovery without leaving the SM,
// with S and P^-1 resident in shared memory, and a second block-per-problem
// kernel runs the merit evaluation and line search; convergence bookkeeping
// stays on the device so that a whole solve is one CUDA graph.
#pragma once

#include <type_traits>

#include "common.cuh"
#include "dynamics.cuh"
#include "dynamics_thread.cuh"
#include "stages.cuh"


namespace gato {

// bounds (mbarrier try_wait calls of about 1 us each) of the waits for bulk
// copies into shared memory: the default wait, and the drain of a copy whose
// wait expired before the CTA stops using its buffer
constexpr int PCG_STAGE_WAIT_TRIES = 1 << 22;
constexpr int PCG_STAGE_DRAIN_TRIES = 1 << 22;

// Per-solver device state handed to every kernel by value.
template <int NQ, typename T>
struct Batch {
    int B, N;
    float solve_ratio;
    int max_pcg_iters;
    float abs_tol;  // PCG absolute floor on |r.z| (1e-6 in the reference, pcg.cuh:85-89)
    int adapt_rho;
    CostParams<T> cp;
    // problem data
    T* xu;
    const T* xs;
    const T* goal;
    const T* fext;         // [B][6]
    int use_fext;          // 0: f_ext all zero, skip the wrench terms
    // KKT system and Schur complement
    T *Q, *R, *q, *r, *A, *Bm, *c, *Qi, *Ri;
    T *S, *P, *gamma, *lambda, *dz;
    // per-problem scalars
    T *rho, *drho, *mu, *tol;
    double *merit_terms;   // [B][NUM_ALPHAS][N]
    double *merit_init, *merit_init0, *merit_final;
    int *pcg_iters, *conv, *sqp_iters;
    int* done;             // device flag: batch converged (fused form)
    // [0] next problem of a persistent launch, [1] CTAs finished, [2] a
    // bounded wait expired (both counters are back at 0 after each launch)
    int* work;
    int* ls_count;         // line-search iterations run (fused form)
    int* status;           // [B] GATO_STATUS_* bits found on the device
    // bounds (mbarrier try_wait calls) of the persistent PCG's waits for its
    // bulk copies: S and P^-1, and the step recovery's A_k, Qi_k
    int wait_tries, wait_tries_dz;
    // per-iteration statistics [iter][B]
    int* h_pcg;
    float *h_ls_min, *h_ls_step;
};

// ------------------------------------------------------------------ merit
// One warp per (knot, alpha); terms[b][alpha][k].
template <int NQ, typename T>
__global__ void k_merit(Batch<NQ, T> bt, DevModel<NQ, T> M, int nalpha, int use_dz, int skip_if_done)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);
    if (skip_if_done && *bt.done) return;
    const int b = blockIdx.y;
    const int wpb = blockDim.x / WARP;
    const int item = blockIdx.x * wpb + warp_id();
    const int N = bt.N;
    if (item >= N * nalpha) return;
    const int k = item % N, j = item / N;
    T* s = smem + warp_id() * MeritSmem<NQ>::SIZE;
    const Dims<NQ> d{N};
    const T alpha = T(1) / (T)(1 << j);
    const T v = merit_knot<NQ, T>(M, cost_of<NQ>(bt.cp, b), N, k, alpha, bt.mu[b], bt.xu + (size_t)b * d.traj(),
                                   use_dz ? bt.dz + (size_t)b * d.traj() : nullptr,
                                   bt.xs + (size_t)b * Dims<NQ>::nx, bt.goal + (size_t)b * d.goal(),
                                   bt.use_fext ? bt.fext + 6 * b : nullptr, s);
    if (lane_id() == 0) bt.merit_terms[((size_t)b * NUM_ALPHAS + j) * N + k] = (double)v;
}

// Sum of the alpha = 1 terms into out[b] (initial / final merit); a
// non-finite merit marks the problem's status.
template <typename Acc>
__global__ void k_merit_sum(int B, int N, const double* terms, double* out, double* out2,
                            int* status)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    Acc s = 0;
    for (int k = 0; k < N; ++k) s += (Acc)terms[(size_t)b * NUM_ALPHAS * N + k];
    out[b] = (double)s;
    if (out2) out2[b] = (double)s;
    if (!isfinite((double)s)) status[b] |= GATO_STATUS_NONFINITE;
}

// Status bits of one line search: no trial step lowered the merit, and
// every trial merit non-finite (the step itself is not finite).
template <typename Acc>
__device__ __forceinline__ int ls_status(const Acc* s_m, bool ok)
{
    int st = ok ? 0 : GATO_STATUS_LS_FAIL;
    bool any = false;
    for (int j = 0; j < NUM_ALPHAS; ++j) any |= isfinite((double)s_m[j]);
    if (!any) st |= GATO_STATUS_NONFINITE;
    return st;
}

// ------------------------------------------------------------------ line search
// lineSearchAndUpdateBatchedKernel (gato/bsqp/kernels/line_search.cuh:12-98),
// one block per problem.  Merit sums over knots are formed here in a fixed
// order (Acc precision) instead of the reference's float atomicAdd.
template <int NQ, typename T, typename Acc>
__global__ void k_line_search(Batch<NQ, T> bt, int it, int skip_if_done)
{
    if (skip_if_done && *bt.done) return;
    const int b = blockIdx.x;
    const int N = bt.N;
    __shared__ Acc s_m[NUM_ALPHAS];
    __shared__ T s_step;
    __shared__ int s_ok;
    const int t = threadIdx.x;
    if (t < NUM_ALPHAS) {
        Acc s = 0;
        const double* tm = bt.merit_terms + ((size_t)b * NUM_ALPHAS + t) * N;
        for (int k = 0; k < N; ++k) s += (Acc)tm[k];
        s_m[t] = s;
    }
    __syncthreads();
    if (t == 0) {
        Acc best = (Acc)1e38;
        int bj = 0;
        for (int j = 0; j < NUM_ALPHAS; ++j)
            if (s_m[j] < best) {
                best = s_m[j];
                bj = j;
            }
        const Acc m0 = (Acc)bt.merit_init[b];
        const bool ok = best < m0;
        bt.status[b] |= ls_status<Acc>(s_m, ok);
        if (bt.adapt_rho) {
            const T dr = bt.drho[b];
            const T fac = T(RHO_FACTOR);
            const T mult = ok ? gmin(dr / fac, T(1) / fac) : gmax(dr * fac, fac);
            bt.drho[b] = mult;
            const T rr = gmax(bt.rho[b] * mult, T(RHO_MIN));
            bt.rho[b] = gmin(rr, T(RHO_MAX));
        }
        T step;
        if (!ok) {
            if (bt.rho[b] > T(RHO_MAX)) bt.rho[b] = T(RHO_INIT);
            step = T(-1);
        } else {
            step = T(1) / (T)(1 << bj);
            bt.merit_init[b] = (double)best;
        }
        s_step = step;
        s_ok = ok;
        if (bt.h_ls_min) {
            bt.h_ls_min[(size_t)it * bt.B + b] = (float)bt.merit_init[b];
            bt.h_ls_step[(size_t)it * bt.B + b] = (float)step;
        }
    }
    __syncthreads();
    if (s_ok) {
        const Dims<NQ> d{N};
        T* x = bt.xu + (size_t)b * d.traj();
        const T* dz = bt.dz + (size_t)b * d.traj();
        const T st = s_step;
        for (int i = t; i < d.traj(); i += blockDim.x) x[i] += st * dz[i];
    }
}

// ------------------------------------------------------------------ merit + line search
// One block per problem, one thread per (step size, knot) sample
// (computeMeritBatchedKernel + lineSearchAndUpdateBatchedKernel,
// gato/bsqp/kernels/merit.cuh:16-92, line_search.cuh:12-98).  The merit sum of
// each step size is formed in knot order in Acc precision.
//   mode 0: merit of XU (alpha = 1, no step)  -> merit_init, merit_init0
//   mode 1: line search over NUM_ALPHAS steps -> rho, step, XU update
//   mode 2: merit of XU                       -> merit_final
template <int NQ, typename T, typename Acc>
__device__ __forceinline__ void merit_ls_body(const Batch<NQ, T>& bt, const DevModel<NQ, T>& M,
                                              int b, int mode, int it, unsigned char* smem_raw)
{
    Acc* terms = reinterpret_cast<Acc*>(smem_raw);
    __shared__ Acc s_m[NUM_ALPHAS];
    __shared__ T s_step;
    __shared__ int s_ok;
    if (mode == 1 && *bt.done) return;
    const int N = bt.N;
    const int nalpha = (mode == 1) ? NUM_ALPHAS : 1;
    const Dims<NQ> d{N};
    const T* xu = bt.xu + (size_t)b * d.traj();
    const T* dz = (mode == 1) ? bt.dz + (size_t)b * d.traj() : nullptr;
    const T mu = bt.mu[b];
    const T* fext = bt.use_fext ? bt.fext + 6 * b : nullptr;
    for (int item = threadIdx.x; item < nalpha * N; item += blockDim.x) {
        const int k = item % N, j = item / N;
        const T alpha = T(1) / (T)(1 << j);
        terms[item] = (Acc)merit_thread<NQ, T>(M, cost_of<NQ>(bt.cp, b), N, k, alpha, mu, xu, dz,
                                               bt.xs + (size_t)b * Dims<NQ>::nx,
                                               bt.goal + (size_t)b * d.goal(), fext);
    }
    __syncthreads();
    const int t = threadIdx.x;
    if (t < nalpha) {
        Acc sum = 0;
        for (int k = 0; k < N; ++k) sum += terms[t * N + k];
        s_m[t] = sum;
    }
    __syncthreads();
    if (mode != 1) {
        if (t == 0) {
            if (!isfinite((double)s_m[0])) bt.status[b] |= GATO_STATUS_NONFINITE;
            if (mode == 0) {
                bt.merit_init[b] = (double)s_m[0];
                bt.merit_init0[b] = (double)s_m[0];
            } else {
                bt.merit_final[b] = (double)s_m[0];
            }
        }
        return;
    }
    if (t == 0) {
        Acc best = (Acc)1e38;
        int bj = 0;
        for (int j = 0; j < NUM_ALPHAS; ++j)
            if (s_m[j] < best) {
                best = s_m[j];
                bj = j;
            }
        const bool ok = best < (Acc)bt.merit_init[b];
        bt.status[b] |= ls_status<Acc>(s_m, ok);
        if (bt.adapt_rho) {
            const T dr = bt.drho[b];
            const T fac = T(RHO_FACTOR);
            const T mult = ok ? gmin(dr / fac, T(1) / fac) : gmax(dr * fac, fac);
            bt.drho[b] = mult;
            const T rr = gmax(bt.rho[b] * mult, T(RHO_MIN));
            bt.rho[b] = gmin(rr, T(RHO_MAX));
        }
        T step;
        if (!ok) {
            if (bt.rho[b] > T(RHO_MAX)) bt.rho[b] = T(RHO_INIT);
            step = T(-1);
        } else {
            step = T(1) / (T)(1 << bj);
            bt.merit_init[b] = (double)best;
        }
        s_step = step;
        s_ok = ok;
        if (bt.h_ls_min) {
            bt.h_ls_min[(size_t)it * bt.B + b] = (float)bt.merit_init[b];
            bt.h_ls_step[(size_t)it * bt.B + b] = (float)step;
        }
    }
    __syncthreads();
    if (s_ok) {
        T* x = bt.xu + (size_t)b * d.traj();
        const T st = s_step;
        for (int i = t; i < d.traj(); i += blockDim.x) x[i] += st * dz[i];
    }
}

template <int NQ, typename T, typename Acc>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 2 : 1) k_merit_ls(Batch<NQ, T> bt, DevModel<NQ, T> M, int mode,
                                                  int it)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    merit_ls_body<NQ, T, Acc>(bt, M, blockIdx.x, mode, it, smem_raw);
}

// ------------------------------------------------------------------ KKT
template <int NQ, typename T>
__global__ void k_kkt(Batch<NQ, T> bt, DevModel<NQ, T> M)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);
    const int b = blockIdx.y;
    const int wpb = blockDim.x / WARP;
    const int k = blockIdx.x * wpb + warp_id();
    const int N = bt.N;
    if (k >= N - 1 || *bt.done) return;  // done: a converged fused-form batch
    const Dims<NQ> d{N};
    constexpr int nx = Dims<NQ>::nx, nu = Dims<NQ>::nu;
    T* s = smem + warp_id() * KktSmem<NQ>::SIZE;
    kkt_knot<NQ, T>(M, cost_of<NQ>(bt.cp, b), N, k, bt.xu + (size_t)b * d.traj(), bt.xs + (size_t)b * nx,
                 bt.goal + (size_t)b * d.goal(), bt.use_fext ? bt.fext + 6 * b : nullptr,
                 bt.Q + (size_t)b * N * nx * nx, bt.R + (size_t)b * N * nu * nu,
                 bt.q + (size_t)b * N * nx, bt.r + (size_t)b * N * nu,
                 bt.A + (size_t)b * N * nx * nx, bt.Bm + (size_t)b * N * nx * nu,
                 bt.c + (size_t)b * N * nx, s);
}

// ------------------------------------------------------------------ Schur
// Inverses Qi_k = (Q_k + rho I_q)^-1 (all k) and Ri_k = R_k^-1 (k < N-1),
// one warp per knot.
template <int NQ, typename T>
__global__ void k_schur_inv(Batch<NQ, T> bt)
{
    if (*bt.done) return;  // fused form: the batch has converged
    const int b = blockIdx.y;
    const int wpb = blockDim.x / WARP;
    const int k = blockIdx.x * wpb + warp_id();
    const int N = bt.N;
    if (k >= N) return;
    constexpr int nx = Dims<NQ>::nx, nu = Dims<NQ>::nu;
    const T rho = bt.rho[b];
    const T* Qk = bt.Q + ((size_t)b * N + k) * nx * nx;
    warp_invert<nx, T>(Qk, rho, bt.Qi + ((size_t)b * N + k) * nx * nx);
    if (k < N - 1) warp_invert<nu, T>(bt.R + ((size_t)b * N + k) * nu * nu, T(0),
                                   bt.Ri + ((size_t)b * N + k) * nu * nu);
}

template <int NQ, typename T>
__global__ void k_schur(Batch<NQ, T> bt)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);
    if (*bt.done) return;
    const int b = blockIdx.y;
    const int wpb = blockDim.x / WARP;
    const int k = blockIdx.x * wpb + warp_id();
    const int N = bt.N;
    if (k >= N) return;
    const Dims<NQ> d{N};
    constexpr int nx = Dims<NQ>::nx, nu = Dims<NQ>::nu;
    T* S = bt.S + (size_t)b * d.b3d();
    T* P = bt.P + (size_t)b * d.b3d();
    T* g = bt.gamma + (size_t)b * d.vecp();
    const T* Qi = bt.Qi + (size_t)b * N * nx * nx;
    if (k == N - 1) {
        schur_first<NQ, T>(bt.rho[b], bt.Q + (size_t)b * N * nx * nx, Qi, bt.q + (size_t)b * N * nx,
                        bt.c + (size_t)b * N * nx, S, P, g);
        return;
    }
    T* s = smem + warp_id() * SchurSmem<NQ>::SIZE;
    schur_knot<NQ, T>(k, bt.rho[b], Qi, bt.Ri + (size_t)b * N * nu * nu, bt.q + (size_t)b * N * nx,
                   bt.r + (size_t)b * N * nu, bt.A + (size_t)b * N * nx * nx,
                   bt.Bm + (size_t)b * N * nx * nu, bt.c + (size_t)b * N * nx, S, P, g, s);
}

template <int NQ, typename T>
__global__ void k_schur_off(Batch<NQ, T> bt)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);
    if (*bt.done) return;
    const int b = blockIdx.y;
    const int wpb = blockDim.x / WARP;
    const int k = blockIdx.x * wpb + warp_id();
    const int N = bt.N;
    if (k >= N - 1) return;
    const Dims<NQ> d{N};
    constexpr int nx = Dims<NQ>::nx;
    T* s = smem + warp_id() * 4 * nx * nx;
    schur_offdiag<NQ, T>(k, bt.S + (size_t)b * d.b3d(), bt.P + (size_t)b * d.b3d(), s);
}

// ------------------------------------------------------------------ PCG
// Block-tridiagonal matrix-vector product over padded vectors
// (btdMatrixVectorProduct, gato/utils/linalg.cuh:174-221): warp w takes block
// rows w, w+W, ...; lane 2*row+half sums half of the 3n columns of one row.
// Returns this lane's partial of out . dotw over the entries it wrote.
template <int NQ, typename T, typename Acc>
__device__ __forceinline__ Acc btd_mv(int N, const T* __restrict__ Mx, const T* __restrict__ vin,
                                      T* __restrict__ vout, const T* __restrict__ dotw)
{
    constexpr int n = 2 * NQ, RD = 3 * n, HALF = RD / 2;
    const int l = lane_id();
    const int row = l >> 1, half = l & 1;
    const int nw = blockDim.x / WARP;
    Acc part = 0;
    for (int br = warp_id(); br < N; br += nw) {
        T acc = T(0);
        if (row < n) {
            const T* mrow = Mx + (size_t)br * n * RD + row * RD + half * HALF;
            const T* v = vin + br * n + half * HALF;
#pragma unroll
            for (int c = 0; c < HALF; ++c) acc += mrow[c] * v[c];
        }
        acc += __shfl_xor_sync(FULL, acc, 1);
        if (row < n && half == 0) {
            const int idx = (br + 1) * n + row;
            vout[idx] = acc;
            part += (Acc)acc * (Acc)dotw[idx];
        }
    }
    return part;
}

template <typename Acc>
__device__ __forceinline__ Acc block_sum(Acc v, Acc* red)
{
    v = warp_sum(v);
    if (lane_id() == 0) red[warp_id()] = v;
    __syncthreads();
    Acc s = 0;
    const int nw = blockDim.x / WARP;
    for (int w = 0; w < nw; ++w) s += red[w];
    return s;
}

// Preconditioned CG on S lambda = gamma for one problem, one block
// (solvePCGBatchedKernel, gato/bsqp/kernels/pcg.cuh:23-147): warm start from
// lambda, stop when |r.z| < 1e-6 + eps |r0.z0|, zero iterations (lambda left
// untouched) when |r0.z0| < 1e-6.  S and P may live in shared or global
// memory.  sv holds 5 padded vectors, red 2*32 Acc.  Returns the iteration
// count.
template <int NQ, typename T, typename Acc>
__device__ int pcg_block(int N, const T* __restrict__ S, const T* __restrict__ P,
                         const T* __restrict__ gamma, T* __restrict__ lam, T eps, int max_iters,
                         T* sv, Acc* red, float abs_floor)
{
    constexpr int n = 2 * NQ;
    const int L = (N + 2) * n;
    const int tid = threadIdx.x, bs = blockDim.x;
    T* x = sv;
    T* r = x + L;
    T* z = r + L;
    T* p = z + L;
    T* Ap = p + L;
    for (int i = tid; i < L; i += bs) {
        x[i] = lam[i];
        r[i] = 0.0f;
        z[i] = 0.0f;
        p[i] = 0.0f;
        Ap[i] = 0.0f;
    }
    __syncthreads();
    btd_mv<NQ, T, Acc>(N, S, x, r, r);
    __syncthreads();
    for (int i = tid; i < L; i += bs) r[i] = gamma[i] - r[i];
    __syncthreads();
    Acc part = btd_mv<NQ, T, Acc>(N, P, r, z, r);
    Acc rho = block_sum<Acc>(part, red);
    for (int i = tid; i < L; i += bs) p[i] = z[i];
    const Acc abs_tol = Acc(abs_floor);
    if (fabs((double)rho) < (double)abs_tol) return 0;
    const Acc rho_init = rho < 0 ? -rho : rho;
    __syncthreads();
    int it = 0;
    for (int i = 0; i < max_iters; ++i) {
        ++it;
        part = btd_mv<NQ, T, Acc>(N, S, p, Ap, p);
        const Acc pAp = block_sum<Acc>(part, red);
        const Acc alpha = rho / pAp;
        const T af = (T)alpha;
        for (int j = tid; j < L; j += bs) {
            x[j] += af * p[j];
            r[j] -= af * Ap[j];
        }
        __syncthreads();
        part = btd_mv<NQ, T, Acc>(N, P, r, z, r);
        const Acc rho_new = block_sum<Acc>(part, red + WARP);
        const Acc arn = rho_new < 0 ? -rho_new : rho_new;
        // the reference's stop (pcg.cuh:128-129); an exact zero also stops (reachable
        // only with a zero tolerance), a NaN runs on to the cap as it does there
        if (arn < abs_tol + (Acc)eps * rho_init || arn == 0) break;
        const Acc beta = rho_new / rho;
        rho = rho_new;
        const T bf = (T)beta;
        for (int j = tid; j < L; j += bs) p[j] = z[j] + bf * p[j];
        __syncthreads();
    }
    __syncthreads();
    for (int i = tid; i < L; i += bs) lam[i] = x[i];
    return it;
}

// Dynamic shared memory of k_pcg: matrices staged when `stage` is set.
// Layout: [S | P (when staged) | 5 padded vectors | reduction slots].
template <int NQ, typename T>
__host__ __device__ inline size_t pcg_smem_bytes(int N, bool stage)
{
    const Dims<NQ> d{N};
    size_t f = 5 * (size_t)d.vecp() + (stage ? 2 * (size_t)d.b3d() : 0);
    return f * sizeof(T) + 2 * WARP * sizeof(double) + 32;
}

template <int NQ, typename T, typename Acc>
__global__ void k_pcg(Batch<NQ, T> bt, int stage, int it_row)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);
    const int b = blockIdx.x;
    const Dims<NQ> d{bt.N};
    int iters = 0;
    if (!bt.conv[b]) {
        const T* S = bt.S + (size_t)b * d.b3d();
        const T* P = bt.P + (size_t)b * d.b3d();
        const size_t mats = stage ? 2 * (size_t)d.b3d() : 0;
        T* sv = smem + mats;
        Acc* red = reinterpret_cast<Acc*>(
            ((uintptr_t)(smem + mats + 5 * d.vecp()) + 15) & ~(uintptr_t)15);
        if (stage) {
            T* sS = smem;
            T* sP = sS + d.b3d();
            const uint4* gS = reinterpret_cast<const uint4*>(S);
            const uint4* gP = reinterpret_cast<const uint4*>(P);
            uint4* tS = reinterpret_cast<uint4*>(sS);
            uint4* tP = reinterpret_cast<uint4*>(sP);
            const int chunks = (int)((size_t)d.b3d() * sizeof(T) / sizeof(uint4));
            for (int i = threadIdx.x; i < chunks; i += blockDim.x) {
                tS[i] = gS[i];
                tP[i] = gP[i];
            }
            __syncthreads();
            S = sS;
            P = sP;
        }
        iters = pcg_block<NQ, T, Acc>(bt.N, S, P, bt.gamma + (size_t)b * d.vecp(),
                                   bt.lambda + (size_t)b * d.vecp(), bt.tol[b], bt.max_pcg_iters,
                                   sv, red, bt.abs_tol);
    }
    if (threadIdx.x == 0) {
        bt.pcg_iters[b] = iters;
        if (it_row >= 0 && bt.h_pcg) bt.h_pcg[(size_t)it_row * bt.B + b] = iters;
    }
}

// ------------------------------------------------------------------ row PCG
// Preconditioned CG with the matrices resident in registers: each thread owns
// RPT rows of one block row of S and P^-1 (3n entries per row) and the
// matching entries of every CG vector; only p and r go through shared memory,
// where a thread reads the 3n-wide window of its block row once with 16-byte
// loads and applies it to all of its rows.  Same iteration as pcg_block
// (gato/bsqp/kernels/pcg.cuh:23-147).  After the solve the block computes the
// step dz of every knot (dz_knot's algebra).
//
// Vectors use a block stride VS: n rounded up to a multiple of 4 whose number
// of 16-byte chunks is odd.  A warp reads the windows of five or six
// consecutive block rows at once; with an odd chunk count those start in
// different bank quads (iiwa14: VS = 20, not 16, which put every other block
// row on the same banks and serialised the load three ways).
__host__ __device__ constexpr int row_vs(int n)
{
    return (((n + 3) / 4) % 2) ? ((n + 3) & ~3) : ((n + 3) & ~3) + 4;
}

// Rows of S and P^-1 per thread in the register-resident PCG: two in FP32
// (each window value loaded from shared memory feeds two rows; one row per
// thread measured 13 % slower), one in FP64.
template <typename T>
__host__ __device__ constexpr int pcg_rows_per_thread()
{
    return 2;
}
// FP64 k_pcg_rows keeps S in registers and P^-1 in shared memory (SmemRows)
template <typename T>
__host__ __device__ constexpr bool pcg_p_in_smem()
{
    return sizeof(T) == 8;
}
// rows per thread of the cluster PCG (both matrices in registers)
template <typename T>
__host__ __device__ constexpr int cluster_rows_per_thread()
{
    return sizeof(T) == 4 ? 2 : 1;
}


template <int NQ, int RPT>
struct SmemRows;

// The scalar divisions of the single-reduction recurrence.  With FP32
// reductions they sit on the CG loop's critical path, so they use the
// hardware's approximate division (__fdividef, within 2 ulp, one reciprocal
// and one multiply instead of the correctly rounded sequence): PCG 2.57 ->
// 2.46 ms per solve on the bench workload, with the trajectory error against
// the FP64 oracle unchanged (median 3.35e-4 -> 3.38e-4, PCG counts equal
// 96.3 % -> 96.2 %, 64 line-search decisions diverging in both).  The mixed
// form's FP64 reductions divide exactly.
template <typename Acc>
__device__ __forceinline__ Acc rec_div(Acc a, Acc b)
{
    if constexpr (sizeof(Acc) == 4) return __fdividef(a, b);
    return a / b;
}

template <int NQ, int RPT>
struct RowPcg {
    static constexpr int n = 2 * NQ, m = NQ, RD = 3 * n, VS = row_vs(n);
    static constexpr int TPB = n / RPT;  // threads per block row
    static_assert(n % RPT == 0, "rows per thread must divide n");
    static constexpr int MAX_THREADS = 512 / RPT;
    __host__ __device__ static int threads(int N) { return ((N * TPB + 31) / 32) * 32; }
    __host__ __device__ static bool fits(int N) { return N * TPB <= MAX_THREADS; }
    // P^-1 in shared memory (SmemRows, SmemRowsF): block row k starts at
    // element k * bstride<E>(), a pad after each block row's n x 3n elements.
    // A lane loads column pairs (2 E) of its rows; the lanes of one
    // shared-memory wavefront (8 for 16-byte loads, 16 for 8-byte) take
    // consecutive rows of a block row and then the first rows of the next.
    // A row is 3n/2 pairs; when that is odd, consecutive rows fall in
    // distinct banks, and the pad makes the next block row continue that
    // sequence, so a wavefront's loads never share a bank (unpadded, rows 8
    // apart collided and every FP64 row load took two wavefronts).
    template <typename E>
    __host__ __device__ static constexpr int ppad()
    {
        constexpr int W = 128 / (2 * (int)sizeof(E)), s = RD / 2;
        return (s % 2) ? ((((TPB - n) * s) % W + W) % W) * 2 : 0;
    }
    template <typename E>
    __host__ __device__ static constexpr int bstride()
    {
        return n * RD + ppad<E>();
    }
    // the FP64 PCG's matrix buffer: S (one copy, unpadded), then P^-1
    // (padded); with p32 P^-1 in FP32 (padded) and a staging area for half
    // of the FP64 P^-1 after it
    __host__ __device__ static size_t psm_buf_bytes(int N, bool p32)
    {
        const size_t s_bytes = (size_t)N * n * RD * sizeof(double);
        size_t p_bytes = (size_t)N * bstride<double>() * sizeof(double);
        if (p32)
            p_bytes = (((size_t)N * bstride<float>() * sizeof(float) + 15) & ~(size_t)15) +
                      s_bytes / 2;
        return s_bytes > p_bytes ? s_bytes : p_bytes;
    }
    // the two CG vectors and the reduction slots; in FP64 also the matrix
    // buffer (pcg_p_in_smem)
    template <typename T>
    __host__ __device__ static size_t smem_bytes(int N)
    {
        const size_t base = 2 * (size_t)(N + 2) * VS * sizeof(T) + 2 * WARP * sizeof(double) + 16;
        if (!pcg_p_in_smem<T>()) return base;
        return base + 16 + psm_buf_bytes(N, false);
    }
    // FP64 with the FP32 preconditioner: its buffer and the FP32 residual window
    __host__ __device__ static size_t smem_bytes_p32(int N)
    {
        const size_t base = 2 * (size_t)(N + 2) * VS * sizeof(double) + 2 * WARP * sizeof(double) + 16;
        return base + 16 + psm_buf_bytes(N, true) + 16 + (size_t)(N + 2) * VS * sizeof(float);
    }
};

// The RPT rows of S or P^-1 a thread holds in registers.  FP32 rows are kept
// as column pairs, so one packed FMA (__ffma2_rn: each lane rounded as
// fmaf) advances the even- and odd-column partial sums of a row together.
template <int NQ, int RPT, typename T>
struct RowMat {
    static constexpr int RD = 6 * NQ;
    T v[RPT][RD];
    // rows j = 0..RPT-1 start at base + j * jstride (zero rows when !act)
    __device__ __forceinline__ void load(const T* base, size_t jstride, bool act)
    {
#pragma unroll
        for (int j = 0; j < RPT; ++j)
#pragma unroll
            for (int c = 0; c < RD; ++c) v[j][c] = act ? base[j * jstride + c] : T(0);
    }
};
template <int NQ, int RPT>
struct RowMat<NQ, RPT, float> {
    static constexpr int RD = 6 * NQ;
    float2 v[RPT][RD / 2];
    __device__ __forceinline__ void load(const float* base, size_t jstride, bool act)
    {
#pragma unroll
        for (int j = 0; j < RPT; ++j) {
            const float2* src = reinterpret_cast<const float2*>(base + j * jstride);
#pragma unroll
            for (int c = 0; c < RD / 2; ++c) v[j][c] = act ? src[c] : make_float2(0.f, 0.f);
        }
    }
};

// out[j] = row[j] . window for the RPT rows of a thread: three blocks of a
// vector at stride VS, four partial sums per row by column mod 4, combined
// as (s0 + s1) + (s2 + s3).  The FP32 form keeps eight (column mod 8): the
// dependent FMA chains are the latency of the CG loop, and halving their
// depth took 6.6 % off the PCG.
template <int NQ, int RPT, typename T>
__device__ __forceinline__ void rows_window_dot(const RowMat<NQ, RPT, T>& row, const T* win,
                                                T (&out)[RPT])
{
    constexpr int n = 2 * NQ, VS = row_vs(n);
    static_assert(sizeof(T) == 8, "FP32 has its own overload");
    T acc[RPT][4];
#pragma unroll
    for (int j = 0; j < RPT; ++j)
#pragma unroll
        for (int a = 0; a < 4; ++a) acc[j][a] = T(0);
#pragma unroll
    for (int blk = 0; blk < 3; ++blk) {
#pragma unroll
        for (int c0 = 0; c0 < n; c0 += 2) {
            const double2 v = *reinterpret_cast<const double2*>(win + blk * VS + c0);
#pragma unroll
            for (int j = 0; j < RPT; ++j) {
                acc[j][c0 & 3] += row.v[j][blk * n + c0] * v.x;
                acc[j][(c0 + 1) & 3] += row.v[j][blk * n + c0 + 1] * v.y;
            }
        }
    }
#pragma unroll
    for (int j = 0; j < RPT; ++j) out[j] = (acc[j][0] + acc[j][1]) + (acc[j][2] + acc[j][3]);
}

template <int NQ, int RPT>
__device__ __forceinline__ void rows_window_dot(const RowMat<NQ, RPT, float>& row,
                                                const float* win, float (&out)[RPT])
{
    constexpr int n = 2 * NQ, VS = row_vs(n);
    static_assert(n % 2 == 0, "column pairs");
    float2 acc[RPT][4];  // column mod 8: (s0, s1), (s2, s3), (s4, s5), (s6, s7)
#pragma unroll
    for (int j = 0; j < RPT; ++j)
#pragma unroll
        for (int a = 0; a < 4; ++a) acc[j][a] = make_float2(0.f, 0.f);
#pragma unroll
    for (int blk = 0; blk < 3; ++blk) {
#pragma unroll
        for (int c0 = 0; c0 < n; c0 += 4) {
            const float4 v = *reinterpret_cast<const float4*>(win + blk * VS + c0);
            const float2 lo = make_float2(v.x, v.y), hi = make_float2(v.z, v.w);
            const int h = ((c0 / 4) & 1) * 2;
#pragma unroll
            for (int j = 0; j < RPT; ++j) {
                acc[j][h] = __ffma2_rn(row.v[j][(blk * n + c0) / 2], lo, acc[j][h]);
                if (c0 + 2 < n)
                    acc[j][h + 1] = __ffma2_rn(row.v[j][(blk * n + c0) / 2 + 1], hi, acc[j][h + 1]);
            }
        }
    }
#pragma unroll
    for (int j = 0; j < RPT; ++j)
        out[j] = ((acc[j][0].x + acc[j][0].y) + (acc[j][1].x + acc[j][1].y)) +
                 ((acc[j][2].x + acc[j][2].y) + (acc[j][3].x + acc[j][3].y));
}

// FP64 P^-1 in shared memory.  An FP64 problem's S and P^-1 (2 x 150 KB for
// iiwa14 N = 32) do not fit in one SM's registers together: S stays in
// registers (RPT rows a thread) and P^-1 is bulk-copied into shared memory
// row-major, [N n][3n] with a pad after each block row (RowPcg::bstride): a
// row is 3n doubles = 21 sixteen-byte chunks for iiwa14 (an odd count), so
// the 16-byte loads of eight threads on consecutive rows fall in eight
// different bank quads, across a block-row boundary too.  The dot product keeps the register form's four partial sums by column mod 4
// and reads each window value once for the thread's RPT rows, so the iterates
// are those of the register form bit for bit.
// horizons whose PCG runs k_pcg_rows (one CTA a problem); longer ones take
// the cluster PCG
template <int NQ, typename T>
__host__ __device__ bool rows_pcg_fits(int N)
{
    return RowPcg<NQ, pcg_rows_per_thread<T>()>::fits(N);
}

template <int NQ, int RPT>
struct SmemRows {
    static constexpr int n = 2 * NQ, RD = 3 * n, TPB = n / RPT;
    const double* base;  // the thread's first row of P^-1 in shared memory; row j at
                         // base + j * TPB * RD
};

template <int NQ, int RPT>
__device__ __forceinline__ void rows_window_dot(const SmemRows<NQ, RPT>& p, const double* win,
                                                double (&out)[RPT])
{
    constexpr int n = 2 * NQ, VS = row_vs(n), TPB = n / RPT, RD = 3 * n;
    double acc[RPT][4];
#pragma unroll
    for (int j = 0; j < RPT; ++j)
#pragma unroll
        for (int a = 0; a < 4; ++a) acc[j][a] = 0.0;
#pragma unroll
    for (int blk = 0; blk < 3; ++blk) {
#pragma unroll
        for (int c0 = 0; c0 < n; c0 += 2) {
            const double2 v = *reinterpret_cast<const double2*>(win + blk * VS + c0);
#pragma unroll
            for (int j = 0; j < RPT; ++j) {
                const double2 m = *reinterpret_cast<const double2*>(
                    p.base + (size_t)j * TPB * RD + blk * n + c0);
                acc[j][c0 & 3] += m.x * v.x;
                acc[j][(c0 + 1) & 3] += m.y * v.y;
            }
        }
    }
#pragma unroll
    for (int j = 0; j < RPT; ++j) out[j] = (acc[j][0] + acc[j][1]) + (acc[j][2] + acc[j][3]);
}

template <typename Acc>
__device__ __forceinline__ Acc rows_block_sum(Acc v, Acc* red)
{
    v = warp_sum(v);
    if (lane_id() == 0) red[warp_id()] = v;
    __syncthreads();
    Acc s = 0;
    const int nw = blockDim.x / WARP;
    for (int w = 0; w < nw; ++w) s += red[w];
    return s;
}

// two block sums at once (one barrier); red holds 2 * WARP slots
template <typename Acc>
__device__ __forceinline__ void rows_block_sum2(Acc& a, Acc& b, Acc* red)
{
    a = warp_sum(a);
    b = warp_sum(b);
    if (lane_id() == 0) {
        red[warp_id()] = a;
        red[WARP + warp_id()] = b;
    }
    __syncthreads();
    Acc sa = 0, sb = 0, ta = 0, tb = 0;  // even and odd warps: half the dependent adds
    const int nw = blockDim.x / WARP;
    if (nw <= 8) {
        // the (up to) eight slots of each sum in 16-byte loads (red is
        // 16-byte aligned; slots past nw are loaded and not used)
        Acc ra[8], rb[8];
#pragma unroll
        for (int w = 0; w < 8; w += 16 / (int)sizeof(Acc)) {
            if constexpr (sizeof(Acc) == 4) {
                const float4 u = *reinterpret_cast<const float4*>(red + w);
                const float4 v = *reinterpret_cast<const float4*>(red + WARP + w);
                ra[w] = u.x, ra[w + 1] = u.y, ra[w + 2] = u.z, ra[w + 3] = u.w;
                rb[w] = v.x, rb[w + 1] = v.y, rb[w + 2] = v.z, rb[w + 3] = v.w;
            } else {
                const double2 u = *reinterpret_cast<const double2*>(red + w);
                const double2 v = *reinterpret_cast<const double2*>(red + WARP + w);
                ra[w] = u.x, ra[w + 1] = u.y;
                rb[w] = v.x, rb[w + 1] = v.y;
            }
        }
#pragma unroll
        for (int w = 0; w < 8; w += 2) {
            if (w < nw) {
                sa += ra[w];
                sb += rb[w];
            }
            if (w + 1 < nw) {
                ta += ra[w + 1];
                tb += rb[w + 1];
            }
        }
    } else {
        for (int w = 0; w < nw; w += 2) {
            sa += red[w];
            sb += red[WARP + w];
            if (w + 1 < nw) {
                ta += red[w + 1];
                tb += red[WARP + w + 1];
            }
        }
    }
    a = sa + ta;
    b = sb + tb;
}

struct NoHook {
    __device__ void operator()() const {}
};
struct NoDzStage {
    __device__ bool operator()() const { return false; }
};

// Sp, Pp: the problem's S and P^-1 (row-major [N n][3n]) in global or shared
// memory (null: bt.S, bt.P).  hook() runs on every thread after the CG loop,
// behind a barrier: Sp and Pp are no longer read.  Adz, Qidz: the problem's
// A_k and Qi_k blocks in shared memory, used by the step recovery on the
// threads where dz_ready() returns true (each thread decides for itself; no
// barrier depends on it), else read from global memory.
// P^-1 in FP32 in shared memory for an FP64 PCG (the FP32-preconditioner
// variant): the same row-major rows, applied to an FP32 copy of the residual
// window with FP32 FMAs, the row sums returned in FP64.  P^-1 only steers the
// CG iteration; the system S, the residual, the inner products and the
// recurrence stay FP64.  Half the shared-memory bytes of the FP64 rows.
template <int NQ, int RPT>
struct SmemRowsF {
    static constexpr int n = 2 * NQ, RD = 3 * n, TPB = n / RPT;
    const float* base;  // as SmemRows
};

template <int NQ, int RPT>
__device__ __forceinline__ void rows_window_dot(const SmemRowsF<NQ, RPT>& p, const float* win,
                                                double (&out)[RPT])
{
    constexpr int n = 2 * NQ, VS = row_vs(n), TPB = n / RPT, RD = 3 * n;
    float acc[RPT][4];
#pragma unroll
    for (int j = 0; j < RPT; ++j)
#pragma unroll
        for (int a = 0; a < 4; ++a) acc[j][a] = 0.f;
#pragma unroll
    for (int blk = 0; blk < 3; ++blk) {
#pragma unroll
        for (int c0 = 0; c0 < n; c0 += 2) {
            const float2 v = *reinterpret_cast<const float2*>(win + blk * VS + c0);
#pragma unroll
            for (int j = 0; j < RPT; ++j) {
                const float2 mm = *reinterpret_cast<const float2*>(
                    p.base + (size_t)j * TPB * RD + blk * n + c0);
                acc[j][c0 & 3] = fmaf(mm.x, v.x, acc[j][c0 & 3]);
                acc[j][(c0 + 1) & 3] = fmaf(mm.y, v.y, acc[j][(c0 + 1) & 3]);
            }
        }
    }
#pragma unroll
    for (int j = 0; j < RPT; ++j)
        out[j] = (double)((acc[j][0] + acc[j][1]) + (acc[j][2] + acc[j][3]));
}

// PSM: P^-1 in shared memory (SmemRows, FP64), S in registers.  An FP64
// problem's S and P^-1 (2 x 150 KB for iiwa14 N = 32) do not fit one SM's
// registers together; the FP64 form with both in registers (one row a
// thread) spilled and ran the PCG in 10.8 ms per solve (iiwa14 N = 32,
// 1024 problems), this one in 8.3.
template <int NQ, typename T, typename Acc, int RPT, class Hook = NoHook,
          class DzReady = NoDzStage, bool PSM = pcg_p_in_smem<T>(), bool P32 = false>
__device__ __forceinline__ void pcg_rows_body(const Batch<NQ, T>& bt, int b, int it_row,
                                              unsigned char* smem_raw, const T* Sp = nullptr,
                                              const T* Pp = nullptr, Hook hook = Hook(),
                                              const T* Adz = nullptr, const T* Qidz = nullptr,
                                              DzReady dz_ready = DzReady())
{
    constexpr bool HOOK = !std::is_same<Hook, NoHook>::value;
    using RP = RowPcg<NQ, RPT>;
    constexpr int n = RP::n, m = RP::m, RD = RP::RD, VS = RP::VS, TPB = RP::TPB;
    if (*bt.done) return;
    const int N = bt.N;
    const Dims<NQ> d{N};
    const int tid = threadIdx.x;
    const bool act = tid < N * TPB;
    const int k = act ? tid / TPB : 0, i0 = act ? tid % TPB : 0;
    const int L = (N + 2) * VS;
    T* pv = reinterpret_cast<T*>(smem_raw);
    T* rv = pv + L;
    Acc* red = reinterpret_cast<Acc*>(((uintptr_t)(rv + L) + 15) & ~(uintptr_t)15);
    // PSM: the bulk copies' mbarrier and the broadcast outcome of a wait
    __shared__ __align__(8) uint64_t s_pbar;
    __shared__ int s_pok;
    auto stage_wait = [&](uint32_t parity) {  // every thread; false: the wait expired
        if (tid == 0) {
            s_pok = mbar_wait_bounded(&s_pbar, parity, bt.wait_tries);
            if (!s_pok) {
                atomicExch(bt.work + 2, 1);
                if (mbar_wait_bounded(&s_pbar, parity, PCG_STAGE_DRAIN_TRIES)) mbar_inval(&s_pbar);
            }
        }
        __syncthreads();
        if (!s_pok) return false;
        if (tid != 0) mbar_try_wait(&s_pbar, parity);  // phase complete: acquires the data
        return true;
    };
    for (int j = tid; j < 2 * L; j += blockDim.x) pv[j] = T(0);
    // P32: the FP32 copy of the residual window, after the matrix buffer
    static_assert(!P32 || PSM, "the FP32 preconditioner is a form of the shared-memory P^-1");
    unsigned char* mbuf = reinterpret_cast<unsigned char*>(((uintptr_t)(red + 2 * WARP) + 15) &
                                                           ~(uintptr_t)15);
    float* rvf = reinterpret_cast<float*>(
        ((uintptr_t)(mbuf + RP::psm_buf_bytes(N, P32)) + 15) & ~(uintptr_t)15);
    if constexpr (P32) {
        for (int j = tid; j < L; j += blockDim.x) rvf[j] = 0.f;
    }
    T* lam = bt.lambda + (size_t)b * d.vecp();
    const int w0 = k * VS;
    int iters = 0;
    T x[RPT];
#pragma unroll
    for (int j = 0; j < RPT; ++j) x[j] = act ? lam[(k + 1) * n + i0 + j * TPB] : T(0);
    if (!bt.conv[b]) {
        // PSM: one shared-memory buffer after the reduction slots takes S by
        // bulk copy, the threads load their S rows from it into registers,
        // then it takes P^-1 (the second copy runs while r = gamma - S x is
        // formed).  Thread 0 waits with a bound and broadcasts the outcome; an
        // expired wait sets bt.work[2] (the host reports GATO_ERR_TIMEOUT and
        // the launch's results are not valid), lets the copy land and ends the
        // problem.
        static_assert(!PSM || sizeof(T) == 8, "P^-1 in shared memory is FP64");
        RowMat<NQ, RPT, T> srow;
        std::conditional_t<P32, SmemRowsF<NQ, RPT>,
                           std::conditional_t<PSM, SmemRows<NQ, RPT>, RowMat<NQ, RPT, T>>>
            prow;
        {
            const size_t row = (size_t)(k * n + i0) * RD;
            const size_t prob = (size_t)b * d.b3d();
            const T* Sg = Sp ? Sp : bt.S + prob;
            const T* Pg = Pp ? Pp : bt.P + prob;
            if constexpr (PSM) {
                T* buf = reinterpret_cast<T*>(mbuf);
                const uint32_t bytes = (uint32_t)(d.b3d() * sizeof(T));
                if (tid == 0) {
                    mbar_init(&s_pbar, 1);
                    fence_mbar_init();
                    fence_proxy_async_shared();
                    mbar_arrive_expect_tx(&s_pbar, bytes);
                    bulk_copy_g2s(buf, Sg, bytes, &s_pbar);
                }
                if (!stage_wait(0)) return;
                srow.load(buf + row, (size_t)TPB * RD, act);
                __syncthreads();  // every S read of the buffer is done
                constexpr int BR = n * RD;  // elements of a block row
                if constexpr (P32) {
                    // P^-1 in two halves: each bulk-copied into a staging
                    // area after the FP32 rows, then rounded to FP32 into
                    // the padded layout
                    constexpr int BSF = RP::template bstride<float>();
                    const size_t half = d.b3d() / 2;
                    float* pf = reinterpret_cast<float*>(buf);
                    T* stg = reinterpret_cast<T*>(
                        ((uintptr_t)(pf + (size_t)N * BSF) + 15) & ~(uintptr_t)15);
                    for (int h = 0; h < 2; ++h) {
                        if (tid == 0) {
                            fence_proxy_async_shared();
                            mbar_arrive_expect_tx(&s_pbar, bytes / 2);
                            bulk_copy_g2s(stg, Pg + h * half, bytes / 2, &s_pbar);
                        }
                        if (!stage_wait(h == 0 ? 1 : 0)) return;
                        for (size_t e = tid; e < half; e += blockDim.x) {
                            const size_t idx = h * half + e;
                            const size_t kb = idx / BR;
                            pf[kb * BSF + (idx - kb * BR)] = (float)stg[e];
                        }
                        __syncthreads();  // the staging area is read before it is refilled
                    }
                    prow.base = pf + (size_t)k * BSF + i0 * RD;
                } else {
                    constexpr int BS = RP::template bstride<double>();
                    if (tid == 0) {
                        fence_proxy_async_shared();
                        mbar_arrive_expect_tx(&s_pbar, bytes);
                        if constexpr (BS == BR) {
                            bulk_copy_g2s(buf, Pg, bytes, &s_pbar);
                        } else {
                            for (int kb = 0; kb < N; ++kb)  // one copy a block row
                                bulk_copy_g2s(buf + (size_t)kb * BS, Pg + (size_t)kb * BR,
                                              (uint32_t)(BR * sizeof(T)), &s_pbar);
                        }
                    }
                    prow.base = buf + (size_t)k * BS + i0 * RD;
                }
            } else {
                srow.load(Sg + row, (size_t)TPB * RD, act);
                prow.load(Pg + row, (size_t)TPB * RD, act);
            }
        }
        T g[RPT], r[RPT], z[RPT], p[RPT], ap[RPT];
#pragma unroll
        for (int j = 0; j < RPT; ++j)
            g[j] = act ? bt.gamma[(size_t)b * d.vecp() + (k + 1) * n + i0 + j * TPB] : T(0);
        __syncthreads();
        if (act) {
#pragma unroll
            for (int j = 0; j < RPT; ++j) pv[(k + 1) * VS + i0 + j * TPB] = x[j];
        }
        __syncthreads();
        rows_window_dot(srow, pv + w0, r);
        Acc part = 0;
#pragma unroll
        for (int j = 0; j < RPT; ++j) {
            r[j] = act ? g[j] - r[j] : T(0);
            if (act) {
                rv[(k + 1) * VS + i0 + j * TPB] = r[j];
                if constexpr (P32) rvf[(k + 1) * VS + i0 + j * TPB] = (float)r[j];
            }
        }
        if constexpr (PSM && !P32) {
            if (!stage_wait(1)) return;  // P^-1 landed (the wait is also the barrier)
        } else {
            __syncthreads();
        }
        if constexpr (P32)
            rows_window_dot(prow, rvf + w0, z);
        else
            rows_window_dot(prow, rv + w0, z);
        const Acc abs_tol = Acc(bt.abs_tol);
        const T eps = bt.tol[b];
        if constexpr (sizeof(T) == 4) {
            // Single-reduction form (Chronopoulos-Gear): w = S z is carried
            // with z, s = S p by recurrence, and r.z, z.w share one block
            // reduction, so an iteration has three barriers instead of four.
            // Same iterates as the reference's recurrence in exact
            // arithmetic; same stopping rule and iteration count.
            T w[RPT], sv[RPT];
            if (act) {
#pragma unroll
                for (int j = 0; j < RPT; ++j) pv[(k + 1) * VS + i0 + j * TPB] = z[j];
            }
            __syncthreads();
            rows_window_dot(srow, pv + w0, w);
            Acc rho = 0, delta = 0;
#pragma unroll
            for (int j = 0; j < RPT; ++j) {
                rho += act ? (Acc)r[j] * (Acc)z[j] : Acc(0);
                delta += act ? (Acc)z[j] * (Acc)w[j] : Acc(0);
            }
            rows_block_sum2<Acc>(rho, delta, red);
            if (!(fabs((double)rho) < (double)abs_tol)) {
                const Acc rho_init = rho < 0 ? -rho : rho;
                Acc alpha = rec_div(rho, delta);
                // delta = 0: nothing to do; a NaN runs on (and stops at the
                // breakdown test), so the problem is not taken as converged
                const bool start = !(delta == 0);
#pragma unroll
                for (int j = 0; j < RPT; ++j) {
                    p[j] = z[j];
                    sv[j] = w[j];
                }
                for (int it = 0; start && it < bt.max_pcg_iters; ++it) {
                    ++iters;
                    const T a = (T)alpha;
#pragma unroll
                    for (int j = 0; j < RPT; ++j) {
                        x[j] += a * p[j];
                        r[j] -= a * sv[j];
                        if (act) rv[(k + 1) * VS + i0 + j * TPB] = r[j];
                    }
                    __syncthreads();
                    rows_window_dot(prow, rv + w0, z);
                    if (act) {
#pragma unroll
                        for (int j = 0; j < RPT; ++j) pv[(k + 1) * VS + i0 + j * TPB] = z[j];
                    }
                    __syncthreads();
                    rows_window_dot(srow, pv + w0, w);
                    Acc rho_new = 0;
                    delta = 0;
#pragma unroll
                    for (int j = 0; j < RPT; ++j) {
                        rho_new += act ? (Acc)r[j] * (Acc)z[j] : Acc(0);
                        delta += act ? (Acc)z[j] * (Acc)w[j] : Acc(0);
                    }
                    rows_block_sum2<Acc>(rho_new, delta, red);
                    const Acc arn = rho_new < 0 ? -rho_new : rho_new;
                    if (arn < abs_tol + (Acc)eps * rho_init || !(arn > 0)) break;
                    const Acc beta = rec_div(rho_new, rho);
                    const Acc rn_a = rec_div(rho_new, alpha);  // independent of beta's division
                    alpha = rec_div(rho_new, delta - beta * rn_a);
                    // breakdown: keep the iterate (tested in Acc, no conversion on the
                    // loop's critical path)
                    if (!isfinite(alpha)) break;
                    rho = rho_new;
                    const T bb = (T)beta;
#pragma unroll
                    for (int j = 0; j < RPT; ++j) {
                        p[j] = z[j] + bb * p[j];
                        sv[j] = w[j] + bb * sv[j];
                    }
                }
                if (act) {
#pragma unroll
                    for (int j = 0; j < RPT; ++j) lam[(k + 1) * n + i0 + j * TPB] = x[j];
                }
            }
        } else {
#pragma unroll
            for (int j = 0; j < RPT; ++j) {
                p[j] = z[j];
                part += act ? (Acc)r[j] * (Acc)z[j] : Acc(0);
            }
            Acc rho = rows_block_sum<Acc>(part, red);
            if (!(fabs((double)rho) < (double)abs_tol)) {
                const Acc rho_init = rho < 0 ? -rho : rho;
                for (int it = 0; it < bt.max_pcg_iters; ++it) {
                    ++iters;
                    if (act) {
#pragma unroll
                        for (int j = 0; j < RPT; ++j) pv[(k + 1) * VS + i0 + j * TPB] = p[j];
                    }
                    __syncthreads();
                    rows_window_dot(srow, pv + w0, ap);
                    part = 0;
#pragma unroll
                    for (int j = 0; j < RPT; ++j) part += act ? (Acc)p[j] * (Acc)ap[j] : Acc(0);
                    const Acc pap = rows_block_sum<Acc>(part, red);
                    if (pap == 0) break;
                    const T alpha = (T)(rho / pap);
#pragma unroll
                    for (int j = 0; j < RPT; ++j) {
                        x[j] += alpha * p[j];
                        r[j] -= alpha * ap[j];
                        if (act) {
                            rv[(k + 1) * VS + i0 + j * TPB] = r[j];
                            if constexpr (P32) rvf[(k + 1) * VS + i0 + j * TPB] = (float)r[j];
                        }
                    }
                    __syncthreads();
                    if constexpr (P32)
                        rows_window_dot(prow, rvf + w0, z);
                    else
                        rows_window_dot(prow, rv + w0, z);
                    part = 0;
#pragma unroll
                    for (int j = 0; j < RPT; ++j) part += act ? (Acc)r[j] * (Acc)z[j] : Acc(0);
                    const Acc rho_new = rows_block_sum<Acc>(part, red + WARP);
                    const Acc arn = rho_new < 0 ? -rho_new : rho_new;
                    if (arn < abs_tol + (Acc)eps * rho_init || arn == 0) break;
                    const T beta = (T)(rho_new / rho);
                    rho = rho_new;
#pragma unroll
                    for (int j = 0; j < RPT; ++j) p[j] = z[j] + beta * p[j];
                }
                if (act) {
#pragma unroll
                    for (int j = 0; j < RPT; ++j) lam[(k + 1) * n + i0 + j * TPB] = x[j];
                }
            }
        }
    }
    // step recovery (computeDzBatchedKernel, schur_linsys.cuh:312-431):
    // res_x = q_k - lambda_k + A_k^T lambda_{k+1}, dz_x = -Qi_k res_x,
    // res_u = r_k + B_k^T lambda_{k+1}, dz_u = -Ri_k res_u
    __syncthreads();
    if constexpr (PSM) {
        if (tid == 0 && !bt.conv[b]) mbar_inval(&s_pbar);  // both copies landed
    }
    if constexpr (HOOK) hook();
    if (act) {
#pragma unroll
        for (int j = 0; j < RPT; ++j) pv[(k + 1) * VS + i0 + j * TPB] = x[j];
    }
    __syncthreads();
    const bool dz_st = dz_ready();
    const T* Ab = dz_st ? Adz : bt.A + (size_t)b * N * n * n;
    const T* Qib = dz_st ? Qidz : bt.Qi + (size_t)b * N * n * n;
    const T* lk1 = pv + (k + 2) * VS;
    T res[RPT], resu[RPT];
#pragma unroll
    for (int j = 0; j < RPT; ++j) {
        res[j] = T(0);
        resu[j] = T(0);
        const int i = i0 + j * TPB;
        if (act) {
            const T* A = Ab + (size_t)k * n * n;
            T acc = T(0);
            if (k < N - 1) {
#pragma unroll
                for (int t = 0; t < n; ++t) acc += lk1[t] * A[i * n + t];
            }
            res[j] = bt.q[((size_t)b * N + k) * n + i] - x[j] + acc;
            bt.q[((size_t)b * N + k) * n + i] = res[j];
            if (i < m) {
                if (k < N - 1) {
                    const T* Bm = bt.Bm + ((size_t)b * N + k) * n * m;
                    T accu = T(0);
#pragma unroll
                    for (int t = 0; t < n; ++t) accu += lk1[t] * Bm[i * n + t];
                    resu[j] = bt.r[((size_t)b * N + k) * m + i] + accu;
                }
                bt.r[((size_t)b * N + k) * m + i] = resu[j];
            }
        }
    }
    __syncthreads();
    if (act) {
#pragma unroll
        for (int j = 0; j < RPT; ++j) {
            const int i = i0 + j * TPB;
            rv[(k + 1) * VS + i] = res[j];
            if (i < m) pv[k * m + i] = resu[j];  // lambda is no longer read
        }
    }
    __syncthreads();
    if (act) {
#pragma unroll
        for (int j = 0; j < RPT; ++j) {
            const int i = i0 + j * TPB;
            const T* Qi = Qib + (size_t)k * n * n;
            const T* rk = rv + (k + 1) * VS;
            T acc = T(0);
#pragma unroll
            for (int t = 0; t < n; ++t) acc += Qi[t * n + i] * rk[t];
            T* dzk = bt.dz + (size_t)b * d.traj() + k * (n + m);
            dzk[i] = -acc;
            if (i < m && k < N - 1) {
                const T* Ri = bt.Ri + ((size_t)b * N + k) * m * m;
                const T* ru = pv + k * m;
                T accu = T(0);
#pragma unroll
                for (int t = 0; t < m; ++t) accu += Ri[t * m + i] * ru[t];
                dzk[n + i] = -accu;
            }
        }
    }
    if (tid == 0) {
        bt.pcg_iters[b] = iters;
        if (bt.h_pcg) bt.h_pcg[(size_t)it_row * bt.B + b] = iters;
    }
}

template <int NQ, typename T, typename Acc, int RPT>
__global__ void __launch_bounds__(RowPcg<NQ, RPT>::MAX_THREADS, 1)
    k_pcg_rows(Batch<NQ, T> bt, int it_row)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    pcg_rows_body<NQ, T, Acc, RPT>(bt, blockIdx.x, it_row, smem_raw);
}

// FP64 k_pcg_rows with P^-1 applied in FP32 (gato_set_fp32_preconditioner)
template <int NQ>
__global__ void __launch_bounds__(RowPcg<NQ, 2>::MAX_THREADS, 1)
    k_pcg_rows_p32(Batch<NQ, double> bt, int it_row)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    pcg_rows_body<NQ, double, double, 2, NoHook, NoDzStage, true, true>(bt, blockIdx.x, it_row,
                                                                         smem_raw);
}

// Persistent FP32 form of k_pcg_rows: one CTA per SM takes problems from a
// counter (bt.work[0]).  When a problem's CG loop ends, the CTA claims the
// next problem and the bulk-copy engine brings its S and P^-1 (2 x 12 N NQ^2
// floats, contiguous per problem) into shared memory while the CTA computes
// the step dz, so the matrices load from shared memory instead of as strided
// rows from HBM.  With dz_stage, a second copy (own mbarrier) brings the
// problem's A_k and Qi_k blocks when its CG loop starts, for the step
// recovery after it; each thread waits on it with its own bound and reads
// global memory if that expires.  Claiming at the end rather than the start of a problem
// keeps the assignment as adaptive as the hardware's block scheduling (the
// early claim cost the adjoint's long, uneven CG runs 8 %).  Per-problem arithmetic is that of
// k_pcg_rows.  Thread 0 alone waits on the copy's mbarrier, with a bound
// (bt.wait_tries); the outcome goes through shared memory so that every
// thread takes the same branch.
// Expired waits set bt.work[2] (the host reports GATO_ERR_TIMEOUT; the
// results of that launch are not valid) and never leave a copy in flight:
//   - S / P^-1: thread 0 waits again, with PCG_STAGE_DRAIN_TRIES, for the
//     copies it issued to land, then the CTA ends;
//   - A_k / Qi_k (bt.wait_tries_dz): the threads that gave up read global
//     memory, the CTA issues no further step-recovery copies (no re-arm of
//     a barrier whose phase may be pending, no parity flip for a phase not
//     seen complete), and before the CTA ends thread 0 waits for the last
//     such copy it issued and did not see land.
template <int NQ>
struct PcgStage {
    __host__ __device__ static size_t matrix_floats(int N) { return (size_t)12 * N * NQ * NQ; }
    __host__ __device__ static size_t block_floats(int N) { return (size_t)4 * N * NQ * NQ; }  // N n x n
    __host__ __device__ static size_t smem_bytes_dz(int N)
    {
        return smem_bytes(N) + 2 * block_floats(N) * sizeof(float);
    }
    __host__ __device__ static size_t offset(int N)
    {
        return (RowPcg<NQ, 2>::template smem_bytes<float>(N) + 127) & ~(size_t)127;
    }
    __host__ __device__ static size_t smem_bytes(int N)
    {
        return offset(N) + 2 * matrix_floats(N) * sizeof(float);
    }
};


template <int NQ, typename Acc>
__global__ void __launch_bounds__(RowPcg<NQ, 2>::MAX_THREADS, 1)
    k_pcg_rows_stream(Batch<NQ, float> bt, int it_row, int dz_stage)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];  // stage offset 128-aligned
    __shared__ __align__(8) uint64_t bar, bar_dz;
    __shared__ int s_next, s_ok, s_dz_dead;
    if (*bt.done) return;
    const int N = bt.N, B = bt.B, tid = threadIdx.x;
    const size_t mat = PcgStage<NQ>::matrix_floats(N);
    float* stS = reinterpret_cast<float*>(smem_raw + PcgStage<NQ>::offset(N));
    float* stP = stS + mat;
    const uint32_t bytes = (uint32_t)(mat * sizeof(float));
    const size_t blk = PcgStage<NQ>::block_floats(N);
    float* stA = stP + mat;
    float* stQi = stA + blk;
    const uint32_t blk_bytes = (uint32_t)(blk * sizeof(float));
    uint32_t parity_dz = 0;
    bool dz_outstanding = false;  // thread 0: a step-recovery copy it has not seen land
    auto fetch = [&](int pb) {  // thread 0; earlier reads of the stage are behind a barrier
        fence_proxy_async_shared();
        mbar_arrive_expect_tx(&bar, 2 * bytes);
        bulk_copy_g2s(stS, bt.S + (size_t)pb * mat, bytes, &bar);
        bulk_copy_g2s(stP, bt.P + (size_t)pb * mat, bytes, &bar);
    };
    int b = blockIdx.x;
    if (tid == 0) {
        mbar_init(&bar, 1);
        mbar_init(&bar_dz, 1);
        fence_mbar_init();
        s_dz_dead = 0;
        if (b < B) fetch(b);
    }
    uint32_t parity = 0;
    while (b < B) {
        __syncthreads();  // the previous problem is done with the vectors and s_next
        if (tid == 0) s_ok = mbar_wait_bounded(&bar, parity, bt.wait_tries);
        __syncthreads();
        if (!s_ok) {
            if (tid == 0) {
                atomicExch(bt.work + 2, 1);
                mbar_wait_bounded(&bar, parity, PCG_STAGE_DRAIN_TRIES);  // let the copies land
            }
            break;
        }
        if (tid != 0) mbar_try_wait(&bar, parity);  // phase complete: acquires the data
        parity ^= 1;
        // a step-recovery wait that expired (any thread, previous problem,
        // behind the barrier above) turns the step-recovery copies off
        const bool dz_on = dz_stage && !s_dz_dead;
        if (dz_on && tid == 0) {  // the previous problem's dz reads are behind a barrier
            fence_proxy_async_shared();
            mbar_arrive_expect_tx(&bar_dz, 2 * blk_bytes);
            bulk_copy_g2s(stA, bt.A + (size_t)b * blk, blk_bytes, &bar_dz);
            bulk_copy_g2s(stQi, bt.Qi + (size_t)b * blk, blk_bytes, &bar_dz);
            dz_outstanding = true;
        }
        auto dz_ready = [&]() {
            if (!dz_on) return false;
            if (mbar_wait_bounded(&bar_dz, parity_dz, bt.wait_tries_dz)) {
                parity_dz ^= 1;
                if (tid == 0) dz_outstanding = false;
                return true;
            }
            atomicExch(bt.work + 2, 1);
            s_dz_dead = 1;
            return false;
        };
        auto next = [&]() {
            if (tid == 0) {
                const int nb = (int)gridDim.x + atomicAdd(bt.work, 1);
                s_next = nb;
                if (nb < B) fetch(nb);
            }
        };
        pcg_rows_body<NQ, float, Acc, 2>(bt, b, it_row, smem_raw, stS, stP, next, stA, stQi,
                                         dz_ready);
        __syncthreads();
        b = s_next;
    }
    if (tid == 0 && dz_outstanding) mbar_wait_bounded(&bar_dz, parity_dz, PCG_STAGE_DRAIN_TRIES);
    if (tid == 0 && atomicAdd(bt.work + 1, 1) == (int)gridDim.x - 1) {
        bt.work[0] = 0;  // last CTA out: ready for the next launch
        bt.work[1] = 0;
    }
}

// ------------------------------------------------------------------ dz
template <int NQ, typename T>
__global__ void k_dz(Batch<NQ, T> bt)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);
    const int b = blockIdx.y;
    const int wpb = blockDim.x / WARP;
    const int k = blockIdx.x * wpb + warp_id();
    const int N = bt.N;
    if (k >= N) return;
    const Dims<NQ> d{N};
    constexpr int nx = Dims<NQ>::nx, nu = Dims<NQ>::nu;
    T* s = smem + warp_id() * 3 * nx;
    dz_knot<NQ, T>(N, k, bt.lambda + (size_t)b * d.vecp(), bt.Qi + (size_t)b * N * nx * nx,
                bt.Ri + (size_t)b * N * nu * nu, bt.q + (size_t)b * N * nx,
                bt.r + (size_t)b * N * nu, bt.A + (size_t)b * N * nx * nx,
                bt.Bm + (size_t)b * N * nx * nu, bt.dz + (size_t)b * d.traj(), s);
}

// ------------------------------------------------------------------ fused
// Convergence bookkeeping of one SQP iteration, one block
// (gato/bsqp/bsqp.cuh:141-167 run on the device): a problem whose PCG took
// zero iterations is converged; the batch is done once the converged count
// reaches B * solve_ratio.
template <int NQ, typename T>
__device__ __forceinline__ void check_body(const Batch<NQ, T>& bt)
{
    __shared__ int s_count;
    if (threadIdx.x == 0) s_count = 0;
    __syncthreads();
    if (*bt.done) return;
    int local = 0;
    for (int b = threadIdx.x; b < bt.B; b += blockDim.x) {
        int cv = bt.conv[b];
        int si = bt.sqp_iters[b];
        if (!cv && bt.pcg_iters[b] >= bt.max_pcg_iters) bt.status[b] |= GATO_STATUS_PCG_MAX_ITER;
        if (bt.pcg_iters[b] == 0) {
            cv = 1;
            si += 1;
        }
        if (cv) local++;
        else si += 1;
        bt.conv[b] = cv;
        bt.sqp_iters[b] = si;
    }
    atomicAdd(&s_count, local);
    __syncthreads();
    if (threadIdx.x == 0) {
        if ((float)s_count >= (float)bt.B * bt.solve_ratio) *bt.done = 1;
        else *bt.ls_count += 1;
    }
}

template <int NQ, typename T>
__global__ void k_check(Batch<NQ, T> bt)
{
    check_body<NQ, T>(bt);
}

// Shared memory of the fused SQP-iteration kernel.
template <int NQ, typename T>
struct FusedLayout {
    int N, warps;
    bool stage;  // S and P^-1 resident in shared memory
    __host__ __device__ size_t scratch_floats() const
    {
        int a = 2 * KktSmem<NQ>::SIZE, bsz = SchurSmem<NQ>::SIZE, c = 4 * (2 * NQ) * (2 * NQ);
        int m = a > bsz ? a : bsz;
        m = m > c ? m : c;
        return (size_t)warps * m;
    }
    __host__ __device__ size_t mats_floats() const
    {
        const Dims<NQ> d{N};
        return stage ? 2 * (size_t)d.b3d() : 0;
    }
    __host__ __device__ size_t vec_floats() const
    {
        const Dims<NQ> d{N};
        return 5 * (size_t)d.vecp();
    }
    __host__ __device__ size_t bytes() const
    {
        // scratch and the PCG vectors are not live at the same time
        size_t s = scratch_floats(), v = vec_floats();
        return (mats_floats() + (s > v ? s : v)) * sizeof(T) + 2 * WARP * sizeof(double) + 16;
    }
};

// One SQP iteration of one problem up to the step (KKT set-up, Schur
// complement, PCG, step recovery), one block.  With with_pcg = 0 it stops
// after the Schur complement (S, P^-1 and gamma left in global memory) and
// k_pcg_rows takes over.
// A group of consecutive warps of a CTA that works on one problem, with its
// own barrier: the whole CTA (barrier 0, __syncthreads) or a fixed slice of
// it synchronised by a named barrier.
struct Team {
    int tid, nthreads, warp, nwarps, bar;
    __device__ static Team cta()
    {
        return Team{(int)threadIdx.x, (int)blockDim.x, warp_id(), (int)(blockDim.x / WARP), 0};
    }
    // slice t of `count` equal slices of the CTA
    __device__ static Team slice(int t, int count)
    {
        const int nt = blockDim.x / count;
        return Team{(int)threadIdx.x - t * nt, nt, warp_id() - t * (nt / WARP), nt / WARP, 1 + t};
    }
    __device__ __forceinline__ void sync() const
    {
        if (bar == 0)
            __syncthreads();
        else
            asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(nthreads) : "memory");
    }
};

// KG: lanes per knot in the KKT stage (16: two knots per warp, 32: one).
// `team` is the set of warps working on this problem (the whole CTA, or half
// of it when a CTA runs two problems at once); with_pcg needs the whole CTA.
// KKT_STAGE / SCHUR_STAGE compile the KKT set-up and the Schur stage (with
// the PCG when with_pcg) in or out, so a kernel that runs one of them is
// allocated the registers of that one alone.
template <int NQ, typename T, typename Acc, int KG = 16, bool KKT_STAGE = true,
          bool SCHUR_STAGE = true>
__device__ __forceinline__ void fused_iter_body(const Batch<NQ, T>& bt, const DevModel<NQ, T>& M,
                                                int b, int stage, int it_row, int with_pcg,
                                                unsigned char* smem_raw,
                                                const Team& team = Team::cta(),
                                                bool with_kkt = true)
{
    T* smem = reinterpret_cast<T*>(smem_raw);
    if (*bt.done) return;
    const int N = bt.N;
    const Dims<NQ> d{N};
    constexpr int nx = Dims<NQ>::nx, nu = Dims<NQ>::nu;
    const int nw = team.nwarps;
    const int wid = team.warp;
    FusedLayout<NQ, T> lay{N, nw, stage != 0};
    T* mats = smem;
    T* work = smem + lay.mats_floats();
    const size_t sc = lay.scratch_floats() / nw;
    T* ws = work + wid * sc;
    size_t wfl = lay.scratch_floats() > lay.vec_floats() ? lay.scratch_floats() : lay.vec_floats();
    Acc* red = reinterpret_cast<Acc*>(((uintptr_t)(work + wfl) + 15) & ~(uintptr_t)15);

    T* Q = bt.Q + (size_t)b * N * nx * nx;
    T* R = bt.R + (size_t)b * N * nu * nu;
    T* qv = bt.q + (size_t)b * N * nx;
    T* rv = bt.r + (size_t)b * N * nu;
    T* A = bt.A + (size_t)b * N * nx * nx;
    T* Bm = bt.Bm + (size_t)b * N * nx * nu;
    T* c = bt.c + (size_t)b * N * nx;
    T* Qi = bt.Qi + (size_t)b * N * nx * nx;
    T* Ri = bt.Ri + (size_t)b * N * nu * nu;
    T* S = stage ? mats : bt.S + (size_t)b * d.b3d();
    T* P = stage ? mats + d.b3d() : bt.P + (size_t)b * d.b3d();
    T* g = bt.gamma + (size_t)b * d.vecp();
    const T rho = bt.rho[b];
    const T* xu = bt.xu + (size_t)b * d.traj();
    const T* fext = bt.use_fext ? bt.fext + 6 * b : nullptr;

    // KKT set-up, two knots per warp (one per half-warp) or one per warp;
    // skipped when a knot-parallel KKT kernel already wrote the blocks
    if (!KKT_STAGE || !with_kkt) {
    } else if constexpr (KG == 32) {
        for (int k = wid; k < N - 1; k += nw)
            kkt_knot<NQ, T, 32>(M, cost_of<NQ>(bt.cp, b), N, k, xu, bt.xs + (size_t)b * nx,
                                bt.goal + (size_t)b * d.goal(), fext, Q, R, qv, rv, A, Bm, c,
                                ws, true);
    } else {
        const int half = lane_id() >> 4;
        const int npairs = N / 2;  // ceil((N - 1) / 2)
        for (int kp = wid; kp < npairs; kp += nw) {
            const int k = 2 * kp + half;
            const bool valid = k < N - 1;
            kkt_knot<NQ, T, 16>(M, cost_of<NQ>(bt.cp, b), N, valid ? k : N - 2, xu, bt.xs + (size_t)b * nx,
                                bt.goal + (size_t)b * d.goal(), fext, Q, R, qv, rv, A, Bm, c,
                                ws + half * KktSmem<NQ>::SIZE, valid);
        }
    }
    if constexpr (!SCHUR_STAGE) return;
    team.sync();
    for (int k = wid; k < N; k += nw) {
        warp_invert<nx, T>(Q + k * nx * nx, rho, Qi + k * nx * nx);
        if (k < N - 1) warp_invert<nu, T>(R + k * nu * nu, T(0), Ri + k * nu * nu);
    }
    if (stage) {
        // the padding blocks of S and P^-1 (row 0 left, row N-1 right) are zero
        for (int i = team.tid; i < nx * 3 * nx; i += team.nthreads) {
            const int y = i / (3 * nx), x = i % (3 * nx);
            if (x < nx) {
                S[y * 3 * nx + x] = 0.0f;
                P[y * 3 * nx + x] = 0.0f;
            } else if (x >= 2 * nx) {
                S[(size_t)(N - 1) * 3 * nx * nx + y * 3 * nx + x] = 0.0f;
                P[(size_t)(N - 1) * 3 * nx * nx + y * 3 * nx + x] = 0.0f;
            }
        }
    }
    team.sync();
    for (int k = wid; k < N; k += nw) {
        if (k == N - 1)
            schur_first<NQ, T>(rho, Q, Qi, qv, c, S, P, g);
        else
            schur_knot<NQ, T>(k, rho, Qi, Ri, qv, rv, A, Bm, c, S, P, g, ws);
    }
    team.sync();
    for (int k = wid; k < N - 1; k += nw) schur_offdiag<NQ, T>(k, S, P, ws);
    if (!with_pcg) return;  // k_pcg_rows continues from S, P^-1 in global memory
    team.sync();
    int iters = 0;
    if (!bt.conv[b])
        iters = pcg_block<NQ, T, Acc>(N, S, P, g, bt.lambda + (size_t)b * d.vecp(), bt.tol[b],
                                   bt.max_pcg_iters, work, red, bt.abs_tol);
    team.sync();
    for (int k = wid; k < N; k += nw)
        dz_knot<NQ, T>(N, k, bt.lambda + (size_t)b * d.vecp(), Qi, Ri, qv, rv, A, Bm,
                    bt.dz + (size_t)b * d.traj(), ws);
    if (team.tid == 0) {
        bt.pcg_iters[b] = iters;
        if (bt.h_pcg) bt.h_pcg[(size_t)it_row * bt.B + b] = iters;
    }
}

// Resident CTAs per SM: four in FP32 (64 registers), two in FP64 (128
// registers; both spill, and both are faster than fewer CTAs without spills:
// FP64 5.36 against 6.48 ms per solve with one CTA at 255 registers)
template <int NQ, typename T, typename Acc>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 2)
    k_fused_iter(Batch<NQ, T> bt, DevModel<NQ, T> M, int stage, int it_row, int with_pcg,
                 int with_kkt)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    fused_iter_body<NQ, T, Acc>(bt, M, blockIdx.x, stage, it_row, with_pcg, smem_raw,
                                Team::cta(), with_kkt != 0);
}

// The two halves of k_fused_iter as separate kernels (CTA per problem, same
// shared-memory layout): the KKT set-up, whose dynamics derivatives need the
// registers (FP32: two CTAs per SM, 128 registers, 720 B spilled; FP64: one,
// 255), and the Schur stage (FP32: four CTAs per SM at 64 registers without
// spills; FP64: two).  The KKT blocks pass through L2 between them.  Against
// the one kernel that does both (FP32 at 64 registers, 2 KB spilled; FP64 at
// 128, 3.8 KB), iiwa14 N = 32 B = 1024, per solve: FP32 2.33 -> 2.03 ms,
// FP64 5.42 -> 3.81 ms; the KKT half at three CTAs per SM (80 registers):
// FP32 2.18 ms; the FP64 KKT half at two CTAs (128 registers, 3.9 KB
// spilled): 4.66 against 3.82 ms.
template <int NQ, typename T, typename Acc>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 2 : 1)
    k_fused_kkt(Batch<NQ, T> bt, DevModel<NQ, T> M, int it_row)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    fused_iter_body<NQ, T, Acc, 16, true, false>(bt, M, blockIdx.x, 0, it_row, 0, smem_raw);
}
template <int NQ, typename T, typename Acc>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 2)
    k_fused_schur(Batch<NQ, T> bt, DevModel<NQ, T> M, int it_row)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    fused_iter_body<NQ, T, Acc, 16, false, true>(bt, M, blockIdx.x, 0, it_row, 0, smem_raw,
                                                  Team::cta(), false);
}

}  // namespace gato
