// Register-resident PCG for long horizons: one thread-block cluster per
// problem.  The S and P^-1 rows of N knots do not fit one SM's registers
// beyond N ~ 36 (iiwa14), so the block rows are split across a cluster of
// C = ceil(N / 32) CTAs (C <= 8; FP64 ceil(N / 16)), each holding up to 32
// (16) block rows exactly as k_pcg_rows does.  CG vectors live in each CTA's shared memory with one halo
// block on each side; the owner of a boundary block also stores it into the
// neighbour CTA's halo through distributed shared memory, and a cluster
// barrier publishes it.  Reductions sum per CTA, every CTA writes its partial
// into every CTA's slot array, and after a cluster barrier each CTA adds the
// C partials in rank order, so all CTAs take bitwise the same stopping
// decision (the cluster barriers stay matched).  Same iteration as
// k_pcg_rows (pcg.cuh:23-147); step recovery follows in the kernel.
#pragma once

#include <cooperative_groups.h>

#include "kernels.cuh"

namespace gato {

template <int NQ, int RPT>
struct ClusterPcg {
    static constexpr int n = 2 * NQ, m = NQ, RD = 3 * n, VS = row_vs(n);
    static constexpr int TPB = n / RPT;
    // block rows per CTA: 32 with two rows a thread (FP32); 16 with one (FP64),
    // so that a thread's S and P^-1 rows (2 x 42 doubles for iiwa14) stay
    // within 255 registers at 224 threads
    static constexpr int MAX_ROWS = RPT == 1 ? 16 : 32;
    static constexpr int MAX_THREADS = 256;
    static constexpr int MAX_CLUSTER = 8;  // portable cluster size
    __host__ __device__ static int ctas(int N) { return (N + MAX_ROWS - 1) / MAX_ROWS; }
    __host__ __device__ static int rows(int N)
    {
        const int C = ctas(N);
        return (N + C - 1) / C;
    }
    __host__ __device__ static int threads(int N) { return ((rows(N) * TPB + 31) / 32) * 32; }
    __host__ __device__ static bool fits(int N)
    {
        const int C = ctas(N);
        return C >= 1 && C <= MAX_CLUSTER && (C - 1) * rows(N) < N;
    }
    template <typename T>
    __host__ __device__ static size_t smem_bytes(int N)
    {
        return 2 * (size_t)(rows(N) + 2) * VS * sizeof(T) +
               (2 * WARP + 2 * MAX_CLUSTER) * sizeof(double) + 32;
    }
};

template <int NQ, typename T, typename Acc, int RPT>
__global__ void __launch_bounds__(ClusterPcg<NQ, RPT>::MAX_THREADS, 1)
    k_pcg_cluster(Batch<NQ, T> bt, int it_row)
{
    namespace cg = cooperative_groups;
    using CP = ClusterPcg<NQ, RPT>;
    constexpr int n = CP::n, m = CP::m, RD = CP::RD, VS = CP::VS, TPB = CP::TPB;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cg::cluster_group cl = cg::this_cluster();
    const int C = (int)cl.num_blocks();
    const int c = (int)cl.block_rank();
    const int b = blockIdx.x / C;
    if (*bt.done) return;  // written by an earlier kernel: the same for the whole cluster
    const int N = bt.N;
    const Dims<NQ> d{N};
    const int KB = CP::rows(N);
    const int r0 = c * KB;
    const int KBc = (N - r0) < KB ? (N - r0) : KB;  // block rows of this CTA
    const int tid = threadIdx.x;
    const bool act = tid < KBc * TPB;
    const int lk = act ? tid / TPB : 0, i0 = act ? tid % TPB : 0;
    const int k = r0 + lk;  // global block row
    const int L = (KB + 2) * VS;
    T* pv = reinterpret_cast<T*>(smem_raw);
    T* rv = pv + L;
    Acc* red = reinterpret_cast<Acc*>(((uintptr_t)(rv + L) + 15) & ~(uintptr_t)15);
    Acc* cred = red + 2 * WARP;  // [2][MAX_CLUSTER] partials of every CTA
    for (int j = tid; j < 2 * L; j += blockDim.x) pv[j] = T(0);
    __syncthreads();
    cl.sync();  // every CTA's halos are zero before any neighbour writes them

    // own block into local smem, boundary blocks into the neighbours' halos
    auto exchange = [&](T* buf, const T* val) {
        if (act) {
#pragma unroll
            for (int j = 0; j < RPT; ++j) {
                const int i = i0 + j * TPB;
                buf[(lk + 1) * VS + i] = val[j];
                if (lk == 0 && c > 0) cl.map_shared_rank(buf, c - 1)[(KB + 1) * VS + i] = val[j];
                if (lk == KBc - 1 && c < C - 1) cl.map_shared_rank(buf, c + 1)[i] = val[j];
            }
        }
        cl.sync();
    };
    // cluster-wide sums of two values, added in rank order on every CTA
    auto csum2 = [&](Acc& a, Acc& e) {
        a = warp_sum(a);
        e = warp_sum(e);
        if (lane_id() == 0) {
            red[warp_id()] = a;
            red[WARP + warp_id()] = e;
        }
        __syncthreads();
        if (tid == 0) {
            Acc sa = 0, se = 0;
            const int nw = blockDim.x / WARP;
            for (int w = 0; w < nw; ++w) {
                sa += red[w];
                se += red[WARP + w];
            }
            for (int q = 0; q < C; ++q) {
                Acc* rem = cl.map_shared_rank(cred, q);
                rem[c] = sa;
                rem[CP::MAX_CLUSTER + c] = se;
            }
        }
        cl.sync();
        Acc sa = 0, se = 0;
        for (int q = 0; q < C; ++q) {
            sa += cred[q];
            se += cred[CP::MAX_CLUSTER + q];
        }
        a = sa;
        e = se;
    };

    T* lam = bt.lambda + (size_t)b * d.vecp();
    const int w0 = lk * VS;
    int iters = 0;
    T x[RPT];
#pragma unroll
    for (int j = 0; j < RPT; ++j) x[j] = act ? lam[(k + 1) * n + i0 + j * TPB] : T(0);
    if (!bt.conv[b]) {  // per problem: the same on every CTA of the cluster
        RowMat<NQ, RPT, T> srow, prow;
        {
            const size_t row = (size_t)b * d.b3d() + (size_t)(k * n + i0) * RD;
            srow.load(bt.S + row, (size_t)TPB * RD, act);
            prow.load(bt.P + row, (size_t)TPB * RD, act);
        }
        T g[RPT], r[RPT], z[RPT], p[RPT], w[RPT];
#pragma unroll
        for (int j = 0; j < RPT; ++j)
            g[j] = act ? bt.gamma[(size_t)b * d.vecp() + (k + 1) * n + i0 + j * TPB] : T(0);
        exchange(pv, x);
        rows_window_dot(srow, pv + w0, r);
#pragma unroll
        for (int j = 0; j < RPT; ++j) r[j] = act ? g[j] - r[j] : T(0);
        exchange(rv, r);
        rows_window_dot(prow, rv + w0, z);
        const Acc abs_tol = Acc(bt.abs_tol);
        const T eps = bt.tol[b];
        if constexpr (sizeof(T) == 4) {
            // single-reduction recurrence, as in k_pcg_rows
            T sv[RPT];
            exchange(pv, z);
            rows_window_dot(srow, pv + w0, w);
            Acc rho = 0, delta = 0;
#pragma unroll
            for (int j = 0; j < RPT; ++j) {
                rho += act ? (Acc)r[j] * (Acc)z[j] : Acc(0);
                delta += act ? (Acc)z[j] * (Acc)w[j] : Acc(0);
            }
            csum2(rho, delta);
            if (!(fabs((double)rho) < (double)abs_tol)) {
                const Acc rho_init = rho < 0 ? -rho : rho;
                Acc alpha = rec_div(rho, delta);
                const bool start = !(delta == 0);  // delta = 0: nothing to do
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
                    }
                    exchange(rv, r);
                    rows_window_dot(prow, rv + w0, z);
                    exchange(pv, z);
                    rows_window_dot(srow, pv + w0, w);
                    Acc rho_new = 0;
                    delta = 0;
#pragma unroll
                    for (int j = 0; j < RPT; ++j) {
                        rho_new += act ? (Acc)r[j] * (Acc)z[j] : Acc(0);
                        delta += act ? (Acc)z[j] * (Acc)w[j] : Acc(0);
                    }
                    csum2(rho_new, delta);
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
            // the reference's two-reduction recurrence
            Acc rho = 0, unused = 0;
#pragma unroll
            for (int j = 0; j < RPT; ++j) {
                p[j] = z[j];
                rho += act ? (Acc)r[j] * (Acc)z[j] : Acc(0);
            }
            csum2(rho, unused);
            if (!(fabs((double)rho) < (double)abs_tol)) {
                const Acc rho_init = rho < 0 ? -rho : rho;
                for (int it = 0; it < bt.max_pcg_iters; ++it) {
                    ++iters;
                    exchange(pv, p);
                    rows_window_dot(srow, pv + w0, w);
                    Acc pap = 0;
                    unused = 0;
#pragma unroll
                    for (int j = 0; j < RPT; ++j) pap += act ? (Acc)p[j] * (Acc)w[j] : Acc(0);
                    csum2(pap, unused);
                    if (pap == 0) break;
                    const T alpha = (T)(rho / pap);
#pragma unroll
                    for (int j = 0; j < RPT; ++j) {
                        x[j] += alpha * p[j];
                        r[j] -= alpha * w[j];
                    }
                    exchange(rv, r);
                    rows_window_dot(prow, rv + w0, z);
                    Acc rho_new = 0;
                    unused = 0;
#pragma unroll
                    for (int j = 0; j < RPT; ++j) rho_new += act ? (Acc)r[j] * (Acc)z[j] : Acc(0);
                    csum2(rho_new, unused);
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
    // step recovery (computeDzBatchedKernel, schur_linsys.cuh:312-431), as in
    // k_pcg_rows; lambda_{k+1} of the last local row comes from the halo
    exchange(pv, x);
    const T* lk1 = pv + (lk + 2) * VS;
    T res[RPT], resu[RPT];
#pragma unroll
    for (int j = 0; j < RPT; ++j) {
        res[j] = T(0);
        resu[j] = T(0);
        const int i = i0 + j * TPB;
        if (act) {
            const T* A = bt.A + ((size_t)b * N + k) * n * n;
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
    __syncthreads();  // local only: no CTA touches another's memory from here on
    if (act) {
#pragma unroll
        for (int j = 0; j < RPT; ++j) {
            const int i = i0 + j * TPB;
            rv[(lk + 1) * VS + i] = res[j];
            if (i < m) pv[lk * m + i] = resu[j];
        }
    }
    __syncthreads();
    if (act) {
#pragma unroll
        for (int j = 0; j < RPT; ++j) {
            const int i = i0 + j * TPB;
            const T* Qi = bt.Qi + ((size_t)b * N + k) * n * n;
            const T* rk = rv + (lk + 1) * VS;
            T acc = T(0);
#pragma unroll
            for (int t = 0; t < n; ++t) acc += Qi[t * n + i] * rk[t];
            T* dzk = bt.dz + (size_t)b * d.traj() + k * (n + m);
            dzk[i] = -acc;
            if (i < m && k < N - 1) {
                const T* Ri = bt.Ri + ((size_t)b * N + k) * m * m;
                const T* ru = pv + lk * m;
                T accu = T(0);
#pragma unroll
                for (int t = 0; t < m; ++t) accu += Ri[t * m + i] * ru[t];
                dzk[n + i] = -accu;
            }
        }
    }
    if (c == 0 && tid == 0) {
        bt.pcg_iters[b] = iters;
        if (bt.h_pcg) bt.h_pcg[(size_t)it_row * bt.B + b] = iters;
    }
}

}  // namespace gato
