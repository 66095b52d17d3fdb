// Mixed batches: problems of several plants and horizons solved together
// (no counterpart in the reference, which compiles one module per plant and
// horizon and one class per power-of-two batch).  Problems are grouped into
// classes (plant, N), each with its own solver buffers; every stage of an SQP
// iteration is ONE persistent launch over all classes: each CTA takes the
// next problem from a device work queue (an atomic counter over a list of
// (class, problem) items sorted longest-first) until the list is exhausted,
// so classes of very different cost share the SMs without a tail per class.
// Long horizons (N beyond one CTA's registers) take the cluster PCG, one
// launch per class, on a parallel branch of the solve graph.
#pragma once

#include "kernels.cuh"

namespace gato {

constexpr int MULTI_MAX_CLASSES = 8;

template <typename T>
struct MultiArgs {
    int nitems;
    const int2* items;  // (class, problem), longest first
    int* head;          // this launch's work-queue counter (zeroed per solve)
    int nq[MULTI_MAX_CLASSES];
    Batch<7, T> b7[MULTI_MAX_CLASSES];
    Batch<6, T> b6[MULTI_MAX_CLASSES];
    DevModel<7, T> m7;
    DevModel<6, T> m6;
};

// next work item for a team (or the whole CTA), or -1 when the queue is empty
__device__ __forceinline__ int queue_next(int* head, int nitems, int* s_item, const Team& team)
{
    team.sync();  // the team has read the previous item
    if (team.tid == 0) *s_item = atomicAdd(head, 1);
    team.sync();
    const int it = *s_item;
    return it < nitems ? it : -1;
}
__device__ __forceinline__ int queue_next(int* head, int nitems, int* s_item)
{
    return queue_next(head, nitems, s_item, Team::cta());
}

// KKT blocks of every queued problem (to global memory).  KG lanes per knot;
// PPB problems per CTA at a time (the CTA's warps split into PPB teams that
// pull work independently, each with team_bytes of shared memory); MINB
// CTAs per SM in FP32 (registers traded for resident warps).
template <typename T, typename Acc, int KG, int PPB, int MINB>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? MINB : 1)
    k_q_kkt(MultiArgs<T> ma, int it_row, int team_bytes)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_item[PPB];
    const int t = PPB == 1 ? 0 : warp_id() / ((int)(blockDim.x / WARP) / PPB);
    const Team team = PPB == 1 ? Team::cta() : Team::slice(t, PPB);
    unsigned char* sm = smem_raw + (size_t)t * team_bytes;
    for (;;) {
        const int it = queue_next(ma.head, ma.nitems, &s_item[t], team);
        if (it < 0) break;
        const int2 w = ma.items[it];
        if (ma.nq[w.x] == 7)
            fused_iter_body<7, T, Acc, KG, true, false>(ma.b7[w.x], ma.m7, w.y, 0, it_row, 0, sm,
                                                        team);
        else
            fused_iter_body<6, T, Acc, KG, true, false>(ma.b6[w.x], ma.m6, w.y, 0, it_row, 0, sm,
                                                        team);
    }
}

// Schur system of every queued problem (S, P^-1, gamma to global memory)
// from the blocks k_q_kkt left there: the two halves of the SQP iteration's
// set-up as separate launches, each compiled for its own occupancy, as
// k_fused_kkt and k_fused_schur are for one class (four CTAs per SM in
// FP32, two in FP64).
template <typename T, typename Acc>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 2)
    k_q_schur(MultiArgs<T> ma, int it_row)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_item;
    for (;;) {
        const int it = queue_next(ma.head, ma.nitems, &s_item);
        if (it < 0) break;
        const int2 w = ma.items[it];
        if (ma.nq[w.x] == 7)
            fused_iter_body<7, T, Acc, 16, false, true>(ma.b7[w.x], ma.m7, w.y, 0, it_row, 0,
                                                        smem_raw, Team::cta(), false);
        else
            fused_iter_body<6, T, Acc, 16, false, true>(ma.b6[w.x], ma.m6, w.y, 0, it_row, 0,
                                                        smem_raw, Team::cta(), false);
    }
}

// register-resident PCG + step of every queued short-horizon problem
template <typename T, typename Acc>
__global__ void __launch_bounds__(RowPcg<7, pcg_rows_per_thread<T>()>::MAX_THREADS, 1)
    k_q_pcg_rows(MultiArgs<T> ma, int it_row)
{
    constexpr int RPT = pcg_rows_per_thread<T>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_item;
    for (;;) {
        const int it = queue_next(ma.head, ma.nitems, &s_item);
        if (it < 0) break;
        const int2 w = ma.items[it];
        if (ma.nq[w.x] == 7)
            pcg_rows_body<7, T, Acc, RPT>(ma.b7[w.x], w.y, it_row, smem_raw);
        else
            pcg_rows_body<6, T, Acc, RPT>(ma.b6[w.x], w.y, it_row, smem_raw);
    }
}

// merit / line search of every queued problem (mode as in k_merit_ls)
template <typename T, typename Acc>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 2 : 1) k_q_merit_ls(MultiArgs<T> ma, int mode, int it_row)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_item;
    for (;;) {
        const int it = queue_next(ma.head, ma.nitems, &s_item);
        if (it < 0) break;
        const int2 w = ma.items[it];
        if (ma.nq[w.x] == 7)
            merit_ls_body<7, T, Acc>(ma.b7[w.x], ma.m7, w.y, mode, it_row, smem_raw);
        else
            merit_ls_body<6, T, Acc>(ma.b6[w.x], ma.m6, w.y, mode, it_row, smem_raw);
    }
}

// convergence bookkeeping, one CTA per class
template <typename T>
__global__ void k_q_check(MultiArgs<T> ma)
{
    const int c = blockIdx.x;
    if (ma.nq[c] == 7)
        check_body<7, T>(ma.b7[c]);
    else
        check_body<6, T>(ma.b6[c]);
}

}  // namespace gato
