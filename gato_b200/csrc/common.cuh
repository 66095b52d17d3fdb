// Shared device-side definitions: the robot model as a by-value kernel
// parameter, solver dimensions, and warp helpers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/gato_b200.h"  // status bits shared with the host

namespace gato {

constexpr int WARP = 32;
constexpr unsigned FULL = 0xffffffffu;
constexpr int NUM_ALPHAS = 8;  // parallel line-search step sizes 2^-j (gato/settings.h:15)

// Penalty adaptation constants of gato/settings.h:17-21 (float in the
// reference).
constexpr float RHO_INIT = 1e-3f;
constexpr float RHO_FACTOR = 1.2f;
constexpr float RHO_MIN = 1e-8f;
constexpr float RHO_MAX = 10.0f;

// Robot model for a chain of NQ revolute joints about their local z axes.
// Built on the host in FP64 from gato_model_t and rounded to FP32.
//   X_i(q) = rot(Rz(q)^T) * [E0 0; C0 E0]   (motion transform parent -> link)
//   FK:   T_i = T_{i-1} * [R0 Rz(q) | P]
template <int NQ, typename T>
struct DevModel {
    T E0[NQ][9];   // row-major rotation block of the fixed joint transform
    T C0[NQ][9];   // row-major coupling block (-E0 * skew(P))
    T R0[NQ][9];   // row-major joint-frame rotation in the parent (E0^T)
    T P[NQ][3];    // joint origin in the parent frame
    T Ibar[NQ][6]; // rotational inertia about the link origin: xx xy xz yy yz zz
    T h[NQ][3];    // first mass moment m * com
    T mass[NQ];
    T qlo[NQ], qhi[NQ], vlo[NQ], vhi[NQ], ulo[NQ], uhi[NQ];
    T gravity;
    int barrier_style;  // 0 exact barrier Hessian, 1 outer product of gradients
};

// Cost weights and time step, as in the BSQP constructor.  `wdiag`, when
// set, holds one problem's diagonal state and control weights
// [Qd_0..Qd_{nx-1}, Rd_0..Rd_{nu-1}]: the cost gains 1/2 Qd_i x_i^2 on every
// state entry and 1/2 Rd_i u_i^2 on every control, replacing the uniform
// qd_cost (velocities) and u_cost.  With Qd = [0, qd_cost], Rd = u_cost it is
// the reference's cost (iiwa14_plant.cuh:275-424).
template <typename T>
struct CostParams {
    T dt;
    T q_cost, qd_cost, u_cost, N_cost, q_lim_cost, vel_lim_cost, ctrl_lim_cost;
    const T* wdiag;
};

// the cost parameters of problem b (offsets the per-problem weights)
template <int NQ, typename T>
__device__ __forceinline__ CostParams<T> cost_of(const CostParams<T>& cp, int b)
{
    CostParams<T> c = cp;
    if (c.wdiag) c.wdiag += (size_t)b * 3 * NQ;
    return c;
}

// precision-generic math
__device__ __forceinline__ void gsincos(float x, float* s, float* c) { sincosf(x, s, c); }
__device__ __forceinline__ void gsincos(double x, double* s, double* c) { sincos(x, s, c); }
__device__ __forceinline__ float glog(float x) { return logf(x); }
__device__ __forceinline__ double glog(double x) { return log(x); }
__device__ __forceinline__ float gabs(float x) { return fabsf(x); }
__device__ __forceinline__ double gabs(double x) { return fabs(x); }
__device__ __forceinline__ float gmin(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ double gmin(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ float gmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double gmax(double a, double b) { return fmax(a, b); }

// Per-problem sizes for a plant with NQ joints and horizon N.
template <int NQ>
struct Dims {
    static constexpr int nq = NQ;
    static constexpr int nx = 2 * NQ;
    static constexpr int nu = NQ;
    static constexpr int nxu = nx + nu;
    static constexpr int nx2 = nx * nx;
    int N;
    __host__ __device__ int traj() const { return nxu * N - nu; }
    __host__ __device__ int vecp() const { return (N + 2) * nx; }   // padded lambda / gamma
    __host__ __device__ int b3d() const { return 3 * nx2 * N; }     // S / Pinv block rows
    __host__ __device__ int goal() const { return 6 * N; }
};

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ int warp_id() { return threadIdx.x >> 5; }

__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}


// ------------------------------------------------------------ bulk copies
// One-dimensional bulk copy global -> shared memory of this CTA, completed on
// an mbarrier (sm_90+ PTX).  Addresses 16-byte aligned, size a multiple of 16.
__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}
// makes an mbarrier's initialisation visible to the bulk-copy engine
__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// orders this thread's earlier shared-memory accesses before later bulk copies
__device__ __forceinline__ void fence_proxy_async_shared()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes,
                                              uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
// true once the phase with the given parity has completed; a call suspends
// the thread for at most about 1 us while it waits
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity), "r"(1000u)
        : "memory");
    return ok != 0;
}
// true once the phase completes, with at most `tries` try_wait calls (0: gives
// up at once without looking)
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int tries)
{
    for (int i = 0; i < tries; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// ends an mbarrier's life (before its memory is initialised again); every
// phase it tracked must have completed
__device__ __forceinline__ void mbar_inval(uint64_t* bar)
{
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

}  // namespace gato
