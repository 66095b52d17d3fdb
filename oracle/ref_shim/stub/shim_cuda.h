/*
 * Single-thread host emulation of the CUDA keywords used by the reference's
 * device headers, so that its GRiD dynamics, plant cost and integrator
 * functions compile with g++ in FP64.  Test infrastructure only: it builds the
 * reference itself into oracle/_ref as a checker for the oracle.
 *
 * One "thread" runs each block-strided loop serially (blockDim = 1).  Warp
 * shuffles return 0 (the identity of the sums they feed); they occur only in
 * the reference's PCG/dot helpers, which this build does not call.
 */
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#define __device__
#define __host__
#define __global__
#define __forceinline__ inline
#define __shared__
#define __launch_bounds__(...)

struct shim_uint3 {
    unsigned x, y, z;
};
extern shim_uint3 threadIdx, blockIdx, blockDim, gridDim;

inline void __syncthreads() {}
inline void __syncwarp(unsigned = 0xffffffffu) {}
inline unsigned __activemask() { return 1u; }
template <class T>
inline T __shfl_down_sync(unsigned, T, unsigned) { return T(0); }
template <class T>
inline T atomicAdd(T* a, T v)
{
    T old = *a;
    *a += v;
    return old;
}
using std::max;
using std::min;
