/* Host stand-in for the reference's gato/utils/cuda.cuh error helpers. */
#pragma once
#include <cuda_runtime.h>
#define gpuErrchk(ans) (ans)
