/*
 * ref_host_shim.h -- lets the reference's CUDA kernel headers
 * (src/gasal_kernels.h and src/kernels/*.h) compile as ordinary host C++.
 *
 * TEST INFRASTRUCTURE ONLY (oracle "A-prime" and the reference CPU arm of the
 * bench).  Each CUDA thread of a launch becomes one call of the kernel
 * function with a thread-local (blockIdx, threadIdx) set by the caller, so the
 * reference's own arithmetic runs unchanged on the host.  Shifts whose count
 * reaches the operand width are undefined behaviour in C++ and may differ
 * from what the GPU build does; only the GPU build pins those.
 */
#ifndef GASAL_REF_HOST_SHIM_H
#define GASAL_REF_HOST_SHIM_H

#include "../include/gasal.h"
#include <climits>
#include <cstdlib>
#include <algorithm>

#undef __global__
#undef __device__
#undef __constant__
#undef __host__
#undef __forceinline__
#define __global__
#define __device__
#define __constant__
#define __host__
#define __forceinline__ inline

struct gb_dim3 { unsigned x, y, z; };
extern thread_local gb_dim3 gb_thread_idx, gb_block_idx;
extern gb_dim3 gb_block_dim, gb_grid_dim;
#define threadIdx gb_thread_idx
#define blockIdx gb_block_idx
#define blockDim gb_block_dim
#define gridDim gb_grid_dim

static inline int max(int a, int b) { return a > b ? a : b; }
static inline int min(int a, int b) { return a < b ? a : b; }

#endif
