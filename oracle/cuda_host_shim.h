/*
 * cuda_host_shim.h -- lets plain CUDA-C kernel text compile as host C++.
 *
 * TEST INFRASTRUCTURE ONLY.  This header is force-included (g++ -include) when
 * oracle/ref_build.py compiles the reference's own RawKernel strings from
 * cloud/solver.py:16-315 into oracle/_ref/libsolverpy_ref.so.  Nothing in the
 * product (realmolecule_b200/) includes it.
 *
 * Model: a launch of grid x block threads becomes an OpenMP loop over blocks
 * (blocks run in parallel, threads of one block run in order).  Kernels that
 * need __syncthreads / shared memory are not compiled through this shim (the
 * build recipe skips them and the oracle restates them instead).
 */
#pragma once
#include <math.h>
#include <stdint.h>

struct rqref_dim3 { unsigned x, y, z; };

/* Per-OS-thread launch coordinates: each OpenMP worker owns its own copy. */
static thread_local rqref_dim3 blockIdx = {0, 0, 0};
static thread_local rqref_dim3 threadIdx = {0, 0, 0};
static thread_local rqref_dim3 blockDim = {1, 1, 1};
static thread_local rqref_dim3 gridDim = {1, 1, 1};

#define __global__
#define __device__
#define __forceinline__ inline

/* Float atomics become OpenMP atomics (cloud/solver.py:310-312 uses them). */
static inline float atomicAdd(float* p, float v) {
  float old;
#pragma omp atomic capture
  { old = *p; *p += v; }
  return old;
}
