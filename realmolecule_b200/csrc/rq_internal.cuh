// rq_internal.cuh -- shared definitions of the librq CUDA kernels (sm_100a).
//
// Layout in HBM: every field is one flat array of S^3 elements, id = i*S^2 + j*S + k
// (k fastest), exactly the reference layout (cloud/solver.py:24-26,
// molecule.js:273-276), so host buffers copy in and out without repacking.
//
// Arithmetic: kernels whose results feed an integer decision (labels) or whose
// outputs are compared bit-for-bit with the reference's own kernels use the
// explicitly rounded intrinsics below (F_ADD ...), which the compiler never
// contracts into FMAs; the order of operations is the reference's.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define F_ADD(a, b) __fadd_rn((a), (b))
#define F_SUB(a, b) __fsub_rn((a), (b))
#define F_MUL(a, b) __fmul_rn((a), (b))
#define F_DIV(a, b) __fdiv_rn((a), (b))
#define F_SQRT(a) __fsqrt_rn((a))

namespace rq {

constexpr int kThreadsK = 32;  // threads along k (contiguous) per block
constexpr int kThreadsJ = 8;   // threads along j per block
constexpr int kMarch = 16;     // planes along i marched by one thread
constexpr int kNmPD = 5;       // new flavour: readout sums per domain (norm, T, V_eK, P rho, P A P)

struct Geo {
  int S;      // points per axis
  int NN;     // S - 1
  long long S2, S3;
};

inline Geo make_geo(int S) {
  Geo g;
  g.S = S;
  g.NN = S - 1;
  g.S2 = (long long)S * S;
  g.S3 = g.S2 * S;
  return g;
}

// Interior march launch: blocks of 32(k) x 8(j) threads, each thread walking kMarch planes in i.
inline dim3 march_grid(const Geo& g, int march = kMarch) {
  int n = g.NN - 1;  // interior points per axis
  return dim3((n + kThreadsK - 1) / kThreadsK, (n + kThreadsJ - 1) / kThreadsJ, (n + march - 1) / march);
}
inline dim3 march_block() { return dim3(kThreadsK, kThreadsJ, 1); }

// ---------------------------------------------------------------------------------------
// Label-keyed FP64 block aggregation.  Each thread carries a running (label, NQ sums)
// pair while it marches; when the label changes the pair is merged into a small
// open-addressing table in shared memory; at block end every used slot is added to the
// global per-domain array with one FP64 atomic per quantity.  A label that finds no free
// slot goes straight to global memory, so the result is exact for any label count.
// ---------------------------------------------------------------------------------------
template <int NQ, int NSLOT = 128>
struct DomTable {
  int keys[NSLOT];
  double vals[NSLOT * NQ];
};

template <int NQ, int NSLOT>
__device__ __forceinline__ void dom_table_init(DomTable<NQ, NSLOT>& t) {
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nt = blockDim.x * blockDim.y * blockDim.z;
  for (int s = tid; s < NSLOT; s += nt) t.keys[s] = -1;
  for (int s = tid; s < NSLOT * NQ; s += nt) t.vals[s] = 0.0;
}

template <int NQ, int NSLOT>
__device__ __forceinline__ void dom_table_add(DomTable<NQ, NSLOT>& t, int label, const double* v, double* global) {
  unsigned slot = ((unsigned)label * 2654435761u) & (NSLOT - 1);
  for (int p = 0; p < NSLOT; ++p) {
    int old = atomicCAS(&t.keys[slot], -1, label);
    if (old == -1 || old == label) {
#pragma unroll
      for (int q = 0; q < NQ; ++q) atomicAdd(&t.vals[slot * NQ + q], v[q]);
      return;
    }
    slot = (slot + 1) & (NSLOT - 1);
  }
#pragma unroll
  for (int q = 0; q < NQ; ++q) atomicAdd(&global[(long long)label * NQ + q], v[q]);
}

template <int NQ, int NSLOT>
__device__ __forceinline__ void dom_table_flush(DomTable<NQ, NSLOT>& t, double* global) {
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nt = blockDim.x * blockDim.y * blockDim.z;
  for (int s = tid; s < NSLOT; s += nt) {
    int k = t.keys[s];
    if (k >= 0) {
#pragma unroll
      for (int q = 0; q < NQ; ++q) atomicAdd(&global[(long long)k * NQ + q], t.vals[s * NQ + q]);
    }
  }
}

// lane of the calling thread in its warp (blocks of any shape)
__device__ __forceinline__ int lane_id() {
  int l;
  asm("mov.u32 %0, %%laneid;" : "=r"(l));
  return l;
}

// Per-thread running sum keyed by label; flushes into the block table on label change.
template <int NQ>
struct RunSum {
  int label;
  double v[NQ];
  __device__ __forceinline__ void reset() {
    label = -1;
#pragma unroll
    for (int q = 0; q < NQ; ++q) v[q] = 0.0;
  }
  template <int NSLOT>
  __device__ __forceinline__ void add(int l, const double* x, DomTable<NQ, NSLOT>& t, double* global) {
    if (l != label) {
      if (label >= 0) dom_table_add(t, label, v, global);
      label = l;
#pragma unroll
      for (int q = 0; q < NQ; ++q) v[q] = x[q];
    } else {
#pragma unroll
      for (int q = 0; q < NQ; ++q) v[q] += x[q];
    }
  }
  template <int NSLOT>
  __device__ __forceinline__ void finish(DomTable<NQ, NSLOT>& t, double* global) {
    if (label >= 0) dom_table_add(t, label, v, global);
  }
  // Same as finish, but must be called by every lane of the warp together: lanes holding the
  // same label first combine their sums with shuffles, so one lane per distinct label touches
  // the shared table (neighbouring k values almost always share a label).
  template <int NSLOT>
  __device__ __forceinline__ void finish_warp(DomTable<NQ, NSLOT>& t, double* global) {
    const unsigned peers = __match_any_sync(0xffffffffu, label);
    const int lane = lane_id();
    double s[NQ];
    if (__all_sync(0xffffffffu, peers == 0xffffffffu)) {
      // one label over the warp (the common case): a butterfly
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        double x = v[q];
        x += __shfl_xor_sync(0xffffffffu, x, 16);
        x += __shfl_xor_sync(0xffffffffu, x, 8);
        x += __shfl_xor_sync(0xffffffffu, x, 4);
        x += __shfl_xor_sync(0xffffffffu, x, 2);
        x += __shfl_xor_sync(0xffffffffu, x, 1);
        s[q] = x;
      }
      if (label >= 0 && lane == 0) dom_table_add(t, label, s, global);
      return;
    }
#pragma unroll
    for (int q = 0; q < NQ; ++q) s[q] = 0.0;
    for (int l = 0; l < 32; ++l) {
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        const double x = __shfl_sync(0xffffffffu, v[q], l);
        if ((peers >> l) & 1u) s[q] += x;
      }
    }
    if (label >= 0 && lane == __ffs(peers) - 1) dom_table_add(t, label, s, global);
  }
};

// Weight Z/N that turns a domain's energy partials (each linear in its density for a fixed P)
// into those of the exactly normalised domain; 1 when Z or the measured norm N is not positive.
inline double domain_norm_weight(double Z, double N) { return (Z > 0.0 && N > 0.0) ? Z / N : 1.0; }

}  // namespace rq
