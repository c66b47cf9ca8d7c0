// batch.cu -- many new-flavour instances with uneven grids stepped together (rq_batch_*).
//
// Every kernel of the schedule is ONE launch over a work list of (instance, tile) items built
// once at creation: block b reads item b, looks up its instance's geometry and buffers, and
// runs the same device body as the single-grid kernel (nm_bodies.cuh) on that tile.  Small
// instances therefore share the GPU instead of each launching a mostly idle grid, and a whole
// schedule period of the batch is one CUDA-graph replay.  The multigrid V-cycle descends level
// by level over the instances that still have a coarser level, solves each instance's coarsest
// level (one block per instance, FP64) when it is reached, and ascends again.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/rq.h"
#include "nm_bodies.cuh"
#include "rq_kernels.h"

namespace rq {

constexpr int kMaxLev = 10;

struct BInst {
  Geo g;
  double h;
  void* U[2];
  void* P[2];
  void* K;
  int* lab[2];
  float* W;
  int nDom, dom0;  // domains of this instance and their offset in the batch-wide arrays
  int nlev;
  Geo lg[kMaxLev];
  double lh[kMaxLev];
  void* lP[kMaxLev];
  void* lf[kMaxLev];
  void* lr[kMaxLev];
  const double* at;  // (x, y, z, Z_nuc) per entry of this instance
  int nAt, at0;      // entries and their offset in the batch-wide force array
  const float4* seeds;
  int nSeed;
  const double* K64;  // fp32 instances of a mixed batch: the FP64 K of its promotion set, read by the readout
  double* cs;         // FP64 working copy of the coarsest level (P and f) for the persistent launch
};

struct BItem {
  int inst, bx, by, bz;
};

// ---------------------------------------------------------------------------------------
// batched kernels: block b works on items[b].  Each copies its instance's geometry into
// registers first: through a reference into the instance table the compiler would re-read it
// after every store, as it cannot prove the field pointers do not alias the table.
// ---------------------------------------------------------------------------------------
template <typename T, bool ACC, bool SR>
__global__ void __launch_bounds__(256) kb_update(const BInst* __restrict__ ins, const BItem* __restrict__ items, int cu,
                                                 int cp, int cl, T half_dv, T dt, double* __restrict__ norms,
                                                 const double* __restrict__ scale, const unsigned* __restrict__ seed,
                                                 unsigned* __restrict__ seed_next, NmTile tile) {
  __shared__ DomTable<1, 128> tab;
  if (SR && blockIdx.x == 0 && threadIdx.x == 0 && threadIdx.y == 0) *seed_next = *seed + 1u;
  const BItem it = items[blockIdx.x];
  const BInst& I = ins[it.inst];
  double* nrm = norms ? norms + I.dom0 : nullptr;
  if (ACC) {
    dom_table_init(tab);
    __syncthreads();
  }
  const Geo g = I.g;
  nm_update_body<T, ACC, false, SR>((const T*)I.U[cu], (T*)I.U[1 - cu], (const T*)I.K, (const T*)I.P[cp], I.lab[cl], g,
                                    half_dv, dt, I.h * I.h * I.h, I.nDom, nrm, tab, it.bx, it.by, it.bz,
                                    scale ? scale + I.dom0 : nullptr, seed, tile);
  if (ACC) {
    __syncthreads();
    dom_table_flush(tab, nrm);
  }
}

template <typename T>
__global__ void __launch_bounds__(256) kb_apply_scale(const BInst* __restrict__ ins, const BItem* __restrict__ items,
                                                      int cu, int cl, const double* __restrict__ scale) {
  const BItem it = items[blockIdx.x];
  const BInst& I = ins[it.inst];
  nm_apply_scale_body<T>((T*)I.U[cu], I.lab[cl], scale + I.dom0, I.g.S3, I.nDom, it.bx);
}

template <typename T>
__global__ void __launch_bounds__(256) kb_norms(const BInst* __restrict__ ins, const BItem* __restrict__ items, int cu,
                                                int cl, double* __restrict__ norms) {
  __shared__ DomTable<1, 128> tab;
  const BItem it = items[blockIdx.x];
  const BInst& I = ins[it.inst];
  dom_table_init(tab);
  __syncthreads();
  nm_norms_body<T>((const T*)I.U[cu], I.lab[cl], I.g.S3, I.h * I.h * I.h, I.nDom, norms + I.dom0, tab, it.bx);
  __syncthreads();
  dom_table_flush(tab, norms + I.dom0);
}

template <typename T, bool FINE>
__global__ void __launch_bounds__(256) kb_rbgs(const BInst* __restrict__ ins, const BItem* __restrict__ items, int lev,
                                               int cu, int cp, int color) {
  const BItem it = items[blockIdx.x];
  const BInst& I = ins[it.inst];
  T* P = FINE ? (T*)I.P[cp] : (T*)I.lP[lev];
  const T* f = FINE ? (const T*)I.U[cu] : (const T*)I.lf[lev];
  const Geo g = I.lg[lev];
  nm_rbgs_body<T, FINE>(P, f, g, (T)(I.lh[lev] * I.lh[lev]), color, it.bx, it.by, it.bz);
}

// residual, full weighting and the zeroed coarse correction of level lev in one pass
template <typename T, bool FINE>
__global__ void __launch_bounds__(256, 4) kb_resrestrict(const BInst* __restrict__ ins, const BItem* __restrict__ items,
                                                      int lev, int cu, int cp, int planes) {
  __shared__ T patch[kNmRrBuf][kNmRrPatch];
  const BItem it = items[blockIdx.x];
  const BInst& I = ins[it.inst];
  const T* P = FINE ? (const T*)I.P[cp] : (const T*)I.lP[lev];
  const T* f = FINE ? (const T*)I.U[cu] : (const T*)I.lf[lev];
  const Geo g = I.lg[lev], gc = I.lg[lev + 1];
  nm_resrestrict_body<T, FINE>(P, f, (T*)I.lf[lev + 1], (T*)I.lP[lev + 1], g, gc, (T)(1.0 / (I.lh[lev] * I.lh[lev])),
                               it.bx, it.by, it.bz, planes, patch);
}

template <typename T>
__global__ void __launch_bounds__(256) kb_prolong(const BInst* __restrict__ ins, const BItem* __restrict__ items, int lev,
                                                  int cp, int planes) {
  const BItem it = items[blockIdx.x];
  const BInst& I = ins[it.inst];
  T* P = lev == 0 ? (T*)I.P[cp] : (T*)I.lP[lev];
  const Geo g = I.lg[lev], gc = I.lg[lev + 1];
  nm_prolong_cells_body<T>((const T*)I.lP[lev + 1], P, g, gc, it.bx, it.by, it.bz, planes);
}

template <typename T>
__global__ void __launch_bounds__(1024) kb_coarsest(const BInst* __restrict__ ins, const BItem* __restrict__ items,
                                                    int lev, int sweeps) {
  extern __shared__ double sm[];
  const BItem it = items[blockIdx.x];
  const BInst& I = ins[it.inst];
  nm_coarsest_body<T>((T*)I.lP[lev], (const T*)I.lf[lev], I.lg[lev], I.lh[lev] * I.lh[lev], sweeps, sm);
}

template <typename T>
__global__ void __launch_bounds__(256) kb_energy(const BInst* __restrict__ ins, const BItem* __restrict__ items, int cu,
                                                 int cp, int cl, double* __restrict__ pd, NmTile tile) {
  __shared__ DomTable<kNmPD, 128> tab;
  const BItem it = items[blockIdx.x];
  const BInst& I = ins[it.inst];
  dom_table_init(tab);
  __syncthreads();
  const Geo g = I.g;
  nm_energy_body<T>((const T*)I.U[cu], (const T*)I.K, (const T*)I.P[cp], I.lab[cl], g, I.h, I.nDom,
                    pd + kNmPD * I.dom0, tab, it.bx, it.by, it.bz, sizeof(T) == sizeof(float) ? I.K64 : nullptr, tile);
  __syncthreads();
  dom_table_flush(tab, pd + kNmPD * I.dom0);
}

template <typename T>
__global__ void __launch_bounds__(256) kb_evolve(const BInst* __restrict__ ins, const BItem* __restrict__ items, int cu,
                                                 int cl, T dt_w, T curv, NmTile tile) {
  const BItem it = items[blockIdx.x];
  const BInst& I = ins[it.inst];
  const Geo g = I.g;
  nm_evolve_body<T>(I.lab[cl], I.lab[1 - cl], (const T*)I.U[cu], I.W, g, dt_w, curv, it.bx, it.by, it.bz, tile);
}

template <typename T>
__global__ void __launch_bounds__(256) kb_potential(const BInst* __restrict__ ins, const BItem* __restrict__ items,
                                                    double sigma_scale) {
  __shared__ double sa[128 * 4];
  const BItem it = items[blockIdx.x];
  const BInst& I = ins[it.inst];
  // fp32 instances of a mixed batch also write the FP64 K of their promotion set (read by the
  // readout, used after a promotion)
  nm_potential_body<T>((T*)I.K, I.at, I.nAt, I.g, I.h, sigma_scale > 0 ? sigma_scale : I.h, it.bx, sa,
                       sizeof(T) == sizeof(float) ? const_cast<double*>(I.K64) : nullptr);
}

template <typename T>
__global__ void __launch_bounds__(256) kb_init(const BInst* __restrict__ ins, const BItem* __restrict__ items) {
  __shared__ float4 ss[256];
  const BItem it = items[blockIdx.x];
  const BInst& I = ins[it.inst];
  nm_init_body<T>((T*)I.U[0], I.lab[0], I.seeds, I.nSeed, I.g, (float)I.h, it.bx, ss);
}

template <typename T>
__global__ void __launch_bounds__(256) kb_force(const BInst* __restrict__ ins, const BItem* __restrict__ items, int cu,
                                                double sigma_scale, double* __restrict__ F) {
  __shared__ double sx[kNmForceTile], sy[kNmForceTile], sz[kNmForceTile], sr[kNmForceTile];
  const BItem it = items[blockIdx.x];
  const BInst& I = ins[it.inst];
  nm_force_body<T>((const T*)I.U[cu], I.at, I.nAt, I.g, I.h, sigma_scale > 0 ? sigma_scale : I.h, F + 3 * I.at0, it.bx,
                   it.by, it.bz, sx, sy, sz, sr);
}

// Sum over the fine interior of the squared residual 2 pi psi^2 - A P (FP64), added into *out:
// the autotuner's multigrid convergence measure.  Row tiling (nm_residual_rows_body's).
template <typename T>
__global__ void __launch_bounds__(256) kb_resnorm(const BInst* __restrict__ ins, const BItem* __restrict__ items, int cu,
                                                  int cp, double* __restrict__ out) {
  __shared__ double part[8];
  const BItem it = items[blockIdx.x];
  const BInst& I = ins[it.inst];
  const Geo g = I.g;
  const T* P = (const T*)I.P[cp];
  const T* U = (const T*)I.U[cu];
  const double ih2 = 1.0 / (I.h * I.h);
  const int j = 1 + it.by * kNmRowTJ + tile_y<32>(), tx = tile_x<32>(), i0 = 1 + it.bz * kNmRowPlanes;
  double acc = 0.0;
  if (j < g.NN) {
    const int iend = min(i0 + kNmRowPlanes, g.NN);
    const long long S = g.S, S2 = g.S2;
    for (int i = i0; i < iend; ++i)
      for (int t = 0; t < 2; ++t) {
        const int k = 1 + it.bx * 64 + tx + 32 * t;
        if (k >= g.NN) continue;
        const long long id = (long long)i * S2 + (long long)j * S + k;
        const double sd = (double)P[id + S2] + (double)P[id - S2] + (double)P[id + S] + (double)P[id - S] +
                          (double)P[id + 1] + (double)P[id - 1];
        const double u = (double)U[id];
        const double r = 6.283185307179586 * u * u + (sd - 6.0 * (double)P[id]) * ih2;
        acc += r * r;
      }
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  const int lin = (int)(threadIdx.x + blockDim.x * threadIdx.y);
  if ((lin & 31) == 0) part[lin >> 5] = acc;
  __syncthreads();
  if (lin == 0) {
    double sum = 0.0;
    for (int w = 0; w < 8; ++w) sum += part[w];
    atomicAdd(out, sum);
  }
}

// ---------------------------------------------------------------------------------------
// The persistent form of a schedule period: ONE launch runs the period's phases (the same
// phases, work lists and bodies as the per-kernel launches above, for both precision sets).
// The items of all phases form one queue, phase after phase and instance after instance within
// a phase; blocks take runs of items from it with one atomic counter.  Every dependency of the
// schedule is within one instance, so an item waits only until its instance's previous non-empty
// phase is complete (a completion counter per (phase, instance)) -- no grid-wide barrier, and
// instances overlap across phases.  Items are taken in queue order, so every item an item waits
// for was taken earlier by a running block: the waits always end.  Each wait is bounded all the
// same (a limit on the global timer): a block that gives up sets bit 1 of the error word and
// leaves, every other block leaves at its next wait, and the host reports RQ_ETIMEOUT.
// ---------------------------------------------------------------------------------------
enum BPhaseKind : int {
  kPhApply, kPhZeroNorms, kPhUpdate, kPhUpdateAcc, kPhScale, kPhRbgs, kPhCoarsest, kPhResidual, kPhRestrict,
  kPhZero, kPhProlong, kPhEvolve
};

struct BPhase {
  int kind, set;          // BPhaseKind; precision set (0: fp32 fields, 1: FP64)
  int lev, color;         // multigrid level and colour
  int cu, cp, cl;         // buffer parities in effect
  int n;                  // items
  const BItem* items;
  const double* scale;    // update: the pending per-domain scale it applies (or null)
  const unsigned* seed;   // update, fp32 unbiased rounding: this step's seed and the next one's slot
  unsigned* seed_next;
};

// A queue entry: `count` consecutive items of one instance in one phase, from item `first`.
struct BChunk {
  int phase, first, count, inst;
};

struct BPersist {
  const BInst* ins;
  const BPhase* prog;
  const BChunk* chunks;   // the queue
  const int2* deps;       // nph x ninst: (previous non-empty phase of the instance or -1, its item count)
  unsigned* done;         // nph x ninst completed items (zeroed before the launch)
  unsigned* queue;        // the next queue index (zeroed before the launch)
  int nph, ninst;
  unsigned total;         // queue length (chunks)
  double half_dv, dt;     // update coefficients (every instance of a batch shares h)
  double* dnorm;          // batch-wide domain norms
  double* scale;          // batch-wide domain scales
  const double* Zdom;
  int sweeps;             // coarsest-level sweeps
  float dt_w, curv;       // level-set pass
  int* err;               // bit 0: non-finite norm; bit 1: a wait gave up
  long long limit_ns;     // bound of every wait
  NmTile tile;            // march tile of the update and level-set items
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

template <typename T>
__device__ __forceinline__ void kb_run_item(const BPersist& a, const BPhase& P, const BItem& it, DomTable<1, 128>& tab) {
  const BInst& I = a.ins[it.inst];
  switch (P.kind) {
    case kPhApply:
      nm_apply_scale_body<T>((T*)I.U[P.cu], I.lab[P.cl], a.scale + I.dom0, I.g.S3, I.nDom, it.bx);
      break;
    case kPhZeroNorms:
      for (int d = threadIdx.x; d < I.nDom; d += blockDim.x) a.dnorm[I.dom0 + d] = 0.0;
      break;
    case kPhScale:
      for (int d = threadIdx.x; d < I.nDom; d += blockDim.x)
        a.scale[I.dom0 + d] = nm_domain_scale(a.dnorm[I.dom0 + d], a.Zdom[I.dom0 + d], a.err);
      break;
    case kPhUpdate:
    case kPhUpdateAcc: {
      const Geo g = I.g;
      const double* sc = P.scale ? P.scale + I.dom0 : nullptr;
      if (P.kind == kPhUpdateAcc) {
        dom_table_init(tab);
        __syncthreads();
        nm_update_body<T, true>((const T*)I.U[P.cu], (T*)I.U[1 - P.cu], (const T*)I.K, (const T*)I.P[P.cp], I.lab[P.cl],
                                g, (T)a.half_dv, (T)a.dt, I.h * I.h * I.h, I.nDom, a.dnorm + I.dom0, tab, it.bx, it.by,
                                it.bz, sc, P.seed, a.tile);
        __syncthreads();
        dom_table_flush(tab, a.dnorm + I.dom0);
      } else {
        nm_update_body<T, false>((const T*)I.U[P.cu], (T*)I.U[1 - P.cu], (const T*)I.K, (const T*)I.P[P.cp],
                                 I.lab[P.cl], g, (T)a.half_dv, (T)a.dt, I.h * I.h * I.h, I.nDom, nullptr, tab, it.bx,
                                 it.by, it.bz, sc, P.seed, a.tile);
      }
      break;
    }
    case kPhRbgs: {
      const Geo g = I.lg[P.lev];
      const T h2 = (T)(I.lh[P.lev] * I.lh[P.lev]);
      if (P.lev == 0)
        nm_rbgs_body<T, true>((T*)I.P[P.cp], (const T*)I.U[P.cu], g, h2, P.color, it.bx, it.by, it.bz);
      else
        nm_rbgs_body<T, false>((T*)I.lP[P.lev], (const T*)I.lf[P.lev], g, h2, P.color, it.bx, it.by, it.bz);
      break;
    }
    case kPhCoarsest:  // one block per instance; the level's FP64 working copy in the instance's scratch
      nm_coarsest_body<T>((T*)I.lP[P.lev], (const T*)I.lf[P.lev], I.lg[P.lev], I.lh[P.lev] * I.lh[P.lev], a.sweeps,
                          I.cs);
      break;
    case kPhResidual: {
      const Geo g = I.lg[P.lev];
      const T ih2 = (T)(1.0 / (I.lh[P.lev] * I.lh[P.lev]));
      if (P.lev == 0)
        nm_residual_rows_body<T, true>((const T*)I.P[P.cp], (const T*)I.U[P.cu], (T*)I.lr[0], g, ih2, it.bx, it.by,
                                       it.bz);
      else
        nm_residual_rows_body<T, false>((const T*)I.lP[P.lev], (const T*)I.lf[P.lev], (T*)I.lr[P.lev], g, ih2, it.bx,
                                        it.by, it.bz);
      break;
    }
    case kPhRestrict: {
      const Geo g = I.lg[P.lev], gc = I.lg[P.lev + 1];
      nm_restrict_body<T>((const T*)I.lr[P.lev], (T*)I.lf[P.lev + 1], g, gc, (long long)it.bx * blockDim.x + threadIdx.x);
      break;
    }
    case kPhZero: {
      const long long S3 = I.lg[P.lev].S3, base = (long long)it.bx * blockDim.x * kNmFlatChunk;
      T* p = (T*)I.lP[P.lev];
      for (int q = 0; q < kNmFlatChunk; ++q) {
        const long long id = base + (long long)q * blockDim.x + threadIdx.x;
        if (id < S3) p[id] = T(0);
      }
      break;
    }
    case kPhProlong: {
      T* Pf = P.lev == 0 ? (T*)I.P[P.cp] : (T*)I.lP[P.lev];
      const Geo g = I.lg[P.lev], gc = I.lg[P.lev + 1];
      nm_prolong_rows_body<T>((const T*)I.lP[P.lev + 1], Pf, g, gc, it.bx, it.by, it.bz);
      break;
    }
    case kPhEvolve: {
      const Geo g = I.g;
      nm_evolve_body<T>(I.lab[P.cl], I.lab[1 - P.cl], (const T*)I.U[P.cu], I.W, g, (T)a.dt_w, (T)a.curv, it.bx, it.by,
                        it.bz, a.tile);
      break;
    }
    default:
      break;
  }
}

// SETS: the precision sets the program uses (bit 0: fp32 fields, bit 1: FP64), so a batch with
// one set compiles only that set's bodies (fewer registers).  The next run of items is taken
// while the block works on the current one.
template <int SETS>
__global__ void __launch_bounds__(256, 4) kb_persist(BPersist a) {
  __shared__ DomTable<1, 128> tab;
  __shared__ BPhase P;                  // phase of the current chunk
  __shared__ BChunk C;
  __shared__ unsigned next;
  __shared__ int ph, ok_ph, ok_inst, stop;  // (ok_ph, ok_inst): a dependency already seen complete
  if (threadIdx.x == 0) {
    ph = -1; ok_ph = -1; ok_inst = -1; stop = 0;
    next = atomicAdd(a.queue, 1u);
  }
  __syncthreads();
  unsigned q = next;
  __syncthreads();
  while (q < a.total) {
    if (threadIdx.x == 0) {
      next = atomicAdd(a.queue, 1u);  // in flight during the chunk
      C = a.chunks[q];
      if (C.phase != ph) { P = a.prog[C.phase]; ph = C.phase; }
      if (ph != ok_ph || C.inst != ok_inst) {
        const int2 d = a.deps[(long long)ph * a.ninst + C.inst];
        if (d.x >= 0) {
          const volatile unsigned* c = a.done + (long long)d.x * a.ninst + C.inst;
          const unsigned long long t0 = global_ns();
          while (*c < (unsigned)d.y) {
            if ((*(volatile int*)a.err & 2) || (long long)(global_ns() - t0) > a.limit_ns) {
              atomicOr(a.err, 2);
              stop = 1;
              break;
            }
            __nanosleep(32);
          }
          __threadfence();
        }
        ok_ph = ph; ok_inst = C.inst;
      }
    }
    __syncthreads();
    if (stop) return;
    for (int k = 0; k < C.count; ++k) {
      const BItem it = P.items[C.first + k];
      if (P.set == 0) {
        if (SETS & 1) kb_run_item<float>(a, P, it, tab);
      } else {
        if (SETS & 2) kb_run_item<double>(a, P, it, tab);
      }
      if (P.kind == kPhUpdateAcc || P.kind == kPhCoarsest) __syncthreads();  // shared table / scratch reuse
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(a.done + (long long)ph * a.ninst + C.inst, (unsigned)C.count);
    }
    q = next;
    __syncthreads();
  }
}

}  // namespace rq

// =========================================================================================
// host side
// =========================================================================================
using namespace rq;

namespace {
// The two precision sets of a batch: every instance holds its fields either in fp32 (kF32) or
// in FP64 (kF64).  A mixed-precision batch starts all-fp32 and moves instances to FP64 one by
// one as they reach the fp32 resolution of their energy; each kernel of a step is then one
// launch per non-empty set.
constexpr int kF32 = 0, kF64 = 1;
}  // namespace

// Work items of one instance for every list; built once at creation, concatenated by build_plans.
struct InstItems {
  std::vector<BItem> march[kMaxLev], rbgs[kMaxLev], restr[kMaxLev], zero[kMaxLev], coarse[kMaxLev], rr[kMaxLev],
      pc[kMaxLev];
  std::vector<BItem> flat16, flat1, force, one;  // one: a single item (per-instance domain work)
};

struct rq_batch {
  int n = 0;
  rq_config cfg{};
  double dv = 0.2;
  std::vector<BInst> hin;         // host copy of the instance table
  std::vector<BInst> hin64;       // mixed batches: each instance's FP64 field set, taken over on promotion
  BInst* din = nullptr;           // device copy
  std::vector<std::vector<rq_atom>> atoms;
  std::vector<void*> allocs;
  int D = 0, A = 0;               // total domains / entries
  double *dnorm = nullptr, *dpd = nullptr, *dF = nullptr, *Zdom = nullptr, *at_all = nullptr, *scale = nullptr;
  int* err = nullptr;
  unsigned* rseed = nullptr;      // the step seed of the fp32 set's unbiased rounding (2 words by parity)
  float4* seeds_all = nullptr;
  int maxlev = 0;
  int rr_pl[kMaxLev] = {}, pr_pl[kMaxLev] = {};  // coarse planes per block of the level's residual-restriction / prolongation
  // work lists, one set per precision
  struct Plan { BItem* d = nullptr; int n = 0, cap = 0; };
  struct Plans {
    Plan march[kMaxLev], rbgs[kMaxLev], restr[kMaxLev], zero[kMaxLev], coarse[kMaxLev], rr[kMaxLev], pc[kMaxLev];
    Plan flat16, flat1, force, one;
  };
  Plans pl[2];
  size_t coarse_smem[kMaxLev] = {};
  cudaStream_t st = nullptr, own = nullptr;
  int cu = 0, cp = 0, cl = 0, steps_done = 0;
  long long launches = 0;
  cudaGraphExec_t graph[32] = {};
  int graph_post[32] = {};
  long long graph_launches[32] = {};
  std::vector<char> active;       // instances still being stepped (solve drops converged ones)
  std::vector<char> f64;          // instances whose fields are FP64 (created so, or promoted)
  std::vector<InstItems> items;   // per-instance work items (built once)
  std::vector<double> lastE;      // last energies per instance (n x RQ_ENERGY_LEN)
  bool pending = false;           // psi awaits the per-domain scale (applied by the next update or a flush)
  int age = 0;                    // updates since psi was last normalised (0: normalised or pending)
  std::string last_error;
  // persistent launches: a schedule period recorded as a program of phases (rec non-null while
  // recording), one program per graph key, the queue and completion counters, the launch's grid
  std::vector<BPhase>* rec = nullptr;
  struct Prog { BPhase* phases = nullptr; BChunk* chunks = nullptr; int2* deps = nullptr; int n = 0, cap = 0, cap_chunks = 0; };
  Prog prog[32];
  unsigned* pcount = nullptr;     // the queue word, then the (phase, instance) completion counters
  size_t pcount_cap = 0;
  int pgrid[4] = {};              // co-resident blocks of kb_persist<sets> (0: not yet queried)
  long long wait_ns = 2000000000LL;
  int extra_arrivals = 0;
  NmTile tile = kNmTile;          // march tile of the update, readout and level-set work lists
  double* dtune = nullptr;        // the autotuner's residual sum
};

#define BCK(call)                                                                  \
  do {                                                                             \
    cudaError_t _e = (call);                                                       \
    if (_e != cudaSuccess) {                                                       \
      b->last_error = std::string(#call) + ": " + cudaGetErrorString(_e);          \
      return _e == cudaErrorMemoryAllocation ? RQ_ENOMEM : RQ_ECUDA;               \
    }                                                                              \
  } while (0)
#define BRC(call)                        \
  do {                                   \
    const int _r = (call);               \
    if (_r != RQ_OK) return _r;          \
  } while (0)

static int balloc(rq_batch* b, void** p, size_t bytes) {
  BCK(cudaMalloc(p, bytes));
  b->allocs.push_back(*p);
  BCK(cudaMemsetAsync(*p, 0, bytes, b->st));
  return RQ_OK;
}
#define BALLOC(ptr, bytes) BRC(balloc(b, (void**)&(ptr), (bytes)))

static int upload_plan(rq_batch* b, rq_batch::Plan& p, const std::vector<BItem>& v) {
  p.n = (int)v.size();
  if (!p.n) return RQ_OK;
  if (p.n > p.cap) {  // the first build allocates the full size; later builds (fewer instances) reuse it
    BALLOC(p.d, sizeof(BItem) * v.size());
    p.cap = p.n;
  }
  BCK(cudaMemcpyAsync(p.d, v.data(), sizeof(BItem) * v.size(), cudaMemcpyHostToDevice, b->st));
  return RQ_OK;
}

static void march_items(std::vector<BItem>& v, int inst, const Geo& g, NmTile tile) {
  const dim3 gr = nm_march_grid(g, tile);
  for (unsigned z = 0; z < gr.z; ++z)
    for (unsigned y = 0; y < gr.y; ++y)
      for (unsigned x = 0; x < gr.x; ++x) v.push_back({inst, (int)x, (int)y, (int)z});
}

static void flat_items(std::vector<BItem>& v, int inst, long long npts, long long per_block) {
  for (long long x = 0; x < (npts + per_block - 1) / per_block; ++x) v.push_back({inst, (int)x, 0, 0});
}

static void make_items(const BInst& I, int q, InstItems& it, NmTile tile, const int* rr_pl, const int* pr_pl) {
  it = InstItems{};
  for (int l = 0; l < I.nlev; ++l) {
    march_items(it.march[l], q, I.lg[l], tile);
    if (l == I.nlev - 1) {
      it.coarse[l].push_back({q, 0, 0, 0});
      continue;
    }
    const int nn = I.lg[l].NN - 1;
    for (int zz = 0; zz < (nn + kNmRowPlanes - 1) / kNmRowPlanes; ++zz)
      for (int y = 0; y < (nn + 7) / 8; ++y)
        for (int x = 0; x < (nn + 63) / 64; ++x) it.rbgs[l].push_back({q, x, y, zz});
    const long long nc = (long long)(I.lg[l + 1].NN - 1) * (I.lg[l + 1].NN - 1) * (I.lg[l + 1].NN - 1);
    flat_items(it.restr[l], q, nc, 256);
    flat_items(it.zero[l], q, I.lg[l + 1].S3, 256 * kNmFlatChunk);
    const int cn = I.lg[l + 1].NN - 1;  // coarse interior of the fused residual + restriction
    for (int zz = 0; zz < (cn + rr_pl[l] - 1) / rr_pl[l]; ++zz)
      for (int y = 0; y < (cn + kNmRrTJ - 1) / kNmRrTJ; ++y)
        for (int x = 0; x < (cn + kNmRrTK - 1) / kNmRrTK; ++x) it.rr[l].push_back({q, x, y, zz});
    const int cc = I.lg[l + 1].NN;  // coarse cells of the prolongation
    for (int zz = 0; zz < (cc + pr_pl[l] - 1) / pr_pl[l]; ++zz)
      for (int y = 0; y < (cc + kNmPrTJ - 1) / kNmPrTJ; ++y)
        for (int x = 0; x < (cc + kNmPrTK - 1) / kNmPrTK; ++x) it.pc[l].push_back({q, x, y, zz});
  }
  it.one.push_back({q, 0, 0, 0});
  flat_items(it.flat16, q, I.g.S3, 256 * kNmFlatChunk);
  flat_items(it.flat1, q, I.g.S3, 256);
  const long long n1 = I.g.NN - 1, ntiles = (n1 * n1 * n1 + kNmForceTile - 1) / kNmForceTile;
  const int groups = (int)std::min<long long>(ntiles, 32);
  for (int ch = 0; ch < (I.nAt + 255) / 256; ++ch)
    for (int t = 0; t < groups; ++t) it.force.push_back({q, t, groups, ch});
}

// Work lists of each precision set over the active instances (all of them at creation; solve
// drops converged ones and moves promoted ones to the FP64 set): concatenations of the
// instances' cached items.  Captured graphs hold the old lists, so they are dropped.
static int build_plans(rq_batch* b) {
  using Items = std::vector<BItem>;
  for (int p = 0; p < 2; ++p) {
    rq_batch::Plans& P = b->pl[p];
    std::vector<int> mine;
    for (int q = 0; q < b->n; ++q)
      if (b->active[q] && (b->f64[q] ? kF64 : kF32) == p) mine.push_back(q);
    auto gather = [&](rq_batch::Plan& plan, auto member) -> int {
      Items v;
      for (int q : mine) {
        const Items& src = member(b->items[q]);
        v.insert(v.end(), src.begin(), src.end());
      }
      return upload_plan(b, plan, v);
    };
    for (int l = 0; l < b->maxlev; ++l) {
      BRC(gather(P.march[l], [l](const InstItems& it) -> const Items& { return it.march[l]; }));
      BRC(gather(P.rbgs[l], [l](const InstItems& it) -> const Items& { return it.rbgs[l]; }));
      BRC(gather(P.restr[l], [l](const InstItems& it) -> const Items& { return it.restr[l]; }));
      BRC(gather(P.zero[l], [l](const InstItems& it) -> const Items& { return it.zero[l]; }));
      BRC(gather(P.rr[l], [l](const InstItems& it) -> const Items& { return it.rr[l]; }));
      BRC(gather(P.pc[l], [l](const InstItems& it) -> const Items& { return it.pc[l]; }));
      BRC(gather(P.coarse[l], [l](const InstItems& it) -> const Items& { return it.coarse[l]; }));
    }
    BRC(gather(P.flat16, [](const InstItems& it) -> const Items& { return it.flat16; }));
    BRC(gather(P.one, [](const InstItems& it) -> const Items& { return it.one; }));
    BRC(gather(P.flat1, [](const InstItems& it) -> const Items& { return it.flat1; }));
    BRC(gather(P.force, [](const InstItems& it) -> const Items& { return it.force; }));
  }
  for (auto& g : b->graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  return RQ_OK;
}

// field buffers of one instance with elements of es bytes (level 0 fields and the multigrid levels)
static int alloc_fields(rq_batch* b, BInst& I, size_t es) {
  const size_t S3 = (size_t)I.g.S3;
  for (int k = 0; k < 2; ++k) {
    BALLOC(I.U[k], S3 * es);
    BALLOC(I.P[k], S3 * es);
  }
  BALLOC(I.K, S3 * es);
  for (int l = 0; l < I.nlev; ++l) {
    const size_t s3 = (size_t)I.lg[l].S3;
    I.lP[l] = I.lf[l] = I.lr[l] = nullptr;
    if (l > 0) {
      BALLOC(I.lP[l], s3 * es);
      BALLOC(I.lf[l], s3 * es);
    }
    if (l < I.nlev - 1) BALLOC(I.lr[l], s3 * es);
  }
  BALLOC(I.cs, 2 * sizeof(double) * (size_t)I.lg[I.nlev - 1].S3);
  return RQ_OK;
}

// Coarse planes per block of each level's residual-restriction and prolongation over all
// instances: 8, halved while the level's launch would have fewer than 8 blocks per SM.
static void b_mg_planes(rq_batch* b) {
  for (int l = 0; l + 1 < b->maxlev; ++l) {
    auto blocks = [&](int planes, bool rr) {
      long long tot = 0;
      for (const BInst& I : b->hin) {
        if (l + 1 >= I.nlev) continue;
        const int n = rr ? I.lg[l + 1].NN - 1 : I.lg[l + 1].NN;
        const int tk = rr ? kNmRrTK : kNmPrTK, tj = rr ? kNmRrTJ : kNmPrTJ;
        tot += (long long)((n + tk - 1) / tk) * ((n + tj - 1) / tj) * ((n + planes - 1) / planes);
      }
      return tot;
    };
    for (int r = 0; r < 2; ++r) {
      int planes = 8;
      while (planes > 1 && blocks(planes, r == 0) < 8LL * 148) planes /= 2;
      (r == 0 ? b->rr_pl : b->pr_pl)[l] = planes;
    }
  }
}

static int build(rq_batch* b) {
  const int n = b->n;
  for (int q = 0; q < n; ++q) {
    BInst& I = b->hin[q];
    BRC(alloc_fields(b, I, b->f64[q] ? sizeof(double) : sizeof(float)));
    for (int k = 0; k < 2; ++k) BALLOC(I.lab[k], (size_t)I.g.S3 * sizeof(int));
    BALLOC(I.W, (size_t)I.g.S3 * sizeof(float));
    const int lc = I.nlev - 1;
    b->coarse_smem[lc] = std::max(b->coarse_smem[lc], sizeof(double) * 2 * (size_t)I.lg[lc].S3);
  }
  // batch-wide per-domain arrays and atom tables
  BALLOC(b->dnorm, sizeof(double) * b->D);
  BALLOC(b->dpd, sizeof(double) * kNmPD * b->D);
  BALLOC(b->Zdom, sizeof(double) * b->D);
  BALLOC(b->scale, sizeof(double) * b->D);
  BALLOC(b->dF, sizeof(double) * 3 * b->A);
  BALLOC(b->at_all, sizeof(double) * 4 * b->A);
  BALLOC(b->seeds_all, sizeof(float4) * b->A);
  BALLOC(b->err, sizeof(int) * 4);
  BALLOC(b->rseed, sizeof(unsigned) * 2);
  std::vector<double> zd(b->D), at(4 * (size_t)b->A);
  std::vector<float4> seeds;
  seeds.reserve(b->A);
  for (int q = 0; q < n; ++q) {
    BInst& I = b->hin[q];
    I.at = b->at_all + 4 * (size_t)I.at0;
    I.seeds = b->seeds_all + seeds.size();
    int ns = 0;
    for (int e = 0; e < I.nAt; ++e) {
      const rq_atom& a = b->atoms[q][e];
      zd[I.dom0 + e] = a.Z;
      double* r = &at[4 * ((size_t)I.at0 + e)];
      r[0] = a.i * I.h; r[1] = a.j * I.h; r[2] = a.k * I.h; r[3] = a.Z_nuc;
      if (a.Z > 0) {
        float4 s;
        s.x = (float)(a.i * I.h); s.y = (float)(a.j * I.h); s.z = (float)(a.k * I.h);
        int idx = e;
        std::memcpy(&s.w, &idx, sizeof(int));
        seeds.push_back(s);
        ns++;
      }
    }
    I.nSeed = ns;
  }
  BCK(cudaMemcpyAsync(b->Zdom, zd.data(), sizeof(double) * b->D, cudaMemcpyHostToDevice, b->st));
  BCK(cudaMemcpyAsync(b->at_all, at.data(), sizeof(double) * at.size(), cudaMemcpyHostToDevice, b->st));
  if (!seeds.empty())
    BCK(cudaMemcpyAsync(b->seeds_all, seeds.data(), sizeof(float4) * seeds.size(), cudaMemcpyHostToDevice, b->st));
  BALLOC(b->din, sizeof(BInst) * n);
  BCK(cudaMemcpyAsync(b->din, b->hin.data(), sizeof(BInst) * n, cudaMemcpyHostToDevice, b->st));
  bool mixed = false;
  for (int q = 0; q < n; ++q) mixed |= !b->f64[q];
  if (mixed) {  // allocated up front, so a promotion during a solve allocates and synchronises nothing
    b->hin64 = b->hin;
    for (int q = 0; q < n; ++q) BRC(alloc_fields(b, b->hin64[q], sizeof(double)));
    // the fp32 instances read their energy with the FP64 K of their promotion set (written by the
    // potential pass of initialisation): the f32 rounding of K then enters the readout at second
    // order only
    for (int q = 0; q < n; ++q)
      if (!b->f64[q]) b->hin[q].K64 = (const double*)b->hin64[q].K;
    BCK(cudaMemcpyAsync(b->din, b->hin.data(), sizeof(BInst) * n, cudaMemcpyHostToDevice, b->st));
  }
  b->items.resize(n);
  b_mg_planes(b);
  for (int q = 0; q < n; ++q) make_items(b->hin[q], q, b->items[q], b->tile, b->rr_pl, b->pr_pl);
  BRC(build_plans(b));
  size_t smax = 0;
  for (int l = 0; l < b->maxlev; ++l) smax = std::max(smax, b->coarse_smem[l]);
  if (smax > 200 * 1024) {
    b->last_error = "coarsest multigrid level too large for the shared-memory FP64 solve";
    return RQ_EINVAL;
  }
  BCK(cudaFuncSetAttribute(kb_coarsest<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smax));
  BCK(cudaFuncSetAttribute(kb_coarsest<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smax));
  BCK(cudaStreamSynchronize(b->st));
  return RQ_OK;
}

int rq_batch_set_active_all(rq_batch* b);

static int b_launch_err(rq_batch* b, const char* what) {
  cudaError_t e = cudaGetLastError();
  b->launches++;
  if (e != cudaSuccess) {
    b->last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return RQ_ECUDA;
  }
  return RQ_OK;
}
#define BL(what) BRC(b_launch_err(b, what))

// f(T(), set) for the fp32 and the FP64 set, in that order
template <class F>
static int each_set(F&& f) {
  const int r = f(float(0), kF32);
  return r != RQ_OK ? r : f(double(0), kF64);
}

// A phase of the period being recorded (persistent launches): kind and work list, with the
// buffer parities in effect at this point of the schedule.
static void b_record(rq_batch* b, int kind, int set, const rq_batch::Plan* pl, int lev = 0, int color = 0) {
  if (!pl || pl->n == 0) return;
  BPhase x{};
  x.kind = kind; x.set = set; x.lev = lev; x.color = color;
  x.cu = b->cu; x.cp = b->cp; x.cl = b->cl;
  x.n = pl->n;
  x.items = pl->d;
  b->rec->push_back(x);
}

template <typename T>
static int b_vcycle(rq_batch* b, int p) {
  const rq_batch::Plans& P = b->pl[p];
  const int pre = b->cfg.mg_pre, post = b->cfg.mg_post;
  const dim3 rb(32, 8);
  auto smooth = [&](int l) -> int {
    for (int color = 0; color < 2; ++color) {
      if (b->rec) {
        b_record(b, kPhRbgs, p, &P.rbgs[l], l, color);
        continue;
      }
      if (l == 0)
        kb_rbgs<T, true><<<P.rbgs[l].n, rb, 0, b->st>>>(b->din, P.rbgs[l].d, l, b->cu, b->cp, color);
      else
        kb_rbgs<T, false><<<P.rbgs[l].n, rb, 0, b->st>>>(b->din, P.rbgs[l].d, l, b->cu, b->cp, color);
      BL("rbgs");
    }
    return RQ_OK;
  };
  for (int l = 0; l < b->maxlev; ++l) {
    if (P.coarse[l].n) {
      if (b->rec) {
        b_record(b, kPhCoarsest, p, &P.coarse[l], l);
      } else {
        kb_coarsest<T><<<P.coarse[l].n, kCoarsestThreads, b->coarse_smem[l], b->st>>>(b->din, P.coarse[l].d, l,
                                                                                     b->cfg.mg_coarse_sweeps);
        BL("coarsest");
      }
    }
    if (!P.rbgs[l].n) continue;
    for (int s = 0; s < pre; ++s) BRC(smooth(l));
    if (b->rec) {
      b_record(b, kPhResidual, p, &P.rbgs[l], l);
      b_record(b, kPhRestrict, p, &P.restr[l], l);
      b_record(b, kPhZero, p, &P.zero[l], l + 1);
      continue;
    }
    // the coarse correction's boundary stays zero from the allocation: only its interior is cleared
    if (l == 0)
      kb_resrestrict<T, true><<<P.rr[l].n, rb, 0, b->st>>>(b->din, P.rr[l].d, l, b->cu, b->cp, b->rr_pl[l]);
    else
      kb_resrestrict<T, false><<<P.rr[l].n, rb, 0, b->st>>>(b->din, P.rr[l].d, l, b->cu, b->cp, b->rr_pl[l]);
    BL("resrestrict");
  }
  for (int l = b->maxlev - 2; l >= 0; --l) {
    if (!P.rbgs[l].n) continue;
    if (b->rec) {
      b_record(b, kPhProlong, p, &P.rbgs[l], l);
    } else {
      kb_prolong<T><<<P.pc[l].n, rb, 0, b->st>>>(b->din, P.pc[l].d, l, b->cp, b->pr_pl[l]);
      BL("prolong");
    }
    for (int s = 0; s < post; ++s) BRC(smooth(l));
  }
  return RQ_OK;
}

template <typename T>
static int b_apply(rq_batch* b, int p) {
  const rq_batch::Plan& f = b->pl[p].flat16;
  if (!f.n) return RQ_OK;
  if (b->rec) {
    b_record(b, kPhApply, p, &f);
    return RQ_OK;
  }
  kb_apply_scale<T><<<f.n, 256, 0, b->st>>>(b->din, f.d, b->cu, b->cl, b->scale);
  BL("apply_scale");
  return RQ_OK;
}

static int b_normalize(rq_batch* b) {
  BCK(cudaMemsetAsync(b->dnorm, 0, sizeof(double) * b->D, b->st));
  BRC(each_set([&](auto tag, int p) -> int {
    using T = decltype(tag);
    const rq_batch::Plan& f = b->pl[p].flat16;
    if (!f.n) return RQ_OK;
    kb_norms<T><<<f.n, 256, 0, b->st>>>(b->din, f.d, b->cu, b->cl, b->dnorm);
    BL("norms");
    return RQ_OK;
  }));
  BCK(nm_norm_scale<double>(b->dnorm, b->Zdom, b->D, b->scale, b->err, b->st));
  b->launches++;
  BRC(each_set([&](auto tag, int p) { return b_apply<decltype(tag)>(b, p); }));
  b->pending = false;
  b->age = 0;
  return RQ_OK;
}

// materialise a pending per-domain normalisation (needed by the multigrid, labels and readouts)
static int b_flush(rq_batch* b) {
  if (!b->pending) return RQ_OK;
  BRC(each_set([&](auto tag, int p) { return b_apply<decltype(tag)>(b, p); }));
  b->pending = false;
  return RQ_OK;
}

// the normalised state every readout reports: flush a pending scale, or normalise now when
// updates ran since the last normalisation
static int b_ready(rq_batch* b) { return b->age == 0 ? b_flush(b) : b_normalize(b); }

static bool any_active(const rq_batch* b) { return b->pl[kF32].march[0].n + b->pl[kF64].march[0].n > 0; }

static int b_step(rq_batch* b, int s) {
  const rq_config& f = b->cfg;
  if (!any_active(b)) return RQ_OK;
  if (s % f.poisson_interval == 0) {
    BRC(b_flush(b));
    BRC(each_set([&](auto tag, int p) { return b_vcycle<decltype(tag)>(b, p); }));
  }
  // normalised after every norm_interval-th update and always after the update that precedes a
  // V-cycle or a label pass (the update commutes with per-domain scales between Poisson solves)
  const bool label_step = s % f.label_interval == 0 && (f.label_until <= 0 || s <= f.label_until);
  const bool norm = (s + 1) % f.norm_interval == 0 || (s + 1) % f.poisson_interval == 0 || label_step;
  // dt = dv h^2 differs per instance only through h: every instance of a batch shares h
  const double hd = 0.5 * b->dv, dt = b->dv * b->hin[0].h * b->hin[0].h;
  const double* sc = b->pending ? b->scale : nullptr;
  if (norm) {
    if (b->rec)
      for (int p = 0; p < 2; ++p) b_record(b, kPhZeroNorms, p, &b->pl[p].one);
    else
      BCK(cudaMemsetAsync(b->dnorm, 0, sizeof(double) * b->D, b->st));
  }
  BRC(each_set([&](auto tag, int p) -> int {
    using T = decltype(tag);
    const rq_batch::Plan& m = b->pl[p].march[0];
    if (!m.n) return RQ_OK;
    const bool sr = p == kF32 && b->cfg.fp32_rounding == 1;
    const unsigned* sd = sr ? b->rseed + b->cu : nullptr;
    unsigned* sn = sr ? b->rseed + (1 - b->cu) : nullptr;
    if (b->rec) {
      b_record(b, norm ? kPhUpdateAcc : kPhUpdate, p, &m);
      b->rec->back().scale = sc;
      b->rec->back().seed = sd;
      b->rec->back().seed_next = sn;
      return RQ_OK;
    }
    double* nrm = norm ? b->dnorm : nullptr;
    if (norm && sr)
      kb_update<T, true, true><<<m.n, nm_march_block(), 0, b->st>>>(b->din, m.d, b->cu, b->cp, b->cl, (T)hd, (T)dt,
                                                                   nrm, sc, sd, sn, b->tile);
    else if (norm)
      kb_update<T, true, false><<<m.n, nm_march_block(), 0, b->st>>>(b->din, m.d, b->cu, b->cp, b->cl, (T)hd, (T)dt,
                                                                    nrm, sc, sd, sn, b->tile);
    else if (sr)
      kb_update<T, false, true><<<m.n, nm_march_block(), 0, b->st>>>(b->din, m.d, b->cu, b->cp, b->cl, (T)hd, (T)dt,
                                                                    nrm, sc, sd, sn, b->tile);
    else
      kb_update<T, false, false><<<m.n, nm_march_block(), 0, b->st>>>(b->din, m.d, b->cu, b->cp, b->cl, (T)hd, (T)dt,
                                                                     nrm, sc, sd, sn, b->tile);
    BL("update");
    return RQ_OK;
  }));
  b->cu ^= 1;
  b->pending = false;
  if (norm) {  // applied by the next update (or a flush)
    if (b->rec) {
      for (int p = 0; p < 2; ++p) b_record(b, kPhScale, p, &b->pl[p].one);
    } else {
      BCK(nm_norm_scale<double>(b->dnorm, b->Zdom, b->D, b->scale, b->err, b->st));
      b->launches++;
    }
    b->pending = true;
  }
  b->age = norm ? 0 : b->age + 1;
  if (label_step) {
    BRC(b_flush(b));
    BRC(each_set([&](auto tag, int p) -> int {
      using T = decltype(tag);
      const rq_batch::Plan& m = b->pl[p].march[0];
      if (!m.n) return RQ_OK;
      if (b->rec) {
        b_record(b, kPhEvolve, p, &m);
        return RQ_OK;
      }
      kb_evolve<T><<<m.n, nm_march_block(), 0, b->st>>>(b->din, m.d, b->cu, b->cl, (T)(float)f.boundary_speed,
                                                       (T)(float)f.curv_reg, b->tile);
      BL("evolve");
      return RQ_OK;
    }));
    b->cl ^= 1;
  }
  return RQ_OK;
}

static int b_initialize(rq_batch* b) {
  b->cu = b->cp = b->cl = 0;
  BRC(each_set([&](auto tag, int p) -> int {
    using T = decltype(tag);
    const rq_batch::Plan& f = b->pl[p].flat1;
    if (!f.n) return RQ_OK;
    kb_potential<T><<<f.n, 256, 0, b->st>>>(b->din, f.d, b->cfg.sigma);
    BL("potential");
    kb_init<T><<<f.n, 256, 0, b->st>>>(b->din, f.d);
    BL("init");
    return RQ_OK;
  }));
  for (int q = 0; q < b->n; ++q) {
    const BInst& I = b->hin[q];
    const size_t es = b->f64[q] ? sizeof(double) : sizeof(float);
    BCK(cudaMemcpyAsync(I.lab[1], I.lab[0], sizeof(int) * I.g.S3, cudaMemcpyDeviceToDevice, b->st));
    BCK(cudaMemsetAsync(I.U[1], 0, es * I.g.S3, b->st));
    for (int k = 0; k < 2; ++k) BCK(cudaMemsetAsync(I.P[k], 0, es * I.g.S3, b->st));
    BCK(launch_fill(I.W, 1.0f, I.g.S3, b->st));
  }
  BRC(b_normalize(b));
  for (int v = 0; v < 10; ++v) BRC(each_set([&](auto tag, int p) { return b_vcycle<decltype(tag)>(b, p); }));
  b->steps_done = 0;
  BCK(cudaStreamSynchronize(b->st));
  return RQ_OK;
}

// -----------------------------------------------------------------------------------------
// C ABI
// -----------------------------------------------------------------------------------------
extern "C" int rq_batch_create(const rq_config* cfgs, const rq_atom* atoms, const int32_t* n_atoms, int32_t n_inst,
                               rq_batch** out) {
  if (!cfgs || !atoms || !n_atoms || !out || n_inst < 1) return RQ_EINVAL;
  *out = nullptr;
  const rq_config& c0 = cfgs[0];
  if (c0.flavor != RQ_FLAVOR_NEW) return RQ_ENOTSUP;
  for (int q = 0; q < n_inst; ++q) {
    const rq_config& c = cfgs[q];
    if (c.flavor != c0.flavor || c.precision != c0.precision || c.NN < 4 || c.NN % 2 || c.screen <= 0 ||
        std::fabs(c.screen / c.NN - c0.screen / c0.NN) > 1e-12 * (c0.screen / c0.NN) || n_atoms[q] < 1)
      return RQ_EINVAL;  // one flavour/precision and one grid spacing h for the whole batch
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return RQ_ENODEV;
  rq_batch* b = new (std::nothrow) rq_batch();
  if (!b) return RQ_ENOMEM;
  b->n = n_inst;
  b->cfg = c0;
  b->f64.assign(n_inst, c0.precision == RQ_PREC_FP64 ? 1 : 0);
  rq_config& f = b->cfg;  // the new flavour's defaults (capi.cu fill_defaults)
  if (f.poisson_interval <= 0) f.poisson_interval = 4;
  if (f.norm_interval <= 0) f.norm_interval = f.poisson_interval;
  if (f.label_interval <= 0) f.label_interval = 20;
  if (f.mg_pre <= 0) f.mg_pre = 1;
  if (f.mg_post <= 0) f.mg_post = 1;
  if (f.mg_coarse_sweeps <= 0) f.mg_coarse_sweeps = 16;
  if (f.boundary_speed <= 0) f.boundary_speed = 0.5;
  if (f.curv_reg == 0) f.curv_reg = 0.15;
  if (f.curv_reg < 0) f.curv_reg = 0;
  if (f.batch_tile == 0) f.batch_tile = kNmTile.lgk | (kNmTile.march << 8);
  b->tile = NmTile{f.batch_tile & 0xff, f.batch_tile >> 8};
  if (b->tile.lgk < 3 || b->tile.lgk > 6 || b->tile.march < 1 || b->tile.march > 64) {
    delete b;
    return RQ_EINVAL;  // 8..64 points along k, 1..64 planes per thread
  }
  b->dv = f.dv > 0 ? f.dv : 0.2;
  if (cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking) != cudaSuccess) {
    delete b;
    return RQ_ECUDA;
  }
  b->st = b->own;
  b->hin.resize(n_inst);
  b->atoms.resize(n_inst);
  const rq_atom* a = atoms;
  for (int q = 0; q < n_inst; ++q) {
    BInst& I = b->hin[q];
    std::memset(&I, 0, sizeof(I));
    const rq_config& c = cfgs[q];
    I.g = make_geo(c.NN + 1);
    I.h = c.screen / c.NN;
    I.nAt = I.nDom = n_atoms[q];
    I.dom0 = I.at0 = b->A;
    b->atoms[q].assign(a, a + n_atoms[q]);
    a += n_atoms[q];
    b->A += n_atoms[q];
    int nl = 1, nn = c.NN;
    const int want = c.mg_levels;
    while (nn % 2 == 0 && (want > 0 ? nl < want : nn / 2 >= 6) && nl < kMaxLev) {
      nn /= 2;
      nl++;
    }
    I.nlev = nl;
    double h = I.h;
    int m = c.NN;
    for (int l = 0; l < nl; ++l) {
      I.lg[l] = make_geo(m + 1);
      I.lh[l] = h;
      h *= 2;
      m /= 2;
    }
    b->maxlev = std::max(b->maxlev, nl);
  }
  b->D = b->A;
  b->active.assign(n_inst, 1);
  int rc = build(b);
  if (rc != RQ_OK) {
    std::fprintf(stderr, "rq_batch_create: %s\n", b->last_error.c_str());
    rq_batch_destroy(b);
    return rc;
  }
  *out = b;
  return RQ_OK;
}

extern "C" void rq_batch_destroy(rq_batch* b) {
  if (!b) return;
  cudaStreamSynchronize(b->st);
  for (auto& g : b->graph)
    if (g) cudaGraphExecDestroy(g);
  for (void* p : b->allocs) cudaFree(p);
  if (b->own) cudaStreamDestroy(b->own);
  delete b;
}

extern "C" const char* rq_batch_last_error(const rq_batch* b) { return b ? b->last_error.c_str() : "null batch"; }

extern "C" int rq_batch_set_stream(rq_batch* b, void* stream) {
  if (!b) return RQ_EINVAL;
  BCK(cudaStreamSynchronize(b->st));
  b->st = stream ? (cudaStream_t)stream : b->own;
  return RQ_OK;
}

extern "C" int rq_batch_initialize(rq_batch* b) {
  if (!b) return RQ_EINVAL;
  return b_initialize(b);
}

static int b_period(const rq_batch* b) {
  auto lcm = [](long x, long y) {
    long a = x, c = y;
    while (c) { long t = a % c; a = c; c = t; }
    return x / a * y;
  };
  const rq_config& f = b->cfg;
  return (int)lcm(lcm(f.poisson_interval, f.norm_interval), f.label_interval);
}

static int b_eager(rq_batch* b, int n) {
  for (int q = 0; q < n; ++q) {
    const int s = b->steps_done + 1;
    BRC(b_step(b, s));
    b->steps_done = s;
  }
  return RQ_OK;
}

// Items of instance q in a recorded phase (0 when q is not in the phase's work list).
static int b_phase_items(const rq_batch* b, const BPhase& x, int q) {
  if (!b->active[q] || (b->f64[q] ? kF64 : kF32) != x.set) return 0;
  const InstItems& it = b->items[q];
  switch (x.kind) {
    case kPhApply: return (int)it.flat16.size();
    case kPhZeroNorms:
    case kPhScale: return 1;
    case kPhUpdate:
    case kPhUpdateAcc:
    case kPhEvolve: return (int)it.march[0].size();
    case kPhRbgs:
    case kPhResidual:
    case kPhProlong: return (int)it.rbgs[x.lev].size();
    case kPhCoarsest: return (int)it.coarse[x.lev].size();
    case kPhRestrict: return (int)it.restr[x.lev].size();
    case kPhZero: return (int)it.zero[x.lev - 1].size();
    default: return 0;
  }
}

// One schedule period as ONE persistent launch: the period is recorded as a program of phases
// (the host state advances exactly as the per-kernel schedule would), with the queue offsets of
// the phases and, per (phase, instance), the instance's previous non-empty phase and its item
// count; all uploaded once per graph key.  The graph holds the zeroing of the counters and the
// cooperative launch of kb_persist over every co-resident block.
static int b_persist_graph(rq_batch* b, int key, int period) {
  // the kernel for the sets in use, and whether the device runs it (checked before recording,
  // which advances the host state)
  int sets = (b->pl[kF32].march[0].n ? 1 : 0) | (b->pl[kF64].march[0].n ? 2 : 0);
  if (!sets) sets = 1;
  void (*kern)(BPersist) = sets == 1 ? kb_persist<1> : sets == 2 ? kb_persist<2> : kb_persist<3>;
  if (b->pgrid[sets] == 0) {
    int dev = 0, nsm = 0, per = 0, coop = 0;
    BCK(cudaGetDevice(&dev));
    BCK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    BCK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    BCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, 256, 0));
    if (!coop || per < 1) {
      b->last_error = "the device cannot run the persistent batch launch (set batch_persistent = 0)";
      return RQ_ENOTSUP;
    }
    b->pgrid[sets] = nsm * per;
  }
  const int pgrid = b->pgrid[sets];
  std::vector<BPhase> prog;
  b->rec = &prog;
  const int rc = b_eager(b, period);
  b->rec = nullptr;
  if (rc != RQ_OK) return rc;
  const int nph = (int)prog.size(), ni = b->n;
  // the queue: per phase, per instance (in work-list order), chunks of up to `per` items, about
  // 4-16 k points each, so a chunk's bookkeeping (dependency check, fence, count) stays small
  // against its work
  std::vector<BChunk> chunks;
  std::vector<int2> deps((size_t)nph * ni);
  std::vector<int> last(ni, -1), lastn(ni, 0);
  for (int k = 0; k < nph; ++k) {
    const int kind = prog[k].kind;
    const int per = (kind == kPhRbgs || kind == kPhResidual || kind == kPhProlong) ? 8
                    : kind == kPhRestrict                                        ? 32
                    : (kind == kPhCoarsest || kind == kPhZeroNorms || kind == kPhScale) ? 1
                                                                                 : 2;
    int first = 0;
    for (int q = 0; q < ni; ++q) {
      deps[(size_t)k * ni + q] = make_int2(last[q], lastn[q] + b->extra_arrivals);
      const int c = b_phase_items(b, prog[k], q);
      for (int o = 0; o < c; o += per) chunks.push_back({k, first + o, std::min(per, c - o), q});
      first += c;
      if (c > 0) { last[q] = k; lastn[q] = c; }
    }
    if (first != prog[k].n) {
      b->last_error = "persistent program: work list and instance item counts disagree";
      return RQ_EINVAL;
    }
  }
  const int nch = (int)chunks.size();
  // device copies: program, queue offsets, dependencies (per key), counters (shared by the keys)
  rq_batch::Prog& G = b->prog[key];
  if (nph > G.cap || nch > G.cap_chunks) {
    BALLOC(G.phases, sizeof(BPhase) * nph);
    BALLOC(G.chunks, sizeof(BChunk) * nch);
    BALLOC(G.deps, sizeof(int2) * (size_t)nph * ni);
    G.cap = nph;
    G.cap_chunks = nch;
  }
  G.n = nph;
  if ((size_t)nph * ni + 1 > b->pcount_cap) {
    BALLOC(b->pcount, sizeof(unsigned) * ((size_t)nph * ni + 1));
    b->pcount_cap = (size_t)nph * ni + 1;
  }
  BCK(cudaMemcpyAsync(G.phases, prog.data(), sizeof(BPhase) * nph, cudaMemcpyHostToDevice, b->st));
  BCK(cudaMemcpyAsync(G.chunks, chunks.data(), sizeof(BChunk) * nch, cudaMemcpyHostToDevice, b->st));
  BCK(cudaMemcpyAsync(G.deps, deps.data(), sizeof(int2) * deps.size(), cudaMemcpyHostToDevice, b->st));
  BCK(cudaStreamSynchronize(b->st));  // the host vectors are copy sources
  BPersist a{};
  a.ins = b->din; a.prog = G.phases; a.chunks = G.chunks; a.deps = G.deps;
  a.queue = b->pcount; a.done = b->pcount + 1;
  a.nph = nph; a.ninst = ni;
  a.total = (unsigned)nch;
  a.half_dv = 0.5 * b->dv; a.dt = b->dv * b->hin[0].h * b->hin[0].h;
  a.dnorm = b->dnorm; a.scale = b->scale; a.Zdom = b->Zdom;
  a.sweeps = b->cfg.mg_coarse_sweeps;
  a.dt_w = (float)b->cfg.boundary_speed; a.curv = (float)b->cfg.curv_reg;
  a.err = b->err;
  a.limit_ns = b->wait_ns;
  a.tile = b->tile;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cudaLaunchConfig_t lc{};
  lc.gridDim = dim3((unsigned)pgrid);
  lc.blockDim = dim3(256);
  lc.dynamicSmemBytes = 0;
  lc.stream = b->st;
  lc.attrs = attr;
  lc.numAttrs = 1;
  BCK(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
  const cudaError_t e1 = cudaMemsetAsync(b->pcount, 0, sizeof(unsigned) * ((size_t)nph * ni + 1), b->st);
  const cudaError_t e2 = cudaLaunchKernelEx(&lc, kern, a);
  cudaGraph_t gr = nullptr;
  cudaError_t e = cudaStreamEndCapture(b->st, &gr);
  if (e == cudaSuccess) e = e1 != cudaSuccess ? e1 : e2;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&b->graph[key], gr, 0);
  if (gr) cudaGraphDestroy(gr);
  BCK(e);
  return RQ_OK;
}

extern "C" int rq_batch_step(rq_batch* b, int32_t n) {
  if (!b || n < 0) return RQ_EINVAL;
  const int period = b_period(b);
  int left = n;
  while (left > 0) {
    const int lu = b->cfg.label_until;
    const bool straddle = lu > 0 && b->steps_done < lu && b->steps_done + period > lu;
    const bool aligned = !straddle && period > 0 && period <= 4096 && b->steps_done % period == 0 && left >= period;
    if (!aligned) {
      int todo = left;
      if (period > 0 && b->steps_done % period != 0) todo = std::min(left, period - b->steps_done % period);
      else if (period > 0 && straddle) todo = std::min(left, period);
      int rc = b_eager(b, todo);
      if (rc != RQ_OK) return rc;
      left -= todo;
      continue;
    }
    const int on = (lu <= 0 || b->steps_done < lu) ? 1 : 0;
    const int key = b->cu | (b->cp << 1) | (b->cl << 2) | (on << 3) | ((b->pending ? 1 : 0) << 4);
    if (!b->graph[key]) {
      const long long l0 = b->launches;
      // the unbiased rounding's step seed advances on the device between steps, which needs the
      // steps in order: that schedule keeps the per-kernel launches
      if (b->cfg.batch_persistent == 1 && b->cfg.fp32_rounding != 1) {
        BRC(b_persist_graph(b, key, period));
        b->launches++;
      } else {
        BCK(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
        int rc = b_eager(b, period);
        cudaGraph_t gr = nullptr;
        cudaError_t e = cudaStreamEndCapture(b->st, &gr);
        if (rc != RQ_OK) {
          if (gr) cudaGraphDestroy(gr);
          return rc;
        }
        BCK(e);
        e = cudaGraphInstantiate(&b->graph[key], gr, 0);
        cudaGraphDestroy(gr);
        BCK(e);
      }
      b->graph_post[key] = b->cu | (b->cp << 1) | (b->cl << 2) | ((b->pending ? 1 : 0) << 4) | (b->age << 5);
      b->graph_launches[key] = b->launches - l0;
      BCK(cudaGraphLaunch(b->graph[key], b->st));
    } else {
      BCK(cudaGraphLaunch(b->graph[key], b->st));
      const int post = b->graph_post[key];
      b->cu = post & 1; b->cp = (post >> 1) & 1; b->cl = (post >> 2) & 1;
      b->pending = (post >> 4) & 1;
      b->age = post >> 5;
      b->steps_done += period;
      b->launches += b->graph_launches[key];
    }
    left -= period;
  }
  return RQ_OK;
}

extern "C" int rq_batch_energy(rq_batch* b, double* out) {
  if (!b || !out) return RQ_EINVAL;
  if (b->lastE.size() != (size_t)b->n * RQ_ENERGY_LEN) b->lastE.assign((size_t)b->n * RQ_ENERGY_LEN, 0.0);
  if (!any_active(b)) {  // nothing active: the cached energies are current
    std::memcpy(out, b->lastE.data(), sizeof(double) * b->lastE.size());
    return RQ_OK;
  }
  BRC(b_ready(b));
  BCK(cudaMemsetAsync(b->dpd, 0, sizeof(double) * kNmPD * b->D, b->st));
  BRC(each_set([&](auto tag, int p) -> int {
    using T = decltype(tag);
    const rq_batch::Plan& m = b->pl[p].march[0];
    if (!m.n) return RQ_OK;
    kb_energy<T><<<m.n, nm_march_block(), 0, b->st>>>(b->din, m.d, b->cu, b->cp, b->cl, b->dpd, b->tile);
    BL("energy");
    return RQ_OK;
  }));
  std::vector<double> pd((size_t)kNmPD * b->D);
  int bad_norm = 0;
  BCK(cudaMemcpyAsync(pd.data(), b->dpd, sizeof(double) * pd.size(), cudaMemcpyDeviceToHost, b->st));
  BCK(cudaMemcpyAsync(&bad_norm, b->err, sizeof(int), cudaMemcpyDeviceToHost, b->st));
  BCK(cudaStreamSynchronize(b->st));
  if (bad_norm) {  // reported once, then cleared
    BCK(cudaMemsetAsync(b->err, 0, sizeof(int), b->st));
    BCK(cudaStreamSynchronize(b->st));
    if (bad_norm & 2) {  // a persistent launch gave up at its barrier: the state is not a valid schedule
      b->last_error = "a bounded wait of the persistent batch launch ran out (rq_batch_set_wait)";
      return RQ_ETIMEOUT;
    }
    // a normalisation met a NaN/Inf domain norm and left that domain unscaled
    b->last_error = "non-finite domain norm in a normalisation";
    return RQ_ENONFINITE;
  }
  for (int q = 0; q < b->n; ++q) {
    const BInst& I = b->hin[q];
    double* o = out + (size_t)q * RQ_ENERGY_LEN;
    if (!b->active[q]) {  // instances dropped by solve keep their last energies
      std::memcpy(o, &b->lastE[(size_t)q * RQ_ENERGY_LEN], sizeof(double) * RQ_ENERGY_LEN);
      continue;
    }
    std::memset(o, 0, sizeof(double) * RQ_ENERGY_LEN);
    double pap = 0;
    for (int d = 0; d < I.nDom; ++d) {  // partials of the exactly normalised domains
      const double* x = &pd[kNmPD * ((size_t)I.dom0 + d)];
      const double w = domain_norm_weight(b->atoms[q][d].Z, x[0]);
      o[RQ_E_T] += w * x[1];
      o[RQ_E_EK] += w * x[2];
      o[RQ_E_EE] += 2.0 * w * x[3];
      pap += x[4];
    }
    o[RQ_E_EE] -= pap / (2.0 * M_PI);  // the P-stationary Hartree energy (nm_energy_readout)
    double ekk = 0;  // point-charge nuclear repulsion (bohr)
    const auto& at = b->atoms[q];
    for (size_t x = 0; x < at.size(); ++x)
      for (size_t y = x + 1; y < at.size(); ++y) {
        if (at[x].Z_nuc <= 0 || at[y].Z_nuc <= 0) continue;
        const double dx = (at[x].i - at[y].i) * I.h, dy = (at[x].j - at[y].j) * I.h, dz = (at[x].k - at[y].k) * I.h;
        ekk += at[x].Z_nuc * at[y].Z_nuc / std::sqrt(dx * dx + dy * dy + dz * dz);
      }
    o[RQ_E_KK] = ekk;
    o[RQ_E_TOTAL] = o[RQ_E_T] + o[RQ_E_EK] + o[RQ_E_EE] + ekk;
    std::memcpy(&b->lastE[(size_t)q * RQ_ENERGY_LEN], o, sizeof(double) * RQ_ENERGY_LEN);
    if (!std::isfinite(o[RQ_E_TOTAL])) {
      b->last_error = "non-finite energy in instance " + std::to_string(q);
      return RQ_ENONFINITE;
    }
  }
  return RQ_OK;
}

extern "C" int rq_batch_forces(rq_batch* b, double* F) {
  if (!b || !F) return RQ_EINVAL;
  for (char a : b->active)
    if (!a) {
      BRC(rq_batch_set_active_all(b));
      break;
    }
  BRC(b_ready(b));
  BCK(cudaMemsetAsync(b->dF, 0, sizeof(double) * 3 * b->A, b->st));
  BRC(each_set([&](auto tag, int p) -> int {
    using T = decltype(tag);
    const rq_batch::Plan& f = b->pl[p].force;
    if (!f.n) return RQ_OK;
    kb_force<T><<<f.n, 256, 0, b->st>>>(b->din, f.d, b->cu, b->cfg.sigma, b->dF);
    BL("force");
    return RQ_OK;
  }));
  BCK(cudaMemcpyAsync(F, b->dF, sizeof(double) * 3 * b->A, cudaMemcpyDeviceToHost, b->st));
  BCK(cudaStreamSynchronize(b->st));
  // add the point-charge nuclear repulsion forces
  for (int q = 0; q < b->n; ++q) {
    const BInst& I = b->hin[q];
    const auto& at = b->atoms[q];
    for (size_t x = 0; x < at.size(); ++x) {
      if (at[x].Z_nuc <= 0) continue;
      for (size_t y = 0; y < at.size(); ++y) {
        if (y == x || at[y].Z_nuc <= 0) continue;
        const double dx = (at[x].i - at[y].i) * I.h, dy = (at[x].j - at[y].j) * I.h, dz = (at[x].k - at[y].k) * I.h;
        const double r2 = dx * dx + dy * dy + dz * dz, w = at[x].Z_nuc * at[y].Z_nuc / (r2 * std::sqrt(r2));
        double* f = F + 3 * ((size_t)I.at0 + x);
        f[0] += w * dx; f[1] += w * dy; f[2] += w * dz;
      }
    }
  }
  return RQ_OK;
}

__global__ void kb_widen(const float* __restrict__ a, double* __restrict__ d, long long n) {
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    d[q] = (double)a[q];
}

// Move instance q of a mixed batch to its FP64 field set for the final refinement (psi must be
// in its normalised state): psi and P are widened into it; its K was computed in FP64 at
// initialisation, its multigrid levels are rebuilt by the next V-cycle, labels and W carry over.
// Nothing is allocated and the host does not wait.  The caller rebuilds the work lists.
static int b_promote(rq_batch* b, int q) {
  if (b->f64[q]) return RQ_OK;
  if (b->hin64.empty()) {
    b->last_error = "no FP64 field set for promotion";
    return RQ_EINVAL;
  }
  BInst& I = b->hin[q];
  const BInst& D = b->hin64[q];
  const long long S3 = I.g.S3;
  kb_widen<<<148 * 4, 256, 0, b->st>>>((const float*)I.U[b->cu], (double*)D.U[b->cu], S3);
  kb_widen<<<148 * 4, 256, 0, b->st>>>((const float*)I.P[b->cp], (double*)D.P[b->cp], S3);
  BCK(cudaGetLastError());
  I = D;
  b->f64[q] = 1;
  // from pageable host memory: the copy has read I when the call returns
  BCK(cudaMemcpyAsync(b->din + q, &I, sizeof(BInst), cudaMemcpyHostToDevice, b->st));
  return RQ_OK;
}

int rq_batch_set_active_all(rq_batch* b) {
  b->active.assign(b->n, 1);
  return build_plans(b);
}

// Converge every instance to |dE| < tol_dE between checks `check_interval` steps apart.  An
// fp32 instance first converges to max(tol_dE, kMixedFloor |E|), the change its fields
// resolve; if that is looser than tol_dE it moves to FP64 right there and refines to tol_dE
// (iterative refinement) while the other instances keep stepping.  Converged instances leave
// the work lists; converged_at[q] is the total step count at convergence (-1: not converged).
extern "C" int rq_batch_solve(rq_batch* b, double tol_dE, int32_t max_steps, int32_t check_interval,
                              int32_t* converged_at, double* E_final) {
  if (!b || max_steps < 0 || check_interval <= 0) return RQ_EINVAL;
  BRC(rq_batch_set_active_all(b));
  std::vector<double> e((size_t)b->n * RQ_ENERGY_LEN), prev(b->n), tol(b->n);
  BRC(rq_batch_energy(b, e.data()));
  for (int q = 0; q < b->n; ++q) {
    prev[q] = e[(size_t)q * RQ_ENERGY_LEN];
    tol[q] = b->f64[q] ? tol_dE : std::max(tol_dE, kMixedFloor * std::fabs(prev[q]));
  }
  std::vector<int> conv(b->n, -1), run(b->n, 0);
  const int need = b->cfg.converge_checks > 0 ? b->cfg.converge_checks : 1;
  int taken = 0, left = b->n;
  while (taken < max_steps && left > 0) {
    const int n = std::min(check_interval, max_steps - taken);
    BRC(rq_batch_step(b, n));
    taken += n;
    BRC(rq_batch_energy(b, e.data()));  // psi is now in its normalised state
    bool changed = false;
    for (int q = 0; q < b->n; ++q) {
      if (!b->active[q]) continue;
      const double E = e[(size_t)q * RQ_ENERGY_LEN], d = std::fabs(E - prev[q]);
      prev[q] = E;
      if (d >= tol[q]) {
        run[q] = 0;
        continue;
      }
      if (!b->f64[q] && tol[q] > tol_dE) {  // fp32 has stalled: refine in FP64 from here
        changed = true;
        BRC(b_promote(b, q));
        tol[q] = tol_dE;
        run[q] = 0;
      } else if (++run[q] >= need) {
        changed = true;
        conv[q] = taken;
        b->active[q] = 0;
        left--;
      }
    }
    if (changed) BRC(build_plans(b));
  }
  BRC(rq_batch_energy(b, e.data()));
  for (int q = 0; q < b->n; ++q) {
    if (converged_at) converged_at[q] = conv[q];
    if (E_final) E_final[q] = e[(size_t)q * RQ_ENERGY_LEN];
  }
  return rq_batch_set_active_all(b);
}

extern "C" int rq_batch_info(const rq_batch* b, int32_t* n_inst, int64_t* total_points, int64_t* interior_points,
                             int64_t* kernel_launches) {
  if (!b) return RQ_EINVAL;
  long long tp = 0, ip = 0;
  for (const auto& I : b->hin) {
    tp += I.g.S3;
    ip += (long long)(I.g.NN - 1) * (I.g.NN - 1) * (I.g.NN - 1);
  }
  if (n_inst) *n_inst = b->n;
  if (total_points) *total_points = tp;
  if (interior_points) *interior_points = ip;
  if (kernel_launches) *kernel_launches = b->launches;
  return RQ_OK;
}

extern "C" int rq_batch_set_wait(rq_batch* b, int64_t limit_ns, int32_t extra_arrivals) {
  if (!b || limit_ns <= 0 || extra_arrivals < 0) return RQ_EINVAL;
  BCK(cudaStreamSynchronize(b->st));
  b->wait_ns = limit_ns;
  b->extra_arrivals = extra_arrivals;
  for (auto& g : b->graph)  // the limits are arguments of the captured launches
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  return RQ_OK;
}

static void b_drop_graphs(rq_batch* b) {
  for (auto& g : b->graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

// the work lists for another march tile (the per-instance items, then the plans)
static int b_retile(rq_batch* b, NmTile t) {
  b->tile = t;
  b->cfg.batch_tile = t.lgk | (t.march << 8);
  for (int q = 0; q < b->n; ++q) make_items(b->hin[q], q, b->items[q], t, b->rr_pl, b->pr_pl);
  return build_plans(b);
}

// sum of the squared fine-grid residual over the active instances
static int b_resnorm(rq_batch* b, double* dsum, double& out) {
  BCK(cudaMemsetAsync(dsum, 0, sizeof(double), b->st));
  BRC(each_set([&](auto tag, int p) -> int {
    using T = decltype(tag);
    const rq_batch::Plan& r = b->pl[p].rbgs[0];
    if (!r.n) return RQ_OK;
    kb_resnorm<T><<<r.n, dim3(32, 8), 0, b->st>>>(b->din, r.d, b->cu, b->cp, dsum);
    BL("resnorm");
    return RQ_OK;
  }));
  BCK(cudaMemcpyAsync(&out, dsum, sizeof(double), cudaMemcpyDeviceToHost, b->st));
  BCK(cudaStreamSynchronize(b->st));
  return RQ_OK;
}

extern "C" int rq_batch_autotune(rq_batch* b, rq_tune_report* out) {
  if (!b || !out) return RQ_EINVAL;
  std::memset(out, 0, sizeof(*out));
  if (!any_active(b)) return RQ_OK;
  const int period = b_period(b);
  BRC(b_ready(b));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  BCK(cudaEventCreate(&e0));
  BCK(cudaEventCreate(&e1));
  auto cleanup = [&]() { cudaEventDestroy(e0); cudaEventDestroy(e1); };
  int rc = RQ_OK;
  // 1. march tile x launch form, timed per step over one captured period
  const NmTile keep = b->tile;
  const int keep_persistent = b->cfg.batch_persistent;
  double best = 1e300;
  int nt = 0;
  for (int lgk : {4, 5})
    for (int march : {8, 16, 32})
      for (int pers : {0, 1}) {
        if (pers && b->cfg.fp32_rounding == 1) continue;  // that schedule keeps the per-kernel launches
        if ((rc = b_retile(b, NmTile{lgk, march})) != RQ_OK) break;
        b->cfg.batch_persistent = pers;
        b_drop_graphs(b);
        if (b->steps_done % period) rc = rq_batch_step(b, period - b->steps_done % period);
        if (rc == RQ_OK) rc = rq_batch_step(b, period);  // captures the period
        if (pers && rc == RQ_ENOTSUP) {  // no cooperative launch here: per-kernel graphs only
          rc = RQ_OK;
          continue;
        }
        if (rc == RQ_OK && cudaEventRecord(e0, b->st) != cudaSuccess) rc = RQ_ECUDA;
        if (rc == RQ_OK) rc = rq_batch_step(b, period);
        if (rc == RQ_OK && cudaEventRecord(e1, b->st) != cudaSuccess) rc = RQ_ECUDA;
        float ms = 0.f;
        if (rc == RQ_OK && (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
          rc = RQ_ECUDA;
        if (rc != RQ_OK) break;
        out->tile[nt] = lgk | (march << 8);
        out->persistent[nt] = pers;
        out->ms_per_step[nt] = ms / period;
        if (out->ms_per_step[nt] < best) { best = out->ms_per_step[nt]; out->best_tile = nt; }
        ++nt;
      }
  out->n_tile = nt;
  if (rc == RQ_OK && nt > 0) {
    const int t = out->tile[out->best_tile];
    rc = b_retile(b, NmTile{t & 0xff, t >> 8});
    b->cfg.batch_persistent = out->persistent[out->best_tile];
    b_drop_graphs(b);
  } else {
    b_retile(b, keep);
    b->cfg.batch_persistent = keep_persistent;
  }
  // 2. smoother sweeps: 3 V-cycles from P = 0 on the current psi, P restored after each
  if (rc == RQ_OK && !b->dtune) rc = balloc(b, (void**)&b->dtune, sizeof(double));
  if (rc == RQ_OK) rc = b_flush(b);
  const int cand[7][3] = {{1, 1, 16}, {2, 1, 16}, {1, 2, 16}, {2, 2, 16}, {1, 1, 8}, {1, 1, 32}, {2, 2, 32}};
  const rq_config keepc = b->cfg;
  double best_eff = -1.0;  // the kept candidate's ms per cycle
  int ns = 0;
  for (int c = 0; c < 7 && rc == RQ_OK; ++c) {
    b->cfg.mg_pre = cand[c][0];
    b->cfg.mg_post = cand[c][1];
    b->cfg.mg_coarse_sweeps = cand[c][2];
    for (int q = 0; q < b->n && rc == RQ_OK; ++q) {
      if (!b->active[q]) continue;
      const BInst& I = b->hin[q];
      const size_t bytes = (b->f64[q] ? sizeof(double) : sizeof(float)) * (size_t)I.g.S3;
      if (cudaMemcpyAsync(I.P[1 - b->cp], I.P[b->cp], bytes, cudaMemcpyDeviceToDevice, b->st) != cudaSuccess ||
          cudaMemsetAsync(I.P[b->cp], 0, bytes, b->st) != cudaSuccess)
        rc = RQ_ECUDA;
    }
    double r0 = 0, r3 = 0;
    if (rc == RQ_OK) rc = b_resnorm(b, b->dtune, r0);
    if (rc == RQ_OK && cudaEventRecord(e0, b->st) != cudaSuccess) rc = RQ_ECUDA;
    for (int v = 0; v < 3 && rc == RQ_OK; ++v)
      rc = each_set([&](auto tag, int p) { return b_vcycle<decltype(tag)>(b, p); });
    if (rc == RQ_OK && cudaEventRecord(e1, b->st) != cudaSuccess) rc = RQ_ECUDA;
    if (rc == RQ_OK) rc = b_resnorm(b, b->dtune, r3);
    float ms = 0.f;
    if (rc == RQ_OK && cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) rc = RQ_ECUDA;
    for (int q = 0; q < b->n && rc == RQ_OK; ++q) {
      if (!b->active[q]) continue;
      const BInst& I = b->hin[q];
      const size_t bytes = (b->f64[q] ? sizeof(double) : sizeof(float)) * (size_t)I.g.S3;
      if (cudaMemcpyAsync(I.P[b->cp], I.P[1 - b->cp], bytes, cudaMemcpyDeviceToDevice, b->st) != cudaSuccess) rc = RQ_ECUDA;
    }
    if (rc != RQ_OK) break;
    const double rho = r0 > 0 ? std::pow(std::sqrt(r3 / r0), 1.0 / 3.0) : 1.0;
    out->pre[ns] = cand[c][0];
    out->post[ns] = cand[c][1];
    out->coarse_sweeps[ns] = cand[c][2];
    out->rho[ns] = rho;
    out->ms_per_cycle[ns] = ms / 3.0;
    ++ns;
  }
  out->n_smooth = ns;
  // The cheapest cycle that reduces the residual at least as well as V(1,1) with 16 coarsest sweeps
  // (candidate 0, to 5 %): one warm-started cycle every poisson_interval steps already keeps P on
  // the ITP state at that rate (mixed and FP64 solves take the same steps), so more smoothing only
  // costs time.
  for (int c = 0; c < ns; ++c)
    if (out->rho[c] <= 1.05 * out->rho[0] && (best_eff < 0 || out->ms_per_cycle[c] < best_eff)) {
      best_eff = out->ms_per_cycle[c];
      out->best_smooth = c;
    }
  if (rc == RQ_OK && ns > 0) {
    b->cfg.mg_pre = out->pre[out->best_smooth];
    b->cfg.mg_post = out->post[out->best_smooth];
    b->cfg.mg_coarse_sweeps = out->coarse_sweeps[out->best_smooth];
  } else {
    b->cfg.mg_pre = keepc.mg_pre;
    b->cfg.mg_post = keepc.mg_post;
    b->cfg.mg_coarse_sweeps = keepc.mg_coarse_sweeps;
  }
  b_drop_graphs(b);  // the periods change with the sweeps
  if (rc == RQ_OK && cudaStreamSynchronize(b->st) != cudaSuccess) rc = RQ_ECUDA;
  cleanup();
  return rc;
}

extern "C" int rq_batch_synchronize(rq_batch* b) {
  if (!b) return RQ_EINVAL;
  BCK(cudaStreamSynchronize(b->st));
  return RQ_OK;
}
