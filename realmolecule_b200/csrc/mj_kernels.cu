// mj_kernels.cu -- the molecule.js flavour of the solver step on sm_100a.
//
// Each kernel restates one WGSL compute shader of molecule.js with the same f32 operations
// in the same order (explicitly rounded), so outputs are bit-identical to the strict-f32
// oracle.  B200-specific changes:
//  * the per-neighbour "inside its label's r_c sphere" tests of updateU (molecule.js:246-259,
//    seven sqrt per cell) are precomputed once per label change into bit 30 of the label word
//    (kMjExcl), so the update reads one int per neighbour like the solver.py flavour;
//  * rhoTotal = psi^2 is computed inside the Jacobi sweep (no separate pass);
//  * the u32 fixed-point norms (molecule.js:912-946) are aggregated per block in shared memory
//    before the global atomics -- integer adds, so the result is bit-exact in any order.
#include <algorithm>

#include "rq_flavors.h"
#include "rq_kernels.h"

namespace rq {

constexpr int kMjExcl = 0x40000000;  // bit 30 of a stored label: cell inside its label's r_c sphere
constexpr int kMjMask = 0x3FFFFFFF;

__device__ __forceinline__ float mj_dist(int ci, int cj, int ck, const MjAtom& a, float h) {
  const float dx = F_MUL(F_SUB((float)ci, (float)a.posI), h);
  const float dy = F_MUL(F_SUB((float)cj, (float)a.posJ), h);
  const float dz = F_MUL(F_SUB((float)ck, (float)a.posK), h);
  return F_SQRT(F_ADD(F_ADD(F_MUL(dx, dx), F_MUL(dy, dy)), F_MUL(dz, dz)));
}

// molecule.js:246-259 isInsideRc(ci, cj, ck, lbl)
__device__ __forceinline__ bool mj_inside_rc(int ci, int cj, int ck, int lbl, const MjAtom* __restrict__ atoms,
                                             int nAt, bool hasBare, float h) {
  const MjAtom a = atoms[lbl];
  if (a.rc > 0.f && mj_dist(ci, cj, ck, a, h) < a.rc) return true;
  if (hasBare)
    for (int n = 0; n < nAt; ++n) {
      const MjAtom b = atoms[n];
      if (b.Z <= 0.f && b.Z_nuc > 0.f && b.rc > 0.f && mj_dist(ci, cj, ck, b, h) < b.rc) return true;
    }
  return false;
}

// inSplitAtom (molecule.js:197-226), d = cell - nucleus in bohr, r = |d|: the entry owns the
// cell iff it lies in its sector.  atan2 is the f64 function rounded once to f32 (WGSL leaves its
// accuracy to the implementation; the oracle does the same).
__device__ bool mj_in_split(float dx, float dy, float dz, float r, const MjSplit& s) {
  if (s.type <= 1u || r < 1e-6f) return true;
  const float axL = fmaxf(F_SQRT(F_ADD(F_ADD(F_MUL(s.ax, s.ax), F_MUL(s.ay, s.ay)), F_MUL(s.az, s.az))), 1e-12f);
  const float a0 = F_DIV(s.ax, axL), a1 = F_DIV(s.ay, axL), a2 = F_DIV(s.az, axL);
  const float dotp = F_ADD(F_ADD(F_MUL(dx, a0), F_MUL(dy, a1)), F_MUL(dz, a2));
  if (s.type == 2u) return s.idx == 0u ? dotp < 0.f : dotp >= 0.f;
  if (s.type == 3u) {
    const float px = F_SUB(dx, F_MUL(dotp, a0)), py = F_SUB(dy, F_MUL(dotp, a1)), pz = F_SUB(dz, F_MUL(dotp, a2));
    float e1x, e1y, e1z;
    if (fabsf(a2) < 0.9f) { e1x = a1; e1y = -a0; e1z = 0.f; } else { e1x = 0.f; e1y = a2; e1z = -a1; }
    const float e1L = fmaxf(F_SQRT(F_ADD(F_ADD(F_MUL(e1x, e1x), F_MUL(e1y, e1y)), F_MUL(e1z, e1z))), 1e-12f);
    e1x = F_DIV(e1x, e1L); e1y = F_DIV(e1y, e1L); e1z = F_DIV(e1z, e1L);
    const float e2x = F_SUB(F_MUL(a1, e1z), F_MUL(a2, e1y)), e2y = F_SUB(F_MUL(a2, e1x), F_MUL(a0, e1z)),
                e2z = F_SUB(F_MUL(a0, e1y), F_MUL(a1, e1x));
    const float pe1 = F_ADD(F_ADD(F_MUL(px, e1x), F_MUL(py, e1y)), F_MUL(pz, e1z));
    const float pe2 = F_ADD(F_ADD(F_MUL(px, e2x), F_MUL(py, e2y)), F_MUL(pz, e2z));
    float th = F_SUB((float)atan2((double)pe2, (double)pe1), s.rot);
    if (th < -3.14159265f) th = F_ADD(th, 6.28318530f);
    if (th > 3.14159265f) th = F_SUB(th, 6.28318530f);
    const unsigned sector = __float2uint_rz(floorf(F_DIV(F_ADD(th, 3.14159265f), 2.09439510f))) % 3u;
    return sector == s.idx;
  }
  return true;
}

// evolveBoundary's cellSectorOK (molecule.js:437-442): d = (cell - nucleus) * h.
__device__ __forceinline__ bool mj_sector_ok(int i, int j, int k, int n, const MjAtom* __restrict__ atoms,
                                             const MjSplit* __restrict__ splits, float h) {
  const MjSplit s = splits[n];
  if (s.type <= 1u) return true;
  const MjAtom a = atoms[n];
  const float dx = F_MUL(F_SUB((float)i, (float)a.posI), h);
  const float dy = F_MUL(F_SUB((float)j, (float)a.posJ), h);
  const float dz = F_MUL(F_SUB((float)k, (float)a.posK), h);
  return mj_in_split(dx, dy, dz, F_SQRT(F_ADD(F_ADD(F_MUL(dx, dx), F_MUL(dy, dy)), F_MUL(dz, dz))), s);
}

__device__ __forceinline__ int mj_pack(int ci, int cj, int ck, int lbl, const MjAtom* atoms, int nAt, bool hasBare,
                                       float h) {
  return lbl | (mj_inside_rc(ci, cj, ck, lbl, atoms, nAt, hasBare, h) ? kMjExcl : 0);
}

// ---------------------------------------------------------------------------------------
// init: molecule.js:1377-1426 gpuInitAccum over all atoms in one pass (identical to its
// 50-atom batches: the running K / bestU / label carry over in the same order) + :1437-1449.
// ---------------------------------------------------------------------------------------
// With PERSIST (moveNuclei's K rebuild, molecule.js:4563-4582) K restarts from 0 but the
// running maximum bestU and the current label persist, so a moved atom can take cells over;
// psi is not touched.  Without PERSIST (initial upload) everything starts from 0 and psi = bestU.
template <bool PERSIST>
__global__ void __launch_bounds__(256) k_mj_init(float* __restrict__ K, float* __restrict__ U, float* __restrict__ bestU,
                                                 int* __restrict__ label, const MjAtom* __restrict__ atoms, int nAt,
                                                 Geo g, float h, float h2, float Rsing, bool hasBare,
                                                 const MjSplit* __restrict__ splits) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= g.S3) return;
  const int S = g.S;
  const int i = (int)(id / g.S2), j = (int)((id / S) % S), kk = (int)(id % S);
  const float xi = F_MUL((float)i, h), yj = F_MUL((float)j, h), zk = F_MUL((float)kk, h);
  float Kval = 0.f, bU = PERSIST ? bestU[id] : 0.f;
  int bestN = PERSIST ? (label[id] & kMjMask) : 0;
  for (int n = 0; n < nAt; ++n) {
    const MjAtom a = atoms[n];
    const float Za = a.Z;
    const float Zn = (a.Z_nuc > 0.f) ? a.Z_nuc : Za;
    if (Za <= 0.f && Zn <= 0.f) continue;
    const float dx = F_SUB(xi, F_MUL((float)a.posI, h));
    const float dy = F_SUB(yj, F_MUL((float)a.posJ, h));
    const float dz = F_SUB(zk, F_MUL((float)a.posK, h));
    const float r2 = F_ADD(F_ADD(F_MUL(dx, dx), F_MUL(dy, dy)), F_MUL(dz, dz));
    const float r = (a.rc > 0.f) ? fmaxf(F_SQRT(F_ADD(r2, F_MUL(0.04f, h2))), a.rc) : fmaxf(F_SQRT(r2), Rsing);
    Kval = F_ADD(Kval, F_DIV(Zn, r));
    const float rReal = F_SQRT(r2);
    const float Ze = a.initZeff;
    const bool okSplit = mj_in_split(dx, dy, dz, rReal, splits[n]);  // the entry's sector (:1413)
    const float uT = (rReal > a.initRcut || Za <= 0.f || !okSplit) ? 0.f
                                                       : F_MUL(F_MUL(F_MUL(Ze, Ze), 0.5641895835f), expf(F_MUL(-Ze, r)));
    if (uT > bU) { bU = uT; bestN = n; }
  }
  K[id] = Kval;
  bestU[id] = bU;
  if (!PERSIST) U[id] = bU;
  label[id] = mj_pack(i, j, kk, bestN, atoms, nAt, hasBare, h);
}

// molecule.js:1337-1370 recomputeK (all S^3 points).
__global__ void __launch_bounds__(256) k_mj_recompute_k(float* __restrict__ K, const MjAtom* __restrict__ atoms,
                                                        int nAt, Geo g, float h, float Rsing) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= g.S3) return;
  const int S = g.S;
  const int i = (int)(id / g.S2), j = (int)((id / S) % S), kk = (int)(id % S);
  float Kval = 0.f;
  for (int n = 0; n < nAt; ++n) {
    const MjAtom a = atoms[n];
    const float Za = a.Z;
    const float Zn = (a.Z_nuc > 0.f) ? a.Z_nuc : Za;
    if (Za <= 0.f && Zn <= 0.f) continue;
    const float di = F_MUL(F_SUB((float)i, (float)a.posI), h);
    const float dj = F_MUL(F_SUB((float)j, (float)a.posJ), h);
    const float dk = F_MUL(F_SUB((float)kk, (float)a.posK), h);
    const float r = F_SQRT(F_ADD(F_ADD(F_MUL(di, di), F_MUL(dj, dj)), F_MUL(dk, dk)));
    const float reff = (a.rc > 0.f) ? fmaxf(r, a.rc) : fmaxf(r, Rsing);
    Kval = F_ADD(Kval, F_DIV(Zn, reff));
  }
  K[id] = Kval;
}

// Recompute the exclusion bit of every stored label (after nuclei move or a label upload).
__global__ void __launch_bounds__(256) k_mj_flags(int* __restrict__ label, const MjAtom* __restrict__ atoms, int nAt,
                                                  Geo g, float h, bool hasBare) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= g.S3) return;
  const int S = g.S;
  const int i = (int)(id / g.S2), j = (int)((id / S) % S), kk = (int)(id % S);
  label[id] = mj_pack(i, j, kk, label[id] & kMjMask, atoms, nAt, hasBare, h);
}

// ---------------------------------------------------------------------------------------
// updateU (molecule.js:263-343, W_CUTOFF = 0): 20 B per interior point.  With ACC the new
// psi's u32 fixed-point norm per label (molecule.js:912-933) is accumulated as well.
// ---------------------------------------------------------------------------------------
// With CHEB the Chebyshev step (molecule.js:345-421): out = omega * (the ITP step) + (1 - omega) *
// psi_{n-1}, where psi_{n-1} is what Uo holds (the input of the previous step), read at the cell
// before it is overwritten.
template <bool ACC, bool CHEB = false>
__global__ void __launch_bounds__(256) k_mj_update(const float* __restrict__ U, float* __restrict__ Uo,
                                                   const float* __restrict__ K, const int* __restrict__ label,
                                                   const float* __restrict__ Pother, Geo g, float half_d, float dt,
                                                   float h3, int nDom, unsigned* __restrict__ unorm,
                                                   float omega = 1.0f) {
  constexpr int NSLOT = 128;
  __shared__ int keys[NSLOT];
  __shared__ unsigned vals[NSLOT];
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  if (ACC) {
    for (int s = tid; s < NSLOT; s += blockDim.x * blockDim.y) { keys[s] = -1; vals[s] = 0u; }
    __syncthreads();
  }
  const int k = 1 + blockIdx.x * kThreadsK + threadIdx.x;
  const int j = 1 + blockIdx.y * kThreadsJ + threadIdx.y;
  const int i0 = 1 + blockIdx.z * kMarch;
  int runL = -1;
  unsigned runV = 0u;
  auto flush_run = [&]() {
    if (runL < 0) return;
    unsigned slot = ((unsigned)runL * 2654435761u) & (NSLOT - 1);
    for (int p = 0; p < NSLOT; ++p) {
      const int old = atomicCAS(&keys[slot], -1, runL);
      if (old == -1 || old == runL) { atomicAdd(&vals[slot], runV); return; }
      slot = (slot + 1) & (NSLOT - 1);
    }
    atomicAdd(&unorm[runL], runV);
  };
  if (k < g.NN && j < g.NN && i0 < g.NN) {
    const int iend = min(i0 + kMarch, g.NN);
    const long long S = g.S, S2 = g.S2;
    long long id = (long long)i0 * S2 + j * S + k;
    float u_m = __ldg(U + id - S2), u_c = __ldg(U + id);
    int l_m = __ldg(label + id - S2), l_c = __ldg(label + id);
    for (int i = i0; i < iend; ++i, id += S2) {
      const float u_p = __ldg(U + id + S2);
      const int l_p = __ldg(label + id + S2);
      float out;
      if (l_c & kMjExcl) {
        out = 0.0f;  // Dirichlet inside the own r_c sphere
      } else {
        const float ujp = __ldg(U + id + S), ujm = __ldg(U + id - S), ukp = __ldg(U + id + 1), ukm = __ldg(U + id - 1);
        const int ljp = __ldg(label + id + S), ljm = __ldg(label + id - S), lkp = __ldg(label + id + 1),
                  lkm = __ldg(label + id - 1);
        // a neighbour is used iff same label and not inside its r_c sphere: packed words equal
        const float a = (l_p == l_c) ? u_p : u_c;
        const float b = (l_m == l_c) ? u_m : u_c;
        const float c = (ljp == l_c) ? ujp : u_c;
        const float d = (ljm == l_c) ? ujm : u_c;
        const float e = (lkp == l_c) ? ukp : u_c;
        const float f = (lkm == l_c) ? ukm : u_c;
        const float lap = F_SUB(F_ADD(F_ADD(F_ADD(F_ADD(F_ADD(a, b), c), d), e), f), F_MUL(6.0f, u_c));
        out = F_ADD(F_ADD(u_c, F_MUL(half_d, lap)),
                    F_MUL(F_MUL(dt, F_SUB(__ldg(K + id), F_MUL(2.0f, __ldg(Pother + id)))), u_c));
        if (CHEB) out = F_ADD(F_MUL(omega, out), F_MUL(F_SUB(1.0f, omega), Uo[id]));
      }
      Uo[id] = out;
      if (ACC) {
        const unsigned contrib = __float2uint_rz(F_MUL(F_MUL(F_MUL(out, out), h3), 16777216.0f));
        const int L = l_c & kMjMask;
        if (L != runL) { flush_run(); runL = L; runV = contrib; } else { runV += contrib; }
      }
      u_m = u_c; u_c = u_p; l_m = l_c; l_c = l_p;
    }
  }
  if (ACC) {
    flush_run();
    __syncthreads();
    for (int s = tid; s < NSLOT; s += blockDim.x * blockDim.y)
      if (keys[s] >= 0) atomicAdd(&unorm[keys[s]], vals[s]);
  }
}

// decodeNorms + the scale of normalize (molecule.js:938-946, :1098-1104): n = f32(acc)*2^-24,
// scale = sqrt(Z/n) if n > 0 and Z > 0 else 1.
__global__ void k_mj_norm_scale(const unsigned* __restrict__ unorm, const MjAtom* __restrict__ atoms, int nDom,
                                float* __restrict__ scale) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= nDom) return;
  const float n = F_MUL((float)unorm[l], 5.9604644775390625e-08f);
  const float Z = atoms[l].Z;
  scale[l] = (n > 0.f && Z > 0.f) ? F_SQRT(F_DIV(Z, n)) : 1.0f;
}

__global__ void __launch_bounds__(256) k_mj_apply_scale(float* __restrict__ U, const int* __restrict__ label,
                                                        const float* __restrict__ scale, Geo g) {
  const int k = 1 + blockIdx.x * kThreadsK + threadIdx.x;
  const int j = 1 + blockIdx.y * kThreadsJ + threadIdx.y;
  const int i0 = 1 + blockIdx.z * kMarch;
  if (k >= g.NN || j >= g.NN || i0 >= g.NN) return;
  const int iend = min(i0 + kMarch, g.NN);
  for (int i = i0; i < iend; ++i) {
    const long long id = (long long)i * g.S2 + (long long)j * g.S + k;
    U[id] = F_MUL(U[id], scale[label[id] & kMjMask]);
  }
}

// Weighted Jacobi with rho = psi^2 inline (molecule.js:723-749, :754-774).  12 B per point.
__global__ void __launch_bounds__(256) k_mj_jacobi(const float* __restrict__ Pin, float* __restrict__ Pout,
                                                   const float* __restrict__ U, Geo g, float h2, float two_pi) {
  const int k = 1 + blockIdx.x * kThreadsK + threadIdx.x;
  const int j = 1 + blockIdx.y * kThreadsJ + threadIdx.y;
  const int i0 = 1 + blockIdx.z * kMarch;
  if (k >= g.NN || j >= g.NN || i0 >= g.NN) return;
  const int iend = min(i0 + kMarch, g.NN);
  const long long S = g.S, S2 = g.S2;
  long long id = (long long)i0 * S2 + j * S + k;
  float p_m = __ldg(Pin + id - S2), p_c = __ldg(Pin + id);
  const float c0 = F_MUL(h2, two_pi);
  for (int i = i0; i < iend; ++i, id += S2) {
    const float p_p = __ldg(Pin + id + S2);
    const float u = __ldg(U + id);
    const float sn = F_ADD(F_ADD(F_ADD(F_ADD(F_ADD(p_p, p_m), __ldg(Pin + id + S)), __ldg(Pin + id - S)),
                                 __ldg(Pin + id + 1)),
                           __ldg(Pin + id - 1));
    const float rhs = F_MUL(c0, F_MUL(u, u));
    Pout[id] = F_ADD(F_MUL(0.3333f, p_c), F_DIV(F_ADD(sn, rhs), 9.0f));
    p_m = p_c; p_c = p_p;
  }
}

// The same weighted Jacobi sweep with the right-hand side read from a density buffer: the
// self-potential solve of the self-interaction correction (jacobiSmooth with rhoTotal bound to
// the single-domain density, molecule.js:723-749, :3024-3030).
__global__ void __launch_bounds__(256) k_mj_jacobi_rho(const float* __restrict__ Pin, float* __restrict__ Pout,
                                                       const float* __restrict__ rho, Geo g, float h2, float two_pi) {
  const int k = 1 + blockIdx.x * kThreadsK + threadIdx.x;
  const int j = 1 + blockIdx.y * kThreadsJ + threadIdx.y;
  const int i0 = 1 + blockIdx.z * kMarch;
  if (k >= g.NN || j >= g.NN || i0 >= g.NN) return;
  const int iend = min(i0 + kMarch, g.NN);
  const long long S = g.S, S2 = g.S2;
  long long id = (long long)i0 * S2 + j * S + k;
  float p_m = __ldg(Pin + id - S2), p_c = __ldg(Pin + id);
  const float c0 = F_MUL(h2, two_pi);
  for (int i = i0; i < iend; ++i, id += S2) {
    const float p_p = __ldg(Pin + id + S2);
    const float sn = F_ADD(F_ADD(F_ADD(F_ADD(F_ADD(p_p, p_m), __ldg(Pin + id + S)), __ldg(Pin + id - S)),
                                 __ldg(Pin + id + 1)),
                           __ldg(Pin + id - 1));
    const float rhs = F_MUL(c0, __ldg(rho + id));
    Pout[id] = F_ADD(F_MUL(0.3333f, p_c), F_DIV(F_ADD(sn, rhs), 9.0f));
    p_m = p_c; p_c = p_p;
  }
}

// ---------------------------------------------------------------------------------------
// the 2-level V-cycle of molecule.js:777-909 (one thread per point; it runs every
// POISSON_INTERVAL steps at most)
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ bool interior_of(long long id, const Geo& g, int& i, int& j, int& k) {
  i = (int)(id / g.S2); j = (int)((id / g.S) % g.S); k = (int)(id % g.S);
  return i >= 1 && i < g.NN && j >= 1 && j < g.NN && k >= 1 && k < g.NN;
}

__global__ void k_mj_rho(const float* __restrict__ U, float* __restrict__ rho, Geo g) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, k;
  if (id >= g.S3 || !interior_of(id, g, i, j, k)) return;
  const float u = U[id];
  rho[id] = F_MUL(u, u);
}

// computeRhoSelf (molecule.js:572-590): psi^2 where the label is m, 0 elsewhere (interior points)
__global__ void k_mj_rho_self(const float* __restrict__ U, const int* __restrict__ label, int m,
                              float* __restrict__ rho, Geo g) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, k;
  if (id >= g.S3 || !interior_of(id, g, i, j, k)) return;
  const float u = U[id];
  rho[id] = ((label[id] & kMjMask) == m) ? F_MUL(u, u) : 0.0f;
}

// subtractPself (molecule.js:694-721): Pother -= Pm * frac where the label is m
__global__ void k_mj_sub_self(const float* __restrict__ Pm, float* __restrict__ Pother, const int* __restrict__ label,
                              int m, float frac, Geo g) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, k;
  if (id >= g.S3 || !interior_of(id, g, i, j, k)) return;
  if ((label[id] & kMjMask) == m) Pother[id] = F_SUB(Pother[id], F_MUL(Pm[id], frac));
}

// computeRhoOther (molecule.js:593-612): psi^2 except where the label is m (interior points)
__global__ void k_mj_rho_other(const float* __restrict__ U, const int* __restrict__ label, int m,
                               float* __restrict__ rho, Geo g) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, k;
  if (id >= g.S3 || !interior_of(id, g, i, j, k)) return;
  const float u = U[id];
  rho[id] = ((label[id] & kMjMask) == m) ? 0.0f : F_MUL(u, u);
}

// copyPotherForLabel (molecule.js:651-671): Pother = Psrc where the label is m
__global__ void k_mj_copy_for_label(const float* __restrict__ Psrc, float* __restrict__ Pother,
                                    const int* __restrict__ label, int m, Geo g) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, k;
  if (id >= g.S3 || !interior_of(id, g, i, j, k)) return;
  if ((label[id] & kMjMask) == m) Pother[id] = Psrc[id];
}

// initPdirect (molecule.js:614-649): P_m = sum over charged n != m of 0.5 / sqrt(r^2 + h^2) (f32,
// truncated integer positions), and Pother += P_m, on interior points
__global__ void k_mj_init_pdirect(const MjAtom* __restrict__ atoms, int nAt, int m, float* __restrict__ Pm,
                                  float* __restrict__ Pother, Geo g, float h, float h2) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, k;
  if (id >= g.S3 || !interior_of(id, g, i, j, k)) return;
  const float xi = F_MUL((float)i, h), yj = F_MUL((float)j, h), zk = F_MUL((float)k, h);
  float val = 0.0f;
  for (int n = 0; n < nAt; ++n) {
    const MjAtom a = atoms[n];
    if (a.Z <= 0.0f || n == m) continue;
    const float dx = F_SUB(xi, F_MUL((float)a.posI, h));
    const float dy = F_SUB(yj, F_MUL((float)a.posJ, h));
    const float dz = F_SUB(zk, F_MUL((float)a.posK, h));
    const float r = F_SQRT(F_ADD(F_ADD(F_ADD(F_MUL(dx, dx), F_MUL(dy, dy)), F_MUL(dz, dz)), h2));
    val = F_ADD(val, F_DIV(0.5f, r));
  }
  Pm[id] = val;
  Pother[id] = F_ADD(Pother[id], val);
}

__global__ void k_mj_residual(const float* __restrict__ Pin, float* __restrict__ R, const float* __restrict__ rho, Geo g,
                              float inv_h2, float two_pi) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, k;
  if (id >= g.S3 || !interior_of(id, g, i, j, k)) return;
  const long long S = g.S, S2 = g.S2;
  const float Pc = Pin[id];
  const float sum = F_ADD(F_ADD(F_ADD(F_ADD(F_ADD(Pin[id + S2], Pin[id - S2]), Pin[id + S]), Pin[id - S]), Pin[id + 1]),
                          Pin[id - 1]);
  const float lap = F_MUL(F_SUB(sum, F_MUL(6.0f, Pc)), inv_h2);
  R[id] = F_SUB(F_MUL(-two_pi, rho[id]), lap);
}

__global__ void k_mj_restrict(const float* __restrict__ fine, float* __restrict__ coarse, Geo g, Geo gc) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int NCM = gc.NN - 1;
  if (q >= (long long)NCM * NCM * NCM) return;
  const int K2 = (int)(q % NCM) + 1, J = (int)((q / NCM) % NCM) + 1, I = (int)(q / ((long long)NCM * NCM)) + 1;
  const int fi = 2 * I, fj = 2 * J, fk = 2 * K2;
  const long long S = g.S, S2 = g.S2;
#define FN(a, b, c) fine[(long long)(a) * S2 + (long long)(b) * S + (c)]
  float val = F_MUL(8.0f, FN(fi, fj, fk));
  float s4 = F_ADD(F_ADD(F_ADD(F_ADD(F_ADD(FN(fi + 1, fj, fk), FN(fi - 1, fj, fk)), FN(fi, fj + 1, fk)), FN(fi, fj - 1, fk)),
                         FN(fi, fj, fk + 1)),
                   FN(fi, fj, fk - 1));
  val = F_ADD(val, F_MUL(4.0f, s4));
  float s2 = FN(fi + 1, fj + 1, fk);
  s2 = F_ADD(s2, FN(fi + 1, fj - 1, fk)); s2 = F_ADD(s2, FN(fi - 1, fj + 1, fk)); s2 = F_ADD(s2, FN(fi - 1, fj - 1, fk));
  s2 = F_ADD(s2, FN(fi + 1, fj, fk + 1)); s2 = F_ADD(s2, FN(fi + 1, fj, fk - 1)); s2 = F_ADD(s2, FN(fi - 1, fj, fk + 1));
  s2 = F_ADD(s2, FN(fi - 1, fj, fk - 1)); s2 = F_ADD(s2, FN(fi, fj + 1, fk + 1)); s2 = F_ADD(s2, FN(fi, fj + 1, fk - 1));
  s2 = F_ADD(s2, FN(fi, fj - 1, fk + 1)); s2 = F_ADD(s2, FN(fi, fj - 1, fk - 1));
  val = F_ADD(val, F_MUL(2.0f, s2));
  float s1 = FN(fi + 1, fj + 1, fk + 1);
  s1 = F_ADD(s1, FN(fi + 1, fj + 1, fk - 1)); s1 = F_ADD(s1, FN(fi + 1, fj - 1, fk + 1)); s1 = F_ADD(s1, FN(fi + 1, fj - 1, fk - 1));
  s1 = F_ADD(s1, FN(fi - 1, fj + 1, fk + 1)); s1 = F_ADD(s1, FN(fi - 1, fj + 1, fk - 1)); s1 = F_ADD(s1, FN(fi - 1, fj - 1, fk + 1));
  s1 = F_ADD(s1, FN(fi - 1, fj - 1, fk - 1));
  val = F_ADD(val, s1);
#undef FN
  coarse[(long long)I * gc.S2 + (long long)J * gc.S + K2] = F_MUL(val, 0.015625f);
}

__global__ void k_mj_coarse_smooth(const float* __restrict__ Ein, float* __restrict__ Eout, const float* __restrict__ f,
                                   Geo gc, float h2) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int NCM = gc.NN - 1;
  if (q >= (long long)NCM * NCM * NCM) return;
  const int K2 = (int)(q % NCM) + 1, J = (int)((q / NCM) % NCM) + 1, I = (int)(q / ((long long)NCM * NCM)) + 1;
  const long long c = (long long)I * gc.S2 + (long long)J * gc.S + K2, SC = gc.S, SC2 = gc.S2;
  const float ec = Ein[c];
  const float sn = F_ADD(F_ADD(F_ADD(F_ADD(F_ADD(Ein[c + SC2], Ein[c - SC2]), Ein[c + SC]), Ein[c - SC]), Ein[c + 1]),
                         Ein[c - 1]);
  const float hc2 = F_MUL(4.0f, h2);
  Eout[c] = F_ADD(F_MUL(0.3333f, ec), F_DIV(F_ADD(sn, F_MUL(hc2, f[c])), 9.0f));
}

__global__ void k_mj_prolong(const float* __restrict__ Ec, float* __restrict__ Pf, Geo g, Geo gc) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, k;
  if (id >= g.S3 || !interior_of(id, g, i, j, k)) return;
  const int NC = gc.NN;
  const int ci = i / 2, cj = j / 2, ck = k / 2;
  const int ci1 = min(ci + (i & 1), NC), cj1 = min(cj + (j & 1), NC), ck1 = min(ck + (k & 1), NC);
  const float wi = (i & 1) ? 0.5f : 1.0f, wj = (j & 1) ? 0.5f : 1.0f, wk = (k & 1) ? 0.5f : 1.0f;
  const float wi1 = F_SUB(1.0f, wi), wj1 = F_SUB(1.0f, wj), wk1 = F_SUB(1.0f, wk);
  const long long SC = gc.S, SC2 = gc.S2;
#define EC(a, b, c) Ec[(long long)(a) * SC2 + (long long)(b) * SC + (c)]
  float corr = 0.0f;
  corr = F_ADD(corr, F_MUL(F_MUL(F_MUL(wi, wj), wk), EC(ci, cj, ck)));
  corr = F_ADD(corr, F_MUL(F_MUL(F_MUL(wi, wj), wk1), EC(ci, cj, ck1)));
  corr = F_ADD(corr, F_MUL(F_MUL(F_MUL(wi, wj1), wk), EC(ci, cj1, ck)));
  corr = F_ADD(corr, F_MUL(F_MUL(F_MUL(wi, wj1), wk1), EC(ci, cj1, ck1)));
  corr = F_ADD(corr, F_MUL(F_MUL(F_MUL(wi1, wj), wk), EC(ci1, cj, ck)));
  corr = F_ADD(corr, F_MUL(F_MUL(F_MUL(wi1, wj), wk1), EC(ci1, cj, ck1)));
  corr = F_ADD(corr, F_MUL(F_MUL(F_MUL(wi1, wj1), wk), EC(ci1, cj1, ck)));
  corr = F_ADD(corr, F_MUL(F_MUL(F_MUL(wi1, wj1), wk1), EC(ci1, cj1, ck1)));
#undef EC
  Pf[id] = F_ADD(Pf[id], F_MUL(0.5f, corr));
}

// ---------------------------------------------------------------------------------------
// evolveBoundary (molecule.js:426-540 without shell splits): snapshot labels in, labels + W
// out; the new label word carries its recomputed exclusion bit.  Locked groups (USER_LOCKED_GROUPS,
// :490-503, compiled into the page's shader): lock[l] has bit g set when label l is in group g; a
// boundary cell whose label and best other label share a group keeps its label, W = max(W, 0.5).
// ---------------------------------------------------------------------------------------
// One plane per block: a cell's pass reuses nothing from the plane before it, and the page runs
// the pass W_STEPS_PER_FRAME times a frame on grids from 32^3 up, where a 16-plane march leaves
// most SMs idle.
constexpr int kEvolveMarch = 1;

__global__ void __launch_bounds__(256) k_mj_evolve(const int* __restrict__ labIn, int* __restrict__ labOut,
                                                   const float* __restrict__ U, float* __restrict__ W,
                                                   const MjAtom* __restrict__ atoms, int nAt, Geo g, float dt_w,
                                                   float curvReg, float h, bool hasBare,
                                                   const unsigned long long* __restrict__ lock,
                                                   const MjSplit* __restrict__ splits) {
  const int k = 1 + blockIdx.x * kThreadsK + threadIdx.x;
  const int j = 1 + blockIdx.y * kThreadsJ + threadIdx.y;
  const int i0 = 1 + blockIdx.z * kEvolveMarch;
  if (k >= g.NN || j >= g.NN || i0 >= g.NN) return;
  const int iend = min(i0 + kEvolveMarch, g.NN);
  const long long S = g.S, S2 = g.S2;
  for (int i = i0; i < iend; ++i) {
    const long long id = (long long)i * S2 + j * S + k;
    const int stored = __ldg(labIn + id);
    const int myL = stored & kMjMask;
    const float uc = __ldg(U + id);
    const float myRho = F_MUL(uc, uc);
    const long long nb[6] = {id + S2, id - S2, id + S, id - S, id + 1, id - 1};
    int bestL = myL;
    float bestRho = 0.f, myCnt = 0.f;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      const int l = __ldg(labIn + nb[q]) & kMjMask;
      if (l == myL) {
        myCnt = F_ADD(myCnt, 1.0f);
      } else {
        const float un = __ldg(U + nb[q]);
        const float r = F_MUL(un, un);
        if (r > bestRho) { bestRho = r; bestL = l; }
      }
    }
    float w = W[id];
    if (myCnt >= 6.0f) {
      W[id] = fmaxf(w, 1.0f);
      labOut[id] = stored;
      continue;
    }
    if ((__ldg(lock + myL) & __ldg(lock + bestL)) != 0ull) {
      W[id] = fmaxf(w, 0.5f);
      labOut[id] = stored;
      continue;
    }
    const float denom = F_ADD(myRho, bestRho);
    const float vel = (denom < 1e-20f) ? 0.0f : F_DIV(F_SUB(myRho, bestRho), denom);
    w = F_ADD(w, F_MUL(dt_w, vel));
    const float curv = F_DIV(F_SUB(myCnt, 3.0f), 3.0f);
    w = F_ADD(w, F_MUL(curvReg, curv));
    int newL = myL;
    if (w < 0.0f) { newL = bestL; w = 0.1f; }
    // shell splits (:514-533): a flip into a domain whose sector excludes the cell is cancelled; a
    // cell outside its own domain's sector goes to the best neighbour whose sector holds it
    const bool myOK = mj_sector_ok(i, j, k, myL, atoms, splits, h);
    if (!mj_sector_ok(i, j, k, newL, atoms, splits, h)) {
      newL = myL;
      w = fmaxf(w, 0.1f);
      if (!myOK && bestL != myL && mj_sector_ok(i, j, k, bestL, atoms, splits, h)) { newL = bestL; w = 0.1f; }
    } else if (!myOK && newL == myL) {
      if (bestL != myL && mj_sector_ok(i, j, k, bestL, atoms, splits, h)) { newL = bestL; w = 0.1f; }
    }
    W[id] = w;
    labOut[id] = (newL == myL) ? stored : mj_pack(i, j, k, newL, atoms, nAt, hasBare, h);
  }
}

// ---------------------------------------------------------------------------------------
// reduceEnergy terms (molecule.js:950-1075) in FP64: per label (norm, T, V_eK, V_ee) plus
// the three dipole sums; exclusion radius max(rc, R_SING) with real distances.
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_mj_energy(const float* __restrict__ U, const float* __restrict__ Pv,
                                                   const float* __restrict__ K, const int* __restrict__ label,
                                                   const MjAtom* __restrict__ atoms, Geo g, float h, float h3,
                                                   float Rsing, int nDom, double* __restrict__ pd,
                                                   double* __restrict__ dip) {
  __shared__ DomTable<4, 128> tab;
  __shared__ double sdip[3][8];
  dom_table_init(tab);
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  __syncthreads();
  RunSum<4> rs;
  rs.reset();
  double dx = 0, dy = 0, dz = 0;
  const int k = 1 + blockIdx.x * kThreadsK + threadIdx.x;
  const int j = 1 + blockIdx.y * kThreadsJ + threadIdx.y;
  const int i0 = 1 + blockIdx.z * kMarch;
  if (k < g.NN && j < g.NN && i0 < g.NN) {
    const int iend = min(i0 + kMarch, g.NN);
    const long long S = g.S, S2 = g.S2;
    for (int i = i0; i < iend; ++i) {
      const long long id = (long long)i * S2 + j * S + k;
      const float v = U[id];
      const float rho = F_MUL(v, v);
      const int L = label[id] & kMjMask;
      const MjAtom a = atoms[L];
      const float rcx = fmaxf(a.rc, Rsing);
      if (mj_dist(i, j, k, a, h) < rcx) continue;
      const bool sip = (label[id + S2] & kMjMask) == L && !(mj_dist(i + 1, j, k, a, h) < rcx);
      const bool sjp = (label[id + S] & kMjMask) == L && !(mj_dist(i, j + 1, k, a, h) < rcx);
      const bool skp = (label[id + 1] & kMjMask) == L && !(mj_dist(i, j, k + 1, a, h) < rcx);
      const double da = sip ? (double)F_SUB(U[id + S2], v) : 0.0;
      const double db = sjp ? (double)F_SUB(U[id + S], v) : 0.0;
      const double dc = skp ? (double)F_SUB(U[id + 1], v) : 0.0;
      const double r3 = (double)rho * (double)h3;
      double q[4] = {r3, 0.5 * (da * da + db * db + dc * dc) * (double)h, -(double)K[id] * r3, (double)Pv[id] * r3};
      rs.add(min(L, nDom - 1), q, tab, pd);
      dx += r3 * (double)F_MUL((float)i, h);
      dy += r3 * (double)F_MUL((float)j, h);
      dz += r3 * (double)F_MUL((float)k, h);
    }
  }
  rs.finish(tab, pd);
  // warp reduce the dipole partials
  for (int o = 16; o > 0; o >>= 1) {
    dx += __shfl_down_sync(0xffffffffu, dx, o);
    dy += __shfl_down_sync(0xffffffffu, dy, o);
    dz += __shfl_down_sync(0xffffffffu, dz, o);
  }
  if ((tid & 31) == 0) { sdip[0][tid >> 5] = dx; sdip[1][tid >> 5] = dy; sdip[2][tid >> 5] = dz; }
  __syncthreads();
  dom_table_flush(tab, pd);
  if (tid < 3) {
    double s = 0;
    for (int w = 0; w < (blockDim.x * blockDim.y) / 32; ++w) s += sdip[tid][w];
    atomicAdd(&dip[tid], s);
  }
}

// ---------------------------------------------------------------------------------------
// gradPtotal (molecule.js:1200-1269): F = 2 Z <grad P> over the integer ball of radius R
// around the (integer) nucleus; one block per atom, FP64 block reduction.
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_mj_gradp(const float* __restrict__ Pt, const MjAtom* __restrict__ atoms,
                                                  Geo g, float inv_h, int R, double* __restrict__ F) {
  __shared__ double red[4][8];
  const int atom = blockIdx.x;
  const MjAtom a = atoms[atom];
  const float ZA = (a.Z <= 0.f) ? a.Z_nuc : a.Z;
  const int tid = threadIdx.x;
  if (ZA <= 0.f) {
    if (tid < 3) F[atom * 3 + tid] = 0.0;
    return;
  }
  const int ci = (int)a.posI, cj = (int)a.posJ, ck = (int)a.posK;
  const int D = 2 * R + 1;
  const long long nball = (long long)D * D * D;
  const float inv2h = F_MUL(0.5f, inv_h);
  const long long S = g.S, S2 = g.S2;
  double sx = 0, sy = 0, sz = 0, cnt = 0;
  for (long long q = tid; q < nball; q += blockDim.x) {
    const int di = (int)(q / ((long long)D * D)) - R, dj = (int)((q / D) % D) - R, dk = (int)(q % D) - R;
    const int ii = ci + di, jj = cj + dj, kk = ck + dk;
    if (ii < 1 || ii >= g.S - 1 || jj < 1 || jj >= g.S - 1 || kk < 1 || kk >= g.S - 1) continue;
    if (di * di + dj * dj + dk * dk > R * R) continue;
    const long long id = (long long)ii * S2 + (long long)jj * S + kk;
    sx += (double)F_MUL(F_SUB(Pt[id + S2], Pt[id - S2]), inv2h);
    sy += (double)F_MUL(F_SUB(Pt[id + S], Pt[id - S]), inv2h);
    sz += (double)F_MUL(F_SUB(Pt[id + 1], Pt[id - 1]), inv2h);
    cnt += 1.0;
  }
  for (int o = 16; o > 0; o >>= 1) {
    sx += __shfl_down_sync(0xffffffffu, sx, o);
    sy += __shfl_down_sync(0xffffffffu, sy, o);
    sz += __shfl_down_sync(0xffffffffu, sz, o);
    cnt += __shfl_down_sync(0xffffffffu, cnt, o);
  }
  if ((tid & 31) == 0) { red[0][tid >> 5] = sx; red[1][tid >> 5] = sy; red[2][tid >> 5] = sz; red[3][tid >> 5] = cnt; }
  __syncthreads();
  if (tid == 0) {
    double t[4] = {0, 0, 0, 0};
    for (int w = 0; w < blockDim.x / 32; ++w)
      for (int c = 0; c < 4; ++c) t[c] += red[c][w];
    const double n = t[3] > 0 ? t[3] : 1.0;
    F[atom * 3 + 0] = 2.0 * (double)ZA * (t[0] / n);
    F[atom * 3 + 1] = 2.0 * (double)ZA * (t[1] / n);
    F[atom * 3 + 2] = 2.0 * (double)ZA * (t[2] / n);
  }
}

// ======================================================================================
// host launchers
// ======================================================================================
static unsigned flat_blocks(long long n) { return (unsigned)((n + 255) / 256); }

cudaError_t launch_mj_init(float* K, float* U, float* bestU, int* label, const MjAtom* atoms, int nAt, const Geo& g,
                           float h, float h2, float Rsing, bool hasBare, bool persist, const MjSplit* splits,
                           cudaStream_t st) {
  if (persist)
    k_mj_init<true><<<flat_blocks(g.S3), 256, 0, st>>>(K, U, bestU, label, atoms, nAt, g, h, h2, Rsing, hasBare, splits);
  else
    k_mj_init<false><<<flat_blocks(g.S3), 256, 0, st>>>(K, U, bestU, label, atoms, nAt, g, h, h2, Rsing, hasBare,
                                                         splits);
  return cudaGetLastError();
}
cudaError_t launch_mj_recompute_k(float* K, const MjAtom* atoms, int nAt, const Geo& g, float h, float Rsing,
                                  cudaStream_t st) {
  k_mj_recompute_k<<<flat_blocks(g.S3), 256, 0, st>>>(K, atoms, nAt, g, h, Rsing);
  return cudaGetLastError();
}
cudaError_t launch_mj_flags(int* label, const MjAtom* atoms, int nAt, const Geo& g, float h, bool hasBare,
                            cudaStream_t st) {
  k_mj_flags<<<flat_blocks(g.S3), 256, 0, st>>>(label, atoms, nAt, g, h, hasBare);
  return cudaGetLastError();
}
cudaError_t launch_mj_update(const float* U, float* Uo, const float* K, const int* label, const float* Pother,
                             const Geo& g, float half_d, float dt, float h3, int nDom, unsigned* unorm,
                             cudaStream_t st) {
  if (g.NN < 2) return cudaSuccess;
  if (unorm)
    k_mj_update<true><<<march_grid(g), march_block(), 0, st>>>(U, Uo, K, label, Pother, g, half_d, dt, h3, nDom, unorm);
  else
    k_mj_update<false><<<march_grid(g), march_block(), 0, st>>>(U, Uo, K, label, Pother, g, half_d, dt, h3, nDom,
                                                                 nullptr);
  return cudaGetLastError();
}
cudaError_t launch_mj_update_cheb(const float* U, float* Uo, const float* K, const int* label, const float* Pother,
                                  const Geo& g, float half_d, float dt, float h3, int nDom, unsigned* unorm,
                                  float omega, cudaStream_t st) {
  if (g.NN < 2) return cudaSuccess;
  if (unorm)
    k_mj_update<true, true><<<march_grid(g), march_block(), 0, st>>>(U, Uo, K, label, Pother, g, half_d, dt, h3, nDom,
                                                                      unorm, omega);
  else
    k_mj_update<false, true><<<march_grid(g), march_block(), 0, st>>>(U, Uo, K, label, Pother, g, half_d, dt, h3, nDom,
                                                                       nullptr, omega);
  return cudaGetLastError();
}
cudaError_t launch_mj_norm_scale(const unsigned* unorm, const MjAtom* atoms, int nDom, float* scale, cudaStream_t st) {
  k_mj_norm_scale<<<(nDom + 127) / 128, 128, 0, st>>>(unorm, atoms, nDom, scale);
  return cudaGetLastError();
}
cudaError_t launch_mj_apply_scale(float* U, const int* label, const float* scale, const Geo& g, cudaStream_t st) {
  if (g.NN < 2) return cudaSuccess;
  k_mj_apply_scale<<<march_grid(g), march_block(), 0, st>>>(U, label, scale, g);
  return cudaGetLastError();
}
cudaError_t launch_mj_jacobi(const float* Pin, float* Pout, const float* U, const Geo& g, float h2, float two_pi,
                             cudaStream_t st) {
  if (g.NN < 2) return cudaSuccess;
  k_mj_jacobi<<<march_grid(g), march_block(), 0, st>>>(Pin, Pout, U, g, h2, two_pi);
  return cudaGetLastError();
}
// molecule.js:2879-2907 (and :3031-3061 for the self-potential): residual of P for the density
// rho, restrict, 10 coarse weighted-Jacobi sweeps from 0, prolongate with P += 0.5 * correction
static cudaError_t mj_vcycle_core(float* P, const float* rho, float* resid, float* Ec0, float* Ec1, float* fc,
                                  const Geo& g, const Geo& gc, float h2, float inv_h2, float two_pi, cudaStream_t st) {
  k_mj_residual<<<flat_blocks(g.S3), 256, 0, st>>>(P, resid, rho, g, inv_h2, two_pi);
  const long long nc = (long long)(gc.NN - 1) * (gc.NN - 1) * (gc.NN - 1);
  k_mj_restrict<<<flat_blocks(nc), 256, 0, st>>>(resid, fc, g, gc);
  cudaError_t e = cudaMemsetAsync(Ec0, 0, sizeof(float) * gc.S3, st);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(Ec1, 0, sizeof(float) * gc.S3, st);
  if (e != cudaSuccess) return e;
  float* E[2] = {Ec0, Ec1};
  for (int cs = 0; cs < 10; ++cs) k_mj_coarse_smooth<<<flat_blocks(nc), 256, 0, st>>>(E[cs % 2], E[(cs + 1) % 2], fc, gc, h2);
  k_mj_prolong<<<flat_blocks(g.S3), 256, 0, st>>>(E[0], P, g, gc);
  return cudaGetLastError();
}

cudaError_t launch_mj_vcycle(float* P, const float* U, float* rho, float* resid, float* Ec0, float* Ec1, float* fc,
                             const Geo& g, const Geo& gc, float h2, float inv_h2, float two_pi, cudaStream_t st) {
  k_mj_rho<<<flat_blocks(g.S3), 256, 0, st>>>(U, rho, g);
  return mj_vcycle_core(P, rho, resid, Ec0, Ec1, fc, g, gc, h2, inv_h2, two_pi, st);
}

cudaError_t launch_mj_direct_init(const MjAtom* atoms, int nAt, int m, float* Pm, float* Pother, const Geo& g, float h,
                                  float h2, cudaStream_t st) {
  k_mj_init_pdirect<<<flat_blocks(g.S3), 256, 0, st>>>(atoms, nAt, m, Pm, Pother, g, h, h2);
  return cudaGetLastError();
}

cudaError_t launch_mj_direct_domain(const float* U, const int* label, float* Pother, int m, float* Pm, float* scratch,
                                    float* rho, const Geo& g, float h2, float two_pi, cudaStream_t st) {
  // molecule.js:2835-2857 for one domain: the density of every other domain, 10 Jacobi sweeps of
  // the persistent P_m (P_m <-> scratch, ending in P_m), then Pother = P_m on the domain
  if (g.NN < 2) return cudaSuccess;
  k_mj_rho_other<<<flat_blocks(g.S3), 256, 0, st>>>(U, label, m, rho, g);
  for (int js = 0; js < 10; ++js)
    k_mj_jacobi_rho<<<march_grid(g), march_block(), 0, st>>>(js % 2 ? scratch : Pm, js % 2 ? Pm : scratch, rho, g, h2,
                                                             two_pi);
  k_mj_copy_for_label<<<flat_blocks(g.S3), 256, 0, st>>>(Pm, Pother, label, m, g);
  return cudaGetLastError();
}

cudaError_t launch_mj_sic_domain(const float* U, const int* label, float* Pother, int m, float frac, float* rho,
                                 float* sic, float* sic2, float* resid, float* Ec0, float* Ec1, float* fc, const Geo& g,
                                 const Geo& gc, float h2, float inv_h2, float two_pi, cudaStream_t st) {
  // molecule.js:3018-3075 for one domain: its density, 4 Jacobi sweeps from 0 (sic <-> sic2),
  // the coarse correction, 4 more sweeps, then Pother -= P_m / Z_m on the domain
  if (g.NN < 2) return cudaSuccess;
  k_mj_rho_self<<<flat_blocks(g.S3), 256, 0, st>>>(U, label, m, rho, g);
  cudaError_t e = cudaMemsetAsync(sic, 0, sizeof(float) * g.S3, st);
  if (e != cudaSuccess) return e;
  for (int js = 0; js < 4; ++js)
    k_mj_jacobi_rho<<<march_grid(g), march_block(), 0, st>>>(js % 2 ? sic2 : sic, js % 2 ? sic : sic2, rho, g, h2,
                                                             two_pi);
  if ((e = mj_vcycle_core(sic, rho, resid, Ec0, Ec1, fc, g, gc, h2, inv_h2, two_pi, st)) != cudaSuccess) return e;
  for (int js = 0; js < 4; ++js)
    k_mj_jacobi_rho<<<march_grid(g), march_block(), 0, st>>>(js % 2 ? sic2 : sic, js % 2 ? sic : sic2, rho, g, h2,
                                                             two_pi);
  k_mj_sub_self<<<flat_blocks(g.S3), 256, 0, st>>>(sic, Pother, label, m, frac, g);
  return cudaGetLastError();
}
cudaError_t launch_mj_evolve(const int* labIn, int* labOut, const float* U, float* W, const MjAtom* atoms, int nAt,
                             const Geo& g, float dt_w, float curvReg, float h, bool hasBare,
                             const unsigned long long* lock, const MjSplit* splits, cudaStream_t st) {
  if (g.NN < 2) return cudaSuccess;
  k_mj_evolve<<<march_grid(g, kEvolveMarch), march_block(), 0, st>>>(labIn, labOut, U, W, atoms, nAt, g, dt_w, curvReg,
                                                                     h, hasBare,
                                                       lock, splits);
  return cudaGetLastError();
}
cudaError_t launch_mj_energy(const float* U, const float* Pv, const float* K, const int* label, const MjAtom* atoms,
                             const Geo& g, float h, float h3, float Rsing, int nDom, double* pd, double* dip,
                             cudaStream_t st) {
  if (g.NN < 2) return cudaSuccess;
  k_mj_energy<<<march_grid(g), march_block(), 0, st>>>(U, Pv, K, label, atoms, g, h, h3, Rsing, nDom, pd, dip);
  return cudaGetLastError();
}
cudaError_t launch_mj_gradp(const float* P, const MjAtom* atoms, int nAt, const Geo& g, float inv_h, int R, double* F,
                            cudaStream_t st) {
  k_mj_gradp<<<nAt, 256, 0, st>>>(P, atoms, g, inv_h, R, F);
  return cudaGetLastError();
}

}  // namespace rq

namespace rq {
__global__ void k_fill(float* __restrict__ f, float v, long long n) {
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    f[q] = v;
}
__global__ void k_unpack(const int* __restrict__ in, int* __restrict__ out, long long n) {
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    out[q] = in[q] & kMjMask;
}
cudaError_t launch_fill(float* f, float v, long long n, cudaStream_t st) {
  k_fill<<<148 * 8, 256, 0, st>>>(f, v, n);
  return cudaGetLastError();
}
cudaError_t launch_unpack_labels(const int* in, int* out, long long n, cudaStream_t st) {
  k_unpack<<<148 * 8, 256, 0, st>>>(in, out, n);
  return cudaGetLastError();
}
}  // namespace rq

namespace rq {

// extractWGSL (molecule.js:1108-1192) with W_CUTOFF = 0 (:84): out = u^2 on the slice k = sk,
// label + 1000 Z of the label, the boundary flags (1 a boundary with density on a side, 2 one
// without), then the K line and the w line along (i, sk, sk)
__global__ void __launch_bounds__(256) k_mj_extract(const float* __restrict__ U, const int* __restrict__ label,
                                                    const float* __restrict__ K, const MjAtom* __restrict__ atoms,
                                                    int nAt, Geo g, int sk, float* __restrict__ out) {
  const int i = blockIdx.x * 16 + threadIdx.x, j = blockIdx.y * 16 + threadIdx.y;
  const int NN = g.S - 1;
  const long long SS = g.S, S2 = g.S2;
  if (i > NN || j > NN) return;
  if (j == 0) {
    out[3 * SS * SS + i] = K[(long long)i * S2 + (long long)sk * SS + sk];
    out[3 * SS * SS + SS + i] = 1.0f;
  }
  if (i < 1 || i >= NN || j < 1 || j >= NN) {
    out[i * SS + j] = 0.0f;
    out[SS * SS + i * SS + j] = 0.0f;
    out[2 * SS * SS + i * SS + j] = 0.0f;
    return;
  }
  const long long idx = (long long)i * S2 + (long long)j * SS + sk;
  const float u = U[idx];
  const int lbl = label[idx] & kMjMask;  // the stored label carries the exclusion bit
  const float Zl = (lbl >= 0 && lbl < nAt) ? atoms[lbl].Z : 0.0f;
  const float dens = __fmul_rn(u, u);
  out[i * SS + j] = dens;
  out[SS * SS + i * SS + j] = __fadd_rn((float)(unsigned)lbl, __fmul_rn(Zl, 1000.0f));
  float bnd = 0.0f;
  if (i > 1 && i < NN - 1) {
    const long long nb = idx + S2;
    if (lbl != (label[nb] & kMjMask)) {
      const float nd = __fmul_rn(U[nb], U[nb]);
      bnd = (dens > 1e-6f || nd > 1e-6f) ? 1.0f : 2.0f;
    }
  }
  if (bnd < 1.5f && j > 1 && j < NN - 1) {
    const long long nb = idx + SS;
    if (lbl != (label[nb] & kMjMask)) {
      const float nd = __fmul_rn(U[nb], U[nb]);
      bnd = (dens > 1e-6f || nd > 1e-6f) ? fmaxf(bnd, 1.0f) : 2.0f;
    }
  }
  out[2 * SS * SS + i * SS + j] = bnd;
}

cudaError_t launch_mj_extract(const float* U, const int* label, const float* K, const MjAtom* atoms, int nAt,
                              const Geo& g, int sk, float* out, cudaStream_t st) {
  const unsigned b = (unsigned)((g.S + 15) / 16);
  k_mj_extract<<<dim3(b, b), dim3(16, 16), 0, st>>>(U, label, K, atoms, nAt, g, sk, out);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------
// LOBPCG frames (molecule.js:1455-1724 shaders, :3265-3740 host).  f32 shaders restated with
// the same operations in the same order; the inner products keep the shaders' workgroup trees;
// the Ritz problems -- double-precision JavaScript in the page, solved on the host between
// dispatches -- run in one device thread with explicitly rounded FP64 operations in the page's
// order, so the whole frame stays on the GPU (no read-back per iteration) and its results are
// those of the page's arithmetic.
// ---------------------------------------------------------------------------------------
#define D_ADD(a, b) __dadd_rn((a), (b))
#define D_SUB(a, b) __dsub_rn((a), (b))
#define D_MUL(a, b) __dmul_rn((a), (b))
#define D_DIV(a, b) __ddiv_rn((a), (b))
#define D_SQRT(a) __dsqrt_rn((a))

// applyH's own isInsideRc (molecule.js:1473-1477): only the label's own r_c sphere.
__device__ __forceinline__ bool lob_inside_rc(int ci, int cj, int ck, int lbl, const MjAtom* __restrict__ atoms,
                                              float h) {
  const MjAtom a = atoms[lbl];
  return a.rc > 0.f && mj_dist(ci, cj, ck, a, h) < a.rc;
}

// applyH (molecule.js:1483-1525): HU = -0.5*lap/h^2 + (-K + 2*Pother)*u, 0 inside the own r_c
// sphere, a neighbour of another label or inside its label's sphere replaced by the centre.
// Without bare nuclei the stored exclusion bit is exactly this test (packed words compare equal
// iff same label and the neighbour is not excluded); with them (BARE) the bit also marks the
// bare nuclei's spheres, which this shader ignores, so the spheres are tested directly.
template <bool BARE>
__global__ void __launch_bounds__(256) k_lob_apply_h(const float* __restrict__ U, float* __restrict__ HU,
                                                     const float* __restrict__ K, const int* __restrict__ label,
                                                     const float* __restrict__ Pother, const MjAtom* __restrict__ atoms,
                                                     Geo g, float h, float inv_h2) {
  // one interior cell per thread: the LOBPCG grids are small, and a march along i would leave
  // most SMs idle (64 blocks at 64^3)
  const int k = 1 + blockIdx.x * 32 + threadIdx.x, j = 1 + blockIdx.y * 8 + threadIdx.y, i = 1 + blockIdx.z;
  if (k >= g.NN || j >= g.NN) return;
  const long long S = g.S, S2 = g.S2;
  const long long id = (long long)i * S2 + j * S + k;
  const int l_c = __ldg(label + id), l_p = __ldg(label + id + S2), l_m = __ldg(label + id - S2);
  const int ljp = __ldg(label + id + S), ljm = __ldg(label + id - S), lkp = __ldg(label + id + 1),
            lkm = __ldg(label + id - 1);
  bool excl, up, um, ujp, ujm, ukp, ukm;  // excl: centre excluded; uX: neighbour X is used
  if (BARE) {
    const int L = l_c & kMjMask;
    excl = lob_inside_rc(i, j, k, L, atoms, h);
    up = (l_p & kMjMask) == L && !lob_inside_rc(i + 1, j, k, l_p & kMjMask, atoms, h);
    um = (l_m & kMjMask) == L && !lob_inside_rc(i - 1, j, k, l_m & kMjMask, atoms, h);
    ujp = (ljp & kMjMask) == L && !lob_inside_rc(i, j + 1, k, ljp & kMjMask, atoms, h);
    ujm = (ljm & kMjMask) == L && !lob_inside_rc(i, j - 1, k, ljm & kMjMask, atoms, h);
    ukp = (lkp & kMjMask) == L && !lob_inside_rc(i, j, k + 1, lkp & kMjMask, atoms, h);
    ukm = (lkm & kMjMask) == L && !lob_inside_rc(i, j, k - 1, lkm & kMjMask, atoms, h);
  } else {
    excl = (l_c & kMjExcl) != 0;
    up = l_p == l_c; um = l_m == l_c; ujp = ljp == l_c; ujm = ljm == l_c; ukp = lkp == l_c; ukm = lkm == l_c;
  }
  float out = 0.0f;
  if (!excl) {
    const float u_c = __ldg(U + id);
    const float a = up ? __ldg(U + id + S2) : u_c;
    const float b = um ? __ldg(U + id - S2) : u_c;
    const float c = ujp ? __ldg(U + id + S) : u_c;
    const float d = ujm ? __ldg(U + id - S) : u_c;
    const float e = ukp ? __ldg(U + id + 1) : u_c;
    const float f = ukm ? __ldg(U + id - 1) : u_c;
    const float lap = F_SUB(F_ADD(F_ADD(F_ADD(F_ADD(F_ADD(a, b), c), d), e), f), F_MUL(6.0f, u_c));
    out = F_ADD(F_MUL(F_MUL(-0.5f, lap), inv_h2), F_MUL(F_ADD(-__ldg(K + id), F_MUL(2.0f, __ldg(Pother + id))), u_c));
  }
  HU[id] = out;
}

// lobpcgInner (molecule.js:1535-1610): interior cells numbered with k fastest; block w thread l
// takes cells w*128+l, then every gridDim*128-th, summing a*b*h^3 for the 12 products over the
// cells of domain m; the block's 128 sums fold pairwise (l += l+s, s = 64 .. 1).
__global__ void __launch_bounds__(kLobWG) k_lob_inner(const float* __restrict__ X, const float* __restrict__ HX,
                                                      const float* __restrict__ W, const float* __restrict__ HW,
                                                      const float* __restrict__ Pv, const float* __restrict__ HP,
                                                      const int* __restrict__ label, int m, Geo g, float h3,
                                                      float* __restrict__ partials) {
  __shared__ float sn[kLobWG][kLobNR + 1];
  const int l = threadIdx.x;
  float acc[kLobNR];
#pragma unroll
  for (int q = 0; q < kLobNR; ++q) acc[q] = 0.0f;
  const unsigned NM = (unsigned)(g.NN - 1), tot = NM * NM * NM, stride = gridDim.x * kLobWG;
  for (unsigned cell = blockIdx.x * kLobWG + l; cell < tot; cell += stride) {
    const unsigned k = cell % NM + 1, j = (cell / NM) % NM + 1, i = cell / (NM * NM) + 1;
    const long long id = (long long)i * g.S2 + (long long)j * g.S + k;
    if ((__ldg(label + id) & kMjMask) != m) continue;
    const float x = __ldg(X + id), hx = __ldg(HX + id), w = __ldg(W + id), hw = __ldg(HW + id), pv = __ldg(Pv + id),
                hp = __ldg(HP + id);
    acc[0] = F_ADD(acc[0], F_MUL(F_MUL(x, x), h3));
    acc[1] = F_ADD(acc[1], F_MUL(F_MUL(x, hx), h3));
    acc[2] = F_ADD(acc[2], F_MUL(F_MUL(w, w), h3));
    acc[3] = F_ADD(acc[3], F_MUL(F_MUL(w, hw), h3));
    acc[4] = F_ADD(acc[4], F_MUL(F_MUL(x, w), h3));
    acc[5] = F_ADD(acc[5], F_MUL(F_MUL(x, hw), h3));
    acc[6] = F_ADD(acc[6], F_MUL(F_MUL(pv, pv), h3));
    acc[7] = F_ADD(acc[7], F_MUL(F_MUL(pv, hp), h3));
    acc[8] = F_ADD(acc[8], F_MUL(F_MUL(x, pv), h3));
    acc[9] = F_ADD(acc[9], F_MUL(F_MUL(x, hp), h3));
    acc[10] = F_ADD(acc[10], F_MUL(F_MUL(w, pv), h3));
    acc[11] = F_ADD(acc[11], F_MUL(F_MUL(w, hp), h3));
  }
#pragma unroll
  for (int q = 0; q < kLobNR; ++q) sn[l][q] = acc[q];
  __syncthreads();
  for (int s = kLobWG / 2; s > 0; s >>= 1) {
    if (l < s)
#pragma unroll
      for (int q = 0; q < kLobNR; ++q) sn[l][q] = F_ADD(sn[l][q], sn[l + s][q]);
    __syncthreads();
  }
  if (l == 0)
#pragma unroll
    for (int q = 0; q < kLobNR; ++q) partials[blockIdx.x * kLobNR + q] = sn[0][q];
}

// JavaScript Math.min / Math.max: NaN if either argument is NaN, -0 below +0.
__device__ __forceinline__ double js_min(double a, double b) {
  if (isnan(a) || isnan(b)) return __longlong_as_double(0x7ff8000000000000LL);
  if (a < b) return a;
  if (b < a) return b;
  return signbit(a) ? a : b;
}
__device__ __forceinline__ double js_max(double a, double b) {
  if (isnan(a) || isnan(b)) return __longlong_as_double(0x7ff8000000000000LL);
  if (a > b) return a;
  if (b > a) return b;
  return signbit(a) ? b : a;
}

// solveRitz2x2 (molecule.js:3265-3295) on ip = the 12 sums: the smaller root lambda of
// det(H - lambda S) = 0 over span{X, W} and its vector scaled to c'Sc = 1.  out = {lambda, c0..c2}.
__device__ void lob_ritz2(const double* ip, double* out) {
  const double a11 = ip[1], a12 = ip[5], a22 = ip[3], s11 = ip[0], s12 = ip[4], s22 = ip[2];
  const double A = D_SUB(D_MUL(s11, s22), D_MUL(s12, s12));
  const double B = -D_SUB(D_ADD(D_MUL(a11, s22), D_MUL(a22, s11)), D_MUL(D_MUL(2.0, a12), s12));
  const double Cq = D_SUB(D_MUL(a11, a22), D_MUL(a12, a12));
  const double disc = D_SUB(D_MUL(B, B), D_MUL(D_MUL(4.0, A), Cq));
  const double sq = D_SQRT(js_max(0.0, disc));
  const double lam1 = D_DIV(D_SUB(-B, sq), D_MUL(2.0, A));
  const double lam2 = D_DIV(D_ADD(-B, sq), D_MUL(2.0, A));
  const double lam = js_min(lam1, lam2);
  const double r1 = D_SUB(a11, D_MUL(lam, s11)), r2 = D_SUB(a12, D_MUL(lam, s12));
  double c0, c1;
  if (fabs(r1) > fabs(r2)) {
    c1 = 1.0;
    c0 = D_DIV(-r2, r1);
  } else if (fabs(r2) > 1e-15) {
    c0 = 1.0;
    c1 = D_DIV(-r1, r2);
  } else {
    c0 = 1.0;
    c1 = 0.0;
  }
  const double norm2 =
      D_ADD(D_ADD(D_MUL(D_MUL(c0, c0), s11), D_MUL(D_MUL(D_MUL(2.0, c0), c1), s12)), D_MUL(D_MUL(c1, c1), s22));
  const double inv = D_DIV(1.0, D_SQRT(js_max(1e-30, norm2)));
  out[0] = lam;
  out[1] = D_MUL(c0, inv);
  out[2] = D_MUL(c1, inv);
  out[3] = 0.0;
}

// solveRitz3x3 (molecule.js:3297-3388) over span{X, W, P}: Cholesky S = L L', the standard
// problem L^-1 H L^-T by 20 sweeps of cyclic Jacobi rotations, the smallest diagonal entry,
// c = L^-T y; the 2x2 problem when the factor is not finite or a diagonal is below 1e-15.
__device__ void lob_ritz3(const double* ip, double* out) {
  const double S[3][3] = {{ip[0], ip[4], ip[8]}, {ip[4], ip[2], ip[10]}, {ip[8], ip[10], ip[6]}};
  const double H[3][3] = {{ip[1], ip[5], ip[9]}, {ip[5], ip[3], ip[11]}, {ip[9], ip[11], ip[7]}};
  double L00 = D_SQRT(js_max(1e-30, S[0][0]));
  double L10 = D_DIV(S[1][0], L00), L20 = D_DIV(S[2][0], L00);
  double L11 = D_SQRT(js_max(1e-30, D_SUB(S[1][1], D_MUL(L10, L10))));
  double L21 = D_DIV(D_SUB(S[2][1], D_MUL(L20, L10)), L11);
  double L22 = D_SQRT(js_max(1e-30, D_SUB(D_SUB(S[2][2], D_MUL(L20, L20)), D_MUL(L21, L21))));
  if (!isfinite(L22) || L00 < 1e-15 || L11 < 1e-15 || L22 < 1e-15) {
    lob_ritz2(ip, out);
    return;
  }
  double Li[3][3] = {{D_DIV(1.0, L00), 0.0, 0.0}, {0.0, D_DIV(1.0, L11), 0.0}, {0.0, 0.0, D_DIV(1.0, L22)}};
  Li[1][0] = D_MUL(D_MUL(-L10, Li[0][0]), Li[1][1]);
  Li[2][0] = D_MUL(-D_ADD(D_MUL(L20, Li[0][0]), D_MUL(L21, Li[1][0])), Li[2][2]);
  Li[2][1] = D_MUL(D_MUL(-L21, Li[1][1]), Li[2][2]);
  double Bm[3][3], A[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s = D_ADD(s, D_MUL(H[i][k], Li[j][k]));
      Bm[i][j] = s;
    }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s = D_ADD(s, D_MUL(Li[i][k], Bm[k][j]));
      A[i][j] = s;
    }
  double V[3][3] = {{1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};
  for (int sweep = 0; sweep < 20; ++sweep)
    for (int e = 0; e < 3; ++e) {
      const int p = e == 2 ? 1 : 0, q = e == 0 ? 1 : 2;  // (0,1), (0,2), (1,2)
      const double apq = A[p][q];
      if (fabs(apq) < 1e-15) continue;
      const double tau = D_DIV(D_SUB(A[q][q], A[p][p]), D_MUL(2.0, apq));
      const double t = D_DIV(tau >= 0 ? 1.0 : -1.0, D_ADD(fabs(tau), D_SQRT(D_ADD(1.0, D_MUL(tau, tau)))));
      const double c = D_DIV(1.0, D_SQRT(D_ADD(1.0, D_MUL(t, t))));
      const double s = D_MUL(t, c);
      const double app = A[p][p], aqq = A[q][q];
      A[p][p] = D_ADD(D_SUB(D_MUL(D_MUL(c, c), app), D_MUL(D_MUL(D_MUL(2.0, s), c), apq)), D_MUL(D_MUL(s, s), aqq));
      A[q][q] = D_ADD(D_ADD(D_MUL(D_MUL(s, s), app), D_MUL(D_MUL(D_MUL(2.0, s), c), apq)), D_MUL(D_MUL(c, c), aqq));
      A[p][q] = 0.0;
      A[q][p] = 0.0;
      for (int r = 0; r < 3; ++r) {
        if (r == p || r == q) continue;
        const double arp = A[r][p], arq = A[r][q];
        A[r][p] = D_SUB(D_MUL(c, arp), D_MUL(s, arq));
        A[p][r] = A[r][p];
        A[r][q] = D_ADD(D_MUL(s, arp), D_MUL(c, arq));
        A[q][r] = A[r][q];
      }
      for (int r = 0; r < 3; ++r) {
        const double vrp = V[r][p], vrq = V[r][q];
        V[r][p] = D_SUB(D_MUL(c, vrp), D_MUL(s, vrq));
        V[r][q] = D_ADD(D_MUL(s, vrp), D_MUL(c, vrq));
      }
    }
  int mi = 0;
  if (A[1][1] < A[mi][mi]) mi = 1;
  if (A[2][2] < A[mi][mi]) mi = 2;
  const double y0 = V[0][mi], y1 = V[1][mi], y2 = V[2][mi];
  out[0] = A[mi][mi];
  out[1] = D_ADD(D_ADD(D_MUL(Li[0][0], y0), D_MUL(Li[1][0], y1)), D_MUL(Li[2][0], y2));
  out[2] = D_ADD(D_MUL(Li[1][1], y1), D_MUL(Li[2][1], y2));
  out[3] = D_MUL(Li[2][2], y2);
}

// lobpcgFinalize (molecule.js:1612-1648) -- thread l adds block results l, l+128, .. in order, the
// same pairwise fold -- and then, in thread 0, the page's host step on the 12 sums:
//   FIRST pass: lambda = <X|HX> / <X|X> in double, stored as f32 (0 when <X|X> <= 0, :3486);
//   second pass: the Ritz problem (3x3 when hasP and <P|P> > 1e-20, else 2x2, :3570-3576), its
//   coefficients stored as f32 (:3581).
// scal: [0] lambda, [1..3] coefficients, [4..15] second-pass sums, [16..27] first-pass sums,
// [28] the Ritz value (f32).
template <bool FIRST>
__global__ void __launch_bounds__(kLobWG) k_lob_finalize(const float* __restrict__ partials, int nwg, int hasP,
                                                         float* __restrict__ scal) {
  __shared__ float wg[kLobWG][kLobNR + 1];
  const int l = threadIdx.x;
  float acc[kLobNR];
#pragma unroll
  for (int q = 0; q < kLobNR; ++q) acc[q] = 0.0f;
  for (int w = l; w < nwg; w += kLobWG)
#pragma unroll
    for (int q = 0; q < kLobNR; ++q) acc[q] = F_ADD(acc[q], partials[w * kLobNR + q]);
#pragma unroll
  for (int q = 0; q < kLobNR; ++q) wg[l][q] = acc[q];
  __syncthreads();
  for (int s = kLobWG / 2; s > 0; s >>= 1) {
    if (l < s)
#pragma unroll
      for (int q = 0; q < kLobNR; ++q) wg[l][q] = F_ADD(wg[l][q], wg[l + s][q]);
    __syncthreads();
  }
  if (l != 0) return;
  double ip[kLobNR];
  for (int q = 0; q < kLobNR; ++q) {
    ip[q] = (double)wg[0][q];
    scal[(FIRST ? 16 : 4) + q] = wg[0][q];
  }
  if (FIRST) {
    scal[0] = ip[0] > 0.0 ? __double2float_rn(D_DIV(ip[1], ip[0])) : 0.0f;
  } else {
    double r[4];
    if (hasP && ip[6] > 1e-20)
      lob_ritz3(ip, r);
    else
      lob_ritz2(ip, r);
    scal[1] = __double2float_rn(r[1]);
    scal[2] = __double2float_rn(r[2]);
    scal[3] = __double2float_rn(r[3]);
    scal[28] = __double2float_rn(r[0]);
  }
}

// lobpcgResidual (molecule.js:1652-1689): on domain m W = (HX - lambda*X) / (3/h^2 + |-K + 2*Pother|
// + 0.1), 0 on every other interior cell; lambda read from the device.
__global__ void __launch_bounds__(256) k_lob_residual(const float* __restrict__ X, const float* __restrict__ HX,
                                                      float* __restrict__ W, const int* __restrict__ label,
                                                      const float* __restrict__ K, const float* __restrict__ Pot,
                                                      const float* __restrict__ lam, int m, Geo g, float inv_h2) {
  const int k = 1 + blockIdx.x * 32 + threadIdx.x, j = 1 + blockIdx.y * 8 + threadIdx.y, i = 1 + blockIdx.z;
  if (k >= g.NN || j >= g.NN) return;
  const long long id = (long long)i * g.S2 + (long long)j * g.S + k;
  if ((__ldg(label + id) & kMjMask) != m) {
    W[id] = 0.0f;
    return;
  }
  const float r = F_SUB(__ldg(HX + id), F_MUL(*lam, __ldg(X + id)));
  const float vEff = fabsf(F_ADD(-__ldg(K + id), F_MUL(2.0f, __ldg(Pot + id))));
  const float diagH = F_ADD(F_ADD(F_MUL(3.0f, inv_h2), vEff), 0.1f);
  W[id] = F_DIV(r, diagH);
}

// lobpcgUpdate (molecule.js:1693-1724): on domain m X = c0*X + c1*W + c2*P, P = c1*W + c2*P.
__global__ void __launch_bounds__(256) k_lob_update(float* __restrict__ X, const float* __restrict__ W,
                                                    float* __restrict__ Pv, const int* __restrict__ label,
                                                    const float* __restrict__ coef, int m, Geo g) {
  const int k = 1 + blockIdx.x * 32 + threadIdx.x, j = 1 + blockIdx.y * 8 + threadIdx.y, i = 1 + blockIdx.z;
  if (k >= g.NN || j >= g.NN) return;
  const long long id = (long long)i * g.S2 + (long long)j * g.S + k;
  if ((__ldg(label + id) & kMjMask) != m) return;
  const float c0 = coef[0], c1 = coef[1], c2 = coef[2];
  const float x = X[id], w = __ldg(W + id), pv = Pv[id];
  X[id] = F_ADD(F_ADD(F_MUL(c0, x), F_MUL(c1, w)), F_MUL(c2, pv));
  Pv[id] = F_ADD(F_MUL(c1, w), F_MUL(c2, pv));
}

// accumNorms (molecule.js:911-930) as its own pass: norm[label] += u32(u*u*h3*2^24) over the
// interior; a warp's lanes with equal labels add their integers first (exact, modulo 2^32 like
// the shader's atomics), one atomic per label and warp.
__global__ void __launch_bounds__(256) k_mj_accum_norms(const float* __restrict__ U, const int* __restrict__ label,
                                                        Geo g, float h3, unsigned* __restrict__ unorm) {
  const int k = 1 + blockIdx.x * 32 + threadIdx.x, j = 1 + blockIdx.y * 8 + threadIdx.y, i = 1 + blockIdx.z;
  int L = -1;
  unsigned v = 0u;
  if (k < g.NN && j < g.NN) {
    const long long id = (long long)i * g.S2 + (long long)j * g.S + k;
    const float u = __ldg(U + id);
    v = __float2uint_rz(F_MUL(F_MUL(F_MUL(u, u), h3), 16777216.0f));
    L = __ldg(label + id) & kMjMask;
  }
  const unsigned peers = __match_any_sync(0xffffffffu, L);
  const unsigned sum = __reduce_add_sync(peers, v);
  if (L >= 0 && (int)threadIdx.x == __ffs(peers) - 1) atomicAdd(&unorm[L], sum);
}

// Copy the six faces (any index 0 or NN) of one label buffer into another: the level-set pass
// writes interior cells only, and in the page its output buffer (label2Buf, molecule.js:3103)
// keeps the face labels of the last full copy (uploadInitialData, :2090).
__global__ void k_copy_faces(const int* __restrict__ src, int* __restrict__ dst, Geo g) {
  const long long n = g.S2;
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 6 * n) return;
  const int face = (int)(q / n);
  const long long r = q % n;
  const int a = (int)(r / g.S), b = (int)(r % g.S);
  int i, j, k;
  switch (face) {
    case 0: i = 0; j = a; k = b; break;
    case 1: i = g.NN; j = a; k = b; break;
    case 2: i = a; j = 0; k = b; break;
    case 3: i = a; j = g.NN; k = b; break;
    case 4: i = a; j = b; k = 0; break;
    default: i = a; j = b; k = g.NN; break;
  }
  const long long id = (long long)i * g.S2 + (long long)j * g.S + k;
  dst[id] = src[id];
}

cudaError_t launch_copy_faces(const int* src, int* dst, const Geo& g, cudaStream_t st) {
  const long long n = 6 * g.S2;
  k_copy_faces<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(src, dst, g);
  return cudaGetLastError();
}

static dim3 lob_cells_grid(const Geo& g) {
  const unsigned n = (unsigned)(g.NN - 1);
  return dim3((n + 31) / 32, (n + 7) / 8, n);
}

int lob_workgroups(const Geo& g) {
  const long long n = g.NN - 1, tot = n * n * n;
  return (int)std::min<long long>(kLobMaxWG, (tot + kLobWG - 1) / kLobWG);
}

cudaError_t launch_lob_apply_h(const float* U, float* HU, const float* K, const int* label, const float* Pother,
                               const MjAtom* atoms, const Geo& g, float h, float inv_h2, bool bare, cudaStream_t st) {
  if (bare)
    k_lob_apply_h<true><<<lob_cells_grid(g), dim3(32, 8), 0, st>>>(U, HU, K, label, Pother, atoms, g, h, inv_h2);
  else
    k_lob_apply_h<false><<<lob_cells_grid(g), dim3(32, 8), 0, st>>>(U, HU, K, label, Pother, atoms, g, h, inv_h2);
  return cudaGetLastError();
}

cudaError_t launch_lob_inner(const float* X, const float* HX, const float* W, const float* HW, const float* Pv,
                             const float* HP, const int* label, int m, const Geo& g, float h3, float* partials,
                             cudaStream_t st) {
  k_lob_inner<<<lob_workgroups(g), kLobWG, 0, st>>>(X, HX, W, HW, Pv, HP, label, m, g, h3, partials);
  return cudaGetLastError();
}

cudaError_t launch_lob_finalize(const float* partials, int nwg, bool first, bool hasP, float* scal, cudaStream_t st) {
  if (first)
    k_lob_finalize<true><<<1, kLobWG, 0, st>>>(partials, nwg, hasP ? 1 : 0, scal);
  else
    k_lob_finalize<false><<<1, kLobWG, 0, st>>>(partials, nwg, hasP ? 1 : 0, scal);
  return cudaGetLastError();
}

cudaError_t launch_lob_residual(const float* X, const float* HX, float* W, const int* label, const float* K,
                                const float* Pot, const float* lam, int m, const Geo& g, float inv_h2, cudaStream_t st) {
  k_lob_residual<<<lob_cells_grid(g), dim3(32, 8), 0, st>>>(X, HX, W, label, K, Pot, lam, m, g, inv_h2);
  return cudaGetLastError();
}

cudaError_t launch_lob_update(float* X, const float* W, float* Pv, const int* label, const float* coef, int m,
                              const Geo& g, cudaStream_t st) {
  k_lob_update<<<lob_cells_grid(g), dim3(32, 8), 0, st>>>(X, W, Pv, label, coef, m, g);
  return cudaGetLastError();
}

cudaError_t launch_mj_accum_norms(const float* U, const int* label, const Geo& g, float h3, unsigned* unorm,
                                  cudaStream_t st) {
  k_mj_accum_norms<<<lob_cells_grid(g), dim3(32, 8), 0, st>>>(U, label, g, h3, unorm);
  return cudaGetLastError();
}

}  // namespace rq
