// nm_bodies.cuh -- device bodies of the new flavour's kernels.
//
// Each body takes its block coordinates explicitly, so the same code runs in two shapes:
// one grid per instance (nm_kernels.cu: the coordinates are blockIdx) and one launch over the
// (instance, tile) work list of a batch of uneven grids (batch_kernels.cu: the coordinates come
// from the work item).  Templated on the field type T (float: mixed path, double: FP64 path);
// point-wise arithmetic is explicitly rounded in the FP64 oracle's operation order
// (oracle/rq_oracle.c, orc_nm_*).
#pragma once
#include "rq_internal.cuh"

namespace rq {

template <typename T> struct Ar;
template <> struct Ar<float> {
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
};
template <> struct Ar<double> {
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
};

constexpr int kNmFlatChunk = 16;     // points per thread of the flat (all S^3) bodies
constexpr int kNmForceTile = 512;    // interior points staged per force tile
constexpr int kNmRowPlanes = 4;      // planes i per block of the row-tiled multigrid bodies
constexpr int kNmRowTJ = 8;           // rows j per block of the row-tiled bodies (block 32 x 8)
// Thread coordinates of a body written for a block of W threads along x, from the linear thread
// index: the body runs the same under a 2-D launch of that shape and under a 1-D launch of the
// same thread count (the persistent batch kernel).
template <int W>
__device__ __forceinline__ int tile_x() { return (int)((threadIdx.x + blockDim.x * threadIdx.y) % W); }
template <int W>
__device__ __forceinline__ int tile_y() { return (int)((threadIdx.x + blockDim.x * threadIdx.y) / W); }
// March tile of the new flavour's stencil bodies (update, readout, level set): 2^lgk points along
// k x 256 / 2^lgk rows j per block of 256 threads, each thread walking `march` planes of i.  The
// single-grid kernels use kNmTile (16 x 16 x 16: 16 wide rows waste fewer lanes than 32 on the
// 47..127-point interiors of the cluster grids); a batch uses the tile its autotuner picked.
struct NmTile {
  int lgk, march;
};
constexpr int kNmTK = 16, kNmTJ = 16;
constexpr NmTile kNmTile{4, kMarch};
inline dim3 nm_march_grid(const Geo& g, NmTile t = kNmTile) {
  const int n = g.NN - 1, tk = 1 << t.lgk, tj = 256 >> t.lgk;
  return dim3((n + tk - 1) / tk, (n + tj - 1) / tj, (n + t.march - 1) / t.march);
}
inline dim3 nm_march_block() { return dim3(kNmTK, kNmTJ, 1); }
// a thread's column (k, j) and first plane i0 in march tile (bx, by, bz)
__device__ __forceinline__ void nm_tile_origin(const NmTile& t, int bx, int by, int bz, int& k, int& j, int& i0) {
  const int lin = (int)(threadIdx.x + blockDim.x * threadIdx.y);
  k = 1 + (bx << t.lgk) + (lin & ((1 << t.lgk) - 1));
  j = 1 + by * (256 >> t.lgk) + (lin >> t.lgk);
  i0 = 1 + bz * t.march;
}
constexpr int kCoarsestThreads = 256; // one block solves the coarsest level (<= 29^3 points)

// FP64 1/sqrt(x) for x in the normal FP32 range: the FP32 hardware estimate y0 (relative error
// e0 below 2^-21) refined by the binomial series (1 - e)^(-1/2) = 1 + e/2 + 3e^2/8 + O(e^3),
// e = 1 - x y0^2 (Householder's third-order step for the reciprocal square root).  The truncation
// is 5e^3/16 < 1e-18 relative, below FP64 rounding; the FP64 work is five FMA-pipe operations
// where the FP64 reciprocal square root costs a slow-pipe estimate and Newton steps.
__device__ __forceinline__ double rsqrt_refined(double x) {
  const double y0 = (double)rsqrtf((float)x);
  const double e = fma(-x * y0, y0, 1.0);
  return fma(y0 * e, fma(0.375, e, 0.5), y0);
}

// The scale that brings a domain of norm n to its charge Z (1 for an empty or non-finite domain;
// a non-finite norm also sets bit 0 of *err).
__device__ __forceinline__ double nm_domain_scale(double n, double Z, int* err) {
  if (!isfinite(n)) {
    atomicOr(err, 1);
    return 1.0;
  }
  return (Z > 0.0 && n > 1e-300) ? sqrt(Z / n) : 1.0;
}

// Squared distance from which erf(r / (sqrt2 sigma)) is 1 to double precision (r / (sqrt2
// sigma) >= 6: erfc(6) = 2e-17): beyond it a Gaussian nucleus is a point charge.
__device__ __forceinline__ double nm_point_r2(double sigma) { return 72.0 * sigma * sigma; }

// ---------------------------------------------------------------------------------------
// K = sum Z erf(r/(sqrt2 sigma))/r in FP64 (K(0) = Z sqrt(2/pi)/sigma); boundary planes 0.
// One block of 256 threads covers points [blk*256, blk*256+256); sa: 512 doubles of smem.
// K64 (optional): the same sums kept in FP64 (the fp32 fields' readout copy), from the same
// pass.
// ---------------------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void nm_potential_body(T* __restrict__ K, const double* __restrict__ at, int nAt,
                                                  const Geo& g, double h, double sigma, long long blk, double* sa,
                                                  double* __restrict__ K64 = nullptr) {
  const long long id = blk * blockDim.x + threadIdx.x;
  const bool inside = id < g.S3;
  int i = 0, j = 0, k = 0;
  if (inside) { i = (int)(id / g.S2); j = (int)((id / g.S) % g.S); k = (int)(id % g.S); }
  const bool interior = inside && i >= 1 && i < g.NN && j >= 1 && j < g.NN && k >= 1 && k < g.NN;
  const double x = i * h, y = j * h, z = k * h;
  const double inv = 1.0 / (1.4142135623730951 * sigma), c0 = 0.7978845608028654 / sigma;  // sqrt(2/pi)
  const double rp2 = nm_point_r2(sigma);
  double v = 0.0;
  for (int base = 0; base < nAt; base += 128) {
    const int cnt = min(128, nAt - base);
    __syncthreads();
    for (int q = threadIdx.x; q < cnt * 4; q += blockDim.x) sa[q] = at[base * 4 + q];
    __syncthreads();
    if (!interior) continue;
    for (int m = 0; m < cnt; ++m) {
      const double Z = sa[m * 4 + 3];
      if (Z <= 0.0) continue;
      const double dx = x - sa[m * 4 + 0], dy = y - sa[m * 4 + 1], dz = z - sa[m * 4 + 2];
      const double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
      if (r2 >= rp2) {  // point charge: Z / r
        v = fma(Z, rsqrt_refined(r2), v);
      } else {
        const double r = sqrt(r2);
        v += (r < 1e-12) ? Z * c0 : Z * erf(r * inv) / r;
      }
    }
  }
  if (inside) {
    K[id] = interior ? (T)v : T(0);
    if (K64) K64[id] = interior ? v : 0.0;
  }
}

// initial state: nearest domain seed (f32 squared distances, first wins ties), psi = exp(-d)
template <typename T>
__device__ __forceinline__ void nm_init_body(T* __restrict__ U, int* __restrict__ label,
                                             const float4* __restrict__ seeds, int nSeed, const Geo& g, float h,
                                             long long blk, float4* ss) {
  const long long id = blk * blockDim.x + threadIdx.x;
  const bool inside = id < g.S3;
  int i = 0, j = 0, k = 0;
  if (inside) { i = (int)(id / g.S2); j = (int)((id / g.S) % g.S); k = (int)(id % g.S); }
  const float x = F_MUL((float)i, h), y = F_MUL((float)j, h), z = F_MUL((float)k, h);
  float best = 3.4e38f;
  int bl = 0;
  for (int base = 0; base < nSeed; base += 256) {
    const int cnt = min(256, nSeed - base);
    __syncthreads();
    if (threadIdx.x < cnt) ss[threadIdx.x] = seeds[base + threadIdx.x];
    __syncthreads();
    for (int m = 0; m < cnt; ++m) {
      const float4 s = ss[m];
      const float dx = F_SUB(x, s.x), dy = F_SUB(y, s.y), dz = F_SUB(z, s.z);
      const float d2 = F_ADD(F_ADD(F_MUL(dx, dx), F_MUL(dy, dy)), F_MUL(dz, dz));
      if (d2 < best) { best = d2; bl = __float_as_int(s.w); }
    }
  }
  if (!inside) return;
  const bool interior = i >= 1 && i < g.NN && j >= 1 && j < g.NN && k >= 1 && k < g.NN;
  label[id] = bl;
  U[id] = interior ? (T)exp(-sqrt((double)best)) : T(0);
}

// Unbiased rounding of the fp32 update.  With round-to-nearest, a change of psi smaller than half
// an ulp is lost at every step and the fp32 iteration stops short of the fixed point.  Instead the
// new value is formed exactly in FP64 and rounded down or up with probability proportional to the
// distance to each neighbour, so its expected value is exact.  The uniform variate is a
// counter-based hash of (grid point, step seed) -- the SplitMix64 finaliser (Steele, Lea and Flood,
// OOPSLA 2014) -- so a run is reproducible.
__device__ __forceinline__ unsigned sr_uniform24(unsigned long long id, unsigned seed) {
  unsigned long long x = id * 0x9E3779B97F4A7C15ull + (unsigned long long)seed * 0xD1B54A32D192ED03ull;
  x ^= x >> 30;
  x *= 0xBF58476D1CE4E5B9ull;
  x ^= x >> 27;
  x *= 0x94D049BB133111EBull;
  x ^= x >> 31;
  return (unsigned)(x >> 40);  // 24 bits
}
__device__ __forceinline__ float sr_round(double v, unsigned u24) {
  const float a = __double2float_rz(v);  // the neighbour toward zero
  const double rem = v - (double)a;      // same sign as v, |rem| < the ulp of a
  if (rem == 0.0) return a;
  const float b = nextafterf(a, v > 0.0 ? 3.0e38f : -3.0e38f);  // the neighbour away from zero
  const double frac = rem / ((double)b - (double)a);             // in (0, 1)
  return (double)u24 * 5.9604644775390625e-08 < frac ? b : a;   // u24 / 2^24
}

// ITP update (same-label Neumann Laplacian) on the march tile (bx, by, bz); with ACC the FP64
// norm of the new psi per label goes through the block table (caller inits and flushes it).
// With a non-null `scale` the stored psi is one normalisation behind.  The update is linear in
// psi and reads only neighbours of the centre's label (a neighbour of another label is replaced
// by the centre value), so the pending per-domain scale multiplies the result once: psi' =
// scale[label] * update(psi), formed in FP64 and rounded once -- normalise-then-update up to
// rounding, without a separate pass over psi.  With a non-null `seed` (fp32 fields) the stored
// value is rounded without bias (sr_round) from its exact FP64 form.
// Same-label neighbour mask of one interior point: bit q set when neighbour q (+i, -i, +j, -j,
// +k, -k) carries the point's label.  The update reads it in place of the six neighbour labels
// while the labels do not change (nm_mask_body writes it after every label change).
constexpr int kNmIp = 1, kNmIm = 2, kNmJp = 4, kNmJm = 8, kNmKp = 16, kNmKm = 32;
__device__ __forceinline__ unsigned char nm_same_label_mask(const int* __restrict__ label, long long id, long long S,
                                                            long long S2) {
  const int l = label[id];
  return (unsigned char)((label[id + S2] == l ? kNmIp : 0) | (label[id - S2] == l ? kNmIm : 0) |
                         (label[id + S] == l ? kNmJp : 0) | (label[id - S] == l ? kNmJm : 0) |
                         (label[id + 1] == l ? kNmKp : 0) | (label[id - 1] == l ? kNmKm : 0));
}

// The mask of every point of S^3 (0 on the boundary planes), flat: 256 * kNmFlatChunk points from blk.
__device__ __forceinline__ void nm_mask_body(const int* __restrict__ label, unsigned char* __restrict__ mask,
                                             const Geo& g, long long blk) {
  const long long base = blk * blockDim.x * kNmFlatChunk;
  for (int q = 0; q < kNmFlatChunk; ++q) {
    const long long id = base + (long long)q * blockDim.x + threadIdx.x;
    if (id >= g.S3) break;
    const int i = (int)(id / g.S2), j = (int)((id / g.S) % g.S), k = (int)(id % g.S);
    const bool interior = i >= 1 && i < g.NN && j >= 1 && j < g.NN && k >= 1 && k < g.NN;
    mask[id] = interior ? nm_same_label_mask(label, id, g.S, g.S2) : (unsigned char)0;
  }
}

// MASK: neighbour-label equality from `mask` (nm_mask_body of the same labels) instead of six label
// loads; the centre label is then read only where it is used (norm accumulation, pending scale).
// The arithmetic is the same, so both forms give the same bits.
// SR: the unbiased rounding of fp32 fields (seed non-null), compiled only where it is asked for
template <typename T, bool ACC, bool MASK = false, bool SR = false>
__device__ __forceinline__ void nm_update_body(const T* __restrict__ U, T* __restrict__ Unew, const T* __restrict__ K,
                                               const T* __restrict__ P, const int* __restrict__ label, const Geo& g,
                                               T half_dv, T dt, double h3, int nDom, double* __restrict__ norms,
                                               DomTable<1, 128>& tab, int bx, int by, int bz,
                                               const double* __restrict__ scale = nullptr,
                                               const unsigned* __restrict__ seed = nullptr,
                                               const NmTile t = kNmTile,
                                               const unsigned char* __restrict__ mask = nullptr) {
  using A = Ar<T>;
  RunSum<1> rs;
  rs.reset();
  int k, j, i0;
  nm_tile_origin(t, bx, by, bz, k, j, i0);
  if (k < g.NN && j < g.NN && i0 < g.NN) {
    const int iend = min(i0 + t.march, g.NN);
    const long long S = g.S, S2 = g.S2;
    long long id = (long long)i0 * S2 + j * S + k;
    const unsigned sd = (SR && seed) ? __ldg(seed) : 0u;
    const bool need_l = !MASK || ACC || scale != nullptr;
    T u_m = __ldg(U + id - S2), u_c = __ldg(U + id);
    int l_m = MASK ? 0 : __ldg(label + id - S2), l_c = need_l ? __ldg(label + id) : 0;
    for (int i = i0; i < iend; ++i, id += S2) {
      const T u_p = __ldg(U + id + S2);
      const T ujp = __ldg(U + id + S), ujm = __ldg(U + id - S), ukp = __ldg(U + id + 1), ukm = __ldg(U + id - 1);
      const T kv = __ldg(K + id), pv = __ldg(P + id);
      T a, b, c, d, e, f;
      int l_p = 0;
      if (MASK) {
        const unsigned m = __ldg(mask + id);
        if (need_l && i + 1 < iend) l_p = __ldg(label + id + S2);
        a = (m & kNmIp) ? u_p : u_c;
        b = (m & kNmIm) ? u_m : u_c;
        c = (m & kNmJp) ? ujp : u_c;
        d = (m & kNmJm) ? ujm : u_c;
        e = (m & kNmKp) ? ukp : u_c;
        f = (m & kNmKm) ? ukm : u_c;
      } else {
        l_p = __ldg(label + id + S2);
        const int ljp = __ldg(label + id + S), ljm = __ldg(label + id - S), lkp = __ldg(label + id + 1),
                  lkm = __ldg(label + id - 1);
        a = (l_p == l_c) ? u_p : u_c;
        b = (l_m == l_c) ? u_m : u_c;
        c = (ljp == l_c) ? ujp : u_c;
        d = (ljm == l_c) ? ujm : u_c;
        e = (lkp == l_c) ? ukp : u_c;
        f = (lkm == l_c) ? ukm : u_c;
      }
      const T lap = A::sub(A::add(A::add(A::add(A::add(A::add(a, b), c), d), e), f), A::mul(T(6), u_c));
      T out;
      if (SR && sizeof(T) == sizeof(float) && seed) {
        // the same f32 terms, summed exactly in FP64, scaled, then one unbiased rounding
        double v = ((double)u_c + (double)A::mul(half_dv, lap)) + (double)A::mul(A::mul(dt, A::sub(kv, A::mul(T(2), pv))), u_c);
        if (scale) v *= __ldg(scale + min(max(l_c, 0), nDom - 1));
        out = (T)sr_round(v, sr_uniform24((unsigned long long)id, sd));
      } else {
        out = A::add(A::add(u_c, A::mul(half_dv, lap)), A::mul(A::mul(dt, A::sub(kv, A::mul(T(2), pv))), u_c));
        if (scale) out = (T)((double)out * __ldg(scale + min(max(l_c, 0), nDom - 1)));
      }
      Unew[id] = out;
      if (ACC) {
        const double r = (double)out * (double)out * h3;
        rs.add(min(max(l_c, 0), nDom - 1), &r, tab, norms);
      }
      u_m = u_c; u_c = u_p; l_m = l_c; l_c = l_p;
    }
  }
  if (ACC) rs.finish_warp(tab, norms);  // every lane of the block reaches this point
}

// U *= scale[label] (FP64 product, rounded once) for labels in [0, nDom) over kNmFlatChunk*256
// points from blk.  With 16-byte aligned fields each thread moves 16-byte vectors of psi (and the
// matching int4 / int2 of labels), kNmFlatChunk points in all; the block covers the same points
// as the scalar walk and every point gets the same product.
template <typename T>
__device__ __forceinline__ void nm_apply_scale_point(T& u, int l, const double* __restrict__ scale, int nDom) {
  if (l >= 0 && l < nDom) u = (T)((double)u * scale[l]);
}

template <typename T>
__device__ __forceinline__ void nm_apply_scale_body(T* __restrict__ U, const int* __restrict__ label,
                                                    const double* __restrict__ scale, long long S3, int nDom,
                                                    long long blk) {
  const long long base = blk * blockDim.x * kNmFlatChunk;
  if ((((unsigned long long)U | (unsigned long long)label) & 15) == 0) {
    constexpr int W = 16 / (int)sizeof(T);  // points per vector
#pragma unroll
    for (int q = 0; q < kNmFlatChunk / W; ++q) {
      const long long e0 = base + ((long long)q * blockDim.x + threadIdx.x) * W;
      if (e0 + W <= S3) {
        if constexpr (sizeof(T) == sizeof(float)) {
          float4 u = *reinterpret_cast<const float4*>(U + e0);
          const int4 l = *reinterpret_cast<const int4*>(label + e0);
          nm_apply_scale_point(u.x, l.x, scale, nDom);
          nm_apply_scale_point(u.y, l.y, scale, nDom);
          nm_apply_scale_point(u.z, l.z, scale, nDom);
          nm_apply_scale_point(u.w, l.w, scale, nDom);
          *reinterpret_cast<float4*>(U + e0) = u;
        } else {
          double2 u = *reinterpret_cast<const double2*>(U + e0);
          const int2 l = *reinterpret_cast<const int2*>(label + e0);
          nm_apply_scale_point(u.x, l.x, scale, nDom);
          nm_apply_scale_point(u.y, l.y, scale, nDom);
          *reinterpret_cast<double2*>(U + e0) = u;
        }
      } else {
        for (long long e = e0; e < S3; ++e) nm_apply_scale_point(U[e], label[e], scale, nDom);
      }
    }
    return;
  }
  for (int q = 0; q < kNmFlatChunk; ++q) {
    const long long id = base + (long long)q * blockDim.x + threadIdx.x;
    if (id >= S3) break;
    nm_apply_scale_point(U[id], label[id], scale, nDom);
  }
}

// FP64 per-label psi^2 h^3 over kNmFlatChunk*256 points from blk (label clipped to [0, nDom))
template <typename T>
__device__ __forceinline__ void nm_norms_body(const T* __restrict__ U, const int* __restrict__ label, long long S3,
                                              double h3, int nDom, double* __restrict__ norms, DomTable<1, 128>& tab,
                                              long long blk) {
  RunSum<1> rs;
  rs.reset();
  const long long base = blk * blockDim.x * kNmFlatChunk;
  for (int q = 0; q < kNmFlatChunk; ++q) {
    const long long id = base + (long long)q * blockDim.x + threadIdx.x;
    if (id >= S3) break;
    const double u = (double)U[id];
    const double r = u * u * h3;
    rs.add(min(max(label[id], 0), nDom - 1), &r, tab, norms);
  }
  rs.finish(tab, norms);
}

// fine-level right-hand side f = (2 pi psi) psi formed from psi on the fly
template <typename T, bool FINE>
__device__ __forceinline__ T rhs_at(const T* __restrict__ f, long long id) {
  if (FINE) {
    const T u = f[id];
    return Ar<T>::mul(Ar<T>::mul((T)6.283185307179586, u), u);
  }
  return f[id];
}

// one colour of a red-black sweep for A P = f, A P = (6P - sum_6 P)/h^2; block (32, 8): each
// thread owns the pair (k0, k0+1) of row j on the kNmRowPlanes planes i from 1 + bz*kNmRowPlanes,
// and on each plane updates the one of the pair that has the colour.  The pass is in place, so
// the compiler may not move a plane's loads above the previous plane's store; they only read
// points of the other colour, which the pass does not change, so all planes' loads are issued
// first (explicitly) and the updates follow.
template <typename T, bool FINE>
__device__ __forceinline__ void nm_rbgs_body(T* __restrict__ P, const T* __restrict__ f, const Geo& g, T h2, int color,
                                             int bx, int by, int bz) {
  using A = Ar<T>;
  const int k0 = 1 + bx * 64 + 2 * tile_x<32>();
  const int j = 1 + by * kNmRowTJ + tile_y<32>();
  const int i0 = 1 + bz * kNmRowPlanes;
  if (j >= g.NN || k0 >= g.NN) return;
  const int iend = min(i0 + kNmRowPlanes, g.NN);
  const long long S = g.S, S2 = g.S2;
  T s[kNmRowPlanes], rhs[kNmRowPlanes];
  long long ids[kNmRowPlanes];
#pragma unroll
  for (int q = 0; q < kNmRowPlanes; ++q) {
    const int i = i0 + q;
    const int k = k0 + ((i + j + k0 + color) & 1);
    ids[q] = (i < iend && k < g.NN) ? (long long)i * S2 + (long long)j * S + k : -1;
    const long long id = ids[q] >= 0 ? ids[q] : S2 + S + 1;  // an interior point: in bounds, not stored
    s[q] = A::add(A::add(A::add(A::add(A::add(P[id + S2], P[id - S2]), P[id + S]), P[id - S]), P[id + 1]), P[id - 1]);
    rhs[q] = rhs_at<T, FINE>(f, id);
  }
#pragma unroll
  for (int q = 0; q < kNmRowPlanes; ++q)
    if (ids[q] >= 0) P[ids[q]] = A::div(A::add(s[q], A::mul(h2, rhs[q])), T(6));
}

// residual f - A P at one interior point from its P values (+i, -i, +j, -j, +k, -k, centre) and
// its right-hand side
template <typename T>
__device__ __forceinline__ T nm_residual_value(T pip, T pim, T pjp, T pjm, T pkp, T pkm, T pc, T rhs, T inv_h2) {
  using A = Ar<T>;
  if (sizeof(T) == sizeof(float)) {
    // fp32 fields: sum_6 P - 6 P cancels most of its digits (P is smooth), so the residual is
    // formed in FP64 from the fp32 values (each operation rounded to nearest) and rounded once --
    // this is what lets the fp32 multigrid reach the fp32 resolution of P instead of stalling at
    // ~1e-4 relative
    const double sd = __dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn((double)pip, (double)pim), (double)pjp),
                                                    (double)pjm), (double)pkp), (double)pkm);
    return (T)__dadd_rn((double)rhs, __dmul_rn(__dsub_rn(sd, __dmul_rn(6.0, (double)pc)), (double)inv_h2));
  }
  const T s = A::add(A::add(A::add(A::add(A::add(pip, pim), pjp), pjm), pkp), pkm);
  return A::add(rhs, A::mul(A::sub(s, A::mul(T(6), pc)), inv_h2));
}

// residual r = f - A P at one interior point
template <typename T, bool FINE>
__device__ __forceinline__ void nm_residual_point(const T* __restrict__ P, const T* __restrict__ f, T* __restrict__ r,
                                                  long long id, long long S, long long S2, T inv_h2) {
  r[id] = nm_residual_value<T>(P[id + S2], P[id - S2], P[id + S], P[id - S], P[id + 1], P[id - 1], P[id],
                               rhs_at<T, FINE>(f, id), inv_h2);
}

// Row tiling shared by the residual and the prolongation: block (32, 8) covers 64 points of k
// on 8 rows j of the kNmRowPlanes planes from i = 1 + bz*kNmRowPlanes; thread x takes
// k = 1 + 64 bx + x and k + 32 on each plane.  Every point is independent (no dependent chain
// along i), so levels of every size fill the SMs, and each warp load is one contiguous run of 32
// values.
#define NM_ROWS_PROLOGUE                                  \
  const int j = 1 + by * kNmRowTJ + tile_y<32>();        \
  const int tx = tile_x<32>();                            \
  const int i0 = 1 + bz * kNmRowPlanes;                   \
  if (j >= g.NN) return;                                  \
  const int iend = min(i0 + kNmRowPlanes, g.NN);          \
  const long long S = g.S, S2 = g.S2;

template <typename T, bool FINE>
__device__ __forceinline__ void nm_residual_rows_body(const T* __restrict__ P, const T* __restrict__ f,
                                                      T* __restrict__ r, const Geo& g, T inv_h2, int bx, int by,
                                                      int bz) {
  NM_ROWS_PROLOGUE
#pragma unroll
  for (int q = 0; q < kNmRowPlanes; ++q) {
    const int i = i0 + q;
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      const int k = 1 + bx * 64 + tx + 32 * t;
      if (i < iend && k < g.NN)
        nm_residual_point<T, FINE>(P, f, r, (long long)i * S2 + (long long)j * S + k, S, S2, inv_h2);
    }
  }
}

// Trilinear prolongation + correction, P += I E_c, on the row tiling.  A fine point averages the
// 1, 2, 4 or 8 coarse values around it, summed in the order (a, b, c) = (i, j, k) offsets with
// k fastest, then divided by their count.  The i and j parities are uniform over a warp's row;
// only the k parity alternates between lanes, and it selects whether a second value is added.
template <typename T>
__device__ __forceinline__ void nm_prolong_rows_body(const T* __restrict__ Ec, T* __restrict__ P, const Geo& g,
                                                     const Geo& gc, int bx, int by, int bz) {
  using A = Ar<T>;
  NM_ROWS_PROLOGUE
  const int oj = j & 1;
#pragma unroll
  for (int q = 0; q < kNmRowPlanes * 2; ++q) {
    const int i = i0 + (q >> 1);
    const int k = 1 + bx * 64 + tx + 32 * (q & 1);
    if (i >= iend || k >= g.NN) continue;
    const int oi = i & 1;
    const long long row0 = (long long)(i >> 1) * gc.S2 + (long long)(j >> 1) * gc.S;
    const int ck = k >> 1, ok = k & 1;
    T v = T(0);
    auto add_row = [&](long long row) {
      v = A::add(v, Ec[row + ck]);
      if (ok) v = A::add(v, Ec[row + ck + 1]);
    };
    add_row(row0);
    if (oj) add_row(row0 + gc.S);
    if (oi) {
      add_row(row0 + gc.S2);
      if (oj) add_row(row0 + gc.S2 + gc.S);
    }
    v = A::div(v, (T)((1 + oi) * (1 + oj) * (1 + ok)));
    const long long id = (long long)i * S2 + (long long)j * S + k;
    P[id] = A::add(P[id], v);
  }
}
#undef NM_ROWS_PROLOGUE

// The same prolongation by coarse cells: thread (x, y) of a block of 256 owns the cells (I, J, K) =
// (I0 + t, by * 8 + y, bx * 32 + x) for `planes` values of t and updates the 2 x 2 x 2 fine
// points (2I + a, 2J + b, 2K + c) of each that are interior.  A fine point with offsets (a, b, c)
// averages the coarse values (I + da, J + db, K + dc) with da <= a, db <= b, dc <= c, added in
// the (da, db, dc) order of nm_prolong_rows_body and scaled by the exact reciprocal of their
// count, so the result is the row body's bit for bit.  Every load is unconditional (no branch
// on parities) and each coarse plane is loaded once per march: 4 coarse and 8 fine loads and 8
// fine stores per cell.
constexpr int kNmPrTK = 32, kNmPrTJ = 8;
template <typename T>
__device__ __forceinline__ void nm_prolong_cells_body(const T* __restrict__ Ec, T* __restrict__ P, const Geo& g,
                                                      const Geo& gc, int bx, int by, int bz, int planes) {
  using A = Ar<T>;
  const int nc = gc.NN;  // coarse cells 0..nc-1 along each axis cover the fine interior 1..NN-1
  const int K = bx * kNmPrTK + tile_x<32>(), J = by * kNmPrTJ + tile_y<32>();
  if (K >= nc || J >= nc) return;
  const int I0 = bz * planes;
  const int Iend = min(I0 + planes, nc);
  const long long S = g.S, S2 = g.S2, Sc = gc.S, Sc2 = gc.S2;
  T c0[2][2], c1[2][2];  // coarse values of planes I and I + 1: [db][dc]
#pragma unroll
  for (int db = 0; db < 2; ++db)
#pragma unroll
    for (int dc = 0; dc < 2; ++dc) c0[db][dc] = Ec[(long long)I0 * Sc2 + (long long)(J + db) * Sc + K + dc];
  for (int I = I0; I < Iend; ++I) {
#pragma unroll
    for (int db = 0; db < 2; ++db)
#pragma unroll
      for (int dc = 0; dc < 2; ++dc) c1[db][dc] = Ec[(long long)(I + 1) * Sc2 + (long long)(J + db) * Sc + K + dc];
#pragma unroll
    for (int a = 0; a < 2; ++a) {
      const int i = 2 * I + a;
      if (i < 1) continue;  // the fine boundary plane
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        const int j = 2 * J + b;
        if (j < 1) continue;
        const long long row = (long long)i * S2 + (long long)j * S;
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          const int k = 2 * K + c;
          if (k < 1) continue;
          T v = A::add(T(0), c0[0][0]);
          if (c) v = A::add(v, c0[0][1]);
          if (b) {
            v = A::add(v, c0[1][0]);
            if (c) v = A::add(v, c0[1][1]);
          }
          if (a) {
            v = A::add(v, c1[0][0]);
            if (c) v = A::add(v, c1[0][1]);
            if (b) {
              v = A::add(v, c1[1][0]);
              if (c) v = A::add(v, c1[1][1]);
            }
          }
          v = A::mul(v, (T)(1.0 / ((1 + a) * (1 + b) * (1 + c))));
          P[row + k] = A::add(P[row + k], v);
        }
      }
    }
#pragma unroll
    for (int db = 0; db < 2; ++db)
#pragma unroll
      for (int dc = 0; dc < 2; ++dc) c0[db][dc] = c1[db][dc];
  }
}

// full weighting (1/64)(8,4,2,1) at coarse interior point number q; loop order a, b, c
template <typename T>
__device__ __forceinline__ void nm_restrict_body(const T* __restrict__ fine, T* __restrict__ coarse, const Geo& g,
                                                 const Geo& gc, long long q) {
  using A = Ar<T>;
  const int n = gc.NN - 1;
  if (q >= (long long)n * n * n) return;
  const int K2 = 1 + (int)(q % n), J = 1 + (int)((q / n) % n), I = 1 + (int)(q / ((long long)n * n));
  T v = T(0);
  for (int a = -1; a <= 1; ++a)
    for (int b = -1; b <= 1; ++b)
      for (int c = -1; c <= 1; ++c) {
        const T w = (T)((a == 0 ? 2 : 1) * (b == 0 ? 2 : 1) * (c == 0 ? 2 : 1));
        v = A::add(v, A::mul(w, fine[(long long)(2 * I + a) * g.S2 + (long long)(2 * J + b) * g.S + (2 * K2 + c)]));
      }
  coarse[(long long)I * gc.S2 + (long long)J * gc.S + K2] = A::div(v, T(64));
}

// Residual and full weighting in one pass: fc = R (f - A P) on the coarse interior without storing
// the fine residual, and the coarse correction Pc (when given) zeroed on the same points.  The
// block (256 threads, read as 32 x 8) owns the coarse points (K, J) = (K0 + x, J0 + y) of a 32 x 8
// tile on `planes` coarse planes from I0, and walks the fine planes 2 I0 - 1 .. 2 Ilast + 1.
// On each fine plane it forms the residual on the 65 x 17 fine patch under the tile into shared
// memory (every thread keeps the P values of its patch points on the planes below and above in
// registers).  One step per coarse plane I forms the fine planes 2I and 2I + 1 and, after one
// barrier, adds the 3 x 3 patch values of the fine planes 2I - 1, 2I and 2I + 1 around each coarse
// point with their weights.  The sums run in the (a, b, c) order of nm_restrict_body and the
// residual is nm_residual_value, so the result is the one of the residual pass and the
// restriction.  A ring of kNmRrBuf (5) patch planes lets the next step's planes be written while
// slower threads still read this step's three: one barrier per coarse plane.
constexpr int kNmRrTK = 32, kNmRrTJ = 8;

// Coarse planes per block of the residual-restriction and prolongation kernels for a launch of
// `blocks_per_plane` blocks on each of n coarse planes: 8, halved while the launch would have
// fewer than 8 blocks per SM (small levels and single grids favour more blocks over the extra
// fine plane a block forms at its chunk's ends).
inline int nm_mg_planes(long long blocks_per_plane, int n) {
  int planes = 8;
  while (planes > 1 && blocks_per_plane * ((n + planes - 1) / planes) < 8LL * 148) planes /= 2;
  return planes;
}
constexpr int kNmRrPK = 2 * kNmRrTK + 1;                      // fine patch row (65 points)
constexpr int kNmRrPatch = kNmRrPK * (2 * kNmRrTJ + 1);       // 65 x 17 fine points
constexpr int kNmRrPer = (kNmRrPatch + 255) / 256;            // patch points per thread
constexpr int kNmRrBuf = 5;                                   // patch planes in the ring

template <typename T, bool FINE>
__device__ __forceinline__ void nm_resrestrict_body(const T* __restrict__ P, const T* __restrict__ f, T* __restrict__ fc,
                                                    T* __restrict__ Pc, const Geo& g, const Geo& gc, T inv_h2, int bx,
                                                    int by, int bz, int planes, T (*patch)[kNmRrPatch]) {
  using A = Ar<T>;
  const int n = gc.NN - 1;  // coarse interior 1..n
  const int I0 = 1 + bz * planes;
  if (I0 > n) return;  // the whole block
  const int Ilast = min(I0 + planes - 1, n);
  const int tx = tile_x<32>(), ty = tile_y<32>(), tid = tx + 32 * ty;
  const int K0 = 1 + bx * kNmRrTK, J0 = 1 + by * kNmRrTJ;
  const int K = K0 + tx, J = J0 + ty;
  const bool own = K <= n && J <= n;
  const long long S = g.S, S2 = g.S2;
  const int fi0 = 2 * I0 - 1;
  // fine (j, k) offset of each patch point of this thread; points outside the grid use the
  // offset of (1, 1) (in bounds, their residuals are not stored)
  int col[kNmRrPer];
  bool in[kNmRrPer];
  T pm[kNmRrPer], pc[kNmRrPer];  // P of each patch point on the planes below and at the next residual plane
#pragma unroll
  for (int m = 0; m < kNmRrPer; ++m) {
    const int p = tid + 256 * m;
    const int fj = 2 * J0 - 1 + p / kNmRrPK, fk = 2 * K0 - 1 + p % kNmRrPK;
    in[m] = p < kNmRrPatch && fj < g.NN && fk < g.NN;
    col[m] = in[m] ? fj * g.S + fk : g.S + 1;
    pm[m] = P[(long long)(fi0 - 1) * S2 + col[m]];
    pc[m] = P[(long long)fi0 * S2 + col[m]];
  }
  auto residual_plane = [&](int i) {  // the residuals of fine plane i into its ring slot
    T* buf = patch[i % kNmRrBuf];
    const long long base = (long long)i * S2;
#pragma unroll
    for (int m = 0; m < kNmRrPer; ++m) {
      const long long id = base + col[m];
      const T pp = P[id + S2];
      const T r = nm_residual_value<T>(pp, pm[m], P[id + S], P[id - S], P[id + 1], P[id - 1], pc[m],
                                       rhs_at<T, FINE>(f, id), inv_h2);
      if (in[m]) buf[tid + 256 * m] = r;
      pm[m] = pc[m];
      pc[m] = pp;
    }
  };
  residual_plane(fi0);
  for (int I = I0; I <= Ilast; ++I) {
    residual_plane(2 * I);
    residual_plane(2 * I + 1);
    __syncthreads();
    if (!own) continue;
    T v = T(0);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const T* q = patch[(2 * I - 1 + a) % kNmRrBuf] + (2 * ty) * kNmRrPK + 2 * tx;  // fine (2J - 1, 2K - 1)
#pragma unroll
      for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int c = 0; c < 3; ++c)
          v = A::add(v, A::mul((T)((a == 1 ? 2 : 1) * (b == 1 ? 2 : 1) * (c == 1 ? 2 : 1)), q[b * kNmRrPK + c]));
    }
    const long long cid = (long long)I * gc.S2 + (long long)J * gc.S + K;
    fc[cid] = A::div(v, T(64));
    if (Pc) Pc[cid] = T(0);
  }
}

// coarsest level: `sweeps` red-black sweeps in FP64 by one block; sm: 2*S^3 doubles of smem
template <typename T>
__device__ __forceinline__ void nm_coarsest_body(T* __restrict__ P, const T* __restrict__ f, const Geo& g, double h2,
                                                 int sweeps, double* sm) {
  double* sP = sm;
  double* sf = sm + g.S3;
  for (long long q = threadIdx.x; q < g.S3; q += blockDim.x) { sP[q] = (double)P[q]; sf[q] = (double)f[q]; }
  __syncthreads();
  const int n = g.NN - 1, S = g.S, S2 = (int)g.S2;  // the coarsest level is at most 29^3 points
  const int nint = n * n * n;
  for (int s = 0; s < sweeps; ++s)
    for (int color = 0; color < 2; ++color) {
      for (int q = threadIdx.x; q < nint; q += blockDim.x) {
        const int k = 1 + q % n, j = 1 + (q / n) % n, i = 1 + q / (n * n);
        if (((i + j + k) & 1) != color) continue;
        const int id = i * S2 + j * S + k;
        const double sum = __dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(sP[id + S2], sP[id - S2]), sP[id + S]),
                                                        sP[id - S]), sP[id + 1]), sP[id - 1]);
        sP[id] = __ddiv_rn(__dadd_rn(sum, __dmul_rn(h2, sf[id])), 6.0);
      }
      __syncthreads();
    }
  for (long long q = threadIdx.x; q < g.S3; q += blockDim.x) P[q] = (T)sP[q];
}

// Per-domain readout sums, kNmPD per domain: (norm, T, V_eK, h^3 sum P rho, h^3 sum P (A P)) on the
// march tile, A = -lap_h with Dirichlet faces (the multigrid's operator).  T counts every
// same-label edge with an interior end point once (forward edges + the edge to the Dirichlet face
// on the first layer).  The last sum is attributed to the point's domain only for bookkeeping: the
// readout uses its total in the P-stationary Hartree energy 2 h^3 sum P rho - (h^3 / 2 pi) sum P A P
// (kNmPD, rq_internal.cuh).
// With K64 (fp32 fields) the nuclear term reads the FP64 potential: the fields evolve with the f32
// rounding of K, and reading the energy with the unrounded K removes that rounding from it at first
// order (the state is stationary, so what is left is second order).
template <typename T>
__device__ __forceinline__ void nm_energy_body(const T* __restrict__ U, const T* __restrict__ K, const T* __restrict__ P,
                                               const int* __restrict__ label, const Geo& g, double h, int nDom,
                                               double* __restrict__ pd, DomTable<kNmPD, 128>& tab, int bx, int by,
                                               int bz, const double* __restrict__ K64 = nullptr,
                                               const NmTile t = kNmTile) {
  RunSum<kNmPD> rs;
  rs.reset();
  const double h3 = h * h * h;
  int k, j, i0;
  nm_tile_origin(t, bx, by, bz, k, j, i0);
  if (k < g.NN && j < g.NN && i0 < g.NN) {
    const int iend = min(i0 + t.march, g.NN);
    const long long S = g.S, S2 = g.S2;
    for (int i = i0; i < iend; ++i) {
      const long long id = (long long)i * S2 + j * S + k;
      const double u = U[id], rho = u * u;
      const int L = label[id];
      if (L < 0 || L >= nDom) continue;
      const double a = (label[id + S2] == L) ? (double)U[id + S2] - u : 0.0;
      const double b = (label[id + S] == L) ? (double)U[id + S] - u : 0.0;
      const double c = (label[id + 1] == L) ? (double)U[id + 1] - u : 0.0;
      double t = a * a + b * b + c * c;
      if (i == 1 && label[id - S2] == L) t += u * u;
      if (j == 1 && label[id - S] == L) t += u * u;
      if (k == 1 && label[id - 1] == L) t += u * u;
      const double pc = (double)P[id];
      const double ap = (6.0 * pc - ((double)P[id + S2] + (double)P[id - S2] + (double)P[id + S] + (double)P[id - S] +
                                     (double)P[id + 1] + (double)P[id - 1])) / (h * h);
      const double kv = K64 ? K64[id] : (double)K[id];
      double v[kNmPD] = {rho * h3, 0.5 * t * h, -kv * rho * h3, pc * rho * h3, pc * ap * h3};
      rs.add(L, v, tab, pd);
    }
  }
  rs.finish_warp(tab, pd);
}

// level-set label update (molecule.js:426-540 rule) on psi of type T, march tile
template <typename T>
__device__ __forceinline__ void nm_evolve_body(const int* __restrict__ labIn, int* __restrict__ labOut,
                                               const T* __restrict__ U, float* __restrict__ W, const Geo& g, T dt_w,
                                               T curvReg, int bx, int by, int bz, const NmTile t = kNmTile) {
  using A = Ar<T>;
  int k, j, i0;
  nm_tile_origin(t, bx, by, bz, k, j, i0);
  if (k >= g.NN || j >= g.NN || i0 >= g.NN) return;
  const int iend = min(i0 + t.march, g.NN);
  const long long S = g.S, S2 = g.S2;
  for (int i = i0; i < iend; ++i) {
    const long long id = (long long)i * S2 + j * S + k;
    const int myL = labIn[id];
    const T uc = U[id];
    const T myRho = A::mul(uc, uc);
    const long long nb[6] = {id + S2, id - S2, id + S, id - S, id + 1, id - 1};
    int bestL = myL;
    T bestRho = T(0), myCnt = T(0);
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      const int l = labIn[nb[q]];
      if (l == myL) {
        myCnt = A::add(myCnt, T(1));
      } else {
        const T un = U[nb[q]];
        const T r = A::mul(un, un);
        if (r > bestRho) { bestRho = r; bestL = l; }
      }
    }
    T w = (T)W[id];
    if (myCnt >= T(6)) {
      W[id] = (float)(w > T(1) ? w : T(1));
      labOut[id] = myL;
      continue;
    }
    const T denom = A::add(myRho, bestRho);
    const T vel = (denom < (T)1e-20f) ? T(0) : A::div(A::sub(myRho, bestRho), denom);
    w = A::add(w, A::mul(dt_w, vel));
    const T curv = A::div(A::sub(myCnt, T(3)), T(3));
    w = A::add(w, A::mul(curvReg, curv));
    int newL = myL;
    if (w < T(0)) { newL = bestL; w = (T)0.1f; }
    W[id] = (float)w;
    labOut[id] = newL;
  }
}

// Gaussian-nucleus force: tiles t = t0, t0+stride, ... of interior points staged in smem as FP64
// (x, y, z, weight) whatever the field type, thread = nucleus a of chunk `chunk`.  With gw ==
// nullptr the Hellmann-Feynman gather F_a = -h^3 sum rho dK/dr (x-R)/r; with a weight field gw =
// dE/dK (one value per grid point) the gradient gather F_a = -dE/dR_a = sum gw dK_a/dr (x-R)/r,
// of which the first is the case gw = -h^3 rho.  The per-nucleus factor (weight scale x Z) is
// applied once, after the sums.
template <typename T>
__device__ __forceinline__ void nm_force_body(const T* __restrict__ U, const double* __restrict__ at, int nAt,
                                              const Geo& g, double h, double sigma, double* __restrict__ F,
                                              long long t0, long long tstride, int chunk, double* sx, double* sy,
                                              double* sz, double* sr, const double* __restrict__ gw = nullptr) {
  const int a = chunk * blockDim.x + threadIdx.x;
  const bool valid = a < nAt && at[a * 4 + 3] > 0.0;
  const double Z = valid ? at[a * 4 + 3] : 0.0;
  const double ax = valid ? at[a * 4 + 0] : 0.0, ay = valid ? at[a * 4 + 1] : 0.0, az = valid ? at[a * 4 + 2] : 0.0;
  const double inv = 1.0 / (1.4142135623730951 * sigma), gs = 0.7978845608028654 / sigma;
  const double inv2 = inv * inv, rp2 = nm_point_r2(sigma);
  const double h3 = h * h * h;
  const long long n1 = g.NN - 1, nInt = n1 * n1 * n1;
  const long long ntiles = (nInt + kNmForceTile - 1) / kNmForceTile;
  double fx = 0, fy = 0, fz = 0;
  for (long long t = t0; t < ntiles; t += tstride) {
    __syncthreads();
    for (int q = threadIdx.x; q < kNmForceTile; q += blockDim.x) {
      const long long v = t * kNmForceTile + q;
      double wt = 0.0, x = 0.0, y = 0.0, z = 0.0;
      if (v < nInt) {
        const int i = 1 + (int)(v / (n1 * n1)), j = 1 + (int)((v / n1) % n1), k = 1 + (int)(v % n1);
        const long long id = (long long)i * g.S2 + (long long)j * g.S + k;
        if (gw) {
          wt = gw[id];
        } else {
          const double u = (double)U[id];
          wt = u * u;
        }
        x = i * h; y = j * h; z = k * h;
      }
      sx[q] = x; sy[q] = y; sz[q] = z; sr[q] = wt;
    }
    __syncthreads();
    if (valid) {
      double lx = 0, ly = 0, lz = 0;  // sum weight x (dK/dr / Z) (x - R) / r
      for (int q = 0; q < kNmForceTile; ++q) {
        const double s = sr[q];
        const double dx = sx[q] - ax, dy = sy[q] - ay, dz = sz[q] - az;
        const double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
        double w;
        if (r2 >= rp2) {  // point charge: dK/dr / r = -Z / r^3
          const double ir = rsqrt_refined(r2);
          w = -s * (ir * ir * ir);
        } else if (r2 < 1e-24) {
          w = 0.0;
        } else {
          const double r = sqrt(r2);
          w = s * (gs * exp(-r2 * inv2) / r - erf(r * inv) / r2) / r;
        }
        lx = fma(w, dx, lx); ly = fma(w, dy, ly); lz = fma(w, dz, lz);
      }
      fx += lx; fy += ly; fz += lz;
    }
  }
  if (valid) {
    const double f = (gw ? 1.0 : -h3) * Z;  // HF: the staged value is rho, its weight -h^3 rho
    atomicAdd(&F[a * 3 + 0], f * fx);
    atomicAdd(&F[a * 3 + 1], f * fy);
    atomicAdd(&F[a * 3 + 2], f * fz);
  }
}

}  // namespace rq
