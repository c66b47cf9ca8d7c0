// nm_farfield.cu -- tiled nuclear sums of the new flavour for grids with many nuclei.
//
// K(x) = sum_a Z_a erf(|x - R_a| / (sqrt2 sigma)) / |x - R_a| and the force gathers
// F_a = sum_x w(x) dK_a/dr (x - R_a) / r are direct sums over every (voxel, nucleus) pair:
// 1e11 pairs for 3000 nuclei on 320^3.  Here the interior is cut into tiles of <= 32^3 points.
// For each tile, the nuclei within kFfFar tile half-widths of its box ("near") are summed
// directly at every point with the exact Gaussian-nucleus terms; the others are point charges
// there (erf = 1 from 6 sqrt2 sigma on) whose summed Coulomb field is harmonic inside the box and
// is represented by its values at a 16^3 tensor grid of Chebyshev points of the box, interpolated
// to the tile's points with the tensor Lagrange basis (three one-axis passes).  Measured worst
// case over atom directions for a 32-point box and nuclei at 3 half-widths: 1.7e-13 relative
// for the potential, 8e-12 relative for its gradient.  The force gather is the exact transpose:
// the tile's weights are anterpolated onto the nodes (W_n = sum_x w(x) L_n(x)) and each far
// nucleus gathers over the nodes, so the tiled forces are the gradient of the tiled energy.
// Pair work at 3000 nuclei on 320^3: 5.3e9 near pairs + 1.2e10 node pairs, against 9.8e10.
#include <algorithm>
#include <cmath>
#include <vector>

#include "nm_bodies.cuh"
#include "rq_ctx.h"
#include "rq_flavors.h"

namespace rq {

constexpr int kFfT = 32;                     // tile points per axis (at most)
constexpr int kFfN = 16;                     // Chebyshev nodes per axis
constexpr int kFfN3 = kFfN * kFfN * kFfN;
constexpr double kFfFar = 3.0;               // near: distance to the tile box below 3 half-widths
constexpr int kFfTabM = kFfT + 1;            // Lagrange tables for tile sizes m = 0..32
// tabs layout: tau[16] (nodes on [-1, 1]), then L[m][p][q] = l_q(t_p), t_p = -1 + 2p/(m-1)
constexpr int kFfTabs = kFfN + kFfTabM * kFfT * kFfN;

struct FfGeo {
  int nt, base, rem;  // tiles per axis; points per tile: base, +1 for the first rem tiles
  double h;
};

__host__ __device__ __forceinline__ void ff_span(const FfGeo& f, int t, int& start, int& m) {
  m = f.base + (t < f.rem ? 1 : 0);
  start = 1 + t * f.base + (t < f.rem ? t : f.rem);
}

struct FfBox {
  double lo[3], hi[3], c[3], a[3], d2;  // bounds, centre, half-width (bohr); squared near radius
  int s[3], m[3];                       // first grid index and point count per axis
};

__device__ __forceinline__ FfBox ff_box(const FfGeo& f, int t) {
  FfBox b;
  const int idx[3] = {t / (f.nt * f.nt), (t / f.nt) % f.nt, t % f.nt};
  double amax = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    ff_span(f, idx[d], b.s[d], b.m[d]);
    b.lo[d] = b.s[d] * f.h;
    b.hi[d] = (b.s[d] + b.m[d] - 1) * f.h;
    b.c[d] = 0.5 * (b.lo[d] + b.hi[d]);
    b.a[d] = 0.5 * (b.hi[d] - b.lo[d]);
    amax = fmax(amax, b.a[d]);
  }
  const double D = kFfFar * amax;
  b.d2 = D * D;
  return b;
}

// the one classification every kernel uses (same operations, so lists and node sums agree)
__device__ __forceinline__ bool ff_near(const FfBox& b, double X, double Y, double Z) {
  const double ex = fmax(fmax(b.lo[0] - X, X - b.hi[0]), 0.0);
  const double ey = fmax(fmax(b.lo[1] - Y, Y - b.hi[1]), 0.0);
  const double ez = fmax(fmax(b.lo[2] - Z, Z - b.hi[2]), 0.0);
  return fma(ex, ex, fma(ey, ey, ez * ez)) < b.d2;
}

// Near lists: per tile the indices of the nuclei near its box, in nucleus order (ordered
// compaction by warp ballots), and their count.  Block of 256 threads per tile.
__global__ void __launch_bounds__(256) k_ff_lists(const double* __restrict__ nuc, int nNuc, FfGeo f,
                                                  int* __restrict__ near_idx, int* __restrict__ near_cnt) {
  __shared__ int wc[8];
  const int t = blockIdx.x;
  const FfBox b = ff_box(f, t);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int cnt = 0;
  for (int base = 0; base < nNuc; base += 256) {
    const int m = base + threadIdx.x;
    const bool nr = m < nNuc && ff_near(b, nuc[m * 4], nuc[m * 4 + 1], nuc[m * 4 + 2]);
    const unsigned bal = __ballot_sync(0xffffffffu, nr);
    if (lane == 0) wc[warp] = __popc(bal);
    __syncthreads();
    int off = cnt + __popc(bal & ((1u << lane) - 1u)), tot = 0;
    for (int w = 0; w < 8; ++w) {
      if (w < warp) off += wc[w];
      tot += wc[w];
    }
    if (nr) near_idx[(long long)t * nNuc + off] = m;
    cnt += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) near_cnt[t] = cnt;
}

// Node values: V[t][qa][qb][qc] = sum over the far nuclei of Z / |node - R| in FP64.  Two blocks
// of 256 threads per tile (blockIdx.x = 2 t + half); thread (qa, qb) owns the 8 nodes qc of its
// half along z (8 accumulators keep the block at ~3 per SM).  Far nuclei of each chunk of 128 are
// compacted into shared memory first.
constexpr int kFfNh = kFfN / 2;
__global__ void __launch_bounds__(256) k_ff_nodes(const double* __restrict__ nuc, int nNuc, FfGeo f,
                                                  const double* __restrict__ tabs, double* __restrict__ Vn) {
  __shared__ double sf[128 * 4];
  __shared__ int wc[8];
  const int t = blockIdx.x >> 1, c0 = (blockIdx.x & 1) * kFfNh;
  const FfBox b = ff_box(f, t);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int qa = threadIdx.x >> 4, qb = threadIdx.x & 15;
  const double xa = b.c[0] + b.a[0] * tabs[qa], yb = b.c[1] + b.a[1] * tabs[qb];
  double zc[kFfNh], v[kFfNh];
#pragma unroll
  for (int q = 0; q < kFfNh; ++q) { zc[q] = b.c[2] + b.a[2] * tabs[c0 + q]; v[q] = 0.0; }
  for (int base = 0; base < nNuc; base += 128) {
    const int m = base + threadIdx.x;
    const bool far = threadIdx.x < 128 && m < nNuc && !ff_near(b, nuc[m * 4], nuc[m * 4 + 1], nuc[m * 4 + 2]);
    const unsigned bal = __ballot_sync(0xffffffffu, far);
    if (lane == 0) wc[warp] = __popc(bal);
    __syncthreads();
    int off = __popc(bal & ((1u << lane) - 1u)), nf = 0;
    for (int w = 0; w < 8; ++w) {
      if (w < warp) off += wc[w];
      nf += wc[w];
    }
    if (far) {
#pragma unroll
      for (int d = 0; d < 4; ++d) sf[off * 4 + d] = nuc[m * 4 + d];
    }
    __syncthreads();
    for (int q = 0; q < nf; ++q) {
      const double dx = xa - sf[q * 4], dy = yb - sf[q * 4 + 1], Z = sf[q * 4 + 2], Zn = sf[q * 4 + 3];
      const double dxy2 = fma(dx, dx, dy * dy);
#pragma unroll
      for (int c = 0; c < kFfNh; ++c) {
        const double dz = zc[c] - Z;
        v[c] = fma(Zn, rsqrt_refined(fma(dz, dz, dxy2)), v[c]);
      }
    }
    __syncthreads();
  }
  double* out = Vn + (long long)t * kFfN3 + (qa * kFfN + qb) * kFfN + c0;
#pragma unroll
  for (int c = 0; c < kFfNh; ++c) out[c] = v[c];
}

// Shared-memory Lagrange tables of one tile: Lx[p][q], Ly[p][q] (row per point) and Lz
// transposed, LzT[q][p] (a warp reading consecutive points p then hits consecutive words).
__device__ __forceinline__ void ff_load_tables(const double* __restrict__ tabs, const FfBox& b, double* Lx, double* Ly,
                                               double* LzT) {
  const double* tx = tabs + kFfN + (long long)b.m[0] * kFfT * kFfN;
  const double* ty = tabs + kFfN + (long long)b.m[1] * kFfT * kFfN;
  const double* tz = tabs + kFfN + (long long)b.m[2] * kFfT * kFfN;
  for (int q = threadIdx.x; q < kFfT * kFfN; q += blockDim.x) {
    Lx[q] = tx[q];
    Ly[q] = ty[q];
    const int p = q / kFfN, n = q % kFfN;
    LzT[n * kFfT + p] = tz[q];
  }
}

// Far part of K at every point of a tile: the tensor interpolation of the node values in three
// one-axis passes (z, then y, then x plane by plane), written to Kd (FP64).  One block of 256
// threads per tile; dynamic shared memory kFfInterpSmem bytes.
constexpr size_t kFfInterpSmem = sizeof(double) * (3 * kFfT * kFfN + kFfN * kFfN * kFfT + kFfN * kFfT * kFfT);

__global__ void __launch_bounds__(256) k_ff_interp(FfGeo f, const double* __restrict__ tabs,
                                                   const double* __restrict__ Vn, double* __restrict__ Kd, Geo g) {
  extern __shared__ double sm[];
  double* Lx = sm;
  double* Ly = Lx + kFfT * kFfN;
  double* LzT = Ly + kFfT * kFfN;
  double* A = LzT + kFfT * kFfN;          // [qa][qb][k]
  double* B = A + kFfN * kFfN * kFfT;     // [qa][j][k]
  double* V = B;                          // node values, read only before B is written
  const int t = blockIdx.x;
  const FfBox b = ff_box(f, t);
  const int mi = b.m[0], mj = b.m[1], mk = b.m[2];
  ff_load_tables(tabs, b, Lx, Ly, LzT);
  const double* vt = Vn + (long long)t * kFfN3;
  for (int q = threadIdx.x; q < kFfN3; q += blockDim.x) V[q] = vt[q];
  __syncthreads();
  for (int q = threadIdx.x; q < kFfN * kFfN * kFfT; q += blockDim.x) {
    const int ab = q / kFfT, k = q % kFfT;
    double s = 0.0;
    if (k < mk) {
#pragma unroll
      for (int c = 0; c < kFfN; ++c) s = fma(V[ab * kFfN + c], LzT[c * kFfT + k], s);
    }
    A[q] = s;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < kFfN * kFfT * kFfT; q += blockDim.x) {
    const int a = q / (kFfT * kFfT), j = (q / kFfT) % kFfT, k = q % kFfT;
    double s = 0.0;
    if (j < mj && k < mk) {
#pragma unroll
      for (int bq = 0; bq < kFfN; ++bq) s = fma(A[(a * kFfN + bq) * kFfT + k], Ly[j * kFfN + bq], s);
    }
    B[q] = s;
  }
  __syncthreads();
  for (int p = 0; p < mi; ++p) {
    const long long ip = (long long)(b.s[0] + p) * g.S2;
    for (int q = threadIdx.x; q < kFfT * kFfT; q += blockDim.x) {
      const int j = q / kFfT, k = q % kFfT;
      if (j >= mj || k >= mk) continue;
      double s = 0.0;
#pragma unroll
      for (int a = 0; a < kFfN; ++a) s = fma(Lx[p * kFfN + a], B[(a * kFfT + j) * kFfT + k], s);
      Kd[ip + (long long)(b.s[1] + j) * g.S + (b.s[2] + k)] = s;
    }
  }
}

// Near part of K and the final write: one block of 256 threads per (tile, plane); thread (jj, kk)
// owns the points (j0 + jj, k0 + kk + 8q), q = 0..3, of the plane.  Kd holds the far part on
// entry and the whole K (FP64) on exit; Kf (optional) receives it rounded to f32.
template <typename T>
__global__ void __launch_bounds__(256) k_ff_near_potential(FfGeo f, const double* __restrict__ nuc, int nNuc,
                                                           const int* __restrict__ near_idx,
                                                           const int* __restrict__ near_cnt, double sigma,
                                                           double* __restrict__ Kd, T* __restrict__ Kf, Geo g) {
  __shared__ double sn[256 * 4];
  const int t = blockIdx.x, p = blockIdx.y;
  const FfBox b = ff_box(f, t);
  if (p >= b.m[0]) return;  // uniform per block
  const int jj = threadIdx.x >> 3, kk = threadIdx.x & 7;
  const bool jin = jj < b.m[1];
  const int i = b.s[0] + p, j = b.s[1] + jj;
  const double x = i * f.h, y = j * f.h;
  double zq[4], acc[4];
  long long id[4];
  bool in[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int kl = kk + 8 * q;
    in[q] = jin && kl < b.m[2];
    const int k = b.s[2] + kl;
    zq[q] = k * f.h;
    id[q] = (long long)i * g.S2 + (long long)j * g.S + k;
    acc[q] = in[q] ? Kd[id[q]] : 0.0;
  }
  const double inv = 1.0 / (1.4142135623730951 * sigma), c0 = 0.7978845608028654 / sigma;
  const double rp2 = nm_point_r2(sigma);
  const int cnt = near_cnt[t];
  const int* lst = near_idx + (long long)t * nNuc;
  for (int base = 0; base < cnt; base += 256) {
    const int nb = min(256, cnt - base);
    __syncthreads();
    if (threadIdx.x < nb) {
      const int m = lst[base + threadIdx.x];
#pragma unroll
      for (int d = 0; d < 4; ++d) sn[threadIdx.x * 4 + d] = nuc[m * 4 + d];
    }
    __syncthreads();
    for (int m = 0; m < nb; ++m) {
      const double dx = x - sn[m * 4], dy = y - sn[m * 4 + 1], Z = sn[m * 4 + 2], Zn = sn[m * 4 + 3];
      const double c2 = fma(dx, dx, dy * dy);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const double dz = zq[q] - Z;
        const double r2 = fma(dz, dz, c2);
        if (r2 >= rp2) {
          acc[q] = fma(Zn, rsqrt_refined(r2), acc[q]);
        } else {
          const double r = sqrt(r2);
          acc[q] += (r < 1e-12) ? Zn * c0 : Zn * erf(r * inv) / r;
        }
      }
    }
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    if (!in[q]) continue;
    Kd[id[q]] = acc[q];
    if (Kf) Kf[id[q]] = (T)acc[q];
  }
}

// The weight of a grid point in a force gather: gw (dE/dK) when given, else the density u^2.
template <typename T>
__device__ __forceinline__ double ff_weight(const T* __restrict__ U, const double* __restrict__ gw, long long id) {
  if (gw) return gw[id];
  const double u = (double)U[id];
  return u * u;
}

// Anterpolation: W[t][qa][qb][qc] = sum over the tile's points of w(x) Lx[p][qa] Ly[j][qb] Lz[k][qc],
// plane by plane (z, then y, then x).  One block of 256 threads per tile; thread (qb, qc) keeps
// the 16 sums over qa in registers.
template <typename T>
__global__ void __launch_bounds__(256) k_ff_anterp(FfGeo f, const double* __restrict__ tabs, const T* __restrict__ U,
                                                   const double* __restrict__ gw, double* __restrict__ Wn, Geo g) {
  __shared__ double Lx[kFfT * kFfN], Ly[kFfT * kFfN], Lz[kFfT * kFfN];  // [p][q]: threads vary in q here
  __shared__ double w[kFfT * kFfT];
  __shared__ double C1[kFfT * kFfN];  // [j][qc]
  const int t = blockIdx.x;
  const FfBox b = ff_box(f, t);
  const int mi = b.m[0], mj = b.m[1], mk = b.m[2];
  for (int q = threadIdx.x; q < kFfT * kFfN; q += blockDim.x) {
    Lx[q] = tabs[kFfN + (long long)mi * kFfT * kFfN + q];
    Ly[q] = tabs[kFfN + (long long)mj * kFfT * kFfN + q];
    Lz[q] = tabs[kFfN + (long long)mk * kFfT * kFfN + q];
  }
  const int qb = threadIdx.x >> 4, qc = threadIdx.x & 15;
  double acc[kFfN];
#pragma unroll
  for (int a = 0; a < kFfN; ++a) acc[a] = 0.0;
  for (int p = 0; p < mi; ++p) {
    const long long ip = (long long)(b.s[0] + p) * g.S2;
    __syncthreads();
    for (int q = threadIdx.x; q < kFfT * kFfT; q += blockDim.x) {
      const int j = q / kFfT, k = q % kFfT;
      w[q] = (j < mj && k < mk) ? ff_weight<T>(U, gw, ip + (long long)(b.s[1] + j) * g.S + (b.s[2] + k)) : 0.0;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < kFfT * kFfN; q += blockDim.x) {
      const int j = q / kFfN, n = q % kFfN;
      double s = 0.0;
      for (int k = 0; k < mk; ++k) s = fma(w[j * kFfT + k], Lz[k * kFfN + n], s);
      C1[q] = s;
    }
    __syncthreads();
    double c2 = 0.0;
    for (int j = 0; j < mj; ++j) c2 = fma(C1[j * kFfN + qc], Ly[j * kFfN + qb], c2);
#pragma unroll
    for (int a = 0; a < kFfN; ++a) acc[a] = fma(Lx[p * kFfN + a], c2, acc[a]);
  }
  double* out = Wn + (long long)t * kFfN3;
#pragma unroll
  for (int a = 0; a < kFfN; ++a) out[(a * kFfN + qb) * kFfN + qc] = acc[a];
}

// Far force: thread = nucleus, block = 128 nuclei x a run of `tpb` tiles.  For each tile the
// nucleus is far from, it gathers sum_n W_n (x_n - R) / |x_n - R|^3 over the tile's nodes
// (its weights in shared memory).  Fraw accumulates sum w (dK/dr / (Z r)) (x - R), i.e. minus
// that sum; the caller's finish applies the per-nucleus factor.
__global__ void __launch_bounds__(128) k_ff_force_far(FfGeo f, int nTiles, int tpb, const double* __restrict__ tabs,
                                                      const double* __restrict__ nuc, int nNuc,
                                                      const double* __restrict__ Wn, double* __restrict__ Fraw) {
  __shared__ double W[kFfN3];
  __shared__ double xs[kFfN], ys[kFfN], zs[kFfN];
  const int n = blockIdx.y * blockDim.x + threadIdx.x;
  const bool valid = n < nNuc;
  const double X = valid ? nuc[n * 4] : 0.0, Y = valid ? nuc[n * 4 + 1] : 0.0, Z = valid ? nuc[n * 4 + 2] : 0.0;
  double fx = 0.0, fy = 0.0, fz = 0.0;
  const int t1 = min(nTiles, (blockIdx.x + 1) * tpb);
  for (int t = blockIdx.x * tpb; t < t1; ++t) {
    const FfBox b = ff_box(f, t);
    __syncthreads();
    const double* wt = Wn + (long long)t * kFfN3;
    for (int q = threadIdx.x; q < kFfN3; q += blockDim.x) W[q] = wt[q];
    if (threadIdx.x < kFfN) {
      xs[threadIdx.x] = b.c[0] + b.a[0] * tabs[threadIdx.x];
      ys[threadIdx.x] = b.c[1] + b.a[1] * tabs[threadIdx.x];
      zs[threadIdx.x] = b.c[2] + b.a[2] * tabs[threadIdx.x];
    }
    __syncthreads();
    if (!valid || ff_near(b, X, Y, Z)) continue;
    double gx = 0.0, gy = 0.0, gz = 0.0;
    for (int a = 0; a < kFfN; ++a) {
      const double dx = xs[a] - X;
      for (int bq = 0; bq < kFfN; ++bq) {
        const double dy = ys[bq] - Y;
        const double dxy2 = fma(dx, dx, dy * dy);
        const double* wr = W + (a * kFfN + bq) * kFfN;
        double s = 0.0, sz = 0.0;
#pragma unroll
        for (int c = 0; c < kFfN; ++c) {
          const double dz = zs[c] - Z;
          const double ir = rsqrt_refined(fma(dz, dz, dxy2));
          const double v = wr[c] * (ir * ir * ir);
          s += v;
          sz = fma(v, dz, sz);
        }
        gx = fma(s, dx, gx);
        gy = fma(s, dy, gy);
        gz += sz;
      }
    }
    fx -= gx; fy -= gy; fz -= gz;
  }
  if (valid) {
    atomicAdd(&Fraw[n * 3 + 0], fx);
    atomicAdd(&Fraw[n * 3 + 1], fy);
    atomicAdd(&Fraw[n * 3 + 2], fz);
  }
}

// Near force: thread = one of 64 near nuclei of a tile (chunk blockIdx.y of its near list); the
// tile's points are staged 256 at a time as FP64 (x, y, z, weight).  Exact Gaussian-nucleus
// terms, as the direct gather.
template <typename T>
__global__ void __launch_bounds__(64) k_ff_force_near(FfGeo f, const double* __restrict__ nuc, int nNuc,
                                                      const int* __restrict__ near_idx,
                                                      const int* __restrict__ near_cnt, const T* __restrict__ U,
                                                      const double* __restrict__ gw, double sigma,
                                                      double* __restrict__ Fraw, Geo g) {
  __shared__ double sx[256], sy[256], sz[256], sw[256];
  const int t = blockIdx.x;
  const int cnt = near_cnt[t];
  if (blockIdx.y * 64 >= cnt) return;  // uniform per block
  const FfBox b = ff_box(f, t);
  const int slot = blockIdx.y * 64 + threadIdx.x;
  const bool valid = slot < cnt;
  const int n = valid ? near_idx[(long long)t * nNuc + slot] : 0;
  const double X = valid ? nuc[n * 4] : 0.0, Y = valid ? nuc[n * 4 + 1] : 0.0, Z = valid ? nuc[n * 4 + 2] : 0.0;
  const double inv = 1.0 / (1.4142135623730951 * sigma), gs = 0.7978845608028654 / sigma;
  const double inv2 = inv * inv, rp2 = nm_point_r2(sigma);
  const int mj = b.m[1], mk = b.m[2];
  const long long npts = (long long)b.m[0] * mj * mk;
  double fx = 0.0, fy = 0.0, fz = 0.0;
  for (long long base = 0; base < npts; base += 256) {
    const int nb = (int)min(256LL, npts - base);
    __syncthreads();
    for (int q = threadIdx.x; q < nb; q += blockDim.x) {
      const long long v = base + q;
      const int p = (int)(v / (mj * mk)), j = (int)((v / mk) % mj), k = (int)(v % mk);
      const int i = b.s[0] + p, jg = b.s[1] + j, kg = b.s[2] + k;
      sx[q] = i * f.h; sy[q] = jg * f.h; sz[q] = kg * f.h;
      sw[q] = ff_weight<T>(U, gw, (long long)i * g.S2 + (long long)jg * g.S + kg);
    }
    __syncthreads();
    if (!valid) continue;
    double lx = 0.0, ly = 0.0, lz = 0.0;
    for (int q = 0; q < nb; ++q) {
      const double s = sw[q];
      const double dx = sx[q] - X, dy = sy[q] - Y, dz = sz[q] - Z;
      const double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
      double w;
      if (r2 >= rp2) {
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
  if (valid) {
    atomicAdd(&Fraw[n * 3 + 0], fx);
    atomicAdd(&Fraw[n * 3 + 1], fy);
    atomicAdd(&Fraw[n * 3 + 2], fz);
  }
}

// F[entry] += (weight scale x Z) Fraw[nucleus]: weight scale 1 for a dE/dK field, -h^3 for rho.
__global__ void k_ff_force_finish(const double* __restrict__ nuc, const int* __restrict__ entry, int nNuc,
                                  const double* __restrict__ Fraw, double wscale, double* __restrict__ F) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= nNuc) return;
  const double fac = wscale * nuc[n * 4 + 3];
  const int e = entry[n];
#pragma unroll
  for (int d = 0; d < 3; ++d) F[e * 3 + d] += fac * Fraw[n * 3 + d];
}

}  // namespace rq

// =========================================================================================
// host side
// =========================================================================================
using namespace rq;

#define CK(call)                                 \
  do {                                           \
    int _rc = rq_cuda(c, (call), #call);         \
    if (_rc != RQ_OK) return _rc;                \
  } while (0)

namespace {

// Chebyshev points tau_q = cos((2q + 1) pi / 32) and, for every tile size m, the Lagrange basis
// of those points at the tile's grid points t_p = -1 + 2p / (m - 1), in long double.
void ff_tables(std::vector<double>& t) {
  t.assign(kFfTabs, 0.0);
  const long double pi = 3.141592653589793238462643383279502884L;
  long double tau[kFfN];
  for (int q = 0; q < kFfN; ++q) {
    tau[q] = std::cos(pi * (2 * q + 1) / (2 * kFfN));
    t[q] = (double)tau[q];
  }
  for (int m = 2; m <= kFfT; ++m)
    for (int p = 0; p < m; ++p) {
      const long double tp = -1.0L + 2.0L * p / (m - 1);
      for (int q = 0; q < kFfN; ++q) {
        long double l = 1.0L;
        for (int r = 0; r < kFfN; ++r)
          if (r != q) l *= (tp - tau[r]) / (tau[q] - tau[r]);
        t[kFfN + ((size_t)m * kFfT + p) * kFfN + q] = (double)l;
      }
    }
}

template <class P>
int ff_alloc(rq_ctx* c, P*& ptr, size_t bytes) {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  return rq_cuda(c, cudaMalloc((void**)&ptr, bytes), "cudaMalloc (tiled nuclear sums)");
}

// Whether the tiles are used, and their layout: ceil(n1 / 32) tiles per axis of base or base + 1
// points.  Far nuclei must be point charges everywhere in a tile: 3 half-widths of the smallest
// tile reach past the Gaussian range (r / (sqrt2 sigma) >= 6).
bool ff_wanted(const rq_ctx* c, int nNuc, int& nt, int& base, int& rem) {
  const int mode = c->cfg.nuclear_sum, n1 = c->g.NN - 1;
  if (mode == 1 || nNuc < 1 || n1 < 32) return false;
  if (mode != 2 && (n1 < 64 || nNuc < 64)) return false;
  nt = (n1 + kFfT - 1) / kFfT;
  base = n1 / nt;
  rem = n1 % nt;
  const double reach = kFfFar * 0.5 * (base - 1) * c->h;
  return reach * reach >= 72.0 * c->sigma * c->sigma;
}

// the compact nuclei, the tiles' near lists (and the buffers, grown as needed)
int ff_plan(rq_ctx* c) {
  rq_ff& F = c->ff;
  std::vector<double> nuc;
  std::vector<int> ent;
  for (int q = 0; q < c->n_atoms; ++q) {
    const rq_atom& a = c->atoms[q];
    if (a.Z_nuc <= 0) continue;
    nuc.insert(nuc.end(), {a.i * c->h, a.j * c->h, a.k * c->h, a.Z_nuc});
    ent.push_back(q);
  }
  const int nNuc = (int)ent.size();
  int nt = 0, base = 0, rem = 0;
  F.active = ff_wanted(c, nNuc, nt, base, rem);
  if (!F.active) return RQ_OK;
  F.nt = nt; F.base = base; F.rem = rem; F.nTiles = nt * nt * nt; F.nNuc = nNuc;
  int rc;
  std::vector<double> tabs;
  if (!F.tabs) {
    ff_tables(tabs);
    if ((rc = ff_alloc(c, F.tabs, sizeof(double) * tabs.size())) != RQ_OK) return rc;
    CK(cudaMemcpyAsync(F.tabs, tabs.data(), sizeof(double) * tabs.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaFuncSetAttribute(k_ff_interp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFfInterpSmem));
  }
  if (nNuc > F.capNuc || F.nTiles > F.capTiles) {
    const int cn = std::max(nNuc, F.capNuc), ct = std::max(F.nTiles, F.capTiles);
    if ((rc = ff_alloc(c, F.nuc, sizeof(double) * 4 * cn)) != RQ_OK) return rc;
    if ((rc = ff_alloc(c, F.entry, sizeof(int) * cn)) != RQ_OK) return rc;
    if ((rc = ff_alloc(c, F.Fraw, sizeof(double) * 3 * cn)) != RQ_OK) return rc;
    if ((rc = ff_alloc(c, F.near_idx, sizeof(int) * (size_t)ct * cn)) != RQ_OK) return rc;
    if ((rc = ff_alloc(c, F.near_cnt, sizeof(int) * ct)) != RQ_OK) return rc;
    if ((rc = ff_alloc(c, F.nodes, sizeof(double) * (size_t)ct * kFfN3)) != RQ_OK) return rc;
    F.capNuc = cn; F.capTiles = ct;
  }
  CK(cudaMemcpyAsync(F.nuc, nuc.data(), sizeof(double) * nuc.size(), cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(F.entry, ent.data(), sizeof(int) * ent.size(), cudaMemcpyHostToDevice, c->st));
  const FfGeo f{F.nt, F.base, F.rem, c->h};
  LAUNCH(RQ_KC_OTHER, 32.0 * nNuc * F.nTiles,
         (k_ff_lists<<<F.nTiles, 256, 0, c->st>>>(F.nuc, nNuc, f, F.near_idx, F.near_cnt), cudaGetLastError()));
  CK(cudaStreamSynchronize(c->st));  // the host vectors above are copy sources
  return RQ_OK;
}

}  // namespace

int nm_nuclear_potential(rq_ctx* c, void* K, double* K64) {
  int rc = ff_plan(c);
  if (rc != RQ_OK) return rc;
  rq_ff& F = c->ff;
  const Geo& g = c->g;
  double* Kd = c->fp64 ? (double*)K : K64;
  if (!F.active || !Kd) {
    if (c->fp64)
      LAUNCH(RQ_KC_OTHER, 8.0 * g.S3, nm_potential<double>((double*)K, c->atoms_nm, c->n_atoms, g, c->h, c->sigma, c->st));
    else
      LAUNCH(RQ_KC_OTHER, (4.0 + (K64 ? 8.0 : 0.0)) * g.S3,
             nm_potential<float>((float*)K, c->atoms_nm, c->n_atoms, g, c->h, c->sigma, c->st, K64));
    return RQ_OK;
  }
  const FfGeo f{F.nt, F.base, F.rem, c->h};
  CK(cudaMemsetAsync(Kd, 0, sizeof(double) * g.S3, c->st));  // faces
  if (!c->fp64) CK(cudaMemsetAsync(K, 0, sizeof(float) * g.S3, c->st));
  LAUNCH(RQ_KC_OTHER, 8.0 * kFfN3 * F.nTiles,
         (k_ff_nodes<<<2 * F.nTiles, 256, 0, c->st>>>(F.nuc, F.nNuc, f, F.tabs, F.nodes), cudaGetLastError()));
  LAUNCH(RQ_KC_OTHER, 8.0 * g.S3,
         (k_ff_interp<<<F.nTiles, 256, kFfInterpSmem, c->st>>>(f, F.tabs, F.nodes, Kd, g), cudaGetLastError()));
  const dim3 grid(F.nTiles, kFfT);
  if (c->fp64)
    LAUNCH(RQ_KC_OTHER, 16.0 * g.S3,
           (k_ff_near_potential<double><<<grid, 256, 0, c->st>>>(f, F.nuc, F.nNuc, F.near_idx, F.near_cnt, c->sigma, Kd,
                                                                 nullptr, g),
            cudaGetLastError()));
  else
    LAUNCH(RQ_KC_OTHER, 20.0 * g.S3,
           (k_ff_near_potential<float><<<grid, 256, 0, c->st>>>(f, F.nuc, F.nNuc, F.near_idx, F.near_cnt, c->sigma, Kd,
                                                                (float*)K, g),
            cudaGetLastError()));
  return RQ_OK;
}

template <typename T>
static int gather_t(rq_ctx* c, const T* U, const double* gw) {
  rq_ff& F = c->ff;
  const Geo& g = c->g;
  const double n1 = g.NN - 1, ni = n1 * n1 * n1;
  if (!F.active) {
    LAUNCH(RQ_KC_FORCES, (gw ? 8.0 : sizeof(T)) * ni,
           nm_force<T>(U, c->atoms_nm, c->n_atoms, g, c->h, c->sigma, c->dF, c->st, gw));
    return RQ_OK;
  }
  const FfGeo f{F.nt, F.base, F.rem, c->h};
  CK(cudaMemsetAsync(F.Fraw, 0, sizeof(double) * 3 * F.nNuc, c->st));
  LAUNCH(RQ_KC_FORCES, (gw ? 8.0 : sizeof(T)) * ni,
         (k_ff_anterp<T><<<F.nTiles, 256, 0, c->st>>>(f, F.tabs, U, gw, F.nodes, g), cudaGetLastError()));
  const int tpb = 4;
  const dim3 gfar((F.nTiles + tpb - 1) / tpb, (F.nNuc + 127) / 128);
  LAUNCH(RQ_KC_FORCES, 8.0 * kFfN3 * F.nTiles,
         (k_ff_force_far<<<gfar, 128, 0, c->st>>>(f, F.nTiles, tpb, F.tabs, F.nuc, F.nNuc, F.nodes, F.Fraw),
          cudaGetLastError()));
  const dim3 gnear(F.nTiles, (F.nNuc + 63) / 64);
  LAUNCH(RQ_KC_FORCES, (gw ? 8.0 : sizeof(T)) * ni,
         (k_ff_force_near<T><<<gnear, 64, 0, c->st>>>(f, F.nuc, F.nNuc, F.near_idx, F.near_cnt, U, gw, c->sigma,
                                                      F.Fraw, g),
          cudaGetLastError()));
  LAUNCH(RQ_KC_FORCES, 48.0 * F.nNuc,
         (k_ff_force_finish<<<(F.nNuc + 127) / 128, 128, 0, c->st>>>(F.nuc, F.entry, F.nNuc, F.Fraw,
                                                                      gw ? 1.0 : -(c->h * c->h * c->h), c->dF),
          cudaGetLastError()));
  return RQ_OK;
}

int nm_gather(rq_ctx* c, const void* U, const double* gw) {
  return c->fp64 ? gather_t<double>(c, (const double*)U, gw) : gather_t<float>(c, (const float*)U, gw);
}

void nm_ff_free(rq_ctx* c) {
  rq_ff& F = c->ff;
  for (void* p : {(void*)F.nuc, (void*)F.entry, (void*)F.near_idx, (void*)F.near_cnt, (void*)F.nodes, (void*)F.tabs,
                  (void*)F.Fraw})
    if (p) cudaFree(p);
  F = rq_ff{};
}
