// nm_kernels.cu -- kernels of the new flavour: Gaussian-smoothed nuclei, red-black
// Gauss-Seidel multigrid for the Hartree half-potential, FP64 per-domain sums, and the
// Hellmann-Feynman / stationary-point gradient with respect to the nuclear centres.
//
// Every kernel is templated on the field type T: float for the mixed path (fp32 fields and
// stencils, FP64 reductions and an FP64 coarsest solve) and double for the plain FP64 path.
// Point-wise arithmetic is explicitly rounded (no FMA contraction) and follows the operation
// order of the FP64 oracle (oracle/rq_oracle.c, orc_nm_*), so the FP64 path reproduces it up
// to the order of the per-domain sums.
#include "rq_kernels.h"

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

// ---------------------------------------------------------------------------------------
// nuclear potential of Gaussian nuclei (width sigma): K = sum Z erf(r/(sqrt2 sigma))/r, FP64
// atoms_nm: (x, y, z in bohr from grid point (0,0,0), Z_nuc) per entry; entries with Z_nuc <= 0
// carry no nucleus.  Boundary planes are 0.
// ---------------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_nm_potential(T* __restrict__ K, const double* __restrict__ at, int nAt, Geo g,
                                                      double h, double sigma) {
  __shared__ double sa[128 * 4];
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool inside = id < g.S3;
  int i = 0, j = 0, k = 0;
  if (inside) { i = (int)(id / g.S2); j = (int)((id / g.S) % g.S); k = (int)(id % g.S); }
  const bool interior = inside && i >= 1 && i < g.NN && j >= 1 && j < g.NN && k >= 1 && k < g.NN;
  const double x = i * h, y = j * h, z = k * h;
  const double inv = 1.0 / (1.4142135623730951 * sigma), c0 = 0.7978845608028654 / sigma;  // sqrt(2/pi)
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
      const double r = sqrt(dx * dx + dy * dy + dz * dz);
      v += (r < 1e-12) ? Z * c0 : Z * erf(r * inv) / r;
    }
  }
  if (inside) K[id] = interior ? (T)v : T(0);
}

// ---------------------------------------------------------------------------------------
// initial state: label = nearest domain seed (f32 squared distances, first index wins ties),
// psi = exp(-|x - seed|).  seeds: (x, y, z, entry index) for every entry with Z > 0.
// ---------------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_nm_init(T* __restrict__ U, int* __restrict__ label,
                                                 const float4* __restrict__ seeds, int nSeed, Geo g, float h) {
  __shared__ float4 ss[256];
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
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

// ---------------------------------------------------------------------------------------
// ITP update (same-label Neumann Laplacian), FP64 domain norms of the new psi with ACC.
// ---------------------------------------------------------------------------------------
template <typename T, bool ACC>
__global__ void __launch_bounds__(256) k_nm_update(const T* __restrict__ U, T* __restrict__ Unew,
                                                   const T* __restrict__ K, const T* __restrict__ P,
                                                   const int* __restrict__ label, Geo g, T half_dv, T dt, double h3,
                                                   int nDom, double* __restrict__ norms) {
  using A = Ar<T>;
  __shared__ DomTable<1, 128> tab;
  if (ACC) dom_table_init(tab);
  if (ACC) __syncthreads();
  RunSum<1> rs;
  rs.reset();
  const int k = 1 + blockIdx.x * kThreadsK + threadIdx.x;
  const int j = 1 + blockIdx.y * kThreadsJ + threadIdx.y;
  const int i0 = 1 + blockIdx.z * kMarch;
  if (k < g.NN && j < g.NN && i0 < g.NN) {
    const int iend = min(i0 + kMarch, g.NN);
    const long long S = g.S, S2 = g.S2;
    long long id = (long long)i0 * S2 + j * S + k;
    T u_m = U[id - S2], u_c = U[id];
    int l_m = label[id - S2], l_c = label[id];
    for (int i = i0; i < iend; ++i, id += S2) {
      const T u_p = U[id + S2];
      const int l_p = label[id + S2];
      const T a = (l_p == l_c) ? u_p : u_c;
      const T b = (l_m == l_c) ? u_m : u_c;
      const T c = (label[id + S] == l_c) ? U[id + S] : u_c;
      const T d = (label[id - S] == l_c) ? U[id - S] : u_c;
      const T e = (label[id + 1] == l_c) ? U[id + 1] : u_c;
      const T f = (label[id - 1] == l_c) ? U[id - 1] : u_c;
      const T lap = A::sub(A::add(A::add(A::add(A::add(A::add(a, b), c), d), e), f), A::mul(T(6), u_c));
      const T out = A::add(A::add(u_c, A::mul(half_dv, lap)), A::mul(A::mul(dt, A::sub(K[id], A::mul(T(2), P[id]))), u_c));
      Unew[id] = out;
      if (ACC) {
        const double r = (double)out * (double)out * h3;
        rs.add(min(max(l_c, 0), nDom - 1), &r, tab, norms);
      }
      u_m = u_c; u_c = u_p; l_m = l_c; l_c = l_p;
    }
  }
  if (ACC) {
    rs.finish(tab, norms);
    __syncthreads();
    dom_table_flush(tab, norms);
  }
}

template <typename T>
__global__ void k_nm_norm_scale(const double* __restrict__ norms, const double* __restrict__ Zdom, int nDom,
                                T* __restrict__ scale, int* __restrict__ err) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= nDom) return;
  const double n = norms[l];
  if (!isfinite(n)) atomicOr(err, 1);
  scale[l] = (Zdom[l] > 0.0 && n > 1e-300) ? (T)sqrt(Zdom[l] / n) : T(1);
}

template <typename T>
__global__ void __launch_bounds__(256) k_nm_apply_scale(T* __restrict__ U, const int* __restrict__ label,
                                                        const T* __restrict__ scale, long long S3, int nDom) {
  for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < S3; id += (long long)gridDim.x * blockDim.x) {
    const int l = label[id];
    if (l < 0 || l >= nDom) continue;
    U[id] = Ar<T>::mul(U[id], scale[l]);
  }
}

// FP64 per-label norms of psi over all S^3 points (label clipped to [0, nDom))
template <typename T>
__global__ void __launch_bounds__(256) k_nm_norms(const T* __restrict__ U, const int* __restrict__ label, long long S3,
                                                  double h3, int nDom, double* __restrict__ norms) {
  __shared__ DomTable<1, 128> tab;
  dom_table_init(tab);
  __syncthreads();
  RunSum<1> rs;
  rs.reset();
  const long long base = (long long)blockIdx.x * blockDim.x * 16;
  for (int q = 0; q < 16; ++q) {
    const long long id = base + (long long)q * blockDim.x + threadIdx.x;
    if (id >= S3) break;
    const double u = (double)U[id];
    const double r = u * u * h3;
    rs.add(min(max(label[id], 0), nDom - 1), &r, tab, norms);
  }
  rs.finish(tab, norms);
  __syncthreads();
  dom_table_flush(tab, norms);
}

// ---------------------------------------------------------------------------------------
// multigrid for A P = f,  A P = (6 P - sum_6 P)/h^2,  f = 2 pi psi^2 on the fine level.
// FINE kernels read psi and form f = (2 pi psi) psi on the fly instead of storing it.
// ---------------------------------------------------------------------------------------
template <typename T, bool FINE>
__device__ __forceinline__ T rhs_at(const T* __restrict__ f, long long id) {
  if (FINE) {
    const T u = f[id];
    return Ar<T>::mul(Ar<T>::mul((T)6.283185307179586, u), u);
  }
  return f[id];
}

// one colour of a red-black Gauss-Seidel sweep: points with (i+j+k)%2 == color
template <typename T, bool FINE>
__global__ void __launch_bounds__(256) k_nm_rbgs(T* __restrict__ P, const T* __restrict__ f, Geo g, T h2, int color) {
  using A = Ar<T>;
  const int k0 = 1 + blockIdx.x * 64 + 2 * threadIdx.x;  // candidates k0, k0+1: one of them has the colour
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  const int i = 1 + blockIdx.z;
  if (j >= g.NN || i >= g.NN) return;
  const int k = k0 + ((i + j + k0 + color) & 1);
  if (k >= g.NN) return;
  const long long S = g.S, S2 = g.S2;
  const long long id = (long long)i * S2 + (long long)j * S + k;
  const T s = A::add(A::add(A::add(A::add(A::add(P[id + S2], P[id - S2]), P[id + S]), P[id - S]), P[id + 1]), P[id - 1]);
  P[id] = A::div(A::add(s, A::mul(h2, rhs_at<T, FINE>(f, id))), T(6));
}

template <typename T, bool FINE>
__global__ void __launch_bounds__(256) k_nm_residual(const T* __restrict__ P, const T* __restrict__ f,
                                                     T* __restrict__ r, Geo g, T inv_h2) {
  using A = Ar<T>;
  const int k = 1 + blockIdx.x * kThreadsK + threadIdx.x;
  const int j = 1 + blockIdx.y * kThreadsJ + threadIdx.y;
  const int i0 = 1 + blockIdx.z * kMarch;
  if (k >= g.NN || j >= g.NN || i0 >= g.NN) return;
  const int iend = min(i0 + kMarch, g.NN);
  const long long S = g.S, S2 = g.S2;
  for (int i = i0; i < iend; ++i) {
    const long long id = (long long)i * S2 + (long long)j * S + k;
    const T s = A::add(A::add(A::add(A::add(A::add(P[id + S2], P[id - S2]), P[id + S]), P[id - S]), P[id + 1]), P[id - 1]);
    r[id] = A::add(rhs_at<T, FINE>(f, id), A::mul(A::sub(s, A::mul(T(6), P[id])), inv_h2));
  }
}

// full weighting (1/64)(8,4,2,1) onto the coarse interior; loop order a, b, c as the oracle
template <typename T>
__global__ void __launch_bounds__(256) k_nm_restrict(const T* __restrict__ fine, T* __restrict__ coarse, Geo g, Geo gc) {
  using A = Ar<T>;
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
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

// trilinear prolongation of the coarse correction, added to the fine level
template <typename T>
__global__ void __launch_bounds__(256) k_nm_prolong(const T* __restrict__ Ec, T* __restrict__ P, Geo g, Geo gc) {
  using A = Ar<T>;
  const int k = 1 + blockIdx.x * kThreadsK + threadIdx.x;
  const int j = 1 + blockIdx.y * kThreadsJ + threadIdx.y;
  const int i0 = 1 + blockIdx.z * kMarch;
  if (k >= g.NN || j >= g.NN || i0 >= g.NN) return;
  const int iend = min(i0 + kMarch, g.NN);
  for (int i = i0; i < iend; ++i) {
    const int ci = i >> 1, cj = j >> 1, ck = k >> 1, oi = i & 1, oj = j & 1, ok = k & 1;
    T v = T(0);
    for (int a = 0; a <= oi; ++a)
      for (int b = 0; b <= oj; ++b)
        for (int c = 0; c <= ok; ++c) v = A::add(v, Ec[(long long)(ci + a) * gc.S2 + (long long)(cj + b) * gc.S + (ck + c)]);
    v = A::div(v, (T)((1 + oi) * (1 + oj) * (1 + ok)));
    const long long id = (long long)i * g.S2 + (long long)j * g.S + k;
    P[id] = A::add(P[id], v);
  }
}

// coarsest level: `sweeps` red-black sweeps in FP64 inside one block (the level fits in shared memory)
template <typename T>
__global__ void __launch_bounds__(1024) k_nm_coarsest(T* __restrict__ P, const T* __restrict__ f, Geo g, double h2,
                                                      int sweeps) {
  extern __shared__ double sm[];
  double* sP = sm;
  double* sf = sm + g.S3;
  for (long long q = threadIdx.x; q < g.S3; q += blockDim.x) { sP[q] = (double)P[q]; sf[q] = (double)f[q]; }
  __syncthreads();
  const int n = g.NN - 1;
  const long long nint = (long long)n * n * n;
  for (int s = 0; s < sweeps; ++s)
    for (int color = 0; color < 2; ++color) {
      for (long long q = threadIdx.x; q < nint; q += blockDim.x) {
        const int k = 1 + (int)(q % n), j = 1 + (int)((q / n) % n), i = 1 + (int)(q / ((long long)n * n));
        if (((i + j + k) & 1) != color) continue;
        const long long id = (long long)i * g.S2 + (long long)j * g.S + k;
        const double sum = __dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(sP[id + g.S2], sP[id - g.S2]), sP[id + g.S]),
                                                        sP[id - g.S]), sP[id + 1]), sP[id - 1]);
        sP[id] = __ddiv_rn(__dadd_rn(sum, __dmul_rn(h2, sf[id])), 6.0);
      }
      __syncthreads();
    }
  for (long long q = threadIdx.x; q < g.S3; q += blockDim.x) P[q] = (T)sP[q];
}

// ---------------------------------------------------------------------------------------
// energies per domain: (norm, T, V_eK, V_ee) in FP64
// ---------------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_nm_energy(const T* __restrict__ U, const T* __restrict__ K,
                                                   const T* __restrict__ P, const int* __restrict__ label, Geo g,
                                                   double h, int nDom, double* __restrict__ pd) {
  __shared__ DomTable<4, 128> tab;
  dom_table_init(tab);
  __syncthreads();
  RunSum<4> rs;
  rs.reset();
  const double h3 = h * h * h;
  const int k = 1 + blockIdx.x * kThreadsK + threadIdx.x;
  const int j = 1 + blockIdx.y * kThreadsJ + threadIdx.y;
  const int i0 = 1 + blockIdx.z * kMarch;
  if (k < g.NN && j < g.NN && i0 < g.NN) {
    const int iend = min(i0 + kMarch, g.NN);
    const long long S = g.S, S2 = g.S2;
    for (int i = i0; i < iend; ++i) {
      const long long id = (long long)i * S2 + j * S + k;
      const double u = U[id], rho = u * u;
      const int L = label[id];
      if (L < 0 || L >= nDom) continue;
      const double a = (label[id + S2] == L) ? (double)U[id + S2] - u : 0.0;
      const double b = (label[id + S] == L) ? (double)U[id + S] - u : 0.0;
      const double c = (label[id + 1] == L) ? (double)U[id + 1] - u : 0.0;
      // every same-label edge with an interior end point is counted once: the forward edges
      // above plus, on the first interior layer, the edge to the Dirichlet face below, so that
      // T is exactly the quadratic form whose gradient is the update's Laplacian
      double t = a * a + b * b + c * c;
      if (i == 1 && label[id - S2] == L) t += u * u;
      if (j == 1 && label[id - S] == L) t += u * u;
      if (k == 1 && label[id - 1] == L) t += u * u;
      double v[4] = {rho * h3, 0.5 * t * h, -(double)K[id] * rho * h3, (double)P[id] * rho * h3};
      rs.add(L, v, tab, pd);
    }
  }
  rs.finish(tab, pd);
  __syncthreads();
  dom_table_flush(tab, pd);
}

// ---------------------------------------------------------------------------------------
// level-set label update (the molecule.js rule, molecule.js:426-540) on psi of type T
// ---------------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_nm_evolve(const int* __restrict__ labIn, int* __restrict__ labOut,
                                                   const T* __restrict__ U, float* __restrict__ W, Geo g, T dt_w,
                                                   T curvReg) {
  using A = Ar<T>;
  const int k = 1 + blockIdx.x * kThreadsK + threadIdx.x;
  const int j = 1 + blockIdx.y * kThreadsJ + threadIdx.y;
  const int i0 = 1 + blockIdx.z * kMarch;
  if (k >= g.NN || j >= g.NN || i0 >= g.NN) return;
  const int iend = min(i0 + kMarch, g.NN);
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

// ---------------------------------------------------------------------------------------
// Force on each nucleus from the electron density with Gaussian nuclei:
// F_a = -h^3 sum_x rho(x) dK_a/dr (x - R_a)/r,  dK/dr = Z (g e^{-r^2/(2 s^2)}/r - erf(r/(sqrt2 s))/r^2)
// (g = sqrt(2/pi)/s).  At a stationary psi (converged, labels frozen) this is minus the exact
// gradient of the discrete energy's electron-nuclear term.  Tiles of interior points are
// staged in shared memory; one thread per nucleus; FP64 accumulation.
// ---------------------------------------------------------------------------------------
constexpr int kNmForceTile = 512;
template <typename T>
__global__ void __launch_bounds__(256) k_nm_force(const T* __restrict__ U, const double* __restrict__ at, int nAt,
                                                  Geo g, double h, double sigma, double* __restrict__ F) {
  // tile staged in the field type: FP64 for the plain path, fp32 for the mixed path
  __shared__ T sx[kNmForceTile], sy[kNmForceTile], sz[kNmForceTile], sr[kNmForceTile];
  const int a = blockIdx.y * blockDim.x + threadIdx.x;
  const bool valid = a < nAt && at[a * 4 + 3] > 0.0;
  const double Z = valid ? at[a * 4 + 3] : 0.0;
  const double ax = valid ? at[a * 4 + 0] : 0.0, ay = valid ? at[a * 4 + 1] : 0.0, az = valid ? at[a * 4 + 2] : 0.0;
  const double inv = 1.0 / (1.4142135623730951 * sigma), gs = 0.7978845608028654 / sigma;
  const double h3 = h * h * h;
  const long long n1 = g.NN - 1, nInt = n1 * n1 * n1;
  const long long ntiles = (nInt + kNmForceTile - 1) / kNmForceTile;
  double fx = 0, fy = 0, fz = 0;
  for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
    __syncthreads();
    for (int q = threadIdx.x; q < kNmForceTile; q += blockDim.x) {
      const long long v = t * kNmForceTile + q;
      T rho = T(0), x = T(0), y = T(0), z = T(0);
      if (v < nInt) {
        const int i = 1 + (int)(v / (n1 * n1)), j = 1 + (int)((v / n1) % n1), k = 1 + (int)(v % n1);
        const double u = (double)U[(long long)i * g.S2 + (long long)j * g.S + k];
        rho = (T)(u * u);
        x = (T)(i * h); y = (T)(j * h); z = (T)(k * h);
      }
      sx[q] = x; sy[q] = y; sz[q] = z; sr[q] = rho;
    }
    __syncthreads();
    if (valid) {
      double lx = 0, ly = 0, lz = 0;
      for (int q = 0; q < kNmForceTile; ++q) {
        const double rho = sr[q];
        if (rho == 0.0) continue;
        const double dx = (double)sx[q] - ax, dy = (double)sy[q] - ay, dz = (double)sz[q] - az;
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (r2 < 1e-24) continue;
        const double r = sqrt(r2);
        double dKdr;
        if (r * inv < 6.0)
          dKdr = Z * (gs * exp(-r2 * inv * inv) / r - erf(r * inv) / r2);
        else
          dKdr = -Z / r2;
        const double w = -h3 * rho * dKdr / r;
        lx += w * dx; ly += w * dy; lz += w * dz;
      }
      fx += lx; fy += ly; fz += lz;
    }
  }
  if (valid) {
    atomicAdd(&F[a * 3 + 0], fx);
    atomicAdd(&F[a * 3 + 1], fy);
    atomicAdd(&F[a * 3 + 2], fz);
  }
}

template <typename T>
__global__ void k_nm_add(T* __restrict__ K, const T* __restrict__ v, long long n) {
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    K[q] = Ar<T>::add(K[q], v[q]);
}

// ======================================================================================
// host launchers (T = float or double)
// ======================================================================================
static unsigned nblk(long long n, int b = 256) { return (unsigned)((n + b - 1) / b); }

template <typename T>
cudaError_t nm_potential(T* K, const double* at, int nAt, const Geo& g, double h, double sigma, cudaStream_t st) {
  k_nm_potential<T><<<nblk(g.S3), 256, 0, st>>>(K, at, nAt, g, h, sigma);
  return cudaGetLastError();
}
template <typename T>
cudaError_t nm_init(T* U, int* label, const float4* seeds, int nSeed, const Geo& g, float h, cudaStream_t st) {
  k_nm_init<T><<<nblk(g.S3), 256, 0, st>>>(U, label, seeds, nSeed, g, h);
  return cudaGetLastError();
}
template <typename T>
cudaError_t nm_update(const T* U, T* Unew, const T* K, const T* P, const int* label, const Geo& g, T half_dv, T dt,
                      double h3, int nDom, double* norms, cudaStream_t st) {
  if (g.NN < 2) return cudaSuccess;
  if (norms)
    k_nm_update<T, true><<<march_grid(g), march_block(), 0, st>>>(U, Unew, K, P, label, g, half_dv, dt, h3, nDom, norms);
  else
    k_nm_update<T, false><<<march_grid(g), march_block(), 0, st>>>(U, Unew, K, P, label, g, half_dv, dt, h3, nDom,
                                                                    nullptr);
  return cudaGetLastError();
}
template <typename T>
cudaError_t nm_normalize(T* U, const int* label, const double* norms, const double* Zdom, int nDom, T* scale, int* err,
                         const Geo& g, cudaStream_t st) {
  k_nm_norm_scale<T><<<nblk(nDom, 128), 128, 0, st>>>(norms, Zdom, nDom, scale, err);
  long long b = nblk(g.S3);
  if (b > 148 * 16) b = 148 * 16;
  k_nm_apply_scale<T><<<(unsigned)b, 256, 0, st>>>(U, label, scale, g.S3, nDom);
  return cudaGetLastError();
}
template <typename T>
cudaError_t nm_norms(const T* U, const int* label, const Geo& g, double h3, int nDom, double* norms, cudaStream_t st) {
  k_nm_norms<T><<<nblk(g.S3, 256 * 16), 256, 0, st>>>(U, label, g.S3, h3, nDom, norms);
  return cudaGetLastError();
}
template <typename T>
cudaError_t nm_rbgs(T* P, const T* f, bool fine, const Geo& g, double h2, int color, cudaStream_t st) {
  const int n = g.NN - 1;
  const dim3 blk(32, 8);
  const dim3 grd((n + 63) / 64, (n + 7) / 8, n);
  if (fine)
    k_nm_rbgs<T, true><<<grd, blk, 0, st>>>(P, f, g, (T)h2, color);
  else
    k_nm_rbgs<T, false><<<grd, blk, 0, st>>>(P, f, g, (T)h2, color);
  return cudaGetLastError();
}
template <typename T>
cudaError_t nm_residual(const T* P, const T* f, bool fine, T* r, const Geo& g, double inv_h2, cudaStream_t st) {
  if (fine)
    k_nm_residual<T, true><<<march_grid(g), march_block(), 0, st>>>(P, f, r, g, (T)inv_h2);
  else
    k_nm_residual<T, false><<<march_grid(g), march_block(), 0, st>>>(P, f, r, g, (T)inv_h2);
  return cudaGetLastError();
}
template <typename T>
cudaError_t nm_restrict(const T* fine, T* coarse, const Geo& g, const Geo& gc, cudaStream_t st) {
  const long long n = gc.NN - 1;
  k_nm_restrict<T><<<nblk(n * n * n), 256, 0, st>>>(fine, coarse, g, gc);
  return cudaGetLastError();
}
template <typename T>
cudaError_t nm_prolong(const T* Ec, T* P, const Geo& g, const Geo& gc, cudaStream_t st) {
  k_nm_prolong<T><<<march_grid(g), march_block(), 0, st>>>(Ec, P, g, gc);
  return cudaGetLastError();
}
template <typename T>
cudaError_t nm_coarsest(T* P, const T* f, const Geo& g, double h2, int sweeps, cudaStream_t st) {
  const size_t smem = sizeof(double) * 2 * (size_t)g.S3;
  if (smem > 200 * 1024) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(k_nm_coarsest<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_nm_coarsest<T><<<1, 1024, smem, st>>>(P, f, g, h2, sweeps);
  return cudaGetLastError();
}
template <typename T>
cudaError_t nm_energy(const T* U, const T* K, const T* P, const int* label, const Geo& g, double h, int nDom, double* pd,
                      cudaStream_t st) {
  if (g.NN < 2) return cudaSuccess;
  k_nm_energy<T><<<march_grid(g), march_block(), 0, st>>>(U, K, P, label, g, h, nDom, pd);
  return cudaGetLastError();
}
template <typename T>
cudaError_t nm_evolve(const int* labIn, int* labOut, const T* U, float* W, const Geo& g, double dt_w, double curvReg,
                      cudaStream_t st) {
  if (g.NN < 2) return cudaSuccess;
  k_nm_evolve<T><<<march_grid(g), march_block(), 0, st>>>(labIn, labOut, U, W, g, (T)(float)dt_w, (T)(float)curvReg);
  return cudaGetLastError();
}
template <typename T>
cudaError_t nm_force(const T* U, const double* at, int nAt, const Geo& g, double h, double sigma, double* F,
                     cudaStream_t st) {
  if (g.NN < 2 || nAt <= 0) return cudaSuccess;
  const long long n1 = g.NN - 1, nInt = n1 * n1 * n1;
  const long long ntiles = (nInt + kNmForceTile - 1) / kNmForceTile;
  const int chunks = (nAt + 255) / 256;
  long long bx = 148 * 8 / chunks;
  if (bx < 1) bx = 1;
  if (bx > ntiles) bx = ntiles;
  k_nm_force<T><<<dim3((unsigned)bx, (unsigned)chunks), 256, 0, st>>>(U, at, nAt, g, h, sigma, F);
  return cudaGetLastError();
}

template <typename T>
cudaError_t nm_add(T* K, const T* v, long long n, cudaStream_t st) {
  k_nm_add<T><<<148 * 8, 256, 0, st>>>(K, v, n);
  return cudaGetLastError();
}

#define RQ_NM_INSTANTIATE(T)                                                                                          \
  template cudaError_t nm_add<T>(T*, const T*, long long, cudaStream_t);                                           \
  RQ_NM_INSTANTIATE2(T)
#define RQ_NM_INSTANTIATE2(T)                                                                                          \
  template cudaError_t nm_potential<T>(T*, const double*, int, const Geo&, double, double, cudaStream_t);           \
  template cudaError_t nm_init<T>(T*, int*, const float4*, int, const Geo&, float, cudaStream_t);                   \
  template cudaError_t nm_update<T>(const T*, T*, const T*, const T*, const int*, const Geo&, T, T, double, int,     \
                                    double*, cudaStream_t);                                                          \
  template cudaError_t nm_normalize<T>(T*, const int*, const double*, const double*, int, T*, int*, const Geo&,     \
                                       cudaStream_t);                                                                \
  template cudaError_t nm_rbgs<T>(T*, const T*, bool, const Geo&, double, int, cudaStream_t);                       \
  template cudaError_t nm_norms<T>(const T*, const int*, const Geo&, double, int, double*, cudaStream_t);           \
  template cudaError_t nm_residual<T>(const T*, const T*, bool, T*, const Geo&, double, cudaStream_t);              \
  template cudaError_t nm_restrict<T>(const T*, T*, const Geo&, const Geo&, cudaStream_t);                          \
  template cudaError_t nm_prolong<T>(const T*, T*, const Geo&, const Geo&, cudaStream_t);                           \
  template cudaError_t nm_coarsest<T>(T*, const T*, const Geo&, double, int, cudaStream_t);                         \
  template cudaError_t nm_energy<T>(const T*, const T*, const T*, const int*, const Geo&, double, int, double*,     \
                                    cudaStream_t);                                                                   \
  template cudaError_t nm_evolve<T>(const int*, int*, const T*, float*, const Geo&, double, double, cudaStream_t);  \
  template cudaError_t nm_force<T>(const T*, const double*, int, const Geo&, double, double, double*, cudaStream_t);
RQ_NM_INSTANTIATE(float)
RQ_NM_INSTANTIATE(double)

}  // namespace rq
