// nm_kernels.cu -- single-grid kernels of the new flavour: Gaussian-smoothed nuclei, red-black
// Gauss-Seidel multigrid for the Hartree half-potential, FP64 per-domain sums, and the
// stationary-point gradient with respect to the nuclear centres.  The point-wise code lives
// in nm_bodies.cuh (shared with the batched kernels); here each body gets its block
// coordinates from blockIdx.  T = float (mixed path) or double (FP64 path).
#include <type_traits>

#include "nm_bodies.cuh"
#include "rq_kernels.h"

namespace rq {

template <typename T>
__global__ void __launch_bounds__(256) k_nm_potential(T* K, const double* at, int nAt, Geo g, double h, double sigma,
                                                      double* K64) {
  __shared__ double sa[128 * 4];
  nm_potential_body<T>(K, at, nAt, g, h, sigma, blockIdx.x, sa, K64);
}

template <typename T>
__global__ void __launch_bounds__(256) k_nm_init(T* U, int* label, const float4* seeds, int nSeed, Geo g, float h) {
  __shared__ float4 ss[256];
  nm_init_body<T>(U, label, seeds, nSeed, g, h, blockIdx.x, ss);
}

// seed[0]: the step seed of the unbiased fp32 rounding (null: round to nearest); the next step's
// seed, seed[0] + 1, goes to seed_next (read and written in different words, so every block reads
// the same value)
__global__ void __launch_bounds__(256) k_nm_mask(const int* __restrict__ label, unsigned char* __restrict__ mask, Geo g) {
  nm_mask_body(label, mask, g, blockIdx.x);
}

// mask: the same-label neighbour mask of `label` (null: the six neighbour labels are read)
template <typename T, bool ACC, bool SR, bool MASK>
__global__ void __launch_bounds__(256) k_nm_update(const T* U, T* Unew, const T* K, const T* P, const int* label, Geo g,
                                                   T half_dv, T dt, double h3, int nDom, double* norms, const double* scale,
                                                   const unsigned* seed, unsigned* seed_next,
                                                   const unsigned char* __restrict__ mask) {
  __shared__ DomTable<1, 128> tab;
  if (SR && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0 && threadIdx.y == 0)
    *seed_next = *seed + 1u;
  if (ACC) {
    dom_table_init(tab);
    __syncthreads();
  }
  nm_update_body<T, ACC, MASK, SR>(U, Unew, K, P, label, g, half_dv, dt, h3, nDom, norms, tab, blockIdx.x, blockIdx.y,
                                   blockIdx.z, scale, seed, kNmTile, mask);
  if (ACC) {
    __syncthreads();
    dom_table_flush(tab, norms);
  }
}

// scale[l] = sqrt(Zdom_l / n_l) (FP64) for every domain of the (concatenated) arrays; a norm
// that is NaN or Inf sets bit 0 of *err and leaves its domain unscaled
template <typename T>
__global__ void k_nm_norm_scale(const double* __restrict__ norms, const double* __restrict__ Zdom, int nDom,
                                double* __restrict__ scale, int* __restrict__ err) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l < nDom) scale[l] = nm_domain_scale(norms[l], Zdom[l], err);
}

template <typename T>
__global__ void __launch_bounds__(256) k_nm_apply_scale(T* U, const int* label, const double* scale, long long S3, int nDom) {
  nm_apply_scale_body<T>(U, label, scale, S3, nDom, blockIdx.x);
}

template <typename T>
__global__ void __launch_bounds__(256) k_nm_norms(const T* U, const int* label, long long S3, double h3, int nDom,
                                                  double* norms) {
  __shared__ DomTable<1, 128> tab;
  dom_table_init(tab);
  __syncthreads();
  nm_norms_body<T>(U, label, S3, h3, nDom, norms, tab, blockIdx.x);
  __syncthreads();
  dom_table_flush(tab, norms);
}

template <typename T, bool FINE>
__global__ void __launch_bounds__(256) k_nm_rbgs(T* P, const T* f, Geo g, T h2, int color) {
  nm_rbgs_body<T, FINE>(P, f, g, h2, color, blockIdx.x, blockIdx.y, blockIdx.z);
}

template <typename T, bool FINE>
__global__ void __launch_bounds__(256, 4) k_nm_resrestrict(const T* P, const T* f, T* fc, T* Pc, Geo g, Geo gc, T inv_h2,
                                                        int planes) {
  __shared__ T patch[kNmRrBuf][kNmRrPatch];
  nm_resrestrict_body<T, FINE>(P, f, fc, Pc, g, gc, inv_h2, blockIdx.x, blockIdx.y, blockIdx.z, planes, patch);
}

template <typename T>
__global__ void __launch_bounds__(256) k_nm_prolong(const T* Ec, T* P, Geo g, Geo gc, int planes) {
  nm_prolong_cells_body<T>(Ec, P, g, gc, blockIdx.x, blockIdx.y, blockIdx.z, planes);
}

template <typename T>
__global__ void __launch_bounds__(1024) k_nm_coarsest(T* P, const T* f, Geo g, double h2, int sweeps) {
  extern __shared__ double sm[];
  nm_coarsest_body<T>(P, f, g, h2, sweeps, sm);
}

template <typename T>
__global__ void __launch_bounds__(256) k_nm_energy(const T* U, const T* K, const T* P, const int* label, Geo g, double h,
                                                   int nDom, double* pd, const double* K64) {
  __shared__ DomTable<kNmPD, 128> tab;
  dom_table_init(tab);
  __syncthreads();
  nm_energy_body<T>(U, K, P, label, g, h, nDom, pd, tab, blockIdx.x, blockIdx.y, blockIdx.z, K64);
  __syncthreads();
  dom_table_flush(tab, pd);
}

template <typename T>
__global__ void __launch_bounds__(256) k_nm_evolve(const int* labIn, int* labOut, const T* U, float* W, Geo g, T dt_w,
                                                   T curvReg) {
  nm_evolve_body<T>(labIn, labOut, U, W, g, dt_w, curvReg, blockIdx.x, blockIdx.y, blockIdx.z);
}

template <typename T>
__global__ void __launch_bounds__(256) k_nm_force(const T* U, const double* at, int nAt, Geo g, double h, double sigma,
                                                  double* F, const double* gw) {
  __shared__ double sx[kNmForceTile], sy[kNmForceTile], sz[kNmForceTile], sr[kNmForceTile];
  nm_force_body<T>(U, at, nAt, g, h, sigma, F, blockIdx.x, gridDim.x, blockIdx.y, sx, sy, sz, sr, gw);
}

template <typename T>
__global__ void k_nm_add(T* __restrict__ K, const T* __restrict__ v, long long n) {
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    K[q] = Ar<T>::add(K[q], v[q]);
}

// ======================================================================================
// host launchers (T = float or double)
// ======================================================================================
static unsigned nblk(long long n, long long b = 256) { return (unsigned)((n + b - 1) / b); }

template <typename T>
cudaError_t nm_potential(T* K, const double* at, int nAt, const Geo& g, double h, double sigma, cudaStream_t st,
                         double* K64) {
  k_nm_potential<T><<<nblk(g.S3), 256, 0, st>>>(K, at, nAt, g, h, sigma, K64);
  return cudaGetLastError();
}
template <typename T>
cudaError_t nm_init(T* U, int* label, const float4* seeds, int nSeed, const Geo& g, float h, cudaStream_t st) {
  k_nm_init<T><<<nblk(g.S3), 256, 0, st>>>(U, label, seeds, nSeed, g, h);
  return cudaGetLastError();
}
template <typename T>
cudaError_t nm_update(const T* U, T* Unew, const T* K, const T* P, const int* label, const Geo& g, T half_dv, T dt,
                      double h3, int nDom, double* norms, cudaStream_t st, const double* scale, const unsigned* seed,
                      unsigned* seed_next, const unsigned char* mask) {
  if (g.NN < 2) return cudaSuccess;
  const dim3 grd = nm_march_grid(g), blk = nm_march_block();
  auto go = [&](auto acc, auto sr, auto msk) {
    k_nm_update<T, decltype(acc)::value, decltype(sr)::value, decltype(msk)::value><<<grd, blk, 0, st>>>(
        U, Unew, K, P, label, g, half_dv, dt, h3, nDom, norms, scale, seed, seed_next, mask);
  };
  using Y = std::true_type;
  using N = std::false_type;
  if (mask) {
    if (norms) { if (seed) go(Y{}, Y{}, Y{}); else go(Y{}, N{}, Y{}); }
    else       { if (seed) go(N{}, Y{}, Y{}); else go(N{}, N{}, Y{}); }
  } else {
    if (norms) { if (seed) go(Y{}, Y{}, N{}); else go(Y{}, N{}, N{}); }
    else       { if (seed) go(N{}, Y{}, N{}); else go(N{}, N{}, N{}); }
  }
  return cudaGetLastError();
}
cudaError_t nm_mask(const int* label, unsigned char* mask, const Geo& g, cudaStream_t st) {
  k_nm_mask<<<nblk(g.S3, 256 * kNmFlatChunk), 256, 0, st>>>(label, mask, g);
  return cudaGetLastError();
}
template <typename T>
cudaError_t nm_apply(T* U, const int* label, const double* scale, int nDom, const Geo& g, cudaStream_t st) {
  k_nm_apply_scale<T><<<nblk(g.S3, 256 * kNmFlatChunk), 256, 0, st>>>(U, label, scale, g.S3, nDom);
  return cudaGetLastError();
}
template <typename T>
cudaError_t nm_normalize(T* U, const int* label, const double* norms, const double* Zdom, int nDom, double* scale, int* err,
                         const Geo& g, cudaStream_t st) {
  k_nm_norm_scale<T><<<nblk(nDom, 128), 128, 0, st>>>(norms, Zdom, nDom, scale, err);
  k_nm_apply_scale<T><<<nblk(g.S3, 256 * kNmFlatChunk), 256, 0, st>>>(U, label, scale, g.S3, nDom);
  return cudaGetLastError();
}
template <typename T>
cudaError_t nm_norm_scale(const double* norms, const double* Zdom, int nDom, double* scale, int* err, cudaStream_t st) {
  k_nm_norm_scale<T><<<nblk(nDom, 128), 128, 0, st>>>(norms, Zdom, nDom, scale, err);
  return cudaGetLastError();
}
template <typename T>
cudaError_t nm_norms(const T* U, const int* label, const Geo& g, double h3, int nDom, double* norms, cudaStream_t st) {
  k_nm_norms<T><<<nblk(g.S3, 256 * kNmFlatChunk), 256, 0, st>>>(U, label, g.S3, h3, nDom, norms);
  return cudaGetLastError();
}
template <typename T>
cudaError_t nm_rbgs(T* P, const T* f, bool fine, const Geo& g, double h2, int color, cudaStream_t st) {
  const int n = g.NN - 1;
  const dim3 blk(32, 8);
  const dim3 grd((n + 63) / 64, (n + 7) / 8, (n + kNmRowPlanes - 1) / kNmRowPlanes);
  if (fine)
    k_nm_rbgs<T, true><<<grd, blk, 0, st>>>(P, f, g, (T)h2, color);
  else
    k_nm_rbgs<T, false><<<grd, blk, 0, st>>>(P, f, g, (T)h2, color);
  return cudaGetLastError();
}
template <typename T>
cudaError_t nm_resrestrict(const T* P, const T* f, bool fine, T* fc, T* Pc, const Geo& g, const Geo& gc, double inv_h2,
                           cudaStream_t st) {
  const int n = gc.NN - 1;
  if (n < 1) return cudaSuccess;
  const long long tiles = (long long)((n + kNmRrTK - 1) / kNmRrTK) * ((n + kNmRrTJ - 1) / kNmRrTJ);
  const int planes = nm_mg_planes(tiles, n);
  const dim3 blk(32, 8), grd((n + kNmRrTK - 1) / kNmRrTK, (n + kNmRrTJ - 1) / kNmRrTJ, (n + planes - 1) / planes);
  if (fine)
    k_nm_resrestrict<T, true><<<grd, blk, 0, st>>>(P, f, fc, Pc, g, gc, (T)inv_h2, planes);
  else
    k_nm_resrestrict<T, false><<<grd, blk, 0, st>>>(P, f, fc, Pc, g, gc, (T)inv_h2, planes);
  return cudaGetLastError();
}
template <typename T>
cudaError_t nm_prolong(const T* Ec, T* P, const Geo& g, const Geo& gc, cudaStream_t st) {
  const int nc = gc.NN;  // coarse cells per axis
  const long long tiles = (long long)((nc + kNmPrTK - 1) / kNmPrTK) * ((nc + kNmPrTJ - 1) / kNmPrTJ);
  const int planes = nm_mg_planes(tiles, nc);
  const dim3 blk(32, 8), grd((nc + kNmPrTK - 1) / kNmPrTK, (nc + kNmPrTJ - 1) / kNmPrTJ, (nc + planes - 1) / planes);
  k_nm_prolong<T><<<grd, blk, 0, st>>>(Ec, P, g, gc, planes);
  return cudaGetLastError();
}
template <typename T>
cudaError_t nm_coarsest(T* P, const T* f, const Geo& g, double h2, int sweeps, cudaStream_t st) {
  const size_t smem = sizeof(double) * 2 * (size_t)g.S3;
  if (smem > 200 * 1024) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(k_nm_coarsest<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_nm_coarsest<T><<<1, kCoarsestThreads, smem, st>>>(P, f, g, h2, sweeps);
  return cudaGetLastError();
}
template <typename T>
cudaError_t nm_energy(const T* U, const T* K, const T* P, const int* label, const Geo& g, double h, int nDom, double* pd,
                      cudaStream_t st, const double* K64) {
  if (g.NN < 2) return cudaSuccess;
  k_nm_energy<T><<<nm_march_grid(g), nm_march_block(), 0, st>>>(U, K, P, label, g, h, nDom, pd, K64);
  return cudaGetLastError();
}
template <typename T>
cudaError_t nm_evolve(const int* labIn, int* labOut, const T* U, float* W, const Geo& g, double dt_w, double curvReg,
                      cudaStream_t st) {
  if (g.NN < 2) return cudaSuccess;
  k_nm_evolve<T><<<nm_march_grid(g), nm_march_block(), 0, st>>>(labIn, labOut, U, W, g, (T)(float)dt_w, (T)(float)curvReg);
  return cudaGetLastError();
}
template <typename T>
cudaError_t nm_force(const T* U, const double* at, int nAt, const Geo& g, double h, double sigma, double* F,
                     cudaStream_t st, const double* gw) {
  if (g.NN < 2 || nAt <= 0) return cudaSuccess;
  const long long n1 = g.NN - 1, nInt = n1 * n1 * n1;
  const long long ntiles = (nInt + kNmForceTile - 1) / kNmForceTile;
  const int chunks = (nAt + 255) / 256;
  long long bx = 148 * 8 / chunks;
  if (bx < 1) bx = 1;
  if (bx > ntiles) bx = ntiles;
  k_nm_force<T><<<dim3((unsigned)bx, (unsigned)chunks), 256, 0, st>>>(U, at, nAt, g, h, sigma, F, gw);
  return cudaGetLastError();
}
template <typename T>
cudaError_t nm_add(T* K, const T* v, long long n, cudaStream_t st) {
  k_nm_add<T><<<148 * 8, 256, 0, st>>>(K, v, n);
  return cudaGetLastError();
}

#define RQ_NM_INSTANTIATE(T)                                                                                          \
  template cudaError_t nm_add<T>(T*, const T*, long long, cudaStream_t);                                           \
  template cudaError_t nm_potential<T>(T*, const double*, int, const Geo&, double, double, cudaStream_t, double*);  \
  template cudaError_t nm_init<T>(T*, int*, const float4*, int, const Geo&, float, cudaStream_t);                   \
  template cudaError_t nm_update<T>(const T*, T*, const T*, const T*, const int*, const Geo&, T, T, double, int,     \
                                    double*, cudaStream_t, const double*, const unsigned*, unsigned*,                \
                                    const unsigned char*);                                                           \
  template cudaError_t nm_apply<T>(T*, const int*, const double*, int, const Geo&, cudaStream_t);                   \
  template cudaError_t nm_normalize<T>(T*, const int*, const double*, const double*, int, double*, int*, const Geo&, \
                                       cudaStream_t);                                                                \
  template cudaError_t nm_norm_scale<T>(const double*, const double*, int, double*, int*, cudaStream_t);            \
  template cudaError_t nm_norms<T>(const T*, const int*, const Geo&, double, int, double*, cudaStream_t);           \
  template cudaError_t nm_rbgs<T>(T*, const T*, bool, const Geo&, double, int, cudaStream_t);                       \
  template cudaError_t nm_resrestrict<T>(const T*, const T*, bool, T*, T*, const Geo&, const Geo&, double,          \
                                         cudaStream_t);                                                            \
  template cudaError_t nm_prolong<T>(const T*, T*, const Geo&, const Geo&, cudaStream_t);                           \
  template cudaError_t nm_coarsest<T>(T*, const T*, const Geo&, double, int, cudaStream_t);                         \
  template cudaError_t nm_energy<T>(const T*, const T*, const T*, const int*, const Geo&, double, int, double*,     \
                                    cudaStream_t, const double*);                                                    \
  template cudaError_t nm_evolve<T>(const int*, int*, const T*, float*, const Geo&, double, double, cudaStream_t);  \
  template cudaError_t nm_force<T>(const T*, const double*, int, const Geo&, double, double, double*, cudaStream_t,  \
                                   const double*);
RQ_NM_INSTANTIATE(float)
RQ_NM_INSTANTIATE(double)

}  // namespace rq
