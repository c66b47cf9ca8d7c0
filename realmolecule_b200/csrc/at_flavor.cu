// at_flavor.cu -- the atom.js per-shell solver (rq_shells_*): one U, W (front) and P field per
// electron shell, the weighted Laplacian div(w grad u), front tracking, and either the
// simultaneous Poisson update or a multigrid Poisson solve per shell (atom.js:1-346).
//
// atom.js updates every field IN PLACE in lexicographic (i, j, k) order: a cell reads the new
// values of its i-1, j-1, k-1 neighbours and the old values of its i+1, j+1, k+1 neighbours.
// That order is kept exactly by a hyperplane wavefront: the cells of the plane i + j + k = t
// depend only on plane t-1 (new) and plane t+1 (old), so each plane is one parallel launch.
// The in-place Gauss-Seidel sweeps of the Poisson solve are pipelined the same way: sweep q
// runs on plane tau - 2q in launch tau, so all sweeps of a smoothing call share one wavefront
// (writes land on planes of one parity, reads on the other).  Arithmetic is that of JS numbers:
// f64 throughout, each Float32Array store rounded to f32, in the reference's operation order;
// only the f64 sums of the normalisation and the energies are summed in a different order.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/rq.h"
#include "rq_internal.cuh"

namespace rq {

constexpr int kAtMaxShells = 8;

struct AtGeo {
  int N, S;
  long long S2, S3;
};

inline AtGeo at_geo(int N) {
  AtGeo g;
  g.N = N; g.S = N + 1; g.S2 = (long long)g.S * g.S; g.S3 = g.S2 * g.S;
  return g;
}

// cell (i, j, k) of plane t for the thread's (i, j); false if the plane has no such cell
__device__ __forceinline__ bool at_plane_cell(const AtGeo& g, int t, int& i, int& j, int& k) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = g.N - 1;
  if (q >= n * n) return false;
  i = 1 + q / n;
  j = 1 + q % n;
  k = t - i - j;
  return k >= 1 && k < g.N;
}

struct AtShellDev {
  int fixed_w;
};

// physicsStep's cell body (atom.js:217-315) for every shell of the cells on plane t.
// acc: E_T, E_ee, E_eK (3) then per shell (ET, Eee, EeK, nrm) -- f64 block sums + atomics.
__global__ void __launch_bounds__(256) k_at_cells(float* __restrict__ U, float* __restrict__ W, float* __restrict__ P,
                                                  const float* __restrict__ K, const AtShellDev* __restrict__ shd,
                                                  int nS, AtGeo g, double h, double d, int simultaneous, int t,
                                                  double* __restrict__ acc) {
  __shared__ double red[3 + 4 * kAtMaxShells];
  for (int q = threadIdx.x; q < 3 + 4 * nS; q += blockDim.x) red[q] = 0.0;
  __syncthreads();
  int i, j, k;
  if (at_plane_cell(g, t, i, j, k)) {
    const double h2 = h * h, h3 = h * h * h, dt = d * h2, PI = 3.141592653589793;
    const long long S3 = g.S3;
    const long long id = (long long)i * g.S2 + (long long)j * g.S + k;
    const long long ip = id + g.S2, im = id - g.S2, jp = id + g.S, jm = id - g.S, kp = id + 1, km = id - 1;
    float c[kAtMaxShells];
    for (int m = 0; m < nS; ++m) {
      c[m] = 0.0f;
      for (int n = 0; n < nS; ++n) {
        if (n != m) c[m] = (float)__dsub_rn((double)c[m], (double)U[n * S3 + id]);
        c[m] = (float)__dmul_rn(0.5, __dadd_rn((double)c[m], (double)U[m * S3 + id]));
      }
    }
    double eT = 0, eEE = 0, eEK = 0;
    for (int m = 0; m < nS; ++m) {
      float* Um = U + m * S3;
      float* Wm = W + m * S3;
      float* Pm = P + m * S3;
      if (!shd[m].fixed_w) {
        const double s6 = __dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn((double)Wm[ip], (double)Wm[im]), (double)Wm[jp]),
                                                        (double)Wm[jm]), (double)Wm[kp]), (double)Wm[km]);
        const double lapW = __ddiv_rn(__dsub_rn(s6, __dmul_rn(6.0, (double)Wm[id])), h2);
        const double gwx = __ddiv_rn(__dsub_rn((double)Wm[ip], (double)Wm[im]), h);
        const double gwy = __ddiv_rn(__dsub_rn((double)Wm[jp], (double)Wm[jm]), h);
        const double gwz = __ddiv_rn(__dsub_rn((double)Wm[kp], (double)Wm[km]), h);
        const double gradW = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(gwx, gwx), __dmul_rn(gwy, gwy)), __dmul_rn(gwz, gwz)));
        const double cm = (double)c[m];
        const double a = __dmul_rn(__dmul_rn(__dmul_rn(2.0, dt), fabs(cm)), lapW);
        const double b = __dmul_rn(__dmul_rn(__dmul_rn(9.0, dt), cm), gradW);
        Wm[id] = (float)__dadd_rn((double)Wm[id], __dadd_rn(a, b));
      }
      const double uid = Um[id], wid = Wm[id], hd = __dmul_rn(0.5, d);
      auto flux = [&](long long pp, long long mm) {
        const double f1 = __dmul_rn(__dmul_rn(__dsub_rn((double)Um[pp], uid), __dadd_rn((double)Wm[pp], wid)), 0.5);
        const double f2 = __dmul_rn(__dmul_rn(__dsub_rn(uid, (double)Um[mm]), __dadd_rn(wid, (double)Wm[mm])), 0.5);
        return __dmul_rn(hd, __dsub_rn(f1, f2));
      };
      const double wlap = __dadd_rn(__dadd_rn(flux(ip, im), flux(jp, jm)), flux(kp, km));
      const double pot = __dmul_rn(__dmul_rn(__dmul_rn(dt, __dsub_rn((double)K[id], __dmul_rn(2.0, (double)Pm[id]))), uid),
                                   wid);
      Um[id] = (float)__dadd_rn(uid, __dadd_rn(wlap, pot));
      // energy where this shell's front dominates (atom.js:258-283)
      const double un = Um[id];
      bool dominated = true;
      for (int n = 0; n < nS; ++n)
        if (n != m && W[n * S3 + id] >= Wm[id]) { dominated = false; break; }
      if (dominated && (double)Wm[id] > 0.01) {
        bool dip = true, djp = true, dkp = true;
        for (int n = 0; n < nS; ++n)
          if (n != m) {
            if (W[n * S3 + ip] >= Wm[ip]) dip = false;
            if (W[n * S3 + jp] >= Wm[jp]) djp = false;
            if (W[n * S3 + kp] >= Wm[kp]) dkp = false;
          }
        const double gx = dip ? __dsub_rn((double)Um[ip], un) : 0.0;
        const double gy = djp ? __dsub_rn((double)Um[jp], un) : 0.0;
        const double gz = dkp ? __dsub_rn((double)Um[kp], un) : 0.0;
        const double tm = __dmul_rn(__dmul_rn(0.5, __dadd_rn(__dadd_rn(__dmul_rn(gx, gx), __dmul_rn(gy, gy)), __dmul_rn(gz, gz))), h);
        const double eem = __dmul_rn(__dmul_rn(__dmul_rn((double)Pm[id], un), un), h3);
        const double ekm = __dmul_rn(__dmul_rn(__dmul_rn(-(double)K[id], un), un), h3);
        const double nrm = __dmul_rn(__dmul_rn(un, un), h3);
        eT += tm; eEE += eem; eEK += ekm;
        atomicAdd(&red[3 + 4 * m], tm);
        atomicAdd(&red[3 + 4 * m + 1], eem);
        atomicAdd(&red[3 + 4 * m + 2], ekm);
        atomicAdd(&red[3 + 4 * m + 3], nrm);
      }
      if (simultaneous) {  // atom.js:286-293
        double rho = 0.0;
        for (int n = 0; n < nS; ++n)
          if (n != m) {
            const double un2 = U[n * S3 + id];
            rho = __dadd_rn(rho, __dmul_rn(__dmul_rn(un2, un2), (double)W[n * S3 + id]));
          }
        const double s6 = __dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn((double)Pm[ip], (double)Pm[im]), (double)Pm[jp]),
                                                        (double)Pm[jm]), (double)Pm[kp]), (double)Pm[km]);
        const double lapP = __ddiv_rn(__dsub_rn(s6, __dmul_rn(6.0, (double)Pm[id])), h2);
        const double inc = __dadd_rn(__dmul_rn(dt, lapP), __dmul_rn(__dmul_rn(__dmul_rn(2.0, PI), dt), rho));
        Pm[id] = (float)__dadd_rn((double)Pm[id], inc);
      }
    }
    atomicAdd(&red[0], eT);
    atomicAdd(&red[1], eEE);
    atomicAdd(&red[2], eEK);
  }
  __syncthreads();
  for (int q = threadIdx.x; q < 3 + 4 * nS; q += blockDim.x)
    if (red[q] != 0.0) atomicAdd(&acc[q], red[q]);
}

// rhs of shell m's Poisson problem: 2 pi sum_{n != m} U_n^2 W_n (atom.js:299-308), interior points
__global__ void k_at_rhs(const float* __restrict__ U, const float* __restrict__ W, float* __restrict__ rhs, int nS, int m,
                         AtGeo g) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = g.N - 1;
  if (q >= n * n * n) return;
  const long long id = (1 + q / (n * n)) * g.S2 + (1 + (q / n) % n) * g.S + 1 + q % n;
  double rho = 0.0;
  for (int s = 0; s < nS; ++s)
    if (s != m) {
      const double u = U[s * g.S3 + id];
      rho = __dadd_rn(rho, __dmul_rn(__dmul_rn(u, u), (double)W[s * g.S3 + id]));
    }
  rhs[id] = (float)__dmul_rn(__dmul_rn(2.0, 3.141592653589793), rho);
}

// launch tau of `iters` pipelined in-place Gauss-Seidel sweeps (atom.js:127-138): sweep s works
// on plane tau - 2 s; thread (s, i, j) takes that sweep's cell of its (i, j) column
__global__ void __launch_bounds__(256) k_at_gs(float* __restrict__ P, const float* __restrict__ rhs, AtGeo g, double h2,
                                               int tau, int iters) {
  const int n = g.N - 1;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n * n * iters) return;
  const int s = q / (n * n), c = q % (n * n);
  const int i = 1 + c / n, j = 1 + c % n, k = tau - 2 * s - i - j;
  if (k < 1 || k >= g.N) return;
  {
    const long long id = (long long)i * g.S2 + (long long)j * g.S + k;
    const double s6 = __dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn((double)P[id + g.S2], (double)P[id - g.S2]),
                                                                (double)P[id + g.S]), (double)P[id - g.S]),
                                          (double)P[id + 1]), (double)P[id - 1]);
    P[id] = (float)__ddiv_rn(__dadd_rn(s6, __dmul_rn(h2, (double)rhs[id])), 6.0);
  }
}

// residual res = rhs + lap P (atom.js:173-184), interior points
__global__ void k_at_residual(const float* __restrict__ P, const float* __restrict__ rhs, float* __restrict__ res,
                              AtGeo g, double h2) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = g.N - 1;
  if (q >= n * n * n) return;
  const long long id = (1 + q / (n * n)) * g.S2 + (1 + (q / n) % n) * g.S + 1 + q % n;
  const double s6 = __dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn((double)P[id + g.S2], (double)P[id - g.S2]),
                                                              (double)P[id + g.S]), (double)P[id - g.S]),
                                        (double)P[id + 1]), (double)P[id - 1]);
  const double lap = __ddiv_rn(__dsub_rn(s6, __dmul_rn(6.0, (double)P[id])), h2);
  res[id] = (float)__dadd_rn((double)rhs[id], lap);
}

// injection to the coarse interior (atom.js:140-153)
__global__ void k_at_restrict(const float* __restrict__ fine, float* __restrict__ coarse, AtGeo g, AtGeo gc) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = gc.N - 1;
  if (q >= n * n * n) return;
  const long long I = 1 + q / (n * n), J = 1 + (q / n) % n, Kc = 1 + q % n;
  coarse[I * gc.S2 + J * gc.S + Kc] = fine[(2 * I) * g.S2 + (2 * J) * g.S + 2 * Kc];
}

// injection-add prolongation (atom.js:155-171): fine interior point x gets coarse floor(x/2)
// when that is a coarse interior point
__global__ void k_at_prolong(const float* __restrict__ Pc, float* __restrict__ P, AtGeo g, AtGeo gc) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = g.N - 1;
  if (q >= n * n * n) return;
  const int i = 1 + (int)(q / (n * n)), j = 1 + (int)((q / n) % n), k = 1 + (int)(q % n);
  const int ci = i >> 1, cj = j >> 1, ck = k >> 1;
  if (ci < 1 || ci >= gc.N || cj < 1 || cj >= gc.N || ck < 1 || ck >= gc.N) return;
  const long long id = (long long)i * g.S2 + (long long)j * g.S + k;
  P[id] = (float)__dadd_rn((double)P[id], (double)Pc[(long long)ci * gc.S2 + (long long)cj * gc.S + ck]);
}

// sum of U^2 h^3 over the interior of shell m (block sums, then FP64 atomics)
__global__ void __launch_bounds__(256) k_at_norm2(const float* __restrict__ U, AtGeo g, double h3, double* __restrict__ out) {
  __shared__ double red[256];
  const long long n = g.N - 1;
  double sum = 0.0;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n * n * n;
       q += (long long)gridDim.x * blockDim.x) {
    const long long id = (1 + q / (n * n)) * g.S2 + (1 + (q / n) % n) * g.S + 1 + q % n;
    const double u = U[id];
    sum += __dmul_rn(__dmul_rn(u, u), h3);
  }
  red[threadIdx.x] = sum;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(out, red[0]);
}

// U *= 1/sqrt(n2) on the interior (atom.js:318-328)
__global__ void k_at_scale(float* __restrict__ U, AtGeo g, const double* __restrict__ n2) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = g.N - 1;
  if (q >= n * n * n) return;
  const long long id = (1 + q / (n * n)) * g.S2 + (1 + (q / n) % n) * g.S + 1 + q % n;
  const double sc = __ddiv_rn(1.0, __dsqrt_rn(*n2));
  U[id] = (float)__dmul_rn((double)U[id], sc);
}

}  // namespace rq

using namespace rq;

struct rq_shells {
  rq_shells_config cfg{};
  std::vector<rq_shell> shells;
  int nS = 0;
  AtGeo g{}, gc{};
  double h = 0;
  float *U = nullptr, *W = nullptr, *P = nullptr, *K = nullptr, *rhs = nullptr, *res = nullptr, *cd = nullptr,
        *Pc = nullptr;
  double* acc = nullptr;  // 3 + 4 nS energy sums, then nS norms
  AtShellDev* shd = nullptr;
  cudaStream_t st = nullptr;
  cudaGraphExec_t graph = nullptr;
  long long launches = 0, graph_launches = 0;
  std::string last_error;
};

#define SCK(call)                                                          \
  do {                                                                     \
    cudaError_t _e = (call);                                               \
    if (_e != cudaSuccess) {                                               \
      s->last_error = std::string(#call) + ": " + cudaGetErrorString(_e);  \
      return _e == cudaErrorMemoryAllocation ? RQ_ENOMEM : RQ_ECUDA;       \
    }                                                                      \
  } while (0)
#define SLAUNCH() SCK(cudaGetLastError()); s->launches++

static unsigned blocks_for(long long n) { return (unsigned)((n + 255) / 256); }

// pipelined Gauss-Seidel: `iters` in-place sweeps of P on grid g in one wavefront
static int at_smooth(rq_shells* s, float* P, const float* rhs, const AtGeo& g, double h2, int iters) {
  const unsigned b = blocks_for((long long)(g.N - 1) * (g.N - 1) * iters);
  for (int tau = 3; tau <= 3 * (g.N - 1) + 2 * (iters - 1); ++tau) {
    k_at_gs<<<b, 256, 0, s->st>>>(P, rhs, g, h2, tau, iters);
    SLAUNCH();
  }
  return RQ_OK;
}

// one physicsStep (atom.js:212-343); the energies land in s->acc
static int at_step(rq_shells* s) {
  const AtGeo& g = s->g;
  const long long nint = (long long)(g.N - 1) * (g.N - 1) * (g.N - 1);
  const double h = s->h, h2 = h * h, h3 = h * h * h;
  SCK(cudaMemsetAsync(s->acc, 0, sizeof(double) * (3 + 5 * s->nS), s->st));
  const unsigned bp = blocks_for((long long)(g.N - 1) * (g.N - 1));
  for (int t = 3; t <= 3 * (g.N - 1); ++t) {
    k_at_cells<<<bp, 256, 0, s->st>>>(s->U, s->W, s->P, s->K, s->shd, s->nS, g, h, s->cfg.d, s->cfg.poisson, t, s->acc);
    SLAUNCH();
  }
  if (!s->cfg.poisson) {  // poissonVcycle per shell (atom.js:186-210, :296-310)
    const AtGeo& gc = s->gc;
    const long long ncint = (long long)(gc.N - 1) * (gc.N - 1) * (gc.N - 1);
    const double hc = h * 2, hc2 = hc * hc;
    for (int m = 0; m < s->nS; ++m) {
      float* Pm = s->P + m * g.S3;
      k_at_rhs<<<blocks_for(nint), 256, 0, s->st>>>(s->U, s->W, s->rhs, s->nS, m, g);
      SLAUNCH();
      int rc = at_smooth(s, Pm, s->rhs, g, h2, 4);
      if (rc != RQ_OK) return rc;
      k_at_residual<<<blocks_for(nint), 256, 0, s->st>>>(Pm, s->rhs, s->res, g, h2);
      SLAUNCH();
      k_at_restrict<<<blocks_for(ncint), 256, 0, s->st>>>(s->res, s->cd, g, gc);
      SLAUNCH();
      SCK(cudaMemsetAsync(s->Pc, 0, sizeof(float) * gc.S3, s->st));
      if ((rc = at_smooth(s, s->Pc, s->cd, gc, hc2, 20)) != RQ_OK) return rc;
      k_at_prolong<<<blocks_for(nint), 256, 0, s->st>>>(s->Pc, Pm, g, gc);
      SLAUNCH();
      if ((rc = at_smooth(s, Pm, s->rhs, g, h2, 4)) != RQ_OK) return rc;
    }
  }
  for (int m = 0; m < s->nS; ++m) {  // normalise each shell over the interior
    double* n2 = s->acc + 3 + 4 * s->nS + m;
    k_at_norm2<<<148 * 2, 256, 0, s->st>>>(s->U + m * g.S3, g, h3, n2);
    SLAUNCH();
    k_at_scale<<<blocks_for(nint), 256, 0, s->st>>>(s->U + m * g.S3, g, n2);
    SLAUNCH();
  }
  return RQ_OK;
}

// atom.js:55-125 on the host (f64, exp from libm, f32 stores), then uploaded
static void at_init_host(const rq_shells* s, std::vector<float>& U, std::vector<float>& W, std::vector<float>& P,
                         std::vector<float>& K) {
  const int NN = s->cfg.NN, nS = s->nS;
  const long long S3 = s->g.S3, S = s->g.S;
  const double scr = s->cfg.screen, h = s->h, h2 = h * h, h3 = h * h * h;
  const int N2 = NN / 2;
  std::vector<double> Rmin(nS), Rmax(nS);
  Rmin[0] = 0; Rmax[0] = s->shells[0].Rmax;
  for (int m = 1; m < nS; ++m) {
    Rmin[m] = s->shells[m - 1].Rmax;
    Rmax[m] = s->shells[m].Rmax ? s->shells[m].Rmax : scr / 2;
  }
  U.assign(S3 * nS, 0.f); W.assign(S3 * nS, 0.f); P.assign(S3 * nS, 0.f); K.assign(S3, 0.f);
  for (int i = 0; i <= NN; ++i)
    for (int j = 0; j <= NN; ++j)
      for (int k = 0; k <= NN; ++k) {
        const long long id = ((long long)i * S + j) * S + k;
        const double r2 = (double)((i - N2) * (i - N2)) * h2 + (double)((j - N2) * (j - N2)) * h2 +
                          (double)((k - N2) * (k - N2)) * h2 + 0.12 * h2;
        const double r = std::sqrt(r2);
        K[id] = (float)(s->cfg.Z_kernel / r);
        for (int m = 0; m < nS; ++m) {
          const rq_shell& c = s->shells[m];
          bool in;
          float& w = W[m * S3 + id];
          if (c.split) {
            if (i == N2) { in = true; w = 0.5f; }
            else in = c.half_index == 0 ? (i < N2) : (i > N2);
          } else if (c.outer_half) {
            in = r >= Rmin[m] && r < Rmax[m] && i > N2;
          } else {
            in = r >= Rmin[m] && r < Rmax[m];
          }
          if (in) {
            U[m * S3 + id] = (float)std::exp(-c.Zeff * r);
            double wv = 1.0;
            const double smoothW = 2 * h;
            if (!c.split) {
              if (Rmin[m] > 0) { const double din = r - Rmin[m]; if (din < smoothW) wv = std::fmin(wv, din / smoothW); }
              const double dout = Rmax[m] - r;
              if (dout < smoothW) wv = std::fmin(wv, dout / smoothW);
            }
            wv = std::fmax(0.01, wv);
            if (w == 0) w = (float)wv;
          }
        }
        for (int m = 0; m < nS; ++m) P[m * S3 + id] = (float)(0.5 / r);
      }
  for (int m = 0; m < nS; ++m) {
    double n2 = 0;
    for (long long id = 0; id < S3; ++id) n2 += (double)U[m * S3 + id] * U[m * S3 + id] * h3;
    const double sc = 1 / std::sqrt(n2);
    for (long long id = 0; id < S3; ++id) U[m * S3 + id] = (float)(U[m * S3 + id] * sc);
  }
}

extern "C" int rq_shells_create(const rq_shells_config* cfg, const rq_shell* shells, int32_t n_shells, rq_shells** out) {
  if (!cfg || !shells || !out || n_shells < 1 || n_shells > kAtMaxShells) return RQ_EINVAL;
  *out = nullptr;
  if (cfg->NN < 8 || cfg->NN % 2 || cfg->screen <= 0 || cfg->d <= 0 || cfg->poisson < 0 || cfg->poisson > 1)
    return RQ_EINVAL;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return RQ_ENODEV;
  rq_shells* s = new (std::nothrow) rq_shells();
  if (!s) return RQ_ENOMEM;
  s->cfg = *cfg;
  s->shells.assign(shells, shells + n_shells);
  s->nS = n_shells;
  s->g = at_geo(cfg->NN);
  s->gc = at_geo(cfg->NN / 2);
  s->h = cfg->screen / cfg->NN;
  auto fail = [&](int rc) {
    std::fprintf(stderr, "rq_shells_create: %s\n", s->last_error.c_str());
    rq_shells_destroy(s);
    return rc;
  };
  int rc = RQ_OK;
  auto alloc = [&](void** p, size_t bytes) -> int {
    if (cudaMalloc(p, bytes) != cudaSuccess) { s->last_error = "cudaMalloc"; return RQ_ENOMEM; }
    if (cudaMemset(*p, 0, bytes) != cudaSuccess) { s->last_error = "cudaMemset"; return RQ_ECUDA; }
    return RQ_OK;
  };
  const size_t S3 = (size_t)s->g.S3, SC3 = (size_t)s->gc.S3;
  if ((rc = alloc((void**)&s->U, sizeof(float) * S3 * n_shells)) || (rc = alloc((void**)&s->W, sizeof(float) * S3 * n_shells)) ||
      (rc = alloc((void**)&s->P, sizeof(float) * S3 * n_shells)) || (rc = alloc((void**)&s->K, sizeof(float) * S3)) ||
      (rc = alloc((void**)&s->rhs, sizeof(float) * S3)) || (rc = alloc((void**)&s->res, sizeof(float) * S3)) ||
      (rc = alloc((void**)&s->cd, sizeof(float) * SC3)) || (rc = alloc((void**)&s->Pc, sizeof(float) * SC3)) ||
      (rc = alloc((void**)&s->acc, sizeof(double) * (3 + 5 * n_shells))) ||
      (rc = alloc((void**)&s->shd, sizeof(AtShellDev) * n_shells)))
    return fail(rc);
  if (cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess) {
    s->last_error = "cudaStreamCreate";
    return fail(RQ_ECUDA);
  }
  std::vector<AtShellDev> hd(n_shells);
  for (int m = 0; m < n_shells; ++m) hd[m].fixed_w = shells[m].fixed_w;
  std::vector<float> U, W, P, K;
  at_init_host(s, U, W, P, K);
  if (cudaMemcpy(s->shd, hd.data(), sizeof(AtShellDev) * n_shells, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(s->U, U.data(), sizeof(float) * U.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(s->W, W.data(), sizeof(float) * W.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(s->P, P.data(), sizeof(float) * P.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(s->K, K.data(), sizeof(float) * K.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
    s->last_error = "initial upload";
    return fail(RQ_ECUDA);
  }
  *out = s;
  return RQ_OK;
}

extern "C" void rq_shells_destroy(rq_shells* s) {
  if (!s) return;
  if (s->st) cudaStreamSynchronize(s->st);
  if (s->graph) cudaGraphExecDestroy(s->graph);
  for (void* p : {(void*)s->U, (void*)s->W, (void*)s->P, (void*)s->K, (void*)s->rhs, (void*)s->res, (void*)s->cd,
                  (void*)s->Pc, (void*)s->acc, (void*)s->shd})
    if (p) cudaFree(p);
  if (s->st) cudaStreamDestroy(s->st);
  delete s;
}

extern "C" const char* rq_shells_last_error(const rq_shells* s) { return s ? s->last_error.c_str() : "null"; }

extern "C" int rq_shells_step(rq_shells* s, int32_t n, double* E, double* per_shell) {
  if (!s || n < 0) return RQ_EINVAL;
  for (int q = 0; q < n; ++q) {
    if (!s->graph) {  // one step is always the same launch sequence: captured once, replayed
      const long long l0 = s->launches;
      SCK(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
      int rc = at_step(s);
      cudaGraph_t gr = nullptr;
      cudaError_t e = cudaStreamEndCapture(s->st, &gr);
      if (rc != RQ_OK) {
        if (gr) cudaGraphDestroy(gr);
        return rc;
      }
      SCK(e);
      e = cudaGraphInstantiate(&s->graph, gr, 0);
      cudaGraphDestroy(gr);
      SCK(e);
      s->graph_launches = s->launches - l0;
    } else {
      s->launches += s->graph_launches;
    }
    SCK(cudaGraphLaunch(s->graph, s->st));
  }
  const int nS = s->nS;
  std::vector<double> acc(3 + 5 * nS);
  SCK(cudaMemcpyAsync(acc.data(), s->acc, sizeof(double) * acc.size(), cudaMemcpyDeviceToHost, s->st));
  SCK(cudaStreamSynchronize(s->st));
  if (E) {
    E[1] = acc[0]; E[2] = acc[2]; E[3] = acc[1];
    E[0] = E[1] + E[2] + E[3];
  }
  if (per_shell)
    for (int m = 0; m < nS; ++m) {
      double* o = per_shell + 5 * m;
      const double* a = &acc[3 + 4 * m];
      o[0] = a[0]; o[1] = a[1]; o[2] = a[2]; o[3] = a[3];
      o[4] = (a[0] + 2 * a[1] + a[2]) / (a[3] != 0 ? a[3] : 1);  // atom.js:340
    }
  return RQ_OK;
}

extern "C" int rq_shells_download(rq_shells* s, int32_t m, float* U, float* W, float* P) {
  if (!s || m < 0 || m >= s->nS) return RQ_EINVAL;
  const size_t S3 = (size_t)s->g.S3;
  if (U) SCK(cudaMemcpyAsync(U, s->U + m * S3, sizeof(float) * S3, cudaMemcpyDeviceToHost, s->st));
  if (W) SCK(cudaMemcpyAsync(W, s->W + m * S3, sizeof(float) * S3, cudaMemcpyDeviceToHost, s->st));
  if (P) SCK(cudaMemcpyAsync(P, s->P + m * S3, sizeof(float) * S3, cudaMemcpyDeviceToHost, s->st));
  SCK(cudaStreamSynchronize(s->st));
  return RQ_OK;
}

extern "C" int rq_shells_upload(rq_shells* s, int32_t m, const float* U, const float* W, const float* P) {
  if (!s || m < 0 || m >= s->nS) return RQ_EINVAL;
  const size_t S3 = (size_t)s->g.S3;
  if (U) SCK(cudaMemcpyAsync(s->U + m * S3, U, sizeof(float) * S3, cudaMemcpyHostToDevice, s->st));
  if (W) SCK(cudaMemcpyAsync(s->W + m * S3, W, sizeof(float) * S3, cudaMemcpyHostToDevice, s->st));
  if (P) SCK(cudaMemcpyAsync(s->P + m * S3, P, sizeof(float) * S3, cudaMemcpyHostToDevice, s->st));
  SCK(cudaStreamSynchronize(s->st));
  return RQ_OK;
}

extern "C" int rq_shells_info(const rq_shells* s, int64_t* kernel_launches) {
  if (!s) return RQ_EINVAL;
  if (kernel_launches) *kernel_launches = s->launches;
  return RQ_OK;
}
