// nm_adjoint.cu -- gradient of the new flavour's energy readout with respect to the nuclear
// positions and an external potential, by a reverse sweep through the last recorded steps.
//
// One forward step s of the new flavour (nm_flavor.cu) acts on the normalised state as
//   [V-cycle]    P <- M P + B f,  f = 2 pi psi^2                 (every poisson_interval steps)
//   update       psi~ = A psi,  A = I + half_dv L + dt diag(K - 2P)   (L: same-label Laplacian)
//   [normalise]  psi = c psi~,  c_d = sqrt(Z_d / (h^3 sum_d psi~^2))
// and the readout is E = sum_d w_d (T_d + V_eK,d + 2 h^3 sum_d P rho) - (h^3 / 2 pi) sum P (A_h P),
// w_d = Z_d / N_d, A_h = -lap_h (the P-stationary Hartree form), with K = K_nuclei(R) + v.
// The reverse sweep starts from dE/dpsi, dE/dP and dE/dK of the readout and applies the
// transposes step by step, newest first:
//   normalise^T  lam <- c (lam - (h^3 / Z) psi <psi, lam>_d)
//   update^T     lam <- A lam (A is symmetric: L is the same-label graph Laplacian with Dirichlet
//                faces), dE/dK += dt psi lam, dE/dP += -2 dt psi lam
//   V-cycle^T    the smoothing colours, the residual, full weighting and trilinear prolongation
//                transposed in reverse order (full weighting^T = prolongation / 8), the coarsest
//                sweeps in reverse; this gives dE/dP before the cycle and dE/df, and
//                lam += 4 pi psi dE/df.
// The labels are integers and held fixed; the state the window starts from is held fixed (a
// warm start).  F_a = -dE/dR_a is then the Hellmann-Feynman-shaped gather with the weight dE/dK
// in place of -h^3 rho (nm_force_body); with no recorded step dE/dK = -h^3 rho and the force is
// the Hellmann-Feynman force, exact at a converged state.  dE/dv = dE/dK.
//
// The reference computes forces with the Hellmann-Feynman integral of its own softened nuclei
// (cloud/solver.py:282-315 computeForceAll, molecule.js:1271-1330) or the Hartree-gradient ball
// (molecule.js:1200-1269); this is the exact derivative of the discrete energy the new flavour
// actually reaches after a finite number of warm-started iterations.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "nm_bodies.cuh"
#include "rq_flavors.h"

using namespace rq;

#define CK(call)                                 \
  do {                                           \
    int _rc = rq_cuda(c, (call), #call);         \
    if (_rc != RQ_OK) return _rc;                \
  } while (0)

namespace {

unsigned nblk(long long n, long long b = 256) { return (unsigned)((n + b - 1) / b); }

// interior point number q -> (i, j, k) and its linear index
struct Pt {
  int i, j, k;
  long long id;
};
// Interior point of a 3-D launch (grid3 / kBlk3): x runs along k, y along j, z is the plane i.  No
// integer division per point, and a block's threads read contiguous rows.
constexpr int kB3x = 64, kB3y = 4;
__device__ __forceinline__ bool interior_pt3(const Geo& g, Pt& p) {
  p.k = 1 + (int)(blockIdx.x * kB3x + threadIdx.x);
  p.j = 1 + (int)(blockIdx.y * kB3y + threadIdx.y);
  p.i = 1 + (int)blockIdx.z;
  p.id = (long long)p.i * g.S2 + (long long)p.j * g.S + p.k;
  return p.k < g.NN && p.j < g.NN && p.i < g.NN;
}
inline dim3 grid3(const Geo& g) {
  const unsigned n = (unsigned)(g.NN - 1);
  return dim3((n + kB3x - 1) / kB3x, (n + kB3y - 1) / kB3y, n);
}
const dim3 kBlk3(kB3x, kB3y, 1);

// dE/dpsi, dE/dP and dE/dK of the readout at psi (nm_energy: E = sum_d w_d Q_d - (h^3 / 2 pi) <P, A P>,
// Q_d = T_d + V_eK,d + 2 h^3 sum_d P rho, w_d = Z_d / N_d).  wq: per domain (w, Q/N).  T = h/2 sum
// over same-label edges (psi_a - psi_b)^2 (edges to a Dirichlet face included), so dT/dpsi = -h L psi
// with the update's Laplacian; dE/dP = 2 w h^3 rho - (h^3 / pi) A P.
template <typename T>
__global__ void __launch_bounds__(256) k_adj_seed(const T* __restrict__ U, const T* __restrict__ K,
                                                  const T* __restrict__ P, const int* __restrict__ label, Geo g,
                                                  double h, int nDom, const double* __restrict__ wq,
                                                  T* __restrict__ lam, T* __restrict__ muP, double* __restrict__ gK,
                                                  const double* __restrict__ K64) {
  Pt p;
  if (!interior_pt3(g, p)) return;
  const long long id = p.id, S = g.S, S2 = g.S2;
  const int L = label[id];
  if (L < 0 || L >= nDom) {
    lam[id] = T(0);
    muP[id] = T(0);
    gK[id] = 0.0;
    return;
  }
  const double h3 = h * h * h, u = (double)U[id];
  const long long nb[6] = {id + S2, id - S2, id + S, id - S, id + 1, id - 1};
  double lap = 0.0;
#pragma unroll
  for (int t = 0; t < 6; ++t)
    if (label[nb[t]] == L) lap += (double)U[nb[t]] - u;
  const double w = wq[2 * L], qn = wq[2 * L + 1];
  const double pc = (double)P[id];
  const double ap = (6.0 * pc - ((double)P[id + S2] + (double)P[id - S2] + (double)P[id + S] + (double)P[id - S] +
                                 (double)P[id + 1] + (double)P[id - 1])) / (h * h);
  const double kv = K64 ? K64[id] : (double)K[id];  // the readout's K (nm_energy_body)
  lam[id] = (T)(w * (-h * lap + 2.0 * h3 * u * (2.0 * pc - kv - qn)));
  muP[id] = (T)(2.0 * w * h3 * u * u - h3 / M_PI * ap);
  gK[id] = -w * h3 * u * u;
}

// per-domain <psi, lam> in FP64 over all S^3 points
template <typename T>
__global__ void __launch_bounds__(256) k_adj_dot(const T* __restrict__ psi, const T* __restrict__ lam,
                                                 const int* __restrict__ label, long long S3, int nDom,
                                                 double* __restrict__ dots) {
  __shared__ DomTable<1, 128> tab;
  dom_table_init(tab);
  __syncthreads();
  RunSum<1> rs;
  rs.reset();
  const long long base = (long long)blockIdx.x * blockDim.x * kNmFlatChunk;
  for (int t = 0; t < kNmFlatChunk; ++t) {
    const long long id = base + (long long)t * blockDim.x + threadIdx.x;
    if (id >= S3) break;
    const int l = label[id];
    if (l < 0 || l >= nDom) continue;
    const double v = (double)psi[id] * (double)lam[id];
    rs.add(l, &v, tab, dots);
  }
  rs.finish(tab, dots);
  __syncthreads();
  dom_table_flush(tab, dots);
}

// per-domain (c, beta) of a transposed normalisation: c = the forward scale, beta = c h^3 <psi, lam> / Z
__global__ void k_adj_norm_coef(const double* __restrict__ scale, const double* __restrict__ Zdom,
                                const double* __restrict__ dots, int nDom, double h3, double* __restrict__ coef) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= nDom) return;
  const double c = scale[d], Z = Zdom[d];
  coef[2 * d] = c;
  coef[2 * d + 1] = Z > 0.0 ? c * h3 * dots[d] / Z : 0.0;
}

// lam <- c lam - beta psi per domain (boundary points hold 0 in both and stay 0)
template <typename T>
__global__ void __launch_bounds__(256) k_adj_norm_apply(T* __restrict__ lam, const T* __restrict__ psi,
                                                        const int* __restrict__ label, const double* __restrict__ coef,
                                                        long long S3, int nDom) {
  const long long base = (long long)blockIdx.x * blockDim.x * kNmFlatChunk;
  for (int t = 0; t < kNmFlatChunk; ++t) {
    const long long id = base + (long long)t * blockDim.x + threadIdx.x;
    if (id >= S3) break;
    const int l = label[id];
    if (l < 0 || l >= nDom) continue;
    lam[id] = (T)(coef[2 * l] * (double)lam[id] - coef[2 * l + 1] * (double)psi[id]);
  }
}

// update^T: out = A(K, P) in (the update's operator applied to lam), gK += dt psi in,
// muP += -2 dt psi in, where psi is the state the forward update started from
template <typename T>
__global__ void __launch_bounds__(256) k_adj_update(const T* __restrict__ in, T* __restrict__ out,
                                                    const T* __restrict__ K, const T* __restrict__ P,
                                                    const int* __restrict__ label, const T* __restrict__ psi, Geo g,
                                                    double half_dv, double dt, double* __restrict__ gK,
                                                    T* __restrict__ muP) {
  Pt p;
  if (!interior_pt3(g, p)) return;
  const long long id = p.id, S = g.S, S2 = g.S2;
  const int L = label[id];
  const double lc = (double)in[id];
  const long long nb[6] = {id + S2, id - S2, id + S, id - S, id + 1, id - 1};
  double lap = 0.0;
#pragma unroll
  for (int t = 0; t < 6; ++t)
    if (label[nb[t]] == L) lap += (double)in[nb[t]] - lc;
  out[id] = (T)(lc + half_dv * lap + dt * ((double)K[id] - 2.0 * (double)P[id]) * lc);
  const double pv = (double)psi[id];
  gK[id] += dt * pv * lc;
  muP[id] = (T)((double)muP[id] - 2.0 * dt * pv * lc);
}

// one colour of a red-black sweep, transposed.  Forward: P <- (sum_6 P + h^2 f) / 6 at the points
// of colour `color` ((i+j+k) % 2 == color).  Transposed: at those points out = 0 and
// muf += h^2/6 in; at the others out = in + (1/6) sum_6 in (every neighbour has colour `color`).
// Boundary entries of the adjoint arrays hold 0 and are never written.
template <typename T>
__global__ void __launch_bounds__(256) k_adj_rbgs(const T* __restrict__ in, T* __restrict__ out, T* __restrict__ muf,
                                                  Geo g, double h2, int color) {
  Pt p;
  if (!interior_pt3(g, p)) return;
  const long long id = p.id, S = g.S, S2 = g.S2;
  const double v = (double)in[id];
  if (((p.i + p.j + p.k) & 1) == color) {
    out[id] = T(0);
    muf[id] = (T)((double)muf[id] + h2 / 6.0 * v);
  } else {
    const double s = (double)in[id + S2] + (double)in[id - S2] + (double)in[id + S] + (double)in[id - S] +
                     (double)in[id + 1] + (double)in[id - 1];
    out[id] = (T)(v + s / 6.0);
  }
}

// residual transposed (forward r = f + (sum_6 P - 6 P) / h^2): muf += mur, muP += (sum_6 mur - 6 mur) / h^2
template <typename T>
__global__ void __launch_bounds__(256) k_adj_residual(const T* __restrict__ mur, T* __restrict__ muP,
                                                      T* __restrict__ muf, Geo g, double inv_h2) {
  Pt p;
  if (!interior_pt3(g, p)) return;
  const long long id = p.id, S = g.S, S2 = g.S2;
  const double r = (double)mur[id];
  const double s = (double)mur[id + S2] + (double)mur[id - S2] + (double)mur[id + S] + (double)mur[id - S] +
                   (double)mur[id + 1] + (double)mur[id - 1];
  muf[id] = (T)((double)muf[id] + r);
  muP[id] = (T)((double)muP[id] + (s - 6.0 * r) * inv_h2);
}

// full weighting transposed: mur = (1/8) trilinear(mufc) at the fine interior points
template <typename T>
__global__ void __launch_bounds__(256) k_adj_restrict(const T* __restrict__ mufc, T* __restrict__ mur, Geo g, Geo gc) {
  Pt p;
  if (!interior_pt3(g, p)) return;
  const int oi = p.i & 1, oj = p.j & 1, ok = p.k & 1;
  double v = 0.0;
  for (int a = 0; a <= oi; ++a)
    for (int b = 0; b <= oj; ++b)
      for (int cc = 0; cc <= ok; ++cc)
        v += (double)mufc[(long long)((p.i >> 1) + a) * gc.S2 + (long long)((p.j >> 1) + b) * gc.S + (p.k >> 1) + cc];
  mur[p.id] = (T)(v / (8.0 * (1 + oi) * (1 + oj) * (1 + ok)));
}

// trilinear prolongation transposed: muPc = (1/8) sum (8,4,2,1 weights) muP at the coarse interior points
template <typename T>
__global__ void __launch_bounds__(256) k_adj_prolong(const T* __restrict__ muP, T* __restrict__ muPc, Geo g, Geo gc) {
  Pt p;
  if (!interior_pt3(gc, p)) return;
  double v = 0.0;
  for (int a = -1; a <= 1; ++a)
    for (int b = -1; b <= 1; ++b)
      for (int cc = -1; cc <= 1; ++cc) {
        const double w = (a == 0 ? 2 : 1) * (b == 0 ? 2 : 1) * (cc == 0 ? 2 : 1);
        v += w * (double)muP[(long long)(2 * p.i + a) * g.S2 + (long long)(2 * p.j + b) * g.S + (2 * p.k + cc)];
      }
  muPc[p.id] = (T)(v / 8.0);
}

// the coarsest level's red-black sweeps transposed, in reverse order, by one block in FP64 shared
// memory: given dE/dP after the solve (which started from P = 0), writes dE/df
template <typename T>
__global__ void __launch_bounds__(1024) k_adj_coarsest(const T* __restrict__ muP, T* __restrict__ muf, Geo g, double h2,
                                                       int sweeps) {
  extern __shared__ double sm[];
  double* sP = sm;
  double* sf = sm + g.S3;
  for (long long q = threadIdx.x; q < g.S3; q += blockDim.x) {
    sP[q] = (double)muP[q];
    sf[q] = 0.0;
  }
  __syncthreads();
  const int n = g.NN - 1, S = g.S, S2 = (int)g.S2;
  const int nint = n * n * n;
  for (int s = sweeps - 1; s >= 0; --s)
    for (int color = 1; color >= 0; --color) {
      for (int q = threadIdx.x; q < nint; q += blockDim.x) {  // the other colour gathers
        const int k = 1 + q % n, j = 1 + (q / n) % n, i = 1 + q / (n * n);
        if (((i + j + k) & 1) == color) continue;
        const int id = i * S2 + j * S + k;
        sP[id] += (sP[id + S2] + sP[id - S2] + sP[id + S] + sP[id - S] + sP[id + 1] + sP[id - 1]) / 6.0;
      }
      __syncthreads();
      for (int q = threadIdx.x; q < nint; q += blockDim.x) {  // this colour: into f, then 0
        const int k = 1 + q % n, j = 1 + (q / n) % n, i = 1 + q / (n * n);
        if (((i + j + k) & 1) != color) continue;
        const int id = i * S2 + j * S + k;
        sf[id] += h2 / 6.0 * sP[id];
        sP[id] = 0.0;
      }
      __syncthreads();
    }
  for (long long q = threadIdx.x; q < g.S3; q += blockDim.x) muf[q] = (T)sf[q];
}

// lam += 4 pi psi muf (the fine right-hand side f = 2 pi psi^2)
template <typename T>
__global__ void __launch_bounds__(256) k_adj_rhs(T* __restrict__ lam, const T* __restrict__ psi, const T* __restrict__ muf,
                                                 Geo g) {
  Pt p;
  if (!interior_pt3(g, p)) return;
  const long long id = p.id;
  lam[id] = (T)((double)lam[id] + 12.566370614359172 * (double)psi[id] * (double)muf[id]);
}

// checkpoint of the state a step starts from: psi with a pending per-domain scale applied
// (FP64 product rounded once, as the update applies it) or a plain copy
template <typename T>
__global__ void __launch_bounds__(256) k_adj_ckpt(const T* __restrict__ U, const int* __restrict__ label,
                                                  const double* __restrict__ scale, T* __restrict__ out, long long S3,
                                                  int nDom) {
  for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < S3;
       id += (long long)gridDim.x * blockDim.x) {
    const T u = U[id];
    if (!scale) {
      out[id] = u;
      continue;
    }
    const int l = label[id];
    out[id] = (l < 0 || l >= nDom) ? u : (T)((double)u * scale[l]);
  }
}

size_t esize(const rq_ctx* c) { return c->fp64 ? sizeof(double) : sizeof(float); }

template <typename T>
T* slot(void* base, long long k, long long S3) {
  return (T*)base + k * S3;
}

// a new P snapshot slot holding the P in effect now.  A window reaches back at most cap steps,
// i.e. over fewer than np - 1 V-cycles, so no step still in the window refers to the slot that
// is overwritten.
int snapshot_p(rq_ctx* c) {
  rq_adj& A = c->adj;
  const size_t bytes = (size_t)c->g.S3 * esize(c);
  const int s = A.next_p % A.np;
  A.next_p++;
  CK(cudaMemcpyAsync((char*)A.psum + (size_t)s * bytes, c->P[c->cp], bytes, cudaMemcpyDeviceToDevice, c->st));
  A.cur_p = s;
  return RQ_OK;
}

}  // namespace

// ----------------------------------------------------------------------------------------
// window management
// ----------------------------------------------------------------------------------------
void nm_adj_free(rq_ctx* c) {
  rq_adj& A = c->adj;
  void* p[] = {A.psi, A.psum, A.scales, A.lam[0], A.lam[1], A.muP[0], A.muP[1], A.muf, A.gK, A.dots, A.coef, A.wq};
  for (void* q : p)
    if (q) cudaFree(q);
  for (auto& L : A.lv)
    for (void* q : {L.mu[0], L.mu[1], L.muf, L.mur})
      if (q) cudaFree(q);
  A = rq_adj();
}

void nm_adj_reset(rq_ctx* c) {
  c->adj.rec.clear();
  c->adj.cur_p = -1;
}

int nm_adj_set_window(rq_ctx* c, int steps) {
  if (steps < 0) return rq_fail(c, RQ_EINVAL, "negative adjoint window");
  nm_adj_free(c);
  if (steps == 0) return RQ_OK;
  rq_adj& A = c->adj;
  const size_t S3 = (size_t)c->g.S3, es = esize(c);
  const int n = c->n_atoms;
  const int pi = std::max(1, c->cfg.poisson_interval);
  const int np = (steps + pi - 1) / pi + 2;
  auto alloc = [&](void** p, size_t bytes) -> bool {
    if (cudaMalloc(p, bytes) != cudaSuccess) return false;
    return cudaMemsetAsync(*p, 0, bytes, c->st) == cudaSuccess;
  };
  bool ok = alloc(&A.psi, (size_t)steps * S3 * es) && alloc(&A.psum, (size_t)np * S3 * es) &&
            alloc((void**)&A.scales, sizeof(double) * (size_t)steps * n) && alloc(&A.lam[0], S3 * es) &&
            alloc(&A.lam[1], S3 * es) && alloc(&A.muP[0], S3 * es) && alloc(&A.muP[1], S3 * es) &&
            alloc(&A.muf, S3 * es) && alloc((void**)&A.gK, S3 * sizeof(double)) &&
            alloc((void**)&A.dots, sizeof(double) * n) && alloc((void**)&A.coef, sizeof(double) * 2 * n) &&
            alloc((void**)&A.wq, sizeof(double) * 2 * n);
  const int levels = (int)c->mg.size();
  A.lv.assign(levels, rq_adj::Level());
  for (int l = 0; ok && l < levels; ++l) {
    const size_t s3 = (size_t)c->mg[l].g.S3;
    if (l > 0) ok = alloc(&A.lv[l].mu[0], s3 * es) && alloc(&A.lv[l].mu[1], s3 * es) && alloc(&A.lv[l].muf, s3 * es);
    if (ok && l < levels - 1) ok = alloc(&A.lv[l].mur, s3 * es);
  }
  if (!ok) {
    nm_adj_free(c);
    return rq_cuda(c, cudaErrorMemoryAllocation, "adjoint window");
  }
  A.cap = steps;
  A.np = np;
  nm_adj_reset(c);
  return cudaStreamSynchronize(c->st) == cudaSuccess ? RQ_OK : rq_cuda(c, cudaGetLastError(), "adjoint window");
}

int nm_adj_record_step(rq_ctx* c, bool vcycle, bool norm) {
  rq_adj& A = c->adj;
  if (vcycle || A.cur_p < 0) {
    int rc = snapshot_p(c);
    if (rc != RQ_OK) return rc;
  }
  if ((int)A.rec.size() == A.cap) A.rec.erase(A.rec.begin());
  rq_adj::Rec r;
  r.psi_slot = (int)(A.next_psi % A.cap);
  A.next_psi++;
  r.p_slot = A.cur_p;
  r.vcycle = vcycle;
  r.norm = norm;
  r.label = false;
  const long long S3 = c->g.S3;
  const double* sc = c->nm_pending ? (const double*)c->scale64 : nullptr;
  if (c->fp64)
    LAUNCH(RQ_KC_OTHER, 20.0 * S3,
           (k_adj_ckpt<double><<<148 * 8, 256, 0, c->st>>>((const double*)c->U[c->cu], c->lab[c->cl], sc,
                                                           slot<double>(A.psi, r.psi_slot, S3), S3, c->n_atoms),
            cudaGetLastError()));
  else
    LAUNCH(RQ_KC_OTHER, 12.0 * S3,
           (k_adj_ckpt<float><<<148 * 8, 256, 0, c->st>>>((const float*)c->U[c->cu], c->lab[c->cl], sc,
                                                          slot<float>(A.psi, r.psi_slot, S3), S3, c->n_atoms),
            cudaGetLastError()));
  A.rec.push_back(r);
  return RQ_OK;
}

int nm_adj_record_scale(rq_ctx* c) {
  rq_adj& A = c->adj;
  if (A.rec.empty()) return RQ_OK;
  const int n = c->n_atoms;
  CK(cudaMemcpyAsync(A.scales + (size_t)A.rec.back().psi_slot * n, c->scale64, sizeof(double) * n,
                     cudaMemcpyDeviceToDevice, c->st));
  return RQ_OK;
}

void nm_adj_record_label(rq_ctx* c) {
  if (!c->adj.rec.empty()) c->adj.rec.back().label = true;
}

// ----------------------------------------------------------------------------------------
// the reverse sweep
// ----------------------------------------------------------------------------------------
namespace {

// transposed normalisation of lam with the forward scales `scale` at the normalised state psi
template <typename T>
int adj_norm(rq_ctx* c, const T* psi, T* lam, const double* scale) {
  rq_adj& A = c->adj;
  const int n = c->n_atoms;
  const long long S3 = c->g.S3;
  CK(cudaMemsetAsync(A.dots, 0, sizeof(double) * n, c->st));
  LAUNCH(RQ_KC_FORCES, 2.0 * sizeof(T) * S3 + 4.0 * S3,
         (k_adj_dot<T><<<nblk(S3, 256 * kNmFlatChunk), 256, 0, c->st>>>(psi, lam, c->lab[c->cl], S3, n, A.dots),
          cudaGetLastError()));
  LAUNCH(RQ_KC_FORCES, 32.0 * n,
         (k_adj_norm_coef<<<nblk(n, 128), 128, 0, c->st>>>(scale, c->Zdom64, A.dots, n, c->h3, A.coef),
          cudaGetLastError()));
  LAUNCH(RQ_KC_FORCES, 3.0 * sizeof(T) * S3 + 4.0 * S3,
         (k_adj_norm_apply<T><<<nblk(S3, 256 * kNmFlatChunk), 256, 0, c->st>>>(lam, psi, c->lab[c->cl], A.coef, S3, n),
          cudaGetLastError()));
  return RQ_OK;
}

// transposed V-cycle on level l: mu[*cur] holds dE/dP of the level after the cycle and becomes
// dE/dP before it; dE/df of the level is accumulated into its muf
template <typename T>
int adj_vcycle(rq_ctx* c, int l, int* cur) {
  rq_adj& A = c->adj;
  const rq_mg_level& L = c->mg[l];
  T* mu[2] = {l == 0 ? (T*)A.muP[0] : (T*)A.lv[l].mu[0], l == 0 ? (T*)A.muP[1] : (T*)A.lv[l].mu[1]};
  T* muf = l == 0 ? (T*)A.muf : (T*)A.lv[l].muf;
  const double h2 = L.h * L.h;
  const long long ni = (long long)(L.g.NN - 1) * (L.g.NN - 1) * (L.g.NN - 1);
  const int last = (int)c->mg.size() - 1;
  if (l == last) {
    const size_t smem = sizeof(double) * 2 * (size_t)L.g.S3;
    CK(cudaFuncSetAttribute(k_adj_coarsest<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    LAUNCH(RQ_KC_MG, 2.0 * sizeof(T) * L.g.S3,
           (k_adj_coarsest<T><<<1, kCoarsestThreads, smem, c->st>>>(mu[*cur], muf, L.g, h2, c->cfg.mg_coarse_sweeps),
            cudaGetLastError()));
    return RQ_OK;
  }
  auto smooth = [&](int sweeps) -> int {
    for (int s = 0; s < sweeps; ++s)
      for (int color = 1; color >= 0; --color) {
        LAUNCH(RQ_KC_MG, 3.5 * sizeof(T) * ni,
               (k_adj_rbgs<T><<<grid3(L.g), kBlk3, 0, c->st>>>(mu[*cur], mu[1 - *cur], muf, L.g, h2, color),
                cudaGetLastError()));
        *cur ^= 1;
      }
    return RQ_OK;
  };
  int rc = smooth(c->cfg.mg_post);
  if (rc != RQ_OK) return rc;
  const rq_mg_level& C = c->mg[l + 1];
  const long long nc = (long long)(C.g.NN - 1) * (C.g.NN - 1) * (C.g.NN - 1);
  int ccur = 0;
  LAUNCH(RQ_KC_MG, sizeof(T) * (ni + nc),
         (k_adj_prolong<T><<<grid3(C.g), kBlk3, 0, c->st>>>(mu[*cur], (T*)A.lv[l + 1].mu[0], L.g, C.g), cudaGetLastError()));
  CK(cudaMemsetAsync(A.lv[l + 1].muf, 0, sizeof(T) * C.g.S3, c->st));
  if ((rc = adj_vcycle<T>(c, l + 1, &ccur)) != RQ_OK) return rc;
  LAUNCH(RQ_KC_MG, sizeof(T) * (ni + nc),
         (k_adj_restrict<T><<<grid3(L.g), kBlk3, 0, c->st>>>((const T*)A.lv[l + 1].muf, (T*)A.lv[l].mur, L.g, C.g),
          cudaGetLastError()));
  LAUNCH(RQ_KC_MG, 5.0 * sizeof(T) * ni,
         (k_adj_residual<T><<<grid3(L.g), kBlk3, 0, c->st>>>((const T*)A.lv[l].mur, mu[*cur], muf, L.g, 1.0 / h2),
          cudaGetLastError()));
  return smooth(c->cfg.mg_pre);
}

template <typename T>
int adjoint_t(rq_ctx* c, double* F, double* dEdv) {
  rq_adj& A = c->adj;
  const int n = c->n_atoms;
  const Geo& g = c->g;
  const long long S3 = g.S3, ni = (long long)(g.NN - 1) * (g.NN - 1) * (g.NN - 1);
  for (const rq_adj::Rec& r : A.rec)
    if (r.label)
      return rq_fail(c, RQ_ENOTSUP,
                     "a label pass ran inside the recorded window: the adjoint holds the labels fixed (set label_until)");
  int rc = nm_ready(c);  // a normalisation it performs is recorded as the last step's
  if (rc != RQ_OK) return rc;
  const T* psi = (const T*)c->U[c->cu];
  const T* K = (const T*)c->K;
  const int* lab = c->lab[c->cl];
  // the readout's per-domain partials -> (Z/N, Q/N)
  CK(cudaMemsetAsync(c->dpd, 0, sizeof(double) * kNmPD * n, c->st));
  LAUNCH(RQ_KC_ENERGY, (4.0 * sizeof(T) + 4.0) * ni,
         nm_energy<T>(psi, K, (const T*)c->P[c->cp], lab, g, c->h, n, c->dpd, c->st, c->K64));
  std::vector<double> pd((size_t)kNmPD * n), wq((size_t)2 * n);
  CK(cudaMemcpyAsync(pd.data(), c->dpd, sizeof(double) * pd.size(), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  for (int d = 0; d < n; ++d) {
    const double* x = &pd[(size_t)kNmPD * d];
    wq[2 * d] = domain_norm_weight(c->atoms[d].Z, x[0]);
    wq[2 * d + 1] = x[0] > 0.0 ? (x[1] + x[2] + 2.0 * x[3]) / x[0] : 0.0;
  }
  CK(cudaMemcpyAsync(A.wq, wq.data(), sizeof(double) * wq.size(), cudaMemcpyHostToDevice, c->st));
  int li = 0, mi = 0;
  T* lam[2] = {(T*)A.lam[0], (T*)A.lam[1]};
  T* muP[2] = {(T*)A.muP[0], (T*)A.muP[1]};
  LAUNCH(RQ_KC_FORCES, (4.0 * sizeof(T) + 4.0 + 2.0 * sizeof(T) + 8.0) * ni,
         (k_adj_seed<T><<<grid3(g), kBlk3, 0, c->st>>>(psi, K, (const T*)c->P[c->cp], lab, g, c->h, n, A.wq, lam[li],
                                                     muP[mi], A.gK, c->K64),
          cudaGetLastError()));
  for (int r = (int)A.rec.size() - 1; r >= 0; --r) {
    const rq_adj::Rec& R = A.rec[r];
    const T* psi_prev = slot<T>(A.psi, R.psi_slot, S3);
    const T* P_s = slot<T>(A.psum, R.p_slot, S3);
    if (R.norm) {
      const T* psi_s = r + 1 < (int)A.rec.size() ? slot<T>(A.psi, A.rec[r + 1].psi_slot, S3) : psi;
      if ((rc = adj_norm<T>(c, psi_s, lam[li], A.scales + (size_t)R.psi_slot * n)) != RQ_OK) return rc;
    }
    LAUNCH(RQ_KC_FORCES, (6.0 * sizeof(T) + 4.0 + 16.0) * ni,
           (k_adj_update<T><<<grid3(g), kBlk3, 0, c->st>>>(lam[li], lam[1 - li], K, P_s, lab, psi_prev, g, c->half_dv,
                                                         c->dt, A.gK, muP[mi]),
            cudaGetLastError()));
    li ^= 1;
    if (R.vcycle) {
      CK(cudaMemsetAsync(A.muf, 0, sizeof(T) * S3, c->st));
      if ((rc = adj_vcycle<T>(c, 0, &mi)) != RQ_OK) return rc;
      LAUNCH(RQ_KC_FORCES, 4.0 * sizeof(T) * ni,
             (k_adj_rhs<T><<<grid3(g), kBlk3, 0, c->st>>>(lam[li], psi_prev, (const T*)A.muf, g), cudaGetLastError()));
    }
  }
  if (F) {
    CK(cudaMemsetAsync(c->dF, 0, sizeof(double) * 3 * n, c->st));
    if ((rc = nm_gather(c, psi, A.gK)) != RQ_OK) return rc;
    CK(cudaMemcpyAsync(F, c->dF, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, c->st));
  }
  if (dEdv) CK(cudaMemcpyAsync(dEdv, A.gK, sizeof(double) * S3, cudaMemcpyDefault, c->st));  // host or device
  CK(cudaStreamSynchronize(c->st));
  return RQ_OK;
}

}  // namespace

int nm_adjoint(rq_ctx* c, double* F, double* dEdv) {
  if (c->adj.cap > 0) return c->fp64 ? adjoint_t<double>(c, F, dEdv) : adjoint_t<float>(c, F, dEdv);
  // no recording window: the gradient of the readout alone (the Hellmann-Feynman terms); the
  // forces alone are the HF gather, dE/dv needs the reverse-sweep buffers for this call
  if (!dEdv) return F ? nm_forces(c, RQ_FORCE_HF, F) : RQ_OK;
  int rc = nm_adj_set_window(c, 1);
  if (rc == RQ_OK) rc = c->fp64 ? adjoint_t<double>(c, F, dEdv) : adjoint_t<float>(c, F, dEdv);
  nm_adj_free(c);
  return rc;
}
