// nm_flavor.cu -- schedule, energies and forces of the new flavour (host side of librq).
//
// Atom list idiom: entries with Z_nuc > 0 are nuclei (Gaussian charge of width sigma), entries
// with Z > 0 are electron domains (their position is the seed of the initial state); labels
// index entries.  One rq_step:
//   every poisson_interval steps one multigrid V-cycle for  -lap P = 2 pi psi^2  (red-black
//     Gauss-Seidel, full weighting, trilinear, coarsest level in FP64);
//   the ITP update psi' = psi + dv/2 lap psi + dt (K - 2P) psi with same-label Neumann faces;
//   every norm_interval steps normalisation to the domain charges (FP64 sums);
//   every label_interval steps the level-set label update (molecule.js:426-540 rule).
// Precision RQ_PREC_MIXED keeps fields in fp32, RQ_PREC_FP64 keeps everything in double.
#include <cmath>
#include <cstring>

#include "rq_flavors.h"
#include "rq_kernels.h"

using namespace rq;

#define CK(call)                                 \
  do {                                           \
    int _rc = rq_cuda(c, (call), #call);         \
    if (_rc != RQ_OK) return _rc;                \
  } while (0)

namespace {
double interior(const Geo& g) {
  const double n = g.NN - 1;
  return n * n * n;
}
size_t esize(const rq_ctx* c) { return c->fp64 ? sizeof(double) : sizeof(float); }
}  // namespace

// the same-label neighbour mask of the current labels (read by the update)
int nm_label_mask(rq_ctx* c) {
  if (!c->nbm) return RQ_OK;
  LAUNCH(RQ_KC_LABELS, 25.0 * c->g.S3, nm_mask(c->lab[c->cl], c->nbm, c->g, c->st));
  return RQ_OK;
}

int nm_alloc_levels(rq_ctx* c) {
  // levels: halve NN while it stays even and the next level keeps NN >= 6, or mg_levels if set
  int levels = 1, NN = c->g.NN;
  const int want = c->cfg.mg_levels;
  while (NN % 2 == 0 && (want > 0 ? levels < want : NN / 2 >= 6)) {
    NN /= 2;
    levels++;
  }
  if (want > 0 && levels != want) return rq_fail(c, RQ_EINVAL, "NN cannot be halved mg_levels-1 times");
  if (levels < 2) return rq_fail(c, RQ_EINVAL, "multigrid needs NN divisible by 2");
  if ((long long)(NN + 1) * (NN + 1) * (NN + 1) * 16 > 200 * 1024)
    return rq_fail(c, RQ_EINVAL, "coarsest multigrid level too large for the FP64 shared-memory solve (NN/2^k > 28)");
  c->mg.assign(levels, rq_mg_level());
  const size_t es = esize(c);
  double h = c->h;
  int nn = c->g.NN;
  for (int l = 0; l < levels; ++l) {
    rq_mg_level& L = c->mg[l];
    L.g = make_geo(nn + 1);
    L.h = h;
    const size_t n = (size_t)L.g.S3 * es;
    if (l > 0) {
      if (cudaMalloc(&L.P, n) != cudaSuccess || cudaMalloc(&L.f, n) != cudaSuccess)
        return rq_cuda(c, cudaErrorMemoryAllocation, "multigrid levels");
      cudaMemsetAsync(L.P, 0, n, c->st);
      cudaMemsetAsync(L.f, 0, n, c->st);
    }
    h *= 2;
    nn /= 2;
  }
  if (cudaMalloc(&c->seeds, sizeof(float4) * c->n_atoms) != cudaSuccess ||
      cudaMalloc(&c->scale64, sizeof(double) * c->n_atoms) != cudaSuccess ||
      cudaMalloc((void**)&c->rseed, sizeof(unsigned) * 2) != cudaSuccess ||
      cudaMalloc((void**)&c->nbm, (size_t)c->g.S3) != cudaSuccess)
    return rq_cuda(c, cudaErrorMemoryAllocation, "seed table");
  cudaMemsetAsync(c->rseed, 0, sizeof(unsigned) * 2, c->st);
  if (!c->fp64 && cudaMalloc((void**)&c->K64, sizeof(double) * (size_t)c->g.S3) != cudaSuccess)
    return rq_cuda(c, cudaErrorMemoryAllocation, "FP64 potential of the readout");
  return RQ_OK;
}

template <typename T>
static int vcycle_level(rq_ctx* c, int l) {
  rq_mg_level& L = c->mg[l];
  const bool fine = l == 0;
  T* P = fine ? (T*)c->P[c->cp] : (T*)L.P;
  const T* f = fine ? (const T*)c->U[c->cu] : (const T*)L.f;
  const double h2 = L.h * L.h;
  const double ip = interior(L.g);
  const int last = (int)c->mg.size() - 1;
  if (l == last) {
    LAUNCH(RQ_KC_MG, 2.0 * sizeof(T) * L.g.S3, nm_coarsest<T>(P, f, L.g, h2, c->cfg.mg_coarse_sweeps, c->st));
    return RQ_OK;
  }
  const int kc = fine ? RQ_KC_POISSON : RQ_KC_MG;
  for (int s = 0; s < c->cfg.mg_pre; ++s)
    for (int color = 0; color < 2; ++color)
      LAUNCH(kc, sizeof(T) * 2.5 * ip, nm_rbgs<T>(P, f, fine, L.g, h2, color, c->st));
  // the residual, its full weighting and the cleared coarse correction in one pass (the coarse
  // boundary stays zero from the allocation)
  rq_mg_level& C = c->mg[l + 1];
  LAUNCH(kc, sizeof(T) * (2.0 * ip + 2.0 * interior(C.g)),
         nm_resrestrict<T>(P, f, fine, (T*)C.f, (T*)C.P, L.g, C.g, 1.0 / h2, c->st));
  int rc = vcycle_level<T>(c, l + 1);
  if (rc != RQ_OK) return rc;
  LAUNCH(RQ_KC_MG, sizeof(T) * (2.0 * ip + interior(C.g)), nm_prolong<T>((const T*)C.P, P, L.g, C.g, c->st));
  for (int s = 0; s < c->cfg.mg_post; ++s)
    for (int color = 0; color < 2; ++color)
      LAUNCH(kc, sizeof(T) * 2.5 * ip, nm_rbgs<T>(P, f, fine, L.g, h2, color, c->st));
  return RQ_OK;
}

static int nm_vcycle(rq_ctx* c) { return c->fp64 ? vcycle_level<double>(c, 0) : vcycle_level<float>(c, 0); }

template <typename T>
static int nm_normalize_t(rq_ctx* c, bool accumulate) {
  T* U = (T*)c->U[c->cu];
  if (accumulate) {
    CK(cudaMemsetAsync(c->dnorm, 0, sizeof(double) * c->n_atoms, c->st));
    LAUNCH(RQ_KC_NORMALIZE, (sizeof(T) + 4.0) * c->g.S3, nm_norms<T>(U, c->lab[c->cl], c->g, c->h3, c->n_atoms, c->dnorm, c->st));
  }
  LAUNCH(RQ_KC_NORMALIZE, (2.0 * sizeof(T) + 4.0) * c->g.S3,
         nm_normalize<T>(U, c->lab[c->cl], c->dnorm, c->Zdom64, c->n_atoms, (double*)c->scale64, c->err, c->g, c->st));
  c->nm_pending = false;
  c->nm_age = 0;
  return RQ_OK;
}

// Apply a pending per-domain normalisation to the stored psi (the update applies it on the
// fly; the multigrid, the label pass and every readout need it materialised).
template <typename T>
static int nm_flush_t(rq_ctx* c) {
  if (!c->nm_pending) return RQ_OK;
  LAUNCH(RQ_KC_NORMALIZE, (2.0 * sizeof(T) + 4.0) * c->g.S3,
         nm_apply<T>((T*)c->U[c->cu], c->lab[c->cl], (const double*)c->scale64, c->n_atoms, c->g, c->st));
  c->nm_pending = false;
  return RQ_OK;
}

int nm_flush(rq_ctx* c) { return c->fp64 ? nm_flush_t<double>(c) : nm_flush_t<float>(c); }

// Bring psi to the normalised state that every readout reports: apply a pending scale, or, when
// updates ran since the last normalisation, normalise now.
template <typename T>
static int nm_ready_t(rq_ctx* c) {
  if (c->nm_age == 0) return nm_flush_t<T>(c);
  int rc = nm_normalize_t<T>(c, true);
  c->nm_age = 0;
  // a readout that normalises changes the state the energy is read from: while steps are
  // recorded it becomes the normalisation of the last recorded step, for the reverse sweep
  if (rc == RQ_OK && c->adj.cap > 0 && !c->adj.rec.empty() && !c->adj.rec.back().norm) {
    c->adj.rec.back().norm = true;
    rc = nm_adj_record_scale(c);
  }
  return rc;
}

int nm_ready(rq_ctx* c) { return c->fp64 ? nm_ready_t<double>(c) : nm_ready_t<float>(c); }

template <typename T>
static int nm_step_t(rq_ctx* c, int s) {
  const rq_config& f = c->cfg;
  int rc;
  if (s % f.poisson_interval == 0) {
    if ((rc = nm_flush_t<T>(c)) != RQ_OK) return rc;
    if ((rc = nm_vcycle(c)) != RQ_OK) return rc;
  }
  // The update is linear in psi and couples only points of one domain, so between two Poisson
  // solves a per-domain scale commutes with it: normalising every step or once before the next
  // V-cycle / label pass gives the same psi there.  Normalise after every norm_interval-th update
  // and always after the update that precedes a V-cycle or ends with a label pass.
  const bool label_step = s % f.label_interval == 0 && (f.label_until <= 0 || s <= f.label_until);
  const bool norm = (s + 1) % f.norm_interval == 0 || (s + 1) % f.poisson_interval == 0 || label_step;
  if (c->adj.cap > 0 && (rc = nm_adj_record_step(c, s % f.poisson_interval == 0, norm)) != RQ_OK) return rc;
  if (norm) CK(cudaMemsetAsync(c->dnorm, 0, sizeof(double) * c->n_atoms, c->st));
  const bool sr = !c->fp64 && f.fp32_rounding == 1;
  // bytes: psi, K, P read, psi' written, the neighbour mask; the centre label where it is needed
  LAUNCH(RQ_KC_UPDATE, (4.0 * sizeof(T) + 1.0 + ((norm || c->nm_pending) ? 4.0 : 0.0)) * interior(c->g),
         nm_update<T>((const T*)c->U[c->cu], (T*)c->U[1 - c->cu], (const T*)c->K, (const T*)c->P[c->cp], c->lab[c->cl],
                      c->g, (T)c->half_dv, (T)c->dt, c->h3, c->n_atoms, norm ? c->dnorm : nullptr, c->st,
                      c->nm_pending ? (const double*)c->scale64 : nullptr, sr ? c->rseed + c->cu : nullptr,
                      sr ? c->rseed + (1 - c->cu) : nullptr, c->nbm));
  c->cu ^= 1;
  c->nm_pending = false;  // the update consumed the pending scale
  if (norm) {  // the scale of this step is applied by the next update (or a flush)
    LAUNCH(RQ_KC_NORMALIZE, 12.0 * c->n_atoms,
           nm_norm_scale<T>(c->dnorm, c->Zdom64, c->n_atoms, (double*)c->scale64, c->err, c->st));
    c->nm_pending = true;
    if (c->adj.cap > 0 && (rc = nm_adj_record_scale(c)) != RQ_OK) return rc;
  }
  c->nm_age = norm ? 0 : c->nm_age + 1;
  if (label_step) {
    if ((rc = nm_flush_t<T>(c)) != RQ_OK) return rc;
    LAUNCH(RQ_KC_LABELS, (sizeof(T) + 12.0) * interior(c->g),
           nm_evolve<T>(c->lab[c->cl], c->lab[1 - c->cl], (const T*)c->U[c->cu], c->W, c->g, f.boundary_speed, f.curv_reg,
                        c->st));
    c->cl ^= 1;
    if ((rc = nm_label_mask(c)) != RQ_OK) return rc;
    if (c->adj.cap > 0) nm_adj_record_label(c);
  }
  return RQ_OK;
}

int nm_step_one(rq_ctx* c, int s) { return c->fp64 ? nm_step_t<double>(c, s) : nm_step_t<float>(c, s); }

__global__ void __launch_bounds__(256) k_nm_add_f2d(double* __restrict__ K, const float* __restrict__ v, long long n) {
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    K[q] += (double)v[q];
}

template <typename T>
static int nm_potential_t(rq_ctx* c) {
  // fp32 fields: the readout's FP64 copy comes from the same pass
  double* K64 = (!c->fp64 && c->K64) ? c->K64 : nullptr;
  int rc = nm_nuclear_potential(c, c->K, K64);
  if (rc != RQ_OK) return rc;
  if (c->Kext) LAUNCH(RQ_KC_OTHER, 3.0 * sizeof(T) * c->g.S3, nm_add<T>((T*)c->K, (const T*)c->Kext, c->g.S3, c->st));
  if (K64) {
    if (c->Kext)
      LAUNCH(RQ_KC_OTHER, 20.0 * c->g.S3,
             (k_nm_add_f2d<<<148 * 8, 256, 0, c->st>>>(c->K64, (const float*)c->Kext, c->g.S3), cudaGetLastError()));
  }
  return RQ_OK;
}

__global__ void __launch_bounds__(256) k_nm_narrow(const double* __restrict__ d, float* __restrict__ a, long long n) {
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    a[q] = (float)d[q];
}

// v: S^3 doubles in host memory or in device memory of this GPU (a device pointer stays on the
// device: no round trip through the host)
int nm_set_external(rq_ctx* c, const double* v) {
  const size_t n = (size_t)c->g.S3;
  if (!v) {
    if (c->Kext) { cudaFree(c->Kext); c->Kext = nullptr; }
  } else {
    if (!c->Kext && cudaMalloc(&c->Kext, n * esize(c)) != cudaSuccess)
      return rq_cuda(c, cudaErrorMemoryAllocation, "external potential");
    cudaPointerAttributes pa{};
    const bool on_device = cudaPointerGetAttributes(&pa, v) == cudaSuccess &&
                           (pa.type == cudaMemoryTypeDevice || pa.type == cudaMemoryTypeManaged);
    cudaGetLastError();  // a plain host pointer may leave an error behind on older drivers
    if (c->fp64) {
      CK(cudaMemcpyAsync(c->Kext, v, n * sizeof(double), cudaMemcpyDefault, c->st));
    } else if (on_device) {
      k_nm_narrow<<<148 * 8, 256, 0, c->st>>>(v, (float*)c->Kext, (long long)n);
      CK(cudaGetLastError());
      c->launches++;
    } else {
      std::vector<float> f(n);
      for (size_t q = 0; q < n; ++q) f[q] = (float)v[q];
      CK(cudaMemcpyAsync(c->Kext, f.data(), n * sizeof(float), cudaMemcpyHostToDevice, c->st));
      CK(cudaStreamSynchronize(c->st));
    }
  }
  return nm_set_atoms(c);  // K = K_nuclei (+ v)
}

int nm_set_atoms(rq_ctx* c) {
  nm_adj_reset(c);  // the recorded steps ran with the old K
  return c->fp64 ? nm_potential_t<double>(c) : nm_potential_t<float>(c);
}

template <typename T>
static int nm_init_t(rq_ctx* c) {
  const size_t n = (size_t)c->g.S3;
  c->cu = c->cp = c->cl = 0;
  int rc = nm_potential_t<T>(c);
  if (rc != RQ_OK) return rc;
  std::vector<float4> seeds;
  for (int q = 0; q < c->n_atoms; ++q) {
    const rq_atom& a = c->atoms[q];
    if (a.Z <= 0) continue;
    float4 s;
    s.x = (float)(a.i * c->h); s.y = (float)(a.j * c->h); s.z = (float)(a.k * c->h);
    int idx = q;
    std::memcpy(&s.w, &idx, sizeof(int));
    seeds.push_back(s);
  }
  if (seeds.empty()) return rq_fail(c, RQ_EINVAL, "the new flavour needs at least one entry with Z > 0 (a domain)");
  CK(cudaMemcpyAsync(c->seeds, seeds.data(), sizeof(float4) * seeds.size(), cudaMemcpyHostToDevice, c->st));
  LAUNCH(RQ_KC_OTHER, (sizeof(T) + 4.0) * n,
         nm_init<T>((T*)c->U[0], c->lab[0], (const float4*)c->seeds, (int)seeds.size(), c->g, (float)c->h, c->st));
  CK(cudaMemcpyAsync(c->lab[1], c->lab[0], n * sizeof(int), cudaMemcpyDeviceToDevice, c->st));
  if ((rc = nm_label_mask(c)) != RQ_OK) return rc;
  CK(cudaMemsetAsync(c->U[1], 0, n * sizeof(T), c->st));
  for (int b = 0; b < 2; ++b) CK(cudaMemsetAsync(c->P[b], 0, n * sizeof(T), c->st));
  LAUNCH(RQ_KC_OTHER, 4.0 * n, launch_fill(c->W, 1.0f, c->g.S3, c->st));
  if ((rc = nm_normalize_t<T>(c, true)) != RQ_OK) return rc;
  for (int v = 0; v < 10; ++v)  // converge the initial Hartree potential
    if ((rc = nm_vcycle(c)) != RQ_OK) return rc;
  return RQ_OK;
}

int nm_initialize(rq_ctx* c) {
  nm_adj_reset(c);
  return c->fp64 ? nm_init_t<double>(c) : nm_init_t<float>(c);
}

__global__ void __launch_bounds__(256) k_nm_widen(const float* __restrict__ a, double* __restrict__ d, long long n) {
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    d[q] = (double)a[q];
}

// Switch a mixed-precision context to FP64 in place, keeping the state it holds: psi (after its
// pending normalisation) and P are widened, K is recomputed in FP64, the multigrid levels are
// reallocated in FP64 and the captured schedule graphs are dropped.  fp32 fields stop resolving
// the energy at a few 1e-8 |E| (updates below half an ulp round away); continuing in FP64 from
// there reaches the FP64 fixed point.
int nm_promote(rq_ctx* c) {
  if (c->fp64) return RQ_OK;
  int rc = nm_flush(c);
  if (rc != RQ_OK) return rc;
  const long long n = c->g.S3;
  const size_t bytes = sizeof(double) * (size_t)n;
  // Every FP64 buffer (fields and multigrid levels) is allocated before anything is freed or
  // swapped: if one allocation fails the context is left exactly as it was (fp32, its captured
  // graphs still valid).
  void* nb[6] = {};  // U0, U1, P0, P1, K, Kext
  void* old[6] = {c->U[0], c->U[1], c->P[0], c->P[1], c->K, c->Kext};
  std::vector<void*> lv;  // new multigrid buffers, in the order of the (L.P, L.f) walk below
  auto undo = [&]() {
    for (void* p : nb)
      if (p) cudaFree(p);
    for (void* p : lv)
      if (p) cudaFree(p);
  };
  for (int q = 0; q < 6; ++q)
    if (old[q] && cudaMalloc(&nb[q], bytes) != cudaSuccess) {
      undo();
      return rq_cuda(c, cudaErrorMemoryAllocation, "promotion to FP64");
    }
  for (const rq_mg_level& L : c->mg)
    for (void* p : {L.P, L.f}) {
      if (!p) continue;
      void* q = nullptr;
      if (cudaMalloc(&q, sizeof(double) * (size_t)L.g.S3) != cudaSuccess) {
        undo();
        return rq_cuda(c, cudaErrorMemoryAllocation, "FP64 multigrid levels");
      }
      lv.push_back(q);
    }
  for (int q = 0; q < 6; ++q)
    if (old[q] && q != 4) {  // K is recomputed below
      k_nm_widen<<<148 * 4, 256, 0, c->st>>>((const float*)old[q], (double*)nb[q], n);
      const cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) {
        cudaStreamSynchronize(c->st);
        undo();
        return rq_cuda(c, e, "promotion to FP64");
      }
      c->launches++;
    }
  size_t li = 0;
  for (const rq_mg_level& L : c->mg)
    for (void* p : {L.P, L.f})
      if (p) cudaMemsetAsync(lv[li++], 0, sizeof(double) * (size_t)L.g.S3, c->st);
  if (cudaStreamSynchronize(c->st) != cudaSuccess) {
    const cudaError_t e = cudaGetLastError();
    undo();
    return rq_cuda(c, e, "promotion to FP64");
  }
  // commit: free the fp32 buffers and swap in the FP64 ones
  for (void* p : old)
    if (p) cudaFree(p);
  c->U[0] = nb[0]; c->U[1] = nb[1]; c->P[0] = nb[2]; c->P[1] = nb[3]; c->K = nb[4]; c->Kext = nb[5];
  li = 0;
  for (rq_mg_level& L : c->mg)
    for (void** p : {&L.P, &L.f})
      if (*p) {
        cudaFree(*p);
        *p = lv[li++];
      }
  c->fp64 = true;
  for (auto& gx : c->graph)
    if (gx) {
      cudaGraphExecDestroy(gx);
      gx = nullptr;
    }
  if ((rc = nm_potential_t<double>(c)) != RQ_OK) return rc;
  if (c->K64) {  // the fields are FP64 now: K itself is the readout's potential
    cudaFree(c->K64);
    c->K64 = nullptr;
  }
  if (c->adj.cap > 0 && (rc = nm_adj_set_window(c, c->adj.cap)) != RQ_OK) return rc;  // FP64 window buffers
  return cudaStreamSynchronize(c->st) == cudaSuccess ? RQ_OK : rq_cuda(c, cudaGetLastError(), "promotion to FP64");
}

// Point-charge nuclear repulsion between entries with Z_nuc > 0 (bohr): thread a sums over all b
// != a (each pair enters twice; the energy is half the per-entry sums, added in entry order).
__global__ void __launch_bounds__(256) k_nm_nuclear(const double* __restrict__ at, int n, double* __restrict__ out) {
  __shared__ double sa[256 * 4];
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = a < n && at[a * 4 + 3] > 0.0;
  const double X = valid ? at[a * 4] : 0.0, Y = valid ? at[a * 4 + 1] : 0.0, Z = valid ? at[a * 4 + 2] : 0.0;
  const double Za = valid ? at[a * 4 + 3] : 0.0;
  double e = 0, fx = 0, fy = 0, fz = 0;
  for (int base = 0; base < n; base += 256) {
    const int cnt = min(256, n - base);
    __syncthreads();
    for (int q = threadIdx.x; q < cnt * 4; q += blockDim.x) sa[q] = at[base * 4 + q];
    __syncthreads();
    if (!valid) continue;
    for (int m = 0; m < cnt; ++m) {
      const double Zb = sa[m * 4 + 3];
      if (Zb <= 0.0 || base + m == a) continue;
      const double dx = X - sa[m * 4], dy = Y - sa[m * 4 + 1], dz = Z - sa[m * 4 + 2];
      const double r2 = dx * dx + dy * dy + dz * dz, r = sqrt(r2), zz = Za * Zb;
      e += zz / r;
      const double w = zz / (r2 * r);
      fx += w * dx; fy += w * dy; fz += w * dz;
    }
  }
  if (a < n) { out[a * 4] = e; out[a * 4 + 1] = fx; out[a * 4 + 2] = fy; out[a * 4 + 3] = fz; }
}

int nm_nuclear_terms(rq_ctx* c, double* E, double* F) {
  const int n = c->n_atoms;
  *E = 0;
  if (n <= 0) return RQ_OK;
  LAUNCH(RQ_KC_FORCES, 32.0 * n, (k_nm_nuclear<<<(n + 255) / 256, 256, 0, c->st>>>(c->atoms_nm, n, c->dpd),
                                  cudaGetLastError()));
  std::vector<double> o((size_t)4 * n);
  CK(cudaMemcpyAsync(o.data(), c->dpd, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  double e = 0;
  for (int a = 0; a < n; ++a) {
    e += o[a * 4];
    F[a * 3] += o[a * 4 + 1]; F[a * 3 + 1] += o[a * 4 + 2]; F[a * 3 + 2] += o[a * 4 + 3];
  }
  *E = 0.5 * e;
  return RQ_OK;
}

// The readout.  Per domain d with norm N_d and charge Z_d the state is read as if exactly
// normalised (weight w_d = Z_d / N_d on its kinetic and nuclear terms, which are linear in its
// density).  The Hartree energy is the P-stationary form
//     E_ee = 2 sum_d w_d h^3 sum_{i in d} P_i rho_i  -  (h^3 / 2 pi) sum_i P_i (A P)_i,
// A = -lap_h with Dirichlet faces: it equals h^3 sum P rho when A P = 2 pi rho (the discrete Poisson
// equation the multigrid solves) and differs from it only at second order in the error of P.  So the
// readout does not follow the lag of P behind psi, nor the error left in P by fp32 fields at first
// order: the mixed path reads within ~4e-8 Ha of the FP64 path on the same method (glycine, 128^3),
// against ~9e-6 Ha with h^3 sum P rho.
int nm_energy(rq_ctx* c, double* out, double* per_domain) {
  const int n = c->n_atoms;
  int frc = nm_ready(c);
  if (frc != RQ_OK) return frc;
  CK(cudaMemsetAsync(c->dpd, 0, sizeof(double) * kNmPD * n, c->st));
  if (c->fp64)
    LAUNCH(RQ_KC_ENERGY, 36 * interior(c->g),
           nm_energy<double>((const double*)c->U[c->cu], (const double*)c->K, (const double*)c->P[c->cp], c->lab[c->cl],
                             c->g, c->h, n, c->dpd, c->st));
  else
    LAUNCH(RQ_KC_ENERGY, 16 * interior(c->g),
           nm_energy<float>((const float*)c->U[c->cu], (const float*)c->K, (const float*)c->P[c->cp], c->lab[c->cl],
                            c->g, c->h, n, c->dpd, c->st, c->K64));
  std::vector<double> pd((size_t)kNmPD * n);
  CK(cudaMemcpyAsync(pd.data(), c->dpd, sizeof(double) * kNmPD * n, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  double T = 0, EK = 0, EE = 0;
  for (int q = 0; q < n; ++q) {
    const double* x = &pd[(size_t)q * kNmPD];
    const double w = domain_norm_weight(c->atoms[q].Z, x[0]);
    const double t = w * x[1], ek = w * x[2], ee = 2.0 * w * x[3] - x[4] / (2.0 * M_PI);
    T += t; EK += ek; EE += ee;
    if (per_domain) {  // the domain's share of the readout; the eigenvalue from its own potential
      double* d = per_domain + (size_t)q * RQ_DOMAIN_LEN;
      d[RQ_D_NORM] = x[0]; d[RQ_D_T] = t; d[RQ_D_EK] = ek; d[RQ_D_EE] = ee;
      const double nr = c->atoms[q].Z > 0 ? c->atoms[q].Z : (x[0] != 0 ? x[0] : 1.0);
      d[RQ_D_EIG] = (t + ek + 2.0 * w * x[3]) / nr;
    }
  }
  out[RQ_E_T] = T; out[RQ_E_EK] = EK; out[RQ_E_EE] = EE;
  return RQ_OK;
}

int nm_forces(rq_ctx* c, int method, double* F) {
  if (method != RQ_FORCE_HF && method != RQ_FORCE_ADJOINT) return RQ_ENOTSUP;
  // the adjoint through the recorded window; with no window it is the Hellmann-Feynman gather
  if (method == RQ_FORCE_ADJOINT && c->adj.cap > 0) return nm_adjoint(c, F, nullptr);
  const int n = c->n_atoms;
  int frc = nm_ready(c);
  if (frc != RQ_OK) return frc;
  CK(cudaMemsetAsync(c->dF, 0, sizeof(double) * 3 * n, c->st));
  if ((frc = nm_gather(c, c->U[c->cu], nullptr)) != RQ_OK) return frc;
  CK(cudaMemcpyAsync(F, c->dF, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return RQ_OK;
}
