// capi.cu -- the C ABI of librq (include/rq.h): context lifecycle, state transfer, the
// per-flavour step schedule (captured as CUDA graphs), energies and forces.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>

#include "rq_ctx.h"
#include "rq_flavors.h"

using namespace rq;

int rq_fail(rq_ctx* c, int code, const std::string& msg) {
  if (c) c->last_error = msg;
  return code;
}

int rq_cuda(rq_ctx* c, cudaError_t e, const char* where) {
  if (e == cudaSuccess) return RQ_OK;
  if (c) c->last_error = std::string(where) + ": " + cudaGetErrorString(e);
  if (e == cudaErrorMemoryAllocation) return RQ_ENOMEM;
  return RQ_ECUDA;
}

#define CK(call)                                        \
  do {                                                  \
    int _rc = rq_cuda(c, (call), #call);                \
    if (_rc != RQ_OK) return _rc;                       \
  } while (0)

static const char* kStatus[] = {"ok", "invalid argument", "out of memory", "CUDA error",
                                "non-finite value", "device wait timed out", "not supported", "no CUDA device"};

extern "C" const char* rq_status_string(int s) {
  if (s > 0 || s < -7) return "unknown status";
  return kStatus[-s];
}

extern "C" const char* rq_last_error(const rq_ctx* c) { return c ? c->last_error.c_str() : "null context"; }

// ----------------------------------------------------------------------------------------
// defaults per flavour
// ----------------------------------------------------------------------------------------
static int count_domains(const std::vector<rq_atom>& a) {
  int n = 0;
  for (auto& x : a) n += (x.Z > 0);
  return n;
}

static double default_dv(const rq_ctx* c) {
  const int ne = count_domains(c->atoms);
  switch (c->cfg.flavor) {
    case RQ_FLAVOR_SOLVER_PY:  // cloud/solver.py:342-351
      return ne > 500 ? 0.005 : ne > 200 ? 0.01 : ne > 100 ? 0.02 : ne > 30 ? 0.03 : 0.12;
    case RQ_FLAVOR_MOLECULE_JS: {  // molecule.js:12-17 NELEC counts Z>0 or Z_nuc>0 entries, :78
      int nel = 0;
      for (auto& x : c->atoms) nel += (x.Z > 0 || x.Z_nuc > 0);
      return nel > 500 ? 0.01 : nel > 100 ? 0.03 : 0.12;
    }
    default:
      return 0.2;  // dt = 0.2 h^2
  }
}

static void fill_defaults(rq_ctx* c) {
  rq_config& f = c->cfg;
  const bool sp = f.flavor == RQ_FLAVOR_SOLVER_PY, mj = f.flavor == RQ_FLAVOR_MOLECULE_JS;
  const bool nm = f.flavor == RQ_FLAVOR_NEW;
  // the new flavour normalises every step: all-electron cores grow by e^{dt |eps|} per step
  if (f.norm_interval <= 0) f.norm_interval = nm ? (f.poisson_interval > 0 ? f.poisson_interval : 4) : 20;
  // new flavour: one V(1,1) every 4 steps (the Hartree potential changes slowly; measured to
  // leave the iteration count and the converged energy unchanged against V(2,2) every 2 steps)
  if (f.poisson_interval <= 0) f.poisson_interval = nm ? 4 : sp ? 2 : 1;
  if (f.label_interval <= 0) f.label_interval = sp ? 5 * f.norm_interval : 20;
  if (f.jacobi_per_step <= 0) f.jacobi_per_step = 2;
  if (f.steps_per_frame <= 0) {  // molecule.js:106
    int nel = 0;
    for (auto& x : c->atoms) nel += (x.Z > 0 || x.Z_nuc > 0);
    f.steps_per_frame = nel <= 30 ? 50 : nel <= 100 ? 5 : 2;
  }
  if (f.vcycle_interval <= 0) f.vcycle_interval = 50;
  if (f.mg_pre <= 0) f.mg_pre = nm ? 1 : 2;
  if (f.mg_post <= 0) f.mg_post = nm ? 1 : 2;
  if (f.mg_coarse_sweeps <= 0) f.mg_coarse_sweeps = 16;
  if (f.boundary_speed <= 0) f.boundary_speed = 0.5;
  if (f.curv_reg == 0) f.curv_reg = 0.15;  // molecule.js:34 default; a negative value switches it off
  if (f.curv_reg < 0) f.curv_reg = 0;
  c->dv = f.dv > 0 ? f.dv : default_dv(c);
  c->half_dv = 0.5 * c->dv;
  c->dt = c->dv * c->h2;
  c->sigma = f.sigma > 0 ? f.sigma : c->h;
}

// ----------------------------------------------------------------------------------------
// atoms -> device tables
// ----------------------------------------------------------------------------------------
static int upload_atoms(rq_ctx* c) {
  const int n = c->n_atoms;
  std::vector<float> a5((size_t)n * 5), zd(n);
  std::vector<double> zd64(n), nm((size_t)n * 4);
  std::vector<MjAtom> mj(n);
  for (int q = 0; q < n; ++q) {
    const rq_atom& a = c->atoms[q];
    a5[q * 5 + 0] = (float)a.i; a5[q * 5 + 1] = (float)a.j; a5[q * 5 + 2] = (float)a.k;
    a5[q * 5 + 3] = (float)a.Z; a5[q * 5 + 4] = (float)a.rc;
    zd[q] = (float)a.Z; zd64[q] = a.Z;
    mj[q] = mj_record(a);
    nm[q * 4 + 0] = a.i * c->h; nm[q * 4 + 1] = a.j * c->h; nm[q * 4 + 2] = a.k * c->h; nm[q * 4 + 3] = a.Z_nuc;
  }
  CK(cudaMemcpyAsync(c->atoms5, a5.data(), sizeof(float) * a5.size(), cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->Zdom, zd.data(), sizeof(float) * n, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->Zdom64, zd64.data(), sizeof(double) * n, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->atoms_mj, mj.data(), sizeof(MjAtom) * n, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->atoms_nm, nm.data(), sizeof(double) * nm.size(), cudaMemcpyHostToDevice, c->st));
  std::vector<int> bstart, bidx, bfar;
  float zmax = 0.f;
  if (c->bin_start) {
    build_atom_bins(a5.data(), n, c->bins_nb, c->bins_bin, bstart, bidx, bfar, zmax);
    CK(cudaMemcpyAsync(c->bin_start, bstart.data(), sizeof(int) * bstart.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->bin_idx, bidx.data(), sizeof(int) * bidx.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->bin_far, bfar.data(), sizeof(int) * bfar.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->bin_zmax, &zmax, sizeof(float), cudaMemcpyHostToDevice, c->st));
  }
  return cudaStreamSynchronize(c->st) == cudaSuccess ? RQ_OK : rq_cuda(c, cudaGetLastError(), "upload_atoms");
}

static void free_ctx(rq_ctx* c) {
  nm_adj_free(c);
  nm_ff_free(c);
  for (auto e : c->evpool) cudaEventDestroy(e);
  for (auto& gx : c->graph)
    if (gx) cudaGraphExecDestroy(gx);
  void* ptrs[] = {c->U[0], c->U[1], c->P[0], c->P[1], c->K, c->W, c->bestU, c->rho, c->Pother, c->resid, c->lab[0], c->lab[1],
                  c->Ec[0], c->Ec[1], c->fc, c->atoms5, c->scratch_atoms5, c->sic, c->sic2, c->pdirect, c->lob, c->lob_part, c->lob_scal, c->lock, c->splits, c->bin_start, c->bin_idx, c->bin_far, c->bin_zmax, c->atoms_mj, c->atoms_nm, c->Zdom, c->Zdom64, c->dnorm,
                  c->dpd, c->dF, c->dsum, c->unorm, c->scale, c->err, c->seeds, c->scale64, c->Kext, c->rseed, c->K64, c->nbm};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (auto& L : c->mg) {
    if (L.P) cudaFree(L.P);
    if (L.f) cudaFree(L.f);
  }
  if (c->own_st) cudaStreamDestroy(c->own_st);
}

static int dalloc(rq_ctx* c, void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) return rq_cuda(c, e, "cudaMalloc");
  e = cudaMemsetAsync(*p, 0, bytes, c->st);
  return rq_cuda(c, e, "cudaMemsetAsync");
}
#define DALLOC(ptr, bytes)                                        \
  do {                                                            \
    int _r = dalloc(c, (void**)&(ptr), (bytes));                  \
    if (_r != RQ_OK) return _r;                                   \
  } while (0)

static int alloc_all(rq_ctx* c) {
  const size_t S3 = (size_t)c->g.S3;
  const size_t es = c->fp64 ? sizeof(double) : sizeof(float);
  const int n = c->n_atoms;
  for (int b = 0; b < 2; ++b) {
    DALLOC(c->U[b], S3 * es);
    DALLOC(c->P[b], S3 * es);
    DALLOC(c->lab[b], S3 * sizeof(int));
  }
  DALLOC(c->K, S3 * es);
  DALLOC(c->W, S3 * sizeof(float));
  if (c->cfg.flavor == RQ_FLAVOR_SOLVER_PY || c->cfg.flavor == RQ_FLAVOR_MOLECULE_JS) DALLOC(c->bestU, S3 * sizeof(float));
  if (c->cfg.flavor == RQ_FLAVOR_MOLECULE_JS) {
    DALLOC(c->rho, S3 * sizeof(float));
    DALLOC(c->Pother, S3 * sizeof(float));
    DALLOC(c->resid, S3 * sizeof(float));
    if (c->cfg.sic) {
      DALLOC(c->sic, S3 * sizeof(float));
      DALLOC(c->sic2, S3 * sizeof(float));
      if (mj_direct(c)) DALLOC(c->pdirect, S3 * sizeof(float) * n);
    }
    DALLOC(c->lock, sizeof(unsigned long long) * n);
    DALLOC(c->splits, sizeof(MjSplit) * n);
    if (c->cfg.lobpcg) {
      DALLOC(c->lob, S3 * sizeof(float) * 5);
      DALLOC(c->lob_part, sizeof(float) * kLobMaxWG * kLobNR);
      DALLOC(c->lob_scal, sizeof(float) * kLobScal);
    }
    const int SC = c->g.NN / 2 + 1;
    c->gc = make_geo(SC);
    const size_t SC3 = (size_t)c->gc.S3;
    DALLOC(c->Ec[0], SC3 * sizeof(float));
    DALLOC(c->Ec[1], SC3 * sizeof(float));
    DALLOC(c->fc, SC3 * sizeof(float));
  }
  DALLOC(c->atoms5, sizeof(float) * 5 * n);
  DALLOC(c->scratch_atoms5, sizeof(float) * 5 * n);
  if (c->cfg.flavor == RQ_FLAVOR_SOLVER_PY) {  // bins of ~1 atom each, at most 64 per axis
    const int S = c->g.S;
    int bin = (int)std::lround(std::cbrt((double)c->g.S3 / std::max(1, n)));
    bin = std::max({bin, 4, (S + 63) / 64});
    c->bins_bin = bin;
    c->bins_nb = (S + bin - 1) / bin;
    DALLOC(c->bin_start, sizeof(int) * ((size_t)c->bins_nb * c->bins_nb * c->bins_nb + 1));
    DALLOC(c->bin_idx, sizeof(int) * n);
    DALLOC(c->bin_far, sizeof(int) * (n + 1));
    DALLOC(c->bin_zmax, sizeof(float));
  }
  DALLOC(c->atoms_mj, sizeof(MjAtom) * n);
  DALLOC(c->atoms_nm, sizeof(double) * 4 * n);
  DALLOC(c->Zdom, sizeof(float) * n);
  DALLOC(c->Zdom64, sizeof(double) * n);
  DALLOC(c->dnorm, sizeof(double) * n);
  DALLOC(c->dpd, sizeof(double) * 5 * n);  // 4 sums per domain (solver.py), 5 (new flavour)
  DALLOC(c->dF, sizeof(double) * 3 * n);
  DALLOC(c->dsum, sizeof(double) * 8);
  DALLOC(c->unorm, sizeof(unsigned) * n);
  DALLOC(c->scale, sizeof(float) * n);
  DALLOC(c->err, sizeof(int) * 4);
  if (c->cfg.flavor == RQ_FLAVOR_NEW) {
    int r = nm_alloc_levels(c);
    if (r != RQ_OK) return r;
  }
  return RQ_OK;
}

extern "C" int rq_create(const rq_config* cfg, const rq_atom* atoms, int32_t n_atoms, rq_ctx** out) {
  if (!cfg || !out || (n_atoms > 0 && !atoms) || n_atoms < 1) return RQ_EINVAL;
  *out = nullptr;
  if (cfg->NN < 4 || cfg->NN % 2 != 0 || cfg->screen <= 0) return RQ_EINVAL;  // molecule.js:155 needs even NN
  if (cfg->flavor < 0 || cfg->flavor > 2 || cfg->precision < 0 || cfg->precision > 1) return RQ_EINVAL;
  if (cfg->precision == RQ_PREC_FP64 && cfg->flavor != RQ_FLAVOR_NEW) return RQ_ENOTSUP;
  if (cfg->sic != 0 && cfg->flavor != RQ_FLAVOR_MOLECULE_JS) return RQ_ENOTSUP;  // SIC is molecule.js's
  if (cfg->lobpcg != 0 && cfg->flavor != RQ_FLAVOR_MOLECULE_JS) return RQ_ENOTSUP;
  if (cfg->lobpcg != 0 && cfg->chebyshev != 0) return RQ_EINVAL;  // the page switches one off (:5472-5478)
  if (cfg->chebyshev != 0) {  // molecule.js's Chebyshev update tests only the own r_c sphere (:368-372)
    if (cfg->flavor != RQ_FLAVOR_MOLECULE_JS) return RQ_ENOTSUP;
    for (int q = 0; q < n_atoms; ++q)
      if (atoms[q].Z == 0 && atoms[q].Z_nuc > 0 && atoms[q].rc > 0) return RQ_ENOTSUP;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return RQ_ENODEV;
  rq_ctx* c = new (std::nothrow) rq_ctx();
  if (!c) return RQ_ENOMEM;
  c->cfg = *cfg;
  c->g = make_geo(cfg->NN + 1);
  c->h = cfg->screen / cfg->NN;
  c->h2 = c->h * c->h;
  c->h3 = c->h2 * c->h;
  c->n_atoms = n_atoms;
  c->atoms.assign(atoms, atoms + n_atoms);
  c->atoms0 = c->atoms;
  c->fp64 = cfg->precision == RQ_PREC_FP64;
  cudaGetDevice(&c->device);
  fill_defaults(c);
  int rc = rq_cuda(c, cudaStreamCreateWithFlags(&c->own_st, cudaStreamNonBlocking), "cudaStreamCreate");
  c->st = c->own_st;
  if (rc == RQ_OK) rc = alloc_all(c);
  if (rc == RQ_OK) rc = upload_atoms(c);
  if (rc == RQ_OK) rc = rq_cuda(c, cudaStreamSynchronize(c->st), "create sync");
  if (rc != RQ_OK) {
    std::fprintf(stderr, "rq_create: %s\n", c->last_error.c_str());
    free_ctx(c);
    delete c;
    return rc;
  }
  *out = c;
  return RQ_OK;
}

extern "C" void rq_destroy(rq_ctx* c) {
  if (!c) return;
  cudaStreamSynchronize(c->st);
  free_ctx(c);
  delete c;
}

extern "C" int rq_set_stream(rq_ctx* c, void* stream) {
  if (!c) return RQ_EINVAL;
  CK(cudaStreamSynchronize(c->st));
  c->st = stream ? (cudaStream_t)stream : c->own_st;
  return RQ_OK;
}

extern "C" int rq_get_info(const rq_ctx* c, rq_info* info) {
  if (!c || !info) return RQ_EINVAL;
  std::memset(info, 0, sizeof(*info));
  info->NN = c->g.NN; info->S = c->g.S; info->n_atoms = c->n_atoms; info->flavor = c->cfg.flavor;
  info->precision = c->cfg.precision; info->steps_done = c->steps_done; info->mg_levels = (int)c->mg.size();
  info->h = c->h; info->dv = c->dv; info->dt = c->dt; info->sigma = c->sigma; info->S3 = c->g.S3;
  info->psi = c->U[c->cu]; info->label = c->lab[c->cl]; info->K = c->K; info->P = c->P[c->cp]; info->W = c->W;
  info->kernel_launches = c->launches;
  return RQ_OK;
}

extern "C" int rq_synchronize(rq_ctx* c) {
  if (!c) return RQ_EINVAL;
  if (c->cfg.flavor == RQ_FLAVOR_NEW) {
    int rc = nm_ready(c);  // device pointers from rq_get_info then hold the normalised psi
    if (rc != RQ_OK) return rc;
  }
  CK(cudaStreamSynchronize(c->st));
  return RQ_OK;
}

// ----------------------------------------------------------------------------------------
// solver.py flavour schedule (cloud/solver.py:402-444, :561-586)
// ----------------------------------------------------------------------------------------
static double interior_points(const Geo& g) {
  const double n = g.NN - 1;
  return n * n * n;
}

static int sp_normalize(rq_ctx* c, bool accumulate) {
  float* U = (float*)c->U[c->cu];
  const double S3 = (double)c->g.S3;
  if (accumulate) {
    CK(cudaMemsetAsync(c->dnorm, 0, sizeof(double) * c->n_atoms, c->st));
    LAUNCH(RQ_KC_NORMALIZE, 8 * S3, launch_norms_flat(U, c->lab[c->cl], c->g, c->h3, c->n_atoms, c->dnorm, c->st));
  }
  LAUNCH(RQ_KC_NORMALIZE, 12.0 * c->n_atoms,
         launch_norm_scale_sp(c->dnorm, c->Zdom, c->n_atoms, c->scale, c->err, c->st));
  LAUNCH(RQ_KC_NORMALIZE, 12 * S3, launch_apply_scale_sp(U, c->lab[c->cl], c->scale, c->g, c->n_atoms, c->st));
  return RQ_OK;
}

static int sp_poisson(rq_ctx* c) {
  const float coeff = (float)(2.0 * M_PI);
  for (int q = 0; q < c->cfg.jacobi_per_step; ++q) {
    LAUNCH(RQ_KC_POISSON, 12 * interior_points(c->g),
           launch_jacobi_sp((float*)c->P[c->cp], (float*)c->P[1 - c->cp], (float*)c->U[c->cu], c->g, (float)c->h2,
                            coeff, c->st));
    c->cp ^= 1;
  }
  return RQ_OK;
}

// One solver.py step (cloud/solver.py:561-586): Poisson every poisson_interval steps (2 Jacobi
// sweeps), the update, normalisation every norm_interval, labels every label_interval.  An update
// and a Jacobi sweep share one pass (k_step_sp): the last sweep of a Poisson step runs fused with
// that step's update, and the first sweep of the NEXT Poisson step runs fused with the update of
// the step before it whenever that step does not normalise (so psi does not change in between).
// That early sweep writes P[1-cp] and leaves cp alone (sp_jdone = 1): every readout still sees
// the P of the last completed Poisson step, and the next Poisson step adopts the buffer.
constexpr int kLabelScanAtoms = 64;  // up to this many atoms the label step scans them all

static int sp_step_one(rq_ctx* c, int s) {
  const rq_config& f = c->cfg;
  const bool poisson = s % f.poisson_interval == 0, norm = s % f.norm_interval == 0;
  const int jps = f.jacobi_per_step;
  const float coeff = (float)(2.0 * M_PI);
  int rc;
  if (norm) CK(cudaMemsetAsync(c->dnorm, 0, sizeof(double) * c->n_atoms, c->st));
  double* nrm = norm ? c->dnorm : nullptr;
  auto fused = [&](bool first) -> int {
    LAUNCH(RQ_KC_UPDATE, 24 * interior_points(c->g),
           launch_step_sp(first, (float*)c->U[c->cu], (float*)c->U[1 - c->cu], (float*)c->K, (float*)c->P[c->cp],
                          (float*)c->P[1 - c->cp], c->lab[c->cl], c->g, (float)c->half_dv, (float)c->dt,
                          (float)c->h2, coeff, c->h3, c->n_atoms, nrm, c->st));
    c->cu ^= 1;
    return RQ_OK;
  };
  bool updated = false;
  if (poisson) {
    int todo = jps;
    if (c->sp_jdone && todo > 0) {  // the first sweep already ran with the previous update
      c->cp ^= 1;
      todo--;
    }
    c->sp_jdone = 0;
    for (int q = 0; q + 1 < todo; ++q) {
      LAUNCH(RQ_KC_POISSON, 12 * interior_points(c->g),
             launch_jacobi_sp((float*)c->P[c->cp], (float*)c->P[1 - c->cp], (float*)c->U[c->cu], c->g, (float)c->h2,
                              coeff, c->st));
      c->cp ^= 1;
    }
    if (todo >= 1) {
      if ((rc = fused(false)) != RQ_OK) return rc;
      c->cp ^= 1;
      updated = true;
    }
  } else if ((s + 1) % f.poisson_interval == 0 && jps >= 1 && !norm) {
    if ((rc = fused(true)) != RQ_OK) return rc;
    c->sp_jdone = 1;
    updated = true;
  }
  if (!updated) {
    LAUNCH(RQ_KC_UPDATE, 20 * interior_points(c->g),
           launch_update_sp((float*)c->U[c->cu], (float*)c->U[1 - c->cu], (float*)c->K, (float*)c->P[c->cp],
                            c->lab[c->cl], c->g, (float)c->half_dv, (float)c->dt, c->h3, c->n_atoms, nrm, c->st));
    c->cu ^= 1;
  }
  if (norm && (rc = sp_normalize(c, false)) != RQ_OK) return rc;
  if (s % f.label_interval == 0 && (f.label_until <= 0 || s <= f.label_until)) {
    // a few atoms: the scan is cheaper than the bin search (same result)
    if (c->n_atoms <= kLabelScanAtoms)
      LAUNCH(RQ_KC_LABELS, 8 * interior_points(c->g),
             launch_labels_sp(c->lab[c->cl], c->lab[1 - c->cl], c->atoms5, c->n_atoms, c->g, (float)c->h,
                              (float)c->h2, c->st));
    else
      LAUNCH(RQ_KC_LABELS, 8 * interior_points(c->g),
             launch_labels_binned_sp(c->lab[c->cl], c->lab[1 - c->cl], c->atoms5, c->n_atoms,
                                     AtomBins{c->bins_nb, c->bins_bin, c->bin_start, c->bin_idx, c->bin_far, c->bin_zmax},
                                     c->g, (float)c->h, (float)c->h2, c->st));
    c->cl ^= 1;
  }
  return RQ_OK;
}

static int sp_initialize(rq_ctx* c) {
  for (int b = 0; b < 2; ++b) {
    CK(cudaMemsetAsync(c->P[b], 0, sizeof(float) * c->g.S3, c->st));
  }
  c->cu = c->cp = c->cl = 0;
  c->sp_jdone = 0;
  LAUNCH(RQ_KC_OTHER, 16.0 * c->g.S3,
         launch_init_sp((float*)c->U[0], c->lab[0], (float*)c->K, c->bestU, c->atoms5, c->n_atoms, c->g, (float)c->h,
                        (float)c->h2, true, c->st));
  CK(cudaMemcpyAsync(c->lab[1], c->lab[0], sizeof(int) * c->g.S3, cudaMemcpyDeviceToDevice, c->st));
  int rc = sp_normalize(c, true);
  if (rc != RQ_OK) return rc;
  for (int q = 0; q < 100; ++q)
    if ((rc = sp_poisson(c)) != RQ_OK) return rc;
  return RQ_OK;
}

// ----------------------------------------------------------------------------------------
// generic step driver with CUDA-graph replay of whole schedule periods
// ----------------------------------------------------------------------------------------
static int step_one(rq_ctx* c, int s) {
  switch (c->cfg.flavor) {
    case RQ_FLAVOR_SOLVER_PY: return sp_step_one(c, s);
    case RQ_FLAVOR_MOLECULE_JS: return mj_step_one(c, s);
    default: return nm_step_one(c, s);
  }
}

static int schedule_period(const rq_ctx* c) {
  const rq_config& f = c->cfg;
  auto lcm = [](long a, long b) { return a / std::gcd(a, b) * b; };
  long p = 1;
  switch (f.flavor) {
    case RQ_FLAVOR_SOLVER_PY: p = lcm(lcm(f.poisson_interval, f.norm_interval), f.label_interval); break;
    case RQ_FLAVOR_MOLECULE_JS:
      p = f.lobpcg ? 1 : (long)f.steps_per_frame * std::max(1, mj_sic_interval(c));
      break;
    default: p = lcm(lcm(f.poisson_interval, f.norm_interval), f.label_interval); break;
  }
  return p > 4096 ? 0 : (int)p;
}

static int run_steps_eager(rq_ctx* c, int n) {
  for (int q = 0; q < n; ++q) {
    int rc = step_one(c, c->steps_done + 1);
    if (rc != RQ_OK) return rc;
    c->steps_done++;
  }
  return RQ_OK;
}

extern "C" int rq_step(rq_ctx* c, int32_t n) {
  if (!c || n < 0) return RQ_EINVAL;
  const int period = schedule_period(c);
  int left = n;
  while (left > 0) {
    // a period that straddles label_until has no single captured pattern: run it eagerly
    const int lu = c->cfg.label_until;
    const bool straddle = lu > 0 && c->steps_done < lu && c->steps_done + period > lu;
    // (a period boundary never leaves an early Jacobi sweep pending: the step before a Poisson step
    // is never the last of a period, as the period is a multiple of poisson_interval)
    // (with SIC, frame 0 never corrects: the first period runs eagerly, the later ones repeat;
    // likewise a first LOBPCG frame, which starts without a search direction)
    // (steps recorded for the adjoint run eagerly: each copies its starting state into the window)
    const bool aligned = !c->prof && !c->cfg.chebyshev && c->adj.cap == 0 && !straddle && period > 0 &&
                         c->steps_done % period == 0 && left >= period &&
                         c->sp_jdone == 0 && !(mj_sic_interval(c) > 0 && c->frame == 0) &&
                         !(c->cfg.lobpcg && c->frame == 0);
    if (!aligned) {
      // run eagerly up to the next period boundary (or all that is left)
      int todo = left;
      if (period > 0 && c->steps_done % period != 0) todo = std::min(left, period - c->steps_done % period);
      int rc = run_steps_eager(c, todo);
      if (rc != RQ_OK) return rc;
      left -= todo;
      continue;
    }
    // one aligned period: replay its CUDA graph (captured on first use for this buffer parity)
    const int labels_on = (lu <= 0 || c->steps_done < lu) ? 1 : 0;
    const int key = c->cu | (c->cp << 1) | (c->cl << 2) | (labels_on << 3) | ((c->nm_pending ? 1 : 0) << 4);
    if (!c->graph[key]) {
      const long long l0 = c->launches;
      CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
      int rc = run_steps_eager(c, period);  // records the work and advances the parities
      cudaGraph_t gr = nullptr;
      cudaError_t e = cudaStreamEndCapture(c->st, &gr);
      if (rc != RQ_OK) {
        if (gr) cudaGraphDestroy(gr);
        return rc;
      }
      CK(e);
      e = cudaGraphInstantiate(&c->graph[key], gr, 0);
      cudaGraphDestroy(gr);
      CK(e);
      c->graph_post[key] = c->cu | (c->cp << 1) | (c->cl << 2) | ((c->nm_pending ? 1 : 0) << 4) | (c->nm_age << 5);
      c->graph_launches[key] = c->launches - l0;
      CK(cudaGraphLaunch(c->graph[key], c->st));
    } else {
      CK(cudaGraphLaunch(c->graph[key], c->st));
      const int post = c->graph_post[key];
      c->cu = post & 1; c->cp = (post >> 1) & 1; c->cl = (post >> 2) & 1;
      c->nm_pending = (post >> 4) & 1;
      c->nm_age = post >> 5;
      c->steps_done += period;
      if (c->cfg.flavor == RQ_FLAVOR_MOLECULE_JS) c->frame += c->cfg.lobpcg ? period : period / c->cfg.steps_per_frame;
      c->launches += c->graph_launches[key];
    }
    left -= period;
  }
  return RQ_OK;
}

extern "C" int rq_set_locked_groups(rq_ctx* c, int32_t n_groups, const int32_t* offsets, const int32_t* members) {
  if (!c || n_groups < 0 || (n_groups > 0 && (!offsets || !members))) return RQ_EINVAL;
  if (c->cfg.flavor != RQ_FLAVOR_MOLECULE_JS) return rq_fail(c, RQ_ENOTSUP, "locked groups are molecule.js's");
  if (n_groups > 64) return rq_fail(c, RQ_ENOTSUP, "at most 64 locked groups");
  std::vector<unsigned long long> mask((size_t)c->n_atoms, 0ull);
  for (int g = 0; g < n_groups; ++g) {
    if (offsets[g] < 0 || offsets[g + 1] < offsets[g]) return rq_fail(c, RQ_EINVAL, "locked group offsets");
    for (int q = offsets[g]; q < offsets[g + 1]; ++q) {
      if (members[q] < 0 || members[q] >= c->n_atoms)
        return rq_fail(c, RQ_EINVAL, "locked group member " + std::to_string(members[q]) + " outside [0, n_atoms)");
      mask[members[q]] |= 1ull << g;
    }
  }
  CK(cudaMemcpyAsync(c->lock, mask.data(), mask.size() * sizeof(unsigned long long), cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  return RQ_OK;
}

extern "C" int rq_set_splits(rq_ctx* c, const rq_split* splits) {
  if (!c) return RQ_EINVAL;
  if (c->cfg.flavor != RQ_FLAVOR_MOLECULE_JS) return rq_fail(c, RQ_ENOTSUP, "shell splits are molecule.js's");
  std::vector<MjSplit> d((size_t)c->n_atoms, MjSplit{0u, 0u, 0.f, 0.f, 1.f, 0.f});
  if (splits)
    for (int n = 0; n < c->n_atoms; ++n) {
      const rq_split& s = splits[n];
      if (s.type < 0 || s.idx < 0) return rq_fail(c, RQ_EINVAL, "negative split type or index");
      d[n] = MjSplit{(uint32_t)s.type, (uint32_t)s.idx, (float)s.axis[0], (float)s.axis[1], (float)s.axis[2],
                     (float)s.rot};
    }
  CK(cudaMemcpyAsync(c->splits, d.data(), d.size() * sizeof(MjSplit), cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  return RQ_OK;
}

extern "C" int rq_set_init_positions(rq_ctx* c, const double* pos, const int32_t* has, int32_t n) {
  if (!c || n < 0 || (n > 0 && (!pos || !has))) return RQ_EINVAL;
  if (c->cfg.flavor != RQ_FLAVOR_MOLECULE_JS) return rq_fail(c, RQ_ENOTSUP, "USER_INIT_POS is molecule.js's");
  c->init_pos.assign(pos, pos + 2 * (size_t)n);
  c->init_has.assign(has, has + n);
  return RQ_OK;
}

extern "C" int rq_set_freeze_boundary(rq_ctx* c, int32_t on) {
  if (!c) return RQ_EINVAL;
  if (c->cfg.flavor != RQ_FLAVOR_MOLECULE_JS) return rq_fail(c, RQ_ENOTSUP, "FREEZE_BOUNDARY is molecule.js's");
  if ((on != 0) != c->freeze) {
    c->freeze = on != 0;
    for (auto& gx : c->graph)  // captured periods hold the old choice
      if (gx) {
        cudaGraphExecDestroy(gx);
        gx = nullptr;
      }
  }
  return RQ_OK;
}

extern "C" int rq_restart(rq_ctx* c) {
  if (!c) return RQ_EINVAL;
  if (c->cfg.flavor != RQ_FLAVOR_MOLECULE_JS) return rq_fail(c, RQ_ENOTSUP, "the restart is molecule.js's");
  c->sp_jdone = 0;
  int rc = mj_restart(c);
  if (rc != RQ_OK) return rc;
  CK(cudaStreamSynchronize(c->st));
  return RQ_OK;
}

extern "C" int rq_initialize(rq_ctx* c) {
  if (!c) return RQ_EINVAL;
  int rc;
  switch (c->cfg.flavor) {
    case RQ_FLAVOR_SOLVER_PY: rc = sp_initialize(c); break;
    case RQ_FLAVOR_MOLECULE_JS: rc = mj_initialize(c); break;
    default: rc = nm_initialize(c); break;
  }
  if (rc != RQ_OK) return rc;
  c->steps_done = 0;
  c->frame = 0;
  c->cheb_omega = 1.0;
  c->cheb_E = 0.0;
  CK(cudaStreamSynchronize(c->st));
  return RQ_OK;
}

// ----------------------------------------------------------------------------------------
// state transfer
// ----------------------------------------------------------------------------------------
// first index of a label outside [0, nAtoms) (atomicMin into *first, which starts above any index)
__global__ void k_check_labels(const int* __restrict__ lab, long long n, int nAtoms, int* first) {
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int l = lab[q];
    if (l < 0 || l >= nAtoms) atomicMin(first, (int)q);
  }
}

// Upload host labels: copied into the spare label buffer and checked there on the device, so a
// rejected upload leaves the state as it was; accepted labels become current and are copied to
// the other buffer (the label pass writes interior points only).
static int upload_labels(rq_ctx* c, const int32_t* label) {
  const size_t n = (size_t)c->g.S3;
  int* spare = c->lab[1 - c->cl];
  CK(cudaMemcpyAsync(spare, label, n * sizeof(int), cudaMemcpyHostToDevice, c->st));
  CK(cudaMemsetAsync(c->err + 2, 0x7f, sizeof(int), c->st));
  k_check_labels<<<148 * 8, 256, 0, c->st>>>(spare, (long long)n, c->n_atoms, c->err + 2);
  CK(cudaGetLastError());
  int first = 0;
  CK(cudaMemcpyAsync(&first, c->err + 2, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (first != 0x7f7f7f7f) {
    CK(cudaMemcpyAsync(spare, c->lab[c->cl], n * sizeof(int), cudaMemcpyDeviceToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    return rq_fail(c, RQ_EINVAL, "label " + std::to_string(label[first]) + " at index " + std::to_string(first) +
                                     " outside [0, n_atoms)");
  }
  c->cl ^= 1;
  CK(cudaMemcpyAsync(c->lab[1 - c->cl], c->lab[c->cl], n * sizeof(int), cudaMemcpyDeviceToDevice, c->st));
  if (c->cfg.flavor == RQ_FLAVOR_NEW) return nm_label_mask(c);
  return RQ_OK;
}

extern "C" int rq_upload_state(rq_ctx* c, const float* psi, const int32_t* label, const float* W, const float* P) {
  if (!c) return RQ_EINVAL;
  if (c->fp64 && (psi || P)) return rq_fail(c, RQ_EINVAL, "FP64 context: use rq_upload_state_f64 for psi/P");
  const size_t n = (size_t)c->g.S3;
  const bool mj = c->cfg.flavor == RQ_FLAVOR_MOLECULE_JS;
  if (label) {
    int rc = upload_labels(c, label);
    if (rc != RQ_OK) return rc;
    if (mj && (rc = mj_refresh_flags(c)) != RQ_OK) return rc;  // r_c-exclusion bits of the new labels
  }
  if (psi || P) c->sp_jdone = 0;  // an early Jacobi sweep used the old psi and P: redo it
  if (psi || P || label) nm_adj_reset(c);  // the recorded steps led to another state
  if (psi) {
    c->nm_pending = false;
    c->nm_age = 0;
    CK(cudaMemcpyAsync(c->U[c->cu], psi, n * sizeof(float), cudaMemcpyHostToDevice, c->st));
    if (mj)  // molecule.js keeps the boundary values of psi (never rewritten): both buffers hold them
      CK(cudaMemcpyAsync(c->U[1 - c->cu], c->U[c->cu], n * sizeof(float), cudaMemcpyDeviceToDevice, c->st));
    else
      CK(launch_zero_faces((float*)c->U[c->cu], c->g, c->st));  // Dirichlet planes are 0
  }
  if (W) CK(cudaMemcpyAsync(c->W, W, n * sizeof(float), cudaMemcpyHostToDevice, c->st));
  if (P) {
    CK(cudaMemcpyAsync(c->P[c->cp], P, n * sizeof(float), cudaMemcpyHostToDevice, c->st));
    CK(launch_zero_faces((float*)c->P[c->cp], c->g, c->st));
    if (c->Pother) CK(cudaMemcpyAsync(c->Pother, c->P[c->cp], n * sizeof(float), cudaMemcpyDeviceToDevice, c->st));
  }
  CK(cudaStreamSynchronize(c->st));
  return RQ_OK;
}

extern "C" int rq_download_state(rq_ctx* c, float* psi, int32_t* label, float* W, float* P) {
  if (!c) return RQ_EINVAL;
  if (c->cfg.flavor == RQ_FLAVOR_NEW && psi) {
    int rc = nm_ready(c);
    if (rc != RQ_OK) return rc;
  }
  if (c->fp64 && (psi || P)) return rq_fail(c, RQ_EINVAL, "FP64 context: use rq_download_state_f64 for psi/P");
  const size_t n = (size_t)c->g.S3;
  if (psi) CK(cudaMemcpyAsync(psi, c->U[c->cu], n * sizeof(float), cudaMemcpyDeviceToHost, c->st));
  if (label) CK(cudaMemcpyAsync(label, c->lab[c->cl], n * sizeof(int), cudaMemcpyDeviceToHost, c->st));
  if (W) CK(cudaMemcpyAsync(W, c->W, n * sizeof(float), cudaMemcpyDeviceToHost, c->st));
  if (P) CK(cudaMemcpyAsync(P, c->P[c->cp], n * sizeof(float), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (label && c->cfg.flavor == RQ_FLAVOR_MOLECULE_JS)
    for (size_t q = 0; q < n; ++q) label[q] &= kMjLabelMask;  // strip the exclusion bit
  return RQ_OK;
}

extern "C" int rq_upload_state_f64(rq_ctx* c, const double* psi, const double* P) {
  if (!c) return RQ_EINVAL;
  if (!c->fp64) return rq_fail(c, RQ_EINVAL, "mixed-precision context: use rq_upload_state");
  const size_t n = (size_t)c->g.S3;
  if (psi || P) nm_adj_reset(c);
  if (psi) {
    c->nm_pending = false;
    c->nm_age = 0;
    CK(cudaMemcpyAsync(c->U[c->cu], psi, n * sizeof(double), cudaMemcpyHostToDevice, c->st));
    CK(launch_zero_faces((double*)c->U[c->cu], c->g, c->st));
  }
  if (P) {
    CK(cudaMemcpyAsync(c->P[c->cp], P, n * sizeof(double), cudaMemcpyHostToDevice, c->st));
    CK(launch_zero_faces((double*)c->P[c->cp], c->g, c->st));
  }
  CK(cudaStreamSynchronize(c->st));
  return RQ_OK;
}

extern "C" int rq_download_state_f64(rq_ctx* c, double* psi, double* P, double* K) {
  if (!c) return RQ_EINVAL;
  if (psi) {
    int rc = nm_ready(c);
    if (rc != RQ_OK) return rc;
  }
  if (!c->fp64) return rq_fail(c, RQ_EINVAL, "mixed-precision context: use rq_download_state");
  const size_t n = (size_t)c->g.S3;
  if (psi) CK(cudaMemcpyAsync(psi, c->U[c->cu], n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  if (P) CK(cudaMemcpyAsync(P, c->P[c->cp], n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  if (K) CK(cudaMemcpyAsync(K, c->K, n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return RQ_OK;
}

extern "C" int rq_download_K(rq_ctx* c, float* K) {
  if (!c || !K) return RQ_EINVAL;
  if (c->fp64) return rq_fail(c, RQ_EINVAL, "FP64 context: use rq_download_state_f64");
  CK(cudaMemcpyAsync(K, c->K, (size_t)c->g.S3 * sizeof(float), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return RQ_OK;
}

// ----------------------------------------------------------------------------------------
// atoms, energies, forces
// ----------------------------------------------------------------------------------------
extern "C" int rq_set_atoms(rq_ctx* c, const rq_atom* atoms, int32_t n) {
  if (!c || !atoms || n != c->n_atoms) return RQ_EINVAL;
  c->atoms.assign(atoms, atoms + n);  // tables are rewritten in place: captured graphs stay valid
  int rc = upload_atoms(c);
  if (rc != RQ_OK) return rc;
  switch (c->cfg.flavor) {
    case RQ_FLAVOR_SOLVER_PY:  // cloud/solver.py:538-548 recomputeK
      CK(launch_init_sp(nullptr, nullptr, (float*)c->K, nullptr, c->atoms5, c->n_atoms, c->g, (float)c->h,
                        (float)c->h2, false, c->st));
      break;
    case RQ_FLAVOR_MOLECULE_JS:
      rc = mj_set_atoms(c);
      break;
    default:
      rc = nm_set_atoms(c);
      break;
  }
  if (rc != RQ_OK) return rc;
  CK(cudaStreamSynchronize(c->st));
  return RQ_OK;
}

extern "C" int rq_set_external_potential(rq_ctx* c, const double* v) {
  if (!c) return RQ_EINVAL;
  if (c->cfg.flavor != RQ_FLAVOR_NEW) return rq_fail(c, RQ_ENOTSUP, "external potential: new flavour only");
  int rc = nm_set_external(c, v);
  if (rc != RQ_OK) return rc;
  CK(cudaStreamSynchronize(c->st));
  return RQ_OK;
}

static void fill_domains(rq_ctx* c, const std::vector<double>& pd, double* out, double* per_domain) {
  double T = 0, EK = 0, EE = 0;
  for (int q = 0; q < c->n_atoms; ++q) {
    T += pd[q * 4 + 1]; EK += pd[q * 4 + 2]; EE += pd[q * 4 + 3];
    if (per_domain) {
      double* d = per_domain + (size_t)q * RQ_DOMAIN_LEN;
      d[RQ_D_NORM] = pd[q * 4]; d[RQ_D_T] = pd[q * 4 + 1]; d[RQ_D_EK] = pd[q * 4 + 2]; d[RQ_D_EE] = pd[q * 4 + 3];
      const double nr = pd[q * 4] != 0 ? pd[q * 4] : 1.0;  // atom.js:340 eigenvalue (|| 1)
      d[RQ_D_EIG] = (pd[q * 4 + 1] + 2 * pd[q * 4 + 3] + pd[q * 4 + 2]) / nr;
    }
  }
  out[RQ_E_T] = T; out[RQ_E_EK] = EK; out[RQ_E_EE] = EE;
}

extern "C" int rq_nuclear_terms(rq_ctx* c, double* E_KK, double* F) {
  if (!c) return RQ_EINVAL;
  const int n = c->n_atoms;
  const double h = c->h;
  std::vector<double> f((size_t)n * 3, 0.0);
  double e = 0;
  if (c->cfg.flavor == RQ_FLAVOR_SOLVER_PY) {
    // cloud/solver.py:462-474 energy and :504-520 forces: softening h^2, charges Z_eff
    for (int a = 0; a < n; ++a) {
      if (c->atoms[a].Z <= 0) continue;
      for (int b = 0; b < n; ++b) {
        if (b == a || c->atoms[b].Z <= 0) continue;
        const double dx = (double)(float)c->atoms[a].i - (double)(float)c->atoms[b].i;
        const double dy = (double)(float)c->atoms[a].j - (double)(float)c->atoms[b].j;
        const double dz = (double)(float)c->atoms[a].k - (double)(float)c->atoms[b].k;
        const double r2 = (dx * dx + dy * dy + dz * dz) * h * h + h * h;
        const double zz = (double)(float)c->atoms[a].Z * (double)(float)c->atoms[b].Z;
        if (b > a) e += zz / std::sqrt(r2);
        const double w = zz / (r2 * std::sqrt(r2));
        f[a * 3] += w * dx * h; f[a * 3 + 1] += w * dy * h; f[a * 3 + 2] += w * dz * h;
      }
    }
  } else if (c->cfg.flavor == RQ_FLAVOR_MOLECULE_JS) {
    mj_nuclear_terms(c, &e, f.data());
  } else {
    const int rc = nm_nuclear_terms(c, &e, f.data());
    if (rc != RQ_OK) return rc;
  }
  if (E_KK) *E_KK = e;
  if (F) std::memcpy(F, f.data(), sizeof(double) * f.size());
  return RQ_OK;
}

extern "C" int rq_energy(rq_ctx* c, double* out, double* per_domain) {
  if (!c || !out) return RQ_EINVAL;
  for (int q = 0; q < RQ_ENERGY_LEN; ++q) out[q] = 0;
  int rc = RQ_OK;
  if (c->cfg.flavor == RQ_FLAVOR_SOLVER_PY) {
    const int n = c->n_atoms;
    CK(cudaMemsetAsync(c->dpd, 0, sizeof(double) * 4 * n, c->st));
    CK(launch_energy_sp((float*)c->U[c->cu], (float*)c->K, (float*)c->P[c->cp], c->lab[c->cl], c->g, c->h, c->h3, n,
                        c->dpd, c->st));
    std::vector<double> pd((size_t)4 * n);
    CK(cudaMemcpyAsync(pd.data(), c->dpd, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    fill_domains(c, pd, out, per_domain);
  } else if (c->cfg.flavor == RQ_FLAVOR_MOLECULE_JS) {
    rc = mj_energy(c, out, per_domain);
  } else {
    rc = nm_energy(c, out, per_domain);
  }
  if (rc != RQ_OK) return rc;
  double ekk = 0;
  if ((rc = rq_nuclear_terms(c, &ekk, nullptr)) != RQ_OK) return rc;
  out[RQ_E_KK] = ekk;
  out[RQ_E_TOTAL] = out[RQ_E_T] + out[RQ_E_EK] + out[RQ_E_EE] + out[RQ_E_KK];
  // a normalisation since the last readout met a NaN/Inf domain norm (the kernel left that
  // domain unscaled and set the word): report it once, then clear the word
  int bad_norm = 0;
  CK(cudaMemcpyAsync(&bad_norm, c->err, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (bad_norm) {
    CK(cudaMemsetAsync(c->err, 0, sizeof(int), c->st));
    CK(cudaStreamSynchronize(c->st));
    return rq_fail(c, RQ_ENONFINITE, "non-finite domain norm in a normalisation");
  }
  for (int q = 0; q < RQ_ENERGY_LEN; ++q)
    if (!std::isfinite(out[q])) return rq_fail(c, RQ_ENONFINITE, "non-finite energy component");
  return RQ_OK;
}

extern "C" int rq_forces(rq_ctx* c, int32_t method, double* F) {
  if (!c || !F) return RQ_EINVAL;
  const int n = c->n_atoms;
  if (c->cfg.flavor == RQ_FLAVOR_SOLVER_PY) {
    if (method != RQ_FORCE_HF && method != RQ_FORCE_ADJOINT) return RQ_ENOTSUP;
    CK(cudaMemsetAsync(c->dF, 0, sizeof(double) * 3 * n, c->st));
    CK(launch_forces_hf_sp((float*)c->U[c->cu], c->atoms5, n, c->g, (float)c->h, (float)c->h2, (float)c->h3, c->dF,
                           c->st));
    CK(cudaMemcpyAsync(F, c->dF, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return RQ_OK;
  }
  if (c->cfg.flavor == RQ_FLAVOR_MOLECULE_JS) return mj_forces(c, method, F);
  return nm_forces(c, method, F);
}

extern "C" int rq_extract(rq_ctx* c, int32_t slice_k, float* out) {
  if (!c || !out) return RQ_EINVAL;
  if (c->cfg.flavor != RQ_FLAVOR_MOLECULE_JS) return rq_fail(c, RQ_ENOTSUP, "the slice buffer is molecule.js's");
  if (slice_k < 1 || slice_k >= c->g.NN) return rq_fail(c, RQ_EINVAL, "slice_k outside the interior");
  const size_t S = (size_t)c->g.S, n = 3 * S * S + 2 * S;
  float* d = nullptr;
  CK(cudaMallocAsync((void**)&d, n * sizeof(float), c->st));
  cudaError_t e = launch_mj_extract((const float*)c->U[c->cu], c->lab[c->cl], (const float*)c->K,
                                    (const MjAtom*)c->atoms_mj, c->n_atoms, c->g, slice_k, d, c->st);
  if (e == cudaSuccess) {
    c->launches++;
    e = cudaMemcpyAsync(out, d, n * sizeof(float), cudaMemcpyDeviceToHost, c->st);
  }
  cudaFreeAsync(d, c->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
  return e == cudaSuccess ? RQ_OK : rq_cuda(c, e, "rq_extract");
}

extern "C" int rq_promote(rq_ctx* c) {
  if (!c) return RQ_EINVAL;
  if (c->cfg.flavor != RQ_FLAVOR_NEW) return rq_fail(c, RQ_ENOTSUP, "promotion to FP64 is for the new flavour");
  const int rc = nm_promote(c);
  if (rc == RQ_OK) c->cfg.precision = RQ_PREC_FP64;
  return rc;
}

extern "C" int rq_set_adjoint_window(rq_ctx* c, int32_t steps) {
  if (!c) return RQ_EINVAL;
  if (c->cfg.flavor != RQ_FLAVOR_NEW) return rq_fail(c, RQ_ENOTSUP, "the adjoint is the new flavour's");
  if (steps < 0) return rq_fail(c, RQ_EINVAL, "negative adjoint window");
  CK(cudaStreamSynchronize(c->st));
  return nm_adj_set_window(c, steps);
}

extern "C" int rq_adjoint(rq_ctx* c, double* F, double* dE_dv) {
  if (!c) return RQ_EINVAL;
  if (c->cfg.flavor != RQ_FLAVOR_NEW) return rq_fail(c, RQ_ENOTSUP, "the adjoint is the new flavour's");
  return nm_adjoint(c, F, dE_dv);
}

extern "C" int rq_solve(rq_ctx* c, double tol_dE, int32_t max_steps, int32_t check_interval, int32_t* steps_taken,
                        double* E_final) {
  if (!c || max_steps < 0 || check_interval <= 0) return RQ_EINVAL;
  double e[RQ_ENERGY_LEN];
  int rc = rq_energy(c, e, nullptr);
  if (rc != RQ_OK) return rc;
  double prev = e[RQ_E_TOTAL];
  const int need = c->cfg.converge_checks > 0 ? c->cfg.converge_checks : 1;
  // a mixed-precision new-flavour context first converges as far as its fp32 fields resolve, then
  // continues in FP64 from there (the same staging as rq_batch_solve)
  bool staged = c->cfg.flavor == RQ_FLAVOR_NEW && !c->fp64;
  double tol = staged ? std::max(tol_dE, kMixedFloor * std::fabs(prev)) : tol_dE;
  int taken = 0, run = 0;
  while (taken < max_steps) {
    const int n = std::min(check_interval, max_steps - taken);
    if ((rc = rq_step(c, n)) != RQ_OK) return rc;
    taken += n;
    if ((rc = rq_energy(c, e, nullptr)) != RQ_OK) return rc;
    const double d = std::fabs(e[RQ_E_TOTAL] - prev);
    prev = e[RQ_E_TOTAL];
    if (d >= tol) {
      run = 0;
      continue;
    }
    if (staged && tol > tol_dE) {  // fp32 has stalled: refine in FP64 from here
      if ((rc = rq_promote(c)) != RQ_OK) return rc;
      staged = false;
      tol = tol_dE;
      run = 0;
      continue;
    }
    if (++run >= need) break;
  }
  if (steps_taken) *steps_taken = taken;
  if (E_final) *E_final = prev;
  return RQ_OK;
}

// ----------------------------------------------------------------------------------------
// single kernels on caller-owned device memory
// ----------------------------------------------------------------------------------------
#define KCHK(call)                                   \
  do {                                               \
    cudaError_t _e = (call);                         \
    if (_e != cudaSuccess) return RQ_ECUDA;          \
  } while (0)

extern "C" int rq_kernel_update_sp(const float* U, float* Unew, const float* K, const float* P, const int32_t* label,
                                   int32_t S, float half_dv, float dtv, void* stream) {
  if (!U || !Unew || !K || !P || !label || S < 3) return RQ_EINVAL;
  Geo g = make_geo(S);
  cudaStream_t st = (cudaStream_t)stream;
  KCHK(launch_update_sp(U, Unew, K, P, label, g, half_dv, dtv, 0.0, 1, nullptr, st));
  KCHK(launch_zero_faces(Unew, g, st));
  return RQ_OK;
}

extern "C" int rq_kernel_jacobi_sp(const float* P, float* Pnew, const float* U, int32_t S, float h2, float coeff,
                                   void* stream) {
  if (!P || !Pnew || !U || S < 3) return RQ_EINVAL;
  Geo g = make_geo(S);
  cudaStream_t st = (cudaStream_t)stream;
  KCHK(launch_jacobi_sp(P, Pnew, U, g, h2, coeff, st));
  KCHK(launch_zero_faces(Pnew, g, st));
  return RQ_OK;
}

extern "C" int rq_kernel_labels_sp(const int32_t* labelIn, int32_t* labelOut, const float* atoms5, int32_t n_atoms,
                                   int32_t S, float h, float h2, void* stream) {
  if (!labelIn || !labelOut || !atoms5 || n_atoms < 1 || S < 3 || labelIn == labelOut) return RQ_EINVAL;
  Geo g = make_geo(S);
  cudaStream_t st = (cudaStream_t)stream;
  KCHK(cudaMemcpyAsync(labelOut, labelIn, sizeof(int) * g.S3, cudaMemcpyDeviceToDevice, st));
  KCHK(launch_labels_sp(labelIn, labelOut, atoms5, n_atoms, g, h, h2, st));
  return RQ_OK;
}

extern "C" int rq_kernel_init_sp(float* U, int32_t* label, float* K, float* bestU, const float* atoms5,
                                 int32_t n_atoms, int32_t S, float h, float h2, void* stream) {
  if (!U || !label || !K || !bestU || !atoms5 || n_atoms < 1 || S < 3) return RQ_EINVAL;
  KCHK(launch_init_sp(U, label, K, bestU, atoms5, n_atoms, make_geo(S), h, h2, true, (cudaStream_t)stream));
  return RQ_OK;
}

extern "C" int rq_kernel_recompute_k_sp(float* K, const float* atoms5, int32_t n_atoms, int32_t S, float h, float h2,
                                        void* stream) {
  if (!K || !atoms5 || n_atoms < 1 || S < 3) return RQ_EINVAL;
  KCHK(launch_init_sp(nullptr, nullptr, K, nullptr, atoms5, n_atoms, make_geo(S), h, h2, false,
                      (cudaStream_t)stream));
  return RQ_OK;
}

extern "C" int rq_kernel_normalize_sp(float* U, const int32_t* label, const float* Zeff, int32_t n_atoms, int32_t S,
                                      float h3, double* norms_out, void* stream) {
  if (!U || !label || !Zeff || n_atoms < 1 || S < 3) return RQ_EINVAL;
  Geo g = make_geo(S);
  cudaStream_t st = (cudaStream_t)stream;
  // scratch for the per-domain sums when the caller passes none, the scale table and the error
  // word; released on every exit, also when a step below fails
  struct Scratch {
    cudaStream_t st;
    void* p[3] = {nullptr, nullptr, nullptr};
    ~Scratch() {
      for (void* q : p)
        if (q) cudaFreeAsync(q, st);
    }
  } tmp{st};
  double* norms = norms_out;
  if (!norms) {
    KCHK(cudaMallocAsync(&tmp.p[0], sizeof(double) * n_atoms, st));
    norms = (double*)tmp.p[0];
  }
  KCHK(cudaMallocAsync(&tmp.p[1], sizeof(float) * n_atoms, st));
  KCHK(cudaMallocAsync(&tmp.p[2], sizeof(int), st));
  float* scale = (float*)tmp.p[1];
  int* err = (int*)tmp.p[2];
  KCHK(cudaMemsetAsync(norms, 0, sizeof(double) * n_atoms, st));
  KCHK(cudaMemsetAsync(err, 0, sizeof(int), st));
  KCHK(launch_norms_flat(U, label, g, (double)h3, n_atoms, norms, st));
  KCHK(launch_norm_scale_sp(norms, Zeff, n_atoms, scale, err, st));
  KCHK(launch_apply_scale_sp(U, label, scale, g, n_atoms, st));
  int err_host = 0;
  KCHK(cudaMemcpyAsync(&err_host, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  KCHK(cudaStreamSynchronize(st));
  return err_host ? RQ_ENONFINITE : RQ_OK;
}

extern "C" int rq_kernel_energy_sp(const float* U, const float* K, const float* P, const int32_t* label,
                                   int32_t n_atoms, int32_t S, float h, float h3, double* per_domain, void* stream) {
  if (!U || !K || !P || !label || !per_domain || n_atoms < 1 || S < 3) return RQ_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  KCHK(cudaMemsetAsync(per_domain, 0, sizeof(double) * 4 * n_atoms, st));
  KCHK(launch_energy_sp(U, K, P, label, make_geo(S), (double)h, (double)h3, n_atoms, per_domain, st));
  return RQ_OK;
}

extern "C" int rq_kernel_forces_hf_sp(const float* U, const float* atoms5, int32_t n_atoms, int32_t S, float h,
                                      float h2, float h3, double* F, void* stream) {
  if (!U || !atoms5 || !F || n_atoms < 1 || S < 3) return RQ_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  KCHK(cudaMemsetAsync(F, 0, sizeof(double) * 3 * n_atoms, st));
  KCHK(launch_forces_hf_sp(U, atoms5, n_atoms, make_geo(S), h, h2, h3, F, st));
  return RQ_OK;
}

// ----------------------------------------------------------------------------------------
// per-kernel profile
// ----------------------------------------------------------------------------------------
extern "C" int rq_profile_begin(rq_ctx* c) {
  if (!c) return RQ_EINVAL;
  CK(cudaStreamSynchronize(c->st));
  c->prec.clear();
  c->evused = 0;
  c->prof = true;
  return RQ_OK;
}

extern "C" int rq_profile_end(rq_ctx* c, rq_profile* out) {
  if (!c || !out) return RQ_EINVAL;
  CK(cudaStreamSynchronize(c->st));
  std::memset(out, 0, sizeof(*out));
  for (auto& r : c->prec) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, r.a, r.b));
    out->launches[r.cls] += 1;
    out->ms[r.cls] += ms;
    out->bytes[r.cls] += r.bytes;
  }
  c->prec.clear();
  c->evused = 0;
  c->prof = false;
  return RQ_OK;
}
