// mj_flavor.cu -- the molecule.js flavour's schedule, energies and forces (host side of librq).
//
// One rq_step of this flavour is one iteration of the s-loop of doSteps (molecule.js:2829-3006);
// every steps_per_frame steps the frame tail runs (Pother <- P, molecule.js:3014-3015, then
// W_STEPS_PER_FRAME level-set passes, :3093-3104).  cfg.sic = 1 takes the reference's own choice
// of Pother: for NELEC <= 5 the direct per-electron Poisson (:2833-2858; persistent P_m solved
// every step, Pother = P_m on domain m), above it the total Poisson with the self-interaction
// correction in the frame tail (:3016-3076) every frame for NELEC <= 15, every 5th for NELEC <=
// 30, never above.  cfg.sic = 0 always takes the total Poisson without the correction.
#include <cmath>
#include <cstring>
#include <map>
#include <tuple>

#include "rq_flavors.h"
#include "rq_kernels.h"

using namespace rq;

#define CK(call)                                 \
  do {                                           \
    int _rc = rq_cuda(c, (call), #call);         \
    if (_rc != RQ_OK) return _rc;                \
  } while (0)

namespace {

struct MjParams {  // the f32 uniform P of molecule.js:175-181 (fillParamsBuf :1829-1836)
  float h, h2, h3, inv_h, inv_h2, dt, half_d, two_pi, dt_w, curvReg, Rsing;
  bool hasBare;
  int nelec;
  double n_electrons;
};

MjParams mj_params(const rq_ctx* c) {
  MjParams p;
  const double h = c->h;
  p.h = (float)h;
  p.h2 = (float)(h * h);
  p.h3 = (float)(h * h * h);
  p.inv_h = (float)(1.0 / h);
  p.inv_h2 = (float)(1.0 / (h * h));
  p.dt = (float)(c->dv * h * h);
  p.half_d = (float)(0.5 * c->dv);
  p.two_pi = (float)(2.0 * M_PI);
  p.dt_w = (float)c->cfg.boundary_speed;
  p.curvReg = (float)c->cfg.curv_reg;
  p.Rsing = (float)(2.0 * h);  // R_SING = 2 h (molecule.js:82)
  p.hasBare = false;
  p.nelec = 0;
  p.n_electrons = 0;
  for (auto& a : c->atoms) {
    if (a.Z == 0 && a.Z_nuc > 0) p.hasBare = true;  // molecule.js:85-91
    if (a.Z > 0 || a.Z_nuc > 0) p.nelec++;
    p.n_electrons += a.Z;
  }
  return p;
}

const MjAtom* atoms_dev(rq_ctx* c) { return (const MjAtom*)c->atoms_mj; }

}  // namespace

static int mj_nelec(const rq_ctx* c) {  // NELEC (molecule.js:12-17)
  int nelec = 0;
  for (auto& a : c->atoms)
    if (a.Z > 0 || a.Z_nuc > 0) nelec++;
  return nelec ? nelec : 3;
}

// The direct per-electron Poisson path (USE_DIRECT_POTHER, molecule.js:111).
bool mj_direct(const rq_ctx* c) {
  return c->cfg.flavor == RQ_FLAVOR_MOLECULE_JS && c->cfg.sic && mj_nelec(c) <= 5;
}

// Frames between self-interaction corrections (SIC_INTERVAL, molecule.js:112), 0 when off.
int mj_sic_interval(const rq_ctx* c) {
  if (c->cfg.flavor != RQ_FLAVOR_MOLECULE_JS || !c->cfg.sic || mj_direct(c)) return 0;
  const int nelec = mj_nelec(c);
  return nelec <= 15 ? 1 : nelec <= 30 ? 5 : 0;
}

namespace {

double interior(const Geo& g) {
  const double n = g.NN - 1;
  return n * n * n;
}

}  // namespace

int mj_initialize(rq_ctx* c) {
  const MjParams p = mj_params(c);
  const size_t n = (size_t)c->g.S3;
  c->cu = c->cp = c->cl = 0;
  // molecule.js uploadInitialData (:1905-2101): K, trial psi and argmax labels over all S^3
  // points; both psi buffers, both label buffers, P = Pother = 0, W = 1.  With USER_INIT_POS
  // (:1909-1921) the trial psi and the labels come from the atoms moved to their init positions
  // (i, j; k kept), then the true records go back and K is rebuilt from 0 by recomputeK
  // (:1959-1981), and the labels' exclusion bits are recomputed for the true positions.
  bool moved = false;
  std::vector<MjAtom> tab((size_t)c->n_atoms);
  for (int q = 0; q < c->n_atoms; ++q) {
    rq_atom a = c->atoms[q];
    if (q < (int)c->init_has.size() && c->init_has[q]) {
      a.i = c->init_pos[2 * q];
      a.j = c->init_pos[2 * q + 1];
      moved = true;
    }
    tab[q] = mj_record(a);
  }
  if (moved) CK(cudaMemcpyAsync(c->atoms_mj, tab.data(), sizeof(MjAtom) * tab.size(), cudaMemcpyHostToDevice, c->st));
  LAUNCH(RQ_KC_OTHER, 12.0 * c->g.S3,
         launch_mj_init((float*)c->K, (float*)c->U[0], c->bestU, c->lab[0], atoms_dev(c), c->n_atoms, c->g, p.h, p.h2,
                        p.Rsing, p.hasBare, false, c->splits, c->st));
  if (moved) {
    for (int q = 0; q < c->n_atoms; ++q) tab[q] = mj_record(c->atoms[q]);
    CK(cudaMemcpyAsync(c->atoms_mj, tab.data(), sizeof(MjAtom) * tab.size(), cudaMemcpyHostToDevice, c->st));
    LAUNCH(RQ_KC_OTHER, 4.0 * c->g.S3,
           launch_mj_recompute_k((float*)c->K, atoms_dev(c), c->n_atoms, c->g, p.h, p.Rsing, c->st));
    LAUNCH(RQ_KC_OTHER, 8.0 * c->g.S3, launch_mj_flags(c->lab[0], atoms_dev(c), c->n_atoms, c->g, p.h, p.hasBare, c->st));
    CK(cudaStreamSynchronize(c->st));  // the table is a copy source
  }
  CK(cudaMemcpyAsync(c->U[1], c->U[0], n * sizeof(float), cudaMemcpyDeviceToDevice, c->st));
  CK(cudaMemcpyAsync(c->lab[1], c->lab[0], n * sizeof(int), cudaMemcpyDeviceToDevice, c->st));
  for (int b = 0; b < 2; ++b) CK(cudaMemsetAsync(c->P[b], 0, n * sizeof(float), c->st));
  CK(cudaMemsetAsync(c->Pother, 0, n * sizeof(float), c->st));
  LAUNCH(RQ_KC_OTHER, 4.0 * c->g.S3, launch_fill(c->W, 1.0f, c->g.S3, c->st));
  if (mj_direct(c) && p.n_electrons > 1) {  // P_m = sum_{n != m} 0.5/r, Pother = sum_m P_m (:2678-2693)
    for (int m = 0; m < c->n_atoms; ++m)
      if (c->atoms[m].Z != 0)
        LAUNCH(RQ_KC_OTHER, 8.0 * c->g.S3,
               launch_mj_direct_init(atoms_dev(c), c->n_atoms, m, c->pdirect + (size_t)m * n, c->Pother, c->g, p.h,
                                     p.h2, c->st));
  }
  return RQ_OK;
}

// The classical-MD backbone's full restart (molecule.js:4236-4286): K, the trial psi and the labels
// rebuilt from scratch at the current positions (all S^3 cells of the current label buffer), P
// cleared; unlike uploadInitialData the level-set W, Pother, the direct path's P_m and the spare
// label buffer (the page's label2Buf, whose faces the next level-set pass hands back) are kept.
int mj_restart(rq_ctx* c) {
  const MjParams p = mj_params(c);
  const size_t n = (size_t)c->g.S3;
  LAUNCH(RQ_KC_OTHER, 12.0 * c->g.S3,
         launch_mj_init((float*)c->K, (float*)c->U[c->cu], c->bestU, c->lab[c->cl], atoms_dev(c), c->n_atoms, c->g, p.h,
                        p.h2, p.Rsing, p.hasBare, false, c->splits, c->st));
  CK(cudaMemcpyAsync(c->U[1 - c->cu], c->U[c->cu], n * sizeof(float), cudaMemcpyDeviceToDevice, c->st));
  LAUNCH(RQ_KC_OTHER, 8.0 * c->g.S3,
         launch_mj_flags(c->lab[1 - c->cl], atoms_dev(c), c->n_atoms, c->g, p.h, p.hasBare, c->st));
  for (int b = 0; b < 2; ++b) CK(cudaMemsetAsync(c->P[b], 0, n * sizeof(float), c->st));
  return RQ_OK;
}

int mj_set_atoms(rq_ctx* c) {
  // moveNuclei's rebuild (molecule.js:4563-4582): K from 0 with the init formula, persistent
  // bestU / labels (a moved atom may take cells over) in the current label buffer, all S^3 cells.
  // The spare buffer stands for the page's label2Buf, which the rebuild does not touch: it keeps
  // its face labels (the next level-set pass hands them back), with exclusion bits for the new
  // positions.
  const MjParams p = mj_params(c);
  LAUNCH(RQ_KC_OTHER, 16.0 * c->g.S3,
         launch_mj_init((float*)c->K, nullptr, c->bestU, c->lab[c->cl], atoms_dev(c), c->n_atoms, c->g, p.h, p.h2,
                        p.Rsing, p.hasBare, true, c->splits, c->st));
  LAUNCH(RQ_KC_OTHER, 8.0 * c->g.S3,
         launch_mj_flags(c->lab[1 - c->cl], atoms_dev(c), c->n_atoms, c->g, p.h, p.hasBare, c->st));
  return RQ_OK;
}

int mj_refresh_flags(rq_ctx* c) {
  const MjParams p = mj_params(c);
  for (int b = 0; b < 2; ++b)
    LAUNCH(RQ_KC_OTHER, 8.0 * c->g.S3,
           launch_mj_flags(c->lab[b], atoms_dev(c), c->n_atoms, c->g, p.h, p.hasBare, c->st));
  return RQ_OK;
}

// The page's Chebyshev omega for the coming step (molecule.js:2924-2949): the spectral bounds of
// the ITP iteration from dv and the previous frame's energy, the omega recurrence, the clamp.
static float mj_cheb_omega(rq_ctx* c) {
  const double dv = c->dv, dtv = dv * (c->h * c->h), E = c->cheb_E;
  const double dtLmax = 6.0 * dv;
  const double dtLmin = dtv * (std::isfinite(E) ? std::max(-100.0, E) : -10.0);
  const double gMax = 1 - dtLmin, gMin = 1 - dtLmax;
  const double q = (gMax - gMin) / (gMax + gMin), rhoSq = q * q;
  double omega;
  if (c->cheb_omega <= 1.0) {
    omega = 1.0;
    c->cheb_omega = 1.001;
  } else if (c->cheb_omega < 1.01) {
    omega = 1.0 / (1.0 - rhoSq / 2.0);
    c->cheb_omega = omega;
  } else {
    omega = 1.0 / (1.0 - rhoSq * c->cheb_omega / 4.0);
    c->cheb_omega = omega;
  }
  return (float)std::min(1.95, std::max(1.0, omega));
}

// One LOBPCG frame (doLOBPCGStep, molecule.js:3323-3740).  Phase 1: the Poisson solve on the current
// psi -- the direct per-electron path, or 4 Jacobi sweeps and the V-cycle (vcycleEnabled, :1815) --
// and Pother: P, minus every domain's own potential when the correction is on (:3405-3451; no
// SIC_INTERVAL here).  Phase 2: per domain 10 iterations (:3460-3588) of H applied to X, the
// Rayleigh quotient, the preconditioned residual W, H applied to W and P, the Ritz problem over
// span{X, W[, P]} and the update of X and P on the domain; the page reads the sums back and solves
// the small problem on the host, here one device thread does it (k_lob_finalize), so no step waits
// for the host.  Phase 3 (:3591-3660): the fixed-point normalisation, one ITP update, the level-set
// passes.  The search direction P persists across frames; frame 0 starts without one.
static int mj_lobpcg_frame(rq_ctx* c) {
  const MjParams p = mj_params(c);
  const rq_config& f = c->cfg;
  const bool poisson = p.n_electrons > 1.0;
  const double ip = interior(c->g);
  const bool direct = mj_direct(c);
  const size_t S3 = (size_t)c->g.S3;
  if (poisson && direct) {
    for (int m = 0; m < c->n_atoms; ++m) {
      if ((float)c->atoms[m].Z == 0.f) continue;
      LAUNCH(RQ_KC_POISSON, 128 * ip,
             launch_mj_direct_domain((float*)c->U[c->cu], c->lab[c->cl], c->Pother, m, c->pdirect + (size_t)m * S3,
                                     c->sic, c->rho, c->g, p.h2, p.two_pi, c->st));
    }
  } else if (poisson) {
    for (int js = 0; js < 4; ++js) {
      LAUNCH(RQ_KC_POISSON, 12 * ip,
             launch_mj_jacobi((float*)c->P[c->cp], (float*)c->P[1 - c->cp], (float*)c->U[c->cu], c->g, p.h2, p.two_pi,
                              c->st));
      c->cp ^= 1;
    }
    LAUNCH(RQ_KC_MG, 40 * ip,
           launch_mj_vcycle((float*)c->P[c->cp], (float*)c->U[c->cu], c->rho, c->resid, c->Ec[0], c->Ec[1], c->fc, c->g,
                            c->gc, p.h2, p.inv_h2, p.two_pi, c->st));
  }
  if (!poisson) {
    CK(cudaMemsetAsync(c->Pother, 0, S3 * sizeof(float), c->st));
  } else if (!direct) {
    CK(cudaMemcpyAsync(c->Pother, c->P[c->cp], S3 * sizeof(float), cudaMemcpyDeviceToDevice, c->st));
    if (f.sic)
      for (int m = 0; m < c->n_atoms; ++m) {
        const float Zm = (float)c->atoms[m].Z;
        if (Zm == 0.f) continue;
        const float frac = Zm > 1.f ? 1.0f / Zm : 1.0f;
        LAUNCH(RQ_KC_MG, 120 * ip,
               launch_mj_sic_domain((float*)c->U[c->cu], c->lab[c->cl], c->Pother, m, frac, c->rho, c->sic, c->sic2,
                                    c->resid, c->Ec[0], c->Ec[1], c->fc, c->g, c->gc, p.h2, p.inv_h2, p.two_pi,
                                    c->st));
      }
  }
  float *HX = c->lob, *LW = HX + S3, *HW = LW + S3, *LP = HW + S3, *HP = LP + S3;
  if (c->frame == 0) CK(cudaMemsetAsync(LP, 0, 2 * S3 * sizeof(float), c->st));  // P and HP
  const int nwg = lob_workgroups(c->g);
  float* X = (float*)c->U[c->cu];
  const MjAtom* at = atoms_dev(c);
  for (int m = 0; m < c->n_atoms; ++m) {
    if ((float)c->atoms[m].Z == 0.f) continue;
    for (int it = 0; it < 10; ++it) {
      const bool hasP = c->frame > 0 || it > 0;
      LAUNCH(RQ_KC_UPDATE, 20 * ip,
             launch_lob_apply_h(X, HX, (float*)c->K, c->lab[c->cl], c->Pother, at, c->g, p.h, p.inv_h2, p.hasBare,
                                c->st));
      if (it == 0 && !hasP) CK(cudaMemsetAsync(LW, 0, 2 * S3 * sizeof(float), c->st));  // W and HW
      LAUNCH(RQ_KC_NORMALIZE, 28 * ip,
             launch_lob_inner(X, HX, LW, HW, LP, HP, c->lab[c->cl], m, c->g, p.h3, c->lob_part, c->st));
      LAUNCH(RQ_KC_NORMALIZE, 48.0 * nwg, launch_lob_finalize(c->lob_part, nwg, true, hasP, c->lob_scal, c->st));
      LAUNCH(RQ_KC_UPDATE, 24 * ip,
             launch_lob_residual(X, HX, LW, c->lab[c->cl], (float*)c->K, c->Pother, c->lob_scal, m, c->g, p.inv_h2,
                                 c->st));
      LAUNCH(RQ_KC_UPDATE, 20 * ip,
             launch_lob_apply_h(LW, HW, (float*)c->K, c->lab[c->cl], c->Pother, at, c->g, p.h, p.inv_h2, p.hasBare,
                                c->st));
      if (hasP)
        LAUNCH(RQ_KC_UPDATE, 20 * ip,
               launch_lob_apply_h(LP, HP, (float*)c->K, c->lab[c->cl], c->Pother, at, c->g, p.h, p.inv_h2, p.hasBare,
                                  c->st));
      LAUNCH(RQ_KC_NORMALIZE, 28 * ip,
             launch_lob_inner(X, HX, LW, HW, LP, HP, c->lab[c->cl], m, c->g, p.h3, c->lob_part, c->st));
      LAUNCH(RQ_KC_NORMALIZE, 48.0 * nwg, launch_lob_finalize(c->lob_part, nwg, false, hasP, c->lob_scal, c->st));
      LAUNCH(RQ_KC_UPDATE, 24 * ip, launch_lob_update(X, LW, LP, c->lab[c->cl], c->lob_scal + 1, m, c->g, c->st));
    }
  }
  CK(cudaMemsetAsync(c->unorm, 0, sizeof(unsigned) * c->n_atoms, c->st));
  LAUNCH(RQ_KC_NORMALIZE, 8 * ip, launch_mj_accum_norms(X, c->lab[c->cl], c->g, p.h3, c->unorm, c->st));
  LAUNCH(RQ_KC_NORMALIZE, 8.0 * c->n_atoms, launch_mj_norm_scale(c->unorm, at, c->n_atoms, c->scale, c->st));
  LAUNCH(RQ_KC_NORMALIZE, 12 * ip, launch_mj_apply_scale(X, c->lab[c->cl], c->scale, c->g, c->st));
  LAUNCH(RQ_KC_UPDATE, 20 * ip,
         launch_mj_update(X, (float*)c->U[1 - c->cu], (float*)c->K, c->lab[c->cl], c->Pother, c->g, p.half_d, p.dt,
                          p.h3, c->n_atoms, nullptr, c->st));
  c->cu ^= 1;
  c->frame++;
  const int wsteps = c->freeze ? 0 : f.steps_per_frame > 1 ? f.steps_per_frame : 1;  // :107; FREEZE_BOUNDARY :3643
  for (int q = 0; q < wsteps; ++q) {
    LAUNCH(RQ_KC_LABELS, 20 * ip,
           launch_mj_evolve(c->lab[c->cl], c->lab[1 - c->cl], (float*)c->U[c->cu], c->W, at, c->n_atoms, c->g, p.dt_w,
                            p.curvReg, p.h, p.hasBare, c->lock, c->splits, c->st));
    c->cl ^= 1;
    // the spare buffer takes the new labels' faces: those of the page's label2Buf
    LAUNCH(RQ_KC_LABELS, 8.0 * 6 * c->g.S2, launch_copy_faces(c->lab[c->cl], c->lab[1 - c->cl], c->g, c->st));
  }
  return RQ_OK;
}

int mj_step_one(rq_ctx* c, int s) {
  if (c->cfg.lobpcg) return mj_lobpcg_frame(c);
  const MjParams p = mj_params(c);
  const rq_config& f = c->cfg;
  const int spf = f.steps_per_frame;
  const int sf = (s - 1) % spf;  // position inside the frame (doSteps' s)
  const bool poisson = p.n_electrons > 1.0;
  const double ip = interior(c->g);
  const bool direct = mj_direct(c);
  if (poisson && direct) {
    for (int m = 0; m < c->n_atoms; ++m) {
      if ((float)c->atoms[m].Z == 0.f) continue;
      LAUNCH(RQ_KC_POISSON, 128 * ip,
             launch_mj_direct_domain((float*)c->U[c->cu], c->lab[c->cl], c->Pother, m,
                                     c->pdirect + (size_t)m * c->g.S3, c->sic, c->rho, c->g, p.h2, p.two_pi, c->st));
    }
  } else if (poisson) {
    for (int js = 0; js < f.jacobi_per_step; ++js) {
      LAUNCH(RQ_KC_POISSON, 12 * ip,
             launch_mj_jacobi((float*)c->P[c->cp], (float*)c->P[1 - c->cp], (float*)c->U[c->cu], c->g, p.h2, p.two_pi,
                              c->st));
      c->cp ^= 1;
    }
    if (sf > 0 && sf % f.vcycle_interval == 0)  // molecule.js:2879
      LAUNCH(RQ_KC_MG, 40 * ip,
             launch_mj_vcycle((float*)c->P[c->cp], (float*)c->U[c->cu], c->rho, c->resid, c->Ec[0], c->Ec[1], c->fc,
                              c->g, c->gc, p.h2, p.inv_h2, p.two_pi, c->st));
  }
  const bool norm = ((sf + 1) % f.norm_interval == 0) || sf == spf - 1;  // molecule.js:2972
  if (norm) CK(cudaMemsetAsync(c->unorm, 0, sizeof(unsigned) * c->n_atoms, c->st));
  if (c->cfg.chebyshev) {
    const float omega = mj_cheb_omega(c);
    LAUNCH(RQ_KC_UPDATE, 24 * ip,
           launch_mj_update_cheb((float*)c->U[c->cu], (float*)c->U[1 - c->cu], (float*)c->K, c->lab[c->cl], c->Pother,
                                 c->g, p.half_d, p.dt, p.h3, c->n_atoms, norm ? c->unorm : nullptr, omega, c->st));
  } else {
    LAUNCH(RQ_KC_UPDATE, 20 * ip,
           launch_mj_update((float*)c->U[c->cu], (float*)c->U[1 - c->cu], (float*)c->K, c->lab[c->cl], c->Pother, c->g,
                            p.half_d, p.dt, p.h3, c->n_atoms, norm ? c->unorm : nullptr, c->st));
  }
  c->cu ^= 1;
  if (norm) {
    LAUNCH(RQ_KC_NORMALIZE, 8.0 * c->n_atoms,
           launch_mj_norm_scale(c->unorm, atoms_dev(c), c->n_atoms, c->scale, c->st));
    LAUNCH(RQ_KC_NORMALIZE, 12 * ip, launch_mj_apply_scale((float*)c->U[c->cu], c->lab[c->cl], c->scale, c->g, c->st));
  }
  if (sf == spf - 1) {
    // frame tail: Pother <- P_buf[0], the self-interaction correction on its frames (the frame
    // counter is the reference's frameCount, incremented before the level-set passes), then the
    // level-set passes on the same psi
    if (!poisson)
      CK(cudaMemsetAsync(c->Pother, 0, (size_t)c->g.S3 * sizeof(float), c->st));
    else if (!direct)  // the direct path builds Pother every step
      CK(cudaMemcpyAsync(c->Pother, c->P[c->cp], (size_t)c->g.S3 * sizeof(float), cudaMemcpyDeviceToDevice, c->st));
    const int sic = mj_sic_interval(c);
    if (poisson && sic > 0 && c->frame > 0 && c->frame % sic == 0) {
      for (int m = 0; m < c->n_atoms; ++m) {
        const float Zm = (float)c->atoms[m].Z;
        if (Zm == 0.f) continue;
        const float frac = Zm > 1.f ? 1.0f / Zm : 1.0f;
        LAUNCH(RQ_KC_MG, 120 * ip,
               launch_mj_sic_domain((float*)c->U[c->cu], c->lab[c->cl], c->Pother, m, frac, c->rho, c->sic, c->sic2,
                                    c->resid, c->Ec[0], c->Ec[1], c->fc, c->g, c->gc, p.h2, p.inv_h2, p.two_pi,
                                    c->st));
      }
    }
    c->frame++;
    const int wsteps = c->freeze ? 0 : spf > 1 ? spf : 1;  // W_STEPS_PER_FRAME (:107); FREEZE_BOUNDARY (:3095)
    for (int q = 0; q < wsteps; ++q) {
      LAUNCH(RQ_KC_LABELS, 20 * ip,
             launch_mj_evolve(c->lab[c->cl], c->lab[1 - c->cl], (float*)c->U[c->cu], c->W, atoms_dev(c), c->n_atoms,
                              c->g, p.dt_w, p.curvReg, p.h, p.hasBare, c->lock, c->splits, c->st));
      c->cl ^= 1;
      LAUNCH(RQ_KC_LABELS, 8.0 * 6 * c->g.S2, launch_copy_faces(c->lab[c->cl], c->lab[1 - c->cl], c->g, c->st));
    }
    if (c->cfg.chebyshev) {  // the page's E at the frame's end feeds the next frame's omega (:3186)
      double e[RQ_ENERGY_LEN], ekk = 0;
      int rc = mj_energy(c, e, nullptr);
      if (rc != RQ_OK) return rc;
      mj_nuclear_terms(c, &ekk, nullptr);
      c->cheb_E = e[RQ_E_T] + e[RQ_E_EK] + e[RQ_E_EE] + ekk;
    }
  }
  return RQ_OK;
}

// Unique nuclei of molecule.js:50-67: entries with Z>0 or Z_nuc>0 grouped by their initial
// grid position key; charge = sum of (Z_nuc || Z); the first entry's current position.
static void mj_unique_nuclei(const rq_ctx* c, std::vector<std::vector<int>>& groups, std::vector<double>& zeff) {
  std::map<std::tuple<double, double, double>, int> key;
  for (int e = 0; e < c->n_atoms; ++e) {
    const rq_atom& a = c->atoms0[e];
    if (a.Z == 0 && a.Z_nuc == 0) continue;
    // the reference keys on the page's atom positions ("i,j,k" strings): exact equality of the
    // creation-time positions
    auto k = std::make_tuple(a.i, a.j, a.k);
    auto it = key.find(k);
    const double z = a.Z_nuc != 0 ? a.Z_nuc : a.Z;
    if (it == key.end()) {
      key[k] = (int)groups.size();
      groups.push_back({e});
      zeff.push_back(z);
    } else {
      groups[it->second].push_back(e);
      zeff[it->second] += z;
    }
  }
}

void mj_nuclear_terms(rq_ctx* c, double* E, double* F) {
  // molecule.js:3170-3185 (E_KK, softening 0.04 h^2) and :3218-3242 (forces, softening h^2)
  std::vector<std::vector<int>> groups;
  std::vector<double> zeff;
  mj_unique_nuclei(c, groups, zeff);
  const double h = c->h;
  double e = 0;
  const size_t G = groups.size();
  for (size_t a = 0; a < G; ++a) {
    const rq_atom& A = c->atoms[groups[a][0]];
    double fx = 0, fy = 0, fz = 0;
    for (size_t b = 0; b < G; ++b) {
      if (b == a) continue;
      const rq_atom& B = c->atoms[groups[b][0]];
      const double dx = (A.i - B.i) * h, dy = (A.j - B.j) * h, dz = (A.k - B.k) * h;
      const double d2 = dx * dx + dy * dy + dz * dz;
      if (b > a) e += zeff[a] * zeff[b] / std::sqrt(d2 + 0.04 * h * h);
      const double r2 = d2 + h * h, r = std::sqrt(r2), inv_r3 = 1.0 / (r * r2);
      fx += zeff[a] * zeff[b] * dx * inv_r3;
      fy += zeff[a] * zeff[b] * dy * inv_r3;
      fz += zeff[a] * zeff[b] * dz * inv_r3;
    }
    if (F)
      for (int q : groups[a]) {
        F[q * 3] = fx; F[q * 3 + 1] = fy; F[q * 3 + 2] = fz;
      }
  }
  *E = e;
}

int mj_energy(rq_ctx* c, double* out, double* per_domain) {
  const MjParams p = mj_params(c);
  const int n = c->n_atoms;
  CK(cudaMemsetAsync(c->dpd, 0, sizeof(double) * 4 * n, c->st));
  CK(cudaMemsetAsync(c->dsum, 0, sizeof(double) * 8, c->st));
  LAUNCH(RQ_KC_ENERGY, 16 * interior(c->g),
         launch_mj_energy((float*)c->U[c->cu], c->Pother, (float*)c->K, c->lab[c->cl], atoms_dev(c), c->g, p.h, p.h3,
                          p.Rsing, n, c->dpd, c->dsum, c->st));
  std::vector<double> pd((size_t)4 * n);
  double dip[3];
  CK(cudaMemcpyAsync(pd.data(), c->dpd, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(dip, c->dsum, sizeof(double) * 3, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  double T = 0, EK = 0, EE = 0;
  for (int q = 0; q < n; ++q) {
    T += pd[q * 4 + 1]; EK += pd[q * 4 + 2]; EE += pd[q * 4 + 3];
    if (per_domain) {
      double* d = per_domain + (size_t)q * RQ_DOMAIN_LEN;
      d[RQ_D_NORM] = pd[q * 4]; d[RQ_D_T] = pd[q * 4 + 1]; d[RQ_D_EK] = pd[q * 4 + 2]; d[RQ_D_EE] = pd[q * 4 + 3];
      const double nr = pd[q * 4] != 0 ? pd[q * 4] : 1.0;
      d[RQ_D_EIG] = (pd[q * 4 + 1] + 2 * pd[q * 4 + 3] + pd[q * 4 + 2]) / nr;
    }
  }
  // per-H exclusion-sphere correction (molecule.js:3130-3139)
  int nH = 0;
  for (auto& a : c->atoms)
    if (a.Z == 1 && a.rc == 0) nH++;
  double raw0 = 0.503, raw1 = -1.028;  // H_RAW[200], the default
  if (c->g.NN == 100 || c->g.NN == 300) { raw0 = 0.5; raw1 = -1.0; }
  T += nH * (0.5 - raw0);
  EK += nH * (-1.0 - raw1);
  out[RQ_E_T] = T; out[RQ_E_EK] = EK; out[RQ_E_EE] = EE;
  // dipole (molecule.js:3141-3161): sum Z_a R_a h - electronic sums
  double dx = 0, dy = 0, dz = 0;
  for (auto& a : c->atoms) {
    if (a.Z == 0) continue;
    dx += a.Z * a.i * c->h; dy += a.Z * a.j * c->h; dz += a.Z * a.k * c->h;
  }
  out[RQ_E_DIPX] = dx - dip[0]; out[RQ_E_DIPY] = dy - dip[1]; out[RQ_E_DIPZ] = dz - dip[2];
  return RQ_OK;
}

int mj_forces(rq_ctx* c, int method, double* F) {
  const MjParams p = mj_params(c);
  const int n = c->n_atoms;
  if (method == RQ_FORCE_GRADP) {
    const int R = std::max(5, (int)std::lround(3.0 / c->h));  // FORCE_RADIUS (molecule.js:1198)
    LAUNCH(RQ_KC_FORCES, 4.0 * n * (2 * R + 1) * (2 * R + 1) * (2 * R + 1),
           launch_mj_gradp(mj_direct(c) ? c->Pother : (float*)c->P[c->cp], atoms_dev(c), n, c->g, p.inv_h, R, c->dF,
                           c->st));  // molecule.js:2703: Pother on the direct path
  } else if (method == RQ_FORCE_HF || method == RQ_FORCE_ADJOINT) {
    // molecule.js:1271-1330: Z_A = Z (or Z_nuc for bare nuclei), integer positions, h^2 softening
    std::vector<float> a5((size_t)n * 5);
    for (int q = 0; q < n; ++q) {
      const rq_atom& a = c->atoms[q];
      a5[q * 5 + 0] = (float)(uint32_t)(a.i < 0 ? 0 : a.i);
      a5[q * 5 + 1] = (float)(uint32_t)(a.j < 0 ? 0 : a.j);
      a5[q * 5 + 2] = (float)(uint32_t)(a.k < 0 ? 0 : a.k);
      a5[q * 5 + 3] = (float)(a.Z <= 0 ? a.Z_nuc : a.Z);
      a5[q * 5 + 4] = 0.f;
    }
    CK(cudaMemcpyAsync(c->scratch_atoms5, a5.data(), sizeof(float) * a5.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemsetAsync(c->dF, 0, sizeof(double) * 3 * n, c->st));
    LAUNCH(RQ_KC_FORCES, 4 * interior(c->g),
           launch_forces_hf_sp((float*)c->U[c->cu], c->scratch_atoms5, n, c->g, p.h, p.h2, p.h3, c->dF, c->st));
  } else {
    return RQ_ENOTSUP;
  }
  CK(cudaMemcpyAsync(F, c->dF, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return RQ_OK;
}
