// rq_flavors.h -- per-flavour schedule entry points used by capi.cu (internal).
#pragma once
#include "rq_ctx.h"

// molecule.js atom record on the device (molecule.js:183-191 without the split fields):
// positions are unsigned integers, as the Uint32Array store of :1882-1884 leaves them.
struct MjAtom {
  uint32_t posI, posJ, posK;
  float Z, rc, Z_nuc, initZeff, initRcut;
};
// The record of one entry: molecule.js:1882-1884 stores positions in a Uint32Array (truncation
// toward zero), the rest as f32; initZeff defaults to Z, initRcut to 1e6.
inline MjAtom mj_record(const rq_atom& a) {
  MjAtom m;
  m.posI = (uint32_t)(a.i < 0 ? 0 : a.i);
  m.posJ = (uint32_t)(a.j < 0 ? 0 : a.j);
  m.posK = (uint32_t)(a.k < 0 ? 0 : a.k);
  m.Z = (float)a.Z;
  m.rc = (float)a.rc;
  m.Z_nuc = (float)a.Z_nuc;
  m.initZeff = (float)(a.init_zeff > 0 ? a.init_zeff : a.Z);
  m.initRcut = (float)(a.init_rcut > 0 ? a.init_rcut : 1e6);
  return m;
}
// An entry's shell split (the atom record's split fields, molecule.js:183-191): type 0/1 whole
// sphere, 2 half space, 3 one of three 120-degree sectors; idx, axis, angular offset rot.
struct MjSplit {
  uint32_t type, idx;
  float ax, ay, az, rot;
};

// molecule.js flavour (mj_flavor.cu)
int mj_initialize(rq_ctx* c);
int mj_restart(rq_ctx* c);
int mj_step_one(rq_ctx* c, int s);
int mj_energy(rq_ctx* c, double* out, double* per_domain);
int mj_forces(rq_ctx* c, int method, double* F);
int mj_set_atoms(rq_ctx* c);
int mj_refresh_flags(rq_ctx* c);
void mj_nuclear_terms(rq_ctx* c, double* E, double* F);

// new flavour (nm_flavor.cu)
int nm_alloc_levels(rq_ctx* c);
int nm_initialize(rq_ctx* c);
int nm_promote(rq_ctx* c);  // mixed -> FP64 in place (psi, P widened; K recomputed)
int nm_step_one(rq_ctx* c, int s);
int nm_energy(rq_ctx* c, double* out, double* per_domain);
int nm_forces(rq_ctx* c, int method, double* F);
int nm_set_atoms(rq_ctx* c);
int nm_set_external(rq_ctx* c, const double* v);
bool mj_direct(const rq_ctx* c);      // molecule.js flavour on the direct per-electron Poisson path
int mj_sic_interval(const rq_ctx* c);  // frames between SIC passes of the molecule.js flavour (0: off)
int nm_flush(rq_ctx* c);  // materialise a pending per-domain normalisation of psi
int nm_ready(rq_ctx* c);  // nm_flush, or normalise now when updates ran since the last normalisation
// adjoint of the new flavour (nm_adjoint.cu)
int nm_adj_set_window(rq_ctx* c, int steps);  // allocate / free the recording window (0: off)
void nm_adj_reset(rq_ctx* c);                 // forget the recorded steps (state or geometry changed)
int nm_adj_record_step(rq_ctx* c, bool vcycle, bool norm);  // before the update of a step
int nm_adj_record_scale(rq_ctx* c);           // after the normalisation scale of that step
void nm_adj_record_label(rq_ctx* c);          // a label pass followed the step
int nm_adjoint(rq_ctx* c, double* F, double* dEdv);
void nm_adj_free(rq_ctx* c);
int nm_nuclear_terms(rq_ctx* c, double* E, double* F);
int nm_label_mask(rq_ctx* c);  // the update's same-label neighbour mask, after a label change
// nuclear sums (nm_farfield.cu): K (field type, and K64 when given) for the current nuclei, tiled
// or direct by cfg.nuclear_sum; a force gather over psi (weight rho) or over gw = dE/dK, added
// into c->dF; the tiles' buffers
int nm_nuclear_potential(rq_ctx* c, void* K, double* K64);
int nm_gather(rq_ctx* c, const void* U, const double* gw);
void nm_ff_free(rq_ctx* c);
