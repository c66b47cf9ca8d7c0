// mj_flavor.cu -- molecule.js flavour (placeholder until its kernels land).
#include "rq_flavors.h"
int mj_initialize(rq_ctx* c) { return rq_fail(c, RQ_ENOTSUP, "molecule.js flavour not built yet"); }
int mj_step_one(rq_ctx* c, int) { return rq_fail(c, RQ_ENOTSUP, "molecule.js flavour not built yet"); }
int mj_energy(rq_ctx* c, double*, double*) { return rq_fail(c, RQ_ENOTSUP, "molecule.js flavour not built yet"); }
int mj_forces(rq_ctx* c, int, double*) { return rq_fail(c, RQ_ENOTSUP, "molecule.js flavour not built yet"); }
int mj_set_atoms(rq_ctx* c) { return rq_fail(c, RQ_ENOTSUP, "molecule.js flavour not built yet"); }
void mj_nuclear_terms(rq_ctx*, double* E, double*) { *E = 0; }
