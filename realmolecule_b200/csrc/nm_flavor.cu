// nm_flavor.cu -- new flavour (placeholder until its kernels land).
#include "rq_flavors.h"
int nm_alloc_levels(rq_ctx*) { return RQ_OK; }
int nm_initialize(rq_ctx* c) { return rq_fail(c, RQ_ENOTSUP, "new flavour not built yet"); }
int nm_step_one(rq_ctx* c, int) { return rq_fail(c, RQ_ENOTSUP, "new flavour not built yet"); }
int nm_energy(rq_ctx* c, double*, double*) { return rq_fail(c, RQ_ENOTSUP, "new flavour not built yet"); }
int nm_forces(rq_ctx* c, int, double*) { return rq_fail(c, RQ_ENOTSUP, "new flavour not built yet"); }
int nm_set_atoms(rq_ctx* c) { return rq_fail(c, RQ_ENOTSUP, "new flavour not built yet"); }
void nm_nuclear_terms(rq_ctx*, double* E, double*) { *E = 0; }
