/*
 * rq.h -- C ABI of librq, the B200-native RealQM real-space solver step.
 *
 * One context (rq_ctx) owns every device buffer of one grid: the density field psi
 * (double-buffered), the int32 domain label per voxel (double-buffered), the nuclear
 * potential K, the Hartree half-potential P, the level-set field W and the FP64
 * per-domain sums.  All entry points return RQ_OK (0) or a negative RQ_E* status;
 * nothing throws or aborts across this boundary.  Host buffers belong to the caller
 * and are copied; device memory belongs to the context.
 *
 * Grid convention (both reference hosts): S = NN+1 points per axis, linear index
 * id = i*S*S + j*S + k (k fastest), the outer planes are Dirichlet boundary
 * (cloud/solver.py:20-30, molecule.js:268-276).  Atom positions are in grid units
 * (x = i*h), like the reference's {i, j, k} atom records.
 *
 * Threading: a context is used by one host thread at a time and issues its work on
 * one CUDA stream (rq_set_stream).  Different contexts are independent.
 *
 * Each entry point cites the reference interface it replaces.
 */
#ifndef RQ_H
#define RQ_H

#include <stdint.h>

#if defined(__GNUC__)
#define RQ_API __attribute__((visibility("default")))
#else
#define RQ_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------- */
#define RQ_OK 0
#define RQ_EINVAL (-1)      /* bad argument (null pointer, size, out-of-range label) */
#define RQ_ENOMEM (-2)      /* device or host allocation failed */
#define RQ_ECUDA (-3)       /* a CUDA runtime call failed (message in rq_last_error) */
#define RQ_ENONFINITE (-4)  /* NaN/Inf detected in an energy or norm (molecule.js:3198-3201) */
#define RQ_ETIMEOUT (-5)    /* a bounded device wait gave up (batched work queue) */
#define RQ_ENOTSUP (-6)     /* option not supported by this flavour */
#define RQ_ENODEV (-7)      /* no CUDA device */

/* ---- flavours and precision ---------------------------------------------------------- */
typedef enum {
  RQ_FLAVOR_MOLECULE_JS = 0, /* molecule.js WGSL step (r_c exclusion, W level set, weighted Jacobi) */
  RQ_FLAVOR_SOLVER_PY = 1,   /* cloud/solver.py CUDA-C step (Jacobi every 2, labels every 100) */
  RQ_FLAVOR_NEW = 2          /* Gaussian nuclei, red-black multigrid, FP64 domain sums */
} rq_flavor;

typedef enum {
  RQ_PREC_MIXED = 0, /* fp32 fields and stencils, FP64 domain sums / energies / coarsest solve */
  RQ_PREC_FP64 = 1   /* every field FP64 (the plain path the mixed path is compared against) */
} rq_precision;

/* ---- configuration (mirrors window.USER_* of molecule.js:4-152 and the config dict of
 *      cloud/solver.py:321-362).  Zero / negative numeric fields take the flavour default. ---- */
typedef struct rq_config {
  int32_t NN;               /* grid intervals per axis (USER_NN / gridN); S = NN+1 */
  int32_t flavor;           /* rq_flavor */
  int32_t precision;        /* rq_precision (RQ_PREC_FP64 only with RQ_FLAVOR_NEW) */
  int32_t norm_interval;    /* normalise every n steps (solver.py 20, molecule.js NORM_INTERVAL 20); new
                               flavour: also always before each V-cycle and label pass (default
                               poisson_interval) */
  double screen;            /* box edge in bohr (USER_SCREEN / screen); h = screen/NN */
  double dv;                /* dt = dv*h^2; <=0 -> flavour table (molecule.js:78, solver.py:342-351) */
  int32_t poisson_interval; /* solver.py: Poisson step every 2; new: one V-cycle every n steps (4) */
  int32_t label_interval;   /* solver.py: 5*norm_interval (100); new: level-set step period */
  int32_t jacobi_per_step;  /* Jacobi sweeps per Poisson step (2 in both references) */
  int32_t steps_per_frame;  /* molecule.js STEPS_PER_FRAME (frame = steps + energy + labels) */
  int32_t vcycle_interval;  /* molecule.js POISSON_INTERVAL (50) */
  int32_t mg_levels;        /* new: multigrid levels (<=0: as deep as NN allows, coarsest >= 4) */
  int32_t mg_pre, mg_post;  /* new: red-black sweeps before / after the coarse correction (1, 1) */
  int32_t mg_coarse_sweeps; /* new: FP64 red-black sweeps on the coarsest level (16) */
  int32_t sic;              /* molecule.js flavour: 1 = the reference's own Pother path (:111-112):
                               <= 5 domains the direct per-electron Poisson (:2833-2858), else the
                               self-interaction correction (:3009-3076) every frame (<= 15 domains)
                               or every 5th (<= 30), none above; 0 = total Poisson, no correction */
  double boundary_speed;    /* molecule.js dt_w (0.5, :135) */
  double curv_reg;          /* molecule.js curvReg (0: 0.15 as :34; < 0: off) */
  double sigma;             /* new: Gaussian nucleus width in bohr (<=0: h) */
  int32_t label_until;      /* labels update only while steps_done < label_until (0: always) */
  int32_t chebyshev;        /* molecule.js flavour, 1: the Chebyshev semi-iterative update instead of plain
                               ITP (molecule.js:345-421, :2915-2962), omega from the page's recurrence and the
                               previous frame's energy; frames run eagerly; not with bare nuclei (Z = 0,
                               Z_nuc > 0, rc > 0: RQ_ENOTSUP) */
  int32_t lobpcg;           /* molecule.js flavour, 1: every step is one LOBPCG frame (doLOBPCGStep,
                               molecule.js:3323-3740; the page's useLOBPCG, :1751): the Poisson solve and
                               Pother, 10 LOBPCG iterations per domain (Ritz problems solved on the device
                               in FP64), normalisation, one ITP update, the level-set passes; not with
                               chebyshev (RQ_EINVAL) */
  int32_t converge_checks;  /* rq_solve / rq_batch_solve: converged after this many consecutive checks with
                               |dE| < tol (molecule.js counts 3 frames within CONVERGENCE_THRESHOLD,
                               :4645-4659); <= 0: 1 */
  int32_t fp32_rounding;    /* new flavour, RQ_PREC_MIXED: 0 = the psi update rounds to nearest; 1 = it rounds
                               without bias (exact FP64 value, rounded down or up with the probability of
                               its position between the two f32 neighbours; a counter-based hash per point
                               and step, so runs repeat) */
  int32_t nuclear_sum;      /* new flavour: how K and the force gathers sum over nuclei.  0 (auto): tiled when
                               the interior has >= 64 points per axis and there are >= 64 nuclei, else direct;
                               1: direct (every nucleus at every voxel); 2: tiled whenever the interior has
                               >= 32 points per axis.  Tiled: per 32^3 tile, nuclei within 3 tile half-widths
                               direct, the rest through a 16^3-node Chebyshev interpolant of their Coulomb
                               field (K within 1e-12 relative of the direct sum; the force gather is its exact
                               transpose) */
  int32_t batch_persistent; /* rq_batch_*: 0 = one launch per kernel and phase, the period captured as one CUDA
                               graph (default: measured fastest on B200); 1 = each schedule period is ONE
                               persistent cooperative launch (blocks take chunks of (instance, tile) items from
                               one queue; an item waits, bounded, only for its instance's previous phase).
                               rq_batch_autotune times both and keeps the faster. */
  int32_t batch_tile;       /* rq_batch_*: march tile of the update, readout and level-set work lists, as
                               log2(points along k) | (planes per thread << 8), 256 threads per tile; 0 = 16 x 16
                               x 16 (4 | 16 << 8).  rq_batch_autotune picks it. */
} rq_config;

/* One entry of the reference atom list: a nucleus and/or one electron domain. */
typedef struct rq_atom {
  double i, j, k;    /* position in grid units; molecule.js stores them as u32 (:1882-1884) */
  double Z;          /* charge of this entry's electron domain (Z_eff); 0 = no domain */
  double Z_nuc;      /* nuclear charge placed here (molecule.js Z_nuc; the Python host sets Z) */
  double rc;         /* pseudopotential core radius in bohr (0 = bare Coulomb) */
  double init_zeff;  /* molecule.js initZeff for the trial psi (<=0: Z) */
  double init_rcut;  /* molecule.js initRcut (<=0: 1e6) */
} rq_atom;

typedef struct rq_ctx rq_ctx;

/* Read-only facts about a context (sizes, chosen defaults, device pointers for zero-copy). */
typedef struct rq_info {
  int32_t NN, S, n_atoms, flavor, precision, steps_done, mg_levels, _pad;
  double h, dv, dt, sigma;
  int64_t S3;
  void* psi;   /* current psi (float* or double* by precision) */
  void* label; /* current int32 labels */
  void* K;     /* nuclear potential (same type as psi) */
  void* P;     /* Hartree half-potential (same type as psi) */
  void* W;     /* level-set field (float*) */
  int64_t kernel_launches; /* librq kernels launched by this context so far (graph replays included) */
} rq_info;

/* Kernel classes for the per-kernel profile (CUDA events around each launch). */
#define RQ_KC_UPDATE 0    /* fused ITP update (+ FP64 domain norms on normalisation steps) */
#define RQ_KC_POISSON 1   /* Jacobi / red-black smoother sweeps on the fine grid */
#define RQ_KC_LABELS 2    /* label / level-set update */
#define RQ_KC_NORMALIZE 3 /* norm scale + apply */
#define RQ_KC_ENERGY 4    /* per-domain energy sums */
#define RQ_KC_FORCES 5    /* force gathers */
#define RQ_KC_MG 6        /* multigrid transfer and coarse levels */
#define RQ_KC_OTHER 7     /* init, potential, copies */
#define RQ_KC_COUNT 8

typedef struct rq_profile {
  int64_t launches[RQ_KC_COUNT];  /* launches per class between begin and end */
  double ms[RQ_KC_COUNT];         /* summed CUDA-event durations (ms) */
  double bytes[RQ_KC_COUNT];      /* summed algorithmic bytes (reads + writes the kernel must do) */
} rq_profile;

/* Energy vector returned by rq_energy (molecule.js:3124-3195, cloud/solver.py:446-476). */
#define RQ_E_TOTAL 0
#define RQ_E_T 1
#define RQ_E_EK 2
#define RQ_E_EE 3
#define RQ_E_KK 4
#define RQ_E_DIPX 5
#define RQ_E_DIPY 6
#define RQ_E_DIPZ 7
#define RQ_ENERGY_LEN 8

/* Per-domain columns of rq_energy's per_domain (n_atoms x 5); atom.js:259-283, :340-342. */
#define RQ_D_NORM 0
#define RQ_D_T 1
#define RQ_D_EK 2
#define RQ_D_EE 3
#define RQ_D_EIG 4
#define RQ_DOMAIN_LEN 5

/* Force methods for rq_forces. */
#define RQ_FORCE_HF 0      /* Hellmann-Feynman integral: cloud/solver.py:282-315, molecule.js:1271-1330 */
#define RQ_FORCE_GRADP 1   /* molecule.js gradPtotal (:1200-1269) */
#define RQ_FORCE_ADJOINT 2 /* new flavour: -dE/dR of the energy readout, by the reverse sweep through the steps
                              recorded since the last reset (rq_set_adjoint_window); without a window the
                              Hellmann-Feynman gather, exact at a converged state.  Other flavours: as HF */

/* ---- lifecycle ---------------------------------------------------------------------- */
/* Replaces RealQMSolver.__init__ (cloud/solver.py:321-400) and molecule.js initGPU buffer
 * set-up (:2263-2347).  Allocates every device buffer of the grid. */
RQ_API int rq_create(const rq_config* cfg, const rq_atom* atoms, int32_t n_atoms, rq_ctx** out);
RQ_API void rq_destroy(rq_ctx* ctx);
/* Binds the context to a CUDA stream (cudaStream_t passed as void*; NULL = the stream the
 * context created for itself).  Pending work on the previous stream is finished first. */
RQ_API int rq_set_stream(rq_ctx* ctx, void* stream);
/* Device pointers in info are the live fields; for the new flavour call rq_synchronize first
 * (it materialises a per-domain normalisation that the next update would otherwise apply). */
RQ_API int rq_get_info(const rq_ctx* ctx, rq_info* info);
RQ_API const char* rq_last_error(const rq_ctx* ctx);
RQ_API const char* rq_status_string(int status);

/* ---- state -------------------------------------------------------------------------- */
/* RealQMSolver.initialize (cloud/solver.py:402-419): trial psi, labels, K, normalise, then
 * 100 Poisson bootstrap steps; molecule.js uploadInitialData (:1905-2101) for that flavour;
 * new flavour: nearest-seed labels, psi ~ exp(-|x-seed|) normalised per domain, one MG solve. */
RQ_API int rq_initialize(rq_ctx* ctx);
/* molecule.js window.FREEZE_BOUNDARY (molecule.js:3095, :3643): with on != 0 the frames skip the
 * level-set passes (labels and W stay as they are; the frame counter still advances); 0 lets the
 * boundaries move again (the page's UNLOCK_AT_STEP, :4621-4624).  molecule.js flavour only. */
RQ_API int rq_set_freeze_boundary(rq_ctx* ctx, int32_t on);
/* molecule.js window.USER_INIT_POS (molecule.js:1905-1981): for the next rq_initialize, the trial psi
 * and the initial labels are built with entry q moved to (pos[2q], pos[2q+1]) in grid units where
 * has[q] != 0 (k unchanged); K is then rebuilt from 0 at the true positions with the page's recomputeK
 * (:1337-1370).  n = 0 clears.  molecule.js flavour only. */
RQ_API int rq_set_init_positions(rq_ctx* ctx, const double* pos, const int32_t* has, int32_t n);
/* The molecule.js classical-MD backbone's full restart (USER_CLASSICAL_MD, molecule.js:4236-4286),
 * after rq_set_atoms with the moved positions: K, the trial psi and the labels rebuilt from scratch,
 * P cleared; unlike rq_initialize the level-set W and Pother (the stale potential the next frame's
 * updates read) are kept.  molecule.js flavour only. */
RQ_API int rq_restart(rq_ctx* ctx);
/* Move nuclei and rebuild K (cloud/solver.py:538-548, molecule.js:4563-4582 without relabel). */
RQ_API int rq_set_atoms(rq_ctx* ctx, const rq_atom* atoms, int32_t n_atoms);
/* molecule.js locked groups (window.USER_LOCKED_GROUPS, molecule.js:490-503, compiled into the
 * page's evolveBoundary shader): group g holds the labels members[offsets[g] .. offsets[g+1]-1]; a
 * boundary cell whose label and best neighbouring label are in one group keeps its label and its
 * level-set value becomes max(W, 0.5).  n_groups = 0 removes the groups.  At most 64 groups
 * (RQ_ENOTSUP above), members in [0, n_atoms) (RQ_EINVAL); molecule.js flavour only. */
RQ_API int rq_set_locked_groups(rq_ctx* ctx, int32_t n_groups, const int32_t* offsets, const int32_t* members);
/* molecule.js shell splits (window.USER_SPLIT_TYPE / _IDX / _AXIS / _ROT, molecule.js:27-32, the atom
 * record's split fields :183-191, inSplitAtom :197-226), one record per atom entry: the entry owns
 * only the cells of its angular sector around its nucleus -- type 2 a half space (idx 0: d.axis < 0,
 * else >= 0), type 3 one of three 120-degree sectors about the axis (sector idx, offset rot in
 * radians); 0, 1 (and 4, which the page leaves unrestricted) the whole sphere.  Used by the trial
 * labelling of rq_initialize and rq_set_atoms (gpuInitAccum, :1377-1426) and by the level-set step
 * (:514-533), so set them before rq_initialize.  NULL removes them.  molecule.js flavour only. */
typedef struct rq_split {
  int32_t type, idx;
  double axis[3];
  double rot;
} rq_split;
RQ_API int rq_set_splits(rq_ctx* ctx, const rq_split* splits);
/* External potential v (S^3 doubles, Ha, in host memory or in this GPU's device memory) added to
 * the nuclear potential K of the new flavour: the update uses K + v and E_eK = -h^3 sum (K + v) rho.
 * NULL removes it.  No reference counterpart: the handle through which dE/dv (rq_adjoint) is
 * exposed to autograd. */
RQ_API int rq_set_external_potential(rq_ctx* ctx, const double* v);
/* Copy a full state in / out (host arrays of S^3 elements; any pointer may be NULL to skip).
 * Labels must lie in [0, n_atoms).  Replaces window.restartWithPositions re-uploads
 * (molecule.js:2127-2147) and direct access to RealQMSolver.U / .label. */
RQ_API int rq_upload_state(rq_ctx* ctx, const float* psi, const int32_t* label, const float* W, const float* P);
RQ_API int rq_download_state(rq_ctx* ctx, float* psi, int32_t* label, float* W, float* P);
RQ_API int rq_upload_state_f64(rq_ctx* ctx, const double* psi, const double* P);
RQ_API int rq_download_state_f64(rq_ctx* ctx, double* psi, double* P, double* K);
RQ_API int rq_download_K(rq_ctx* ctx, float* K);

/* ---- the solver step ------------------------------------------------------------------- */
/* n solver steps on the flavour schedule: the loop body of RealQMSolver.run
 * (cloud/solver.py:561-591) or the s-loop of molecule.js doSteps (:2829-3006) with the
 * frame tail (:3009-3104) every steps_per_frame steps.  Asynchronous on the stream. */
RQ_API int rq_step(rq_ctx* ctx, int32_t n_steps);
/* Energies (FP64 sums).  out[RQ_ENERGY_LEN]; per_domain may be NULL or n_atoms*RQ_DOMAIN_LEN.
 * Synchronises the stream.  Returns RQ_ENONFINITE if any component is NaN/Inf. */
RQ_API int rq_energy(rq_ctx* ctx, double* out, double* per_domain);
/* Electronic forces on every atom entry (n_atoms x 3, FP64), without nuclear-nuclear terms.
 * cloud/solver.py _compute_forces (:478-502); molecule.js gradPtotal / HF (:1200-1330). */
RQ_API int rq_forces(rq_ctx* ctx, int32_t method, double* F);
/* Nuclear-nuclear energy and forces with the flavour's softening (host-side terms of
 * cloud/solver.py:462-474, :504-520 and molecule.js:3170-3185, :3218-3242). */
RQ_API int rq_nuclear_terms(rq_ctx* ctx, double* E_KK, double* F /* n_atoms x 3 or NULL */);
/* Step until |E_n - E_{n-1}| < tol_dE on converge_checks consecutive checks every check_interval
 * steps.  New flavour, RQ_PREC_MIXED: a context first converges to max(tol_dE, 1e-12 |E|), the change
 * between checks its fp32 fields resolve; if that is looser than tol_dE it is promoted to FP64 in
 * place (rq_promote) and continues to tol_dE, as rq_batch_solve does. */
/* molecule.js flavour: extractWGSL (molecule.js:1108-1192, W_CUTOFF = 0) as a headless buffer of
 * 3 S^2 + 2 S floats -- u^2 on the slice k = slice_k, label + 1000 Z of the label, boundary flags,
 * then the K line and the w line along (i, slice_k, slice_k).  1 <= slice_k < NN. */
RQ_API int rq_extract(rq_ctx* ctx, int32_t slice_k, float* out);
/* No counterpart in the reference.  New flavour, RQ_PREC_MIXED: continue in FP64 from the current
 * state (psi and P widened, K recomputed in FP64); the context is RQ_PREC_FP64 afterwards.  fp32
 * fields stop resolving the energy at a few 1e-8 |E|; a mixed solve followed by this and more
 * steps reaches the FP64 fixed point.  No-op on an FP64 context; RQ_ENOTSUP for other flavours. */
RQ_API int rq_promote(rq_ctx* ctx);
RQ_API int rq_solve(rq_ctx* ctx, double tol_dE, int32_t max_steps, int32_t check_interval, int32_t* steps_taken,
             double* E_final);
/* Exact gradients of the new flavour's energy readout (no single reference call site: the reference
 * forces are the Hellmann-Feynman integral cloud/solver.py:282-315 / molecule.js:1271-1330 and the
 * Hartree-gradient ball molecule.js:1200-1269, exact only at convergence).
 * rq_set_adjoint_window(ctx, K): from now on every rq_step records the state each step starts
 * from, keeping the last K steps (K x S^3 psi, K / poisson_interval + 2 x S^3 P and K x n_atoms
 * scales of device memory; 0 switches recording off).  Recorded steps run eagerly (no CUDA-graph
 * replay).  The window forgets its steps whenever the state or the geometry changes
 * (rq_initialize, rq_set_atoms, rq_set_external_potential, uploads, rq_promote): the state at that
 * moment is the fixed starting point of the gradient.
 * rq_adjoint(ctx, F, dE_dv): reverse sweep from the current readout back through the recorded steps
 * (update, per-domain normalisation and multigrid V-cycle transposed, labels held fixed), giving
 * F = -dE/dR of every entry (n_atoms x 3 in host memory, electronic part, NULL to skip) and dE/dv
 * for an external potential (S^3 doubles in host or device memory, NULL to skip).  The gradient is exact for the energy reached from the
 * window's starting state when every step since it fits in the window; with more steps the sweep
 * stops at the oldest kept step.  RQ_ENOTSUP if a label pass ran inside the window (set
 * label_until).  Synchronises. */
RQ_API int rq_set_adjoint_window(rq_ctx* ctx, int32_t steps);
RQ_API int rq_adjoint(rq_ctx* ctx, double* F, double* dE_dv);
RQ_API int rq_synchronize(rq_ctx* ctx);
/* Per-kernel timing (the reference only times whole frames, molecule.js:2823, :3168,
 * and whole runs, cloud/solver.py:559-597): between begin and end every launch of the context
 * is bracketed by CUDA events on its stream.  Work recorded while profiling runs eagerly
 * (no CUDA-graph replay).  end synchronises and fills *out. */
RQ_API int rq_profile_begin(rq_ctx* ctx);
RQ_API int rq_profile_end(rq_ctx* ctx, rq_profile* out);

/* ---- batches of independent new-flavour instances with uneven grids ----------------------
 * No single reference call site: the reference runs one molecule per process (cloud/app.py:70-87
 * loops jobs serially).  A batch steps n_inst instances in lockstep; every kernel of the
 * schedule is one launch over an (instance, tile) work list, and a schedule period is one CUDA
 * graph.  cfgs[q] gives each instance's NN and screen (one flavour RQ_FLAVOR_NEW, one precision
 * and one grid spacing h for the batch; the intervals of cfgs[0] apply to all).  atoms holds the
 * entries of instance 0, then instance 1, ... (n_atoms[q] each). */
typedef struct rq_batch rq_batch;
RQ_API int rq_batch_create(const rq_config* cfgs, const rq_atom* atoms, const int32_t* n_atoms, int32_t n_inst,
                           rq_batch** out);
RQ_API void rq_batch_destroy(rq_batch* b);
RQ_API const char* rq_batch_last_error(const rq_batch* b);
RQ_API int rq_batch_set_stream(rq_batch* b, void* stream);
RQ_API int rq_batch_initialize(rq_batch* b);
RQ_API int rq_batch_step(rq_batch* b, int32_t n_steps);
/* out: n_inst x RQ_ENERGY_LEN (dipole entries 0).  Synchronises. */
RQ_API int rq_batch_energy(rq_batch* b, double* out);
/* Forces on every entry (sum of n_atoms x 3, instance-major), electronic + nuclear repulsion. */
RQ_API int rq_batch_forces(rq_batch* b, double* F);
/* Steps until every instance's |dE| between checks is below tol_dE; converged_at[q] = step count
 * at which instance q converged (-1 if not within max_steps); E_final[q] its last energy. */
RQ_API int rq_batch_solve(rq_batch* b, double tol_dE, int32_t max_steps, int32_t check_interval, int32_t* converged_at,
                          double* E_final);
RQ_API int rq_batch_info(const rq_batch* b, int32_t* n_inst, int64_t* total_points, int64_t* interior_points,
                         int64_t* kernel_launches);
RQ_API int rq_batch_synchronize(rq_batch* b);

/* Bounds of the persistent batch launch's waits (batch_persistent = 1; no reference counterpart: the
 * reference steps one molecule at a time).  An item of the launch waits until its instance's previous
 * phase is complete; every such wait gives up after limit_ns nanoseconds (default 2e9) and then every
 * block leaves the launch; the next readout (rq_batch_energy, rq_batch_solve) returns RQ_ETIMEOUT, and
 * the state must be re-initialised.  extra_arrivals > 0 makes every wait need that many completions
 * more than there are, so every wait runs out (a test of the timeout path on a healthy device).  Drops
 * the captured periods. */
RQ_API int rq_batch_set_wait(rq_batch* b, int64_t limit_ns, int32_t extra_arrivals);

/* The batch's own autotuner (no reference counterpart).  Needs an initialised batch; its timing runs
 * are steps of the solve (the state moves on as under rq_batch_step) and leave the multigrid
 * correction P as it was.
 *   1. March tile x launch form: each candidate (tiles 16 x 16 and 32 x 8 points with 8, 16 or 32
 *      planes per thread; per-kernel graph or persistent launch) runs one schedule period to capture
 *      it and one timed by CUDA events; the fastest per step is kept.
 *   2. Smoother sweeps (mg_pre, mg_post, mg_coarse_sweeps): from P = 0 each candidate runs 3 V-cycles
 *      on the batch's current psi (rho: fine-grid residual reduction per cycle); the cheapest cycle
 *      whose rho is within 5 % of V(1,1)'s is kept (a warm-started cycle every poisson_interval steps
 *      at V(1,1)'s rate already keeps P on the ITP state).
 * The kept values go into the batch's configuration (batch_tile, batch_persistent, mg_*), and the
 * report lists every candidate. */
typedef struct rq_tune_report {
  int32_t n_tile;                  /* tile x launch candidates timed */
  int32_t tile[12], persistent[12];
  double ms_per_step[12];
  int32_t n_smooth;                /* smoother candidates */
  int32_t pre[8], post[8], coarse_sweeps[8];
  double rho[8], ms_per_cycle[8];
  int32_t best_tile, best_smooth;  /* indices of the kept candidates */
  int32_t reserved[6];
} rq_tune_report;
RQ_API int rq_batch_autotune(rq_batch* b, rq_tune_report* out);

/* ---- atom.js per-shell solver (atom.js:1-346) ----------------------------------------------
 * Replaces atom.js's module state and physicsStep(): one U (density amplitude), W (front) and P
 * (Hartree potential of the other shells) field per electron shell on an S^3 grid (S = NN+1)
 * centred on one nucleus of charge Z_kernel.  The in-place lexicographic sweep of the reference
 * runs as a hyperplane wavefront, so every f32 store is the reference's; only the FP64 sums of
 * the normalisation and the energies are summed in another order. */
typedef struct rq_shells rq_shells;
typedef struct rq_shells_config {
  int32_t NN;       /* USER_NN (even) */
  int32_t poisson;  /* USER_POISSON: 0 'multigrid' (default), 1 'simultaneous' */
  double screen;    /* USER_SCREEN, box edge in bohr */
  double Z_kernel;  /* USER_Z_KERNEL */
  double d;         /* USER_D: dt = d h^2 */
  int32_t reserved[4];
} rq_shells_config;
typedef struct rq_shell {  /* one entry of USER_SHELLS */
  double ne, Rmax, Zeff;   /* Rmax 0: screen/2 for shells after the first */
  int32_t split;           /* 1: split 'halfspace' */
  int32_t half_index;      /* halfIndex of a half-space shell */
  int32_t outer_half;      /* outerHalf */
  int32_t fixed_w;         /* fixedW: the front of this shell does not move */
} rq_shell;
/* at most 8 shells; the initial state (atom.js:55-125) is built at creation */
RQ_API int rq_shells_create(const rq_shells_config* cfg, const rq_shell* shells, int32_t n_shells, rq_shells** out);
RQ_API void rq_shells_destroy(rq_shells* s);
RQ_API const char* rq_shells_last_error(const rq_shells* s);
/* n physicsStep() calls (atom.js:212-343).  E (4 or NULL) = {E, E_T, E_eK, E_ee} of the last one;
 * per_shell (n_shells x 5 or NULL) = {ET_m, Eee_m, EeK_m, nrm_m, eig_m}.  Synchronises. */
RQ_API int rq_shells_step(rq_shells* s, int32_t n, double* E, double* per_shell);
RQ_API int rq_shells_download(rq_shells* s, int32_t shell, float* U, float* W, float* P);
RQ_API int rq_shells_upload(rq_shells* s, int32_t shell, const float* U, const float* W, const float* P);
RQ_API int rq_shells_info(const rq_shells* s, int64_t* kernel_launches);

/* ---- mol_fast.js multi-field solver (mol_fast.js:1-1651) ------------------------------------
 * Replaces mol_fast.js's GPU state and doSteps()/computeForces(): one U (density amplitude),
 * W (front) and P (Hartree potential of its own density) field per electron, one electron per
 * nucleus (at most 16), all electrons advanced by one fused pass per step (competition front,
 * weighted Laplacian, Hartree of the others, Poisson), the reference's f32 tree reductions for
 * the norms and energies, normalisation every 20 steps and at the end of a frame, and the
 * two-level Poisson correction of every electron every vcycle_interval steps of a frame.  The
 * f32 arithmetic follows the shaders' operation order (no contraction). */
typedef struct rq_mf rq_mf;
typedef struct rq_mf_config {
  int32_t NN;                 /* USER_NN (even) */
  int32_t shell_mode;         /* USER_SHELL_MODE: rc / r_out / angular split per orbital */
  int32_t vcycle;             /* USER_VCYCLE !== false */
  int32_t vcycle_interval;    /* USER_VCYCLE_INTERVAL (50) */
  int32_t coarse_iters;       /* USER_COARSE_ITERS (10) */
  int32_t r_out_release_step; /* USER_R_OUT_RELEASE_STEP; < 0: never */
  int32_t full_self;          /* USER_FULL_SELF */
  int32_t reserved0;
  double screen;              /* USER_SCREEN, box edge in bohr (15) */
  double kinetic_coeff;       /* USER_KINETIC_COEFF (0.5) */
  double kc_multi;            /* USER_KC_MULTI (1) */
  double beta_pauli;          /* USER_BETA_PAULI (0) */
  double field_x;             /* USER_FIELD_X (0) */
  double alpha_tf;            /* USER_ALPHA_TF (0) */
  double line_j_offset;       /* USER_LINE_J_OFFSET (0) */
  int32_t reserved[8];
} rq_mf_config;
typedef struct rq_mf_nucleus {  /* one entry of USER_NUCLEI plus its USER_NORM_TARGETS value */
  double i, j, k;               /* grid coordinates */
  double Z, rc, r_out, tilt_y, tilt_x, hs;
  double z_init;                /* initial decay rate (the page's default: Z > 0 ? Z : 1) */
  double norm_target;           /* occupation (1) */
  double split_axis[3];         /* raw axis, normalised by the library */
  int32_t split;                /* 0 sphere, 2 hemi, 3 third, 4 tetra, 5 hemi_third */
  int32_t split_idx;
  int32_t split_fix;            /* 1: enforce the split every step */
  int32_t reserved;
} rq_mf_nucleus;
/* the initial state of uploadInitialData (mol_fast.js:941-1046) is built at creation */
RQ_API int rq_mf_create(const rq_mf_config* cfg, const rq_mf_nucleus* nuclei, int32_t n, rq_mf** out);
RQ_API void rq_mf_destroy(rq_mf* s);
RQ_API const char* rq_mf_last_error(const rq_mf* s);
/* doSteps(n) (mol_fast.js:1237-1322) without its host epilogue: the f32 sums of the frame's last
 * reduction into sums (n_electrons + 6 or NULL: norm^2 per electron, T, V_eK, V_ee, dipole x,y,z).
 * Synchronises. */
RQ_API int rq_mf_step(rq_mf* s, int32_t n, float* sums);
/* the force shader (mol_fast.js:500-563): 2 Z <grad sum_m P_m> per nucleus into F (3n, f32). */
RQ_API int rq_mf_forces(rq_mf* s, float* F);
/* moved nuclei (stepNuclei, mol_fast.js:1375-1410): grid positions (3n doubles), the f32 copy in
 * the parameters and K rebuilt on the device (recomputeK_WGSL, :565-587). */
RQ_API int rq_mf_set_positions(rq_mf* s, const double* ijk);
/* the slice of extractWGSL (mol_fast.js:595-640) as a headless buffer of 3 n S^2 floats. */
RQ_API int rq_mf_extract(rq_mf* s, float* out);
/* fields of electron m (S^3 each, NULL = skip); an upload writes both buffer sets, as
 * uploadInitialData (:1039-1044) does, so the next frame reads the uploaded boundary too */
RQ_API int rq_mf_download(rq_mf* s, int32_t m, float* U, float* W, float* P);
RQ_API int rq_mf_upload(rq_mf* s, int32_t m, const float* U, const float* W, const float* P);
RQ_API int rq_mf_download_K(rq_mf* s, float* K);
RQ_API int rq_mf_info(const rq_mf* s, int64_t* kernel_launches, int64_t* steps_done);

/* ---- realqm_rb.js red-black multi-field solver (realqm_rb.js:1-1222) -------------------------
 * Replaces realqm_rb.js's GPU state, doSteps(), computeEnergy() and extractSlice(): one U, W, P
 * field per electron (each nucleus carries `ne` electrons, 2..16 in all), updated in place by
 * red-black colouring -- per step rho_total and each electron's competitor, then the red and
 * the black passes (front and amplitude, then the potential) -- and normalised with the
 * reference's f32 grid-stride reduction whenever the frame-local step index is a multiple of 5.
 * The f32 arithmetic follows the shaders' operation order (no contraction). */
typedef struct rq_rb rq_rb;
typedef struct rq_rb_config {
  int32_t NN;       /* USER_NN (100) */
  int32_t reserved0;
  double screen;    /* USER_SCREEN, box edge in bohr (8) */
  int32_t reserved[8];
} rq_rb_config;
typedef struct rq_rb_nucleus {  /* one entry of USER_NUCLEI */
  double i, j, k;               /* grid coordinates */
  double Z, rc;                 /* rc > 0: the initial front is cut at rc bohr */
  double rc_excl;               /* > 0: u and w held at 0 within rc_excl bohr of the nucleus */
  int32_t ne;                   /* electrons of this nucleus (ne = 2: the left / right half split) */
  int32_t reserved;
} rq_rb_nucleus;
/* norm_targets: one occupation per electron (USER_NORM_TARGETS) or NULL (the nucleus' ne).
 * The initial state (runInitKernels and the r_c masks, :720-801, :519-544, :615-644) is built
 * at creation. */
RQ_API int rq_rb_create(const rq_rb_config* cfg, const rq_rb_nucleus* nuclei, int32_t n_nuclei,
                        const double* norm_targets, rq_rb** out);
RQ_API void rq_rb_destroy(rq_rb* s);
RQ_API const char* rq_rb_last_error(const rq_rb* s);
/* doSteps(n) (:891-965).  Synchronises. */
RQ_API int rq_rb_step(rq_rb* s, int32_t n);
/* computeEnergy (:982-1045) summed in FP64: out = {E_T, E_eK, E_ee} (without V_KK). */
RQ_API int rq_rb_energy(rq_rb* s, double* out);
/* extractSlice (:1047-1066) as a headless buffer of S*S*(3n+1) floats. */
RQ_API int rq_rb_slice(rq_rb* s, float* out);
RQ_API int rq_rb_download(rq_rb* s, int32_t m, float* U, float* W, float* P);
RQ_API int rq_rb_upload(rq_rb* s, int32_t m, const float* U, const float* W, const float* P);
RQ_API int rq_rb_download_K(rq_rb* s, float* K);
RQ_API int rq_rb_info(const rq_rb* s, int64_t* kernel_launches, int64_t* steps_done);

/* ---- single kernels on caller-owned device memory (zero-copy PyTorch interop) ---------------
 * Pointers are device pointers of S^3 elements; `stream` is a cudaStream_t or NULL.  These run
 * exactly the kernels rq_step uses and exist for kernel-level parity checks and custom drivers. */
/* cloud/solver.py:61-90 updateU (S^3 interior update, boundary written 0). */
RQ_API int rq_kernel_update_sp(const float* U, float* Unew, const float* K, const float* P, const int32_t* label,
                        int32_t S, float half_dv, float dtv, void* stream);
/* cloud/solver.py:181-208 computeRho + jacobiStep fused: Pnew = (sum P + coeff*U^2*h2)/6. */
RQ_API int rq_kernel_jacobi_sp(const float* P, float* Pnew, const float* U, int32_t S, float h2, float coeff, void* stream);
/* cloud/solver.py:92-147 boundaryEvolve with snapshot semantics (read labelIn, write labelOut). */
RQ_API int rq_kernel_labels_sp(const int32_t* labelIn, int32_t* labelOut, const float* atoms5, int32_t n_atoms,
                        int32_t S, float h, float h2, void* stream);
/* cloud/solver.py:16-59 initTrial (U, label, K, bestU). */
RQ_API int rq_kernel_init_sp(float* U, int32_t* label, float* K, float* bestU, const float* atoms5, int32_t n_atoms,
                      int32_t S, float h, float h2, void* stream);
/* cloud/solver.py:149-179 recomputeK. */
RQ_API int rq_kernel_recompute_k_sp(float* K, const float* atoms5, int32_t n_atoms, int32_t S, float h, float h2,
                             void* stream);
/* FP64 per-label sums of psi^2*h3 (label clipped to [0,n) like cloud/solver.py:427), then
 * normalizeU (:210-225) with scale sqrt(Z/n).  norms_out (n doubles, device) may be NULL.
 * Synchronises the stream; RQ_ENONFINITE when a domain's norm is NaN/Inf as an f32 (that
 * domain is left unscaled). */
RQ_API int rq_kernel_normalize_sp(float* U, const int32_t* label, const float* Zeff, int32_t n_atoms, int32_t S, float h3,
                           double* norms_out, void* stream);
/* No counterpart in the reference.  The same normalisation as rq_kernel_normalize_sp, for
 * callers that cannot allocate device memory (for example a host framework whose own caching
 * allocator owns the GPU memory, or a solver loop that must not allocate once it runs): its
 * scratch -- the per-domain FP64 sums, the scale table and an error word -- lives in one fixed
 * device array inside the library, so the call allocates and frees nothing.
 * Limit: n_atoms <= RQ_NOALLOC_MAX_DOMAINS, otherwise RQ_EINVAL and nothing runs.
 * The array is shared by every call on a device and keeps the last call's contents (each call
 * clears what it sums into first); calls that overlap on the GPU race on it, so order them on
 * one stream.  The first call in each CUDA context looks up the array's device address (cached
 * per context: a context created again after cudaDeviceReset, or a non-primary context the
 * caller made current, gets its own look-up); make it before starting any stream capture in
 * that context.  The per-domain sums are not returned.  Like rq_kernel_normalize_sp it
 * synchronises the stream and returns RQ_ENONFINITE for a NaN/Inf domain norm. */
#define RQ_NOALLOC_MAX_DOMAINS 16384
RQ_API int rq_kernel_normalize_sp_noalloc(float* U, const int32_t* label, const float* Zeff, int32_t n_atoms, int32_t S,
                                          float h3, void* stream);
/* Per-label FP64 (norm, T, V_eK, V_ee) of cloud/solver.py:246-256 into per_domain (n x 4, device). */
RQ_API int rq_kernel_energy_sp(const float* U, const float* K, const float* P, const int32_t* label, int32_t n_atoms,
                        int32_t S, float h, float h3, double* per_domain, void* stream);
/* cloud/solver.py:282-315 computeForceAll with FP64 accumulation into F (n x 3, device). */
RQ_API int rq_kernel_forces_hf_sp(const float* U, const float* atoms5, int32_t n_atoms, int32_t S, float h, float h2,
                           float h3, double* F, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* RQ_H */
