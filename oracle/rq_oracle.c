/*
 * rq_oracle.c -- CPU restatement of the RealQM solver step (TEST INFRASTRUCTURE).
 *
 * This file is the oracle: tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg call it to check or time the CUDA product.  The product path
 * (realmolecule_b200/) never links or calls it.
 *
 * Three flavours are restated, each function citing the reference lines it follows:
 *   sp_*  cloud/solver.py   (CUDA-C strings compiled by CuPy/NVRTC)
 *   mj_*  molecule.js       (WGSL compute shaders)
 *   nm_*  the FP64 "new method" (Gaussian nuclei, red-black multigrid), which has no
 *         reference counterpart; its parity is "FP64 oracle of the same method".
 *
 * Arithmetic rules: f32 functions use plain IEEE single operations in the order the
 * reference writes them (built with -ffp-contract=off, no fast-math), so integer
 * and label results are bit-exact and field updates are bit-exact whenever the
 * CUDA kernel uses the same non-contracted order.  Reductions are FP64 with a
 * fixed per-plane order so that results do not depend on the thread count.
 *
 * Grid convention (both references): S = NN+1 points per axis, linear index
 * id = i*S*S + j*S + k with k fastest (cloud/solver.py:24-26, molecule.js:273-276);
 * the outer planes i,j,k in {0, NN} are Dirichlet boundary.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define IDX(i, j, k, S) ((int64_t)(i) * (S) * (S) + (int64_t)(j) * (S) + (k))

static inline int interior(int i, int j, int k, int NN) {
  return i >= 1 && i < NN && j >= 1 && j < NN && k >= 1 && k < NN;
}

/* ======================================================================
 * solver.py flavour
 * ==================================================================== */

/* cloud/solver.py:16-59 initTrial: K = sum Z/r_soft, trial u = Z^2/sqrt(pi) e^{-Zr},
 * label = argmax (first wins ties).  atoms5 = [i,j,k,Z,rc] floats per atom. */
void orc_sp_init_trial(float* U, int32_t* label, float* K, float* bestU, const float* atoms5,
                       int nAtoms, int S, float h, float h2) {
  const int NN = S - 1;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < S; ++i)
    for (int j = 0; j < S; ++j)
      for (int k = 0; k < S; ++k) {
        int64_t id = IDX(i, j, k, S);
        if (!interior(i, j, k, NN)) { U[id] = 0.f; label[id] = 0; K[id] = 0.f; bestU[id] = 0.f; continue; }
        float xi = (float)i * h, yj = (float)j * h, zk = (float)k * h;
        float bU = 0.f, Kval = 0.f;
        int bestN = 0;
        const float inv_sqrt_pi = 0.5641895835f;
        for (int n = 0; n < nAtoms; ++n) {
          float Za = atoms5[n * 5 + 3];
          if (Za <= 0.f) continue;
          float rc = atoms5[n * 5 + 4];
          float dx = xi - atoms5[n * 5 + 0] * h;
          float dy = yj - atoms5[n * 5 + 1] * h;
          float dz = zk - atoms5[n * 5 + 2] * h;
          float r2 = dx * dx + dy * dy + dz * dz;
          float r = (rc > 0.f) ? fmaxf(sqrtf(r2 + 0.04f * h2), rc) : sqrtf(r2 + h2);
          Kval += Za / r;
          float uT = Za * Za * inv_sqrt_pi * expf(-Za * r);
          if (uT > bU) { bU = uT; bestN = n; }
        }
        K[id] = Kval; bestU[id] = bU; label[id] = bestN; U[id] = bU;
      }
}

/* cloud/solver.py:149-179 recomputeK (same K as initTrial, no trial/labels). */
void orc_sp_recompute_K(float* K, const float* atoms5, int nAtoms, int S, float h, float h2) {
  const int NN = S - 1;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < S; ++i)
    for (int j = 0; j < S; ++j)
      for (int k = 0; k < S; ++k) {
        int64_t id = IDX(i, j, k, S);
        if (!interior(i, j, k, NN)) { K[id] = 0.f; continue; }
        float xi = (float)i * h, yj = (float)j * h, zk = (float)k * h, Kval = 0.f;
        for (int n = 0; n < nAtoms; ++n) {
          float Za = atoms5[n * 5 + 3];
          if (Za <= 0.f) continue;
          float rc = atoms5[n * 5 + 4];
          float dx = xi - atoms5[n * 5 + 0] * h;
          float dy = yj - atoms5[n * 5 + 1] * h;
          float dz = zk - atoms5[n * 5 + 2] * h;
          float r2 = dx * dx + dy * dy + dz * dz;
          float r = (rc > 0.f) ? fmaxf(sqrtf(r2 + 0.04f * h2), rc) : sqrtf(r2 + h2);
          Kval += Za / r;
        }
        K[id] = Kval;
      }
}

/* cloud/solver.py:61-90 updateU: same-label Neumann 7-point Laplacian, then
 * Unew = u + half_dv*lap + dtv*(K - 2P)*u; boundary planes written 0. */
void orc_sp_update(const float* U, float* Unew, const float* K, const float* P, const int32_t* label,
                   int S, float half_dv, float dtv) {
  const int NN = S - 1;
  const int64_t S2 = (int64_t)S * S;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < S; ++i)
    for (int j = 0; j < S; ++j)
      for (int k = 0; k < S; ++k) {
        int64_t id = IDX(i, j, k, S);
        if (!interior(i, j, k, NN)) { Unew[id] = 0.f; continue; }
        int32_t L = label[id];
        float u = U[id];
        float uip = (label[id + S2] == L) ? U[id + S2] : u;
        float uim = (label[id - S2] == L) ? U[id - S2] : u;
        float ujp = (label[id + S] == L) ? U[id + S] : u;
        float ujm = (label[id - S] == L) ? U[id - S] : u;
        float ukp = (label[id + 1] == L) ? U[id + 1] : u;
        float ukm = (label[id - 1] == L) ? U[id - 1] : u;
        float lap = uip + uim + ujp + ujm + ukp + ukm - 6.0f * u;
        Unew[id] = u + half_dv * lap + dtv * (K[id] - 2.0f * P[id]) * u;
      }
}

/* cloud/solver.py:92-147 boundaryEvolve decision for one interior cell, reading
 * labels from `lab`.  Returns the new label (== current label when no flip). */
static inline int32_t sp_boundary_cell(const int32_t* lab, const float* atoms5, int nAtoms, int S,
                                       int i, int j, int k, float h, float h2) {
  const int64_t S2 = (int64_t)S * S;
  int64_t id = IDX(i, j, k, S);
  float xi = (float)i * h, yj = (float)j * h, zk = (float)k * h;
  int32_t cur = lab[id];
  int otherCount = 0;
  const int64_t nb[6] = {id + S2, id - S2, id + S, id - S, id + 1, id - 1};
  for (int n = 0; n < 6; ++n)
    if (lab[nb[n]] != cur) otherCount++;
  if (otherCount == 0) return cur;
  float curScore = 0.f, bestScore = 0.f;
  int32_t bestN = cur;
  for (int n = 0; n < nAtoms; ++n) {
    float Za = atoms5[n * 5 + 3];
    if (Za <= 0.f) continue;
    float dx = xi - atoms5[n * 5 + 0] * h;
    float dy = yj - atoms5[n * 5 + 1] * h;
    float dz = zk - atoms5[n * 5 + 2] * h;
    float r2 = dx * dx + dy * dy + dz * dz + h2;
    float score = Za / sqrtf(r2);
    if (n == cur) curScore = score;
    if (score > bestScore) { bestScore = score; bestN = n; }
  }
  if (bestN != cur && bestScore > curScore * 1.1f && otherCount >= 2) return bestN;
  return cur;
}

/* Snapshot semantics (read labelIn, write labelOut): the deterministic form of
 * cloud/solver.py:92-147, whose in-place write (:143-145) races on a GPU. */
void orc_sp_boundary_snapshot(const int32_t* labelIn, int32_t* labelOut, const float* atoms5, int nAtoms,
                              int S, float h, float h2) {
  const int NN = S - 1;
  const int64_t S3 = (int64_t)S * S * S;
  memcpy(labelOut, labelIn, (size_t)S3 * sizeof(int32_t));
#pragma omp parallel for schedule(static)
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k)
        labelOut[IDX(i, j, k, S)] = sp_boundary_cell(labelIn, atoms5, nAtoms, S, i, j, k, h, h2);
}

/* In-place, lexicographic order: what the reference kernel produces when its
 * threads run one after another in index order.  Used only to pin the decision
 * rule against the reference kernel run serially on the host. */
void orc_sp_boundary_inplace_lex(int32_t* label, const float* atoms5, int nAtoms, int S, float h, float h2) {
  const int NN = S - 1;
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k)
        label[IDX(i, j, k, S)] = sp_boundary_cell(label, atoms5, nAtoms, S, i, j, k, h, h2);
}

/* cloud/solver.py:181-208 computeRho + jacobiStep: Pnew = (sum_6 P + coeff*rho*h2)/6. */
void orc_sp_jacobi(const float* P, float* Pnew, const float* U, int S, float h2, float coeff) {
  const int NN = S - 1;
  const int64_t S2 = (int64_t)S * S;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < S; ++i)
    for (int j = 0; j < S; ++j)
      for (int k = 0; k < S; ++k) {
        int64_t id = IDX(i, j, k, S);
        if (!interior(i, j, k, NN)) { Pnew[id] = 0.f; continue; }
        float rho = U[id] * U[id];
        float sumN = P[id + S2] + P[id - S2] + P[id + S] + P[id - S] + P[id + 1] + P[id - 1];
        Pnew[id] = (sumN + coeff * rho * h2) / 6.0f;
      }
}

/* cloud/solver.py:421-427 norms as numpy/cupyx computes them on the host:
 * rho = U*U*h3 in f32, scatter_add in index order into f32 (np.add.at). */
void orc_sp_norms_f32_seq(const float* U, const int32_t* label, int64_t S3, int nAtoms, float h3, float* norms) {
  for (int n = 0; n < nAtoms; ++n) norms[n] = 0.f;
  for (int64_t id = 0; id < S3; ++id) {
    int32_t l = label[id];
    if (l < 0) l = 0;
    if (l > nAtoms - 1) l = nAtoms - 1;
    norms[l] += (U[id] * U[id]) * h3;
  }
}

/* Per-label FP64 sums of psi^2 h^3 over ALL points (the reference sums the whole
 * array; boundary points are zero), with the label clipped like :427. */
void orc_sp_norms_f64(const float* U, const int32_t* label, int S, int nAtoms, double h3, double* norms) {
  const int64_t S2 = (int64_t)S * S;
  double* part = (double*)calloc((size_t)S * nAtoms, sizeof(double));
#pragma omp parallel for schedule(static)
  for (int i = 0; i < S; ++i) {
    double* pp = part + (size_t)i * nAtoms;
    for (int64_t q = 0; q < S2; ++q) {
      int64_t id = i * S2 + q;
      int32_t l = label[id];
      if (l < 0) l = 0;
      if (l > nAtoms - 1) l = nAtoms - 1;
      double u = (double)U[id];
      pp[l] += u * u * h3;
    }
  }
  for (int n = 0; n < nAtoms; ++n) norms[n] = 0.0;
  for (int i = 0; i < S; ++i)
    for (int n = 0; n < nAtoms; ++n) norms[n] += part[(size_t)i * nAtoms + n];
  free(part);
}

/* cloud/solver.py:210-225 normalizeU: U *= sqrt(Z/n) for labels in range with Z>0, n>1e-20. */
void orc_sp_normalize(float* U, const int32_t* label, const float* norms, const float* Zeff, int64_t S3, int nAtoms) {
#pragma omp parallel for schedule(static)
  for (int64_t id = 0; id < S3; ++id) {
    int32_t l = label[id];
    if (l < 0 || l >= nAtoms) continue;
    float z = Zeff[l];
    if (z <= 0.f) continue;
    float n = norms[l];
    if (n > 1e-20f) U[id] *= sqrtf(z / n);
  }
}

/* cloud/solver.py:227-280 computeEnergy, restated: per thread T/VeK/Vee terms in f32,
 * a shared-memory tree per block of `block` threads, then block partials added in
 * block order (the reference adds them with float atomics in arbitrary order). */
void orc_sp_energy_blocktree(const float* U, const float* K, const float* P, const int32_t* label, float* out,
                             int S, float h, float h3, int block) {
  const int NN = S - 1;
  const int64_t S2 = (int64_t)S * S, S3 = S2 * S;
  const int64_t nblk = (S3 + block - 1) / block;
  float* bp = (float*)malloc(sizeof(float) * 3 * (size_t)nblk);
#pragma omp parallel
  {
    float* sd = (float*)malloc(sizeof(float) * 3 * (size_t)block);
#pragma omp for schedule(static)
    for (int64_t b = 0; b < nblk; ++b) {
      for (int t = 0; t < block; ++t) {
        int64_t id = b * block + t;
        float lT = 0.f, lK = 0.f, lE = 0.f;
        if (id < S3) {
          int i = (int)(id / S2), j = (int)((id / S) % S), k = (int)(id % S);
          if (interior(i, j, k, NN)) {
            float u = U[id], rho = u * u;
            int32_t L = label[id];
            float dui = (label[id + S2] == L) ? U[id + S2] - u : 0.f;
            float duj = (label[id + S] == L) ? U[id + S] - u : 0.f;
            float duk = (label[id + 1] == L) ? U[id + 1] - u : 0.f;
            lT = 0.5f * (dui * dui + duj * duj + duk * duk) * h;
            lK = -K[id] * rho * h3;
            lE = P[id] * rho * h3;
          }
        }
        sd[t] = lT; sd[t + block] = lK; sd[t + 2 * block] = lE;
      }
      for (int s = block / 2; s > 0; s >>= 1)
        for (int t = 0; t < s; ++t) {
          sd[t] += sd[t + s]; sd[t + block] += sd[t + block + s]; sd[t + 2 * block] += sd[t + 2 * block + s];
        }
      bp[3 * b] = sd[0]; bp[3 * b + 1] = sd[block]; bp[3 * b + 2] = sd[2 * block];
    }
    free(sd);
  }
  out[0] = out[1] = out[2] = 0.f;
  for (int64_t b = 0; b < nblk; ++b) { out[0] += bp[3 * b]; out[1] += bp[3 * b + 1]; out[2] += bp[3 * b + 2]; }
  free(bp);
}

/* Same energy terms (cloud/solver.py:246-256) accumulated in FP64, total and per
 * label: out[0..2] = T, V_eK, V_ee; per_domain (nDom x 4, may be NULL) = norm, T,
 * V_eK, V_ee of each label (labels outside [0,nDom) are skipped there). */
void orc_sp_energy_f64(const float* U, const float* K, const float* P, const int32_t* label, int S, double h,
                       double h3, double* out, int nDom, double* per_domain) {
  const int NN = S - 1;
  const int64_t S2 = (int64_t)S * S;
  double* part = (double*)calloc((size_t)S * 3, sizeof(double));
  double* pd = per_domain ? (double*)calloc((size_t)S * nDom * 4, sizeof(double)) : NULL;
#pragma omp parallel for schedule(static)
  for (int i = 1; i < NN; ++i) {
    double t = 0, vk = 0, ve = 0;
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        int64_t id = IDX(i, j, k, S);
        double u = U[id], rho = u * u;
        int32_t L = label[id];
        double dui = (label[id + S2] == L) ? (double)U[id + S2] - u : 0.0;
        double duj = (label[id + S] == L) ? (double)U[id + S] - u : 0.0;
        double duk = (label[id + 1] == L) ? (double)U[id + 1] - u : 0.0;
        double lt = 0.5 * (dui * dui + duj * duj + duk * duk) * h;
        double lk = -(double)K[id] * rho * h3, le = (double)P[id] * rho * h3;
        t += lt; vk += lk; ve += le;
        if (pd && L >= 0 && L < nDom) {
          double* q = pd + ((size_t)i * nDom + L) * 4;
          q[0] += rho * h3; q[1] += lt; q[2] += lk; q[3] += le;
        }
      }
    part[3 * i] = t; part[3 * i + 1] = vk; part[3 * i + 2] = ve;
  }
  out[0] = out[1] = out[2] = 0;
  for (int i = 0; i < S; ++i) { out[0] += part[3 * i]; out[1] += part[3 * i + 1]; out[2] += part[3 * i + 2]; }
  if (pd) {
    memset(per_domain, 0, sizeof(double) * nDom * 4);
    for (int i = 0; i < S; ++i)
      for (int q = 0; q < nDom * 4; ++q) per_domain[q] += pd[(size_t)i * nDom * 4 + q];
    free(pd);
  }
  free(part);
}

/* cloud/solver.py:282-315 computeForceAll (Hellmann-Feynman), FP64 accumulation:
 * F_n += Z_n rho h^3 (x - R_n) / (|x-R_n|^2 + h^2)^{3/2} over interior points with rho >= 1e-20.
 * Per-voxel terms are evaluated in f32 as the reference does. */
void orc_sp_forces(const float* U, const float* atoms5, int nAtoms, int S, float h, float h2, float h3, double* F) {
  const int NN = S - 1;
  double* part = (double*)calloc((size_t)S * nAtoms * 3, sizeof(double));
#pragma omp parallel for schedule(static)
  for (int i = 1; i < NN; ++i) {
    double* pp = part + (size_t)i * nAtoms * 3;
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        int64_t id = IDX(i, j, k, S);
        float rho = U[id] * U[id];
        if (rho < 1e-20f) continue;
        float xi = (float)i * h, yj = (float)j * h, zk = (float)k * h;
        for (int n = 0; n < nAtoms; ++n) {
          float Za = atoms5[n * 5 + 3];
          if (Za <= 0.f) continue;
          float dx = xi - atoms5[n * 5 + 0] * h;
          float dy = yj - atoms5[n * 5 + 1] * h;
          float dz = zk - atoms5[n * 5 + 2] * h;
          float r2 = dx * dx + dy * dy + dz * dz + h2;
          float inv_r3 = 1.0f / (r2 * sqrtf(r2));
          float w = Za * rho * inv_r3 * h3;
          pp[n * 3 + 0] += (double)(w * dx);
          pp[n * 3 + 1] += (double)(w * dy);
          pp[n * 3 + 2] += (double)(w * dz);
        }
      }
  }
  memset(F, 0, sizeof(double) * nAtoms * 3);
  for (int i = 0; i < S; ++i)
    for (int q = 0; q < nAtoms * 3; ++q) F[q] += part[(size_t)i * nAtoms * 3 + q];
  free(part);
}

/* ======================================================================
 * molecule.js flavour
 * ==================================================================== */

/* Atom record as molecule.js packs it (molecule.js:183-191, :1875-1903): positions are
 * stored in a Uint32Array, so fractional grid positions are truncated. */
typedef struct {
  uint32_t posI, posJ, posK;
  float Z, rc, Z_nuc, initZeff, initRcut;
} orc_mj_atom;

static inline float mj_dist(int ci, int cj, int ck, const orc_mj_atom* a, float h) {
  float dx = ((float)ci - (float)a->posI) * h;
  float dy = ((float)cj - (float)a->posJ) * h;
  float dz = ((float)ck - (float)a->posK) * h;
  return sqrtf(dx * dx + dy * dy + dz * dz);
}

/* Shell split of an entry (window.USER_SPLIT_TYPE/_IDX/_AXIS/_ROT, molecule.js:27-32, the atom
 * record's split fields :183-191): type 0/1 = whole sphere, 2 = half space, 3 = 120-degree sector. */
typedef struct {
  uint32_t type, idx;
  float ax, ay, az, rot;
} orc_mj_split;

/* inSplitAtom (molecule.js:197-226); d = cell - nucleus in bohr, r = |d|.  atan2 is the f64
 * function rounded once to f32 (WGSL leaves its accuracy to the implementation). */
static int mj_in_split(float dx, float dy, float dz, float r, const orc_mj_split* s) {
  if (s->type <= 1u || r < 1e-6f) return 1;
  const float axL = fmaxf(sqrtf(s->ax * s->ax + s->ay * s->ay + s->az * s->az), 1e-12f);
  const float a0 = s->ax / axL, a1 = s->ay / axL, a2 = s->az / axL;
  const float dotp = dx * a0 + dy * a1 + dz * a2;
  if (s->type == 2u) return s->idx == 0u ? dotp < 0.f : dotp >= 0.f;
  if (s->type == 3u) {
    const float px = dx - dotp * a0, py = dy - dotp * a1, pz = dz - dotp * a2;
    float e1x, e1y, e1z;
    if (fabsf(a2) < 0.9f) { e1x = a1; e1y = -a0; e1z = 0.f; } else { e1x = 0.f; e1y = a2; e1z = -a1; }
    const float e1L = fmaxf(sqrtf(e1x * e1x + e1y * e1y + e1z * e1z), 1e-12f);
    e1x = e1x / e1L; e1y = e1y / e1L; e1z = e1z / e1L;
    const float e2x = a1 * e1z - a2 * e1y, e2y = a2 * e1x - a0 * e1z, e2z = a0 * e1y - a1 * e1x;
    const float pe1 = px * e1x + py * e1y + pz * e1z, pe2 = px * e2x + py * e2y + pz * e2z;
    float th = (float)atan2((double)pe2, (double)pe1) - s->rot;
    if (th < -3.14159265f) th = th + 6.28318530f;
    if (th > 3.14159265f) th = th - 6.28318530f;
    const uint32_t sector = ((uint32_t)floorf((th + 3.14159265f) / 2.09439510f)) % 3u;
    return sector == s->idx;
  }
  return 1;
}

/* evolveBoundary's cellSectorOK (molecule.js:437-442): d = (cell - nucleus) * h. */
static int mj_sector_ok(int i, int j, int k, uint32_t n, const orc_mj_atom* atoms, const orc_mj_split* splits, float h) {
  if (!splits || splits[n].type <= 1u) return 1;
  const float dx = ((float)i - (float)atoms[n].posI) * h;
  const float dy = ((float)j - (float)atoms[n].posJ) * h;
  const float dz = ((float)k - (float)atoms[n].posK) * h;
  return mj_in_split(dx, dy, dz, sqrtf(dx * dx + dy * dy + dz * dz), &splits[n]);
}

/* molecule.js:246-259 isInsideRc (own r_c sphere; bare nuclei when present). */
static inline int mj_inside_rc(int ci, int cj, int ck, uint32_t lbl, const orc_mj_atom* atoms, int nElec,
                               int hasBare, float h) {
  float rc = atoms[lbl].rc;
  if (rc > 0.f && mj_dist(ci, cj, ck, &atoms[lbl], h) < rc) return 1;
  if (hasBare)
    for (int n = 0; n < nElec; ++n)
      if (atoms[n].Z <= 0.f && atoms[n].Z_nuc > 0.f && atoms[n].rc > 0.f)
        if (mj_dist(ci, cj, ck, &atoms[n], h) < atoms[n].rc) return 1;
  return 0;
}

/* molecule.js:263-343 updateU with W_CUTOFF = 0 (the default, :83): Dirichlet 0
 * inside the own r_c sphere; a neighbour of another label or inside its label's
 * r_c sphere is replaced by the centre value.  Interior cells only are written. */
void orc_mj_update(const float* U, float* Uo, const float* K, const uint32_t* label, const float* Pother,
                   const orc_mj_atom* atoms, int nElec, int hasBare, int S, float h, float half_d, float dt) {
  const int NN = S - 1;
  const int64_t S2 = (int64_t)S * S;
#pragma omp parallel for schedule(static)
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        int64_t id = IDX(i, j, k, S);
        uint32_t L = label[id];
        if (mj_inside_rc(i, j, k, L, atoms, nElec, hasBare, h)) { Uo[id] = 0.f; continue; }
        float uc = U[id];
        uint32_t lip = label[id + S2], lim = label[id - S2], ljp = label[id + S], ljm = label[id - S];
        uint32_t lkp = label[id + 1], lkm = label[id - 1];
        int eip = mj_inside_rc(i + 1, j, k, lip, atoms, nElec, hasBare, h);
        int eim = mj_inside_rc(i - 1, j, k, lim, atoms, nElec, hasBare, h);
        int ejp = mj_inside_rc(i, j + 1, k, ljp, atoms, nElec, hasBare, h);
        int ejm = mj_inside_rc(i, j - 1, k, ljm, atoms, nElec, hasBare, h);
        int ekp = mj_inside_rc(i, j, k + 1, lkp, atoms, nElec, hasBare, h);
        int ekm = mj_inside_rc(i, j, k - 1, lkm, atoms, nElec, hasBare, h);
        float uip = (lip == L && !eip) ? U[id + S2] : uc;
        float uim = (lim == L && !eim) ? U[id - S2] : uc;
        float ujp = (ljp == L && !ejp) ? U[id + S] : uc;
        float ujm = (ljm == L && !ejm) ? U[id - S] : uc;
        float ukp = (lkp == L && !ekp) ? U[id + 1] : uc;
        float ukm = (lkm == L && !ekm) ? U[id - 1] : uc;
        float lap = uip + uim + ujp + ujm + ukp + ukm - 6.0f * uc;
        Uo[id] = uc + half_d * lap + dt * (K[id] - 2.0f * Pother[id]) * uc;
      }
}

/* molecule.js:426-540 evolveBoundary without locked groups or shell splits
 * (both off unless a page sets them, :490-503): snapshot read labelIn, write labelOut and W. */
/* chebyshevStepWGSL (molecule.js:345-421): the ITP step of orc_mj_update blended with psi_{n-1},
 * which Uo holds on entry: Uo = omega * step + (1 - omega) * Uo; cells inside their own r_c are 0.
 * (The shader tests only the own label's r_c sphere, as orc_mj_update does without bare nuclei.) */
void orc_mj_update_cheb(const float* U, float* Uo, const float* K, const uint32_t* label, const float* Pother,
                        const orc_mj_atom* atoms, int nElec, int S, float h, float half_d, float dt, float omega) {
  const int NN = S - 1;
  const int64_t S2 = (int64_t)S * S;
#pragma omp parallel for schedule(static)
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        int64_t id = IDX(i, j, k, S);
        uint32_t L = label[id];
        if (mj_inside_rc(i, j, k, L, atoms, nElec, 0, h)) { Uo[id] = 0.f; continue; }
        float uc = U[id];
        uint32_t lip = label[id + S2], lim = label[id - S2], ljp = label[id + S], ljm = label[id - S];
        uint32_t lkp = label[id + 1], lkm = label[id - 1];
        float uip = (lip == L && !mj_inside_rc(i + 1, j, k, lip, atoms, nElec, 0, h)) ? U[id + S2] : uc;
        float uim = (lim == L && !mj_inside_rc(i - 1, j, k, lim, atoms, nElec, 0, h)) ? U[id - S2] : uc;
        float ujp = (ljp == L && !mj_inside_rc(i, j + 1, k, ljp, atoms, nElec, 0, h)) ? U[id + S] : uc;
        float ujm = (ljm == L && !mj_inside_rc(i, j - 1, k, ljm, atoms, nElec, 0, h)) ? U[id - S] : uc;
        float ukp = (lkp == L && !mj_inside_rc(i, j, k + 1, lkp, atoms, nElec, 0, h)) ? U[id + 1] : uc;
        float ukm = (lkm == L && !mj_inside_rc(i, j, k - 1, lkm, atoms, nElec, 0, h)) ? U[id - 1] : uc;
        float lap = uip + uim + ujp + ujm + ukp + ukm - 6.0f * uc;
        float step = uc + half_d * lap + dt * (K[id] - 2.0f * Pother[id]) * uc;
        Uo[id] = omega * step + (1.0f - omega) * Uo[id];
      }
}

/* evolveBoundary (molecule.js:426-540).  Locked groups (:490-503): lock[l] has bit g set when
 * label l is in group g (lock may be NULL); a boundary cell whose label and best other label share
 * a group keeps its label with W = max(W, 0.5).  Shell splits (:514-533, splits may be NULL): a
 * flip into a domain whose sector excludes the cell is cancelled, and a cell outside its own
 * domain's sector goes to the best neighbour whose sector holds it. */
void orc_mj_evolve_boundary(const uint32_t* labelIn, uint32_t* labelOut, const float* U, float* W, int S,
                            float dt_w, float curvReg, const uint64_t* lock, const orc_mj_atom* atoms,
                            const orc_mj_split* splits, float h) {
  const int NN = S - 1;
  const int64_t S2 = (int64_t)S * S;
#pragma omp parallel for schedule(static)
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        int64_t id = IDX(i, j, k, S);
        uint32_t myL = labelIn[id];
        float myRho = U[id] * U[id];
        const int64_t nb[6] = {id + S2, id - S2, id + S, id - S, id + 1, id - 1};
        uint32_t bestL = myL;
        float bestRho = 0.f, myCnt = 0.f;
        for (int q = 0; q < 6; ++q) {
          uint32_t l = labelIn[nb[q]];
          if (l == myL) myCnt += 1.0f;
          else {
            float r = U[nb[q]] * U[nb[q]];
            if (r > bestRho) { bestRho = r; bestL = l; }
          }
        }
        float w = W[id];
        if (myCnt >= 6.0f) { w = fmaxf(w, 1.0f); W[id] = w; labelOut[id] = myL; continue; }
        if (lock && (lock[myL] & lock[bestL])) { W[id] = fmaxf(w, 0.5f); labelOut[id] = myL; continue; }
        float denom = myRho + bestRho;
        float vel = (denom < 1e-20f) ? 0.0f : (myRho - bestRho) / denom;
        w += dt_w * vel;
        float curv = (myCnt - 3.0f) / 3.0f;
        w += curvReg * curv;
        uint32_t newL = myL;
        if (w < 0.0f) { newL = bestL; w = 0.1f; }
        const int myOK = mj_sector_ok(i, j, k, myL, atoms, splits, h);
        if (!mj_sector_ok(i, j, k, newL, atoms, splits, h)) {
          newL = myL;
          w = fmaxf(w, 0.1f);
          if (!myOK && bestL != myL && mj_sector_ok(i, j, k, bestL, atoms, splits, h)) { newL = bestL; w = 0.1f; }
        } else if (!myOK && newL == myL) {
          if (bestL != myL && mj_sector_ok(i, j, k, bestL, atoms, splits, h)) { newL = bestL; w = 0.1f; }
        }
        W[id] = w;
        labelOut[id] = newL;
      }
}

/* molecule.js:723-749 weighted Jacobi: Pout = 0.3333*Pc + (sum_6 + h2*2pi*rho)/9. */
void orc_mj_jacobi(const float* Pin, float* Pout, const float* rho, int S, float h2, float two_pi) {
  const int NN = S - 1;
  const int64_t S2 = (int64_t)S * S;
#pragma omp parallel for schedule(static)
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        int64_t id = IDX(i, j, k, S);
        float Pc = Pin[id];
        float sn = Pin[id + S2] + Pin[id - S2] + Pin[id + S] + Pin[id - S] + Pin[id + 1] + Pin[id - 1];
        float rhs = h2 * two_pi * rho[id];
        Pout[id] = 0.3333f * Pc + (sn + rhs) / 9.0f;
      }
}

/* molecule.js:754-774 computeRho (interior only). */
void orc_mj_rho(const float* U, float* rho, int S) {
  const int NN = S - 1;
#pragma omp parallel for schedule(static)
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) { int64_t id = IDX(i, j, k, S); float u = U[id]; rho[id] = u * u; }
}

/* molecule.js:572-590 computeRhoSelf: rho = psi^2 where label == m, 0 elsewhere (interior only). */
void orc_mj_rho_self(const float* U, const uint32_t* label, uint32_t m, float* rho, int S) {
  const int NN = S - 1;
#pragma omp parallel for schedule(static)
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        int64_t id = IDX(i, j, k, S);
        float u = U[id];
        rho[id] = label[id] == m ? u * u : 0.0f;
      }
}

/* molecule.js:694-721 subtractPself: Pother -= Pm * frac where label == m, with frac = 1/Z_m when
   Z_m > 1 and 1 otherwise (f32). */
void orc_mj_sub_self(const float* Pm, float* Pother, const uint32_t* label, uint32_t m, float Zm, int S) {
  const int NN = S - 1;
  const float frac = Zm > 1.0f ? 1.0f / Zm : 1.0f;
#pragma omp parallel for schedule(static)
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        int64_t id = IDX(i, j, k, S);
        if (label[id] == m) Pother[id] = Pother[id] - Pm[id] * frac;
      }
}

/* molecule.js:593-612 computeRhoOther: rho = psi^2 except where label == m (interior only). */
void orc_mj_rho_other(const float* U, const uint32_t* label, uint32_t m, float* rho, int S) {
  const int NN = S - 1;
#pragma omp parallel for schedule(static)
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        int64_t id = IDX(i, j, k, S);
        float u = U[id];
        rho[id] = label[id] == m ? 0.0f : u * u;
      }
}

/* molecule.js:651-671 copyPotherForLabel: Pother = Psrc where label == m. */
void orc_mj_copy_for_label(const float* Psrc, float* Pother, const uint32_t* label, uint32_t m, int S) {
  const int NN = S - 1;
#pragma omp parallel for schedule(static)
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        int64_t id = IDX(i, j, k, S);
        if (label[id] == m) Pother[id] = Psrc[id];
      }
}

/* molecule.js:614-649 initPdirect: Pm = sum over n != m with Z_n > 0 of 0.5/sqrt(r^2 + h^2) at the
   truncated positions (f32, atoms in index order); Pother += Pm. */
void orc_mj_init_pdirect(const orc_mj_atom* atoms, int nAt, uint32_t m, float* Pm, float* Pother, int S, float h,
                         float h2) {
  const int NN = S - 1;
#pragma omp parallel for schedule(static)
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        int64_t id = IDX(i, j, k, S);
        float xi = (float)i * h, yj = (float)j * h, zk = (float)k * h, val = 0.0f;
        for (int n = 0; n < nAt; ++n) {
          if (atoms[n].Z <= 0.0f || (uint32_t)n == m) continue;
          float dx = xi - (float)atoms[n].posI * h, dy = yj - (float)atoms[n].posJ * h, dz = zk - (float)atoms[n].posK * h;
          float r = sqrtf(dx * dx + dy * dy + dz * dz + h2);
          val += 0.5f / r;
        }
        Pm[id] = val;
        Pother[id] += val;
      }
}

/* molecule.js:777-803 residual r = -2pi*rho - lap(P)/h^2 (sign as written). */
void orc_mj_residual(const float* Pin, float* R, const float* rho, int S, float inv_h2, float two_pi) {
  const int NN = S - 1;
  const int64_t S2 = (int64_t)S * S;
#pragma omp parallel for schedule(static)
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        int64_t id = IDX(i, j, k, S);
        float Pc = Pin[id];
        float lap = (Pin[id + S2] + Pin[id - S2] + Pin[id + S] + Pin[id - S] + Pin[id + 1] + Pin[id - 1] - 6.0f * Pc) *
                    inv_h2;
        R[id] = -two_pi * rho[id] - lap;
      }
}

/* molecule.js:806-839 27-point full weighting (8/4/2/1)/64 onto SC = NN/2+1. */
void orc_mj_restrict(const float* fine, float* coarse, int S, int SC) {
  const int NC = SC - 1;
  const int64_t S2 = (int64_t)S * S;
#pragma omp parallel for schedule(static)
  for (int I = 1; I < NC; ++I)
    for (int J = 1; J < NC; ++J)
      for (int K2 = 1; K2 < NC; ++K2) {
        int fi = 2 * I, fj = 2 * J, fk = 2 * K2;
#define F(a, b, c) fine[(int64_t)(a) * S2 + (int64_t)(b) * S + (c)]
        float val = 8.0f * F(fi, fj, fk);
        val += 4.0f * (F(fi + 1, fj, fk) + F(fi - 1, fj, fk) + F(fi, fj + 1, fk) + F(fi, fj - 1, fk) +
                       F(fi, fj, fk + 1) + F(fi, fj, fk - 1));
        val += 2.0f * (F(fi + 1, fj + 1, fk) + F(fi + 1, fj - 1, fk) + F(fi - 1, fj + 1, fk) + F(fi - 1, fj - 1, fk) +
                       F(fi + 1, fj, fk + 1) + F(fi + 1, fj, fk - 1) + F(fi - 1, fj, fk + 1) + F(fi - 1, fj, fk - 1) +
                       F(fi, fj + 1, fk + 1) + F(fi, fj + 1, fk - 1) + F(fi, fj - 1, fk + 1) + F(fi, fj - 1, fk - 1));
        val += F(fi + 1, fj + 1, fk + 1) + F(fi + 1, fj + 1, fk - 1) + F(fi + 1, fj - 1, fk + 1) +
               F(fi + 1, fj - 1, fk - 1) + F(fi - 1, fj + 1, fk + 1) + F(fi - 1, fj + 1, fk - 1) +
               F(fi - 1, fj - 1, fk + 1) + F(fi - 1, fj - 1, fk - 1);
#undef F
        coarse[IDX(I, J, K2, SC)] = val * 0.015625f;
      }
}

/* molecule.js:842-867 coarse weighted Jacobi with hc^2 = 4 h^2. */
void orc_mj_coarse_smooth(const float* Ein, float* Eout, const float* f, int SC, float h2) {
  const int NC = SC - 1;
  const int64_t SC2 = (int64_t)SC * SC;
#pragma omp parallel for schedule(static)
  for (int I = 1; I < NC; ++I)
    for (int J = 1; J < NC; ++J)
      for (int K2 = 1; K2 < NC; ++K2) {
        int64_t c = IDX(I, J, K2, SC);
        float ec = Ein[c];
        float sn = Ein[c + SC2] + Ein[c - SC2] + Ein[c + SC] + Ein[c - SC] + Ein[c + 1] + Ein[c - 1];
        float hc2 = 4.0f * h2;
        Eout[c] = 0.3333f * ec + (sn + hc2 * f[c]) / 9.0f;
      }
}

/* molecule.js:870-909 trilinear prolongation, Pf += 0.5*corr (sign/damping as written). */
void orc_mj_prolong(const float* Ec, float* Pf, int S, int SC) {
  const int NN = S - 1, NC = SC - 1;
  const int64_t S2 = (int64_t)S * S, SC2 = (int64_t)SC * SC;
#pragma omp parallel for schedule(static)
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        int ci = i / 2, cj = j / 2, ck = k / 2;
        int ci1 = ci + (i & 1); if (ci1 > NC) ci1 = NC;
        int cj1 = cj + (j & 1); if (cj1 > NC) cj1 = NC;
        int ck1 = ck + (k & 1); if (ck1 > NC) ck1 = NC;
        float wi = (i & 1) ? 0.5f : 1.0f, wj = (j & 1) ? 0.5f : 1.0f, wk = (k & 1) ? 0.5f : 1.0f;
        float wi1 = 1.0f - wi, wj1 = 1.0f - wj, wk1 = 1.0f - wk;
#define E(a, b, c) Ec[(int64_t)(a) * SC2 + (int64_t)(b) * SC + (c)]
        float corr = 0.0f;
        corr += wi * wj * wk * E(ci, cj, ck);
        corr += wi * wj * wk1 * E(ci, cj, ck1);
        corr += wi * wj1 * wk * E(ci, cj1, ck);
        corr += wi * wj1 * wk1 * E(ci, cj1, ck1);
        corr += wi1 * wj * wk * E(ci1, cj, ck);
        corr += wi1 * wj * wk1 * E(ci1, cj, ck1);
        corr += wi1 * wj1 * wk * E(ci1, cj1, ck);
        corr += wi1 * wj1 * wk1 * E(ci1, cj1, ck1);
#undef E
        Pf[(int64_t)i * S2 + (int64_t)j * S + k] += 0.5f * corr;
      }
}

/* molecule.js:912-946 fixed-point norms: norm[l] += u32(u*u*h3*2^24) (truncation),
 * decoded as f32(sum) * 2^-24.  The u32 sum wraps modulo 2^32 like WGSL atomics. */
void orc_mj_norms_fixed(const float* U, const uint32_t* label, int S, float h3, int nDom, uint32_t* acc,
                        float* normFloat) {
  const int NN = S - 1;
  for (int n = 0; n < nDom; ++n) acc[n] = 0u;
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        int64_t id = IDX(i, j, k, S);
        float v = U[id];
        uint32_t c = (uint32_t)(v * v * h3 * 16777216.0f);
        acc[label[id]] += c;
      }
  for (int n = 0; n < nDom; ++n) normFloat[n] = (float)acc[n] * (1.0f / 16777216.0f);
}

/* molecule.js:1077-1105 normalize: U *= sqrt(Z/n) when n > 0 and Z > 0 (interior only). */
void orc_mj_normalize(float* U, const float* normFloat, const uint32_t* label, const orc_mj_atom* atoms, int S) {
  const int NN = S - 1;
#pragma omp parallel for schedule(static)
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        int64_t id = IDX(i, j, k, S);
        uint32_t l = label[id];
        float n = normFloat[l], Z = atoms[l].Z;
        if (n > 0.f && Z > 0.f) U[id] *= sqrtf(Z / n);
      }
}

/* molecule.js:950-1075 reduceEnergy terms accumulated in FP64 (the reference sums in f32):
 * out = {T, V_eK, V_ee, dipX, dipY, dipZ}; exclusion sphere radius max(rc, R_SING). */
void orc_mj_energy(const float* U, const float* Pv, const float* K, const uint32_t* label, const orc_mj_atom* atoms,
                   int S, float h, float h3, float Rsing, double* out) {
  const int NN = S - 1;
  const int64_t S2 = (int64_t)S * S;
  double* part = (double*)calloc((size_t)S * 6, sizeof(double));
#pragma omp parallel for schedule(static)
  for (int i = 1; i < NN; ++i) {
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        int64_t id = IDX(i, j, k, S);
        float v = U[id], rho = v * v;
        uint32_t L = label[id];
        const orc_mj_atom* a = &atoms[L];
        float rcx = fmaxf(a->rc, Rsing);
#define EXCL(ci, cj, ck) (mj_dist((ci), (cj), (ck), a, h) < rcx)
        if (EXCL(i, j, k)) continue;
        int sip = label[id + S2] == L && !EXCL(i + 1, j, k);
        int sjp = label[id + S] == L && !EXCL(i, j + 1, k);
        int skp = label[id + 1] == L && !EXCL(i, j, k + 1);
#undef EXCL
        float da = sip ? U[id + S2] - v : 0.f;
        float db = sjp ? U[id + S] - v : 0.f;
        float dc = skp ? U[id + 1] - v : 0.f;
        acc[0] += 0.5 * ((double)da * da + (double)db * db + (double)dc * dc) * h;
        acc[1] += -(double)K[id] * rho * h3;
        acc[2] += (double)Pv[id] * rho * h3;
        acc[3] += (double)rho * ((float)i * h) * h3;
        acc[4] += (double)rho * ((float)j * h) * h3;
        acc[5] += (double)rho * ((float)k * h) * h3;
      }
    for (int q = 0; q < 6; ++q) part[6 * i + q] = acc[q];
  }
  for (int q = 0; q < 6; ++q) out[q] = 0;
  for (int i = 0; i < S; ++i)
    for (int q = 0; q < 6; ++q) out[q] += part[6 * i + q];
  free(part);
}

/* molecule.js:1200-1269 gradPtotal: F = 2 Z <grad P> over the integer ball |d|^2 <= R^2
 * around the (integer) nucleus, central differences; FP64 accumulation of the f32 terms. */
void orc_mj_force_gradP(const float* Pt, const orc_mj_atom* atoms, int nElec, int S, float inv_h, int R, double* F) {
  const int64_t S2 = (int64_t)S * S;
  for (int a = 0; a < nElec; ++a) {
    float ZA = (atoms[a].Z <= 0.f) ? atoms[a].Z_nuc : atoms[a].Z;
    if (ZA <= 0.f) { F[3 * a] = F[3 * a + 1] = F[3 * a + 2] = 0; continue; }
    int ci = (int)atoms[a].posI, cj = (int)atoms[a].posJ, ck = (int)atoms[a].posK;
    float inv2h = 0.5f * inv_h;
    double sx = 0, sy = 0, sz = 0, cnt = 0;
    for (int di = -R; di <= R; ++di) {
      int ii = ci + di;
      if (ii < 1 || ii >= S - 1) continue;
      for (int dj = -R; dj <= R; ++dj) {
        int jj = cj + dj;
        if (jj < 1 || jj >= S - 1) continue;
        for (int dk = -R; dk <= R; ++dk) {
          int kk = ck + dk;
          if (kk < 1 || kk >= S - 1) continue;
          if (di * di + dj * dj + dk * dk > R * R) continue;
          int64_t id = (int64_t)ii * S2 + (int64_t)jj * S + kk;
          sx += (double)((Pt[id + S2] - Pt[id - S2]) * inv2h);
          sy += (double)((Pt[id + S] - Pt[id - S]) * inv2h);
          sz += (double)((Pt[id + 1] - Pt[id - 1]) * inv2h);
          cnt += 1;
        }
      }
    }
    if (cnt > 0) { sx /= cnt; sy /= cnt; sz /= cnt; }
    F[3 * a] = 2.0 * ZA * sx; F[3 * a + 1] = 2.0 * ZA * sy; F[3 * a + 2] = 2.0 * ZA * sz;
  }
}

/* molecule.js:1271-1330 direct HF force with h^2 softening over the interior. */
void orc_mj_force_hf(const float* U, const orc_mj_atom* atoms, int nElec, int S, float h, float h2, double* F) {
  const int NN = S - 1;
  const float h3 = h * h * h;
  for (int a = 0; a < nElec; ++a) {
    float ZA = (atoms[a].Z <= 0.f) ? atoms[a].Z_nuc : atoms[a].Z;
    F[3 * a] = F[3 * a + 1] = F[3 * a + 2] = 0;
    if (ZA <= 0.f) continue;
    float Ri = (float)atoms[a].posI * h, Rj = (float)atoms[a].posJ * h, Rk = (float)atoms[a].posK * h;
    double fx = 0, fy = 0, fz = 0;
#pragma omp parallel for reduction(+ : fx, fy, fz) schedule(static)
    for (int i = 1; i < NN; ++i)
      for (int j = 1; j < NN; ++j)
        for (int k = 1; k < NN; ++k) {
          float di = (float)i * h - Ri, dj = (float)j * h - Rj, dk = (float)k * h - Rk;
          float r2 = di * di + dj * dj + dk * dk + h2;
          float r = sqrtf(r2);
          float inv_r3 = 1.0f / (r * r2);
          int64_t id = IDX(i, j, k, S);
          float rho = U[id] * U[id];
          float w = rho * inv_r3 * h3;
          fx += (double)(di * w); fy += (double)(dj * w); fz += (double)(dk * w);
        }
    F[3 * a] = ZA * fx; F[3 * a + 1] = ZA * fy; F[3 * a + 2] = ZA * fz;
  }
}

/* molecule.js:1377-1426 gpuInitAccum over all atoms in one pass plus :1437-1449 final copy:
 * K = sum Zn/r_eff, trial u = Ze^2/sqrt(pi) e^{-Ze r} (0 beyond initRcut or for bare nuclei),
 * label = argmax (strict >, first wins).  K/bestU/label start from 0/0/0 over ALL S^3 points. */
void orc_mj_init(float* K, float* U, uint32_t* label, const orc_mj_atom* atoms, int nElec, int S, float h,
                 float h2, float Rsing, const orc_mj_split* splits) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < S; ++i)
    for (int j = 0; j < S; ++j)
      for (int kk = 0; kk < S; ++kk) {
        int64_t id = IDX(i, j, kk, S);
        float xi = (float)i * h, yj = (float)j * h, zk = (float)kk * h;
        float Kval = 0.f, bU = 0.f;
        uint32_t bestN = 0;
        for (int n = 0; n < nElec; ++n) {
          float Za = atoms[n].Z;
          float Zn = (atoms[n].Z_nuc > 0.f) ? atoms[n].Z_nuc : Za;
          if (Za <= 0.f && Zn <= 0.f) continue;
          float dx = xi - (float)atoms[n].posI * h;
          float dy = yj - (float)atoms[n].posJ * h;
          float dz = zk - (float)atoms[n].posK * h;
          float r2 = dx * dx + dy * dy + dz * dz;
          float r = (atoms[n].rc > 0.f) ? fmaxf(sqrtf(r2 + 0.04f * h2), atoms[n].rc) : fmaxf(sqrtf(r2), Rsing);
          Kval += Zn / r;
          float Ze = atoms[n].initZeff;
          float rReal = sqrtf(r2);
          const int okSplit = !splits || mj_in_split(dx, dy, dz, rReal, &splits[n]);
          float uT = (rReal > atoms[n].initRcut || Za <= 0.f || !okSplit) ? 0.f
                                                                            : Ze * Ze * 0.5641895835f * expf(-Ze * r);
          if (uT > bU) { bU = uT; bestN = (uint32_t)n; }
        }
        K[id] = Kval; U[id] = bU; label[id] = bestN;
      }
}

/* molecule.js:1337-1370 recomputeK_WGSL: K from 0 over all S^3 points from the atoms' stored (u32)
 * positions, distances ((f32)i - (f32)posI) * h, r_eff = max(r, rc) for pseudopotential atoms and
 * max(r, R_SING) for bare Coulomb ones.  uploadInitialData runs it after a USER_INIT_POS
 * initialisation, at the restored nucleus positions (:1959-1981). */
void orc_mj_recompute_k(float* K, const orc_mj_atom* atoms, int nElec, int S, float h, float Rsing) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < S; ++i)
    for (int j = 0; j < S; ++j)
      for (int kk = 0; kk < S; ++kk) {
        float Kval = 0.f;
        for (int n = 0; n < nElec; ++n) {
          float Za = atoms[n].Z;
          float Zn = (atoms[n].Z_nuc > 0.f) ? atoms[n].Z_nuc : Za;
          if (Za <= 0.f && Zn <= 0.f) continue;
          float di = ((float)i - (float)atoms[n].posI) * h;
          float dj = ((float)j - (float)atoms[n].posJ) * h;
          float dk = ((float)kk - (float)atoms[n].posK) * h;
          float r = sqrtf(di * di + dj * dj + dk * dk);
          float reff = (atoms[n].rc > 0.f) ? fmaxf(r, atoms[n].rc) : fmaxf(r, Rsing);
          Kval += Zn / reff;
        }
        K[IDX(i, j, kk, S)] = Kval;
      }
}

/* molecule.js:4563-4582 + :1377-1426: moveNuclei's K rebuild -- K from 0 with the init
 * formula, the running maximum bestU and the current labels persist (an atom may take cells
 * over); psi is not touched. */
void orc_mj_init_persist(float* K, float* bestU, uint32_t* label, const orc_mj_atom* atoms, int nElec, int S, float h,
                         float h2, float Rsing, const orc_mj_split* splits) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < S; ++i)
    for (int j = 0; j < S; ++j)
      for (int kk = 0; kk < S; ++kk) {
        int64_t id = IDX(i, j, kk, S);
        float xi = (float)i * h, yj = (float)j * h, zk = (float)kk * h;
        float Kval = 0.f, bU = bestU[id];
        uint32_t bestN = label[id];
        for (int n = 0; n < nElec; ++n) {
          float Za = atoms[n].Z;
          float Zn = (atoms[n].Z_nuc > 0.f) ? atoms[n].Z_nuc : Za;
          if (Za <= 0.f && Zn <= 0.f) continue;
          float dx = xi - (float)atoms[n].posI * h;
          float dy = yj - (float)atoms[n].posJ * h;
          float dz = zk - (float)atoms[n].posK * h;
          float r2 = dx * dx + dy * dy + dz * dz;
          float r = (atoms[n].rc > 0.f) ? fmaxf(sqrtf(r2 + 0.04f * h2), atoms[n].rc) : fmaxf(sqrtf(r2), Rsing);
          Kval += Zn / r;
          float Ze = atoms[n].initZeff;
          float rReal = sqrtf(r2);
          const int okSplit = !splits || mj_in_split(dx, dy, dz, rReal, &splits[n]);
          float uT = (rReal > atoms[n].initRcut || Za <= 0.f || !okSplit) ? 0.f
                                                                            : Ze * Ze * 0.5641895835f * expf(-Ze * r);
          if (uT > bU) { bU = uT; bestN = (uint32_t)n; }
        }
        K[id] = Kval; bestU[id] = bU; label[id] = bestN;
      }
}

/* ======================================================================
 * FP64 new method (Gaussian nuclei, red-black multigrid).  No reference counterpart.
 * ==================================================================== */

/* Gaussian-smeared nucleus of charge Z and width sigma: K(r) = Z erf(r/(sqrt2 sigma))/r,
 * K(0) = Z sqrt(2/pi)/sigma.  xyz are atom centres in bohr relative to grid point (0,0,0). */
void orc_nm_potential(double* K, const double* xyz, const double* Z, int nAt, int S, double h, double sigma) {
  const int NN = S - 1;
  const double c0 = sqrt(2.0 / M_PI) / sigma, inv = 1.0 / (sqrt(2.0) * sigma);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < S; ++i)
    for (int j = 0; j < S; ++j)
      for (int k = 0; k < S; ++k) {
        int64_t id = IDX(i, j, k, S);
        if (!interior(i, j, k, NN)) { K[id] = 0; continue; }
        double v = 0;
        for (int a = 0; a < nAt; ++a) {
          double dx = i * h - xyz[3 * a], dy = j * h - xyz[3 * a + 1], dz = k * h - xyz[3 * a + 2];
          double r = sqrt(dx * dx + dy * dy + dz * dz);
          v += (r < 1e-12) ? Z[a] * c0 : Z[a] * erf(r * inv) / r;
        }
        K[id] = v;
      }
}

/* FP64 ITP update of the new method: same-label Neumann Laplacian, psi' = psi +
 * half_dv*lap + dt*(K - 2P)*psi (the solver.py update with FP64 fields). */
void orc_nm_update(const double* U, double* Unew, const double* K, const double* P, const int32_t* label, int S,
                   double half_dv, double dt) {
  const int NN = S - 1;
  const int64_t S2 = (int64_t)S * S;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < S; ++i)
    for (int j = 0; j < S; ++j)
      for (int k = 0; k < S; ++k) {
        int64_t id = IDX(i, j, k, S);
        if (!interior(i, j, k, NN)) { Unew[id] = 0; continue; }
        int32_t L = label[id];
        double u = U[id];
        double s = ((label[id + S2] == L) ? U[id + S2] : u) + ((label[id - S2] == L) ? U[id - S2] : u) +
                   ((label[id + S] == L) ? U[id + S] : u) + ((label[id - S] == L) ? U[id - S] : u) +
                   ((label[id + 1] == L) ? U[id + 1] : u) + ((label[id - 1] == L) ? U[id - 1] : u);
        Unew[id] = u + half_dv * (s - 6.0 * u) + dt * (K[id] - 2.0 * P[id]) * u;
      }
}

/* One red-black Gauss-Seidel sweep (red = (i+j+k) even first) for -lap(P)/h^2 = f,
 * i.e. P = (sum_6 P + h^2 f)/6, on a level with S points per axis. */
static void nm_rbgs(double* P, const double* f, int S, double h2) {
  const int NN = S - 1;
  const int64_t S2 = (int64_t)S * S;
  for (int color = 0; color < 2; ++color) {
#pragma omp parallel for schedule(static)
    for (int i = 1; i < NN; ++i)
      for (int j = 1; j < NN; ++j)
        for (int k = 1 + ((i + j + 1 + color) & 1); k < NN; k += 2) {
          int64_t id = IDX(i, j, k, S);
          P[id] = (P[id + S2] + P[id - S2] + P[id + S] + P[id - S] + P[id + 1] + P[id - 1] + h2 * f[id]) / 6.0;
        }
  }
}

static void nm_residual(const double* P, const double* f, double* r, int S, double inv_h2) {
  const int NN = S - 1;
  const int64_t S2 = (int64_t)S * S;
  memset(r, 0, sizeof(double) * (size_t)S * S * S);
#pragma omp parallel for schedule(static)
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        int64_t id = IDX(i, j, k, S);
        r[id] = f[id] + (P[id + S2] + P[id - S2] + P[id + S] + P[id - S] + P[id + 1] + P[id - 1] - 6.0 * P[id]) *
                            inv_h2;
      }
}

/* full weighting (1/64)(8,4,2,1) onto the next coarser vertex-centred level */
static void nm_restrict(const double* fine, double* coarse, int S, int SC) {
  const int NC = SC - 1;
  const int64_t S2 = (int64_t)S * S;
  memset(coarse, 0, sizeof(double) * (size_t)SC * SC * SC);
#pragma omp parallel for schedule(static)
  for (int I = 1; I < NC; ++I)
    for (int J = 1; J < NC; ++J)
      for (int K2 = 1; K2 < NC; ++K2) {
        double v = 0;
        for (int a = -1; a <= 1; ++a)
          for (int b = -1; b <= 1; ++b)
            for (int c = -1; c <= 1; ++c) {
              double w = (a == 0 ? 2.0 : 1.0) * (b == 0 ? 2.0 : 1.0) * (c == 0 ? 2.0 : 1.0);
              v += w * fine[(int64_t)(2 * I + a) * S2 + (int64_t)(2 * J + b) * S + (2 * K2 + c)];
            }
        coarse[IDX(I, J, K2, SC)] = v / 64.0;
      }
}

/* trilinear prolongation of the coarse correction, added to the fine solution */
static void nm_prolong_add(const double* Ec, double* P, int S, int SC) {
  const int NN = S - 1;
  const int64_t SC2 = (int64_t)SC * SC;
#pragma omp parallel for schedule(static)
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        int ci = i >> 1, cj = j >> 1, ck = k >> 1;
        int oi = i & 1, oj = j & 1, ok = k & 1;
        double v = 0;
        for (int a = 0; a <= oi; ++a)
          for (int b = 0; b <= oj; ++b)
            for (int c = 0; c <= ok; ++c) v += Ec[(int64_t)(ci + a) * SC2 + (int64_t)(cj + b) * SC + (ck + c)];
        v /= (double)((1 + oi) * (1 + oj) * (1 + ok));
        P[IDX(i, j, k, S)] += v;
      }
}

/* V(pre,post) cycle on -lap P = f with `levels` levels (NN divisible by 2^(levels-1)),
 * coarsest level solved by `coarse_sweeps` RBGS sweeps.  FP64 throughout. */
static void nm_vcycle_rec(double* P, const double* f, int S, double h, int levels, int pre, int post,
                          int coarse_sweeps) {
  double h2 = h * h;
  if (levels <= 1) {
    for (int s = 0; s < coarse_sweeps; ++s) nm_rbgs(P, f, S, h2);
    return;
  }
  for (int s = 0; s < pre; ++s) nm_rbgs(P, f, S, h2);
  int SC = (S - 1) / 2 + 1;
  size_t nf = (size_t)S * S * S, nc = (size_t)SC * SC * SC;
  double* r = (double*)malloc(sizeof(double) * nf);
  double* rc = (double*)malloc(sizeof(double) * nc);
  double* ec = (double*)calloc(nc, sizeof(double));
  nm_residual(P, f, r, S, 1.0 / h2);
  nm_restrict(r, rc, S, SC);
  nm_vcycle_rec(ec, rc, SC, 2 * h, levels - 1, pre, post, coarse_sweeps);
  nm_prolong_add(ec, P, S, SC);
  for (int s = 0; s < post; ++s) nm_rbgs(P, f, S, h2);
  free(r); free(rc); free(ec);
}

/* Poisson for the Hartree half-potential: lap P = -2 pi rho  <=>  -lap P = 2 pi psi^2. */
void orc_nm_vcycle(double* P, const double* U, int S, double h, int levels, int pre, int post, int coarse_sweeps) {
  size_t n = (size_t)S * S * S;
  double* f = (double*)malloc(sizeof(double) * n);
  for (size_t q = 0; q < n; ++q) f[q] = 2.0 * M_PI * U[q] * U[q];
  nm_vcycle_rec(P, f, S, h, levels, pre, post, coarse_sweeps);
  free(f);
}

/* Per-label FP64 sums of the new flavour's readout, 5 per domain: norm, T, V_eK, h^3 sum P rho and
 * h^3 sum P (A P) with A = -lap_h (Dirichlet faces; attributed to the point's label).  out[0..2]: the
 * sums of T, V_eK and h^3 sum P rho over the domains. */
void orc_nm_energy(const double* U, const double* K, const double* P, const int32_t* label, int S, double h,
                   double* out, int nDom, double* per_domain) {
  const int NN = S - 1;
  const int64_t S2 = (int64_t)S * S;
  const double h3 = h * h * h;
  double* pd = (double*)calloc((size_t)S * nDom * 5, sizeof(double));
#pragma omp parallel for schedule(static)
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        int64_t id = IDX(i, j, k, S);
        double u = U[id], rho = u * u;
        int32_t L = label[id];
        if (L < 0 || L >= nDom) continue;
        double a = (label[id + S2] == L) ? U[id + S2] - u : 0.0;
        double b = (label[id + S] == L) ? U[id + S] - u : 0.0;
        double c = (label[id + 1] == L) ? U[id + 1] - u : 0.0;
        /* every same-label edge with an interior end point once: forward edges plus the edge
           to the Dirichlet face below on the first interior layer (psi = 0 there) */
        double t = a * a + b * b + c * c;
        if (i == 1 && label[id - S2] == L) t += u * u;
        if (j == 1 && label[id - S] == L) t += u * u;
        if (k == 1 && label[id - 1] == L) t += u * u;
        double* q = pd + ((size_t)i * nDom + L) * 5;
        double ap = (6.0 * P[id] - (P[id + S2] + P[id - S2] + P[id + S] + P[id - S] + P[id + 1] + P[id - 1])) / (h * h);
        q[0] += rho * h3; q[1] += 0.5 * t * h; q[2] += -K[id] * rho * h3;
        q[3] += P[id] * rho * h3; q[4] += P[id] * ap * h3;
      }
  memset(per_domain, 0, sizeof(double) * nDom * 5);
  for (int i = 0; i < S; ++i)
    for (int q = 0; q < nDom * 5; ++q) per_domain[q] += pd[(size_t)i * nDom * 5 + q];
  out[0] = out[1] = out[2] = 0;
  for (int d = 0; d < nDom; ++d) { out[0] += per_domain[5 * d + 1]; out[1] += per_domain[5 * d + 2]; out[2] += per_domain[5 * d + 3]; }
  free(pd);
}

/* Normalise FP64 psi to charge Zdom[l] per label from the per_domain norms (column 0). */
void orc_nm_normalize(double* U, const int32_t* label, int64_t S3, int nDom, const double* Zdom, const double* norms) {
#pragma omp parallel for schedule(static)
  for (int64_t id = 0; id < S3; ++id) {
    int32_t l = label[id];
    if (l < 0 || l >= nDom) continue;
    double n = norms[l];
    if (n > 1e-300 && Zdom[l] > 0) U[id] *= sqrt(Zdom[l] / n);
  }
}

/* Hellmann-Feynman / stationary-point gradient of E_eK = -h^3 sum K rho with Gaussian
 * nuclei: dE/dR_a = -h^3 sum rho dK_a/dR_a, where dK_a/dR_a = -dK_a/dr * (x-R)/|x-R|.
 * Returns the FORCE -dE/dR (without the nuclear-nuclear part). */
void orc_nm_force(const double* U, const double* xyz, const double* Z, int nAt, int S, double h, double sigma,
                  double* F) {
  const int NN = S - 1;
  const double h3 = h * h * h, inv = 1.0 / (sqrt(2.0) * sigma), g = sqrt(2.0 / M_PI) / sigma;
  for (int a = 0; a < nAt; ++a) {
    double fx = 0, fy = 0, fz = 0;
#pragma omp parallel for reduction(+ : fx, fy, fz) schedule(static)
    for (int i = 1; i < NN; ++i)
      for (int j = 1; j < NN; ++j)
        for (int k = 1; k < NN; ++k) {
          double dx = i * h - xyz[3 * a], dy = j * h - xyz[3 * a + 1], dz = k * h - xyz[3 * a + 2];
          double r2 = dx * dx + dy * dy + dz * dz, r = sqrt(r2);
          if (r < 1e-12) continue;
          double u = U[IDX(i, j, k, S)], rho = u * u;
          /* d/dr [erf(r*inv)/r] = (g e^{-r^2 inv^2})/r - erf(r inv)/r^2 */
          double dKdr = Z[a] * (g * exp(-r2 * inv * inv) / r - erf(r * inv) / r2);
          /* F = -dE/dR = -(h^3 sum rho dK/dr (x-R)/r)  since dK/dR = -dK/dr (x-R)/r and E=-sum K rho h3 */
          double w = -h3 * rho * dKdr / r;
          fx += w * dx; fy += w * dy; fz += w * dz;
        }
    F[3 * a] = fx; F[3 * a + 1] = fy; F[3 * a + 2] = fz;
  }
}

/* Initial state of the new method: label = nearest domain seed by f32 squared distance
 * (first seed wins ties), psi = exp(-sqrt(d2)) in FP64, boundary psi = 0.  seeds: x,y,z (f32,
 * bohr) and the entry index of each domain seed. */
void orc_nm_init(double* U, int32_t* label, const float* seeds_xyz, const int32_t* seed_idx, int nSeed, int S, float h) {
  const int NN = S - 1;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < S; ++i)
    for (int j = 0; j < S; ++j)
      for (int k = 0; k < S; ++k) {
        int64_t id = IDX(i, j, k, S);
        float x = (float)i * h, y = (float)j * h, z = (float)k * h;
        float best = 3.4e38f;
        int bl = 0;
        for (int m = 0; m < nSeed; ++m) {
          float dx = x - seeds_xyz[3 * m], dy = y - seeds_xyz[3 * m + 1], dz = z - seeds_xyz[3 * m + 2];
          float d2 = dx * dx + dy * dy + dz * dz;
          if (d2 < best) { best = d2; bl = seed_idx[m]; }
        }
        label[id] = bl;
        U[id] = interior(i, j, k, NN) ? exp(-sqrt((double)best)) : 0.0;
      }
}

/* The molecule.js level-set rule (molecule.js:426-540) on FP64 psi, snapshot labels. */
void orc_nm_evolve(const int32_t* labelIn, int32_t* labelOut, const double* U, float* W, int S, double dt_w,
                   double curvReg) {
  const int NN = S - 1;
  const int64_t S2 = (int64_t)S * S;
  memcpy(labelOut, labelIn, sizeof(int32_t) * (size_t)S2 * S);
#pragma omp parallel for schedule(static)
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        int64_t id = IDX(i, j, k, S);
        int32_t myL = labelIn[id];
        double myRho = U[id] * U[id];
        const int64_t nb[6] = {id + S2, id - S2, id + S, id - S, id + 1, id - 1};
        int32_t bestL = myL;
        double bestRho = 0, myCnt = 0;
        for (int q = 0; q < 6; ++q) {
          int32_t l = labelIn[nb[q]];
          if (l == myL) myCnt += 1.0;
          else {
            double r = U[nb[q]] * U[nb[q]];
            if (r > bestRho) { bestRho = r; bestL = l; }
          }
        }
        double w = (double)W[id];
        if (myCnt >= 6.0) { W[id] = (float)(w > 1.0 ? w : 1.0); labelOut[id] = myL; continue; }
        double denom = myRho + bestRho;
        double vel = (denom < (double)1e-20f) ? 0.0 : (myRho - bestRho) / denom;
        w = w + dt_w * vel;
        double curv = (myCnt - 3.0) / 3.0;
        w = w + curvReg * curv;
        int32_t newL = myL;
        if (w < 0.0) { newL = bestL; w = (double)0.1f; }
        W[id] = (float)w;
        labelOut[id] = newL;
      }
}

/* The same level-set rule on fp32 psi with every operation in f32 (the mixed-precision path's
 * label pass): products, sums and the quotient each rounded to single precision, in the order of
 * orc_nm_evolve.  dt_w and curvReg are the f32 values of the parameters. */
void orc_nm_evolve_f32(const int32_t* labelIn, int32_t* labelOut, const float* U, float* W, int S, float dt_w,
                       float curvReg) {
  const int NN = S - 1;
  const int64_t S2 = (int64_t)S * S;
  memcpy(labelOut, labelIn, sizeof(int32_t) * (size_t)S2 * S);
#pragma omp parallel for schedule(static)
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        int64_t id = IDX(i, j, k, S);
        int32_t myL = labelIn[id];
        float uc = U[id];
        float myRho = uc * uc;
        const int64_t nb[6] = {id + S2, id - S2, id + S, id - S, id + 1, id - 1};
        int32_t bestL = myL;
        float bestRho = 0.0f, myCnt = 0.0f;
        for (int q = 0; q < 6; ++q) {
          int32_t l = labelIn[nb[q]];
          if (l == myL) myCnt = myCnt + 1.0f;
          else {
            float un = U[nb[q]];
            float r = un * un;
            if (r > bestRho) { bestRho = r; bestL = l; }
          }
        }
        float w = W[id];
        if (myCnt >= 6.0f) { W[id] = w > 1.0f ? w : 1.0f; labelOut[id] = myL; continue; }
        float denom = myRho + bestRho;
        float vel = (denom < 1e-20f) ? 0.0f : (myRho - bestRho) / denom;
        w = w + dt_w * vel;
        float curv = (myCnt - 3.0f) / 3.0f;
        w = w + curvReg * curv;
        int32_t newL = myL;
        if (w < 0.0f) { newL = bestL; w = 0.1f; }
        W[id] = w;
        labelOut[id] = newL;
      }
}

/* ====================================================================
 * atom.js flavour: per-shell fields U[m], W[m], P[m] (atom.js:1-346).  JS numbers are f64 and
 * every Float32Array store rounds to f32; loops run in the reference's lexicographic in-place
 * order.  Fields are nShells consecutive S^3 blocks.
 * ==================================================================== */

typedef struct {
  double ne, Rmax, Zeff;                    /* shellConfig[m].ne / .Rmax / .Zeff */
  int32_t split, half_index, outer_half, fixed_w;  /* 'halfspace', .halfIndex, .outerHalf, .fixedW */
} orc_shell;

/* atom.js:55-125: K, U, W, P on all S^3 points, then each U normalised over all points. */
void orc_at_init(float* U, float* W, float* P, float* K, const orc_shell* sh, int nS, int NN, double scr,
                 double Zk) {
  const int S = NN + 1;
  const int64_t S3 = (int64_t)S * S * S;
  const double h = scr / NN, h2 = h * h, h3 = h * h * h;
  const int N2 = NN / 2;
  double Rmin[16], Rmax[16];
  Rmin[0] = 0; Rmax[0] = sh[0].Rmax;
  for (int m = 1; m < nS; ++m) { Rmin[m] = sh[m - 1].Rmax; Rmax[m] = sh[m].Rmax ? sh[m].Rmax : scr / 2; }
  memset(U, 0, sizeof(float) * S3 * nS);
  memset(W, 0, sizeof(float) * S3 * nS);
  for (int i = 0; i <= NN; ++i)
    for (int j = 0; j <= NN; ++j)
      for (int k = 0; k <= NN; ++k) {
        const int64_t id = IDX(i, j, k, S);
        const double r2 = (double)((i - N2) * (i - N2)) * h2 + (double)((j - N2) * (j - N2)) * h2 +
                          (double)((k - N2) * (k - N2)) * h2 + 0.12 * h2;
        const double r = sqrt(r2);
        K[id] = (float)(Zk / r);
        for (int m = 0; m < nS; ++m) {
          float* Um = U + m * S3; float* Wm = W + m * S3;
          int in;
          if (sh[m].split) {
            if (i == N2) { in = 1; Wm[id] = 0.5f; }
            else in = sh[m].half_index == 0 ? (i < N2) : (i > N2);
          } else if (sh[m].outer_half) {
            in = r >= Rmin[m] && r < Rmax[m] && i > N2;
          } else {
            in = r >= Rmin[m] && r < Rmax[m];
          }
          if (in) {
            Um[id] = (float)exp(-sh[m].Zeff * r);
            double w = 1.0;
            const double smoothW = 2 * h;
            if (!sh[m].split) {
              if (Rmin[m] > 0) { const double din = r - Rmin[m]; if (din < smoothW) w = fmin(w, din / smoothW); }
              const double dout = Rmax[m] - r;
              if (dout < smoothW) w = fmin(w, dout / smoothW);
            }
            w = fmax(0.01, w);
            if (Wm[id] == 0) Wm[id] = (float)w;
          }
        }
        for (int m = 0; m < nS; ++m) P[m * S3 + id] = (float)(0.5 / r);
      }
  for (int m = 0; m < nS; ++m) {
    float* Um = U + m * S3;
    double n2 = 0;
    for (int64_t id = 0; id < S3; ++id) n2 += (double)Um[id] * Um[id] * h3;
    const double sc = 1 / sqrt(n2);
    for (int64_t id = 0; id < S3; ++id) Um[id] = (float)(Um[id] * sc);
  }
}

/* atom.js:127-138 in-place lexicographic Jacobi-labelled (Gauss-Seidel) sweeps */
static void at_gs(float* P, const float* rhs, int N, double h2, int nIter) {
  const int S = N + 1;
  const int64_t S2 = (int64_t)S * S;
  for (int it = 0; it < nIter; ++it)
    for (int i = 1; i < N; ++i)
      for (int j = 1; j < N; ++j)
        for (int k = 1; k < N; ++k) {
          const int64_t id = i * S2 + (int64_t)j * S + k;
          P[id] = (float)(((double)P[id + S2] + P[id - S2] + P[id + S] + P[id - S] + P[id + 1] + P[id - 1] +
                           h2 * rhs[id]) / 6);
        }
}

/* atom.js:186-210 poissonVcycle: 4 sweeps, residual, injection to N/2, 20 coarse sweeps from 0,
   injection-add prolongation, 4 sweeps. */
void orc_at_vcycle(float* P, const float* rhs, int N, double h) {
  const int S = N + 1, Nc = N / 2, Sc = Nc + 1;
  const int64_t S2 = (int64_t)S * S, S3 = S2 * S, Sc2 = (int64_t)Sc * Sc;
  const double h2 = h * h;
  at_gs(P, rhs, N, h2, 4);
  float* res = (float*)calloc(S3, sizeof(float));
  for (int i = 1; i < N; ++i)
    for (int j = 1; j < N; ++j)
      for (int k = 1; k < N; ++k) {
        const int64_t id = i * S2 + (int64_t)j * S + k;
        const double lap = ((double)P[id + S2] + P[id - S2] + P[id + S] + P[id - S] + P[id + 1] + P[id - 1] -
                            6 * (double)P[id]) / h2;
        res[id] = (float)(rhs[id] + lap);
      }
  float* cd = (float*)calloc(Sc2 * Sc, sizeof(float));
  for (int i = 1; i < Nc; ++i)
    for (int j = 1; j < Nc; ++j)
      for (int k = 1; k < Nc; ++k) cd[i * Sc2 + (int64_t)j * Sc + k] = res[(2 * i) * S2 + (int64_t)(2 * j) * S + 2 * k];
  const double hc = h * 2, hc2 = hc * hc;
  float* Pc = (float*)calloc(Sc2 * Sc, sizeof(float));
  at_gs(Pc, cd, Nc, hc2, 20);
  for (int i = 1; i < Nc; ++i)
    for (int j = 1; j < Nc; ++j)
      for (int k = 1; k < Nc; ++k) {
        const double val = Pc[i * Sc2 + (int64_t)j * Sc + k];
        for (int di = 0; di <= 1; ++di)
          for (int dj = 0; dj <= 1; ++dj)
            for (int dk = 0; dk <= 1; ++dk) {
              const int fi = 2 * i + di, fj = 2 * j + dj, fk = 2 * k + dk;
              if (fi > 0 && fi < N && fj > 0 && fj < N && fk > 0 && fk < N) {
                const int64_t f = fi * S2 + (int64_t)fj * S + fk;
                P[f] = (float)(P[f] + val);
              }
            }
      }
  at_gs(P, rhs, N, h2, 4);
  free(res); free(cd); free(Pc);
}

/* atom.js:212-343 physicsStep.  E4 = {E, E_T, E_eK, E_ee}; per_shell (nS x 4) = {ET, Eee, EeK, nrm}. */
void orc_at_step(float* U, float* W, float* P, const float* K, const orc_shell* sh, int nS, int NN, double scr,
                 double d, int simultaneous, double* E4, double* per_shell) {
  const int S = NN + 1;
  const int64_t S2 = (int64_t)S * S, S3 = S2 * S;
  const double h = scr / NN, h2 = h * h, h3 = h * h * h, dt = d * h2, PI = 3.141592653589793;
  float c[16];
  double ET = 0, Eee = 0, EeK = 0;
  for (int q = 0; q < 4 * nS; ++q) per_shell[q] = 0;
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        const int64_t id = i * S2 + (int64_t)j * S + k;
        for (int m = 0; m < nS; ++m) {
          c[m] = 0;
          for (int n = 0; n < nS; ++n) {
            if (n != m) c[m] = (float)((double)c[m] - U[n * S3 + id]);
            c[m] = (float)(0.5 * ((double)c[m] + U[m * S3 + id]));
          }
        }
        const int64_t ip = id + S2, im = id - S2, jp = id + S, jm = id - S, kp = id + 1, km = id - 1;
        for (int m = 0; m < nS; ++m) {
          float* Um = U + m * S3; float* Wm = W + m * S3; float* Pm = P + m * S3;
          if (!sh[m].fixed_w) {
            const double lapW = ((double)Wm[ip] + Wm[im] + Wm[jp] + Wm[jm] + Wm[kp] + Wm[km] - 6 * (double)Wm[id]) / h2;
            const double gwx = ((double)Wm[ip] - Wm[im]) / h, gwy = ((double)Wm[jp] - Wm[jm]) / h,
                         gwz = ((double)Wm[kp] - Wm[km]) / h;
            const double gradW = sqrt(gwx * gwx + gwy * gwy + gwz * gwz);
            Wm[id] = (float)(Wm[id] + (2 * dt * fabs((double)c[m]) * lapW + 9 * dt * (double)c[m] * gradW));
          }
          const double wlap =
              0.5 * d * (((double)Um[ip] - Um[id]) * ((double)Wm[ip] + Wm[id]) * 0.5 -
                         ((double)Um[id] - Um[im]) * ((double)Wm[id] + Wm[im]) * 0.5) +
              0.5 * d * (((double)Um[jp] - Um[id]) * ((double)Wm[jp] + Wm[id]) * 0.5 -
                         ((double)Um[id] - Um[jm]) * ((double)Wm[id] + Wm[jm]) * 0.5) +
              0.5 * d * (((double)Um[kp] - Um[id]) * ((double)Wm[kp] + Wm[id]) * 0.5 -
                         ((double)Um[id] - Um[km]) * ((double)Wm[id] + Wm[km]) * 0.5);
          Um[id] = (float)(Um[id] + (wlap + dt * ((double)K[id] - 2 * (double)Pm[id]) * Um[id] * Wm[id]));
          int dominated = 1;
          for (int n = 0; n < nS; ++n)
            if (n != m && W[n * S3 + id] >= Wm[id]) { dominated = 0; break; }
          if (dominated && Wm[id] > 0.01) {
            int dip = 1, djp = 1, dkp = 1;
            for (int n = 0; n < nS; ++n)
              if (n != m) {
                if (W[n * S3 + ip] >= Wm[ip]) dip = 0;
                if (W[n * S3 + jp] >= Wm[jp]) djp = 0;
                if (W[n * S3 + kp] >= Wm[kp]) dkp = 0;
              }
            const double gx = dip ? (double)Um[ip] - Um[id] : 0, gy = djp ? (double)Um[jp] - Um[id] : 0,
                         gz = dkp ? (double)Um[kp] - Um[id] : 0;
            const double tm = 0.5 * (gx * gx + gy * gy + gz * gz) * h;
            const double eem = (double)Pm[id] * Um[id] * Um[id] * h3;
            const double ekm = -(double)K[id] * Um[id] * Um[id] * h3;
            ET += tm; Eee += eem; EeK += ekm;
            per_shell[4 * m] += tm; per_shell[4 * m + 1] += eem; per_shell[4 * m + 2] += ekm;
            per_shell[4 * m + 3] += (double)Um[id] * Um[id] * h3;
          }
          if (simultaneous) {
            double rhoOther = 0;
            for (int n = 0; n < nS; ++n)
              if (n != m) rhoOther += (double)U[n * S3 + id] * U[n * S3 + id] * W[n * S3 + id];
            const double lapP = ((double)Pm[ip] + Pm[im] + Pm[jp] + Pm[jm] + Pm[kp] + Pm[km] - 6 * (double)Pm[id]) / h2;
            Pm[id] = (float)(Pm[id] + (dt * lapP + 2 * PI * dt * rhoOther));
          }
        }
      }
  if (!simultaneous) {
    float* rhs = (float*)calloc(S3, sizeof(float));
    for (int m = 0; m < nS; ++m) {
      for (int i = 1; i < NN; ++i)
        for (int j = 1; j < NN; ++j)
          for (int k = 1; k < NN; ++k) {
            const int64_t id = i * S2 + (int64_t)j * S + k;
            double rhoOther = 0;
            for (int n = 0; n < nS; ++n)
              if (n != m) rhoOther += (double)U[n * S3 + id] * U[n * S3 + id] * W[n * S3 + id];
            rhs[id] = (float)(2 * PI * rhoOther);
          }
      orc_at_vcycle(P + m * S3, rhs, NN, h);
    }
    free(rhs);
  }
  for (int m = 0; m < nS; ++m) {
    float* Um = U + m * S3;
    double n2 = 0;
    for (int i = 1; i < NN; ++i)
      for (int j = 1; j < NN; ++j)
        for (int k = 1; k < NN; ++k) { const double u = Um[IDX(i, j, k, S)]; n2 += u * u * h3; }
    const double sc = 1 / sqrt(n2);
    for (int i = 1; i < NN; ++i)
      for (int j = 1; j < NN; ++j)
        for (int k = 1; k < NN; ++k) { const int64_t id = IDX(i, j, k, S); Um[id] = (float)(Um[id] * sc); }
  }
  E4[0] = ET + EeK + Eee; E4[1] = ET; E4[2] = EeK; E4[3] = Eee;
}

/* ======================================================================
 * mol_fast.js multi-field solver (mol_fast.js:1-1651), f32 WGSL semantics
 *
 * One U, W, P field per electron (one electron per nucleus), field m at offset m*S3.
 * Every function follows the shader it names in the reference's operation order, with
 * plain IEEE single operations (no contraction); the reductions repeat the shaders'
 * workgroup trees exactly, so the f32 sums are the reference's bit for bit.
 * ==================================================================== */

#define MF_MAX 16
typedef struct {
  int32_t NN, S, N2, n, shell_mode, pad0;
  float h, h2, inv_h, inv_h2, dt, half_d, h3, two_pi;
  float R_out, field_x, alpha_tf, full_self;
  float kc, kc_multi, beta, pad1;
  float atoms[MF_MAX][4]; /* i, j, k, Z */
  float rcs[MF_MAX][4];   /* rc, norm target, tilt_x, tilt_y */
  float r_out[MF_MAX];
  int32_t split_type[MF_MAX], split_idx[MF_MAX], split_fix[MF_MAX], split_group[MF_MAX];
  float ax[MF_MAX][4];
} orc_mf_params;

/* pow and atan2: the f64 functions rounded once to f32 (WGSL leaves their accuracy to the
 * implementation; the CUDA side does the same) */
static inline float mf_pow(float x, float y) { return (float)pow((double)x, (double)y); }
static inline float mf_atan2(float y, float x) { return (float)atan2((double)y, (double)x); }

/* the smooth rc cusp t^2 (3 - 2t) on w (mol_fast.js:188-193, :255-260) */
static inline float mf_cusp(float r, float rc, float h) {
  const float edge = rc - 3.0f * h;
  const float t = fminf(fmaxf((r - edge) / (rc - edge), 0.0f), 1.0f);
  return t * t * (3.0f - 2.0f * t);
}

static inline float mf_dot3(const float* a, float x, float y, float z) { return a[0] * x + a[1] * y + a[2] * z; }

/* the three-sector index around axis ax (mol_fast.js:206-216) */
static inline uint32_t mf_third_sector(const float* ax, float x, float y, float z) {
  const float dotA = mf_dot3(ax, x, y, z);
  const float px = x - dotA * ax[0], py = y - dotA * ax[1], pz = z - dotA * ax[2];
  float e1[3];
  if (fabsf(ax[2]) < 0.9f) { e1[0] = ax[1]; e1[1] = -ax[0]; e1[2] = 0.0f; }
  else { e1[0] = 0.0f; e1[1] = ax[2]; e1[2] = -ax[1]; }
  const float L = sqrtf(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
  e1[0] = e1[0] / L; e1[1] = e1[1] / L; e1[2] = e1[2] / L;
  const float e2[3] = {ax[1] * e1[2] - ax[2] * e1[1], ax[2] * e1[0] - ax[0] * e1[2], ax[0] * e1[1] - ax[1] * e1[0]};
  float theta = mf_atan2(mf_dot3(e2, px, py, pz), mf_dot3(e1, px, py, pz)) - 0.0f;
  if (theta < -3.141592653589793f) theta = theta + 6.283185307179586f;
  if (theta > 3.141592653589793f) theta = theta - 6.283185307179586f;
  return ((uint32_t)floorf((theta + 3.141592653589793f) / 2.094395102393195f)) % 3u;
}

/* the angular split enforcement of SHELL_MODE (mol_fast.js:196-246); rel in grid cells */
static inline int mf_in_sector(const orc_mf_params* p, int m, float x, float y, float z, float r_m) {
  const int t = p->split_type[m];
  const uint32_t sidx = (uint32_t)p->split_idx[m];
  const float* ax = p->ax[m];
  if (t == 2) {
    const float d = mf_dot3(ax, x, y, z);
    return sidx == 0 ? d < 0.0f : d >= 0.0f;
  }
  if (t == 3) return mf_third_sector(ax, x, y, z) == sidx;
  if (t == 4) {
    if (r_m > 1e-6f) {
      const float ux = x / r_m, uy = y / r_m, uz = z / r_m;
      uint32_t best = 0;
      float bestD = 1.0f * ux + 1.0f * uy + 1.0f * uz;
      const float d1 = 1.0f * ux + -1.0f * uy + -1.0f * uz;
      if (d1 > bestD) { bestD = d1; best = 1; }
      const float d2 = -1.0f * ux + 1.0f * uy + -1.0f * uz;
      if (d2 > bestD) { bestD = d2; best = 2; }
      const float d3 = -1.0f * ux + -1.0f * uy + 1.0f * uz;
      if (d3 > bestD) { bestD = d3; best = 3; }
      return best == sidx;
    }
    return 1;
  }
  if (t == 5) {
    const float d = mf_dot3(ax, x, y, z);
    if (sidx == 0) return d >= 0.0f;
    if (d >= 0.0f) return 0;
    return mf_third_sector(ax, x, y, z) == sidx - 1u;
  }
  return 1;
}

/* updateWGSL (mol_fast.js:134-351): front w, amplitude u and potential P of every electron,
 * reading the old buffers (Ui, Wi, Pi) and writing the new ones at the interior cells. */
void orc_mf_update(const orc_mf_params* p, const float* Ui, const float* Wi, const float* Pi, const float* K,
                   float* Uo, float* Wo, float* Po) {
  const int NN = p->NN, S = p->S, n = p->n;
  const int64_t S2 = (int64_t)S * S, S3 = S2 * S;
#pragma omp parallel for schedule(static)
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        const int64_t id = i * S2 + (int64_t)j * S + k;
        for (int m = 0; m < n; ++m) {
          const int64_t o = m * S3;
          const float uc = Ui[o + id];
          float umax = 0.0f;
          for (int q = 0; q < n; ++q) {
            if (q == m) continue;
            const float un = Ui[q * S3 + id];
            if (un > umax) umax = un;
          }
          const float cm = uc - umax;
          const float wc = Wi[o + id];
          const float wip = Wi[o + id + S2], wim = Wi[o + id - S2];
          const float wjp = Wi[o + id + S], wjm = Wi[o + id - S];
          const float wkp = Wi[o + id + 1], wkm = Wi[o + id - 1];
          const float lw = (wip + wim + wjp + wjm + wkp + wkm - 6.0f * wc) * p->inv_h2;
          const float gx = (wip - wim) * p->inv_h, gy = (wjp - wjm) * p->inv_h, gz = (wkp - wkm) * p->inv_h;
          float nw = wc + 0.05f * p->dt * fabsf(cm) * lw + 1.0f * p->dt * cm * sqrtf(gx * gx + gy * gy + gz * gz);
          nw = fminf(fmaxf(nw, 0.0f), 1.0f);
          if (p->shell_mode) {
            const float rc_m = p->rcs[m][0];
            const float ro_m = p->r_out[m] * p->R_out;
            const float dxm = (float)i - p->atoms[m][0], dym = (float)j - p->atoms[m][1], dzm = (float)k - p->atoms[m][2];
            const float r_m = sqrtf(dxm * dxm + dym * dym + dzm * dzm) * p->h;
            if (rc_m > 0.0f && r_m < rc_m) nw = fminf(nw, mf_cusp(r_m, rc_m, p->h));
            if (ro_m > 0.0f && r_m > ro_m) nw = (r_m <= ro_m + p->h) ? nw : 0.0f;
            if (p->split_type[m] != 0 && p->split_fix[m] == 1 && !mf_in_sector(p, m, dxm, dym, dzm, r_m)) nw = 0.0f;
          } else {
            for (int a = 0; a < n; ++a) {
              const float dx = (float)i - p->atoms[a][0], dy = (float)j - p->atoms[a][1], dz = (float)k - p->atoms[a][2];
              const float r = sqrtf(dx * dx + dy * dy + dz * dz) * p->h;
              const float rc_a = p->rcs[a][0];
              if (rc_a > 0.0f && r < rc_a) nw = fminf(nw, mf_cusp(r, rc_a, p->h));
            }
          }
          Wo[o + id] = nw;
          float Ptot = 0.0f, Pgrp = 0.0f;
          for (int q = 0; q < n; ++q) {
            const float Pn = Pi[q * S3 + id];
            Ptot += Pn;
            if (p->split_group[q] == p->split_group[m]) Pgrp += Pn;
          }
          const float selfN = p->rcs[m][1];
          const float fm_multi = p->full_self > 0.5f ? 0.0f : 1.0f / selfN;
          const float fm = selfN > 1.0f ? fm_multi : 1.0f;
          const float Vother = 2.0f * (Ptot - fm * Pgrp);
          const float rho_m = uc * uc;
          const float V_TF = (selfN > 1.0f && p->alpha_tf > 0.0f) ? p->alpha_tf * mf_pow(fmaxf(rho_m, 1e-20f), 0.6666667f) : 0.0f;
          const float tilt_y = p->rcs[m][3], tilt_x = p->rcs[m][2];
          const float x_au = ((float)i - (float)p->N2) * p->h;
          const float y_au = ((float)j - (float)p->N2) * p->h;
          const float V_tilt = -tilt_x * x_au - tilt_y * y_au;
          float rho_other = 0.0f;
          for (int q = 0; q < n; ++q) {
            if (q == m) continue;
            const float un = Ui[q * S3 + id];
            rho_other += un * un;
          }
          const float V_Pauli = p->beta * rho_other;
          const float uip = Ui[o + id + S2], uim = Ui[o + id - S2];
          const float ujp = Ui[o + id + S], ujm = Ui[o + id - S];
          const float ukp = Ui[o + id + 1], ukm = Ui[o + id - 1];
          const float k_mult = selfN > 1.0f ? p->kc_multi : 1.0f;
          const float hd = p->half_d * k_mult;
          Uo[o + id] = uc + hd * ((uip - uc) * (wip + nw) * 0.5f - (uc - uim) * (nw + wim) * 0.5f) +
                       hd * ((ujp - uc) * (wjp + nw) * 0.5f - (uc - ujm) * (nw + wjm) * 0.5f) +
                       hd * ((ukp - uc) * (wkp + nw) * 0.5f - (uc - ukm) * (nw + wkm) * 0.5f) +
                       p->dt * (K[id] - Vother - V_TF - V_tilt - V_Pauli - p->field_x * x_au) * uc * wc;
          const float Pc = Pi[o + id];
          Po[o + id] = Pc +
                       p->dt * (Pi[o + id + S2] + Pi[o + id - S2] + Pi[o + id + S] + Pi[o + id - S] + Pi[o + id + 1] +
                                Pi[o + id - 1] - 6.0f * Pc) * p->inv_h2 +
                       p->two_pi * p->dt * uc * uc;
        }
      }
}

/* reduceWGSL + finalizeWGSL (mol_fast.js:353-472): per-cell f32 terms, 128-cell workgroups over
 * the interior in linear order, the shared-memory trees, and the single finalize workgroup.
 * sums: n norms^2, T, V_eK, V_ee, dipole x, y, z. */
void orc_mf_reduce(const orc_mf_params* p, const float* U, const float* W, const float* Pv, const float* K,
                   float* sums) {
  const int NN = p->NN, S = p->S, n = p->n, NR = n + 6;
  const int64_t S2 = (int64_t)S * S, S3 = S2 * S;
  const int64_t NM = NN - 1, tot = NM * NM * NM;
  const int64_t nwg = (tot + 127) / 128;
  float* part = (float*)calloc((size_t)(nwg * NR), sizeof(float));
#pragma omp parallel for schedule(static)
  for (int64_t wg = 0; wg < nwg; ++wg) {
    float sn[128 * (MF_MAX + 6)];
    for (int q = 0; q < 128 * NR; ++q) sn[q] = 0.0f;
    for (int lid = 0; lid < 128; ++lid) {
      const int64_t cell = wg * 128 + lid;
      if (cell >= tot) continue;
      const int k = (int)(cell % NM) + 1, j = (int)((cell / NM) % NM) + 1, i = (int)(cell / (NM * NM)) + 1;
      const int64_t id = i * S2 + (int64_t)j * S + k;
      float T = 0.0f, VeK = 0.0f, Vee = 0.0f, dx = 0.0f, dy = 0.0f, dz = 0.0f;
      const float xc = ((float)i - (float)p->N2) * p->h;
      const float yc = ((float)j - (float)p->N2) * p->h;
      const float zc = ((float)k - (float)p->N2) * p->h;
      float Ptot = 0.0f;
      for (int q = 0; q < n; ++q) Ptot += Pv[q * S3 + id];
      for (int m = 0; m < n; ++m) {
        const int64_t o = m * S3;
        const float v = U[o + id];
        sn[lid * NR + m] = v * v * p->h3;
        if (W[o + id] > 0.1f) {
          const float a = U[o + id + S2] - v, b = U[o + id + S] - v, c = U[o + id + 1] - v;
          const float kmt = p->rcs[m][1] > 1.0f ? p->kc_multi : 1.0f;
          T += kmt * p->kc * (a * a + b * b + c * c) * p->h;
        }
        VeK -= K[id] * v * v * p->h3;
        const float rho_cell = v * v * p->h3;
        dx -= rho_cell * xc;
        dy -= rho_cell * yc;
        dz -= rho_cell * zc;
        const float selfN = p->rcs[m][1];
        const float fm = selfN > 1.0f ? 1.0f / selfN : 1.0f;
        Vee += (Ptot - fm * Pv[o + id]) * v * v * p->h3;
        if (selfN > 1.0f && p->alpha_tf > 0.0f) T += 0.6f * p->alpha_tf * mf_pow(fmaxf(v * v, 1e-20f), 1.6666667f) * p->h3;
        const float tilt = p->rcs[m][3];
        if (tilt != 0.0f) T += (-tilt) * yc * v * v * p->h3;
      }
      sn[lid * NR + n] = T;
      sn[lid * NR + n + 1] = VeK;
      sn[lid * NR + n + 2] = Vee;
      sn[lid * NR + n + 3] = dx;
      sn[lid * NR + n + 4] = dy;
      sn[lid * NR + n + 5] = dz;
    }
    for (int s = 64; s > 0; s >>= 1)
      for (int lid = 0; lid < s; ++lid)
        for (int x = 0; x < NR; ++x) sn[lid * NR + x] += sn[(lid + s) * NR + x];
    for (int x = 0; x < NR; ++x) part[wg * NR + x] = sn[x];
  }
  float* wgs = (float*)calloc((size_t)(128 * NR), sizeof(float));
  for (int lid = 0; lid < 128; ++lid)
    for (int64_t q = lid; q < nwg; q += 128)
      for (int x = 0; x < NR; ++x) wgs[lid * NR + x] += part[q * NR + x];
  for (int s = 64; s > 0; s >>= 1)
    for (int lid = 0; lid < s; ++lid)
      for (int x = 0; x < NR; ++x) wgs[lid * NR + x] += wgs[(lid + s) * NR + x];
  for (int x = 0; x < NR; ++x) sums[x] = wgs[x];
  free(wgs);
  free(part);
}

/* normalizeWGSL (mol_fast.js:474-492) */
void orc_mf_normalize(const orc_mf_params* p, float* U, const float* sums) {
  const int NN = p->NN, S = p->S;
  const int64_t S2 = (int64_t)S * S, S3 = S2 * S;
  for (int m = 0; m < p->n; ++m) {
    const float nrm = sums[m], tgt = p->rcs[m][1];
    if (!(nrm > 0.0f && tgt > 0.0f)) continue;
    const float sc = sqrtf(tgt / nrm);
    for (int i = 1; i < NN; ++i)
      for (int j = 1; j < NN; ++j)
        for (int k = 1; k < NN; ++k) U[m * S3 + i * S2 + (int64_t)j * S + k] *= sc;
  }
}

/* the per-electron V-cycle of doSteps (mol_fast.js:1262-1289) for electron m: rhoSource,
 * residualPm, restrict, cleared coarse error, coarse_iters weighted-Jacobi sweeps (ping-pong,
 * prolongation always reading buffer 0) and prolongCorrectPm (:645-785). */
void orc_mf_vcycle(const orc_mf_params* p, const float* U, float* P, int m, int coarse_iters) {
  const int NN = p->NN, S = p->S, NC = NN / 2, SC = NC + 1;
  const int64_t S2 = (int64_t)S * S, S3 = S2 * S, SC2 = (int64_t)SC * SC, SC3 = SC2 * SC;
  const float* Um = U + m * S3;
  float* Pm = P + m * S3;
  float* rho = (float*)malloc(sizeof(float) * S3);
  float* res = (float*)calloc((size_t)S3, sizeof(float));
  float* rhs = (float*)calloc((size_t)SC3, sizeof(float));
  float* E0 = (float*)calloc((size_t)SC3, sizeof(float));
  float* E1 = (float*)calloc((size_t)SC3, sizeof(float));
  for (int64_t id = 0; id < S3; ++id) rho[id] = Um[id] * Um[id];
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        const int64_t id = i * S2 + (int64_t)j * S + k;
        const float Pc = Pm[id];
        const float lap = (Pm[id + S2] + Pm[id - S2] + Pm[id + S] + Pm[id - S] + Pm[id + 1] + Pm[id - 1] - 6.0f * Pc) * p->inv_h2;
        res[id] = -p->two_pi * rho[id] - lap;
      }
#define MFF(a, b, c) res[(int64_t)(a) * S2 + (int64_t)(b) * S + (c)]
  for (int I = 1; I < NC; ++I)
    for (int J = 1; J < NC; ++J)
      for (int L = 1; L < NC; ++L) {
        const int fi = 2 * I, fj = 2 * J, fk = 2 * L;
        float val = 8.0f * MFF(fi, fj, fk);
        val += 4.0f * (MFF(fi + 1, fj, fk) + MFF(fi - 1, fj, fk) + MFF(fi, fj + 1, fk) + MFF(fi, fj - 1, fk) +
                       MFF(fi, fj, fk + 1) + MFF(fi, fj, fk - 1));
        val += 2.0f * (MFF(fi + 1, fj + 1, fk) + MFF(fi + 1, fj - 1, fk) + MFF(fi - 1, fj + 1, fk) + MFF(fi - 1, fj - 1, fk) +
                       MFF(fi + 1, fj, fk + 1) + MFF(fi + 1, fj, fk - 1) + MFF(fi - 1, fj, fk + 1) + MFF(fi - 1, fj, fk - 1) +
                       MFF(fi, fj + 1, fk + 1) + MFF(fi, fj + 1, fk - 1) + MFF(fi, fj - 1, fk + 1) + MFF(fi, fj - 1, fk - 1));
        val += MFF(fi + 1, fj + 1, fk + 1) + MFF(fi + 1, fj + 1, fk - 1) + MFF(fi + 1, fj - 1, fk + 1) +
               MFF(fi + 1, fj - 1, fk - 1) + MFF(fi - 1, fj + 1, fk + 1) + MFF(fi - 1, fj + 1, fk - 1) +
               MFF(fi - 1, fj - 1, fk + 1) + MFF(fi - 1, fj - 1, fk - 1);
        rhs[I * SC2 + (int64_t)J * SC + L] = val * 0.015625f;
      }
#undef MFF
  const float hc2 = 4.0f * p->h2;
  for (int cs = 0; cs < coarse_iters; ++cs) {
    const float* Ein = (cs % 2) ? E1 : E0;
    float* Eout = (cs % 2) ? E0 : E1;
    for (int I = 1; I < NC; ++I)
      for (int J = 1; J < NC; ++J)
        for (int L = 1; L < NC; ++L) {
          const int64_t c = I * SC2 + (int64_t)J * SC + L;
          const float sum = Ein[c + SC2] + Ein[c - SC2] + Ein[c + SC] + Ein[c - SC] + Ein[c + 1] + Ein[c - 1];
          Eout[c] = 0.3333f * Ein[c] + (sum + hc2 * rhs[c]) / 9.0f;
        }
  }
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        const int ci = i / 2, cj = j / 2, ck = k / 2;
        const int ci1 = ci + (i & 1) < NC ? ci + (i & 1) : NC;
        const int cj1 = cj + (j & 1) < NC ? cj + (j & 1) : NC;
        const int ck1 = ck + (k & 1) < NC ? ck + (k & 1) : NC;
        const float wi = (i & 1) ? 0.5f : 1.0f, wj = (j & 1) ? 0.5f : 1.0f, wk = (k & 1) ? 0.5f : 1.0f;
        const float wi1 = 1.0f - wi, wj1 = 1.0f - wj, wk1 = 1.0f - wk;
#define MFE(a, b, c) E0[(int64_t)(a) * SC2 + (int64_t)(b) * SC + (c)]
        float corr = 0.0f;
        corr += wi * wj * wk * MFE(ci, cj, ck);
        corr += wi * wj * wk1 * MFE(ci, cj, ck1);
        corr += wi * wj1 * wk * MFE(ci, cj1, ck);
        corr += wi * wj1 * wk1 * MFE(ci, cj1, ck1);
        corr += wi1 * wj * wk * MFE(ci1, cj, ck);
        corr += wi1 * wj * wk1 * MFE(ci1, cj, ck1);
        corr += wi1 * wj1 * wk * MFE(ci1, cj1, ck);
        corr += wi1 * wj1 * wk1 * MFE(ci1, cj1, ck1);
#undef MFE
        Pm[i * S2 + (int64_t)j * S + k] += 0.5f * corr;
      }
  free(rho); free(res); free(rhs); free(E0); free(E1);
}

/* forceWGSL (mol_fast.js:500-563): 2 Z <grad sum_m P_m> over the ball of radius 4 cells */
void orc_mf_force(const orc_mf_params* p, const float* P, float* F) {
  const int S = p->S, n = p->n;
  const int64_t S2 = (int64_t)S * S, S3 = S2 * S;
  const float inv2h = 0.5f * p->inv_h;
  for (int a = 0; a < n; ++a) {
    const float Z = p->atoms[a][3];
    if (Z <= 0.0f) { F[3 * a] = F[3 * a + 1] = F[3 * a + 2] = 0.0f; continue; }
    const int ci = (int)p->atoms[a][0], cj = (int)p->atoms[a][1], ck = (int)p->atoms[a][2];
    float sx = 0.0f, sy = 0.0f, sz = 0.0f, count = 0.0f;
    for (int di = -4; di <= 4; ++di) {
      const int ii = ci + di;
      if (ii < 1 || ii >= S - 1) continue;
      for (int dj = -4; dj <= 4; ++dj) {
        const int jj = cj + dj;
        if (jj < 1 || jj >= S - 1) continue;
        for (int dk = -4; dk <= 4; ++dk) {
          const int kk = ck + dk;
          if (kk < 1 || kk >= S - 1) continue;
          if ((float)(di * di + dj * dj + dk * dk) > 16.0f) continue;
          float xp = 0, xm = 0, yp = 0, ym = 0, zp = 0, zm = 0;
          for (int m = 0; m < n; ++m) {
            const float* Pm = P + m * S3;
            xp += Pm[(ii + 1) * S2 + (int64_t)jj * S + kk];
            xm += Pm[(ii - 1) * S2 + (int64_t)jj * S + kk];
            yp += Pm[ii * S2 + (int64_t)(jj + 1) * S + kk];
            ym += Pm[ii * S2 + (int64_t)(jj - 1) * S + kk];
            zp += Pm[ii * S2 + (int64_t)jj * S + kk + 1];
            zm += Pm[ii * S2 + (int64_t)jj * S + kk - 1];
          }
          sx += (xp - xm) * inv2h;
          sy += (yp - ym) * inv2h;
          sz += (zp - zm) * inv2h;
          count += 1.0f;
        }
      }
    }
    const float avg = count > 0.0f ? 1.0f / count : 0.0f;
    F[3 * a] = 2.0f * Z * sx * avg;
    F[3 * a + 1] = 2.0f * Z * sy * avg;
    F[3 * a + 2] = 2.0f * Z * sz * avg;
  }
}

/* recomputeK_WGSL (mol_fast.js:565-587) */
void orc_mf_recompute_k(const orc_mf_params* p, float* K) {
  const int S = p->S;
  const int64_t S2 = (int64_t)S * S, S3 = S2 * S;
#pragma omp parallel for schedule(static)
  for (int64_t id = 0; id < S3; ++id) {
    const int k = (int)(id % S), j = (int)((id / S) % S), i = (int)(id / S2);
    float Kv = 0.0f;
    for (int a = 0; a < p->n; ++a) {
      const float Z = p->atoms[a][3];
      if (Z <= 0.0f) continue;
      const float di = ((float)i - p->atoms[a][0]) * p->h, dj = ((float)j - p->atoms[a][1]) * p->h,
                  dk = ((float)k - p->atoms[a][2]) * p->h;
      Kv += Z / sqrtf(di * di + dj * dj + dk * dk + 4.0f * p->h2);
    }
    K[id] = Kv;
  }
}

/* extractWGSL (mol_fast.js:595-640) into out (3 n S^2 floats, zero-filled by the caller) */
void orc_mf_extract(const orc_mf_params* p, const float* U, const float* W, const float* Pv, float* out) {
  const int S = p->S, n = p->n, N2 = p->N2;
  const int64_t S2 = (int64_t)S * S, S3 = S2 * S, SS = S;
  for (int i = 0; i <= p->NN; ++i)
    for (int j = 0; j <= p->NN; ++j)
      for (int m = 0; m < n; ++m) {
        const int64_t idx2 = m * S3 + i * S2 + (int64_t)j * S + N2;
        out[m * SS * SS + i * SS + j] = W[idx2] > 0.1f ? U[idx2] : 0.0f;
        if (j == 0) {
          const int64_t line = i * S2 + (int64_t)N2 * S + N2, ml = m * S3 + line;
          out[n * SS * SS + m * SS + i] = U[ml];
          out[2 * n * SS * SS + m * SS + i] = W[ml];
          float Ps = 0.0f;
          for (int q = 0; q < n; ++q) Ps += Pv[q * S3 + line];
          if (m == 0) out[n * SS * SS + n * SS + i] = 2.0f * Ps;
          const float selfN = p->rcs[m][1];
          float Vp = 0.0f;
          if (selfN > 1.0f && p->alpha_tf > 0.0f) Vp = p->alpha_tf * mf_pow(fmaxf(U[ml] * U[ml], 1e-20f), 0.6666667f);
          out[n * SS * SS + (n + 1 + m) * SS + i] = Vp;
        }
      }
}

/* inSplit (mol_fast.js:878-939), JS numbers (f64); the axis is the raw USER_NUCLEI one */
static int mf_in_split_f64(double dx, double dy, double dz, double r, int split, int idx, const double* axr) {
  if (split == 0 || split == 1 || r < 1e-6) return 1;
  double L = sqrt(axr[0] * axr[0] + axr[1] * axr[1] + axr[2] * axr[2]);
  if (L == 0) L = 1;
  const double a0 = axr[0] / L, a1 = axr[1] / L, a2 = axr[2] / L;
  const double PI = 3.141592653589793;
  if (split == 2) {
    const double d = dx * a0 + dy * a1 + dz * a2;
    return idx == 0 ? d < 0 : d >= 0;
  }
  if (split == 3 || split == 5) {
    const double d = dx * a0 + dy * a1 + dz * a2;
    if (split == 5) {
      if (idx == 0) return d >= 0;
      if (d >= 0) return 0;
    }
    const double px = dx - d * a0, py = dy - d * a1, pz = dz - d * a2;
    double e1x, e1y, e1z;
    if (fabs(a2) < 0.9) { e1x = a1; e1y = -a0; e1z = 0; }
    else { e1x = 0; e1y = a2; e1z = -a1; }
    double e1L = sqrt(e1x * e1x + e1y * e1y + e1z * e1z);
    if (e1L == 0) e1L = 1;
    e1x /= e1L; e1y /= e1L; e1z /= e1L;
    const double e2x = a1 * e1z - a2 * e1y, e2y = a2 * e1x - a0 * e1z, e2z = a0 * e1y - a1 * e1x;
    const double pe1 = px * e1x + py * e1y + pz * e1z, pe2 = px * e2x + py * e2y + pz * e2z;
    double theta = atan2(pe2, pe1) - 0;
    if (theta < -PI) theta += 2 * PI;
    if (theta > PI) theta -= 2 * PI;
    const int sector = (int)fmod(floor((theta + PI) / (2 * PI / 3)), 3.0);
    return split == 3 ? sector == idx : sector == idx - 1;
  }
  if (split == 4) {
    static const double vs[4][3] = {{1, 1, 1}, {1, -1, -1}, {-1, 1, -1}, {-1, -1, 1}};
    const double u0 = dx / r, u1 = dy / r, u2 = dz / r;
    int best = 0;
    double bestDot = -INFINITY;
    for (int v = 0; v < 4; ++v) {
      const double d = vs[v][0] * u0 + vs[v][1] * u1 + vs[v][2] * u2;
      if (d > bestDot) { bestDot = d; best = v; }
    }
    return best == idx;
  }
  return 1;
}

/* uploadInitialData (mol_fast.js:941-1046) in JS numbers with f32 stores.  nuc: n records of 16
 * doubles {i, j, k, Z, rc, r_out, hs, z_init, norm_target, split, split_idx, ax0, ax1, ax2, -, -}. */
void orc_mf_init(int NN, double screen, int n, const double* nuc, float* K, float* U, float* W, float* P) {
  const int S = NN + 1;
  const int64_t S2 = (int64_t)S * S, S3 = S2 * S;
  const double hv = screen / NN, h2v = hv * hv, h3v = hv * hv * hv, soft = 4 * h2v, R_init = 3.0;
  const double midI0 = (nuc[0] + nuc[16 * (n - 1)]) / 2;
#pragma omp parallel for schedule(static)
  for (int i = 0; i <= NN; ++i)
    for (int j = 0; j <= NN; ++j)
      for (int k = 0; k <= NN; ++k) {
        const int64_t id = i * S2 + (int64_t)j * S + k;
        double Kacc = 0, rl[MF_MAX], ul[MF_MAX];
        int bestM = -1;
        double bestU = -1;
        for (int a = 0; a < n; ++a) {
          const double* c = nuc + 16 * a;
          const double dx = (i - c[0]) * hv, dy = (j - c[1]) * hv, dz = (k - c[2]) * hv;
          const double r_soft = sqrt(dx * dx + dy * dy + dz * dz + soft);
          const double r = sqrt(dx * dx + dy * dy + dz * dz);
          Kacc += c[3] / r_soft;
          const double z = c[7];
          const double uh = exp(-z * r);
          rl[a] = r; ul[a] = uh;
          const double tg = c[8] != 0 ? c[8] : 1;
          const double uw = sqrt(tg * z * z * z) * uh;
          const double roa = c[5];
          const int okR = !(roa > 0 && r > roa + hv);
          const double hs = c[6];
          const int okHS = hs == 0 || ((hs > 0) == (i > midI0));
          const int okS = mf_in_split_f64(dx, dy, dz, r, (int)c[9], (int)c[10], c + 11);
          if (okR && okHS && okS && uw > bestU) { bestU = uw; bestM = a; }
        }
        K[id] = (float)Kacc;
        for (int m = 0; m < n; ++m) {
          const double rc = nuc[16 * m + 4];
          double u = ul[m];
          if (rc > 0 && rl[m] < rc) {
            const double edge = rc - 3 * hv;
            const double t = fmax(0, fmin(1, (rl[m] - edge) / (rc - edge)));
            u *= t * t * (3 - 2 * t);
          }
          U[m * S3 + id] = (float)u;
          W[m * S3 + id] = 0.0f;
        }
        if (bestM >= 0 && rl[bestM] < R_init) {
          const double rc = nuc[16 * bestM + 4], ro = nuc[16 * bestM + 5];
          double w = 1.0;
          if (rc > 0 && rl[bestM] < rc) {
            const double edge = rc - 3 * hv;
            const double t = fmax(0, fmin(1, (rl[bestM] - edge) / (rc - edge)));
            w = t * t * (3 - 2 * t);
          }
          if (ro > 0 && rl[bestM] > ro + hv) w = 0;
          W[bestM * S3 + id] = (float)w;
        }
        for (int m = 0; m < n; ++m) P[m * S3 + id] = (float)(0.5 * nuc[16 * m + 3] / (rl[m] + h2v));
      }
  for (int m = 0; m < n; ++m) {
    double nrm = 0;
    for (int64_t id = 0; id < S3; ++id) nrm += (double)U[m * S3 + id] * (double)U[m * S3 + id];
    nrm *= h3v;
    const double tg = nuc[16 * m + 8];
    if (nrm > 0 && tg > 0) {
      const double sc = sqrt(tg / nrm);
      for (int64_t id = 0; id < S3; ++id) U[m * S3 + id] = (float)(U[m * S3 + id] * sc);
    }
  }
}

/* ======================================================================
 * realqm_rb.js red-black multi-field solver (realqm_rb.js:1-1222), f32 WGSL semantics
 *
 * One U, W, P field per electron (field m at offset m*S3), updated IN PLACE by red-black
 * colouring; exp is the f64 function rounded once to f32 (WGSL leaves its accuracy to the
 * implementation; the CUDA side does the same).
 * ==================================================================== */

typedef struct {
  int32_t NN, S, N2, n;   /* n electrons */
  float h, h2, inv_h, inv_h2, dt, half_d, two_pi, h3;
  float tgt[MF_MAX];      /* occupation (norm target) per electron */
} orc_rb_params;

/* rhoTotal (realqm_rb.js:190-215) and uNearest (:225-251): rho = u0^2 + u1^2 + ... and, per
 * electron, the max of the other electrons' u in index order, at every interior cell */
void orc_rb_rho_nearest(const orc_rb_params* p, const float* U, float* rho, float* unear) {
  const int NN = p->NN, S = p->S, n = p->n;
  const int64_t S2 = (int64_t)S * S, S3 = S2 * S;
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        const int64_t id = i * S2 + (int64_t)j * S + k;
        float r = U[id] * U[id];
        for (int m = 1; m < n; ++m) r = r + U[m * S3 + id] * U[m * S3 + id];
        rho[id] = r;
        for (int m = 0; m < n; ++m) {
          int first = 1;
          float v = 0.0f;
          for (int q = 0; q < n; ++q) {
            if (q == m) continue;
            const float u = U[q * S3 + id];
            if (first) { v = u; first = 0; }
            else v = fmaxf(v, u);
          }
          unear[m * S3 + id] = v;
        }
      }
}

/* fusedWU_RB_WGSL (realqm_rb.js:256-311) for electron m on the cells of one colour, in place */
void orc_rb_wu(const orc_rb_params* p, int m, int color, float* U, float* W, const float* unear, const float* K,
               const float* P, const float* mask) {
  const int NN = p->NN, S = p->S;
  const int64_t S2 = (int64_t)S * S, S3 = S2 * S;
  float* u = U + m * S3;
  float* w = W + m * S3;
  const float* un = unear + m * S3;
  const float* Pm = P + m * S3;
  const float* mk = mask + m * S3;
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        if ((i + j + k) % 2 != color) continue;
        const int64_t id = i * S2 + (int64_t)j * S + k;
        const float c = 0.1f * (u[id] - un[id]);
        const float wc = w[id];
        const float lap_w = w[id + S2] + w[id - S2] + w[id + S] + w[id - S] + w[id + 1] + w[id - 1] - 6.0f * wc;
        const float gwx = (w[id + S2] - w[id - S2]) * p->inv_h;
        const float gwy = (w[id + S] - w[id - S]) * p->inv_h;
        const float gwz = (w[id + 1] - w[id - 1]) * p->inv_h;
        const float grad_w = sqrtf(gwx * gwx + gwy * gwy + gwz * gwz);
        w[id] = wc + 0.5f * p->dt * fabsf(c) * lap_w * p->inv_h2 + 10.0f * p->dt * c * grad_w;
        const float wc2 = w[id];
        const float uc = u[id];
        const float fxp = (u[id + S2] - uc) * (w[id + S2] + wc2) * 0.5f;
        const float fxm = (uc - u[id - S2]) * (wc2 + w[id - S2]) * 0.5f;
        const float fyp = (u[id + S] - uc) * (w[id + S] + wc2) * 0.5f;
        const float fym = (uc - u[id - S]) * (wc2 + w[id - S]) * 0.5f;
        const float fzp = (u[id + 1] - uc) * (w[id + 1] + wc2) * 0.5f;
        const float fzm = (uc - u[id - 1]) * (wc2 + w[id - 1]) * 0.5f;
        const float wlap = (fxp - fxm) + (fyp - fym) + (fzp - fzm);
        const float u_new = uc + p->half_d * wlap + p->dt * (K[id] - 2.0f * Pm[id]) * uc * wc2;
        u[id] = u_new * mk[id];
        w[id] = w[id] * mk[id];
      }
}

/* updateP_RB_WGSL (realqm_rb.js:318-353) for electron m on the cells of one colour, in place */
void orc_rb_p(const orc_rb_params* p, int m, int color, float* P, const float* U, const float* rho) {
  const int NN = p->NN, S = p->S;
  const int64_t S2 = (int64_t)S * S, S3 = S2 * S;
  float* Pm = P + m * S3;
  const float* u = U + m * S3;
  const float selfN = p->tgt[m];
  const float selfFrac = selfN > 1.0f ? 1.0f / selfN : 1.0f;
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        if ((i + j + k) % 2 != color) continue;
        const int64_t id = i * S2 + (int64_t)j * S + k;
        const float Pc = Pm[id];
        const float lap = Pm[id + S2] + Pm[id - S2] + Pm[id + S] + Pm[id - S] + Pm[id + 1] + Pm[id - 1] - 6.0f * Pc;
        const float us = u[id];
        const float ro = fmaxf(rho[id] - selfFrac * us * us, 0.0f);
        Pm[id] = Pc + p->dt * (lap * p->inv_h2 + p->two_pi * ro);
      }
}

/* reduceNormWGSL + normalizeWGSL (realqm_rb.js:356-422) for electron m: nwg workgroups of 128
 * threads, each thread a grid-stride f32 sum over the interior, the workgroup tree, then the
 * sequential f32 sum of the partials and the scale sqrt(tgt / norm).  Returns the norm. */
float orc_rb_normalize(const orc_rb_params* p, int m, float* U) {
  const int NN = p->NN, S = p->S;
  const int64_t S2 = (int64_t)S * S, S3 = S2 * S;
  const int64_t NM = NN - 1, tot = NM * NM * NM;
  int64_t nwg = (tot + 127) / 128;
  if (nwg > 256) nwg = 256;
  const int64_t stride = nwg * 128;
  float* u = U + m * S3;
  float part[256];
  for (int64_t wg = 0; wg < nwg; ++wg) {
    float sd[128];
    for (int lid = 0; lid < 128; ++lid) {
      float acc = 0.0f;
      for (int64_t cell = wg * 128 + lid; cell < tot; cell += stride) {
        const int k = (int)(cell % NM) + 1, j = (int)((cell / NM) % NM) + 1, i = (int)(cell / (NM * NM)) + 1;
        const float v = u[i * S2 + (int64_t)j * S + k];
        acc += v * v * p->h3;
      }
      sd[lid] = acc;
    }
    for (int s = 64; s > 0; s >>= 1)
      for (int lid = 0; lid < s; ++lid) sd[lid] += sd[lid + s];
    part[wg] = sd[0];
  }
  float norm = 0.0f;
  for (int64_t q = 0; q < nwg; ++q) norm += part[q];
  if (norm > 0.0f) {
    const float sc = sqrtf(p->tgt[m] / norm);
    for (int i = 1; i < NN; ++i)
      for (int j = 1; j < NN; ++j)
        for (int k = 1; k < NN; ++k) u[i * S2 + (int64_t)j * S + k] *= sc;
  }
  return norm;
}

/* computeEnergy (realqm_rb.js:982-1045) in JS numbers (h, h3 the page's f64 spacing):
 * out = {E_T, E_eK, E_ee} */
void orc_rb_energy(const orc_rb_params* p, const float* U, const float* W, const float* P, const float* K, double h,
                   double h3, double* out) {
  const int NN = p->NN, S = p->S, n = p->n;
  const int64_t S2 = (int64_t)S * S, S3 = S2 * S;
  double ET = 0, EK = 0, EE = 0;
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        const int64_t id = i * S2 + (int64_t)j * S + k;
        for (int m = 0; m < n; ++m) {
          const float* u = U + m * S3;
          const float* w = W + m * S3;
          const double v = u[id], rho = v * v;
          if (w[id] > 0.1) {
            double g2 = 0;
            if (w[id + S2] > 0.1) { const double g = u[id + S2] - v; g2 += g * g; }
            if (w[id + S] > 0.1) { const double g = u[id + S] - v; g2 += g * g; }
            if (w[id + 1] > 0.1) { const double g = u[id + 1] - v; g2 += g * g; }
            ET += 0.5 * g2 * h;
          }
          EK += -(double)K[id] * rho * h3;
          EE += (double)P[m * S3 + id] * rho * h3;
        }
      }
  out[0] = ET; out[1] = EK; out[2] = EE;
}

/* the init shader (realqm_rb.js:104-186) run as runInitKernels does (:720-801): K accumulated
 * nucleus by nucleus (f32), then each electron's u, w, P on its Voronoi cell (at most 8 rivals),
 * split half and 3 bohr sphere.  nuc: nn records of 8 floats {i, j, k, Z, rc, ne, -, -};
 * enuc: the nucleus of each electron.  U, W, P, K are zero on entry. */
void orc_rb_init(const orc_rb_params* p, int nn, const float* nuc, const int32_t* enuc, float* K, float* U, float* W,
                 float* P) {
  const int NN = p->NN, S = p->S, n = p->n, N2 = p->N2;
  const int64_t S2 = (int64_t)S * S, S3 = S2 * S;
  for (int a = 0; a < nn; ++a) {
    const float* c = nuc + 8 * a;
    for (int i = 1; i < NN; ++i)
      for (int j = 1; j < NN; ++j)
        for (int k = 1; k < NN; ++k) {
          const float dx = ((float)i - c[0]) * p->h, dy = ((float)j - c[1]) * p->h, dz = ((float)k - c[2]) * p->h;
          const float r2 = dx * dx + dy * dy + dz * dz;
          K[i * S2 + (int64_t)j * S + k] += c[3] / sqrtf(r2 + 1.2f * p->h2);
        }
  }
  for (int m = 0; m < n; ++m) {
    const int a = enuc[m];
    const float* c = nuc + 8 * a;
    int sib = 0;
    for (int q = 0; q < m; ++q) sib += enuc[q] == a;
    const int splitDir = (int)c[5] == 1 ? 2 : (sib == 0 ? 0 : 1);
    float riv[8][3];
    int nriv = 0;
    for (int b = 0; b < nn && nriv < 8; ++b)
      if (b != a) { riv[nriv][0] = nuc[8 * b]; riv[nriv][1] = nuc[8 * b + 1]; riv[nriv][2] = nuc[8 * b + 2]; ++nriv; }
    for (int i = 1; i < NN; ++i)
      for (int j = 1; j < NN; ++j)
        for (int k = 1; k < NN; ++k) {
          const int64_t id = i * S2 + (int64_t)j * S + k;
          const float dx = ((float)i - c[0]) * p->h, dy = ((float)j - c[1]) * p->h, dz = ((float)k - c[2]) * p->h;
          const float r2 = dx * dx + dy * dy + dz * dz;
          const float r_soft = sqrtf(r2 + 1.2f * p->h2);
          const float r_au = sqrtf(r2);
          int inV = 1;
          for (int q = 0; q < nriv; ++q) {
            const float ex = ((float)i - riv[q][0]) * p->h, ey = ((float)j - riv[q][1]) * p->h,
                        ez = ((float)k - riv[q][2]) * p->h;
            if (r2 > ex * ex + ey * ey + ez * ez) inV = 0;
          }
          const int inRc = c[4] <= 0.0f || r_au < c[4];
          const int inSplit = splitDir == 2 ? 1 : (splitDir == 0 ? (unsigned)i < (unsigned)(N2 - 1) : (unsigned)i > (unsigned)(N2 + 1));
          const int inSph = r_au < 3.0f;
          if (inV && inSplit && inRc && inSph) W[m * S3 + id] = 1.0f;
          if (inV && inSplit && inSph) U[m * S3 + id] = (float)exp((double)(-0.5f * c[3] * r_soft));
          P[m * S3 + id] = 0.5f / r_soft;
        }
  }
}

/* extractSliceWGSL (realqm_rb.js:429-457): per pixel (i, j) of the k = N2 plane, u, w, P of every
 * electron then K; out has S*S*(3n+1) floats */
void orc_rb_slice(const orc_rb_params* p, const float* U, const float* W, const float* P, const float* K, float* out) {
  const int S = p->S, n = p->n, N1 = S;
  const int64_t S2 = (int64_t)S * S, S3 = S2 * S;
  const int stride = 3 * n + 1;
  for (int g = 0; g < N1 * N1; ++g) {
    const int j = g / N1, i = g % N1;
    const int64_t id = i * S2 + (int64_t)j * S + p->N2;
    for (int m = 0; m < n; ++m) {
      out[(int64_t)g * stride + 3 * m] = U[m * S3 + id];
      out[(int64_t)g * stride + 3 * m + 1] = W[m * S3 + id];
      out[(int64_t)g * stride + 3 * m + 2] = P[m * S3 + id];
    }
    out[(int64_t)g * stride + stride - 1] = K[id];
  }
}

/* ======================================================================
 * molecule.js LOBPCG frame (shaders molecule.js:1455-1724, host :3265-3740; the page's
 * useLOBPCG switch, off by default, :1751).  f32 shaders restated with the same operation
 * order; the Ritz solves are the page's double-precision JavaScript.
 * ==================================================================== */

/* applyH's own isInsideRc (molecule.js:1473-1477): only the label's own r_c sphere. */
static inline int lob_inside_rc(int ci, int cj, int ck, uint32_t lbl, const orc_mj_atom* atoms, float h) {
  const float rc = atoms[lbl].rc;
  if (rc <= 0.f) return 0;
  return mj_dist(ci, cj, ck, &atoms[lbl], h) < rc;
}

/* applyH (molecule.js:1483-1525): HU = -0.5*lap/h^2 + (-K + 2*Pother)*u on interior cells, 0 inside
 * the own r_c sphere; a neighbour of another label or inside its label's sphere counts as the
 * centre value (Neumann). */
void orc_lob_apply_h(const float* U, float* HU, const float* K, const uint32_t* label, const float* Pother,
                     const orc_mj_atom* atoms, int S, float h, float inv_h2) {
  const int NN = S - 1;
  const int64_t S2 = (int64_t)S * S;
#pragma omp parallel for schedule(static)
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        const int64_t id = IDX(i, j, k, S);
        const uint32_t L = label[id];
        if (lob_inside_rc(i, j, k, L, atoms, h)) { HU[id] = 0.f; continue; }
        const float uc = U[id];
        const uint32_t lip = label[id + S2], lim = label[id - S2], ljp = label[id + S], ljm = label[id - S];
        const uint32_t lkp = label[id + 1], lkm = label[id - 1];
        const float uip = (lip == L && !lob_inside_rc(i + 1, j, k, lip, atoms, h)) ? U[id + S2] : uc;
        const float uim = (lim == L && !lob_inside_rc(i - 1, j, k, lim, atoms, h)) ? U[id - S2] : uc;
        const float ujp = (ljp == L && !lob_inside_rc(i, j + 1, k, ljp, atoms, h)) ? U[id + S] : uc;
        const float ujm = (ljm == L && !lob_inside_rc(i, j - 1, k, ljm, atoms, h)) ? U[id - S] : uc;
        const float ukp = (lkp == L && !lob_inside_rc(i, j, k + 1, lkp, atoms, h)) ? U[id + 1] : uc;
        const float ukm = (lkm == L && !lob_inside_rc(i, j, k - 1, lkm, atoms, h)) ? U[id - 1] : uc;
        const float lap = uip + uim + ujp + ujm + ukp + ukm - 6.0f * uc;
        HU[id] = -0.5f * lap * inv_h2 + (-K[id] + 2.0f * Pother[id]) * uc;
      }
}

/* lobpcgInner + lobpcgFinalize (molecule.js:1535-1648): the 12 f32 inner products over the
 * cells of domain m -- <X|X> <X|HX> <W|W> <W|HW> <X|W> <X|HW> <P|P> <P|HP> <X|P> <X|HP> <W|P>
 * <W|HP>, each term a*b*h^3 -- summed in the shaders' order.  Interior cells are numbered with k
 * fastest; workgroup w (of nwg = min(256, ceil(cells/128))) thread l takes cells w*128+l, then
 * every nwg*128-th; the 128 per-thread sums of a workgroup fold pairwise (l += l+s for s = 64 ..
 * 1); the one finalize workgroup's thread l adds workgroup results l, l+128, .. in order and
 * folds the same way. */
#define LOB_NR 12
#define LOB_WG 128
void orc_lob_inner(const float* X, const float* HX, const float* W, const float* HW, const float* Pv,
                   const float* HP, const uint32_t* label, uint32_t m, int S, float h3, float* sums) {
  const int NM = S - 2;
  const int64_t tot = (int64_t)NM * NM * NM;
  const int nwg = (int)((tot + LOB_WG - 1) / LOB_WG) < 256 ? (int)((tot + LOB_WG - 1) / LOB_WG) : 256;
  const int64_t stride = (int64_t)nwg * LOB_WG;
  float* part = (float*)calloc((size_t)nwg * LOB_NR, sizeof(float));
#pragma omp parallel for schedule(static)
  for (int w = 0; w < nwg; ++w) {
    float sn[LOB_WG][LOB_NR];
    for (int l = 0; l < LOB_WG; ++l) {
      for (int q = 0; q < LOB_NR; ++q) sn[l][q] = 0.f;
      for (int64_t cell = (int64_t)w * LOB_WG + l; cell < tot; cell += stride) {
        const int k = (int)(cell % NM) + 1, j = (int)((cell / NM) % NM) + 1, i = (int)(cell / ((int64_t)NM * NM)) + 1;
        const int64_t id = IDX(i, j, k, S);
        if (label[id] != m) continue;
        const float x = X[id], hx = HX[id], wv = W[id], hw = HW[id], pv = Pv[id], hp = HP[id];
        sn[l][0] += x * x * h3;
        sn[l][1] += x * hx * h3;
        sn[l][2] += wv * wv * h3;
        sn[l][3] += wv * hw * h3;
        sn[l][4] += x * wv * h3;
        sn[l][5] += x * hw * h3;
        sn[l][6] += pv * pv * h3;
        sn[l][7] += pv * hp * h3;
        sn[l][8] += x * pv * h3;
        sn[l][9] += x * hp * h3;
        sn[l][10] += wv * pv * h3;
        sn[l][11] += wv * hp * h3;
      }
    }
    for (int s = LOB_WG / 2; s > 0; s >>= 1)
      for (int l = 0; l < s; ++l)
        for (int q = 0; q < LOB_NR; ++q) sn[l][q] += sn[l + s][q];
    for (int q = 0; q < LOB_NR; ++q) part[(size_t)w * LOB_NR + q] = sn[0][q];
  }
  float wg[LOB_WG][LOB_NR];
  for (int l = 0; l < LOB_WG; ++l) {
    for (int q = 0; q < LOB_NR; ++q) wg[l][q] = 0.f;
    for (int w = l; w < nwg; w += LOB_WG)
      for (int q = 0; q < LOB_NR; ++q) wg[l][q] += part[(size_t)w * LOB_NR + q];
  }
  for (int s = LOB_WG / 2; s > 0; s >>= 1)
    for (int l = 0; l < s; ++l)
      for (int q = 0; q < LOB_NR; ++q) wg[l][q] += wg[l + s][q];
  for (int q = 0; q < LOB_NR; ++q) sums[q] = wg[0][q];
  free(part);
}

/* lobpcgResidual (molecule.js:1652-1689): W = (HX - lambda*X) / (3/h^2 + |-K + 2*Pother| + 0.1) on
 * domain m, 0 on every other interior cell. */
void orc_lob_residual(const float* X, const float* HX, float* W, const uint32_t* label, const float* K,
                      const float* Pot, float lam, uint32_t m, int S, float inv_h2) {
  const int NN = S - 1;
#pragma omp parallel for schedule(static)
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        const int64_t id = IDX(i, j, k, S);
        if (label[id] != m) { W[id] = 0.f; continue; }
        const float r = HX[id] - lam * X[id];
        const float vEff = fabsf(-K[id] + 2.0f * Pot[id]);
        const float diagH = 3.0f * inv_h2 + vEff + 0.1f;
        W[id] = r / diagH;
      }
}

/* lobpcgUpdate (molecule.js:1693-1724): on domain m, X = c0*X + c1*W + c2*P and P = c1*W + c2*P. */
void orc_lob_update(float* X, const float* W, float* Pv, const uint32_t* label, float c0, float c1, float c2,
                    uint32_t m, int S) {
  const int NN = S - 1;
#pragma omp parallel for schedule(static)
  for (int i = 1; i < NN; ++i)
    for (int j = 1; j < NN; ++j)
      for (int k = 1; k < NN; ++k) {
        const int64_t id = IDX(i, j, k, S);
        if (label[id] != m) continue;
        const float x = X[id], w = W[id], pv = Pv[id];
        X[id] = c0 * x + c1 * w + c2 * pv;
        Pv[id] = c1 * w + c2 * pv;
      }
}

/* Math.min / Math.max of JavaScript: NaN if either argument is NaN, -0 below +0. */
static double js_min(double a, double b) {
  if (a != a || b != b) return NAN;
  if (a < b) return a;
  if (b < a) return b;
  return signbit(a) ? a : b;
}
static double js_max(double a, double b) {
  if (a != a || b != b) return NAN;
  if (a > b) return a;
  if (b > a) return b;
  return signbit(a) ? b : a;
}

/* solveRitz2x2 (molecule.js:3265-3295): the smaller root of det(H - lambda S) = 0 over span{X, W},
 * its vector scaled to c'Sc = 1.  ip = the 12 sums; out = {lambda, c0, c1, c2}. */
void orc_lob_ritz2(const double* ip, double* out) {
  const double a11 = ip[1], a12 = ip[5], a22 = ip[3];
  const double s11 = ip[0], s12 = ip[4], s22 = ip[2];
  const double A = s11 * s22 - s12 * s12;
  const double B = -(a11 * s22 + a22 * s11 - 2 * a12 * s12);
  const double Cq = a11 * a22 - a12 * a12;
  const double disc = B * B - 4 * A * Cq;
  const double sq = sqrt(js_max(0, disc));
  const double lam1 = (-B - sq) / (2 * A), lam2 = (-B + sq) / (2 * A);
  const double lam = js_min(lam1, lam2);
  const double r1 = a11 - lam * s11, r2 = a12 - lam * s12;
  double c0, c1;
  if (fabs(r1) > fabs(r2)) {
    c1 = 1;
    c0 = -r2 / r1;
  } else if (fabs(r2) > 1e-15) {
    c0 = 1;
    c1 = -r1 / r2;
  } else {
    c0 = 1;
    c1 = 0;
  }
  const double norm2 = c0 * c0 * s11 + 2 * c0 * c1 * s12 + c1 * c1 * s22;
  const double inv = 1 / sqrt(js_max(1e-30, norm2));
  out[0] = lam;
  out[1] = c0 * inv;
  out[2] = c1 * inv;
  out[3] = 0;
}

/* solveRitz3x3 (molecule.js:3297-3388) over span{X, W, P}: Cholesky S = L L', the standard problem
 * L^-1 H L^-T by 20 sweeps of cyclic Jacobi rotations, the smallest diagonal entry, c = L^-T y;
 * the 2x2 solve when the Cholesky factor is not finite or has a diagonal below 1e-15. */
void orc_lob_ritz3(const double* ip, double* out) {
  const double S[3][3] = {{ip[0], ip[4], ip[8]}, {ip[4], ip[2], ip[10]}, {ip[8], ip[10], ip[6]}};
  const double H[3][3] = {{ip[1], ip[5], ip[9]}, {ip[5], ip[3], ip[11]}, {ip[9], ip[11], ip[7]}};
  double L[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  L[0][0] = sqrt(js_max(1e-30, S[0][0]));
  L[1][0] = S[1][0] / L[0][0];
  L[2][0] = S[2][0] / L[0][0];
  L[1][1] = sqrt(js_max(1e-30, S[1][1] - L[1][0] * L[1][0]));
  L[2][1] = (S[2][1] - L[2][0] * L[1][0]) / L[1][1];
  L[2][2] = sqrt(js_max(1e-30, S[2][2] - L[2][0] * L[2][0] - L[2][1] * L[2][1]));
  if (!isfinite(L[2][2]) || L[0][0] < 1e-15 || L[1][1] < 1e-15 || L[2][2] < 1e-15) {
    orc_lob_ritz2(ip, out);
    return;
  }
  double Li[3][3] = {{1 / L[0][0], 0, 0}, {0, 1 / L[1][1], 0}, {0, 0, 1 / L[2][2]}};
  Li[1][0] = -L[1][0] * Li[0][0] * Li[1][1];
  Li[2][0] = -(L[2][0] * Li[0][0] + L[2][1] * Li[1][0]) * Li[2][2];
  Li[2][1] = -L[2][1] * Li[1][1] * Li[2][2];
  double Bm[3][3], A[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += H[i][k] * Li[j][k];
      Bm[i][j] = s;
    }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += Li[i][k] * Bm[k][j];
      A[i][j] = s;
    }
  double V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  static const int PQ[3][2] = {{0, 1}, {0, 2}, {1, 2}};
  for (int sweep = 0; sweep < 20; ++sweep)
    for (int e = 0; e < 3; ++e) {
      const int p = PQ[e][0], q = PQ[e][1];
      const double apq = A[p][q];
      if (fabs(apq) < 1e-15) continue;
      const double tau = (A[q][q] - A[p][p]) / (2 * apq);
      const double t = (tau >= 0 ? 1 : -1) / (fabs(tau) + sqrt(1 + tau * tau));
      const double c = 1 / sqrt(1 + t * t);
      const double s = t * c;
      const double app = A[p][p], aqq = A[q][q];
      A[p][p] = c * c * app - 2 * s * c * apq + s * s * aqq;
      A[q][q] = s * s * app + 2 * s * c * apq + c * c * aqq;
      A[p][q] = 0;
      A[q][p] = 0;
      for (int r = 0; r < 3; ++r) {
        if (r == p || r == q) continue;
        const double arp = A[r][p], arq = A[r][q];
        A[r][p] = c * arp - s * arq;
        A[p][r] = A[r][p];
        A[r][q] = s * arp + c * arq;
        A[q][r] = A[r][q];
      }
      for (int r = 0; r < 3; ++r) {
        const double vrp = V[r][p], vrq = V[r][q];
        V[r][p] = c * vrp - s * vrq;
        V[r][q] = s * vrp + c * vrq;
      }
    }
  int mi = 0;
  if (A[1][1] < A[mi][mi]) mi = 1;
  if (A[2][2] < A[mi][mi]) mi = 2;
  const double y0 = V[0][mi], y1 = V[1][mi], y2 = V[2][mi];
  out[0] = A[mi][mi];
  out[1] = Li[0][0] * y0 + Li[1][0] * y1 + Li[2][0] * y2;
  out[2] = Li[1][1] * y1 + Li[2][1] * y2;
  out[3] = Li[2][2] * y2;
}
