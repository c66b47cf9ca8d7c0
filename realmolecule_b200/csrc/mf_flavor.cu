// mf_flavor.cu -- the mol_fast.js multi-field solver (rq_mf_*): one U (density amplitude), W
// (front) and P (Hartree potential of its own density) field per electron, one electron per
// nucleus, all fields double-buffered (mol_fast.js:1-1651).
//
// The reference dispatches one invocation per (cell, electron) and re-reads every other
// electron's U and P at the cell.  Here one thread owns a cell and walks the electrons: the
// cross-electron terms (the competitor max, sum_n P_n, the split-group sum) come from one read
// of each field at the cell, and the per-electron stencils follow.  All f32 arithmetic is the
// shaders' own operation order with explicit round-to-nearest operations (no contraction).
// The norm/energy reduction keeps the reference's 128-cell workgroup trees and its single
// finalize workgroup, so the f32 sums (and every normalisation scale) are the reference's.
// The two-level Poisson correction runs for all electrons at once (per-electron scratch);
// each electron's correction depends only on its own fields, as in the sequential loop.
// The initial state (uploadInitialData) is computed on the device in FP64 with f32 stores.
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "../../include/rq.h"
#include "rq_internal.cuh"

namespace rq {

constexpr int kMfMax = 16;

struct MfParams {  // writeParams (mol_fast.js:838-874) plus the constants templated into the shaders
  int NN, S, N2, n, shell_mode, any_rc;
  float h, h2, inv_h, inv_h2, dt, half_d, h3, two_pi;
  float R_out, field_x, alpha_tf, full_self;
  float kc, kc_multi, beta, pad1;
  float4 atoms[kMfMax];  // i, j, k, Z
  float4 rcs[kMfMax];    // rc, norm target, tilt_x, tilt_y
  float r_out[kMfMax];
  int split_type[kMfMax], split_idx[kMfMax], split_fix[kMfMax], split_group[kMfMax];
  float4 ax[kMfMax];
  // per-electron constants of the shaders, formed on the host with the same f32 operations:
  // upd = (fm, half_d * k_mult, 1 if the Thomas-Fermi term is on, tilt_x) of updateWGSL,
  // red = (fm without USER_FULL_SELF, k_mult * KINETIC_COEFF, same flag, tilt_y) of reduceWGSL
  float4 upd[kMfMax], red[kMfMax];
  unsigned gmask[kMfMax];  // bit q set: electron q is in this electron's split group
};

constexpr int kMfNucLen = 16;  // doubles per nucleus record of the initialiser

// WGSL leaves the accuracy of pow and atan2 to the implementation; both sides of the parity
// tests use the f64 function rounded once to f32 (within an f32 ulp of the exact value)
__device__ __forceinline__ float mf_pow(float x, float y) { return (float)pow((double)x, (double)y); }
__device__ __forceinline__ float mf_atan2(float y, float x) { return (float)atan2((double)y, (double)x); }

__device__ __forceinline__ float mf_cusp(float r, float rc, float h) {  // mol_fast.js:188-193
  const float edge = F_SUB(rc, F_MUL(3.0f, h));
  const float t = fminf(fmaxf(F_DIV(F_SUB(r, edge), F_SUB(rc, edge)), 0.0f), 1.0f);
  return F_MUL(F_MUL(t, t), F_SUB(3.0f, F_MUL(2.0f, t)));
}

__device__ __forceinline__ float mf_dot(float4 a, float x, float y, float z) {
  return F_ADD(F_ADD(F_MUL(a.x, x), F_MUL(a.y, y)), F_MUL(a.z, z));
}

// the three-sector index around ax (mol_fast.js:206-216)
__device__ unsigned mf_third_sector(float4 ax, float x, float y, float z) {
  const float d = mf_dot(ax, x, y, z);
  const float px = F_SUB(x, F_MUL(d, ax.x)), py = F_SUB(y, F_MUL(d, ax.y)), pz = F_SUB(z, F_MUL(d, ax.z));
  float e1x, e1y, e1z;
  if (fabsf(ax.z) < 0.9f) { e1x = ax.y; e1y = -ax.x; e1z = 0.0f; }
  else { e1x = 0.0f; e1y = ax.z; e1z = -ax.y; }
  const float L = F_SQRT(F_ADD(F_ADD(F_MUL(e1x, e1x), F_MUL(e1y, e1y)), F_MUL(e1z, e1z)));
  e1x = F_DIV(e1x, L); e1y = F_DIV(e1y, L); e1z = F_DIV(e1z, L);
  const float e2x = F_SUB(F_MUL(ax.y, e1z), F_MUL(ax.z, e1y));
  const float e2y = F_SUB(F_MUL(ax.z, e1x), F_MUL(ax.x, e1z));
  const float e2z = F_SUB(F_MUL(ax.x, e1y), F_MUL(ax.y, e1x));
  const float pe2 = F_ADD(F_ADD(F_MUL(px, e2x), F_MUL(py, e2y)), F_MUL(pz, e2z));
  const float pe1 = F_ADD(F_ADD(F_MUL(px, e1x), F_MUL(py, e1y)), F_MUL(pz, e1z));
  float theta = F_SUB(mf_atan2(pe2, pe1), 0.0f);
  if (theta < -3.141592653589793f) theta = F_ADD(theta, 6.283185307179586f);
  if (theta > 3.141592653589793f) theta = F_SUB(theta, 6.283185307179586f);
  return ((unsigned)floorf(F_DIV(F_ADD(theta, 3.141592653589793f), 2.094395102393195f))) % 3u;
}

// SHELL_MODE angular split (mol_fast.js:196-246); (x, y, z) in grid cells from the nucleus
__device__ bool mf_in_sector(const MfParams* __restrict__ p, int m, float x, float y, float z, float r_m) {
  const int t = p->split_type[m];
  const unsigned sidx = (unsigned)p->split_idx[m];
  const float4 ax = p->ax[m];
  if (t == 2) {
    const float d = mf_dot(ax, x, y, z);
    return sidx == 0u ? d < 0.0f : d >= 0.0f;
  }
  if (t == 3) return mf_third_sector(ax, x, y, z) == sidx;
  if (t == 4) {
    if (r_m > 1e-6f) {
      const float ux = F_DIV(x, r_m), uy = F_DIV(y, r_m), uz = F_DIV(z, r_m);
      unsigned best = 0;
      float bestD = F_ADD(F_ADD(F_MUL(1.0f, ux), F_MUL(1.0f, uy)), F_MUL(1.0f, uz));
      const float d1 = F_ADD(F_ADD(F_MUL(1.0f, ux), F_MUL(-1.0f, uy)), F_MUL(-1.0f, uz));
      if (d1 > bestD) { bestD = d1; best = 1; }
      const float d2 = F_ADD(F_ADD(F_MUL(-1.0f, ux), F_MUL(1.0f, uy)), F_MUL(-1.0f, uz));
      if (d2 > bestD) { bestD = d2; best = 2; }
      const float d3 = F_ADD(F_ADD(F_MUL(-1.0f, ux), F_MUL(-1.0f, uy)), F_MUL(1.0f, uz));
      if (d3 > bestD) { bestD = d3; best = 3; }
      return best == sidx;
    }
    return true;
  }
  if (t == 5) {
    const float d = mf_dot(ax, x, y, z);
    if (sidx == 0u) return d >= 0.0f;
    if (d >= 0.0f) return false;
    return mf_third_sector(ax, x, y, z) == sidx - 1u;
  }
  return true;
}

constexpr int kMfTK = 32, kMfTJ = 8;


// updateWGSL (mol_fast.js:134-351) for every electron of one interior cell.  One thread owns a
// cell: the cross-electron terms (sum_q P_q, the competitor max) come from one read of each
// electron's U and P at the cell.  The competitor max over the other electrons is the largest U
// of the cell unless this electron holds it (then the second largest): both are exact
// selections, equal to the shader's sequential scan.  The register cap (4 blocks of 256 per SM)
// lets the per-electron stencil loads of enough warps overlap; the kernel is bound by the
// instruction issue of the unfused f32 arithmetic, not by DRAM.
template <int NMAX, bool SHELL>
__global__ void __launch_bounds__(256, 4) k_mf_update(const MfParams* __restrict__ p, const float* __restrict__ Ui,
                                                      const float* __restrict__ Wi, const float* __restrict__ Pi,
                                                      const float* __restrict__ K, float* __restrict__ Uo,
                                                      float* __restrict__ Wo, float* __restrict__ Po) {
  const int NN = p->NN;
  const int k = blockIdx.x * kMfTK + threadIdx.x + 1;
  const int j = blockIdx.y * kMfTJ + threadIdx.y + 1;
  const int i = blockIdx.z + 1;
  if (k >= NN || j >= NN) return;
  const long long S = p->S, S2 = S * S, S3 = S2 * S;
  const long long id = (long long)i * S2 + (long long)j * S + k;
  const int n = p->n;
  float Ptot = 0.0f, max1 = 0.0f, max2 = 0.0f;
  int arg1 = -1;
#pragma unroll
  for (int q = 0; q < NMAX; ++q)
    if (q < n) {
      Ptot = F_ADD(Ptot, __ldg(Pi + q * S3 + id));
      const float u = __ldg(Ui + q * S3 + id);
      if (u > max1) { max2 = max1; max1 = u; arg1 = q; }
      else if (u > max2) max2 = u;
    }
  const float h = p->h, dt = p->dt, inv_h = p->inv_h, inv_h2 = p->inv_h2;
  // frozen-core mode: the rc cusps of all nuclei act on every electron's front; min is exact,
  // so the cap over the nuclei is taken once per cell (mol_fast.js:249-262)
  float cap = 2.0f;
  if (!SHELL && p->any_rc) {
    for (int a = 0; a < n; ++a) {
      const float4 at = p->atoms[a];
      const float rc_a = p->rcs[a].x;
      const float dx = F_SUB((float)i, at.x), dy = F_SUB((float)j, at.y), dz = F_SUB((float)k, at.z);
      const float r = F_MUL(F_SQRT(F_ADD(F_ADD(F_MUL(dx, dx), F_MUL(dy, dy)), F_MUL(dz, dz))), h);
      if (rc_a > 0.0f && r < rc_a) cap = fminf(cap, mf_cusp(r, rc_a, h));
    }
  }
  const float Kc = __ldg(K + id);
  const float x_au = F_MUL(F_SUB((float)i, (float)p->N2), h);
  const float y_au = F_MUL(F_SUB((float)j, (float)p->N2), h);
  const float beta = p->beta, two_pi_dt = F_MUL(p->two_pi, dt), fxx = F_MUL(p->field_x, x_au);
  const float dt005 = F_MUL(0.05f, dt), dt1 = F_MUL(1.0f, dt);
  const int s1 = (int)S, s2 = (int)S2;  // stencil offsets within one field (S^3 < 2^31)
#pragma unroll 1
  for (int m = 0; m < n; ++m) {
    const long long o = m * S3 + id;
    const float* __restrict__ u = Ui + o;
    const float* __restrict__ w = Wi + o;
    const float* __restrict__ pp = Pi + o;
    const float uc = __ldg(u), wc = __ldg(w), Pc = __ldg(pp);
    const float wip = __ldg(w + s2), wim = __ldg(w - s2), wjp = __ldg(w + s1), wjm = __ldg(w - s1);
    const float wkp = __ldg(w + 1), wkm = __ldg(w - 1);
    const float uip = __ldg(u + s2), uim = __ldg(u - s2), ujp = __ldg(u + s1), ujm = __ldg(u - s1);
    const float ukp = __ldg(u + 1), ukm = __ldg(u - 1);
    const float pip = __ldg(pp + s2), pim = __ldg(pp - s2), pjp = __ldg(pp + s1), pjm = __ldg(pp - s1);
    const float pkp = __ldg(pp + 1), pkm = __ldg(pp - 1);
    const float4 cu = p->upd[m];
    const float tilt_y = p->rcs[m].w;
    const unsigned gm = p->gmask[m];
    const float umax = m == arg1 ? max2 : max1;
    float Pgrp, rho_other = 0.0f;
    if (gm == (1u << m)) {  // no split siblings: the group sum is this electron's own P
      Pgrp = F_ADD(0.0f, Pc);
    } else {
      Pgrp = 0.0f;
      for (int q = 0; q < n; ++q)
        if ((gm >> q) & 1u) Pgrp = F_ADD(Pgrp, __ldg(Pi + q * S3 + id));
    }
    if (beta != 0.0f) {  // V_Pauli; with beta = 0 it is 0 * (a finite sum of squares) = 0
      for (int q = 0; q < n; ++q)
        if (q != m) {
          const float un = __ldg(Ui + q * S3 + id);
          rho_other = F_ADD(rho_other, F_MUL(un, un));
        }
    }
    const float cm = F_SUB(uc, umax);
    const float lw =
        F_MUL(F_SUB(F_ADD(F_ADD(F_ADD(F_ADD(F_ADD(wip, wim), wjp), wjm), wkp), wkm), F_MUL(6.0f, wc)), inv_h2);
    const float gx = F_MUL(F_SUB(wip, wim), inv_h), gy = F_MUL(F_SUB(wjp, wjm), inv_h),
                gz = F_MUL(F_SUB(wkp, wkm), inv_h);
    float nw = F_ADD(F_ADD(wc, F_MUL(F_MUL(dt005, fabsf(cm)), lw)),
                     F_MUL(F_MUL(dt1, cm), F_SQRT(F_ADD(F_ADD(F_MUL(gx, gx), F_MUL(gy, gy)), F_MUL(gz, gz)))));
    nw = fminf(fmaxf(nw, 0.0f), 1.0f);
    if (SHELL) {
      const float4 at = p->atoms[m];
      const float rc_m = p->rcs[m].x;
      const float ro_m = F_MUL(p->r_out[m], p->R_out);
      const float dxm = F_SUB((float)i, at.x), dym = F_SUB((float)j, at.y), dzm = F_SUB((float)k, at.z);
      const float r_m = F_MUL(F_SQRT(F_ADD(F_ADD(F_MUL(dxm, dxm), F_MUL(dym, dym)), F_MUL(dzm, dzm))), h);
      if (rc_m > 0.0f && r_m < rc_m) nw = fminf(nw, mf_cusp(r_m, rc_m, h));
      if (ro_m > 0.0f && r_m > ro_m) nw = (r_m <= F_ADD(ro_m, h)) ? nw : 0.0f;
      if (p->split_type[m] != 0 && p->split_fix[m] == 1 && !mf_in_sector(p, m, dxm, dym, dzm, r_m)) nw = 0.0f;
    } else if (cap <= 1.0f) {
      nw = fminf(nw, cap);
    }
    Wo[o] = nw;
    const float Vother = F_MUL(2.0f, F_SUB(Ptot, F_MUL(cu.x, Pgrp)));
    const float V_TF = cu.z != 0.0f ? F_MUL(p->alpha_tf, mf_pow(fmaxf(F_MUL(uc, uc), 1e-20f), 0.6666667f)) : 0.0f;
    const float V_tilt = F_SUB(F_MUL(-cu.w, x_au), F_MUL(tilt_y, y_au));
    const float V_Pauli = F_MUL(beta, rho_other);
    const float hd = cu.y;
    const float fx = F_SUB(F_MUL(F_MUL(F_SUB(uip, uc), F_ADD(wip, nw)), 0.5f), F_MUL(F_MUL(F_SUB(uc, uim), F_ADD(nw, wim)), 0.5f));
    const float fy = F_SUB(F_MUL(F_MUL(F_SUB(ujp, uc), F_ADD(wjp, nw)), 0.5f), F_MUL(F_MUL(F_SUB(uc, ujm), F_ADD(nw, wjm)), 0.5f));
    const float fz = F_SUB(F_MUL(F_MUL(F_SUB(ukp, uc), F_ADD(wkp, nw)), 0.5f), F_MUL(F_MUL(F_SUB(uc, ukm), F_ADD(nw, wkm)), 0.5f));
    const float pot = F_SUB(F_SUB(F_SUB(F_SUB(F_SUB(Kc, Vother), V_TF), V_tilt), V_Pauli), fxx);
    Uo[o] = F_ADD(F_ADD(F_ADD(F_ADD(uc, F_MUL(hd, fx)), F_MUL(hd, fy)), F_MUL(hd, fz)),
                  F_MUL(F_MUL(F_MUL(dt, pot), uc), wc));
    const float lap = F_SUB(F_ADD(F_ADD(F_ADD(F_ADD(F_ADD(pip, pim), pjp), pjm), pkp), pkm), F_MUL(6.0f, Pc));
    Po[o] = F_ADD(F_ADD(Pc, F_MUL(F_MUL(dt, lap), inv_h2)), F_MUL(F_MUL(two_pi_dt, uc), uc));
  }
}

// reduceWGSL (mol_fast.js:353-444): 128 interior cells in linear order per block, per-cell f32
// terms, the shared-memory tree of the reference.  partials: one row of NR = n + 6 per block.
__global__ void __launch_bounds__(128) k_mf_reduce(const MfParams* __restrict__ p, const float* __restrict__ U,
                                                   const float* __restrict__ W, const float* __restrict__ Pv,
                                                   const float* __restrict__ K, float* __restrict__ part) {
  extern __shared__ float sn[];
  const int n = p->n, NR = n + 6, lid = threadIdx.x;
  for (int x = 0; x < NR; ++x) sn[lid * NR + x] = 0.0f;
  const long long NM = p->NN - 1, tot = NM * NM * NM;
  const long long cell = (long long)blockIdx.x * 128 + lid;
  if (cell < tot) {
    const int k = (int)(cell % NM) + 1, j = (int)((cell / NM) % NM) + 1, i = (int)(cell / (NM * NM)) + 1;
    const long long S = p->S, S2 = S * S, S3 = S2 * S;
    const long long id = (long long)i * S2 + (long long)j * S + k;
    const float h = p->h, h3 = p->h3;
    float T = 0.0f, VeK = 0.0f, Vee = 0.0f, dx = 0.0f, dy = 0.0f, dz = 0.0f;
    const float xc = F_MUL(F_SUB((float)i, (float)p->N2), h);
    const float yc = F_MUL(F_SUB((float)j, (float)p->N2), h);
    const float zc = F_MUL(F_SUB((float)k, (float)p->N2), h);
    float Ptot = 0.0f;
    for (int q = 0; q < n; ++q) Ptot = F_ADD(Ptot, __ldg(Pv + q * S3 + id));
    const float Kc = __ldg(K + id);
    for (int m = 0; m < n; ++m) {
      const long long o = m * S3 + id;
      const float v = __ldg(U + o);
      const float4 cr = p->red[m];
      const float vv = F_MUL(v, v);
      sn[lid * NR + m] = F_MUL(vv, h3);
      if (__ldg(W + o) > 0.1f) {
        const float a = F_SUB(__ldg(U + o + S2), v), b = F_SUB(__ldg(U + o + S), v), c = F_SUB(__ldg(U + o + 1), v);
        T = F_ADD(T, F_MUL(F_MUL(cr.y, F_ADD(F_ADD(F_MUL(a, a), F_MUL(b, b)), F_MUL(c, c))), h));
      }
      VeK = F_SUB(VeK, F_MUL(F_MUL(F_MUL(Kc, v), v), h3));
      const float rho_cell = F_MUL(vv, h3);
      dx = F_SUB(dx, F_MUL(rho_cell, xc));
      dy = F_SUB(dy, F_MUL(rho_cell, yc));
      dz = F_SUB(dz, F_MUL(rho_cell, zc));
      Vee = F_ADD(Vee, F_MUL(F_MUL(F_MUL(F_SUB(Ptot, F_MUL(cr.x, __ldg(Pv + o))), v), v), h3));
      if (cr.z != 0.0f)
        T = F_ADD(T, F_MUL(F_MUL(F_MUL(0.6f, p->alpha_tf), mf_pow(fmaxf(vv, 1e-20f), 1.6666667f)), h3));
      const float tilt = cr.w;
      if (tilt != 0.0f) T = F_ADD(T, F_MUL(F_MUL(F_MUL(F_MUL(-tilt, yc), v), v), h3));
    }
    sn[lid * NR + n] = T;
    sn[lid * NR + n + 1] = VeK;
    sn[lid * NR + n + 2] = Vee;
    sn[lid * NR + n + 3] = dx;
    sn[lid * NR + n + 4] = dy;
    sn[lid * NR + n + 5] = dz;
  }
  __syncthreads();
  for (int s = 64; s > 0; s >>= 1) {
    if (lid < s)
      for (int x = 0; x < NR; ++x) sn[lid * NR + x] = F_ADD(sn[lid * NR + x], sn[(lid + s) * NR + x]);
    __syncthreads();
  }
  if (lid < NR) part[(long long)blockIdx.x * NR + lid] = sn[lid];
}

// finalizeWGSL (mol_fast.js:446-472): the single workgroup's strided sums and tree, one block
// per slot (the slots never mix, so each block repeats the reference's order for its slot)
__global__ void __launch_bounds__(128) k_mf_finalize(const MfParams* __restrict__ p, const float* __restrict__ part,
                                                     long long nwg, float* __restrict__ sums) {
  __shared__ float wg[128];
  const int NR = p->n + 6, x = blockIdx.x, lid = threadIdx.x;
  float acc = 0.0f;
#pragma unroll 4
  for (long long q = lid; q < nwg; q += 128) acc = F_ADD(acc, __ldg(part + q * NR + x));
  wg[lid] = acc;
  __syncthreads();
  for (int s = 64; s > 0; s >>= 1) {
    if (lid < s) wg[lid] = F_ADD(wg[lid], wg[lid + s]);
    __syncthreads();
  }
  if (lid == 0) sums[x] = wg[0];
}

// normalizeWGSL (mol_fast.js:474-492)
__global__ void __launch_bounds__(256) k_mf_normalize(const MfParams* __restrict__ p, float* __restrict__ U,
                                                      const float* __restrict__ sums) {
  const int NN = p->NN;
  const int k = blockIdx.x * kMfTK + threadIdx.x + 1;
  const int j = blockIdx.y * kMfTJ + threadIdx.y + 1;
  const int i = blockIdx.z + 1;
  if (k >= NN || j >= NN) return;
  const long long S = p->S, S2 = S * S, S3 = S2 * S;
  const long long id = (long long)i * S2 + (long long)j * S + k;
  for (int m = 0; m < p->n; ++m) {
    const float nrm = sums[m], tgt = p->rcs[m].y;
    if (nrm > 0.0f && tgt > 0.0f) U[m * S3 + id] = F_MUL(U[m * S3 + id], F_SQRT(F_DIV(tgt, nrm)));
  }
}

// rhoSourceWGSL + residualPmWGSL (mol_fast.js:645-690) for every electron (blockIdx.z = i-1 + NM m)
__global__ void __launch_bounds__(256) k_mf_residual(const MfParams* __restrict__ p, const float* __restrict__ U,
                                                     const float* __restrict__ P, float* __restrict__ res) {
  const int NN = p->NN, NM = NN - 1;
  const int k = blockIdx.x * kMfTK + threadIdx.x + 1;
  const int j = blockIdx.y * kMfTJ + threadIdx.y + 1;
  const int i = blockIdx.z % NM + 1, m = blockIdx.z / NM;
  if (k >= NN || j >= NN) return;
  const long long S = p->S, S2 = S * S, S3 = S2 * S;
  const long long o = m * S3 + (long long)i * S2 + (long long)j * S + k;
  const float Pc = __ldg(P + o);
  const float lap = F_MUL(F_SUB(F_ADD(F_ADD(F_ADD(F_ADD(F_ADD(__ldg(P + o + S2), __ldg(P + o - S2)), __ldg(P + o + S)),
                                                    __ldg(P + o - S)),
                                              __ldg(P + o + 1)),
                                        __ldg(P + o - 1)),
                                  F_MUL(6.0f, Pc)),
                          p->inv_h2);
  const float u = __ldg(U + o);
  res[o] = F_SUB(F_MUL(-p->two_pi, F_MUL(u, u)), lap);
}

// restrictWGSL (mol_fast.js:692-725), blockIdx.z = I-1 + (NC-1) m
__global__ void __launch_bounds__(256) k_mf_restrict(const MfParams* __restrict__ p, const float* __restrict__ fine,
                                                     float* __restrict__ coarse) {
  const int NC = p->NN / 2, NCM = NC - 1;
  const int K2 = blockIdx.x * kMfTK + threadIdx.x + 1;
  const int J = blockIdx.y * kMfTJ + threadIdx.y + 1;
  const int I = blockIdx.z % NCM + 1, m = blockIdx.z / NCM;
  if (K2 >= NC || J >= NC) return;
  const long long S = p->S, S2 = S * S, S3 = S2 * S;
  const long long SC = NC + 1, SC2 = SC * SC, SC3 = SC2 * SC;
  const float* f = fine + m * S3;
  const long long c = (2LL * I) * S2 + (2LL * J) * S + 2LL * K2;
  auto F = [&](int a, int b, int d) { return __ldg(f + c + a * S2 + b * S + d); };
  float val = F_MUL(8.0f, F(0, 0, 0));
  val = F_ADD(val, F_MUL(4.0f, F_ADD(F_ADD(F_ADD(F_ADD(F_ADD(F(1, 0, 0), F(-1, 0, 0)), F(0, 1, 0)), F(0, -1, 0)), F(0, 0, 1)),
                                     F(0, 0, -1))));
  float e = F_ADD(F(1, 1, 0), F(1, -1, 0));
  e = F_ADD(e, F(-1, 1, 0)); e = F_ADD(e, F(-1, -1, 0));
  e = F_ADD(e, F(1, 0, 1)); e = F_ADD(e, F(1, 0, -1)); e = F_ADD(e, F(-1, 0, 1)); e = F_ADD(e, F(-1, 0, -1));
  e = F_ADD(e, F(0, 1, 1)); e = F_ADD(e, F(0, 1, -1)); e = F_ADD(e, F(0, -1, 1)); e = F_ADD(e, F(0, -1, -1));
  val = F_ADD(val, F_MUL(2.0f, e));
  float v = F_ADD(F(1, 1, 1), F(1, 1, -1));
  v = F_ADD(v, F(1, -1, 1)); v = F_ADD(v, F(1, -1, -1)); v = F_ADD(v, F(-1, 1, 1)); v = F_ADD(v, F(-1, 1, -1));
  v = F_ADD(v, F(-1, -1, 1)); v = F_ADD(v, F(-1, -1, -1));
  val = F_ADD(val, v);
  coarse[m * SC3 + (long long)I * SC2 + (long long)J * SC + K2] = F_MUL(val, 0.015625f);
}

// coarseSmoothWGSL (mol_fast.js:727-751), blockIdx.z = I-1 + (NC-1) m
__global__ void __launch_bounds__(256) k_mf_coarse(const MfParams* __restrict__ p, const float* __restrict__ Ein,
                                                   float* __restrict__ Eout, const float* __restrict__ rhs) {
  const int NC = p->NN / 2, NCM = NC - 1;
  const int K2 = blockIdx.x * kMfTK + threadIdx.x + 1;
  const int J = blockIdx.y * kMfTJ + threadIdx.y + 1;
  const int I = blockIdx.z % NCM + 1, m = blockIdx.z / NCM;
  if (K2 >= NC || J >= NC) return;
  const long long SC = NC + 1, SC2 = SC * SC, SC3 = SC2 * SC;
  const long long c = m * SC3 + (long long)I * SC2 + (long long)J * SC + K2;
  const float sum = F_ADD(F_ADD(F_ADD(F_ADD(F_ADD(Ein[c + SC2], Ein[c - SC2]), Ein[c + SC]), Ein[c - SC]), Ein[c + 1]), Ein[c - 1]);
  Eout[c] = F_ADD(F_MUL(0.3333f, Ein[c]), F_DIV(F_ADD(sum, F_MUL(F_MUL(4.0f, p->h2), rhs[c])), 9.0f));
}

// prolongCorrectPmWGSL (mol_fast.js:753-785), blockIdx.z = i-1 + NM m
__global__ void __launch_bounds__(256) k_mf_prolong(const MfParams* __restrict__ p, const float* __restrict__ Ec,
                                                    float* __restrict__ P) {
  const int NN = p->NN, NM = NN - 1, NC = NN / 2;
  const int k = blockIdx.x * kMfTK + threadIdx.x + 1;
  const int j = blockIdx.y * kMfTJ + threadIdx.y + 1;
  const int i = blockIdx.z % NM + 1, m = blockIdx.z / NM;
  if (k >= NN || j >= NN) return;
  const long long S = p->S, S2 = S * S, S3 = S2 * S;
  const long long SC = NC + 1, SC2 = SC * SC, SC3 = SC2 * SC;
  const int ci = i / 2, cj = j / 2, ck = k / 2;
  const int ci1 = min(ci + (i & 1), NC), cj1 = min(cj + (j & 1), NC), ck1 = min(ck + (k & 1), NC);
  const float wi = (i & 1) ? 0.5f : 1.0f, wj = (j & 1) ? 0.5f : 1.0f, wk = (k & 1) ? 0.5f : 1.0f;
  const float wi1 = F_SUB(1.0f, wi), wj1 = F_SUB(1.0f, wj), wk1 = F_SUB(1.0f, wk);
  const float* E = Ec + m * SC3;
  auto e = [&](int a, int b, int c) { return __ldg(E + (long long)a * SC2 + (long long)b * SC + c); };
  float corr = 0.0f;
  corr = F_ADD(corr, F_MUL(F_MUL(F_MUL(wi, wj), wk), e(ci, cj, ck)));
  corr = F_ADD(corr, F_MUL(F_MUL(F_MUL(wi, wj), wk1), e(ci, cj, ck1)));
  corr = F_ADD(corr, F_MUL(F_MUL(F_MUL(wi, wj1), wk), e(ci, cj1, ck)));
  corr = F_ADD(corr, F_MUL(F_MUL(F_MUL(wi, wj1), wk1), e(ci, cj1, ck1)));
  corr = F_ADD(corr, F_MUL(F_MUL(F_MUL(wi1, wj), wk), e(ci1, cj, ck)));
  corr = F_ADD(corr, F_MUL(F_MUL(F_MUL(wi1, wj), wk1), e(ci1, cj, ck1)));
  corr = F_ADD(corr, F_MUL(F_MUL(F_MUL(wi1, wj1), wk), e(ci1, cj1, ck)));
  corr = F_ADD(corr, F_MUL(F_MUL(F_MUL(wi1, wj1), wk1), e(ci1, cj1, ck1)));
  const long long o = m * S3 + (long long)i * S2 + (long long)j * S + k;
  P[o] = F_ADD(P[o], F_MUL(0.5f, corr));
}

// forceWGSL (mol_fast.js:500-563): the ball's terms in parallel, summed by one thread in the
// reference's (di, dj, dk) order
__global__ void __launch_bounds__(256) k_mf_force(const MfParams* __restrict__ p, const float* __restrict__ P,
                                                  float* __restrict__ F) {
  __shared__ float tx[729], ty[729], tz[729];
  __shared__ unsigned char ok[729];
  const int a = blockIdx.x;
  const float4 at = p->atoms[a];
  if (at.w <= 0.0f) {
    if (threadIdx.x == 0) F[3 * a] = F[3 * a + 1] = F[3 * a + 2] = 0.0f;
    return;
  }
  const int S = p->S, n = p->n;
  const long long S2 = (long long)S * S, S3 = S2 * S;
  const int ci = (int)at.x, cj = (int)at.y, ck = (int)at.z;
  const float inv2h = F_MUL(0.5f, p->inv_h);
  for (int t = threadIdx.x; t < 729; t += blockDim.x) {
    const int di = t / 81 - 4, dj = (t / 9) % 9 - 4, dk = t % 9 - 4;
    const int ii = ci + di, jj = cj + dj, kk = ck + dk;
    const bool v = ii >= 1 && ii < S - 1 && jj >= 1 && jj < S - 1 && kk >= 1 && kk < S - 1 &&
                   !((float)(di * di + dj * dj + dk * dk) > 16.0f);
    ok[t] = v;
    if (v) {
      float xp = 0.0f, xm = 0.0f, yp = 0.0f, ym = 0.0f, zp = 0.0f, zm = 0.0f;
      const long long c = (long long)ii * S2 + (long long)jj * S + kk;
      for (int m = 0; m < n; ++m) {
        const float* Pm = P + m * S3 + c;
        xp = F_ADD(xp, __ldg(Pm + S2)); xm = F_ADD(xm, __ldg(Pm - S2));
        yp = F_ADD(yp, __ldg(Pm + S)); ym = F_ADD(ym, __ldg(Pm - S));
        zp = F_ADD(zp, __ldg(Pm + 1)); zm = F_ADD(zm, __ldg(Pm - 1));
      }
      tx[t] = F_MUL(F_SUB(xp, xm), inv2h);
      ty[t] = F_MUL(F_SUB(yp, ym), inv2h);
      tz[t] = F_MUL(F_SUB(zp, zm), inv2h);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float sx = 0.0f, sy = 0.0f, sz = 0.0f, count = 0.0f;
    for (int t = 0; t < 729; ++t)
      if (ok[t]) {
        sx = F_ADD(sx, tx[t]); sy = F_ADD(sy, ty[t]); sz = F_ADD(sz, tz[t]);
        count = F_ADD(count, 1.0f);
      }
    const float avg = count > 0.0f ? F_DIV(1.0f, count) : 0.0f;
    const float z2 = F_MUL(2.0f, at.w);
    F[3 * a] = F_MUL(F_MUL(z2, sx), avg);
    F[3 * a + 1] = F_MUL(F_MUL(z2, sy), avg);
    F[3 * a + 2] = F_MUL(F_MUL(z2, sz), avg);
  }
}

// recomputeK_WGSL (mol_fast.js:565-587) over all S^3 points
__global__ void __launch_bounds__(256) k_mf_recompute_k(const MfParams* __restrict__ p, float* __restrict__ K) {
  const long long S = p->S, S2 = S * S, S3 = S2 * S;
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= S3) return;
  const int k = (int)(id % S), j = (int)((id / S) % S), i = (int)(id / S2);
  const float h = p->h, soft = F_MUL(4.0f, p->h2);
  float Kv = 0.0f;
  for (int a = 0; a < p->n; ++a) {
    const float4 at = p->atoms[a];
    if (at.w <= 0.0f) continue;
    const float di = F_MUL(F_SUB((float)i, at.x), h), dj = F_MUL(F_SUB((float)j, at.y), h),
                dk = F_MUL(F_SUB((float)k, at.z), h);
    Kv = F_ADD(Kv, F_DIV(at.w, F_SQRT(F_ADD(F_ADD(F_ADD(F_MUL(di, di), F_MUL(dj, dj)), F_MUL(dk, dk)), soft))));
  }
  K[id] = Kv;
}

// extractWGSL (mol_fast.js:595-640)
__global__ void __launch_bounds__(256) k_mf_extract(const MfParams* __restrict__ p, const float* __restrict__ U,
                                                    const float* __restrict__ W, const float* __restrict__ Pv,
                                                    float* __restrict__ out) {
  const int i = blockIdx.x * 16 + threadIdx.x, j = blockIdx.y * 16 + threadIdx.y;
  const int NN = p->NN, n = p->n, N2 = p->N2;
  if (i > NN || j > NN) return;
  const long long SS = NN + 1, S2 = SS * SS, S3 = S2 * SS;
  for (int m = 0; m < n; ++m) {
    const long long idx2 = m * S3 + (long long)i * S2 + (long long)j * SS + N2;
    out[m * SS * SS + i * SS + j] = W[idx2] > 0.1f ? U[idx2] : 0.0f;
    if (j == 0) {
      const long long line = (long long)i * S2 + (long long)N2 * SS + N2, ml = m * S3 + line;
      out[n * SS * SS + m * SS + i] = U[ml];
      out[2 * n * SS * SS + m * SS + i] = W[ml];
      float Ps = 0.0f;
      for (int q = 0; q < n; ++q) Ps = F_ADD(Ps, Pv[q * S3 + line]);
      if (m == 0) out[n * SS * SS + n * SS + i] = F_MUL(2.0f, Ps);
      float Vp = 0.0f;
      if (p->rcs[m].y > 1.0f && p->alpha_tf > 0.0f) Vp = F_MUL(p->alpha_tf, mf_pow(fmaxf(F_MUL(U[ml], U[ml]), 1e-20f), 0.6666667f));
      out[n * SS * SS + (n + 1 + m) * SS + i] = Vp;
    }
  }
}

// ---- initial state (uploadInitialData, mol_fast.js:941-1046): JS numbers, f32 stores --------

// inSplit (mol_fast.js:878-939) on the raw USER_NUCLEI axis
__device__ bool mf_in_split_f64(double dx, double dy, double dz, double r, int split, int idx, const double* axr) {
  if (split == 0 || split == 1 || r < 1e-6) return true;
  double L = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(axr[0], axr[0]), __dmul_rn(axr[1], axr[1])), __dmul_rn(axr[2], axr[2])));
  if (L == 0) L = 1;
  const double a0 = axr[0] / L, a1 = axr[1] / L, a2 = axr[2] / L;
  const double PI = 3.141592653589793;
  auto dot3 = [](double x, double y, double z, double u, double v, double w) {
    return __dadd_rn(__dadd_rn(__dmul_rn(x, u), __dmul_rn(y, v)), __dmul_rn(z, w));
  };
  if (split == 2) {
    const double d = dot3(dx, dy, dz, a0, a1, a2);
    return idx == 0 ? d < 0 : d >= 0;
  }
  if (split == 3 || split == 5) {
    const double d = dot3(dx, dy, dz, a0, a1, a2);
    if (split == 5) {
      if (idx == 0) return d >= 0;
      if (d >= 0) return false;
    }
    const double px = __dsub_rn(dx, __dmul_rn(d, a0)), py = __dsub_rn(dy, __dmul_rn(d, a1)), pz = __dsub_rn(dz, __dmul_rn(d, a2));
    double e1x, e1y, e1z;
    if (fabs(a2) < 0.9) { e1x = a1; e1y = -a0; e1z = 0; }
    else { e1x = 0; e1y = a2; e1z = -a1; }
    double e1L = sqrt(dot3(e1x, e1y, e1z, e1x, e1y, e1z));
    if (e1L == 0) e1L = 1;
    e1x /= e1L; e1y /= e1L; e1z /= e1L;
    const double e2x = __dsub_rn(__dmul_rn(a1, e1z), __dmul_rn(a2, e1y));
    const double e2y = __dsub_rn(__dmul_rn(a2, e1x), __dmul_rn(a0, e1z));
    const double e2z = __dsub_rn(__dmul_rn(a0, e1y), __dmul_rn(a1, e1x));
    const double pe1 = dot3(px, py, pz, e1x, e1y, e1z), pe2 = dot3(px, py, pz, e2x, e2y, e2z);
    double theta = atan2(pe2, pe1) - 0;
    if (theta < -PI) theta += 2 * PI;
    if (theta > PI) theta -= 2 * PI;
    const int sector = (int)fmod(floor((theta + PI) / (2 * PI / 3)), 3.0);
    return split == 3 ? sector == idx : sector == idx - 1;
  }
  if (split == 4) {
    const double vs[4][3] = {{1, 1, 1}, {1, -1, -1}, {-1, 1, -1}, {-1, -1, 1}};
    const double u0 = dx / r, u1 = dy / r, u2 = dz / r;
    int best = 0;
    double bestDot = -INFINITY;
    for (int v = 0; v < 4; ++v) {
      const double d = dot3(vs[v][0], vs[v][1], vs[v][2], u0, u1, u2);
      if (d > bestDot) { bestDot = d; best = v; }
    }
    return best == idx;
  }
  return true;
}

__global__ void __launch_bounds__(256) k_mf_init(const double* __restrict__ nuc, int n, int NN, double hv, double midI0,
                                                 float* __restrict__ K, float* __restrict__ U, float* __restrict__ W,
                                                 float* __restrict__ P) {
  const long long S = NN + 1, S2 = S * S, S3 = S2 * S;
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= S3) return;
  const int k = (int)(id % S), j = (int)((id / S) % S), i = (int)(id / S2);
  const double h2v = __dmul_rn(hv, hv), soft = __dmul_rn(4.0, h2v), R_init = 3.0;
  double Kacc = 0, rl[kMfMax], ul[kMfMax];
  int bestM = -1;
  double bestU = -1;
  for (int a = 0; a < n; ++a) {
    const double* c = nuc + kMfNucLen * a;
    const double dx = __dmul_rn(__dsub_rn((double)i, c[0]), hv), dy = __dmul_rn(__dsub_rn((double)j, c[1]), hv),
                 dz = __dmul_rn(__dsub_rn((double)k, c[2]), hv);
    const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
    const double r_soft = __dsqrt_rn(__dadd_rn(r2, soft));
    const double r = __dsqrt_rn(r2);
    Kacc = __dadd_rn(Kacc, __ddiv_rn(c[3], r_soft));
    const double z = c[7];
    const double uh = exp(-__dmul_rn(z, r));
    rl[a] = r;
    ul[a] = uh;
    const double tg = c[8] != 0 ? c[8] : 1.0;
    const double uw = __dmul_rn(__dsqrt_rn(__dmul_rn(__dmul_rn(__dmul_rn(tg, z), z), z)), uh);
    const double roa = c[5];
    const bool okR = !(roa > 0 && r > __dadd_rn(roa, hv));
    const double hs = c[6];
    const bool okHS = hs == 0 || ((hs > 0) == ((double)i > midI0));
    const bool okS = mf_in_split_f64(dx, dy, dz, r, (int)c[9], (int)c[10], c + 11);
    if (okR && okHS && okS && uw > bestU) { bestU = uw; bestM = a; }
  }
  K[id] = (float)Kacc;
  for (int m = 0; m < n; ++m) {
    const double rc = nuc[kMfNucLen * m + 4];
    double u = ul[m];
    if (rc > 0 && rl[m] < rc) {
      const double edge = __dsub_rn(rc, __dmul_rn(3.0, hv));
      const double t = fmax(0.0, fmin(1.0, __ddiv_rn(__dsub_rn(rl[m], edge), __dsub_rn(rc, edge))));
      u = __dmul_rn(u, __dmul_rn(__dmul_rn(t, t), __dsub_rn(3.0, __dmul_rn(2.0, t))));
    }
    U[m * S3 + id] = (float)u;
    W[m * S3 + id] = 0.0f;
    P[m * S3 + id] = (float)__ddiv_rn(__dmul_rn(0.5, nuc[kMfNucLen * m + 3]), __dadd_rn(rl[m], h2v));
  }
  if (bestM >= 0 && rl[bestM] < R_init) {
    const double rc = nuc[kMfNucLen * bestM + 4], ro = nuc[kMfNucLen * bestM + 5];
    double w = 1.0;
    if (rc > 0 && rl[bestM] < rc) {
      const double edge = __dsub_rn(rc, __dmul_rn(3.0, hv));
      const double t = fmax(0.0, fmin(1.0, __ddiv_rn(__dsub_rn(rl[bestM], edge), __dsub_rn(rc, edge))));
      w = __dmul_rn(__dmul_rn(t, t), __dsub_rn(3.0, __dmul_rn(2.0, t)));
    }
    if (ro > 0 && rl[bestM] > __dadd_rn(ro, hv)) w = 0;
    W[bestM * S3 + id] = (float)w;
  }
}

// FP64 sum of U^2 of electron blockIdx.y over all S^3 points (the pre-normalisation of
// uploadInitialData, mol_fast.js:1024-1037)
__global__ void __launch_bounds__(256) k_mf_init_norm(const float* __restrict__ U, long long S3, double* __restrict__ acc) {
  __shared__ double red[256];
  const float* Um = U + blockIdx.y * S3;
  double s = 0;
  for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < S3; id += (long long)gridDim.x * blockDim.x) {
    const double u = Um[id];
    s = __dadd_rn(s, __dmul_rn(u, u));
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(acc + blockIdx.y, red[0]);
}

__global__ void __launch_bounds__(256) k_mf_init_scale(float* __restrict__ U, long long S3, const double* __restrict__ acc,
                                                       const double* __restrict__ nuc, double h3v) {
  const int m = blockIdx.y;
  const double nrm = __dmul_rn(acc[m], h3v), tg = nuc[kMfNucLen * m + 8];
  if (!(nrm > 0 && tg > 0)) return;
  const double sc = __dsqrt_rn(__ddiv_rn(tg, nrm));
  float* Um = U + m * S3;
  for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < S3; id += (long long)gridDim.x * blockDim.x)
    Um[id] = (float)__dmul_rn((double)Um[id], sc);
}

}  // namespace rq

using namespace rq;

struct rq_mf {
  rq_mf_config cfg{};
  std::vector<rq_mf_nucleus> nuc;
  int n = 0, NN = 0, S = 0, nr = 0;
  long long S3 = 0, SC3 = 0, nwg = 0;
  MfParams hp{};
  MfParams* dp = nullptr;
  float *U[2] = {}, *W[2] = {}, *P[2] = {}, *K = nullptr;
  float *res = nullptr, *rhsC = nullptr, *errC[2] = {};
  float *part = nullptr, *sums = nullptr, *force = nullptr, *slice = nullptr;
  int cur = 0;
  bool r_out_enforce = true;
  long long t_step = 0, launches = 0;
  cudaStream_t st = nullptr;
  std::map<std::pair<int, int>, std::pair<cudaGraphExec_t, long long>> graphs;  // (n, cur) -> graph, launches
  std::string last_error;
};

#define MCK(call)                                                          \
  do {                                                                     \
    cudaError_t _e = (call);                                               \
    if (_e != cudaSuccess) {                                               \
      s->last_error = std::string(#call) + ": " + cudaGetErrorString(_e);  \
      return _e == cudaErrorMemoryAllocation ? RQ_ENOMEM : RQ_ECUDA;       \
    }                                                                      \
  } while (0)
#define MLAUNCH() MCK(cudaGetLastError()); s->launches++

namespace {

// JS toFixed(6) of a number, as the shader text carries it, then the literal's f32 value
float fixed6(double v) {
  char buf[64];
  std::snprintf(buf, sizeof buf, "%.6f", v);
  return (float)std::strtod(buf, nullptr);
}

void mf_fill_params(rq_mf* s) {
  MfParams& p = s->hp;
  std::memset(&p, 0, sizeof p);
  const rq_mf_config& c = s->cfg;
  const double hv = c.screen / c.NN, h2v = hv * hv, h3v = hv * hv * hv, dv = 0.12;
  p.NN = c.NN; p.S = c.NN + 1; p.N2 = c.NN / 2; p.n = s->n; p.shell_mode = c.shell_mode ? 1 : 0;
  p.h = (float)hv; p.h2 = (float)h2v; p.inv_h = (float)(1 / hv); p.inv_h2 = (float)(1 / h2v);
  p.dt = (float)(dv * h2v); p.half_d = (float)(c.kinetic_coeff * dv); p.h3 = (float)h3v;
  p.two_pi = (float)(2 * M_PI);
  p.R_out = s->r_out_enforce ? 1.0f : 0.0f;
  p.field_x = (float)c.field_x; p.alpha_tf = (float)c.alpha_tf; p.full_self = c.full_self ? 1.0f : 0.0f;
  p.kc = fixed6(c.kinetic_coeff); p.kc_multi = fixed6(c.kc_multi); p.beta = fixed6(c.beta_pauli);
  for (int a = 0; a < s->n; ++a) {
    const rq_mf_nucleus& q = s->nuc[a];
    p.atoms[a] = make_float4((float)q.i, (float)q.j, (float)q.k, (float)q.Z);
    p.rcs[a] = make_float4((float)q.rc, (float)q.norm_target, (float)q.tilt_x, (float)q.tilt_y);
    p.r_out[a] = fixed6(q.r_out);
    if (p.rcs[a].x > 0.0f) p.any_rc = 1;
    p.split_type[a] = q.split;
    p.split_idx[a] = q.split_idx;
    p.split_fix[a] = q.split_fix ? 1 : 0;
    const double* v = q.split_axis;
    double L = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (L == 0) L = 1;
    p.ax[a] = make_float4(fixed6(v[0] / L), fixed6(v[1] / L), fixed6(v[2] / L), 0.0f);
    // split siblings at one site share their Hartree subtraction (mol_fast.js:124-132)
    int g = a;
    if (q.split != 0)
      for (int b = 0; b < a; ++b) {
        const rq_mf_nucleus& o = s->nuc[b];
        if (o.split == q.split && o.i == q.i && o.j == q.j && o.k == q.k) { g = b; break; }
      }
    p.split_group[a] = g;
  }
  if (s->n == kMfMax) p.rcs[kMfMax - 1].z = (float)c.line_j_offset;  // the reference's last rcs slot
  for (int a = 0; a < s->n; ++a) {
    const float selfN = p.rcs[a].y;
    const float km = selfN > 1.0f ? p.kc_multi : 1.0f;
    const float fm = selfN > 1.0f ? (p.full_self > 0.5f ? 0.0f : 1.0f / selfN) : 1.0f;
    const float tf = (selfN > 1.0f && p.alpha_tf > 0.0f) ? 1.0f : 0.0f;
    p.upd[a] = make_float4(fm, p.half_d * km, tf, p.rcs[a].z);
    p.red[a] = make_float4(selfN > 1.0f ? 1.0f / selfN : 1.0f, km * p.kc, tf, p.rcs[a].w);
    unsigned gmask = 0;
    for (int b = 0; b < s->n; ++b)
      if (p.split_group[b] == p.split_group[a]) gmask |= 1u << b;
    p.gmask[a] = gmask;
  }
}

int mf_upload_params(rq_mf* s) {
  MCK(cudaMemcpyAsync(s->dp, &s->hp, sizeof(MfParams), cudaMemcpyHostToDevice, s->st));
  return RQ_OK;
}

dim3 mf_grid(int NN, int planes) {
  const int NM = NN - 1;
  return dim3((NM + kMfTK - 1) / kMfTK, (NM + kMfTJ - 1) / kMfTJ, planes);
}

int mf_launch_update(rq_mf* s, int c) {
  const int nx = 1 - c;
  const dim3 g = mf_grid(s->NN, s->NN - 1), b(kMfTK, kMfTJ);
  const bool sh = s->cfg.shell_mode != 0;
#define MF_UPD(NM_, SH_) \
  k_mf_update<NM_, SH_><<<g, b, 0, s->st>>>(s->dp, s->U[c], s->W[c], s->P[c], s->K, s->U[nx], s->W[nx], s->P[nx])
  if (s->n <= 4) { if (sh) MF_UPD(4, true); else MF_UPD(4, false); }
  else if (s->n <= 8) { if (sh) MF_UPD(8, true); else MF_UPD(8, false); }
  else { if (sh) MF_UPD(16, true); else MF_UPD(16, false); }
#undef MF_UPD
  MLAUNCH();
  return RQ_OK;
}

int mf_launch_reduce(rq_mf* s, int c) {
  k_mf_reduce<<<(unsigned)s->nwg, 128, sizeof(float) * 128 * s->nr, s->st>>>(s->dp, s->U[c], s->W[c], s->P[c], s->K, s->part);
  MLAUNCH();
  k_mf_finalize<<<s->nr, 128, 0, s->st>>>(s->dp, s->part, s->nwg, s->sums);
  MLAUNCH();
  return RQ_OK;
}

int mf_vcycle(rq_mf* s, int c) {
  const int NN = s->NN, NC = NN / 2;
  k_mf_residual<<<mf_grid(NN, (NN - 1) * s->n), dim3(kMfTK, kMfTJ), 0, s->st>>>(s->dp, s->U[c], s->P[c], s->res);
  MLAUNCH();
  k_mf_restrict<<<mf_grid(NC, (NC - 1) * s->n), dim3(kMfTK, kMfTJ), 0, s->st>>>(s->dp, s->res, s->rhsC);
  MLAUNCH();
  MCK(cudaMemsetAsync(s->errC[0], 0, sizeof(float) * s->SC3 * s->n, s->st));
  MCK(cudaMemsetAsync(s->errC[1], 0, sizeof(float) * s->SC3 * s->n, s->st));
  for (int q = 0; q < s->cfg.coarse_iters; ++q) {
    k_mf_coarse<<<mf_grid(NC, (NC - 1) * s->n), dim3(kMfTK, kMfTJ), 0, s->st>>>(s->dp, s->errC[q % 2], s->errC[1 - q % 2], s->rhsC);
    MLAUNCH();
  }
  k_mf_prolong<<<mf_grid(NN, (NN - 1) * s->n), dim3(kMfTK, kMfTJ), 0, s->st>>>(s->dp, s->errC[0], s->P[c]);
  MLAUNCH();
  return RQ_OK;
}

// the launch sequence of doSteps(n) (mol_fast.js:1244-1291) starting from buffer set c
int mf_frame(rq_mf* s, int n, int c) {
  int rc;
  for (int q = 0; q < n; ++q) {
    const int nx = 1 - c;
    if ((rc = mf_launch_update(s, c)) != RQ_OK) return rc;
    if ((q + 1) % 20 == 0 || q == n - 1) {
      if ((rc = mf_launch_reduce(s, nx)) != RQ_OK) return rc;
      k_mf_normalize<<<mf_grid(s->NN, s->NN - 1), dim3(kMfTK, kMfTJ), 0, s->st>>>(s->dp, s->U[nx], s->sums);
      MLAUNCH();
    }
    if (s->cfg.vcycle && (q + 1) % s->cfg.vcycle_interval == 0)
      if ((rc = mf_vcycle(s, nx)) != RQ_OK) return rc;
    c = nx;
  }
  return RQ_OK;
}

}  // namespace

extern "C" int rq_mf_create(const rq_mf_config* cfg, const rq_mf_nucleus* nuclei, int32_t n, rq_mf** out) {
  if (!cfg || !nuclei || !out || n < 1 || n > kMfMax) return RQ_EINVAL;
  *out = nullptr;
  if (cfg->NN < 8 || cfg->NN % 2 || !(cfg->screen > 0) || cfg->vcycle_interval < 1 || cfg->coarse_iters < 0)
    return RQ_EINVAL;
  for (int a = 0; a < n; ++a) {
    const int sp = nuclei[a].split;
    if (sp < 0 || sp > 5 || sp == 1) return RQ_EINVAL;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return RQ_ENODEV;
  rq_mf* s = new (std::nothrow) rq_mf();
  if (!s) return RQ_ENOMEM;
  s->cfg = *cfg;
  s->nuc.assign(nuclei, nuclei + n);
  s->n = n; s->NN = cfg->NN; s->S = cfg->NN + 1; s->nr = n + 6;
  s->S3 = (long long)s->S * s->S * s->S;
  const long long SC = cfg->NN / 2 + 1;
  s->SC3 = SC * SC * SC;
  const long long NM = cfg->NN - 1;
  s->nwg = (NM * NM * NM + 127) / 128;
  auto fail = [&](int rc) {
    std::fprintf(stderr, "rq_mf_create: %s\n", s->last_error.c_str());
    rq_mf_destroy(s);
    return rc;
  };
  auto alloc = [&](void** p, size_t bytes) -> int {
    if (cudaMalloc(p, bytes) != cudaSuccess) { s->last_error = "cudaMalloc"; return RQ_ENOMEM; }
    if (cudaMemset(*p, 0, bytes) != cudaSuccess) { s->last_error = "cudaMemset"; return RQ_ECUDA; }
    return RQ_OK;
  };
  const size_t F = sizeof(float), fld = F * (size_t)s->S3 * n, cfld = F * (size_t)s->SC3 * n;
  int rc = RQ_OK;
  for (int b = 0; b < 2 && rc == RQ_OK; ++b)
    if ((rc = alloc((void**)&s->U[b], fld)) || (rc = alloc((void**)&s->W[b], fld)) || (rc = alloc((void**)&s->P[b], fld)) ||
        (rc = alloc((void**)&s->errC[b], cfld)))
      break;
  if (rc == RQ_OK &&
      ((rc = alloc((void**)&s->K, F * s->S3)) || (rc = alloc((void**)&s->res, fld)) || (rc = alloc((void**)&s->rhsC, cfld)) ||
       (rc = alloc((void**)&s->part, F * (size_t)s->nwg * s->nr)) || (rc = alloc((void**)&s->sums, F * s->nr)) ||
       (rc = alloc((void**)&s->force, F * 3 * n)) || (rc = alloc((void**)&s->slice, F * 3 * (size_t)n * s->S * s->S)) ||
       (rc = alloc((void**)&s->dp, sizeof(MfParams)))))
    ;
  if (rc != RQ_OK) return fail(rc);
  if (cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess) {
    s->last_error = "cudaStreamCreate";
    return fail(RQ_ECUDA);
  }
  mf_fill_params(s);
  if ((rc = mf_upload_params(s)) != RQ_OK) return fail(rc);
  // initial state on the device
  std::vector<double> rec((size_t)kMfNucLen * n, 0.0);
  for (int a = 0; a < n; ++a) {
    const rq_mf_nucleus& q = nuclei[a];
    double* r = rec.data() + kMfNucLen * a;
    r[0] = q.i; r[1] = q.j; r[2] = q.k; r[3] = q.Z; r[4] = q.rc; r[5] = q.r_out; r[6] = q.hs; r[7] = q.z_init;
    r[8] = q.norm_target; r[9] = q.split; r[10] = q.split_idx;
    r[11] = q.split_axis[0]; r[12] = q.split_axis[1]; r[13] = q.split_axis[2];
  }
  double* dnuc = nullptr;
  double* acc = nullptr;
  if ((rc = alloc((void**)&dnuc, sizeof(double) * rec.size())) || (rc = alloc((void**)&acc, sizeof(double) * n))) {
    if (dnuc) cudaFree(dnuc);
    return fail(rc);
  }
  const double hv = cfg->screen / cfg->NN;
  const double midI0 = (nuclei[0].i + nuclei[n - 1].i) / 2;
  cudaError_t e = cudaMemcpyAsync(dnuc, rec.data(), sizeof(double) * rec.size(), cudaMemcpyHostToDevice, s->st);
  if (e == cudaSuccess) {
    k_mf_init<<<(unsigned)((s->S3 + 255) / 256), 256, 0, s->st>>>(dnuc, n, cfg->NN, hv, midI0, s->K, s->U[0], s->W[0], s->P[0]);
    k_mf_init_norm<<<dim3(592, n), 256, 0, s->st>>>(s->U[0], s->S3, acc);
    k_mf_init_scale<<<dim3(592, n), 256, 0, s->st>>>(s->U[0], s->S3, acc, dnuc, hv * hv * hv);
    s->launches += 3;
    e = cudaGetLastError();
  }
  for (const auto& pr : {std::make_pair(s->U[1], s->U[0]), std::make_pair(s->W[1], s->W[0]), std::make_pair(s->P[1], s->P[0])})
    if (e == cudaSuccess) e = cudaMemcpyAsync(pr.first, pr.second, fld, cudaMemcpyDeviceToDevice, s->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
  cudaFree(dnuc);
  cudaFree(acc);
  if (e != cudaSuccess) {
    s->last_error = std::string("initial state: ") + cudaGetErrorString(e);
    return fail(RQ_ECUDA);
  }
  *out = s;
  return RQ_OK;
}

extern "C" void rq_mf_destroy(rq_mf* s) {
  if (!s) return;
  if (s->st) cudaStreamSynchronize(s->st);
  for (auto& kv : s->graphs) cudaGraphExecDestroy(kv.second.first);
  for (int b = 0; b < 2; ++b)
    for (void* p : {(void*)s->U[b], (void*)s->W[b], (void*)s->P[b], (void*)s->errC[b]})
      if (p) cudaFree(p);
  for (void* p : {(void*)s->K, (void*)s->res, (void*)s->rhsC, (void*)s->part, (void*)s->sums, (void*)s->force,
                  (void*)s->slice, (void*)s->dp})
    if (p) cudaFree(p);
  if (s->st) cudaStreamDestroy(s->st);
  delete s;
}

extern "C" const char* rq_mf_last_error(const rq_mf* s) { return s ? s->last_error.c_str() : "null"; }

extern "C" int rq_mf_step(rq_mf* s, int32_t n, float* sums) {
  if (!s || n < 0) return RQ_EINVAL;
  if (s->cfg.r_out_release_step >= 0 && s->r_out_enforce && s->t_step >= s->cfg.r_out_release_step) {
    s->r_out_enforce = false;  // mol_fast.js:1239-1243
    s->hp.R_out = 0.0f;
    int rc = mf_upload_params(s);
    if (rc != RQ_OK) return rc;
  }
  if (n > 0) {
    const auto key = std::make_pair((int)n, s->cur);
    auto it = s->graphs.find(key);
    if (it == s->graphs.end()) {  // a frame of n steps is one fixed launch sequence: captured once
      const long long l0 = s->launches;
      MCK(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
      int rc = mf_frame(s, n, s->cur);
      cudaGraph_t gr = nullptr;
      cudaError_t e = cudaStreamEndCapture(s->st, &gr);
      if (rc != RQ_OK) {
        if (gr) cudaGraphDestroy(gr);
        return rc;
      }
      MCK(e);
      cudaGraphExec_t ex = nullptr;
      e = cudaGraphInstantiate(&ex, gr, 0);
      cudaGraphDestroy(gr);
      MCK(e);
      it = s->graphs.emplace(key, std::make_pair(ex, s->launches - l0)).first;
      s->launches = l0;
    }
    MCK(cudaGraphLaunch(it->second.first, s->st));
    s->launches += it->second.second;
    s->cur ^= (n & 1);
    s->t_step += n;
  }
  if (sums) MCK(cudaMemcpyAsync(sums, s->sums, sizeof(float) * s->nr, cudaMemcpyDeviceToHost, s->st));
  MCK(cudaStreamSynchronize(s->st));
  return RQ_OK;
}

extern "C" int rq_mf_forces(rq_mf* s, float* F) {
  if (!s || !F) return RQ_EINVAL;
  k_mf_force<<<s->n, 256, 0, s->st>>>(s->dp, s->P[s->cur], s->force);
  MLAUNCH();
  MCK(cudaMemcpyAsync(F, s->force, sizeof(float) * 3 * s->n, cudaMemcpyDeviceToHost, s->st));
  MCK(cudaStreamSynchronize(s->st));
  return RQ_OK;
}

extern "C" int rq_mf_set_positions(rq_mf* s, const double* ijk) {
  if (!s || !ijk) return RQ_EINVAL;
  for (int a = 0; a < s->n; ++a) {
    s->nuc[a].i = ijk[3 * a]; s->nuc[a].j = ijk[3 * a + 1]; s->nuc[a].k = ijk[3 * a + 2];
    s->hp.atoms[a].x = (float)ijk[3 * a];
    s->hp.atoms[a].y = (float)ijk[3 * a + 1];
    s->hp.atoms[a].z = (float)ijk[3 * a + 2];
  }
  int rc = mf_upload_params(s);
  if (rc != RQ_OK) return rc;
  k_mf_recompute_k<<<(unsigned)((s->S3 + 255) / 256), 256, 0, s->st>>>(s->dp, s->K);
  MLAUNCH();
  MCK(cudaStreamSynchronize(s->st));
  return RQ_OK;
}

extern "C" int rq_mf_extract(rq_mf* s, float* out) {
  if (!s || !out) return RQ_EINVAL;
  const int c = s->cur;
  const unsigned g = (unsigned)((s->S + 15) / 16);
  k_mf_extract<<<dim3(g, g), dim3(16, 16), 0, s->st>>>(s->dp, s->U[c], s->W[c], s->P[c], s->slice);
  MLAUNCH();
  MCK(cudaMemcpyAsync(out, s->slice, sizeof(float) * 3 * (size_t)s->n * s->S * s->S, cudaMemcpyDeviceToHost, s->st));
  MCK(cudaStreamSynchronize(s->st));
  return RQ_OK;
}

extern "C" int rq_mf_download(rq_mf* s, int32_t m, float* U, float* W, float* P) {
  if (!s || m < 0 || m >= s->n) return RQ_EINVAL;
  const size_t S3 = (size_t)s->S3, off = (size_t)m * S3;
  const int c = s->cur;
  if (U) MCK(cudaMemcpyAsync(U, s->U[c] + off, sizeof(float) * S3, cudaMemcpyDeviceToHost, s->st));
  if (W) MCK(cudaMemcpyAsync(W, s->W[c] + off, sizeof(float) * S3, cudaMemcpyDeviceToHost, s->st));
  if (P) MCK(cudaMemcpyAsync(P, s->P[c] + off, sizeof(float) * S3, cudaMemcpyDeviceToHost, s->st));
  MCK(cudaStreamSynchronize(s->st));
  return RQ_OK;
}

extern "C" int rq_mf_upload(rq_mf* s, int32_t m, const float* U, const float* W, const float* P) {
  if (!s || m < 0 || m >= s->n) return RQ_EINVAL;
  const size_t S3 = (size_t)s->S3, off = (size_t)m * S3;
  for (int c = 0; c < 2; ++c) {  // both buffer sets, as uploadInitialData writes them
    if (U) MCK(cudaMemcpyAsync(s->U[c] + off, U, sizeof(float) * S3, cudaMemcpyHostToDevice, s->st));
    if (W) MCK(cudaMemcpyAsync(s->W[c] + off, W, sizeof(float) * S3, cudaMemcpyHostToDevice, s->st));
    if (P) MCK(cudaMemcpyAsync(s->P[c] + off, P, sizeof(float) * S3, cudaMemcpyHostToDevice, s->st));
  }
  MCK(cudaStreamSynchronize(s->st));
  return RQ_OK;
}

extern "C" int rq_mf_download_K(rq_mf* s, float* K) {
  if (!s || !K) return RQ_EINVAL;
  MCK(cudaMemcpyAsync(K, s->K, sizeof(float) * s->S3, cudaMemcpyDeviceToHost, s->st));
  MCK(cudaStreamSynchronize(s->st));
  return RQ_OK;
}

extern "C" int rq_mf_info(const rq_mf* s, int64_t* kernel_launches, int64_t* steps_done) {
  if (!s) return RQ_EINVAL;
  if (kernel_launches) *kernel_launches = s->launches;
  if (steps_done) *steps_done = s->t_step;
  return RQ_OK;
}
