// sp_kernels.cu -- the cloud/solver.py flavour of the solver step on sm_100a.
//
// Every kernel here restates one RawKernel of cloud/solver.py:16-315 with the same
// per-point arithmetic in the same order (explicitly rounded, never contracted), so
// single-kernel outputs are bit-identical to the reference kernel text compiled for
// the host.  What changes is the execution shape: interior-only 32x8-thread blocks
// that march 16 planes along i keeping the i-1/i/i+1 column in registers, rho = psi^2
// computed inside the Jacobi sweep instead of a separate pass, and FP64 per-domain sums
// aggregated per block instead of f32 scatter_add / atomics.
#include <algorithm>

#include "rq_kernels.h"

namespace rq {

// ---------------------------------------------------------------------------------------
// K1: ITP update (cloud/solver.py:61-90).  With ACC, also the FP64 norm of the NEW psi per
// label (cloud/solver.py:421-427, label clipped to [0, nDom)) for the normalisation step.
// Algorithmic traffic: read psi, label, K, P; write psi' = 20 B per interior point.
// ---------------------------------------------------------------------------------------
template <bool ACC>
__global__ void __launch_bounds__(256) k_update_sp(const float* __restrict__ U, float* __restrict__ Unew,
                                                   const float* __restrict__ K, const float* __restrict__ P,
                                                   const int* __restrict__ label, Geo g, float half_dv, float dtv,
                                                   double h3, int nDom, double* __restrict__ norms) {
  __shared__ DomTable<1, 128> tab;
  if (ACC) dom_table_init(tab);
  if (ACC) __syncthreads();
  RunSum<1> rs;
  rs.reset();
  const int k = 1 + blockIdx.x * kThreadsK + threadIdx.x;
  const int j = 1 + blockIdx.y * kThreadsJ + threadIdx.y;
  const int i0 = 1 + blockIdx.z * kMarch;
  if (k < g.NN && j < g.NN && i0 < g.NN) {
    const int iend = min(i0 + kMarch, g.NN);
    const long long S = g.S, S2 = g.S2;
    long long id = (long long)i0 * S2 + j * S + k;
    float u_m = __ldg(U + id - S2), u_c = __ldg(U + id);
    int l_m = __ldg(label + id - S2), l_c = __ldg(label + id);
    for (int i = i0; i < iend; ++i, id += S2) {
      const float u_p = __ldg(U + id + S2);
      const int l_p = __ldg(label + id + S2);
      const float ujp = __ldg(U + id + S), ujm = __ldg(U + id - S), ukp = __ldg(U + id + 1), ukm = __ldg(U + id - 1);
      const int ljp = __ldg(label + id + S), ljm = __ldg(label + id - S), lkp = __ldg(label + id + 1),
                lkm = __ldg(label + id - 1);
      const float kv = __ldg(K + id), pv = __ldg(P + id);
      const float a = (l_p == l_c) ? u_p : u_c;
      const float b = (l_m == l_c) ? u_m : u_c;
      const float c = (ljp == l_c) ? ujp : u_c;
      const float d = (ljm == l_c) ? ujm : u_c;
      const float e = (lkp == l_c) ? ukp : u_c;
      const float f = (lkm == l_c) ? ukm : u_c;
      const float lap = F_SUB(F_ADD(F_ADD(F_ADD(F_ADD(F_ADD(a, b), c), d), e), f), F_MUL(6.0f, u_c));
      const float out =
          F_ADD(F_ADD(u_c, F_MUL(half_dv, lap)), F_MUL(F_MUL(dtv, F_SUB(kv, F_MUL(2.0f, pv))), u_c));
      Unew[id] = out;
      if (ACC) {
        double r = (double)out * (double)out * h3;
        int lc = min(max(l_c, 0), nDom - 1);
        rs.add(lc, &r, tab, norms);
      }
      u_m = u_c; u_c = u_p; l_m = l_c; l_c = l_p;
    }
  }
  if (ACC) {
    rs.finish(tab, norms);
    __syncthreads();
    dom_table_flush(tab, norms);
  }
}

// ---------------------------------------------------------------------------------------
// Jacobi sweep fused with computeRho (cloud/solver.py:181-208):
// Pnew = (sum_6 P + coeff*(U*U)*h2)/6.  Traffic: read P, U; write Pnew = 12 B/point.
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_jacobi_sp(const float* __restrict__ P, float* __restrict__ Pnew,
                                                   const float* __restrict__ U, Geo g, float h2, float coeff) {
  const int k = 1 + blockIdx.x * kThreadsK + threadIdx.x;
  const int j = 1 + blockIdx.y * kThreadsJ + threadIdx.y;
  const int i0 = 1 + blockIdx.z * kMarch;
  if (k >= g.NN || j >= g.NN || i0 >= g.NN) return;
  const int iend = min(i0 + kMarch, g.NN);
  const long long S = g.S, S2 = g.S2;
  long long id = (long long)i0 * S2 + j * S + k;
  float p_m = __ldg(P + id - S2), p_c = __ldg(P + id);
  for (int i = i0; i < iend; ++i, id += S2) {
    const float p_p = __ldg(P + id + S2);
    const float u = __ldg(U + id);
    const float rho = F_MUL(u, u);
    const float sumN = F_ADD(F_ADD(F_ADD(F_ADD(F_ADD(p_p, p_m), __ldg(P + id + S)), __ldg(P + id - S)),
                                   __ldg(P + id + 1)),
                             __ldg(P + id - 1));
    Pnew[id] = F_DIV(F_ADD(sumN, F_MUL(F_MUL(coeff, rho), h2)), 6.0f);
    p_m = p_c; p_c = p_p;
  }
}

// ---------------------------------------------------------------------------------------
// One pass that does an ITP update and a Jacobi sweep together.  The update reads P only at
// the centre and the sweep reads psi only at the centre, so on a march both are local:
//   FIRST = false: Pnew = jacobi(P, rho = psi^2), then psi' = update(psi, Pnew)   (the last sweep
//                  of a Poisson step, then that step's update);
//   FIRST = true:  psi' = update(psi, P), then Pnew = jacobi(P, rho = psi'^2)     (a step's update,
//                  then the first sweep of the next step's Poisson solve).
// The per-point arithmetic is that of k_update_sp and k_jacobi_sp, so both outputs are
// bit-identical to the two separate kernels.  Traffic: read psi, label, K, P; write psi', P' =
// 24 B per interior point instead of 20 + 12.
// ---------------------------------------------------------------------------------------
template <bool FIRST, bool ACC>
__global__ void __launch_bounds__(256) k_step_sp(const float* __restrict__ U, float* __restrict__ Unew,
                                                 const float* __restrict__ K, const float* __restrict__ P,
                                                 float* __restrict__ Pnew, const int* __restrict__ label, Geo g,
                                                 float half_dv, float dtv, float h2, float coeff, double h3, int nDom,
                                                 double* __restrict__ norms) {
  __shared__ DomTable<1, 128> tab;
  if (ACC) dom_table_init(tab);
  if (ACC) __syncthreads();
  RunSum<1> rs;
  rs.reset();
  const int k = 1 + blockIdx.x * kThreadsK + threadIdx.x;
  const int j = 1 + blockIdx.y * kThreadsJ + threadIdx.y;
  const int i0 = 1 + blockIdx.z * kMarch;
  if (k < g.NN && j < g.NN && i0 < g.NN) {
    const int iend = min(i0 + kMarch, g.NN);
    const long long S = g.S, S2 = g.S2;
    long long id = (long long)i0 * S2 + j * S + k;
    float u_m = __ldg(U + id - S2), u_c = __ldg(U + id);
    int l_m = __ldg(label + id - S2), l_c = __ldg(label + id);
    float p_m = __ldg(P + id - S2), p_c = __ldg(P + id);
    for (int i = i0; i < iend; ++i, id += S2) {
      const float u_p = __ldg(U + id + S2), p_p = __ldg(P + id + S2);
      const int l_p = __ldg(label + id + S2);
      const float ujp = __ldg(U + id + S), ujm = __ldg(U + id - S), ukp = __ldg(U + id + 1), ukm = __ldg(U + id - 1);
      const int ljp = __ldg(label + id + S), ljm = __ldg(label + id - S), lkp = __ldg(label + id + 1),
                lkm = __ldg(label + id - 1);
      const float sumN = F_ADD(F_ADD(F_ADD(F_ADD(F_ADD(p_p, p_m), __ldg(P + id + S)), __ldg(P + id - S)),
                                     __ldg(P + id + 1)),
                               __ldg(P + id - 1));
      const float kv = __ldg(K + id);
      const float a = (l_p == l_c) ? u_p : u_c;
      const float b = (l_m == l_c) ? u_m : u_c;
      const float c = (ljp == l_c) ? ujp : u_c;
      const float d = (ljm == l_c) ? ujm : u_c;
      const float e = (lkp == l_c) ? ukp : u_c;
      const float f = (lkm == l_c) ? ukm : u_c;
      const float lap = F_SUB(F_ADD(F_ADD(F_ADD(F_ADD(F_ADD(a, b), c), d), e), f), F_MUL(6.0f, u_c));
      float pv = p_c;
      if (!FIRST) {
        pv = F_DIV(F_ADD(sumN, F_MUL(F_MUL(coeff, F_MUL(u_c, u_c)), h2)), 6.0f);
        Pnew[id] = pv;
      }
      const float out =
          F_ADD(F_ADD(u_c, F_MUL(half_dv, lap)), F_MUL(F_MUL(dtv, F_SUB(kv, F_MUL(2.0f, pv))), u_c));
      Unew[id] = out;
      if (FIRST) Pnew[id] = F_DIV(F_ADD(sumN, F_MUL(F_MUL(coeff, F_MUL(out, out)), h2)), 6.0f);
      if (ACC) {
        double r = (double)out * (double)out * h3;
        int lc = min(max(l_c, 0), nDom - 1);
        rs.add(lc, &r, tab, norms);
      }
      u_m = u_c; u_c = u_p; l_m = l_c; l_c = l_p; p_m = p_c; p_c = p_p;
    }
  }
  if (ACC) {
    rs.finish(tab, norms);
    __syncthreads();
    dom_table_flush(tab, norms);
  }
}

// ---------------------------------------------------------------------------------------
// Label step (cloud/solver.py:92-147) with snapshot semantics: reads labelIn, writes
// labelOut for interior points.  A boundary cell (>= 1 foreign neighbour) flips to the
// atom of largest Z/sqrt(r^2+h^2) when that beats the current atom's score by 10 % and
// >= 2 neighbours are foreign.  Pure integer outcome of IEEE f32 comparisons.
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_labels_sp(const int* __restrict__ labIn, int* __restrict__ labOut,
                                                   const float* __restrict__ atoms5, int nAtoms, Geo g, float h,
                                                   float h2) {
  const int k = 1 + blockIdx.x * kThreadsK + threadIdx.x;
  const int j = 1 + blockIdx.y * kThreadsJ + threadIdx.y;
  const int i0 = 1 + blockIdx.z * kMarch;
  if (k >= g.NN || j >= g.NN || i0 >= g.NN) return;
  const int iend = min(i0 + kMarch, g.NN);
  const long long S = g.S, S2 = g.S2;
  const float yj = F_MUL((float)j, h), zk = F_MUL((float)k, h);
  for (int i = i0; i < iend; ++i) {
    const long long id = (long long)i * S2 + j * S + k;
    const int cur = __ldg(labIn + id);
    int other = (__ldg(labIn + id + S2) != cur) + (__ldg(labIn + id - S2) != cur) + (__ldg(labIn + id + S) != cur) +
                (__ldg(labIn + id - S) != cur) + (__ldg(labIn + id + 1) != cur) + (__ldg(labIn + id - 1) != cur);
    int out = cur;
    if (other >= 2) {  // a cell with one foreign neighbour never flips: its argmax is not needed
      const float xi = F_MUL((float)i, h);
      float curScore = 0.f, bestScore = 0.f;
      int bestN = cur;
      for (int n = 0; n < nAtoms; ++n) {
        const float Za = __ldg(atoms5 + n * 5 + 3);
        if (Za <= 0.f) continue;
        const float dx = F_SUB(xi, F_MUL(__ldg(atoms5 + n * 5 + 0), h));
        const float dy = F_SUB(yj, F_MUL(__ldg(atoms5 + n * 5 + 1), h));
        const float dz = F_SUB(zk, F_MUL(__ldg(atoms5 + n * 5 + 2), h));
        const float r2 = F_ADD(F_ADD(F_ADD(F_MUL(dx, dx), F_MUL(dy, dy)), F_MUL(dz, dz)), h2);
        const float score = F_DIV(Za, F_SQRT(r2));
        if (n == cur) curScore = score;
        if (score > bestScore) { bestScore = score; bestN = n; }
      }
      if (bestN != cur && bestScore > F_MUL(curScore, 1.1f) && other >= 2) out = bestN;
    }
    labOut[id] = out;
  }
}

// The same label step with the argmax over atoms found through atom bins instead of a scan of
// every atom.  Candidate atoms are visited bin ring by bin ring around the cell (far list
// first); after ring r every unvisited atom is at least d_min away, so its score is at most
// zmax / sqrt(d_min^2 + h^2).  The search stops once that bound -- taken with an absolute
// 1e-3 bohr margin on d_min and a 1e-5 relative margin on the score, far above f32 rounding of
// the per-atom score -- is below the best score found.  Each candidate's score is the scan's
// expression, and ties go to the lower atom index (the scan keeps the first maximum), so the
// winner and its score are those of the scan.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ float sp_atom_score(const float* __restrict__ atoms5, int n, float xi, float yj, float zk,
                                               float h, float h2) {
  const float Za = __ldg(atoms5 + n * 5 + 3);
  const float dx = F_SUB(xi, F_MUL(__ldg(atoms5 + n * 5 + 0), h));
  const float dy = F_SUB(yj, F_MUL(__ldg(atoms5 + n * 5 + 1), h));
  const float dz = F_SUB(zk, F_MUL(__ldg(atoms5 + n * 5 + 2), h));
  const float r2 = F_ADD(F_ADD(F_ADD(F_MUL(dx, dx), F_MUL(dy, dy)), F_MUL(dz, dz)), h2);
  return F_DIV(Za, F_SQRT(r2));
}

__global__ void __launch_bounds__(256) k_labels_binned_sp(const int* __restrict__ labIn, int* __restrict__ labOut,
                                                          const float* __restrict__ atoms5, int nAtoms, AtomBins B,
                                                          Geo g, float h, float h2) {
  const int k = 1 + blockIdx.x * kThreadsK + threadIdx.x;
  const int j = 1 + blockIdx.y * kThreadsJ + threadIdx.y;
  const int i0 = 1 + blockIdx.z * kMarch;
  if (k >= g.NN || j >= g.NN || i0 >= g.NN) return;
  const int iend = min(i0 + kMarch, g.NN);
  const long long S = g.S, S2 = g.S2;
  const float yj = F_MUL((float)j, h), zk = F_MUL((float)k, h);
  const double zmax = (double)__ldg(B.zmax);
  for (int i = i0; i < iend; ++i) {
    const long long id = (long long)i * S2 + j * S + k;
    const int cur = __ldg(labIn + id);
    int other = (__ldg(labIn + id + S2) != cur) + (__ldg(labIn + id - S2) != cur) + (__ldg(labIn + id + S) != cur) +
                (__ldg(labIn + id - S) != cur) + (__ldg(labIn + id + 1) != cur) + (__ldg(labIn + id - 1) != cur);
    int out = cur;
    if (other >= 2) {
      const float xi = F_MUL((float)i, h);
      float curScore = 0.f;
      if (cur >= 0 && cur < nAtoms && __ldg(atoms5 + cur * 5 + 3) > 0.f)
        curScore = sp_atom_score(atoms5, cur, xi, yj, zk, h, h2);
      bool found = false;
      float bs = 0.f;
      int bn = cur;
      auto visit = [&](int n) {
        const float sc = sp_atom_score(atoms5, n, xi, yj, zk, h, h2);
        if (!found || sc > bs || (sc == bs && n < bn)) { bs = sc; bn = n; found = true; }
      };
      const int nfar = __ldg(B.far);
      for (int q = 0; q < nfar; ++q) visit(__ldg(B.far + 1 + q));
      const int c0[3] = {min(i / B.bin, B.nb - 1), min(j / B.bin, B.nb - 1), min(k / B.bin, B.nb - 1)};
      const int p[3] = {i, j, k};
      for (int r = 0; r < B.nb; ++r) {
        for (int a = max(c0[0] - r, 0); a <= min(c0[0] + r, B.nb - 1); ++a)
          for (int b = max(c0[1] - r, 0); b <= min(c0[1] + r, B.nb - 1); ++b) {
            const bool edge_ab = abs(a - c0[0]) == r || abs(b - c0[1]) == r;
            for (int c = max(c0[2] - r, 0); c <= min(c0[2] + r, B.nb - 1); ++c) {
              if (!edge_ab && abs(c - c0[2]) != r) continue;  // ring r only
              const int bin = (a * B.nb + b) * B.nb + c;
              for (int q = __ldg(B.start + bin); q < __ldg(B.start + bin + 1); ++q) visit(__ldg(B.idx + q));
            }
          }
        // distance (grid units) from the cell to the nearest unvisited bin
        double dmin = 1e30;
        for (int ax = 0; ax < 3; ++ax) {
          if (c0[ax] - r > 0) dmin = fmin(dmin, (double)(p[ax] - (c0[ax] - r) * B.bin));
          if (c0[ax] + r < B.nb - 1) dmin = fmin(dmin, (double)((c0[ax] + r + 1) * B.bin - p[ax]));
        }
        if (dmin >= 1e29) break;  // every bin visited
        const double d = fmax(dmin * (double)h - 1e-3, 0.0);
        if (found && zmax / sqrt(d * d + (double)h2) * (1.0 + 1e-5) < (double)bs) break;
      }
      if (found && bn != cur && bs > F_MUL(curScore, 1.1f)) out = bn;
    }
    labOut[id] = out;
  }
}

void build_atom_bins(const float* atoms5, int n, int nb, int bin, std::vector<int>& start, std::vector<int>& idx,
                     std::vector<int>& far, float& zmax) {
  const long long nbins = (long long)nb * nb * nb;
  start.assign(nbins + 1, 0);
  idx.assign(n, 0);
  far.assign(n + 1, 0);
  zmax = 0.f;
  std::vector<long long> where(n, -1);
  const double lim = (double)nb * bin;
  for (int q = 0; q < n; ++q) {
    const float* a = atoms5 + 5 * q;
    if (!(a[3] > 0.f)) continue;  // the scan skips atoms without charge
    zmax = std::max(zmax, a[3]);
    const double x = a[0], y = a[1], z = a[2];
    if (x >= 0 && y >= 0 && z >= 0 && x < lim && y < lim && z < lim) {
      where[q] = ((long long)(x / bin) * nb + (long long)(y / bin)) * nb + (long long)(z / bin);
      start[where[q] + 1]++;
    } else {
      far[1 + far[0]++] = q;
    }
  }
  for (long long b = 0; b < nbins; ++b) start[b + 1] += start[b];
  std::vector<int> fill(start.begin(), start.end() - 1);
  for (int q = 0; q < n; ++q)
    if (where[q] >= 0) idx[fill[where[q]]++] = q;
}

cudaError_t launch_labels_binned_sp(const int* labIn, int* labOut, const float* atoms5, int nAtoms, AtomBins bins,
                                    const Geo& g, float h, float h2, cudaStream_t st) {
  if (g.NN < 2) return cudaSuccess;
  k_labels_binned_sp<<<march_grid(g), march_block(), 0, st>>>(labIn, labOut, atoms5, nAtoms, bins, g, h, h2);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------
// Nuclear potential and trial state (cloud/solver.py:16-59, :149-179).  Atoms are staged
// through shared memory in chunks; all S^3 points are written (boundary = 0).
// ---------------------------------------------------------------------------------------
template <bool TRIAL>
__global__ void __launch_bounds__(256) k_init_sp(float* __restrict__ U, int* __restrict__ label, float* __restrict__ K,
                                                 float* __restrict__ bestU, const float* __restrict__ atoms5,
                                                 int nAtoms, Geo g, float h, float h2) {
  __shared__ float sa[256 * 5];
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool inside = id < g.S3;
  const int S = g.S;
  const int i = inside ? (int)(id / g.S2) : 0, j = inside ? (int)((id / S) % S) : 0, k = inside ? (int)(id % S) : 0;
  const bool interior = inside && i >= 1 && i < g.NN && j >= 1 && j < g.NN && k >= 1 && k < g.NN;
  const float xi = F_MUL((float)i, h), yj = F_MUL((float)j, h), zk = F_MUL((float)k, h);
  const float inv_sqrt_pi = 0.5641895835f;
  float bU = 0.f, Kval = 0.f;
  int bestN = 0;
  for (int base = 0; base < nAtoms; base += 256) {
    const int cnt = min(256, nAtoms - base);
    __syncthreads();
    for (int q = threadIdx.x; q < cnt * 5; q += blockDim.x) sa[q] = atoms5[base * 5 + q];
    __syncthreads();
    if (interior) {
      for (int m = 0; m < cnt; ++m) {
        const float Za = sa[m * 5 + 3];
        if (Za <= 0.f) continue;
        const float rc = sa[m * 5 + 4];
        const float dx = F_SUB(xi, F_MUL(sa[m * 5 + 0], h));
        const float dy = F_SUB(yj, F_MUL(sa[m * 5 + 1], h));
        const float dz = F_SUB(zk, F_MUL(sa[m * 5 + 2], h));
        const float r2 = F_ADD(F_ADD(F_MUL(dx, dx), F_MUL(dy, dy)), F_MUL(dz, dz));
        const float r = (rc > 0.f) ? fmaxf(F_SQRT(F_ADD(r2, F_MUL(0.04f, h2))), rc) : F_SQRT(F_ADD(r2, h2));
        Kval = F_ADD(Kval, F_DIV(Za, r));
        if (TRIAL) {
          const float uT = F_MUL(F_MUL(F_MUL(Za, Za), inv_sqrt_pi), expf(F_MUL(-Za, r)));
          if (uT > bU) { bU = uT; bestN = base + m; }
        }
      }
    }
  }
  if (!inside) return;
  K[id] = Kval;
  if (TRIAL) {
    bestU[id] = bU;
    label[id] = bestN;
    U[id] = bU;
  }
}

// ---------------------------------------------------------------------------------------
// Normalisation (cloud/solver.py:421-432, :210-225).
// ---------------------------------------------------------------------------------------
// FP64 per-label psi^2 h^3 over all S^3 points, label clipped to [0, nDom).
__global__ void __launch_bounds__(256) k_norms_flat(const float* __restrict__ U, const int* __restrict__ label,
                                                    long long S3, double h3, int nDom, double* __restrict__ norms) {
  __shared__ DomTable<1, 128> tab;
  dom_table_init(tab);
  __syncthreads();
  RunSum<1> rs;
  rs.reset();
  const long long per = 16;
  long long base = ((long long)blockIdx.x * blockDim.x) * per;
  for (long long q = 0; q < per; ++q) {
    long long id = base + q * blockDim.x + threadIdx.x;
    if (id >= S3) break;
    double u = U[id];
    double r = u * u * h3;
    int l = min(max(label[id], 0), nDom - 1);
    rs.add(l, &r, tab, norms);
  }
  rs.finish(tab, norms);
  __syncthreads();
  dom_table_flush(tab, norms);
}

// scale[l] = sqrt(Z_l / n_l) when Z_l > 0 and n_l > 1e-20 (f32 like the reference), else 1.
// A norm that is not finite as an f32 (NaN or Inf in the FP64 sum, or a finite sum above
// FLT_MAX) sets bit 0 of *err and leaves the domain unscaled: sqrt(z / inf) would zero it.
__global__ void k_norm_scale_sp(const double* __restrict__ norms, const float* __restrict__ Zeff, int nDom,
                                float* __restrict__ scale, int* __restrict__ err) {
  int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= nDom) return;
  const float z = Zeff[l];
  const float n = (float)norms[l];
  if (!isfinite(n)) {
    atomicOr(err, 1);
    scale[l] = 1.0f;
    return;
  }
  scale[l] = (z > 0.f && n > 1e-20f) ? F_SQRT(F_DIV(z, n)) : 1.0f;
}

// U *= scale[label] over all S^3 points; labels outside [0, nDom) are left unscaled.
__global__ void __launch_bounds__(256) k_apply_scale_sp(float* __restrict__ U, const int* __restrict__ label,
                                                        const float* __restrict__ scale, long long S3, int nDom) {
  long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  for (; id < S3; id += (long long)gridDim.x * blockDim.x) {
    int l = label[id];
    if (l < 0 || l >= nDom) continue;
    U[id] = F_MUL(U[id], scale[l]);
  }
}

// ---------------------------------------------------------------------------------------
// Energies per domain (cloud/solver.py:227-280 terms, FP64): (norm, T, V_eK, V_ee).
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_energy_sp(const float* __restrict__ U, const float* __restrict__ K,
                                                   const float* __restrict__ P, const int* __restrict__ label, Geo g,
                                                   double h, double h3, int nDom, double* __restrict__ pd) {
  __shared__ DomTable<4, 128> tab;
  dom_table_init(tab);
  __syncthreads();
  RunSum<4> rs;
  rs.reset();
  const int k = 1 + blockIdx.x * kThreadsK + threadIdx.x;
  const int j = 1 + blockIdx.y * kThreadsJ + threadIdx.y;
  const int i0 = 1 + blockIdx.z * kMarch;
  if (k < g.NN && j < g.NN && i0 < g.NN) {
    const int iend = min(i0 + kMarch, g.NN);
    const long long S = g.S, S2 = g.S2;
    for (int i = i0; i < iend; ++i) {
      const long long id = (long long)i * S2 + j * S + k;
      const double u = U[id], rho = u * u;
      const int L = label[id];
      const double a = (label[id + S2] == L) ? (double)U[id + S2] - u : 0.0;
      const double b = (label[id + S] == L) ? (double)U[id + S] - u : 0.0;
      const double c = (label[id + 1] == L) ? (double)U[id + 1] - u : 0.0;
      double v[4] = {rho * h3, 0.5 * (a * a + b * b + c * c) * h, -(double)K[id] * rho * h3,
                     (double)P[id] * rho * h3};
      rs.add(min(max(L, 0), nDom - 1), v, tab, pd);
    }
  }
  rs.finish(tab, pd);
  __syncthreads();
  dom_table_flush(tab, pd);
}

// ---------------------------------------------------------------------------------------
// Hellmann-Feynman forces (cloud/solver.py:282-315).  Each block stages a tile of interior
// points (x, y, z, rho) in shared memory and each thread owns one atom, so every pair is
// evaluated once with no per-pair atomics; partials are FP64, one atomic per block/atom.
// ---------------------------------------------------------------------------------------
constexpr int kForceTile = 512;
__global__ void __launch_bounds__(256) k_forces_hf_sp(const float* __restrict__ U, const float* __restrict__ atoms5,
                                                      int nAtoms, Geo g, float h, float h2, float h3,
                                                      double* __restrict__ F) {
  __shared__ float sx[kForceTile], sy[kForceTile], sz[kForceTile], sr[kForceTile];
  const int a = blockIdx.y * blockDim.x + threadIdx.x;
  const bool valid = a < nAtoms;
  const float Za = valid ? atoms5[a * 5 + 3] : 0.f;
  const float ax = valid ? F_MUL(atoms5[a * 5 + 0], h) : 0.f;
  const float ay = valid ? F_MUL(atoms5[a * 5 + 1], h) : 0.f;
  const float az = valid ? F_MUL(atoms5[a * 5 + 2], h) : 0.f;
  const long long n1 = g.NN - 1, nInt = n1 * n1 * n1;
  const long long ntiles = (nInt + kForceTile - 1) / kForceTile;
  double fx = 0, fy = 0, fz = 0;
  for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
    __syncthreads();
    for (int q = threadIdx.x; q < kForceTile; q += blockDim.x) {
      long long v = t * kForceTile + q;
      float rho = 0.f, x = 0.f, y = 0.f, z = 0.f;
      if (v < nInt) {
        int i = 1 + (int)(v / (n1 * n1)), j = 1 + (int)((v / n1) % n1), k = 1 + (int)(v % n1);
        float u = U[(long long)i * g.S2 + (long long)j * g.S + k];
        rho = F_MUL(u, u);
        if (rho < 1e-20f) rho = 0.f;
        x = F_MUL((float)i, h); y = F_MUL((float)j, h); z = F_MUL((float)k, h);
      }
      sx[q] = x; sy[q] = y; sz[q] = z; sr[q] = rho;
    }
    __syncthreads();
    if (valid && Za > 0.f) {
      float lx = 0.f, ly = 0.f, lz = 0.f;
      for (int q = 0; q < kForceTile; ++q) {
        const float rho = sr[q];
        const float dx = F_SUB(sx[q], ax), dy = F_SUB(sy[q], ay), dz = F_SUB(sz[q], az);
        const float r2 = F_ADD(F_ADD(F_ADD(F_MUL(dx, dx), F_MUL(dy, dy)), F_MUL(dz, dz)), h2);
        const float inv_r3 = F_DIV(1.0f, F_MUL(r2, F_SQRT(r2)));
        const float w = F_MUL(F_MUL(F_MUL(Za, rho), inv_r3), h3);
        lx += w * dx; ly += w * dy; lz += w * dz;
      }
      fx += lx; fy += ly; fz += lz;
    }
  }
  if (valid && Za > 0.f) {
    atomicAdd(&F[a * 3 + 0], fx);
    atomicAdd(&F[a * 3 + 1], fy);
    atomicAdd(&F[a * 3 + 2], fz);
  }
}

// ---------------------------------------------------------------------------------------
// Boundary faces to zero (Dirichlet planes the reference rewrites every step).
// ---------------------------------------------------------------------------------------
template <typename T>
__global__ void k_zero_faces(T* __restrict__ f, Geo g) {
  const long long n = g.S2;
  long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 6 * n) return;
  const int face = (int)(q / n);
  const long long r = q % n;
  const int a = (int)(r / g.S), b = (int)(r % g.S);
  int i, j, k;
  switch (face) {
    case 0: i = 0; j = a; k = b; break;
    case 1: i = g.NN; j = a; k = b; break;
    case 2: i = a; j = 0; k = b; break;
    case 3: i = a; j = g.NN; k = b; break;
    case 4: i = a; j = b; k = 0; break;
    default: i = a; j = b; k = g.NN; break;
  }
  f[(long long)i * g.S2 + (long long)j * g.S + k] = T(0);
}

// ======================================================================================
// host launchers
// ======================================================================================
cudaError_t launch_update_sp(const float* U, float* Unew, const float* K, const float* P, const int* label,
                             const Geo& g, float half_dv, float dtv, double h3, int nDom, double* norms,
                             cudaStream_t st) {
  if (g.NN < 2) return cudaSuccess;
  if (norms)
    k_update_sp<true><<<march_grid(g), march_block(), 0, st>>>(U, Unew, K, P, label, g, half_dv, dtv, h3, nDom,
                                                                norms);
  else
    k_update_sp<false><<<march_grid(g), march_block(), 0, st>>>(U, Unew, K, P, label, g, half_dv, dtv, h3, nDom,
                                                                 nullptr);
  return cudaGetLastError();
}

cudaError_t launch_jacobi_sp(const float* P, float* Pnew, const float* U, const Geo& g, float h2, float coeff,
                             cudaStream_t st) {
  if (g.NN < 2) return cudaSuccess;
  k_jacobi_sp<<<march_grid(g), march_block(), 0, st>>>(P, Pnew, U, g, h2, coeff);
  return cudaGetLastError();
}

cudaError_t launch_step_sp(bool first, const float* U, float* Unew, const float* K, const float* P, float* Pnew,
                           const int* label, const Geo& g, float half_dv, float dtv, float h2, float coeff, double h3,
                           int nDom, double* norms, cudaStream_t st) {
  if (g.NN < 2) return cudaSuccess;
  const dim3 grd = march_grid(g), blk = march_block();
  if (first && norms)
    k_step_sp<true, true><<<grd, blk, 0, st>>>(U, Unew, K, P, Pnew, label, g, half_dv, dtv, h2, coeff, h3, nDom, norms);
  else if (first)
    k_step_sp<true, false><<<grd, blk, 0, st>>>(U, Unew, K, P, Pnew, label, g, half_dv, dtv, h2, coeff, h3, nDom,
                                                nullptr);
  else if (norms)
    k_step_sp<false, true><<<grd, blk, 0, st>>>(U, Unew, K, P, Pnew, label, g, half_dv, dtv, h2, coeff, h3, nDom,
                                                norms);
  else
    k_step_sp<false, false><<<grd, blk, 0, st>>>(U, Unew, K, P, Pnew, label, g, half_dv, dtv, h2, coeff, h3, nDom,
                                                 nullptr);
  return cudaGetLastError();
}

cudaError_t launch_labels_sp(const int* labIn, int* labOut, const float* atoms5, int nAtoms, const Geo& g, float h,
                             float h2, cudaStream_t st) {
  if (g.NN < 2) return cudaSuccess;
  k_labels_sp<<<march_grid(g), march_block(), 0, st>>>(labIn, labOut, atoms5, nAtoms, g, h, h2);
  return cudaGetLastError();
}

cudaError_t launch_init_sp(float* U, int* label, float* K, float* bestU, const float* atoms5, int nAtoms,
                           const Geo& g, float h, float h2, bool trial, cudaStream_t st) {
  const unsigned blocks = (unsigned)((g.S3 + 255) / 256);
  if (trial)
    k_init_sp<true><<<blocks, 256, 0, st>>>(U, label, K, bestU, atoms5, nAtoms, g, h, h2);
  else
    k_init_sp<false><<<blocks, 256, 0, st>>>(U, label, K, bestU, atoms5, nAtoms, g, h, h2);
  return cudaGetLastError();
}

cudaError_t launch_norms_flat(const float* U, const int* label, const Geo& g, double h3, int nDom, double* norms,
                              cudaStream_t st) {
  const long long per = 16 * 256;
  const unsigned blocks = (unsigned)((g.S3 + per - 1) / per);
  k_norms_flat<<<blocks, 256, 0, st>>>(U, label, g.S3, h3, nDom, norms);
  return cudaGetLastError();
}

cudaError_t launch_norm_scale_sp(const double* norms, const float* Zeff, int nDom, float* scale, int* err,
                                 cudaStream_t st) {
  k_norm_scale_sp<<<(nDom + 127) / 128, 128, 0, st>>>(norms, Zeff, nDom, scale, err);
  return cudaGetLastError();
}

cudaError_t launch_apply_scale_sp(float* U, const int* label, const float* scale, const Geo& g, int nDom,
                                  cudaStream_t st) {
  long long blocks = (g.S3 + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_apply_scale_sp<<<(unsigned)blocks, 256, 0, st>>>(U, label, scale, g.S3, nDom);
  return cudaGetLastError();
}

cudaError_t launch_energy_sp(const float* U, const float* K, const float* P, const int* label, const Geo& g, double h,
                             double h3, int nDom, double* pd, cudaStream_t st) {
  if (g.NN < 2) return cudaSuccess;
  k_energy_sp<<<march_grid(g), march_block(), 0, st>>>(U, K, P, label, g, h, h3, nDom, pd);
  return cudaGetLastError();
}

cudaError_t launch_forces_hf_sp(const float* U, const float* atoms5, int nAtoms, const Geo& g, float h, float h2,
                                float h3, double* F, cudaStream_t st) {
  if (g.NN < 2 || nAtoms <= 0) return cudaSuccess;
  const long long n1 = g.NN - 1, nInt = n1 * n1 * n1;
  const long long ntiles = (nInt + kForceTile - 1) / kForceTile;
  const int chunks = (nAtoms + 255) / 256;
  long long bx = 148 * 8 / chunks;
  if (bx < 1) bx = 1;
  if (bx > ntiles) bx = ntiles;
  k_forces_hf_sp<<<dim3((unsigned)bx, (unsigned)chunks), 256, 0, st>>>(U, atoms5, nAtoms, g, h, h2, h3, F);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_zero_faces(T* f, const Geo& g, cudaStream_t st) {
  const long long n = 6 * g.S2;
  k_zero_faces<T><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(f, g);
  return cudaGetLastError();
}
template cudaError_t launch_zero_faces<float>(float*, const Geo&, cudaStream_t);
template cudaError_t launch_zero_faces<double>(double*, const Geo&, cudaStream_t);

}  // namespace rq
