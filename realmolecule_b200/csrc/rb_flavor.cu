// rb_flavor.cu -- the realqm_rb.js red-black multi-field solver (rq_rb_*): one U (density
// amplitude), W (front) and P (Hartree potential of the others) field per electron, updated in
// place by red-black colouring (realqm_rb.js:1-1222).
//
// The reference launches one pass per electron for every stage of a step (uNearest, red W+U,
// red P, black W+U, black P).  The electrons of a colour touch disjoint data -- W+U of m writes
// u_m, w_m; P of m reads u_m at the cell itself, the precomputed rho_total and P_m of the other
// colour -- so one thread here owns a cell of the colour and runs W+U then P for every electron.
// The per-step rho_total and competitor max come from one pass (the competitor of electron m is
// the cell's largest u unless m holds it, then the second largest: exact selections, equal to the
// reference's max chain).  A step is three launches; a frame is one CUDA graph.  The f32
// arithmetic is the shaders' in their order (explicit round-to-nearest operations); the norm
// reduction keeps the reference's grid-stride partial sums and workgroup trees, so the scales are
// the reference's; the energies are the host formula in FP64.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/rq.h"
#include "rq_internal.cuh"

namespace rq {

constexpr int kRbMax = 16;
constexpr int kRbTK = 32, kRbTJ = 8;  // a block: 32 cells of one colour along k (64 k) x 8 j

struct RbParams {
  int NN, S, N2, n;
  float h, h2, inv_h, inv_h2, dt, half_d, two_pi, h3;
  float self_frac[kRbMax];  // 1/selfN for selfN > 1, else 1 (updateP_RB_WGSL)
  int masked[kRbMax];       // the electron's nucleus has an r_c exclusion mask
};

struct RbCell {
  long long id;
  int i, j, k;
};

// the thread's cell of colour `color` in plane blockIdx.z + 1; false when outside the interior
__device__ __forceinline__ bool rb_cell(const RbParams& p, int color, RbCell& c) {
  c.i = blockIdx.z + 1;
  c.j = blockIdx.y * kRbTJ + threadIdx.y + 1;
  const int k0 = 1 + ((c.i + c.j + 1 + color) & 1);  // (i + j + k0) % 2 == color
  c.k = k0 + 2 * (blockIdx.x * kRbTK + threadIdx.x);
  if (c.j >= p.NN || c.k >= p.NN) return false;
  c.id = (long long)c.i * p.S * p.S + (long long)c.j * p.S + c.k;
  return true;
}

// rhoTotal (realqm_rb.js:190-215) and the inputs of uNearest (:225-251): per interior cell
// (rho_total, largest u, second largest u, index of the largest)
__global__ void __launch_bounds__(256) k_rb_rho_top2(const RbParams p, const float* __restrict__ U,
                                                     float4* __restrict__ top) {
  const int k = blockIdx.x * 32 + threadIdx.x + 1, j = blockIdx.y * 8 + threadIdx.y + 1, i = blockIdx.z + 1;
  if (k >= p.NN || j >= p.NN) return;
  const long long S3 = (long long)p.S * p.S * p.S;
  const long long id = (long long)i * p.S * p.S + (long long)j * p.S + k;
  float rho = 0.0f, m1 = -INFINITY, m2 = -INFINITY;
  int a1 = -1;
  for (int q = 0; q < p.n; ++q) {
    const float u = __ldg(U + q * S3 + id);
    rho = q == 0 ? F_MUL(u, u) : F_ADD(rho, F_MUL(u, u));
    if (u > m1) { m2 = m1; m1 = u; a1 = q; }
    else if (u > m2) m2 = u;
  }
  top[id] = make_float4(rho, m1, m2, __int_as_float(a1));
}

// fusedWU_RB_WGSL (:256-311) then updateP_RB_WGSL (:318-353) of every electron on one cell of
// the colour, in place
__global__ void __launch_bounds__(256) k_rb_color(const RbParams p, int color, float* __restrict__ U,
                                                  float* __restrict__ W, float* __restrict__ P,
                                                  const float* __restrict__ K, const float4* __restrict__ top,
                                                  const unsigned char* __restrict__ mask) {
  RbCell c;
  if (!rb_cell(p, color, c)) return;
  const long long S = p.S, S2 = S * S, S3 = S2 * S;
  const float4 t = top[c.id];
  const int a1 = __float_as_int(t.w);
  const float Kc = __ldg(K + c.id);
  const float dt = p.dt, inv_h = p.inv_h, inv_h2 = p.inv_h2;
  const float dt05 = F_MUL(0.5f, dt), dt10 = F_MUL(10.0f, dt);
  for (int m = 0; m < p.n; ++m) {
    float* u = U + m * S3 + c.id;
    float* w = W + m * S3 + c.id;
    float* Pm = P + m * S3 + c.id;
    const float un = m == a1 ? t.z : t.y;
    const float uc = *u;
    const float cc = F_MUL(0.1f, F_SUB(uc, un));
    const float wc = *w;
    const float wxp = w[S2], wxm = w[-S2], wyp = w[S], wym = w[-S], wzp = w[1], wzm = w[-1];
    const float lap_w = F_SUB(F_ADD(F_ADD(F_ADD(F_ADD(F_ADD(wxp, wxm), wyp), wym), wzp), wzm), F_MUL(6.0f, wc));
    const float gwx = F_MUL(F_SUB(wxp, wxm), inv_h), gwy = F_MUL(F_SUB(wyp, wym), inv_h),
                gwz = F_MUL(F_SUB(wzp, wzm), inv_h);
    const float grad_w = F_SQRT(F_ADD(F_ADD(F_MUL(gwx, gwx), F_MUL(gwy, gwy)), F_MUL(gwz, gwz)));
    const float wc2 = F_ADD(F_ADD(wc, F_MUL(F_MUL(F_MUL(dt05, fabsf(cc)), lap_w), inv_h2)), F_MUL(F_MUL(dt10, cc), grad_w));
    const float fxp = F_MUL(F_MUL(F_SUB(u[S2], uc), F_ADD(wxp, wc2)), 0.5f);
    const float fxm = F_MUL(F_MUL(F_SUB(uc, u[-S2]), F_ADD(wc2, wxm)), 0.5f);
    const float fyp = F_MUL(F_MUL(F_SUB(u[S], uc), F_ADD(wyp, wc2)), 0.5f);
    const float fym = F_MUL(F_MUL(F_SUB(uc, u[-S]), F_ADD(wc2, wym)), 0.5f);
    const float fzp = F_MUL(F_MUL(F_SUB(u[1], uc), F_ADD(wzp, wc2)), 0.5f);
    const float fzm = F_MUL(F_MUL(F_SUB(uc, u[-1]), F_ADD(wc2, wzm)), 0.5f);
    const float wlap = F_ADD(F_ADD(F_SUB(fxp, fxm), F_SUB(fyp, fym)), F_SUB(fzp, fzm));
    const float Pc = *Pm;
    float un_new = F_ADD(F_ADD(uc, F_MUL(p.half_d, wlap)), F_MUL(F_MUL(F_MUL(dt, F_SUB(Kc, F_MUL(2.0f, Pc))), uc), wc2));
    float wn_new = wc2;
    if (p.masked[m]) {
      const float mk = mask[m * S3 + c.id] ? 1.0f : 0.0f;
      un_new = F_MUL(un_new, mk);
      wn_new = F_MUL(wn_new, mk);
    }
    *u = un_new;
    *w = wn_new;
    const float lap = F_SUB(F_ADD(F_ADD(F_ADD(F_ADD(F_ADD(Pm[S2], Pm[-S2]), Pm[S]), Pm[-S]), Pm[1]), Pm[-1]), F_MUL(6.0f, Pc));
    const float ro = fmaxf(F_SUB(t.x, F_MUL(F_MUL(p.self_frac[m], un_new), un_new)), 0.0f);
    *Pm = F_ADD(Pc, F_MUL(dt, F_ADD(F_MUL(lap, inv_h2), F_MUL(p.two_pi, ro))));
  }
}

// reduceNormWGSL (:356-394): blockIdx.y = electron; nwg blocks of 128 threads, each thread a
// grid-stride f32 sum over the interior cells in linear order, then the workgroup tree
__global__ void __launch_bounds__(128) k_rb_norm_partial(const RbParams p, const float* __restrict__ U,
                                                         float* __restrict__ part) {
  __shared__ float sd[128];
  const int m = blockIdx.y, lid = threadIdx.x;
  const long long NM = p.NN - 1, tot = NM * NM * NM, stride = (long long)gridDim.x * 128;
  const long long S = p.S, S2 = S * S, S3 = S2 * S;
  const float* u = U + m * S3;
  float acc = 0.0f;
  for (long long cell = (long long)blockIdx.x * 128 + lid; cell < tot; cell += stride) {
    const int k = (int)(cell % NM) + 1, j = (int)((cell / NM) % NM) + 1, i = (int)(cell / (NM * NM)) + 1;
    const float v = __ldg(u + (long long)i * S2 + (long long)j * S + k);
    acc = F_ADD(acc, F_MUL(F_MUL(v, v), p.h3));
  }
  sd[lid] = acc;
  __syncthreads();
  for (int s = 64; s > 0; s >>= 1) {
    if (lid < s) sd[lid] = F_ADD(sd[lid], sd[lid + s]);
    __syncthreads();
  }
  if (lid == 0) part[m * gridDim.x + blockIdx.x] = sd[0];
}

// normalizeWGSL's sum of the partials (:398-422), once per electron: norm and scale
__global__ void k_rb_norm_scale(const RbParams p, const float* __restrict__ part, int nwg,
                                const float* __restrict__ tgt, float2* __restrict__ scale) {
  const int m = threadIdx.x;
  if (m >= p.n) return;
  float norm = 0.0f;
  for (int q = 0; q < nwg; ++q) norm = F_ADD(norm, part[m * nwg + q]);
  scale[m] = make_float2(norm, norm > 0.0f ? F_SQRT(F_DIV(tgt[m], norm)) : 1.0f);
}

__global__ void __launch_bounds__(256) k_rb_normalize(const RbParams p, float* __restrict__ U,
                                                      const float2* __restrict__ scale) {
  const int k = blockIdx.x * 32 + threadIdx.x + 1, j = blockIdx.y * 8 + threadIdx.y + 1, i = blockIdx.z + 1;
  if (k >= p.NN || j >= p.NN) return;
  const long long S3 = (long long)p.S * p.S * p.S;
  const long long id = (long long)i * p.S * p.S + (long long)j * p.S + k;
  for (int m = 0; m < p.n; ++m) {
    const float2 sc = scale[m];
    if (sc.x > 0.0f) U[m * S3 + id] = F_MUL(U[m * S3 + id], sc.y);
  }
}

// computeEnergy (:982-1045) in FP64 (h, h3 the page's f64 spacing): acc = {E_T, E_eK, E_ee}
__global__ void __launch_bounds__(256) k_rb_energy(const RbParams p, const float* __restrict__ U,
                                                   const float* __restrict__ W, const float* __restrict__ P,
                                                   const float* __restrict__ K, double h, double h3,
                                                   double* __restrict__ acc) {
  __shared__ double red[3][256];
  const int k = blockIdx.x * 32 + threadIdx.x + 1, j = blockIdx.y * 8 + threadIdx.y + 1, i = blockIdx.z + 1;
  const int tid = threadIdx.y * 32 + threadIdx.x;
  double eT = 0, eK = 0, eE = 0;
  if (k < p.NN && j < p.NN) {
    const long long S = p.S, S2 = S * S, S3 = S2 * S;
    const long long id = (long long)i * S2 + (long long)j * S + k;
    const double Kc = K[id];
    for (int m = 0; m < p.n; ++m) {
      const float* u = U + m * S3 + id;
      const float* w = W + m * S3 + id;
      const double v = u[0], rho = __dmul_rn(v, v);
      if ((double)w[0] > 0.1) {
        double g2 = 0;
        if ((double)w[S2] > 0.1) { const double g = __dsub_rn((double)u[S2], v); g2 = __dadd_rn(g2, __dmul_rn(g, g)); }
        if ((double)w[S] > 0.1) { const double g = __dsub_rn((double)u[S], v); g2 = __dadd_rn(g2, __dmul_rn(g, g)); }
        if ((double)w[1] > 0.1) { const double g = __dsub_rn((double)u[1], v); g2 = __dadd_rn(g2, __dmul_rn(g, g)); }
        eT += __dmul_rn(__dmul_rn(0.5, g2), h);
      }
      eK += __dmul_rn(__dmul_rn(-Kc, rho), h3);
      eE += __dmul_rn(__dmul_rn((double)P[m * S3 + id], rho), h3);
    }
  }
  red[0][tid] = eT; red[1][tid] = eK; red[2][tid] = eE;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (tid < s)
      for (int q = 0; q < 3; ++q) red[q][tid] += red[q][tid + s];
    __syncthreads();
  }
  if (tid < 3) atomicAdd(acc + tid, red[tid][0]);
}

// extractSliceWGSL (:429-457): per pixel (i, j) of the k = N2 plane u, w, P of every electron, then K
__global__ void __launch_bounds__(256) k_rb_slice(const RbParams p, const float* __restrict__ U,
                                                  const float* __restrict__ W, const float* __restrict__ P,
                                                  const float* __restrict__ K, float* __restrict__ out) {
  const int N1 = p.S;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= N1 * N1) return;
  const int j = g / N1, i = g % N1;
  const long long S2 = (long long)p.S * p.S, S3 = S2 * p.S;
  const long long id = (long long)i * S2 + (long long)j * p.S + p.N2;
  const int stride = 3 * p.n + 1;
  for (int m = 0; m < p.n; ++m) {
    out[(long long)g * stride + 3 * m] = U[m * S3 + id];
    out[(long long)g * stride + 3 * m + 1] = W[m * S3 + id];
    out[(long long)g * stride + 3 * m + 2] = P[m * S3 + id];
  }
  out[(long long)g * stride + stride - 1] = K[id];
}

// ---- initial state (runInitKernels, :720-801, with the init shader :104-186) -----------------
struct RbNucDev {
  float i, j, k, Z, rc;
  int ne;
};

// K accumulated nucleus by nucleus at the interior cells (f32, in the reference's order)
__global__ void __launch_bounds__(256) k_rb_init_k(const RbParams p, const RbNucDev* __restrict__ nuc, int nn,
                                                   float* __restrict__ K) {
  const int k = blockIdx.x * 32 + threadIdx.x + 1, j = blockIdx.y * 8 + threadIdx.y + 1, i = blockIdx.z + 1;
  if (k >= p.NN || j >= p.NN) return;
  const long long id = (long long)i * p.S * p.S + (long long)j * p.S + k;
  float Kv = K[id];
  const float soft = F_MUL(1.2f, p.h2);
  for (int a = 0; a < nn; ++a) {
    const RbNucDev c = nuc[a];
    const float dx = F_MUL(F_SUB((float)i, c.i), p.h), dy = F_MUL(F_SUB((float)j, c.j), p.h),
                dz = F_MUL(F_SUB((float)k, c.k), p.h);
    const float r2 = F_ADD(F_ADD(F_MUL(dx, dx), F_MUL(dy, dy)), F_MUL(dz, dz));
    Kv = F_ADD(Kv, F_DIV(c.Z, F_SQRT(F_ADD(r2, soft))));
  }
  K[id] = Kv;
}

// electron m's u, w, P on its Voronoi cell (blockIdx.z = i-1 + NM m)
__global__ void __launch_bounds__(256) k_rb_init_fields(const RbParams p, const RbNucDev* __restrict__ nuc, int nn,
                                                        const int* __restrict__ enuc, float* __restrict__ U,
                                                        float* __restrict__ W, float* __restrict__ P) {
  const int NM = p.NN - 1;
  const int k = blockIdx.x * 32 + threadIdx.x + 1, j = blockIdx.y * 8 + threadIdx.y + 1;
  const int i = blockIdx.z % NM + 1, m = blockIdx.z / NM;
  if (k >= p.NN || j >= p.NN) return;
  const long long S3 = (long long)p.S * p.S * p.S;
  const long long id = (long long)i * p.S * p.S + (long long)j * p.S + k;
  const int a = enuc[m];
  const RbNucDev c = nuc[a];
  int sib = 0;
  for (int q = 0; q < m; ++q) sib += enuc[q] == a;
  const int splitDir = c.ne == 1 ? 2 : (sib == 0 ? 0 : 1);
  const float dx = F_MUL(F_SUB((float)i, c.i), p.h), dy = F_MUL(F_SUB((float)j, c.j), p.h),
              dz = F_MUL(F_SUB((float)k, c.k), p.h);
  const float r2 = F_ADD(F_ADD(F_MUL(dx, dx), F_MUL(dy, dy)), F_MUL(dz, dz));
  const float r_soft = F_SQRT(F_ADD(r2, F_MUL(1.2f, p.h2)));
  const float r_au = F_SQRT(r2);
  bool inV = true;
  int nriv = 0;
  for (int b = 0; b < nn && nriv < 8; ++b) {  // the first 8 other nuclei (MAX_RIVALS)
    if (b == a) continue;
    ++nriv;
    const RbNucDev r = nuc[b];
    const float ex = F_MUL(F_SUB((float)i, r.i), p.h), ey = F_MUL(F_SUB((float)j, r.j), p.h),
                ez = F_MUL(F_SUB((float)k, r.k), p.h);
    if (r2 > F_ADD(F_ADD(F_MUL(ex, ex), F_MUL(ey, ey)), F_MUL(ez, ez))) inV = false;
  }
  const bool inRc = c.rc <= 0.0f || r_au < c.rc;
  const bool inSplit = splitDir == 2 ? true : (splitDir == 0 ? (unsigned)i < (unsigned)(p.N2 - 1) : (unsigned)i > (unsigned)(p.N2 + 1));
  const bool inSph = r_au < 3.0f;
  if (inV && inSplit && inRc && inSph) W[m * S3 + id] = 1.0f;
  if (inV && inSplit && inSph) U[m * S3 + id] = (float)exp((double)F_MUL(F_MUL(-0.5f, c.Z), r_soft));
  P[m * S3 + id] = F_DIV(0.5f, r_soft);
}

// the r_c exclusion mask (realqm_rb.js:522-542, in JS numbers) of electron blockIdx.y around its
// nucleus' grid point; the initial u and w are zeroed inside it (:617-644)
__global__ void k_rb_init_mask(const RbParams p, const double* __restrict__ excl, float* __restrict__ U,
                               float* __restrict__ W, unsigned char* __restrict__ mask) {
  const int m = blockIdx.y;
  const double* e = excl + 5 * m;  // {rc_excl, i, j, k, rcCells}
  const double rc = e[0];
  if (!(rc > 0)) return;
  const int rcc = (int)e[4], side = 2 * rcc + 1;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)side * side * side) return;
  const int di = (int)(t / ((long long)side * side)) - rcc, dj = (int)((t / side) % side) - rcc, dk = (int)(t % side) - rcc;
  const double gi = e[1] + di, gj = e[2] + dj, gk = e[3] + dk;
  if (gi < 0 || gi >= p.S || gj < 0 || gj >= p.S || gk < 0 || gk >= p.S) return;
  const double hd = excl[5 * kRbMax];  // the page's f64 spacing
  const double x = __dmul_rn((double)di, hd), y = __dmul_rn((double)dj, hd), z = __dmul_rn((double)dk, hd);
  const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
  if (r2 < __dmul_rn(rc, rc)) {
    const long long S3 = (long long)p.S * p.S * p.S;
    const long long id = (long long)gi * p.S * p.S + (long long)gj * p.S + (long long)gk;
    mask[m * S3 + id] = 0;
    U[m * S3 + id] = 0.0f;
    W[m * S3 + id] = 0.0f;
  }
}

}  // namespace rq

using namespace rq;

struct rq_rb {
  rq_rb_config cfg{};
  std::vector<rq_rb_nucleus> nuc;
  std::vector<int> enuc;
  std::vector<double> tgt;
  int n = 0, nwg = 0;
  long long S3 = 0;
  double h = 0;
  RbParams p{};
  float *U = nullptr, *W = nullptr, *P = nullptr, *K = nullptr, *part = nullptr, *tgt_d = nullptr, *slice = nullptr;
  float4* top = nullptr;
  float2* scale = nullptr;
  unsigned char* mask = nullptr;
  double* acc = nullptr;
  long long t_step = 0, launches = 0;
  cudaStream_t st = nullptr;
  std::map<int, std::pair<cudaGraphExec_t, long long>> graphs;
  std::string last_error;
};

#define BCK(call)                                                          \
  do {                                                                     \
    cudaError_t _e = (call);                                               \
    if (_e != cudaSuccess) {                                               \
      s->last_error = std::string(#call) + ": " + cudaGetErrorString(_e);  \
      return _e == cudaErrorMemoryAllocation ? RQ_ENOMEM : RQ_ECUDA;       \
    }                                                                      \
  } while (0)
#define BLAUNCH() BCK(cudaGetLastError()); s->launches++

namespace {

dim3 rb_cells_grid(int NN, int planes) {
  const int NM = NN - 1;
  return dim3((NM + 31) / 32, (NM + 7) / 8, planes);
}

dim3 rb_color_grid(int NN) {  // 32 threads cover 64 consecutive k
  const int NM = NN - 1;
  return dim3((NM + 2 * kRbTK - 1) / (2 * kRbTK), (NM + kRbTJ - 1) / kRbTJ, NM);
}

// doSteps(n) (realqm_rb.js:891-965): per step rho/competitor, the red pass, the black pass, and
// the normalisation of every electron when the frame-local step index is a multiple of 5
int rb_frame(rq_rb* s, int n) {
  const int NN = s->cfg.NN;
  for (int q = 0; q < n; ++q) {
    k_rb_rho_top2<<<rb_cells_grid(NN, NN - 1), dim3(32, 8), 0, s->st>>>(s->p, s->U, s->top);
    BLAUNCH();
    for (int color = 0; color < 2; ++color) {
      k_rb_color<<<rb_color_grid(NN), dim3(kRbTK, kRbTJ), 0, s->st>>>(s->p, color, s->U, s->W, s->P, s->K, s->top, s->mask);
      BLAUNCH();
    }
    if (q % 5 == 0) {
      k_rb_norm_partial<<<dim3(s->nwg, s->n), 128, 0, s->st>>>(s->p, s->U, s->part);
      BLAUNCH();
      k_rb_norm_scale<<<1, 32, 0, s->st>>>(s->p, s->part, s->nwg, s->tgt_d, s->scale);
      BLAUNCH();
      k_rb_normalize<<<rb_cells_grid(NN, NN - 1), dim3(32, 8), 0, s->st>>>(s->p, s->U, s->scale);
      BLAUNCH();
    }
  }
  return RQ_OK;
}

}  // namespace

extern "C" int rq_rb_create(const rq_rb_config* cfg, const rq_rb_nucleus* nuclei, int32_t n_nuclei,
                            const double* norm_targets, rq_rb** out) {
  if (!cfg || !nuclei || !out || n_nuclei < 1) return RQ_EINVAL;
  *out = nullptr;
  if (cfg->NN < 8 || !(cfg->screen > 0)) return RQ_EINVAL;
  int nel = 0;
  for (int a = 0; a < n_nuclei; ++a) {
    if (nuclei[a].ne < 0) return RQ_EINVAL;
    nel += nuclei[a].ne;
  }
  if (nel < 2 || nel > kRbMax) return RQ_EINVAL;  // the competitor needs another electron
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return RQ_ENODEV;
  rq_rb* s = new (std::nothrow) rq_rb();
  if (!s) return RQ_ENOMEM;
  s->cfg = *cfg;
  s->nuc.assign(nuclei, nuclei + n_nuclei);
  for (int a = 0; a < n_nuclei; ++a)
    for (int e = 0; e < nuclei[a].ne; ++e) s->enuc.push_back(a);
  s->n = nel;
  for (int m = 0; m < nel; ++m) s->tgt.push_back(norm_targets ? norm_targets[m] : (double)nuclei[s->enuc[m]].ne);
  const int NN = cfg->NN, S = NN + 1;
  s->S3 = (long long)S * S * S;
  s->h = cfg->screen / NN;
  const long long NM = NN - 1, tot = NM * NM * NM;
  s->nwg = (int)std::min<long long>(256, (tot + 127) / 128);
  RbParams& p = s->p;
  const double h = s->h, h2 = h * h, h3 = h * h * h, dv = 0.1;
  p.NN = NN; p.S = S; p.N2 = (int)std::floor(NN / 2.0); p.n = nel;
  p.dt = (float)(dv * h2); p.half_d = (float)(0.5 * dv); p.two_pi = (float)(2 * M_PI);
  p.h = (float)h; p.h2 = (float)h2; p.inv_h = (float)(1 / h); p.inv_h2 = (float)(1 / h2); p.h3 = (float)h3;
  for (int m = 0; m < nel; ++m) {
    const float selfN = (float)s->tgt[m];
    p.self_frac[m] = selfN > 1.0f ? 1.0f / selfN : 1.0f;
    p.masked[m] = nuclei[s->enuc[m]].rc_excl > 0;
  }
  auto fail = [&](int rc) {
    std::fprintf(stderr, "rq_rb_create: %s\n", s->last_error.c_str());
    rq_rb_destroy(s);
    return rc;
  };
  auto alloc = [&](void** ptr, size_t bytes) -> int {
    if (cudaMalloc(ptr, bytes) != cudaSuccess) { s->last_error = "cudaMalloc"; return RQ_ENOMEM; }
    if (cudaMemset(*ptr, 0, bytes) != cudaSuccess) { s->last_error = "cudaMemset"; return RQ_ECUDA; }
    return RQ_OK;
  };
  const size_t fld = sizeof(float) * (size_t)s->S3 * nel;
  int rc;
  if ((rc = alloc((void**)&s->U, fld)) || (rc = alloc((void**)&s->W, fld)) || (rc = alloc((void**)&s->P, fld)) ||
      (rc = alloc((void**)&s->K, sizeof(float) * s->S3)) || (rc = alloc((void**)&s->top, sizeof(float4) * s->S3)) ||
      (rc = alloc((void**)&s->part, sizeof(float) * 256 * nel)) || (rc = alloc((void**)&s->tgt_d, sizeof(float) * nel)) ||
      (rc = alloc((void**)&s->scale, sizeof(float2) * nel)) || (rc = alloc((void**)&s->acc, sizeof(double) * 3)) ||
      (rc = alloc((void**)&s->mask, (size_t)s->S3 * nel)) ||
      (rc = alloc((void**)&s->slice, sizeof(float) * (size_t)S * S * (3 * nel + 1))))
    return fail(rc);
  if (cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess) {
    s->last_error = "cudaStreamCreate";
    return fail(RQ_ECUDA);
  }
  // initial state on the device
  std::vector<float> tf(nel);
  for (int m = 0; m < nel; ++m) tf[m] = (float)s->tgt[m];
  std::vector<RbNucDev> hn(n_nuclei);
  for (int a = 0; a < n_nuclei; ++a)
    hn[a] = RbNucDev{(float)nuclei[a].i, (float)nuclei[a].j, (float)nuclei[a].k, (float)nuclei[a].Z, (float)nuclei[a].rc,
                     nuclei[a].ne};
  std::vector<double> ex(5 * kRbMax + 1, 0.0);
  int max_side = 1;
  for (int m = 0; m < nel; ++m) {
    const rq_rb_nucleus& c = nuclei[s->enuc[m]];
    if (!(c.rc_excl > 0)) continue;
    // the reference indexes its mask with the nucleus' grid position: only whole positions mark cells
    if (c.i != std::floor(c.i) || c.j != std::floor(c.j) || c.k != std::floor(c.k)) continue;
    const int rcc = (int)std::ceil(c.rc_excl / h) + 1;
    ex[5 * m] = c.rc_excl; ex[5 * m + 1] = c.i; ex[5 * m + 2] = c.j; ex[5 * m + 3] = c.k; ex[5 * m + 4] = rcc;
    max_side = std::max(max_side, 2 * rcc + 1);
  }
  ex[5 * kRbMax] = h;
  RbNucDev* dn = nullptr;
  int* de = nullptr;
  double* dx = nullptr;
  if ((rc = alloc((void**)&dn, sizeof(RbNucDev) * n_nuclei)) || (rc = alloc((void**)&de, sizeof(int) * nel)) ||
      (rc = alloc((void**)&dx, sizeof(double) * ex.size()))) {
    for (void* q : {(void*)dn, (void*)de, (void*)dx}) if (q) cudaFree(q);
    return fail(rc);
  }
  cudaError_t e = cudaMemcpyAsync(dn, hn.data(), sizeof(RbNucDev) * n_nuclei, cudaMemcpyHostToDevice, s->st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(de, s->enuc.data(), sizeof(int) * nel, cudaMemcpyHostToDevice, s->st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dx, ex.data(), sizeof(double) * ex.size(), cudaMemcpyHostToDevice, s->st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(s->tgt_d, tf.data(), sizeof(float) * nel, cudaMemcpyHostToDevice, s->st);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->mask, 1, (size_t)s->S3 * nel, s->st);
  if (e == cudaSuccess) {
    k_rb_init_k<<<rb_cells_grid(NN, NN - 1), dim3(32, 8), 0, s->st>>>(p, dn, n_nuclei, s->K);
    k_rb_init_fields<<<rb_cells_grid(NN, (NN - 1) * nel), dim3(32, 8), 0, s->st>>>(p, dn, n_nuclei, de, s->U, s->W, s->P);
    const long long cube = (long long)max_side * max_side * max_side;
    k_rb_init_mask<<<dim3((unsigned)((cube + 255) / 256), nel), 256, 0, s->st>>>(p, dx, s->U, s->W, s->mask);
    s->launches += 3;
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
  for (void* q : {(void*)dn, (void*)de, (void*)dx}) cudaFree(q);
  if (e != cudaSuccess) {
    s->last_error = std::string("initial state: ") + cudaGetErrorString(e);
    return fail(RQ_ECUDA);
  }
  *out = s;
  return RQ_OK;
}

extern "C" void rq_rb_destroy(rq_rb* s) {
  if (!s) return;
  if (s->st) cudaStreamSynchronize(s->st);
  for (auto& kv : s->graphs) cudaGraphExecDestroy(kv.second.first);
  for (void* q : {(void*)s->U, (void*)s->W, (void*)s->P, (void*)s->K, (void*)s->top, (void*)s->part, (void*)s->tgt_d,
                  (void*)s->scale, (void*)s->acc, (void*)s->mask, (void*)s->slice})
    if (q) cudaFree(q);
  if (s->st) cudaStreamDestroy(s->st);
  delete s;
}

extern "C" const char* rq_rb_last_error(const rq_rb* s) { return s ? s->last_error.c_str() : "null"; }

extern "C" int rq_rb_step(rq_rb* s, int32_t n) {
  if (!s || n < 0) return RQ_EINVAL;
  if (n > 0) {
    auto it = s->graphs.find(n);
    if (it == s->graphs.end()) {  // a frame of n steps is one fixed launch sequence: captured once
      const long long l0 = s->launches;
      BCK(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
      int rc = rb_frame(s, n);
      cudaGraph_t gr = nullptr;
      cudaError_t e = cudaStreamEndCapture(s->st, &gr);
      if (rc != RQ_OK) {
        if (gr) cudaGraphDestroy(gr);
        return rc;
      }
      BCK(e);
      cudaGraphExec_t ex = nullptr;
      e = cudaGraphInstantiate(&ex, gr, 0);
      cudaGraphDestroy(gr);
      BCK(e);
      it = s->graphs.emplace(n, std::make_pair(ex, s->launches - l0)).first;
      s->launches = l0;
    }
    BCK(cudaGraphLaunch(it->second.first, s->st));
    s->launches += it->second.second;
    s->t_step += n;
  }
  BCK(cudaStreamSynchronize(s->st));
  return RQ_OK;
}

extern "C" int rq_rb_energy(rq_rb* s, double* out) {
  if (!s || !out) return RQ_EINVAL;
  const int NN = s->cfg.NN;
  BCK(cudaMemsetAsync(s->acc, 0, sizeof(double) * 3, s->st));
  k_rb_energy<<<rb_cells_grid(NN, NN - 1), dim3(32, 8), 0, s->st>>>(s->p, s->U, s->W, s->P, s->K, s->h,
                                                                    s->h * s->h * s->h, s->acc);
  BLAUNCH();
  BCK(cudaMemcpyAsync(out, s->acc, sizeof(double) * 3, cudaMemcpyDeviceToHost, s->st));
  BCK(cudaStreamSynchronize(s->st));
  return RQ_OK;
}

extern "C" int rq_rb_slice(rq_rb* s, float* out) {
  if (!s || !out) return RQ_EINVAL;
  const int S = s->p.S;
  k_rb_slice<<<(S * S + 255) / 256, 256, 0, s->st>>>(s->p, s->U, s->W, s->P, s->K, s->slice);
  BLAUNCH();
  BCK(cudaMemcpyAsync(out, s->slice, sizeof(float) * (size_t)S * S * (3 * s->n + 1), cudaMemcpyDeviceToHost, s->st));
  BCK(cudaStreamSynchronize(s->st));
  return RQ_OK;
}

extern "C" int rq_rb_download(rq_rb* s, int32_t m, float* U, float* W, float* P) {
  if (!s || m < 0 || m >= s->n) return RQ_EINVAL;
  const size_t S3 = (size_t)s->S3, off = (size_t)m * S3;
  if (U) BCK(cudaMemcpyAsync(U, s->U + off, sizeof(float) * S3, cudaMemcpyDeviceToHost, s->st));
  if (W) BCK(cudaMemcpyAsync(W, s->W + off, sizeof(float) * S3, cudaMemcpyDeviceToHost, s->st));
  if (P) BCK(cudaMemcpyAsync(P, s->P + off, sizeof(float) * S3, cudaMemcpyDeviceToHost, s->st));
  BCK(cudaStreamSynchronize(s->st));
  return RQ_OK;
}

extern "C" int rq_rb_upload(rq_rb* s, int32_t m, const float* U, const float* W, const float* P) {
  if (!s || m < 0 || m >= s->n) return RQ_EINVAL;
  const size_t S3 = (size_t)s->S3, off = (size_t)m * S3;
  if (U) BCK(cudaMemcpyAsync(s->U + off, U, sizeof(float) * S3, cudaMemcpyHostToDevice, s->st));
  if (W) BCK(cudaMemcpyAsync(s->W + off, W, sizeof(float) * S3, cudaMemcpyHostToDevice, s->st));
  if (P) BCK(cudaMemcpyAsync(s->P + off, P, sizeof(float) * S3, cudaMemcpyHostToDevice, s->st));
  BCK(cudaStreamSynchronize(s->st));
  return RQ_OK;
}

extern "C" int rq_rb_download_K(rq_rb* s, float* K) {
  if (!s || !K) return RQ_EINVAL;
  BCK(cudaMemcpyAsync(K, s->K, sizeof(float) * s->S3, cudaMemcpyDeviceToHost, s->st));
  BCK(cudaStreamSynchronize(s->st));
  return RQ_OK;
}

extern "C" int rq_rb_info(const rq_rb* s, int64_t* kernel_launches, int64_t* steps_done) {
  if (!s) return RQ_EINVAL;
  if (kernel_launches) *kernel_launches = s->launches;
  if (steps_done) *steps_done = s->t_step;
  return RQ_OK;
}
