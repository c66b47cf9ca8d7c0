// rq_kernels.h -- host launchers of the librq kernels (internal to the library).
#pragma once
#include <vector>
#include "rq_internal.cuh"

namespace rq {

// ---- solver.py flavour (sp_kernels.cu) --------------------------------------------------
cudaError_t launch_update_sp(const float* U, float* Unew, const float* K, const float* P, const int* label,
                             const Geo& g, float half_dv, float dtv, double h3, int nDom, double* norms,
                             cudaStream_t st);
// update and Jacobi sweep in one pass (first: update then the sweep on the new psi; else the
// sweep then the update with the new P)
cudaError_t launch_step_sp(bool first, const float* U, float* Unew, const float* K, const float* P, float* Pnew,
                           const int* label, const Geo& g, float half_dv, float dtv, float h2, float coeff, double h3,
                           int nDom, double* norms, cudaStream_t st);
cudaError_t launch_jacobi_sp(const float* P, float* Pnew, const float* U, const Geo& g, float h2, float coeff,
                             cudaStream_t st);
cudaError_t launch_labels_sp(const int* labIn, int* labOut, const float* atoms5, int nAtoms, const Geo& g, float h,
                             float h2, cudaStream_t st);
// Atoms with Z > 0 sorted into cubic bins of `bin` grid units over [0, nb*bin)^3 (the grid box);
// atoms outside it are on a far list.  Built on the host by build_atom_bins.
struct AtomBins {
  int nb, bin;
  const int* start;   // nb^3 + 1 offsets into idx
  const int* idx;     // atom indices, bin by bin
  const int* far;     // far[0] = count, far[1..count] = atom indices
  const float* zmax;  // largest Z of any atom (device value, so captured graphs see updates)
};
// host: fill start/idx/far (sizes nb^3+1, n, n+1) and zmax for atoms5 (n x 5, grid units)
void build_atom_bins(const float* atoms5, int n, int nb, int bin, std::vector<int>& start, std::vector<int>& idx,
                     std::vector<int>& far, float& zmax);
// the label step with the argmax over atoms found through the bins (same result as launch_labels_sp)
cudaError_t launch_labels_binned_sp(const int* labIn, int* labOut, const float* atoms5, int nAtoms, AtomBins bins,
                                    const Geo& g, float h, float h2, cudaStream_t st);
cudaError_t launch_init_sp(float* U, int* label, float* K, float* bestU, const float* atoms5, int nAtoms,
                           const Geo& g, float h, float h2, bool trial, cudaStream_t st);
cudaError_t launch_norms_flat(const float* U, const int* label, const Geo& g, double h3, int nDom, double* norms,
                              cudaStream_t st);
cudaError_t launch_norm_scale_sp(const double* norms, const float* Zeff, int nDom, float* scale, int* err,
                                 cudaStream_t st);
cudaError_t launch_apply_scale_sp(float* U, const int* label, const float* scale, const Geo& g, int nDom,
                                  cudaStream_t st);
cudaError_t launch_energy_sp(const float* U, const float* K, const float* P, const int* label, const Geo& g, double h,
                             double h3, int nDom, double* pd, cudaStream_t st);
cudaError_t launch_forces_hf_sp(const float* U, const float* atoms5, int nAtoms, const Geo& g, float h, float h2,
                                float h3, double* F, cudaStream_t st);
template <typename T>
cudaError_t launch_zero_faces(T* f, const Geo& g, cudaStream_t st);

// ---- molecule.js flavour (mj_kernels.cu); labels carry the r_c-exclusion flag in bit 30 ---
}  // namespace rq
struct MjAtom;
struct MjSplit;
namespace rq {
constexpr int kMjExclBit = 0x40000000;
constexpr int kMjLabelMask = 0x3FFFFFFF;
cudaError_t launch_mj_init(float* K, float* U, float* bestU, int* label, const MjAtom* atoms, int nAt, const Geo& g,
                           float h, float h2, float Rsing, bool hasBare, bool persist,
                           const MjSplit* splits, cudaStream_t st);
cudaError_t launch_mj_recompute_k(float* K, const MjAtom* atoms, int nAt, const Geo& g, float h, float Rsing,
                                  cudaStream_t st);
cudaError_t launch_mj_flags(int* label, const MjAtom* atoms, int nAt, const Geo& g, float h, bool hasBare,
                            cudaStream_t st);
cudaError_t launch_mj_update(const float* U, float* Uo, const float* K, const int* label, const float* Pother,
                             const Geo& g, float half_d, float dt, float h3, int nDom, unsigned* unorm, cudaStream_t st);
cudaError_t launch_mj_norm_scale(const unsigned* unorm, const MjAtom* atoms, int nDom, float* scale, cudaStream_t st);
cudaError_t launch_mj_update_cheb(const float* U, float* Uo, const float* K, const int* label, const float* Pother,
                                  const Geo& g, float half_d, float dt, float h3, int nDom, unsigned* unorm,
                                  float omega, cudaStream_t st);
cudaError_t launch_mj_extract(const float* U, const int* label, const float* K, const MjAtom* atoms, int nAt,
                              const Geo& g, int sk, float* out, cudaStream_t st);
cudaError_t launch_mj_apply_scale(float* U, const int* label, const float* scale, const Geo& g, cudaStream_t st);
cudaError_t launch_mj_jacobi(const float* Pin, float* Pout, const float* U, const Geo& g, float h2, float two_pi,
                             cudaStream_t st);
cudaError_t launch_mj_vcycle(float* P, const float* U, float* rho, float* resid, float* Ec0, float* Ec1, float* fc,
                             const Geo& g, const Geo& gc, float h2, float inv_h2, float two_pi, cudaStream_t st);
// the direct per-electron Poisson of small systems (molecule.js:2833-2858, :614-671): P_m init and
// one step's solve for domain m (Pm persistent; rho, scratch are scratch)
cudaError_t launch_mj_direct_init(const MjAtom* atoms, int nAt, int m, float* Pm, float* Pother, const Geo& g, float h,
                                  float h2, cudaStream_t st);
cudaError_t launch_mj_direct_domain(const float* U, const int* label, float* Pother, int m, float* Pm, float* scratch,
                                    float* rho, const Geo& g, float h2, float two_pi, cudaStream_t st);
// the self-interaction correction of one domain m (molecule.js:3018-3075); rho, sic, sic2, resid,
// Ec0, Ec1 and fc are scratch
cudaError_t launch_mj_sic_domain(const float* U, const int* label, float* Pother, int m, float frac, float* rho,
                                 float* sic, float* sic2, float* resid, float* Ec0, float* Ec1, float* fc, const Geo& g,
                                 const Geo& gc, float h2, float inv_h2, float two_pi, cudaStream_t st);
// lock: per label the bit set of its locked groups (all 0 without groups)
cudaError_t launch_mj_evolve(const int* labIn, int* labOut, const float* U, float* W, const MjAtom* atoms, int nAt,
                             const Geo& g, float dt_w, float curvReg, float h, bool hasBare,
                             const unsigned long long* lock, const MjSplit* splits, cudaStream_t st);
cudaError_t launch_mj_energy(const float* U, const float* Pv, const float* K, const int* label, const MjAtom* atoms,
                             const Geo& g, float h, float h3, float Rsing, int nDom, double* pd, double* dip,
                             cudaStream_t st);
cudaError_t launch_mj_gradp(const float* P, const MjAtom* atoms, int nAt, const Geo& g, float inv_h, int R, double* F,
                            cudaStream_t st);
cudaError_t launch_fill(float* f, float v, long long n, cudaStream_t st);
// the six faces of label buffer src copied into dst
cudaError_t launch_copy_faces(const int* src, int* dst, const Geo& g, cudaStream_t st);
// LOBPCG frames (molecule.js:1455-1724): inner products in workgroups of kLobWG threads, at most
// kLobMaxWG of them (molecule.js:1533-1534); kLobScal floats of per-iteration scalars
constexpr int kLobNR = 12, kLobWG = 128, kLobMaxWG = 256, kLobScal = 32;
int lob_workgroups(const Geo& g);
cudaError_t launch_lob_apply_h(const float* U, float* HU, const float* K, const int* label, const float* Pother,
                               const MjAtom* atoms, const Geo& g, float h, float inv_h2, bool bare, cudaStream_t st);
cudaError_t launch_lob_inner(const float* X, const float* HX, const float* W, const float* HW, const float* Pv,
                             const float* HP, const int* label, int m, const Geo& g, float h3, float* partials,
                             cudaStream_t st);
cudaError_t launch_lob_finalize(const float* partials, int nwg, bool first, bool hasP, float* scal, cudaStream_t st);
cudaError_t launch_lob_residual(const float* X, const float* HX, float* W, const int* label, const float* K,
                                const float* Pot, const float* lam, int m, const Geo& g, float inv_h2, cudaStream_t st);
cudaError_t launch_lob_update(float* X, const float* W, float* Pv, const int* label, const float* coef, int m,
                              const Geo& g, cudaStream_t st);
cudaError_t launch_mj_accum_norms(const float* U, const int* label, const Geo& g, float h3, unsigned* unorm,
                                  cudaStream_t st);

// ---- new flavour (nm_kernels.cu), T = float (mixed) or double (FP64) --------------------
// |dE| between checks, relative to |E|, below which fp32 fields stop resolving the energy: a
// mixed-precision solve that needs less is promoted to FP64 there.  With the P-stationary readout
// (nm_energy) the fp32 readout changes smoothly between checks down to ~1e-13 |E| (glycine, 128^3);
// read as h^3 sum P rho it jittered at ~1e-9 |E|, which needed promotion at 3e-9 |E|.
constexpr double kMixedFloor = 1e-12;
template <typename T>
// K64 (optional): FP64 copy of the same sums, from the same pass
cudaError_t nm_potential(T* K, const double* at, int nAt, const Geo& g, double h, double sigma, cudaStream_t st,
                         double* K64 = nullptr);
template <typename T>
cudaError_t nm_init(T* U, int* label, const float4* seeds, int nSeed, const Geo& g, float h, cudaStream_t st);
template <typename T>
cudaError_t nm_update(const T* U, T* Unew, const T* K, const T* P, const int* label, const Geo& g, T half_dv, T dt,
                      double h3, int nDom, double* norms, cudaStream_t st, const double* scale = nullptr,
                      const unsigned* seed = nullptr, unsigned* seed_next = nullptr,
                      const unsigned char* mask = nullptr);
// the same-label neighbour mask of `label` (S^3 bytes; bit q: neighbour q has the point's label)
cudaError_t nm_mask(const int* label, unsigned char* mask, const Geo& g, cudaStream_t st);
template <typename T>
cudaError_t nm_apply(T* U, const int* label, const double* scale, int nDom, const Geo& g, cudaStream_t st);
template <typename T>
cudaError_t nm_normalize(T* U, const int* label, const double* norms, const double* Zdom, int nDom, double* scale, int* err,
                         const Geo& g, cudaStream_t st);
template <typename T>
cudaError_t nm_norm_scale(const double* norms, const double* Zdom, int nDom, double* scale, int* err, cudaStream_t st);
template <typename T>
cudaError_t nm_norms(const T* U, const int* label, const Geo& g, double h3, int nDom, double* norms, cudaStream_t st);
template <typename T>
cudaError_t nm_rbgs(T* P, const T* f, bool fine, const Geo& g, double h2, int color, cudaStream_t st);
// fc = R (f - A P) (the residual and its full weighting in one pass) and Pc = 0 on the coarse interior
template <typename T>
cudaError_t nm_resrestrict(const T* P, const T* f, bool fine, T* fc, T* Pc, const Geo& g, const Geo& gc, double inv_h2,
                           cudaStream_t st);
template <typename T>
cudaError_t nm_prolong(const T* Ec, T* P, const Geo& g, const Geo& gc, cudaStream_t st);
template <typename T>
cudaError_t nm_coarsest(T* P, const T* f, const Geo& g, double h2, int sweeps, cudaStream_t st);
template <typename T>
cudaError_t nm_energy(const T* U, const T* K, const T* P, const int* label, const Geo& g, double h, int nDom, double* pd,
                      cudaStream_t st, const double* K64 = nullptr);
template <typename T>
cudaError_t nm_evolve(const int* labIn, int* labOut, const T* U, float* W, const Geo& g, double dt_w, double curvReg,
                      cudaStream_t st);
template <typename T>
cudaError_t nm_add(T* K, const T* v, long long n, cudaStream_t st);
// HF gather (gw null) or the gradient gather with the weight field gw = dE/dK (S^3 doubles)
template <typename T>
cudaError_t nm_force(const T* U, const double* at, int nAt, const Geo& g, double h, double sigma, double* F,
                     cudaStream_t st, const double* gw = nullptr);
cudaError_t launch_unpack_labels(const int* in, int* out, long long n, cudaStream_t st);

}  // namespace rq
