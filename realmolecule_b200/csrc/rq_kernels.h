// rq_kernels.h -- host launchers of the librq kernels (internal to the library).
#pragma once
#include "rq_internal.cuh"

namespace rq {

// ---- solver.py flavour (sp_kernels.cu) --------------------------------------------------
cudaError_t launch_update_sp(const float* U, float* Unew, const float* K, const float* P, const int* label,
                             const Geo& g, float half_dv, float dtv, double h3, int nDom, double* norms,
                             cudaStream_t st);
cudaError_t launch_jacobi_sp(const float* P, float* Pnew, const float* U, const Geo& g, float h2, float coeff,
                             cudaStream_t st);
cudaError_t launch_labels_sp(const int* labIn, int* labOut, const float* atoms5, int nAtoms, const Geo& g, float h,
                             float h2, cudaStream_t st);
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

}  // namespace rq
