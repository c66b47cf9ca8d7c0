// noalloc.cu -- rq_kernel_normalize_sp_noalloc: the solver.py normalisation on caller-owned
// device memory without any device allocation.
//
// Who needs this: rq_kernel_normalize_sp obtains its scratch (the per-domain FP64 sums, the
// per-domain scale table and an error word) from the stream-ordered allocator on every call.
// Some hosts cannot allow that: a host framework whose own caching allocator has already
// claimed the device memory and forbids outside allocations, or a long-running solver loop
// that must not allocate after start-up because an allocation can stall or fragment device
// memory in the middle of a run.  This variant keeps its scratch in one fixed array in device
// global memory instead, sized for at most RQ_NOALLOC_MAX_DOMAINS domains.
//
// Behaviour of the shared scratch:
//  * the array lives for as long as the library is loaded, on every GPU that loads it
//    (RQ_NOALLOC_MAX_DOMAINS * 12 bytes + 256 bytes per GPU);
//  * every call uses the same array, and it keeps what the last call left there: each call
//    zeroes the per-domain sums and the error word before using them;
//  * two calls whose work overlaps on the GPU (different streams, or different host threads
//    with no ordering between them) race on the array; order such calls on one stream.
//
// Set-up: the device address of the array belongs to one CUDA context (one load of this
// module in it).  The first call in a context looks it up (cudaGetSymbolAddress, with that
// context current) and caches it under the context's unique id, so a primary context created
// again after cudaDeviceReset, or another context the caller made current, gets its own
// look-up instead of a stale address.  Make the first call in each context before starting any
// stream capture in it.
//
// Errors: like rq_kernel_normalize_sp, the call reads the error word back (it synchronises the
// stream) and returns RQ_ENONFINITE when a domain's norm was NaN or Inf; that domain is left
// unscaled.
#include <mutex>
#include <vector>

#include <cuda.h>

#include "../../include/rq.h"
#include "rq_kernels.h"

namespace {

constexpr int kMaxDomains = RQ_NOALLOC_MAX_DOMAINS;

// [0, 8*max): FP64 per-domain sums; [8*max, 12*max): f32 scale table; then the error word.
constexpr size_t kScratchBytes = (size_t)kMaxDomains * 12 + 256;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

struct CachedAddr {
  unsigned long long ctx_id;
  void* addr;
};

std::mutex g_setup_mutex;
CtxGetCurrentFn g_ctx_current = nullptr;
CtxGetIdFn g_ctx_id = nullptr;
std::vector<CachedAddr> g_scratch_addr;

// Unique id of the current CUDA context (0 with an error if there is none after the runtime
// has set up its primary context).  Caller holds g_setup_mutex.
cudaError_t current_context_id(unsigned long long* id) {
  if (!g_ctx_current || !g_ctx_id) {
    cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = cudaDriverEntryPointSymbolNotFound;
    cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", (void**)&g_ctx_current, cudaEnableDefault, &q1);
    if (e == cudaSuccess) e = cudaGetDriverEntryPoint("cuCtxGetId", (void**)&g_ctx_id, cudaEnableDefault, &q2);
    if (e != cudaSuccess) return e;
    if (q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess) {
      g_ctx_current = nullptr;
      g_ctx_id = nullptr;
      return cudaErrorNotSupported;
    }
  }
  CUcontext ctx = nullptr;
  if (g_ctx_current(&ctx) != CUDA_SUCCESS) return cudaErrorContextIsDestroyed;
  if (!ctx) {
    // no context current yet: let the runtime bring up the device's primary context (the symbol
    // look-up does that and allocates nothing), then ask again
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    if (g_ctx_current(&ctx) != CUDA_SUCCESS || !ctx) return cudaErrorContextIsDestroyed;
  }
  return g_ctx_id(ctx, id) == CUDA_SUCCESS ? cudaSuccess : cudaErrorContextIsDestroyed;
}

// Device address of g_noalloc_scratch in the current context (looked up once per context).
cudaError_t scratch_address(void** out) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  unsigned long long id = 0;
  cudaError_t e = current_context_id(&id);
  if (e != cudaSuccess) return e;
  for (const CachedAddr& c : g_scratch_addr)
    if (c.ctx_id == id) {
      *out = c.addr;
      return cudaSuccess;
    }
  void* p = nullptr;
  e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return e;
  g_scratch_addr.push_back({id, p});
  *out = p;
  return cudaSuccess;
}

}  // namespace

extern "C" int rq_kernel_normalize_sp_noalloc(float* U, const int32_t* label, const float* Zeff, int32_t n_atoms,
                                              int32_t S, float h3, void* stream) {
  if (!U || !label || !Zeff || n_atoms < 1 || S < 3) return RQ_EINVAL;
  if (n_atoms > kMaxDomains) return RQ_EINVAL;  // more domains than the fixed scratch holds
  void* base = nullptr;
  if (scratch_address(&base) != cudaSuccess) return RQ_ECUDA;
  unsigned char* b = (unsigned char*)base;
  double* norms = (double*)b;
  float* scale = (float*)(b + (size_t)kMaxDomains * 8);
  int* err = (int*)(b + (size_t)kMaxDomains * 12);
  const rq::Geo g = rq::make_geo(S);
  cudaStream_t st = (cudaStream_t)stream;
  if (cudaMemsetAsync(norms, 0, sizeof(double) * n_atoms, st) != cudaSuccess) return RQ_ECUDA;
  if (cudaMemsetAsync(err, 0, sizeof(int), st) != cudaSuccess) return RQ_ECUDA;
  if (rq::launch_norms_flat(U, label, g, (double)h3, n_atoms, norms, st) != cudaSuccess) return RQ_ECUDA;
  if (rq::launch_norm_scale_sp(norms, Zeff, n_atoms, scale, err, st) != cudaSuccess) return RQ_ECUDA;
  if (rq::launch_apply_scale_sp(U, label, scale, g, n_atoms, st) != cudaSuccess) return RQ_ECUDA;
  // the error word back into host memory (a pageable stack variable: no allocation)
  int err_host = 0;
  if (cudaMemcpyAsync(&err_host, err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return RQ_ECUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return RQ_ECUDA;
  return err_host ? RQ_ENONFINITE : RQ_OK;
}
