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
// Set-up: the first call on each device looks up the device address of the array
// (cudaGetSymbolAddress, with that device current) and caches it; make that first call on a
// device before starting any stream capture on it.
#include <mutex>

#include "../../include/rq.h"
#include "rq_kernels.h"

namespace {

constexpr int kMaxDomains = RQ_NOALLOC_MAX_DOMAINS;
constexpr int kMaxDevices = 64;

// [0, 8*max): FP64 per-domain sums; [8*max, 12*max): f32 scale table; then the error word.
constexpr size_t kScratchBytes = (size_t)kMaxDomains * 12 + 256;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_setup_mutex;
void* g_scratch_addr[kMaxDevices] = {};

// Returns the device address of g_noalloc_scratch on the current device (set up once per device).
cudaError_t scratch_address(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
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
  return RQ_OK;
}
