// fdrstats without device allocation.
//
// fdr_stats() obtains its scratch space from the stream-ordered allocator.  Some callers
// cannot allow that: a real-time acquisition pipeline that forbids device allocation once it
// is running (an allocation may have to wait on the device or fail when memory is tight), or
// a host program whose device memory is fully reserved by its own pool allocator, where any
// allocation by this library can fail.  fdr_stats_noalloc() computes the same statistics
// (the same Float32 pairwise kernels, bit for bit) with its scratch space in a fixed,
// file-scope device array instead.
//
// The array is a static __device__ symbol, so every GPU that loads this library holds it
// (FDR_STATS_NOALLOC_MAX_COLUMNS * 16 + 32 bytes) until the process exits.  Host code cannot
// use the symbol's name as a device address; its address is looked up with
// cudaGetSymbolAddress once per device and CUDA context (a context that is torn down and
// created again, e.g. after cudaDeviceReset, loads the module again and gets a new address)
// and passed to the kernels.
#include <math.h>

#include <mutex>

#include "fdr_internal.cuh"

namespace fdr {

// Partial sums per column: at most kNoallocParts CTAs per column, two passes (sum, centred
// squares).  Every slot a call reads is written earlier in the same call, so nothing needs
// clearing between calls.
constexpr int kNoallocParts = 2;
constexpr long long kNoallocPartFloats = 2LL * kNoallocParts * FDR_STATS_NOALLOC_MAX_COLUMNS;

// [0, kNoallocPartFloats): partials; then three doubles: m, s, threshold.
static __device__ __align__(256) float g_stats_scratch[kNoallocPartFloats + 8];

typedef int (*PFN_ctx_get_current)(void**);

// cuCtxGetCurrent from the driver, through the runtime (no link against libcuda).
static PFN_ctx_get_current ctx_get_current() {
  static const PFN_ctx_get_current fn = []() -> PFN_ctx_get_current {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess && q == cudaDriverEntryPointSuccess)
      return (PFN_ctx_get_current)p;
    return nullptr;
  }();
  return fn;
}

struct ScratchSlot {
  void* ctx = nullptr;
  float* addr = nullptr;
};
static ScratchSlot g_scratch_slots[64];
static std::mutex g_scratch_mu;

// Device address of g_stats_scratch on the current device, looked up on the first call
// per device and context, with that device current.
static int scratch_address(float** out) {
  int dev = 0;
  FDR_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    set_error(FDR_ERR_INVALID_ARGUMENT, "fdr_stats_noalloc: device ordinal %d >= 64", dev);
    return FDR_ERR_INVALID_ARGUMENT;
  }
  void* ctx = nullptr;
  PFN_ctx_get_current get = ctx_get_current();
  if (get != nullptr && get(&ctx) == 0 && ctx == nullptr) {
    // no context current on this thread yet: cudaSetDevice initialises the device's primary
    // context and makes it current (CUDA 12), without allocating
    FDR_CUDA(cudaSetDevice(dev));
    if (get(&ctx) != 0) ctx = nullptr;
  }
  if (get == nullptr || ctx == nullptr) {
    set_error(FDR_ERR_CUDA, "fdr_stats_noalloc: cuCtxGetCurrent unavailable");
    return FDR_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  ScratchSlot& slot = g_scratch_slots[dev];
  if (slot.addr == nullptr || slot.ctx != ctx) {
    void* p = nullptr;
    FDR_CUDA(cudaGetSymbolAddress(&p, g_stats_scratch));
    slot.addr = static_cast<float*>(p);
    slot.ctx = ctx;
  }
  *out = slot.addr;
  return FDR_OK;
}

}  // namespace fdr

using namespace fdr;

extern "C" int fdr_stats_noalloc(const float* fdr, int64_t Nf, int64_t Nr, double* m, double* s,
                                 fdr_stream_t stream) {
  FDR_CHECK_ARG(fdr && m && s, "fdr_stats_noalloc: NULL argument");
  FDR_CHECK_ARG(Nf >= 1 && Nr >= 1, "fdr_stats_noalloc: bad sizes Nf=%lld Nr=%lld",
                (long long)Nf, (long long)Nr);
  FDR_CHECK_ARG(Nr <= FDR_STATS_NOALLOC_MAX_COLUMNS,
                "fdr_stats_noalloc: Nr=%lld exceeds the fixed scratch capacity of %d columns; "
                "use fdr_stats", (long long)Nr, FDR_STATS_NOALLOC_MAX_COLUMNS);
  float* scratch = nullptr;
  FDR_TRY(scratch_address(&scratch));
  cudaStream_t st = (cudaStream_t)stream;
  double* ms = reinterpret_cast<double*>(scratch + kNoallocPartFloats);
  FDR_TRY(pairwise_stats_launch(nullptr, fdr, 1, Nf, Nr, scratch, kNoallocParts, ms, 0, 0.0, st));
  double h[3] = {0.0, 0.0, 0.0};
  FDR_CUDA(cudaMemcpyAsync(h, ms, sizeof(h), cudaMemcpyDeviceToHost, st));
  FDR_CUDA(cudaStreamSynchronize(st));
  *m = h[0];
  *s = h[1];
  return FDR_OK;
}
