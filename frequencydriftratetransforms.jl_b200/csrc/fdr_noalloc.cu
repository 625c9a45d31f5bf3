// fdrstats without device allocation.
//
// fdr_stats() obtains its per-column accumulators from the stream-ordered allocator.  Some
// callers cannot allow that: a real-time acquisition pipeline that forbids device
// allocation once it is running (an allocation may have to wait on the device or fail when
// memory is tight), or a host program whose device memory is fully reserved by its own pool
// allocator, where any allocation by this library can fail.  fdr_stats_noalloc() computes
// the same statistics with its scratch space in a fixed, file-scope device array instead.
//
// The array is a static __device__ symbol, so every GPU that loads this library holds it
// (FDR_STATS_NOALLOC_MAX_COLUMNS * 16 + 16 bytes) until the process exits.  Host code cannot
// use the symbol's name as a device address; its address is looked up once per device with
// cudaGetSymbolAddress and passed to the kernels.
#include <math.h>

#include <mutex>

#include "fdr_internal.cuh"

namespace fdr {

constexpr int kNoallocThreads = 256;

// [0, 2*MAX): per-column sum and sum of squares; [2*MAX, 2*MAX+2): mean, minimum std.
static __device__ __align__(256) double g_stats_scratch[2 * FDR_STATS_NOALLOC_MAX_COLUMNS + 2];

static double* g_scratch_addr[64];
static std::mutex g_scratch_mu;

// Device address of g_stats_scratch on the current device (set up on first use).
static int scratch_address(double** out) {
  int dev = 0;
  FDR_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    set_error(FDR_ERR_INVALID_ARGUMENT, "fdr_stats_noalloc: device ordinal %d >= 64", dev);
    return FDR_ERR_INVALID_ARGUMENT;
  }
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    FDR_CUDA(cudaGetSymbolAddress(&p, g_stats_scratch));
    g_scratch_addr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_addr[dev];
  return FDR_OK;
}

__global__ void noalloc_clear_kernel(double* __restrict__ acc, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) acc[i] = 0.0;
}

// grid.x: chunks of rows, grid.y: columns.
__global__ void __launch_bounds__(kNoallocThreads)
noalloc_moments_kernel(const float* __restrict__ fdr, long long Nf, double* __restrict__ acc) {
  const long long col = blockIdx.y;
  const float* x = fdr + col * Nf;
  double s1 = 0.0, s2 = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < Nf;
       i += (long long)gridDim.x * blockDim.x) {
    const double v = (double)x[i];
    s1 += v;
    s2 += v * v;
  }
  for (int o = 16; o > 0; o >>= 1) {
    s1 += __shfl_down_sync(0xffffffffu, s1, o);
    s2 += __shfl_down_sync(0xffffffffu, s2, o);
  }
  __shared__ double r1[kNoallocThreads / 32], r2[kNoallocThreads / 32];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { r1[w] = s1; r2[w] = s2; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int i = 0; i < kNoallocThreads / 32; ++i) { a += r1[i]; b += r2[i]; }
    atomicAdd(acc + 2 * col, a);
    atomicAdd(acc + 2 * col + 1, b);
  }
}

__global__ void noalloc_finalize_kernel(double* __restrict__ acc, long long ncols, long long Nf,
                                        double* __restrict__ ms) {
  __shared__ double smin[256];
  __shared__ int snan[256];
  double best = INFINITY;
  int nan = 0;
  for (long long c = threadIdx.x; c < ncols; c += blockDim.x) {
    const double s1 = acc[2 * c], s2 = acc[2 * c + 1];
    const double mean = s1 / (double)Nf;
    double var = (s2 - s1 * mean) / (double)(Nf - 1);
    if (var < 0) var = 0;
    const double sd = sqrt(var);
    if (isnan(sd)) nan = 1;
    best = fmin(best, sd);
  }
  smin[threadIdx.x] = best;
  snan[threadIdx.x] = nan;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = INFINITY;
    int anynan = 0;
    for (int i = 0; i < blockDim.x; ++i) { b = fmin(b, smin[i]); anynan |= snan[i]; }
    ms[0] = acc[0] / (double)Nf;
    ms[1] = anynan ? NAN : b;
  }
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
  double* scratch = nullptr;
  FDR_TRY(scratch_address(&scratch));
  cudaStream_t st = (cudaStream_t)stream;
  double* acc = scratch;
  double* ms = scratch + 2 * FDR_STATS_NOALLOC_MAX_COLUMNS;
  const int nacc = (int)(2 * Nr);
  noalloc_clear_kernel<<<(unsigned)std::max(1, std::min(64, (nacc + 255) / 256)), 256, 0, st>>>(acc, nacc);
  FDR_LAUNCH_CHECK("noalloc_clear_kernel");
  const long long rows_blocks = std::max<long long>(
      1, std::min<long long>(cdiv(Nf, kNoallocThreads * 8),
                             std::max<long long>(1, (long long)sm_count() * 8 / Nr)));
  noalloc_moments_kernel<<<dim3((unsigned)rows_blocks, (unsigned)Nr), kNoallocThreads, 0, st>>>(fdr, Nf, acc);
  FDR_LAUNCH_CHECK("noalloc_moments_kernel");
  noalloc_finalize_kernel<<<1, 256, 0, st>>>(acc, Nr, Nf, ms);
  FDR_LAUNCH_CHECK("noalloc_finalize_kernel");
  double h[2] = {0.0, 0.0};
  FDR_CUDA(cudaMemcpyAsync(h, ms, sizeof(h), cudaMemcpyDeviceToHost, st));
  FDR_CUDA(cudaStreamSynchronize(st));
  *m = h[0];
  *s = h[1];
  return FDR_OK;
}
