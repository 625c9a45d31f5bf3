// Library-wide C entry points (version, errors, synchronisation, zdtutils.jl helpers) and
// the internal host utilities declared in fdr_internal.cuh.
#include <stdarg.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <mutex>

#include "fdr_internal.cuh"
#include "zdt_ws.cuh"

namespace fdr {

static thread_local std::string g_last_error;
static std::atomic<long long> g_launches{0};

void count_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// Readers of the debug builds' per-file fault words (registered by static initialisers).
static std::vector<int (*)(unsigned long long*)>& debug_readers() {
  static std::vector<int (*)(unsigned long long*)> v;
  return v;
}
static std::mutex g_debug_mu;

void register_debug_reader(int (*take)(unsigned long long*)) {
  std::lock_guard<std::mutex> lock(g_debug_mu);
  debug_readers().push_back(take);
}

int debug_take_fault(unsigned long long* word) {
  std::lock_guard<std::mutex> lock(g_debug_mu);
  unsigned long long first = 0;
  for (auto fn : debug_readers()) {
    unsigned long long w = 0;
    fn(&w);
    if (w && !first) first = w;
  }
  *word = first;
  return FDR_OK;
}

void set_error(int status, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = std::string(fdr_status_string(status)) + ": " + buf;
}

int cuda_status(cudaError_t e, const char* what) {
  int st = (e == cudaErrorMemoryAllocation) ? FDR_ERR_OUT_OF_MEMORY
           : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) ? FDR_ERR_NO_DEVICE
                                                                          : FDR_ERR_CUDA;
  // Clear a non-sticky error so later calls on this thread start clean.
  (void)cudaGetLastError();
  set_error(st, "%s failed: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
  return st;
}

int64_t nextprod(const int64_t* factors, int nfactors, int64_t n) {
  static const int64_t deflt[3] = {2, 3, 5};
  if (factors == nullptr || nfactors <= 0) { factors = deflt; nfactors = 3; }
  for (int i = 0; i < nfactors; ++i)
    if (factors[i] < 2) return -1;
  if (n <= 1) return 1;
  // Smallest product of powers of the factors that is >= n, by depth-first search over the
  // exponents (the search space is tiny for the sizes used here).
  int64_t best = INT64_MAX;
  struct Rec {
    const int64_t* f;
    int nf;
    int64_t n;
    int64_t* best;
    void go(int i, int64_t cur) {
      if (cur >= n) { if (cur < *best) *best = cur; return; }
      if (i == nf) return;
      int64_t v = cur;
      while (true) {
        go(i + 1, v);
        if (v >= n || v > INT64_MAX / f[i]) break;
        v *= f[i];
      }
    }
  } r{factors, nfactors, n, &best};
  r.go(0, 1);
  return best == INT64_MAX ? -1 : best;
}

// Small host arrays (matrix pointers, rate blocks) reach the device as kernel parameters, 512
// bytes per launch, not through a host-to-device copy: such a copy can queue behind a large
// transfer that the caller has in flight on a copy engine (the next spectrogram of a pipeline),
// and every kernel after it would wait for that transfer to finish.
struct WordChunk {
  uint32_t w[128];
};

__global__ void store_words_kernel(WordChunk c, int n, uint32_t* __restrict__ dst) {
  if ((int)threadIdx.x < n) dst[threadIdx.x] = c.w[threadIdx.x];
}

int upload_words(void* dev, const void* host, size_t bytes, cudaStream_t s) {
  FDR_CHECK_ARG(bytes % 4 == 0 && (reinterpret_cast<uintptr_t>(dev) & 3) == 0,
                "upload of %zu bytes: not whole aligned 32-bit words", bytes);
  const uint32_t* h = static_cast<const uint32_t*>(host);
  const size_t n = bytes / 4;
  for (size_t off = 0; off < n; off += 128) {
    WordChunk c;
    const int k = (int)std::min<size_t>(128, n - off);
    memcpy(c.w, h + off, sizeof(uint32_t) * k);
    store_words_kernel<<<1, 128, 0, s>>>(c, k, static_cast<uint32_t*>(dev) + off);
    FDR_LAUNCH_CHECK("store_words_kernel");
  }
  return FDR_OK;
}

// Mapped pinned host words for the small results of a call (proto-hit counts, thresholds),
// one buffer per host thread, grown on demand.  A kernel stores the results there over the
// bus: a device-to-host copy would again go through a copy engine and wait behind an
// unrelated host-to-device transfer in flight.
namespace {
struct PinnedStaging {
  void* p = nullptr;
  void* d = nullptr;
  size_t n = 0;
  ~PinnedStaging() {
    if (p) (void)cudaFreeHost(p);
  }
};
thread_local PinnedStaging t_staging;
}  // namespace

int pinned_staging(size_t bytes, void** host, void** dev) {
  if (t_staging.n < bytes) {
    if (t_staging.p) (void)cudaFreeHost(t_staging.p);
    t_staging = PinnedStaging();
    const size_t n = std::max<size_t>(bytes, 256);
    void* p = nullptr;
    void* d = nullptr;
    FDR_CUDA(cudaHostAlloc(&p, n, cudaHostAllocMapped | cudaHostAllocPortable));
    const cudaError_t e = cudaHostGetDevicePointer(&d, p, 0);
    if (e != cudaSuccess) {
      (void)cudaFreeHost(p);
      return cuda_status(e, "cudaHostGetDevicePointer");
    }
    t_staging.p = p;
    t_staging.d = d;
    t_staging.n = n;
  }
  *host = t_staging.p;
  *dev = t_staging.d;
  return FDR_OK;
}

int device_view(void* p, void** dp, const char* what) {
  cudaPointerAttributes a;
  const cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    set_error(FDR_ERR_INVALID_ARGUMENT, "%s: not a CUDA-accessible pointer", what);
    return FDR_ERR_INVALID_ARGUMENT;
  }
  if (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) {
    *dp = p;
    return FDR_OK;
  }
  if (a.type == cudaMemoryTypeHost && a.devicePointer != nullptr) {
    *dp = a.devicePointer;
    return FDR_OK;
  }
  set_error(FDR_ERR_INVALID_ARGUMENT, "%s: neither device memory nor mapped pinned host memory", what);
  return FDR_ERR_INVALID_ARGUMENT;
}

// Stream-ordered scratch comes from a memory pool owned by the library, one per device, that
// keeps up to kScratchKeep bytes reserved across synchronisations.  (The device's default pool
// releases everything at each synchronisation, so every allocation after one maps fresh
// memory, which costs tens of microseconds per call.)
static constexpr uint64_t kScratchKeep = 256ull << 20;

static int scratch_pool(cudaMemPool_t* out) {
  static std::mutex mu;
  static cudaMemPool_t pools[64] = {};
  int dev = 0;
  FDR_CUDA(cudaGetDevice(&dev));
  FDR_CHECK_ARG(dev >= 0 && dev < 64, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lock(mu);
  if (!pools[dev]) {
    cudaMemPoolProps props;
    memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    FDR_CUDA(cudaMemPoolCreate(&pool, &props));
    uint64_t keep = kScratchKeep;
    FDR_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    pools[dev] = pool;
  }
  *out = pools[dev];
  return FDR_OK;
}

int scratch_alloc(void** p, size_t bytes, cudaStream_t s) {
  *p = nullptr;
  if (bytes == 0) return FDR_OK;
  cudaMemPool_t pool = nullptr;
  FDR_TRY(scratch_pool(&pool));
  FDR_CUDA(cudaMallocFromPoolAsync(p, bytes, pool, s));
  return FDR_OK;
}

void scratch_free(void* p, cudaStream_t s) {
  if (p) cudaFreeAsync(p, s);
}

int sm_count() {
  static int cached[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  if (dev < 64 && cached[dev]) return cached[dev];
  int n = 0;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
    n = 148;
  if (dev < 64) cached[dev] = n;
  return n;
}

}  // namespace fdr

extern "C" {

const char* fdr_version(void) { return "fdr_b200 0.1.0 (sm_100a)"; }

const char* fdr_last_error_string(void) { return fdr::g_last_error.c_str(); }

int64_t fdr_kernel_launches(void) { return fdr::g_launches.load(std::memory_order_relaxed); }

const char* fdr_status_string(int status) {
  switch (status) {
    case FDR_OK: return "FDR_OK";
    case FDR_ERR_INVALID_ARGUMENT: return "FDR_ERR_INVALID_ARGUMENT";
    case FDR_ERR_UNSUPPORTED_SIZE: return "FDR_ERR_UNSUPPORTED_SIZE";
    case FDR_ERR_UNSUPPORTED_WINDOW: return "FDR_ERR_UNSUPPORTED_WINDOW";
    case FDR_ERR_OUT_OF_MEMORY: return "FDR_ERR_OUT_OF_MEMORY";
    case FDR_ERR_CUDA: return "FDR_ERR_CUDA";
    case FDR_ERR_CAPACITY: return "FDR_ERR_CAPACITY";
    case FDR_ERR_NO_DEVICE: return "FDR_ERR_NO_DEVICE";
    default: return "FDR_ERR_UNKNOWN";
  }
}

int fdr_selftest_bounded_wait(int64_t limit_ns, fdr_stream_t stream) {
  FDR_CHECK_ARG(limit_ns > 0 && limit_ns <= 1000000000LL, "selftest: limit must be in (0, 1 s]");
  return fdr::bounded_wait_selftest((unsigned long long)limit_ns, (cudaStream_t)stream);
}

int fdr_synchronize(fdr_stream_t stream) {
  if (stream) {
    FDR_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
  } else {
    FDR_CUDA(cudaDeviceSynchronize());
  }
  const int st = fdr::fused_take_fault();
  if (st != FDR_OK) return st;
  unsigned long long w = 0;
  fdr::debug_take_fault(&w);
  if (w) {
    fdr::set_error(FDR_ERR_CUDA, "debug index check failed (source unit %u, line %u)",
                   (unsigned)((w >> 32) & 0x7fffffffu), (unsigned)(w & 0xffffffffu));
    return FDR_ERR_CUDA;
  }
  return FDR_OK;
}

int fdr_debug_build(void) {
#ifdef FDR_DEBUG
  return 1;
#else
  return 0;
#endif
}

int fdr_debug_fault(uint64_t* word, fdr_stream_t stream) {
  FDR_CHECK_ARG(word != nullptr, "fdr_debug_fault: NULL argument");
  if (stream) {
    FDR_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
  } else {
    FDR_CUDA(cudaDeviceSynchronize());
  }
  unsigned long long w = 0;
  fdr::debug_take_fault(&w);
  *word = (uint64_t)w;
  return FDR_OK;
}

int64_t fdr_calc_nl(int64_t Nt, int64_t Nr, const int64_t* factors, int nfactors) {
  if (Nt < 1 || Nr < 1) return -1;
  return fdr::nextprod(factors, nfactors, Nt + Nr - 1);
}

int64_t fdr_grow_nr(int64_t Nt, int64_t Nr, const int64_t* factors, int nfactors) {
  int64_t nl = fdr_calc_nl(Nt, Nr, factors, nfactors);
  return nl < 0 ? -1 : nl - Nt + 1;
}

int64_t fdr_estimate_memory(int64_t Nf, int64_t Nt, int64_t Nr, int64_t Ni, int64_t No,
                            const int64_t* factors, int nfactors) {
  int64_t Nl = fdr_calc_nl(Nt, Nr, factors, nfactors);
  if (Nl < 0 || Nf < 1) return -1;
  Ni += 3;
  const int64_t Nz = 3;
  return 4 * ((Nf * Nt) * Ni + (Nf * Nl) * Nz + (Nf * Nr) * No);
}

}  // extern "C"
