// Internal helpers shared by the FDR CUDA translation units (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string>
#include <vector>

#include "../../include/fdr_b200.h"

namespace fdr {

// ------------------------------------------------------------------------------------
// Error reporting: every C entry point returns an fdr_status; the message of the last
// failure on the calling host thread is kept for fdr_last_error_string().
// ------------------------------------------------------------------------------------
void set_error(int status, const char* fmt, ...);
int cuda_status(cudaError_t e, const char* what);

#define FDR_CHECK_ARG(cond, ...)                                              \
  do {                                                                        \
    if (!(cond)) {                                                            \
      fdr::set_error(FDR_ERR_INVALID_ARGUMENT, __VA_ARGS__);                  \
      return FDR_ERR_INVALID_ARGUMENT;                                        \
    }                                                                         \
  } while (0)

#define FDR_CUDA(call)                                                        \
  do {                                                                        \
    cudaError_t e__ = (call);                                                 \
    if (e__ != cudaSuccess) return fdr::cuda_status(e__, #call);              \
  } while (0)

#define FDR_TRY(call)                                                         \
  do {                                                                        \
    int s__ = (call);                                                         \
    if (s__ != FDR_OK) return s__;                                            \
  } while (0)

// Counts a kernel launch (fdr_kernel_launches) and checks the launch error; placed after
// every <<<>>> launch of the library.
void count_launch(int n = 1);
#define FDR_LAUNCH_CHECK(what)                                                \
  do {                                                                        \
    fdr::count_launch();                                                      \
    FDR_CUDA(cudaPeekAtLastError());                                          \
  } while (0)

// ------------------------------------------------------------------------------------
// Debug build (-DFDR_DEBUG, libfdrb200_debug.so): FDR_DBG_OK(cond) guards a device memory
// access; a false condition records the first violation of the translation unit (its
// FDR_TU_ID and source line) in a device word and the access is skipped.  fdr_synchronize
// reads and clears every unit's word and reports a violation as FDR_ERR_CUDA.  In the
// normal build FDR_DBG_OK(cond) is `true` and costs nothing.
// ------------------------------------------------------------------------------------
void register_debug_reader(int (*take)(unsigned long long*));
int debug_take_fault(unsigned long long* word);  // first recorded violation, 0 if none
#ifndef FDR_TU_ID
#define FDR_TU_ID 0
#endif
#ifdef FDR_DEBUG
namespace dbg {
static __device__ unsigned long long fault_word;
static int take(unsigned long long* out) {
  unsigned long long w = 0;
  if (cudaMemcpyFromSymbol(&w, fault_word, sizeof(w)) != cudaSuccess) {
    (void)cudaGetLastError();
    *out = 0;
    return 0;
  }
  if (w) {
    const unsigned long long z = 0;
    (void)cudaMemcpyToSymbol(fault_word, &z, sizeof(z));
  }
  *out = w;
  return 0;
}
struct Registration {
  Registration() { register_debug_reader(&take); }
};
static Registration registration;
__device__ __forceinline__ bool check(bool ok, unsigned line) {
  if (!ok)
    atomicCAS(&fault_word, 0ull, (1ull << 63) | ((unsigned long long)FDR_TU_ID << 32) | line);
  return ok;
}
}  // namespace dbg
#define FDR_DBG_OK(cond) (fdr::dbg::check((cond), __LINE__))
#else
#define FDR_DBG_OK(cond) (true)
#endif

// ------------------------------------------------------------------------------------
// Complex helpers (float2 = complex64 with .x real, .y imaginary)
// ------------------------------------------------------------------------------------
// Complex add / subtract: one packed FP32 add (FADD2) on sm_100 (the same IEEE round-to-nearest
// sums as two scalar adds; measured 6% faster output and 1% faster czt passes).
#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ >= 1000)
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
#else
__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
#endif
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__host__ __device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// multiply by +i (s=+1) or -i (s=-1)
__host__ __device__ __forceinline__ float2 cmul_i(float2 a, int s) {
  return s > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}
// (a.x + i a.y) * (b.x + i b.y) with each product rounded separately and no FMA
// contraction, as Julia's ComplexF32 `*` computes it.
__device__ __forceinline__ float2 cmul_rn(float2 a, float2 b) {
  return make_float2(__fsub_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)),
                     __fadd_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}

// cispi(x) = exp(i*pi*x) for a float argument (CUDA's sincospif reduces x exactly).
__device__ __forceinline__ float2 cispif(float x) {
  float s, c;
  sincospif(x, &s, &c);
  return make_float2(c, s);
}

// exp(i*pi*h) where h = num / den half-turns is given exactly as an integer fraction
// reduced in integer arithmetic: the residue (num mod 2*den) is exact, only the final
// conversion of the residue to a float in [-1, 1) rounds.
__device__ __forceinline__ float2 cispi_frac(long long num, long long den2 /* = 2*den */) {
  long long r = num % den2;
  if (r < 0) r += den2;
  // h = 2*r/den2 in [0, 2); map to [-1, 1)
  double h = 2.0 * (double)r / (double)den2;
  if (h >= 1.0) h -= 2.0;
  return cispif((float)h);
}

// exp(i*pi*h) for a double h reduced modulo 2 in double precision first.
__device__ __forceinline__ float2 cispi_d(double h) {
  double r = h - 2.0 * rint(0.5 * h);
  return cispif((float)r);
}

// ------------------------------------------------------------------------------------
// Small host utilities
// ------------------------------------------------------------------------------------
int64_t nextprod(const int64_t* factors, int nfactors, int64_t n);
bool factorize(int64_t n, std::vector<int>& radices, int max_prime);
inline int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }
inline bool is_pow2(int64_t n) { return n > 0 && (n & (n - 1)) == 0; }
inline int ilog2(int64_t n) { int l = 0; while ((int64_t(1) << l) < n) ++l; return l; }

// Temporary device memory from the stream-ordered pool.
int scratch_alloc(void** p, size_t bytes, cudaStream_t s);
void scratch_free(void* p, cudaStream_t s);
// Stream-ordered store of a small host array (whole 32-bit words) into device memory by
// kernel parameters (no copy engine).
int upload_words(void* dev, const void* host, size_t bytes, cudaStream_t s);
// Per-host-thread mapped pinned buffer of at least `bytes` for the small results of a call,
// written by kernels through *dev and read through *host after a synchronisation.
int pinned_staging(size_t bytes, void** host, void** dev);
// The address kernels use for a caller's buffer: device or managed memory as is, mapped
// pinned host memory through its device pointer; anything else is FDR_ERR_INVALID_ARGUMENT.
int device_view(void* p, void** dp, const char* what);

// Current device's SM count (cached per device).
int sm_count();

// fdrutils.cu helpers shared with the ZDT driver.
int upload_ptrs(const void* const* host, int64_t nb, void*** dev, cudaStream_t s);
int stats_device(const float* const* d_mats, int64_t nb, int64_t Nf, int64_t Nrb, double* d_ms,
                 int snr_mode, double snr, cudaStream_t s);
// Float32 fdrstats in the reference's pairwise order over nb*Nrb columns (device pointer
// array d_mats, or the contiguous matrix `base` when d_mats is NULL).  `part` holds
// 2*ncols*pairwise_stats_parts(Nf, ncols, smax) floats of scratch; d_ms receives m, s and
// the threshold fdrdenormalize(snr, m, s) (snr_mode FDR_SNR_F64 / FDR_SNR_F32).  leafmax,
// when set, receives the maximum of every pairwise leaf (the proto-hit gate).
int pairwise_stats_parts(long long Nf, long long ncols, int smax);
int pairwise_stats_launch(const float* const* d_mats, const float* base, long long nb, long long Nf,
                          long long Nrb, float* part, int smax, double* d_ms, int snr_mode,
                          double snr, cudaStream_t s, float* leafmax = nullptr);
// findprotohits(...; snr=true): fdrstats, the threshold in snr_mode's type (d_ms = m, s,
// threshold) and the proto-hits, reading again only the leaves whose maximum reaches the
// threshold.  Synchronises s.
int snr_protohits_run(const float* const* d_mats, int64_t nb, int64_t Nf, int64_t Nrb, double* d_ms,
                      int snr_mode, double snr, int64_t* hits, int64_t capacity, int64_t* count,
                      double* thr_used, cudaStream_t s);
int moments_accumulate(const float* x, long long Nf, long long ncols, double* acc, cudaStream_t s);
int stats_finalize_launch(const double* acc, long long ncols, long long Nf, double* d_ms,
                          cudaStream_t s);
int threshold_launch(const double* d_ms, int snr_mode, double snr, double* d_thr, cudaStream_t s);
int hits_run(const float* const* d_mats, int64_t nb, int64_t Nf, int64_t Nrb, double thr_host,
             const double* d_thr, int64_t* hits, int64_t capacity, int64_t* count,
             double* thr_used, cudaStream_t s);

}  // namespace fdr
