// Brute-force integer-shift FDR (src/intfdr.jl of FrequencyDriftRateTransforms.jl).
//
// intfdr! (intfdr.jl:34-45) materialises an Nf x Nt x Nr work array of circularly shifted
// columns and reduces it with Base's sum! over dims=2, which starts from 0f0 and adds the
// columns one after another in time order.  Here each output element is formed directly
// from the spectrogram with the same sequence of float32 additions, so the result is
// bit-identical without the work array: fdr[n, j] = (((0 + s[n+n_0, 0]) + s[n+n_1, 1]) + ...)
// with n_t = round(rate_j * t) (intfdr.jl:10, ties to even) and indices modulo Nf.
#include <math.h>

#define FDR_TU_ID 3
#include "fdr_internal.cuh"

namespace fdr {

constexpr int kShiftParamWords = 4096;  // shifts carried in one launch's parameters
constexpr int kIntfdrThreads = 256;
constexpr int kIntfdrVec = 4;            // channels per thread

struct ShiftTable {
  int32_t sh[kShiftParamWords];  // shift (mod Nf) of rate jj at time t: sh[jj*Nt + t]
};

__global__ void __launch_bounds__(kIntfdrThreads)
intfdr_kernel(const float* __restrict__ spec, long long Nf, int Nt, int nrates,
              float* __restrict__ fdr, const __grid_constant__ ShiftTable tab) {
  const long long base = (long long)blockIdx.x * (kIntfdrThreads * kIntfdrVec) + threadIdx.x;
  for (int jj = 0; jj < nrates; ++jj) {
    float acc[kIntfdrVec];
#pragma unroll
    for (int v = 0; v < kIntfdrVec; ++v) acc[v] = 0.0f;
    for (int t = 0; t < Nt; ++t) {
      const long long sh = tab.sh[jj * Nt + t];
      const float* col = spec + (long long)t * Nf;
#pragma unroll
      for (int v = 0; v < kIntfdrVec; ++v) {
        const long long n = base + v * kIntfdrThreads;
        if (n < Nf) {
          long long idx = n + sh;
          if (idx >= Nf) idx -= Nf;
          if (FDR_DBG_OK(idx >= 0 && idx < Nf)) acc[v] = __fadd_rn(acc[v], __ldg(col + idx));
        }
      }
    }
    float* out = fdr + (long long)jj * Nf;
#pragma unroll
    for (int v = 0; v < kIntfdrVec; ++v) {
      const long long n = base + v * kIntfdrThreads;
      if (n < Nf) out[n] = acc[v];
    }
  }
}

// Tiled form for shift sets that stay close together (every rate of a launch within a
// window of each column): a CTA stages, per time step t, the spectrogram channels
// [n0 + lo_t, n0 + TN + hi_t] (modulo Nf) in shared memory and forms its TN output channels
// of every rate from there, with the same sequence of float32 additions.  Each spectrogram
// element is then read from HBM about once per CTA instead of once per rate.
constexpr int kTiledMaxNt = 64;
constexpr int kTiledMaxWords = 24576;  // shared-memory window floats (96 KB)

struct TiledTable {
  int32_t rel[kShiftParamWords];  // shift of rate jj at time t, minus lo_t: rel[jj*Nt + t]
  int32_t lo[kTiledMaxNt];        // smallest signed shift at time t (in (-Nf/2, Nf/2])
  int32_t off[kTiledMaxNt + 1];   // start of time step t's window in shared memory
};

template <int TNV>  // TN = TNV * kIntfdrThreads output channels per CTA
__global__ void __launch_bounds__(kIntfdrThreads)
intfdr_tiled_kernel(const float* __restrict__ spec, long long Nf, int Nt, int nrates,
                    float* __restrict__ fdr, const __grid_constant__ TiledTable tab) {
  constexpr int TN = TNV * kIntfdrThreads;
  extern __shared__ float win[];
  const long long n0 = (long long)blockIdx.x * TN;
  for (int t = 0; t < Nt; ++t) {
    const float* col = spec + (long long)t * Nf;
    const int len = tab.off[t + 1] - tab.off[t];
    long long idx = (n0 + tab.lo[t]) % Nf;
    if (idx < 0) idx += Nf;
    for (int i = threadIdx.x; i < len; i += kIntfdrThreads) {
      long long g = idx + i;
      if (g >= Nf) g -= Nf;  // len <= TN + Nf/4 < Nf: one wrap at most
      if (FDR_DBG_OK(g >= 0 && g < Nf && tab.off[t] + i < kTiledMaxWords)) win[tab.off[t] + i] = __ldg(col + g);
    }
  }
  __syncthreads();
  // the TNV channels of a thread are independent sums: interleaved, each in time order
  for (int jj = 0; jj < nrates; ++jj) {
    float acc[TNV];
#pragma unroll
    for (int v = 0; v < TNV; ++v) acc[v] = 0.0f;
    for (int t = 0; t < Nt; ++t) {
      const float* w = win + tab.off[t] + tab.rel[jj * Nt + t] + threadIdx.x;
#pragma unroll
      for (int v = 0; v < TNV; ++v)
        if (FDR_DBG_OK(tab.off[t] + tab.rel[jj * Nt + t] + (int)threadIdx.x + v * kIntfdrThreads < tab.off[t + 1]))
          acc[v] = __fadd_rn(acc[v], w[v * kIntfdrThreads]);
    }
#pragma unroll
    for (int v = 0; v < TNV; ++v) {
      const long long n = n0 + threadIdx.x + v * kIntfdrThreads;
      if (n < Nf) fdr[(long long)jj * Nf + n] = acc[v];
    }
  }
}

__global__ void intshift_kernel(const float* __restrict__ din, long long Nf, int Nt,
                                float* __restrict__ dout, const __grid_constant__ ShiftTable tab) {
  const long long total = Nf * Nt;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long t = e / Nf, n = e - t * Nf;
    long long idx = n + tab.sh[t];
    if (idx >= Nf) idx -= Nf;
    if (FDR_DBG_OK(idx >= 0 && idx < Nf)) dout[e] = din[idx + t * Nf];
  }
}

// round(rate * t) as Julia computes it for a Float64 or Float32 rate, reduced mod Nf.
static int64_t shift_of(double rate, int64_t t, int rate_type) {
  double v;
  if (rate_type == FDR_RATES_F32) {
    volatile float p = (float)rate * (float)t;  // single-precision product, rounded once
    v = (double)nearbyintf(p);
  } else {
    v = nearbyint(rate * (double)t);
  }
  return (int64_t)v;
}

static int32_t mod_nf(int64_t sh, int64_t Nf) {
  int64_t m = sh % Nf;
  if (m < 0) m += Nf;
  return (int32_t)m;
}

// Tiled launch of rates [j0, j0 + nr) if their shifts fit the shared-memory windows;
// false if not (the caller uses the untiled kernel).
static bool run_intfdr_tiled(const float* spec, int64_t Nf, int64_t Nt, int64_t j0, int64_t nr,
                             float* fdr, const std::vector<int32_t>& sh, cudaStream_t s, int* status) {
  *status = FDR_OK;
  if (Nt > kTiledMaxNt || nr * Nt > kShiftParamWords || Nf < 2 * kIntfdrThreads) return false;
  TiledTable tab;
  int64_t spans = 0;
  for (int64_t t = 0; t < Nt; ++t) {
    int64_t lo = 0, hi = 0;
    for (int64_t j = 0; j < nr; ++j) {
      int64_t v = sh[(j0 + j) * Nt + t];  // in [0, Nf)
      if (v > Nf / 2) v -= Nf;            // signed representative in (-Nf/2, Nf/2]
      if (j == 0 || v < lo) lo = v;
      if (j == 0 || v > hi) hi = v;
    }
    if (hi - lo > Nf / 4) return false;
    tab.lo[t] = (int32_t)lo;
    spans += hi - lo;
    for (int64_t j = 0; j < nr; ++j) {
      int64_t v = sh[(j0 + j) * Nt + t];
      if (v > Nf / 2) v -= Nf;
      tab.rel[j * Nt + t] = (int32_t)(v - lo);
    }
  }
  int TN = 0;
  for (int tn = 1024; tn >= 256; tn /= 2)  // TN <= Nf/2 and spans <= Nf/4: windows < Nf
    if (Nt * (int64_t)tn + spans <= kTiledMaxWords && 2 * (int64_t)tn <= Nf) { TN = tn; break; }
  if (TN == 0) return false;
  tab.off[0] = 0;
  for (int64_t t = 0; t < Nt; ++t) {
    int64_t hi = 0;
    for (int64_t j = 0; j < nr; ++j) hi = std::max<int64_t>(hi, tab.rel[j * Nt + t]);
    tab.off[t + 1] = tab.off[t] + (int32_t)(TN + hi);  // channels n0 + lo .. n0 + TN - 1 + hi
  }
  const size_t smem = sizeof(float) * (size_t)tab.off[Nt];
  cudaError_t ea = cudaSuccess;
#define TILED(V)                                                                                \
  if (TN == V * kIntfdrThreads) {                                                               \
    ea = cudaFuncSetAttribute(intfdr_tiled_kernel<V>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                              (int)(sizeof(float) * kTiledMaxWords));                           \
    if (ea == cudaSuccess)                                                                      \
      intfdr_tiled_kernel<V><<<(unsigned)cdiv(Nf, TN), kIntfdrThreads, smem, s>>>(             \
          spec, Nf, (int)Nt, (int)nr, fdr + j0 * Nf, tab);                                      \
  }
  TILED(1) TILED(2) TILED(4)
#undef TILED
  if (ea != cudaSuccess) { *status = cuda_status(ea, "intfdr tiled attribute"); return true; }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) *status = cuda_status(e, "intfdr_tiled_kernel");
  return true;
}

static int run_intfdr(const float* spec, int64_t Nf, int64_t Nt, int64_t Nr, float* fdr,
                      const std::vector<int32_t>& sh, cudaStream_t s) {
  FDR_CHECK_ARG(Nt <= kShiftParamWords, "intfdr: Nt=%lld exceeds %d", (long long)Nt,
                kShiftParamWords);
  const int64_t chunk = std::max<int64_t>(1, kShiftParamWords / Nt);
  const unsigned gx = (unsigned)cdiv(Nf, kIntfdrThreads * kIntfdrVec);
  ShiftTable tab;
  for (int64_t j0 = 0; j0 < Nr; j0 += chunk) {
    const int64_t nr = std::min(chunk, Nr - j0);
    int st = FDR_OK;
    if (run_intfdr_tiled(spec, Nf, Nt, j0, nr, fdr, sh, s, &st)) {
      if (st != FDR_OK) return st;
      continue;
    }
    memcpy(tab.sh, sh.data() + j0 * Nt, sizeof(int32_t) * nr * Nt);
    intfdr_kernel<<<gx, kIntfdrThreads, 0, s>>>(spec, Nf, (int)Nt, (int)nr, fdr + j0 * Nf, tab);
    FDR_LAUNCH_CHECK("intfdr_kernel");
  }
  return FDR_OK;
}

}  // namespace fdr

using namespace fdr;

extern "C" {

int fdr_intshift(const float* din, int64_t Nf, int64_t Nt, double rate, int rate_type,
                 float* dout, fdr_stream_t stream) {
  FDR_CHECK_ARG(din && dout, "intshift!: NULL array");
  FDR_CHECK_ARG(Nf >= 1 && Nt >= 1, "intshift!: bad sizes");
  FDR_CHECK_ARG(Nt <= kShiftParamWords, "intshift!: Nt too large");
  FDR_CHECK_ARG(rate_type == FDR_RATES_F64 || rate_type == FDR_RATES_F32, "intshift!: bad rate type");
  ShiftTable tab;
  for (int64_t t = 0; t < Nt; ++t) tab.sh[t] = mod_nf(shift_of(rate, t, rate_type), Nf);
  const long long total = Nf * Nt;
  unsigned g = (unsigned)std::max<long long>(1, std::min<long long>(cdiv(total, 256), sm_count() * 16LL));
  intshift_kernel<<<g, 256, 0, (cudaStream_t)stream>>>(din, Nf, (int)Nt, dout, tab);
  FDR_LAUNCH_CHECK("intshift_kernel");
  return FDR_OK;
}

int fdr_intfdr(const float* spec, int64_t Nf, int64_t Nt, const double* rates, int64_t Nr,
               int rate_type, float* fdr, fdr_stream_t stream) {
  FDR_CHECK_ARG(spec && fdr, "intfdr!: NULL array");
  FDR_CHECK_ARG(Nf >= 1 && Nt >= 1 && Nr >= 0, "intfdr!: bad sizes");
  FDR_CHECK_ARG(Nr == 0 || rates, "intfdr!: rates is NULL");
  FDR_CHECK_ARG(rate_type == FDR_RATES_F64 || rate_type == FDR_RATES_F32, "intfdr!: bad rate type");
  std::vector<int32_t> sh((size_t)(Nr * Nt));
  for (int64_t j = 0; j < Nr; ++j)
    for (int64_t t = 0; t < Nt; ++t) sh[j * Nt + t] = mod_nf(shift_of(rates[j], t, rate_type), Nf);
  return run_intfdr(spec, Nf, Nt, Nr, fdr, sh, (cudaStream_t)stream);
}

int fdr_intfdr_shifts(const float* spec, int64_t Nf, int64_t Nt, const int64_t* shifts,
                      int64_t Nr, float* fdr, fdr_stream_t stream) {
  FDR_CHECK_ARG(spec && fdr, "intfdr!: NULL array");
  FDR_CHECK_ARG(Nf >= 1 && Nt >= 1 && Nr >= 0, "intfdr!: bad sizes");
  FDR_CHECK_ARG(Nr == 0 || shifts, "intfdr!: shifts is NULL");
  std::vector<int32_t> sh((size_t)(Nr * Nt));
  for (int64_t i = 0; i < Nr * Nt; ++i) sh[i] = mod_nf(shifts[i], Nf);
  return run_intfdr(spec, Nf, Nt, Nr, fdr, sh, (cudaStream_t)stream);
}

}  // extern "C"
