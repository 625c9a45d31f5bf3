// Fourier-domain shift FDR (src/fftfdr.jl of FrequencyDriftRateTransforms.jl):
// fftfdr_workspace (:39-59), fftfdr_workspace! (:69-84), fdshiftsum! (:86-96),
// fdshift! (:104-111), fftfdr! (:126-134).
//
// The phasor of time step t and channel-bin k is cispi(2*k*t*r/Nf) with the argument
// formed in Float32 exactly as the reference does (fftfdr.jl:10-12): Float32(2*k*t) * r,
// then / Float32(Nf), each rounded once.  The sum over t runs in time order from zero in
// complex float32, as Base's sum! over dims=2 accumulates.
#include <string.h>

#include "fft_engine.cuh"

struct fdr_fft_ws {
  int64_t Nf = 0, Nt = 0, K = 0;
  float2* F = nullptr;        // dest_rfft (K x Nt)
  float2* P = nullptr;        // dest_phasor (K x Nt)
  float2* S = nullptr;        // per-rate sums (K x kRateChunk)
  float2* rscratch = nullptr;
  int64_t rscratch_pairs = 0;
};

namespace fdr {

constexpr int kRateChunk = 32;

struct RateParams {
  float r[kRateChunk];
};

__device__ __forceinline__ float2 phasor_ref(long long k, long long t, float r, float Nf_f) {
  float x = __fdiv_rn(__fmul_rn(__ll2float_rn(2 * k * t), r), Nf_f);
  return cispif(x);
}

// S[k + jj*K] = sum_t F[k, t] * phasor(k, t, r_jj)
__global__ void phasor_sum_kernel(const float2* __restrict__ F, long long K, long long Nt,
                                  long long Nf, int nr, float2* __restrict__ S,
                                  const __grid_constant__ RateParams rp) {
  const long long total = K * nr;
  const float Nf_f = __ll2float_rn(Nf);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long jj = e / K, k = e - jj * K;
    const float r = rp.r[jj];
    float2 acc = make_float2(0.f, 0.f);
    for (long long t = 0; t < Nt; ++t) {
      float2 p = cmul_rn(F[k + t * K], phasor_ref(k, t, r, Nf_f));
      acc = make_float2(__fadd_rn(acc.x, p.x), __fadd_rn(acc.y, p.y));
    }
    S[e] = acc;
  }
}

// P[k, t] = F[k, t] * phasor(k, t, r)
__global__ void phasor_kernel(const float2* __restrict__ F, long long K, long long Nt, long long Nf,
                              float r, float2* __restrict__ P) {
  const long long total = K * Nt;
  const float Nf_f = __ll2float_rn(Nf);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long t = e / K, k = e - t * K;
    P[e] = cmul_rn(F[e], phasor_ref(k, t, r, Nf_f));
  }
}

static unsigned grid_1d(long long total) {
  long long b = cdiv(total, 256);
  long long cap = (long long)sm_count() * 16;
  return (unsigned)std::max(1LL, std::min(b, cap));
}

static void release(fdr_fft_ws* ws) {
  if (!ws) return;
  cudaFree(ws->F);
  cudaFree(ws->P);
  cudaFree(ws->S);
  cudaFree(ws->rscratch);
  delete ws;
}

}  // namespace fdr

using namespace fdr;

extern "C" {

int fdr_fftfdr_workspace(fdr_fft_ws** out, const float* spectrogram, int64_t Nf, int64_t Nt,
                         fdr_stream_t stream) {
  FDR_CHECK_ARG(out && spectrogram, "fftfdr_workspace: NULL argument");
  FDR_CHECK_ARG(Nf >= 1 && Nt >= 1, "fftfdr_workspace: bad sizes");
  *out = nullptr;
  fdr_fft_ws* ws = new fdr_fft_ws();
  ws->Nf = Nf; ws->Nt = Nt; ws->K = Nf / 2 + 1;
  const int64_t K = ws->K;
  const int64_t per = real_fft_scratch_per_pair(Nf);
  int64_t pairs = cdiv(std::max<int64_t>(Nt, kRateChunk), 2);
  const int64_t cap = std::max<int64_t>(1, (int64_t(256) << 20) / (int64_t)(per * sizeof(float2)));
  ws->rscratch_pairs = std::min(pairs, cap);
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = cudaMalloc(&ws->F, sizeof(float2) * K * Nt);
  if (e == cudaSuccess) e = cudaMalloc(&ws->P, sizeof(float2) * K * Nt);
  if (e == cudaSuccess) e = cudaMalloc(&ws->S, sizeof(float2) * K * kRateChunk);
  if (e == cudaSuccess) e = cudaMalloc(&ws->rscratch, sizeof(float2) * per * ws->rscratch_pairs);
  if (e != cudaSuccess) {
    int st = cuda_status(e, "fftfdr_workspace allocation");
    release(ws);
    return st;
  }
  int st = fdr_fftfdr_workspace_update(ws, spectrogram, Nf, Nt, stream);
  if (st != FDR_OK) { release(ws); return st; }
  *out = ws;
  return FDR_OK;
}

int fdr_fftfdr_workspace_update(fdr_fft_ws* ws, const float* spectrogram, int64_t Nf, int64_t Nt,
                                fdr_stream_t stream) {
  FDR_CHECK_ARG(ws && spectrogram, "fftfdr_workspace!: NULL argument");
  // fftfdr.jl:71-76
  FDR_CHECK_ARG(Nf == ws->Nf && Nt == ws->Nt, "input spectrogram has unexpected size");
  return rfft_columns(spectrogram, Nf, Nt, Nf, ws->F, ws->K, ws->rscratch, ws->rscratch_pairs,
                      (cudaStream_t)stream);
}

int fdr_fftfdr_destroy(fdr_fft_ws* ws) {
  if (ws) {
    cudaDeviceSynchronize();
    release(ws);
  }
  return FDR_OK;
}

int fdr_fftfdr_rfft_buffer(fdr_fft_ws* ws, void** F) {
  FDR_CHECK_ARG(ws && F, "NULL argument");
  *F = ws->F;
  return FDR_OK;
}

int fdr_fdshiftsum(fdr_fft_ws* ws, float rate, float* dest, fdr_stream_t stream) {
  FDR_CHECK_ARG(ws && dest, "fdshiftsum!: NULL argument");
  return fdr_fftfdr(ws, &rate, 1, dest, stream);
}

int fdr_fdshift(fdr_fft_ws* ws, float rate, float* dest, fdr_stream_t stream) {
  FDR_CHECK_ARG(ws && dest, "fdshift!: NULL argument");
  cudaStream_t s = (cudaStream_t)stream;
  phasor_kernel<<<grid_1d(ws->K * ws->Nt), 256, 0, s>>>(ws->F, ws->K, ws->Nt, ws->Nf, rate, ws->P);
  FDR_LAUNCH_CHECK("phasor_kernel");
  return irfft_columns(ws->P, ws->K, ws->Nt, ws->Nf, dest, ws->Nf, ws->rscratch,
                       ws->rscratch_pairs, s);
}

int fdr_fftfdr(fdr_fft_ws* ws, const float* rates, int64_t Nr, float* fdr, fdr_stream_t stream) {
  FDR_CHECK_ARG(ws && fdr, "fftfdr!: NULL argument");
  FDR_CHECK_ARG(Nr >= 0 && (Nr == 0 || rates), "fftfdr!: bad rates");
  cudaStream_t s = (cudaStream_t)stream;
  RateParams rp;
  for (int64_t j0 = 0; j0 < Nr; j0 += kRateChunk) {
    const int nr = (int)std::min<int64_t>(kRateChunk, Nr - j0);
    memset(&rp, 0, sizeof(rp));
    for (int i = 0; i < nr; ++i) rp.r[i] = rates[j0 + i];
    phasor_sum_kernel<<<grid_1d(ws->K * nr), 256, 0, s>>>(ws->F, ws->K, ws->Nt, ws->Nf, nr, ws->S, rp);
    FDR_LAUNCH_CHECK("phasor_sum_kernel");
    FDR_TRY(irfft_columns(ws->S, ws->K, nr, ws->Nf, fdr + j0 * ws->Nf, ws->Nf, ws->rscratch,
                          ws->rscratch_pairs, s));
  }
  return FDR_OK;
}

}  // extern "C"
