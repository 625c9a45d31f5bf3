// Chirp-Z De-Doppler Transform (ZDT) workspace and staged stages, following
// src/zdtfdr.jl of FrequencyDriftRateTransforms.jl: input! (:209-212), preprocess!
// (:221-239), convolve! (:249-253), postprocess! (:297-321), output! (:328-331),
// computeV! (:173-187) and the zdtfdr! driver (:349-378).
//
// Phase arguments: by default each chirp factor is computed from the same Float32
// argument the reference forms (e.g. vlow: Float32(-k*l^2) * dr / Float32(Nf),
// zdtfdr.jl:141), with every product and quotient rounded separately (no FMA
// contraction), and cispi evaluated by sincospif.  With FDR_ZDT_EXACT_PHASE the argument
// is formed and reduced modulo 2 in float64 instead, which removes the reference's
// argument rounding (about 4e-5 half-turns at k*l^2 ~ 2^33).
#include <string.h>

#include "fft_engine.cuh"
#include "zdt_ws.cuh"

namespace fdr {

__device__ __forceinline__ float f32_of_i64(long long v) { return __ll2float_rn(v); }

// prephase(k, l, r0, dr, Nf) = cispi(k*l*(l*dr + 2*r0)/Nf)   (zdtfdr.jl:196-198)
__device__ __forceinline__ float2 prephase_ref(long long k, long long l, float r0, float dr,
                                               float Nf_f) {
  float inner = __fadd_rn(__fmul_rn(f32_of_i64(l), dr), __fmul_rn(2.0f, r0));
  float x = __fdiv_rn(__fmul_rn(f32_of_i64(k * l), inner), Nf_f);
  return cispif(x);
}
__device__ __forceinline__ float2 prephase_exact(long long k, long long l, float r0, float dr,
                                                 double Nf) {
  double kl = (double)(k * l);
  double h = (kl * (double)l * (double)dr + 2.0 * kl * (double)r0) / Nf;
  return cispi_d(h);
}

// vlow(k, l, dr, Nf) = cispi(-k*l^2*dr/Nf)   (zdtfdr.jl:140-142)
__device__ __forceinline__ float2 vlow_ref(long long k, long long l, float dr, float Nf_f) {
  float x = __fdiv_rn(__fmul_rn(f32_of_i64(-k * l * l), dr), Nf_f);
  return cispif(x);
}
__device__ __forceinline__ float2 vlow_exact(long long k, long long l, float dr, double Nf) {
  double h = -((double)(k * l * l) * (double)dr) / Nf;
  return cispi_d(h);
}

// postphase(k, l, dr, Nf) = cispi(k*l*l*dr/Nf)   (zdtfdr.jl:268-270)
__device__ __forceinline__ float2 postphase_ref(long long k, long long l, float dr, float Nf_f) {
  float x = __fdiv_rn(__fmul_rn(f32_of_i64(k * l * l), dr), Nf_f);
  return cispif(x);
}
__device__ __forceinline__ float2 postphase_exact(long long k, long long l, float dr, double Nf) {
  double h = ((double)(k * l * l) * (double)dr) / Nf;
  return cispi_d(h);
}

__global__ void zdt_preprocess_kernel(const float2* __restrict__ F, float2* __restrict__ Y,
                                      long long K, long long Nt, long long Nl, long long Nf,
                                      float r0, float dr, int exact) {
  const long long total = K * Nl;
  const float Nf_f = __ll2float_rn(Nf);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long l = e / K, k = e - l * K;
    float2 v = make_float2(0.f, 0.f);
    if (l < Nt) {
      float2 ph = exact ? prephase_exact(k, l, r0, dr, (double)Nf) : prephase_ref(k, l, r0, dr, Nf_f);
      v = cmul_rn(F[e], ph);
    }
    Y[e] = v;
  }
}

__global__ void zdt_vinit_kernel(float2* __restrict__ V, long long K, long long Nt, long long Nr,
                                 long long Nl, long long Nf, float dr, int exact) {
  const long long total = K * Nl;
  const float Nf_f = __ll2float_rn(Nf);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long l = e / K, k = e - l * K;
    float2 v = make_float2(0.f, 0.f);
    long long m = -1;
    if (l < Nr) m = l;                        // vlow   (zdtfdr.jl:181)
    else if (l >= Nl - Nt + 1) m = Nl - l;    // vhigh  (zdtfdr.jl:184, :159-161)
    if (m >= 0) v = exact ? vlow_exact(k, m, dr, (double)Nf) : vlow_ref(k, m, dr, Nf_f);
    V[e] = v;
  }
}

// window: 0 rect, 1 hamming, 2 custom (float64 values w[k])
__global__ void zdt_postprocess_kernel(float2* __restrict__ Y, long long K, long long Nr,
                                       long long Nf, float dr, int exact, int window,
                                       const double* __restrict__ wk) {
  const long long total = K * Nr;
  const float Nf_f = __ll2float_rn(Nf);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long l = e / K, k = e - l * K;
    float2 ph = exact ? postphase_exact(k, l, dr, (double)Nf) : postphase_ref(k, l, dr, Nf_f);
    float2 y = Y[e];
    if (window == 0) {
      Y[e] = cmul_rn(y, ph);
    } else {
      // cispi(...)::ComplexF32 * w(k, Nf)::Float64 promotes to ComplexF64 and the product
      // with Ys is rounded to ComplexF32 on store (zdtfdr.jl:268-270, :299-300).
      double w;
      if (window == 1) {
        double x = 2.0 * (double)k / (double)Nf;
        w = 0.53836 + 0.46164 * cospi(x);
      } else {
        w = wk[k];
      }
      double cr = (double)ph.x * w, ci = (double)ph.y * w;
      double yr = (double)y.x, yi = (double)y.y;
      Y[e] = make_float2((float)(yr * cr - yi * ci), (float)(yr * ci + yi * cr));
    }
  }
}

static unsigned grid_1d(long long total) {
  long long b = cdiv(total, 256);
  long long cap = (long long)sm_count() * 16;
  return (unsigned)max(1LL, min(b, cap));
}

void zdt_mark(fdr_zdt* ws, const char* name, cudaStream_t s) {
  if (!ws->timing) return;
  cudaEvent_t e;
  if (cudaEventCreate(&e) != cudaSuccess) return;
  cudaEventRecord(e, s);
  ws->events.push_back(e);
  ws->ev_names.push_back(name);
}

static int zdt_ensure_staged(fdr_zdt* ws, cudaStream_t s);

int zdt_stage_input(fdr_zdt* ws, const float* spec, cudaStream_t s) {
  FDR_CHECK_ARG(spec != nullptr, "input!: spectrogram is NULL");
  FDR_TRY(zdt_ensure_staged(ws, s));
  FDR_TRY(rfft_columns(spec, ws->Nf, ws->Nt, ws->Nf, ws->F, ws->K, ws->rscratch,
                       ws->rscratch_pairs, s));
  ws->F_valid = true;
  ws->A_valid = false;
  return FDR_OK;
}

int zdt_ensure_F(fdr_zdt* ws, cudaStream_t s) {
  if (ws->F_valid) return FDR_OK;
  if (ws->fused && ws->A_valid) {
    FDR_TRY(zdt_fused_A_to_F(ws, s));
    ws->F_valid = true;
    return FDR_OK;
  }
  // Never given a spectrogram: F is whatever the caller left there (the reference's F is
  // uninitialised memory in that case too); treat it as valid.
  ws->F_valid = true;
  return FDR_OK;
}

static int zdt_compute_V(fdr_zdt* ws, cudaStream_t s);

// Y, V and the real-FFT scratch of the staged stages.  Workspaces that run zdtfdr! on the
// fused kernels allocate them (and compute V) on the first staged call only.
static int zdt_ensure_staged(fdr_zdt* ws, cudaStream_t s) {
  if (ws->Y && ws->V && ws->rscratch) return FDR_OK;
  const int64_t K = ws->K, Nl = ws->Nl;
  const int64_t per = real_fft_scratch_per_pair(ws->Nf);
  if (!ws->Y) {
    FDR_CUDA(cudaMalloc(&ws->Y, sizeof(float2) * K * Nl));
    ws->bytes += (int64_t)sizeof(float2) * K * Nl;
  }
  if (!ws->rscratch) {
    FDR_CUDA(cudaMalloc(&ws->rscratch, sizeof(float2) * per * ws->rscratch_pairs));
    ws->bytes += (int64_t)sizeof(float2) * per * ws->rscratch_pairs;
  }
  if (!ws->V) {
    FDR_CUDA(cudaMalloc(&ws->V, sizeof(float2) * K * Nl));
    ws->bytes += (int64_t)sizeof(float2) * K * Nl;
    FDR_TRY(zdt_compute_V(ws, s));
  }
  return FDR_OK;
}

static int zdt_preprocess(fdr_zdt* ws, float r0, cudaStream_t s) {
  FDR_TRY(zdt_ensure_staged(ws, s));
  FDR_TRY(zdt_ensure_F(ws, s));
  zdt_preprocess_kernel<<<grid_1d(ws->K * ws->Nl), 256, 0, s>>>(
      ws->F, ws->Y, ws->K, ws->Nt, ws->Nl, ws->Nf, r0, ws->dr,
      (ws->flags & FDR_ZDT_EXACT_PHASE) ? 1 : 0);
  FDR_LAUNCH_CHECK("zdt_preprocess_kernel");
  return FDR_OK;
}

static int zdt_convolve(fdr_zdt* ws, cudaStream_t s) {
  FDR_TRY(zdt_ensure_staged(ws, s));
  FDR_TRY(fft_strided_inplace(ws->Y, ws->Nl, ws->K, ws->K, 1, -1, 1.f, ws->V, s));
  FDR_TRY(fft_strided_inplace(ws->Y, ws->Nl, ws->K, ws->K, 1, +1, 1.f / (float)ws->Nl, nullptr, s));
  return FDR_OK;
}

static int zdt_postprocess(fdr_zdt* ws, int window, const double* wk, cudaStream_t s) {
  if (window < 0 || window > 2) {
    set_error(FDR_ERR_UNSUPPORTED_WINDOW, "unsupported window type (%d)", window);
    return FDR_ERR_UNSUPPORTED_WINDOW;
  }
  FDR_CHECK_ARG(window != FDR_WINDOW_CUSTOM || wk != nullptr,
                "postprocess!: custom window values are NULL");
  FDR_TRY(zdt_ensure_staged(ws, s));
  zdt_postprocess_kernel<<<grid_1d(ws->K * ws->Nr), 256, 0, s>>>(
      ws->Y, ws->K, ws->Nr, ws->Nf, ws->dr, (ws->flags & FDR_ZDT_EXACT_PHASE) ? 1 : 0, window, wk);
  FDR_LAUNCH_CHECK("zdt_postprocess_kernel");
  return FDR_OK;
}

static int zdt_output(fdr_zdt* ws, float* dest, cudaStream_t s) {
  FDR_CHECK_ARG(dest != nullptr, "output!: dest is NULL");
  FDR_TRY(zdt_ensure_staged(ws, s));
  return irfft_columns(ws->Y, ws->K, ws->Nr, ws->Nf, dest, ws->Nf, ws->rscratch,
                       ws->rscratch_pairs, s);
}

static int zdt_compute_V(fdr_zdt* ws, cudaStream_t s) {
  zdt_vinit_kernel<<<grid_1d(ws->K * ws->Nl), 256, 0, s>>>(
      ws->V, ws->K, ws->Nt, ws->Nr, ws->Nl, ws->Nf, ws->dr,
      (ws->flags & FDR_ZDT_EXACT_PHASE) ? 1 : 0);
  FDR_LAUNCH_CHECK("zdt_vinit_kernel");
  return fft_strided_inplace(ws->V, ws->Nl, ws->K, ws->K, 1, -1, 1.f, nullptr, s);
}

// One staged ZDT (zdtfdr.jl:355-358) for a given r0 into dest.
int zdt_staged_run(fdr_zdt* ws, float r0, float* dest, int window, const double* wk, double* acc,
                   cudaStream_t s) {
  FDR_TRY(zdt_preprocess(ws, r0, s));
  zdt_mark(ws, "preprocess", s);
  FDR_TRY(zdt_convolve(ws, s));
  zdt_mark(ws, "convolve", s);
  FDR_TRY(zdt_postprocess(ws, window, wk, s));
  zdt_mark(ws, "postprocess", s);
  FDR_TRY(zdt_output(ws, dest, s));
  if (acc) FDR_TRY(moments_accumulate(dest, ws->Nf, ws->Nr, acc, s));
  zdt_mark(ws, "output", s);
  return FDR_OK;
}

static bool fft_len_ok(long long N) {
  int radix[kMaxStages], nst;
  if (N <= kMaxCtaElems) return plan_radices(N, radix, &nst);
  for (long long a = 2; a <= kMaxCtaElems; ++a) {
    if (N % a) continue;
    long long b = N / a;
    if (b > kMaxCtaElems) continue;
    if (plan_radices(a, radix, &nst) && plan_radices(b, radix, &nst)) return true;
  }
  return false;
}

static void release(fdr_zdt* ws) {
  if (!ws) return;
  cudaFree(ws->F);
  cudaFree(ws->Y);
  cudaFree(ws->V);
  cudaFree(ws->rscratch);
  zdt_fused_release(ws);
  for (auto e : ws->events) cudaEventDestroy(e);
  delete ws;
}

}  // namespace fdr

using namespace fdr;

extern "C" {

int fdr_zdt_create(fdr_zdt** out, const float* spectrogram, int64_t Nf, int64_t Nt, float r0,
                   float dr, int64_t Nr, const int64_t* factors, int nfactors, uint32_t flags,
                   fdr_stream_t stream) {
  FDR_CHECK_ARG(out != nullptr, "ZDTWorkspace: output handle pointer is NULL");
  *out = nullptr;
  FDR_CHECK_ARG(Nf >= 1 && Nt >= 1 && Nr >= 1, "ZDTWorkspace: bad sizes Nf=%lld Nt=%lld Nr=%lld",
                (long long)Nf, (long long)Nt, (long long)Nr);
  FDR_CHECK_ARG(nfactors >= 0 && nfactors <= 8, "ZDTWorkspace: at most 8 factors");
  int64_t Nl = fdr_calc_nl(Nt, Nr, factors, nfactors);
  FDR_CHECK_ARG(Nl > 0, "ZDTWorkspace: invalid factors");
  if (!fft_len_ok(Nf)) {
    set_error(FDR_ERR_UNSUPPORTED_SIZE, "ZDTWorkspace: Nf=%lld has a prime factor > %d or "
              "cannot be split into two factors <= %d", (long long)Nf, kMaxRadixPrime, kMaxCtaElems);
    return FDR_ERR_UNSUPPORTED_SIZE;
  }
  if (Nl > kMaxCtaElems || !fft_len_ok(Nl)) {
    set_error(FDR_ERR_UNSUPPORTED_SIZE, "ZDTWorkspace: Nl=%lld unsupported (max %d, prime "
              "factors <= %d); use fewer rates per batch", (long long)Nl, kMaxCtaElems, kMaxRadixPrime);
    return FDR_ERR_UNSUPPORTED_SIZE;
  }
  cudaStream_t s = (cudaStream_t)stream;
  fdr_zdt* ws = new fdr_zdt();
  ws->Nf = Nf; ws->Nt = Nt; ws->Nr = Nr; ws->Nl = Nl; ws->K = Nf / 2 + 1;
  ws->r0 = r0; ws->dr = dr; ws->flags = flags;
  if (factors && nfactors > 0) ws->factors.assign(factors, factors + nfactors);
  else ws->factors = {2, 3, 5};
  cudaGetDevice(&ws->device);
  const int64_t K = ws->K;
  // Real-FFT scratch: enough pairs for the larger of Nt and Nr, capped at ~256 MiB.
  const int64_t per = real_fft_scratch_per_pair(Nf);
  int64_t pairs = cdiv(std::max(Nt, Nr), 2);
  const int64_t cap = std::max<int64_t>(1, (int64_t(256) << 20) / (int64_t)(per * sizeof(float2)));
  ws->rscratch_pairs = std::min(pairs, cap);
  auto fail = [&](cudaError_t e, const char* what) {
    int st = cuda_status(e, what);
    release(ws);
    return st;
  };
  cudaError_t e;
  if ((e = cudaMalloc(&ws->F, sizeof(float2) * K * Nt)) != cudaSuccess) return fail(e, "cudaMalloc(F)");
  ws->bytes = (int64_t)sizeof(float2) * K * Nt;
  (void)per;
  int st = FDR_OK;
  if (!(flags & FDR_ZDT_STAGED_ONLY) && zdt_fused_eligible(Nf, Nt, Nr)) {
    st = zdt_fused_setup(ws);
  } else {
    st = zdt_ensure_staged(ws, s);  // allocates Y, V, scratch and computes V (computeV!)
  }
  if (st != FDR_OK) { release(ws); return st; }
  if (spectrogram) st = fdr_zdt_input(ws, spectrogram, stream);
  if (st == FDR_OK) {
    e = s ? cudaStreamSynchronize(s) : cudaDeviceSynchronize();
    if (e != cudaSuccess) st = cuda_status(e, "ZDTWorkspace synchronize");
  }
  if (st != FDR_OK) { release(ws); return st; }
  *out = ws;
  return FDR_OK;
}

int fdr_zdt_destroy(fdr_zdt* ws) {
  if (ws) {
    cudaDeviceSynchronize();
    release(ws);
  }
  return FDR_OK;
}

int fdr_zdt_get_info(const fdr_zdt* ws, fdr_zdt_info* info) {
  FDR_CHECK_ARG(ws && info, "fdr_zdt_get_info: NULL argument");
  memset(info, 0, sizeof(*info));
  info->Nf = ws->Nf; info->Nt = ws->Nt; info->Nr = ws->Nr; info->Nl = ws->Nl; info->K = ws->K;
  info->r0 = ws->r0; info->dr = ws->dr; info->flags = ws->flags; info->fused = ws->fused ? 1 : 0;
  info->bytes = ws->bytes;
  info->nfactors = (int32_t)std::min<size_t>(8, ws->factors.size());
  for (int i = 0; i < info->nfactors; ++i) info->factors[i] = ws->factors[i];
  return FDR_OK;
}

int fdr_zdt_fused_split(int64_t Nf, int64_t Nt, int64_t Nr, uint32_t flags, int64_t* P, int64_t* Q) {
  FDR_CHECK_ARG(P && Q, "fdr_zdt_fused_split: NULL argument");
  if ((flags & FDR_ZDT_STAGED_ONLY) || !zdt_fused_eligible(Nf, Nt, Nr)) {
    set_error(FDR_ERR_UNSUPPORTED_SIZE, "fdr_zdt_fused_split: Nf=%lld Nt=%lld Nr=%lld runs the staged kernels",
              (long long)Nf, (long long)Nt, (long long)Nr);
    return FDR_ERR_UNSUPPORTED_SIZE;
  }
  int pl = 0, ql = 0;
  fused_split_log2(Nf, Nt, &pl, &ql);
  *P = (int64_t)1 << pl;
  *Q = (int64_t)1 << ql;
  return FDR_OK;
}

int fdr_zdt_buffers(fdr_zdt* ws, void** F, void** Y, void** V) {
  FDR_CHECK_ARG(ws != nullptr, "fdr_zdt_buffers: NULL workspace");
  if (F) {
    // Callers may read F directly: make sure it reflects the last input!.
    FDR_TRY(zdt_ensure_F(ws, nullptr));
    FDR_CUDA(cudaDeviceSynchronize());
    *F = ws->F;
  }
  if (Y || V) {
    FDR_TRY(zdt_ensure_staged(ws, nullptr));
    FDR_CUDA(cudaDeviceSynchronize());
  }
  if (Y) *Y = ws->Y;
  if (V) *V = ws->V;
  return FDR_OK;
}

// The fused kernels read the spectrogram and write the FDR in 8-byte pairs of floats, so
// their pointers must be 8-byte aligned (cudaMalloc'd and CuArray storage, and its columns
// for even Nf, always are); any other pointer is rejected before a kernel is launched.
static int check_pair_aligned(const void* p, const char* what) {
  if ((reinterpret_cast<uintptr_t>(p) & 7) != 0) {
    set_error(FDR_ERR_INVALID_ARGUMENT, "%s: the fused path needs an 8-byte aligned device "
              "pointer (got %p)", what, p);
    return FDR_ERR_INVALID_ARGUMENT;
  }
  return FDR_OK;
}

int fdr_zdt_input(fdr_zdt* ws, const float* spectrogram, fdr_stream_t stream) {
  FDR_CHECK_ARG(ws != nullptr, "input!: NULL workspace");
  FDR_CHECK_ARG(spectrogram != nullptr, "input!: spectrogram is NULL");
  cudaStream_t s = (cudaStream_t)stream;
  if (ws->fused) {
    FDR_TRY(check_pair_aligned(spectrogram, "input!: spectrogram"));
    FDR_TRY(zdt_fused_input(ws, spectrogram, s));
    ws->A_valid = true;
    ws->F_valid = false;
    return FDR_OK;
  }
  return zdt_stage_input(ws, spectrogram, s);
}

int fdr_zdt_preprocess(fdr_zdt* ws, float r0, fdr_stream_t stream) {
  FDR_CHECK_ARG(ws != nullptr, "preprocess!: NULL workspace");
  return zdt_preprocess(ws, r0, (cudaStream_t)stream);
}

int fdr_zdt_convolve(fdr_zdt* ws, fdr_stream_t stream) {
  FDR_CHECK_ARG(ws != nullptr, "convolve!: NULL workspace");
  return zdt_convolve(ws, (cudaStream_t)stream);
}

int fdr_zdt_postprocess(fdr_zdt* ws, int window, const double* custom_window,
                        fdr_stream_t stream) {
  FDR_CHECK_ARG(ws != nullptr, "postprocess!: NULL workspace");
  return zdt_postprocess(ws, window, custom_window, (cudaStream_t)stream);
}

int fdr_zdt_output(fdr_zdt* ws, float* dest, fdr_stream_t stream) {
  FDR_CHECK_ARG(ws != nullptr, "output!: NULL workspace");
  return zdt_output(ws, dest, (cudaStream_t)stream);
}

static int zdt_execute(fdr_zdt* ws, const float* spectrogram, const float* r0s, int64_t nbatch,
                       float* const* dests, int window, const double* custom_window, double* acc,
                       fdr_stream_t stream) {
  FDR_CHECK_ARG(ws != nullptr, "zdtfdr!: NULL workspace");
  FDR_CHECK_ARG(nbatch >= 0, "zdtfdr!: negative batch count");
  FDR_CHECK_ARG(nbatch == 0 || dests != nullptr, "zdtfdr!: dests is NULL");
  if (window < 0 || window > 2) {
    set_error(FDR_ERR_UNSUPPORTED_WINDOW, "unsupported window type (%d)", window);
    return FDR_ERR_UNSUPPORTED_WINDOW;
  }
  FDR_CHECK_ARG(window != FDR_WINDOW_CUSTOM || custom_window != nullptr,
                "zdtfdr!: custom window values are NULL");
  for (int64_t b = 0; b < nbatch; ++b) FDR_CHECK_ARG(dests[b] != nullptr, "zdtfdr!: dests[%lld] is NULL", (long long)b);
  const bool use_fused = ws->fused && !(ws->flags & FDR_ZDT_STAGED_ONLY);
  if (use_fused)
    for (int64_t b = 0; b < nbatch; ++b) FDR_TRY(check_pair_aligned(dests[b], "zdtfdr!: dest"));
  if (ws->fused && spectrogram) FDR_TRY(check_pair_aligned(spectrogram, "zdtfdr!: spectrogram"));
  cudaStream_t s = (cudaStream_t)stream;
  zdt_mark(ws, "start", s);
  if (spectrogram) {
    FDR_TRY(fdr_zdt_input(ws, spectrogram, stream));
    zdt_mark(ws, "input", s);
  }
  for (int64_t b = 0; b < nbatch; ++b) {
    const float r0 = r0s ? r0s[b] : ws->r0;
    if (use_fused) {
      FDR_TRY(zdt_fused_run(ws, r0, dests[b], window, custom_window, acc ? acc + 2 * b * ws->Nr : nullptr, s));
    } else {
      FDR_TRY(zdt_staged_run(ws, r0, dests[b], window, custom_window, acc ? acc + 2 * b * ws->Nr : nullptr, s));
    }
  }
  return FDR_OK;
}

// zdtfdr! over 8-rate blocks of the workspace's rate grid in one pass (fused path only).
static int zdt_execute_blocks(fdr_zdt* ws, const float* spectrogram, const int32_t* blocks,
                              int64_t nblocks, float* dest, int window, const double* custom_window,
                              double* acc, cudaStream_t s) {
  FDR_CHECK_ARG(ws != nullptr && blocks != nullptr && dest != nullptr, "zdtfdr blocks: NULL argument");
  FDR_CHECK_ARG(nblocks >= 1, "zdtfdr blocks: need at least one block");
  if (window < 0 || window > 2) {
    set_error(FDR_ERR_UNSUPPORTED_WINDOW, "unsupported window type (%d)", window);
    return FDR_ERR_UNSUPPORTED_WINDOW;
  }
  FDR_CHECK_ARG(window != FDR_WINDOW_CUSTOM || custom_window != nullptr,
                "zdtfdr blocks: custom window values are NULL");
  if (!ws->fused || (ws->flags & FDR_ZDT_STAGED_ONLY)) {
    set_error(FDR_ERR_UNSUPPORTED_SIZE, "zdtfdr blocks: needs the fused path (power-of-two Nf, Nt <= 64)");
    return FDR_ERR_UNSUPPORTED_SIZE;
  }
  for (int64_t i = 0; i < nblocks; ++i)
    FDR_CHECK_ARG(blocks[i] >= 0 && 8LL * (blocks[i] + 1) <= ws->Nr,
                  "zdtfdr blocks: block %lld = %d outside the workspace's %lld rates", (long long)i,
                  (int)blocks[i], (long long)ws->Nr);
  FDR_CHECK_ARG(4 * nblocks <= ws->W_pairs, "zdtfdr blocks: more than Nr/8 blocks");
  FDR_TRY(check_pair_aligned(dest, "zdtfdr blocks: dest"));
  if (spectrogram) FDR_TRY(check_pair_aligned(spectrogram, "zdtfdr blocks: spectrogram"));
  // the kernels take the rate index of each block's first rate
  std::vector<int> base((size_t)nblocks);
  for (int64_t i = 0; i < nblocks; ++i) base[(size_t)i] = 8 * (int)blocks[i];
  int* d_blk = nullptr;
  FDR_TRY(scratch_alloc((void**)&d_blk, sizeof(int) * nblocks, s));
  int st = upload_words(d_blk, base.data(), sizeof(int) * nblocks, s);
  zdt_mark(ws, "start", s);
  if (st == FDR_OK && spectrogram) {
    st = fdr_zdt_input(ws, spectrogram, s);
    zdt_mark(ws, "input", s);
  }
  if (st == FDR_OK) st = zdt_fused_run_blocks(ws, d_blk, nblocks, dest, window, custom_window, acc, s);
  scratch_free(d_blk, s);
  return st;
}

static void clear_events(fdr_zdt* ws) {
  for (auto e : ws->events) cudaEventDestroy(e);
  ws->events.clear();
  ws->ev_names.clear();
}

int fdr_zdt_execute(fdr_zdt* ws, const float* spectrogram, const float* r0s, int64_t nbatch,
                    float* const* dests, int window, const double* custom_window,
                    fdr_stream_t stream) {
  return zdt_execute(ws, spectrogram, r0s, nbatch, dests, window, custom_window, nullptr, stream);
}

int fdr_zdtfdr_protohits(fdr_zdt* ws, const float* spectrogram, const float* r0s, int64_t nbatch,
                         float* const* dests, int window, const double* custom_window,
                         double threshold, int snr, int64_t* hits, int64_t capacity,
                         int64_t* count, double* threshold_used, fdr_stream_t stream) {
  FDR_CHECK_ARG(ws != nullptr && count != nullptr, "zdtfdr_protohits: NULL argument");
  FDR_CHECK_ARG(nbatch >= 1, "zdtfdr_protohits: need at least one dest");
  FDR_CHECK_ARG(capacity >= 0 && (capacity == 0 || hits != nullptr), "zdtfdr_protohits: bad hit buffer");
  FDR_CHECK_ARG(snr == 0 || snr == FDR_SNR_F64 || snr == FDR_SNR_F32,
                "zdtfdr_protohits: snr must be 0, FDR_SNR_F64 or FDR_SNR_F32 (got %d)", snr);
  *count = 0;
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t ncols = nbatch * ws->Nr;
  const bool fast = (ws->flags & FDR_ZDT_FAST_STATS) != 0;
  double* acc = nullptr;  // [2*ncols moments (fast statistics)], then m, s, threshold
  if (snr) {
    FDR_TRY(scratch_alloc((void**)&acc, sizeof(double) * ((fast ? 2 * ncols : 0) + 3), s));
    if (fast) FDR_CUDA(cudaMemsetAsync(acc, 0, sizeof(double) * 2 * ncols, s));
  }
  int st = zdt_execute(ws, spectrogram, r0s, nbatch, dests, window, custom_window,
                       fast ? acc : nullptr, stream);
  double* d_ms = acc ? acc + (fast ? 2 * ncols : 0) : nullptr;
  void** d_mats = nullptr;
  if (st == FDR_OK) st = upload_ptrs((const void* const*)dests, nbatch, &d_mats, s);
  if (st == FDR_OK && snr && !fast) {
    st = snr_protohits_run((const float* const*)d_mats, nbatch, ws->Nf, ws->Nr, d_ms, snr, threshold,
                           hits, capacity, count, threshold_used, s);
  } else {
    if (st == FDR_OK && snr) {
      st = stats_finalize_launch(acc, ncols, ws->Nf, d_ms, s);
      if (st == FDR_OK) st = threshold_launch(d_ms, snr, threshold, d_ms + 2, s);
    }
    if (st == FDR_OK)
      st = hits_run((const float* const*)d_mats, nbatch, ws->Nf, ws->Nr, threshold,
                    snr ? d_ms + 2 : nullptr, hits, capacity, count, threshold_used, s);
  }
  scratch_free(d_mats, s);
  scratch_free(acc, s);
  return st;
}

int fdr_zdt_execute_blocks(fdr_zdt* ws, const float* spectrogram, const int32_t* blocks,
                           int64_t nblocks, float* dest, int window, const double* custom_window,
                           fdr_stream_t stream) {
  return zdt_execute_blocks(ws, spectrogram, blocks, nblocks, dest, window, custom_window, nullptr,
                            (cudaStream_t)stream);
}

int fdr_zdtfdr_blocks_protohits(fdr_zdt* ws, const float* spectrogram, const int32_t* blocks,
                                int64_t nblocks, float* dest, int window, const double* custom_window,
                                double threshold, int snr, int64_t* hits, int64_t capacity,
                                int64_t* count, double* threshold_used, fdr_stream_t stream) {
  FDR_CHECK_ARG(ws != nullptr && count != nullptr, "zdtfdr_blocks_protohits: NULL argument");
  FDR_CHECK_ARG(nblocks >= 1, "zdtfdr_blocks_protohits: need at least one block");
  FDR_CHECK_ARG(capacity >= 0 && (capacity == 0 || hits != nullptr), "zdtfdr_blocks_protohits: bad hit buffer");
  FDR_CHECK_ARG(snr == 0 || snr == FDR_SNR_F64 || snr == FDR_SNR_F32,
                "zdtfdr_blocks_protohits: snr must be 0, FDR_SNR_F64 or FDR_SNR_F32 (got %d)", snr);
  *count = 0;
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t ncols = 8 * nblocks;
  const bool fast = (ws->flags & FDR_ZDT_FAST_STATS) != 0;
  double* acc = nullptr;  // [2*ncols moments (fast statistics)], then m, s, threshold
  if (snr) {
    FDR_TRY(scratch_alloc((void**)&acc, sizeof(double) * ((fast ? 2 * ncols : 0) + 3), s));
    if (fast) FDR_CUDA(cudaMemsetAsync(acc, 0, sizeof(double) * 2 * ncols, s));
  }
  int st = zdt_execute_blocks(ws, spectrogram, blocks, nblocks, dest, window, custom_window,
                              fast ? acc : nullptr, s);
  double* d_ms = acc ? acc + (fast ? 2 * ncols : 0) : nullptr;
  void** d_mats = nullptr;
  float* const dl[1] = {dest};
  if (st == FDR_OK) st = upload_ptrs((const void* const*)dl, 1, &d_mats, s);
  if (st == FDR_OK && snr && !fast) {
    st = snr_protohits_run((const float* const*)d_mats, 1, ws->Nf, ncols, d_ms, snr, threshold, hits,
                           capacity, count, threshold_used, s);
  } else {
    if (st == FDR_OK && snr) {
      st = stats_finalize_launch(acc, ncols, ws->Nf, d_ms, s);
      if (st == FDR_OK) st = threshold_launch(d_ms, snr, threshold, d_ms + 2, s);
    }
    if (st == FDR_OK)
      st = hits_run((const float* const*)d_mats, 1, ws->Nf, ncols, threshold,
                    snr ? d_ms + 2 : nullptr, hits, capacity, count, threshold_used, s);
  }
  scratch_free(d_mats, s);
  scratch_free(acc, s);
  return st;
}

int fdr_zdt_set_timing(fdr_zdt* ws, int enable) {
  FDR_CHECK_ARG(ws != nullptr, "NULL workspace");
  ws->timing = enable != 0;
  clear_events(ws);
  return FDR_OK;
}

int fdr_zdt_stage_times(fdr_zdt* ws, float* times_ms, int max_stages, int* nstages,
                        const char** stage_names) {
  FDR_CHECK_ARG(ws != nullptr && nstages != nullptr, "NULL argument");
  *nstages = 0;
  if (ws->events.size() < 2) { clear_events(ws); return FDR_OK; }
  FDR_CUDA(cudaEventSynchronize(ws->events.back()));
  // Sum, per stage name, the time between each stage mark and the mark before it within
  // the same call (a call starts at a "start" mark), over every call recorded since the
  // last query.
  std::vector<const char*> names;
  std::vector<float> sums;
  for (size_t i = 1; i < ws->events.size(); ++i) {
    if (strcmp(ws->ev_names[i], "start") == 0) continue;
    float ms = 0.f;
    FDR_CUDA(cudaEventElapsedTime(&ms, ws->events[i - 1], ws->events[i]));
    size_t j = 0;
    while (j < names.size() && strcmp(names[j], ws->ev_names[i]) != 0) ++j;
    if (j == names.size()) { names.push_back(ws->ev_names[i]); sums.push_back(0.f); }
    sums[j] += ms;
  }
  int n = 0;
  for (; n < (int)names.size() && n < max_stages; ++n) {
    if (times_ms) times_ms[n] = sums[n];
    if (stage_names) stage_names[n] = names[n];
  }
  *nstages = n;
  clear_events(ws);
  return FDR_OK;
}

}  // extern "C"
