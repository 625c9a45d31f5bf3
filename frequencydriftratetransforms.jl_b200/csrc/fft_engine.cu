// Generic batched FFT engine: see fft_engine.cuh.
#include <math.h>
#include <string.h>

#include <map>
#include <mutex>

#include "fft_device.cuh"
#include "fft_engine.cuh"

namespace fdr {

// ------------------------------------------------------------------------------------
// Planning
// ------------------------------------------------------------------------------------
bool plan_radices(long long L, int* radix, int* nst) {
  int n = 0;
  long long m = L;
  while (m % 8 == 0 && n < kMaxStages) { radix[n++] = 8; m /= 8; }
  while (m % 4 == 0 && n < kMaxStages) { radix[n++] = 4; m /= 4; }
  while (m % 2 == 0 && n < kMaxStages) { radix[n++] = 2; m /= 2; }
  for (int p = 3; p <= kMaxRadixPrime && m > 1; p += 2) {
    while (m % p == 0 && n < kMaxStages) { radix[n++] = p; m /= p; }
  }
  *nst = n;
  return m == 1;
}

int get_roots(long long L, const float2** roots) {
  static std::mutex mu;
  static std::map<std::pair<int, long long>, float2*> cache;
  int dev = 0;
  FDR_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  auto key = std::make_pair(dev, L);
  auto it = cache.find(key);
  if (it != cache.end()) { *roots = it->second; return FDR_OK; }
  std::vector<float2> h((size_t)L);
  for (long long m = 0; m < L; ++m) {
    // exp(-2*pi*i*m/L) with the angle reduced to the first half-turn pair in double
    double a = -2.0 * (double)m / (double)L;  // half-turns
    double c = cos(M_PI * a), sn = sin(M_PI * a);
    h[(size_t)m] = make_float2((float)c, (float)sn);
  }
  float2* d = nullptr;
  FDR_CUDA(cudaMalloc(&d, sizeof(float2) * (size_t)L));
  FDR_CUDA(cudaMemcpy(d, h.data(), sizeof(float2) * (size_t)L, cudaMemcpyHostToDevice));
  cache[key] = d;
  *roots = d;
  return FDR_OK;
}

// ------------------------------------------------------------------------------------
// Small DFT kernels on register arrays.  sign: -1 forward, +1 backward.
// ------------------------------------------------------------------------------------
__device__ __forceinline__ float2 root_at(const float2* roots, int m, int sign) {
  float2 w = __ldg(roots + m);
  return sign > 0 ? cconj(w) : w;
}

// One Stockham stage of radix R over bpc transforms of length L held in shared memory.
template <int R>
__device__ __forceinline__ void stage_fixed(const float2* __restrict__ A, float2* __restrict__ B,
                                            int L, int bpc, int Ns, int sign,
                                            const float2* roots) {
  const int nbf = L / R;
  const int total = nbf * bpc;
  const int stride = L / (Ns * R);
  for (int j = threadIdx.x; j < total; j += blockDim.x) {
    const int i = j / nbf;
    const int jj = j - i * nbf;
    const int k = jj % Ns;
    const float2* a = A + (size_t)i * L;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = a[jj + r * nbf];
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], root_at(roots, r * k * stride, sign));
    }
    Dft<R>::run(v, sign);
    const int base = (jj / Ns) * Ns * R + k;
    float2* b = B + (size_t)i * L;
#pragma unroll
    for (int r = 0; r < R; ++r) b[base + r * Ns] = v[r];
  }
}

// Direct DFT stage for any radix R <= kMaxRadixPrime (one output per thread iteration).
__device__ void stage_generic(const float2* __restrict__ A, float2* __restrict__ B, int L,
                              int bpc, int Ns, int R, int sign, const float2* roots) {
  const int nbf = L / R;
  const int total = nbf * bpc * R;
  const int stride = L / (Ns * R);
  const int rstep = L / R;  // roots[q*rstep] = exp(-2*pi*i*q/R)
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int m = e % R;
    const int j = e / R;
    const int i = j / nbf;
    const int jj = j - i * nbf;
    const int k = jj % Ns;
    const float2* a = A + (size_t)i * L;
    float2 acc = make_float2(0.f, 0.f);
    for (int r = 0; r < R; ++r) {
      float2 v = a[jj + r * nbf];
      if (Ns > 1 && r > 0) v = cmul(v, root_at(roots, r * k * stride, sign));
      int q = (r * m) % R;
      acc = cadd(acc, cmul(v, root_at(roots, q * rstep, sign)));
    }
    const int base = (jj / Ns) * Ns * R + k;
    B[(size_t)i * L + base + m * Ns] = acc;
  }
}

__global__ void __launch_bounds__(256) fft_pass_kernel(PassDesc d) {
  extern __shared__ float2 sm[];
  const int L = d.L, bpc = d.bpc;
  const long long b1_0 = (long long)blockIdx.x * bpc;
  const int nb = (int)min((long long)bpc, d.nb1 - b1_0);
  const int total = L * bpc;
  for (long long b0 = blockIdx.y; b0 < d.nb0; b0 += gridDim.y) {
    float2* A = sm;
    float2* B = sm + (size_t)L * bpc;
    // load
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      int i, l;
      if (d.ld_b1_fast) { i = e % bpc; l = e / bpc; } else { l = e % L; i = e / L; }
      float2 v = make_float2(0.f, 0.f);
      if (i < nb) v = d.in[b0 * d.is0 + (b1_0 + i) * d.is1 + (long long)l * d.isl];
      A[(size_t)i * L + l] = v;
    }
    __syncthreads();
    int Ns = 1;
    for (int s = 0; s < d.nst; ++s) {
      const int R = d.radix[s];
      switch (R) {
        case 2: stage_fixed<2>(A, B, L, bpc, Ns, d.sign, d.roots); break;
        case 3: stage_fixed<3>(A, B, L, bpc, Ns, d.sign, d.roots); break;
        case 4: stage_fixed<4>(A, B, L, bpc, Ns, d.sign, d.roots); break;
        case 5: stage_fixed<5>(A, B, L, bpc, Ns, d.sign, d.roots); break;
        case 8: stage_fixed<8>(A, B, L, bpc, Ns, d.sign, d.roots); break;
        default: stage_generic(A, B, L, bpc, Ns, R, d.sign, d.roots); break;
      }
      __syncthreads();
      float2* t = A; A = B; B = t;
      Ns *= R;
    }
    // store
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      int i, l;
      if (d.st_b1_fast) { i = e % bpc; l = e / bpc; } else { l = e % L; i = e / L; }
      if (i >= nb) continue;
      float2 v = A[(size_t)i * L + l];
      const long long b1 = b1_0 + i;
      if (d.tw_n) {
        const long long b = d.tw_dim == 1 ? b1 : b0;
        const long long m = ((long long)l * b) % d.tw_n;
        double sn, cs;
        sincospi(2.0 * (double)m / (double)d.tw_n, &sn, &cs);
        v = cmul(v, make_float2((float)cs, (float)(d.sign * sn)));
      }
      if (d.mul) v = cmul(v, d.mul[b0 * d.ms0 + b1 * d.ms1 + (long long)l * d.msl]);
      v = cscale(v, d.scale);
      d.out[b0 * d.os0 + b1 * d.os1 + (long long)l * d.osl] = v;
    }
    __syncthreads();
  }
}

int launch_pass(PassDesc d, cudaStream_t s) {
  if (!plan_radices(d.L, d.radix, &d.nst)) {
    set_error(FDR_ERR_UNSUPPORTED_SIZE, "FFT length %d has a prime factor > %d", d.L,
              kMaxRadixPrime);
    return FDR_ERR_UNSUPPORTED_SIZE;
  }
  FDR_TRY(get_roots(d.L, &d.roots));
  static bool attr_set[64] = {false};
  int dev = 0;
  FDR_CUDA(cudaGetDevice(&dev));
  const size_t smem = sizeof(float2) * 2 * (size_t)d.L * d.bpc;
  if (dev < 64 && !attr_set[dev]) {
    FDR_CUDA(cudaFuncSetAttribute(fft_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(sizeof(float2) * 2 * kMaxCtaElems)));
    attr_set[dev] = true;
  }
  if (d.nb0 <= 0 || d.nb1 <= 0) return FDR_OK;
  dim3 grid((unsigned)cdiv(d.nb1, d.bpc), (unsigned)min(d.nb0, 65535LL));
  fft_pass_kernel<<<grid, 256, smem, s>>>(d);
  FDR_LAUNCH_CHECK("fft_pass_kernel");
  return FDR_OK;
}

static int pick_bpc(long long L, long long nb1) {
  long long b = kMaxCtaElems / L;
  if (b < 1) b = 1;
  long long p = 1;
  while (p * 2 <= b && p * 2 <= 64) p *= 2;
  if (p > nb1) {
    p = 1;
    while (p * 2 <= nb1) p *= 2;
  }
  return (int)p;
}

static PassDesc blank_pass() {
  PassDesc d;
  memset(&d, 0, sizeof(d));
  d.scale = 1.f;
  d.nb0 = 1;
  return d;
}

int fft_strided_inplace(float2* buf, long long L, long long sl, long long nb, long long sb,
                        int sign, float scale, const float2* mul, cudaStream_t s) {
  if (L > kMaxCtaElems) {
    set_error(FDR_ERR_UNSUPPORTED_SIZE, "strided FFT length %lld exceeds %d", L, kMaxCtaElems);
    return FDR_ERR_UNSUPPORTED_SIZE;
  }
  PassDesc d = blank_pass();
  d.in = buf; d.out = buf; d.mul = mul;
  d.L = (int)L;
  d.nb0 = 1; d.nb1 = nb;
  d.is1 = sb; d.isl = sl; d.os1 = sb; d.osl = sl; d.ms1 = sb; d.msl = sl;
  d.sign = sign; d.scale = scale;
  d.bpc = pick_bpc(L, nb);
  d.ld_b1_fast = d.st_b1_fast = (sb == 1) ? 1 : 0;
  return launch_pass(d, s);
}

static void split_len(long long N, long long* L1, long long* L2) {
  // N = L1 * L2 with both <= kMaxCtaElems, L2 (the contiguous inner length) near sqrt(N).
  long long best1 = 0, best2 = 0;
  for (long long a = 2; a <= kMaxCtaElems; ++a) {
    if (N % a) continue;
    long long b = N / a;
    if (b > kMaxCtaElems) continue;
    if (best1 == 0 || llabs(a - b) < llabs(best1 - best2)) { best1 = a; best2 = b; }
  }
  *L1 = best1;
  *L2 = best2;
}

int fft_contig(const float2* in, long long ldin, float2* out, long long ldout, long long N,
               long long ncol, int sign, float scale, float2* tmp, cudaStream_t s) {
  if (N <= kMaxCtaElems) {
    PassDesc d = blank_pass();
    d.in = in; d.out = out;
    d.L = (int)N;
    d.nb0 = 1; d.nb1 = ncol;
    d.is1 = ldin; d.isl = 1; d.os1 = ldout; d.osl = 1;
    d.sign = sign; d.scale = scale;
    d.bpc = pick_bpc(N, ncol);
    d.ld_b1_fast = d.st_b1_fast = 0;
    return launch_pass(d, s);
  }
  long long L1, L2;
  split_len(N, &L1, &L2);
  if (L1 == 0) {
    set_error(FDR_ERR_UNSUPPORTED_SIZE, "FFT length %lld cannot be split into two factors <= %d",
              N, kMaxCtaElems);
    return FDR_ERR_UNSUPPORTED_SIZE;
  }
  FDR_CHECK_ARG(tmp != nullptr, "four-step FFT needs scratch");
  // Pass 1: n = n2 + L2*n1; DFT over n1 (stride L2) for each n2; twiddle exp(sign*2pi i k1 n2/N)
  PassDesc d = blank_pass();
  d.in = in; d.out = tmp;
  d.L = (int)L1;
  d.nb0 = ncol; d.nb1 = L2;
  d.is0 = ldin; d.is1 = 1; d.isl = L2;
  d.os0 = N; d.os1 = 1; d.osl = L2;
  d.sign = sign; d.scale = 1.f;
  d.tw_n = N; d.tw_dim = 1;
  d.bpc = pick_bpc(L1, L2);
  d.ld_b1_fast = d.st_b1_fast = 1;
  FDR_TRY(launch_pass(d, s));
  // Pass 2: for each k1, DFT over n2 (contiguous) -> out[k1 + L1*k2]
  PassDesc e = blank_pass();
  e.in = tmp; e.out = out;
  e.L = (int)L2;
  e.nb0 = ncol; e.nb1 = L1;
  e.is0 = N; e.is1 = L2; e.isl = 1;
  e.os0 = ldout; e.os1 = 1; e.osl = L1;
  e.sign = sign; e.scale = scale;
  e.bpc = pick_bpc(L2, L1);
  e.ld_b1_fast = 0; e.st_b1_fast = 1;
  return launch_pass(e, s);
}

long long real_fft_scratch_per_pair(long long N) {
  return N <= kMaxCtaElems ? N : 2 * N;
}

// z[p][n] = in[n, 2p] + i*in[n, 2p+1]
__global__ void pack_real_pairs(const float* __restrict__ in, long long ldin, long long ncol,
                                long long N, long long p0, long long np, float2* __restrict__ z) {
  const long long total = N * np;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long p = e / N, n = e - p * N;
    const long long c0 = 2 * (p0 + p), c1 = c0 + 1;
    float a = in[n + c0 * ldin];
    float b = c1 < ncol ? in[n + c1 * ldin] : 0.f;
    z[e] = make_float2(a, b);
  }
}

// F[k, 2p] = (Z[k] + conj Z[-k]) / 2, F[k, 2p+1] = (Z[k] - conj Z[-k]) / (2i)
__global__ void unpack_r2c(const float2* __restrict__ Z, long long N, long long K, long long ncol,
                           long long p0, long long np, float2* __restrict__ F, long long ldF) {
  const long long total = K * np;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long p = e / K, k = e - p * K;
    const float2* z = Z + p * N;
    float2 a = z[k];
    float2 b = cconj(z[k == 0 ? 0 : N - k]);
    const long long c0 = 2 * (p0 + p), c1 = c0 + 1;
    F[k + c0 * ldF] = make_float2(0.5f * (a.x + b.x), 0.5f * (a.y + b.y));
    if (c1 < ncol) {
      // (a - b) / (2i) = -i (a - b) / 2
      float2 d = csub(a, b);
      F[k + c1 * ldF] = make_float2(0.5f * d.y, -0.5f * d.x);
    }
  }
}

// C[p][k] = S_a[k] + i S_b[k] for k <= N/2, conj(S_a[N-k]) + i conj(S_b[N-k]) above.
__global__ void pack_c2r(const float2* __restrict__ S, long long ldS, long long ncol, long long N,
                         long long K, long long p0, long long np, float2* __restrict__ C) {
  const long long total = N * np;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long p = e / N, k = e - p * N;
    const long long c0 = 2 * (p0 + p), c1 = c0 + 1;
    const bool upper = k >= K;
    const long long kk = upper ? N - k : k;
    float2 a = S[kk + c0 * ldS];
    float2 b = c1 < ncol ? S[kk + c1 * ldS] : make_float2(0.f, 0.f);
    const bool real_bin = (kk == 0) || ((N % 2 == 0) && kk == N / 2);
    if (real_bin) { a.y = 0.f; b.y = 0.f; }
    if (upper) { a = cconj(a); b = cconj(b); }
    C[e] = make_float2(a.x - b.y, a.y + b.x);  // a + i b
  }
}

__global__ void unpack_c2r(const float2* __restrict__ z, long long N, long long ncol, long long p0,
                           long long np, float* __restrict__ out, long long ldout) {
  const long long total = N * np;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long p = e / N, n = e - p * N;
    const long long c0 = 2 * (p0 + p), c1 = c0 + 1;
    float2 v = z[e];
    out[n + c0 * ldout] = v.x;
    if (c1 < ncol) out[n + c1 * ldout] = v.y;
  }
}

static unsigned grid_for(long long total) {
  long long b = cdiv(total, 256);
  long long cap = (long long)sm_count() * 32;
  return (unsigned)max(1LL, min(b, cap));
}

int rfft_columns(const float* in, long long ldin, long long ncol, long long N, float2* F,
                 long long ldF, float2* scratch, long long pairs_per_chunk, cudaStream_t s) {
  const long long K = N / 2 + 1;
  const long long npairs = cdiv(ncol, 2);
  const long long per = real_fft_scratch_per_pair(N);
  for (long long p0 = 0; p0 < npairs; p0 += pairs_per_chunk) {
    const long long np = min(pairs_per_chunk, npairs - p0);
    // packed pairs in z; the four-step's first pass runs in place on z, the second
    // writes zo
    float2* z = scratch;
    float2* zo = (N <= kMaxCtaElems) ? scratch : scratch + N * np;
    float2* tmp = z;
    (void)per;
    pack_real_pairs<<<grid_for(N * np), 256, 0, s>>>(in, ldin, ncol, N, p0, np, z);
    FDR_LAUNCH_CHECK("pack_real_pairs");
    FDR_TRY(fft_contig(z, N, zo, N, N, np, -1, 1.f, tmp, s));
    unpack_r2c<<<grid_for(K * np), 256, 0, s>>>(zo, N, K, ncol, p0, np, F, ldF);
    FDR_LAUNCH_CHECK("unpack_r2c");
  }
  return FDR_OK;
}

int irfft_columns(const float2* S, long long ldS, long long ncol, long long N, float* out,
                  long long ldout, float2* scratch, long long pairs_per_chunk, cudaStream_t s) {
  const long long K = N / 2 + 1;
  const long long npairs = cdiv(ncol, 2);
  for (long long p0 = 0; p0 < npairs; p0 += pairs_per_chunk) {
    const long long np = min(pairs_per_chunk, npairs - p0);
    float2* c = scratch;
    float2* co = (N <= kMaxCtaElems) ? scratch : scratch + N * np;
    float2* tmp = c;
    pack_c2r<<<grid_for(N * np), 256, 0, s>>>(S, ldS, ncol, N, K, p0, np, c);
    FDR_LAUNCH_CHECK("pack_c2r");
    FDR_TRY(fft_contig(c, N, co, N, N, np, +1, 1.f / (float)N, tmp, s));
    unpack_c2r<<<grid_for(N * np), 256, 0, s>>>(co, N, ncol, p0, np, out, ldout);
    FDR_LAUNCH_CHECK("unpack_c2r");
  }
  return FDR_OK;
}

}  // namespace fdr
