// Taylor-tree integer FDR (fdr_taylor_tree).
//
// The reference computes integer-shift FDRs by brute force (intfdr, intfdr.jl:34-45) and
// notes that "the Taylor Tree algorithm" would remove the redundant additions but is not
// included (the reference's README.md:88-92).  This is that algorithm for Nt = 2^m time steps: FDR column d
// (total drift d channels over the Nt-1 step intervals, rate d/(Nt-1) channels per step,
// |d| <= Nt-1) is the sum of the spectrogram along a tree path built recursively: a path of
// drift d over 2L steps is the path of drift floor(d/2) over the first L steps followed by
// the path of drift floor(d/2) over the last L steps started ceil(d/2) channels further
// (towards lower channels for negative d).  Over all drifts this costs m*Nt additions per
// channel instead of Nt*(2Nt-1).  Paths with d = 0 and |d| = Nt-1 are the straight lines of
// intfdr at rates 0 and +-1; other paths stay within a channel or two of round(d*t/(Nt-1))
// and are given exactly by taylor_shifts in the host code.  Channels wrap around modulo Nf
// like intshift! (intfdr.jl:7-26): column d at channel n sums s[(n + p_d(t)) mod Nf, t].
//
// One CTA per tile of C channels: the tile plus Nt-1 halo channels either side, all Nt
// steps, are staged in shared memory once; the m stages run between two more buffers; the
// positive and the negative trees are formed one after the other from the staged input.
// Additions are float32, in a fixed order, so the result is deterministic.
#include "fdr_internal.cuh"

namespace fdr {

constexpr int kTaylorThreads = 256;

// Tile shape for NT steps: C channels per CTA, W = C + 2*(NT-1) staged channels, rows
// stored with PAD spare floats either side (PAD >= the largest shift, NT/2) so that the
// shifted reads need no bounds test (the spare floats only feed outputs that are dropped).
template <int NT>
struct TaylorShape {
  static constexpr int C = NT <= 32 ? 256 : 64;
  static constexpr int H = NT - 1;
  static constexpr int W = C + 2 * H;
  static constexpr int PAD = NT / 2;
  static constexpr int WS = W + 2 * PAD;  // row stride
  static constexpr size_t SMEM = sizeof(float) * 3 * NT * WS;
  static_assert(W <= 2 * kTaylorThreads, "each thread stages at most two channels");
  static_assert(SMEM <= 227 * 1024, "shared memory per CTA");
};

// One stage of the tree: from blocks of length L (rows r = block*L + drift) in src to
// blocks of length 2L in dst; thread j handles channels j and j + kTaylorThreads.
template <int SIGN, int NT, int L>
__device__ __forceinline__ void taylor_stage(const float* __restrict__ src, float* __restrict__ dst) {
  using S = TaylorShape<NT>;
  const int w0 = threadIdx.x, w1 = threadIdx.x + kTaylorThreads;
  const bool h1 = w1 < S::W;
#pragma unroll
  for (int r = 0; r < NT; ++r) {
    const int B = r / (2 * L), d = r % (2 * L);  // compile-time after unrolling
    const float* top = src + (2 * B * L + d / 2) * S::WS + S::PAD;
    const float* bot = src + ((2 * B + 1) * L + d / 2) * S::WS + S::PAD + SIGN * ((d + 1) / 2);
    float* o = dst + r * S::WS + S::PAD;
    if (w0 < S::W) o[w0] = top[w0] + bot[w0];
    if (h1) o[w1] = top[w1] + bot[w1];
  }
  __syncthreads();
}

// Runs the stages L = 1, 2, ..., NT/2 from src through the buffers a and b (src is left
// untouched); returns the buffer holding the final rows (row d = drift |d|).
template <int SIGN, int NT, int L>
__device__ __forceinline__ float* taylor_stages(const float* src, float* a, float* b) {
  if constexpr (L >= NT) {
    return const_cast<float*>(src);
  } else {
    taylor_stage<SIGN, NT, L>(src, a);
    return taylor_stages<SIGN, NT, 2 * L>(a, b, a);
  }
}

template <int NT>
__global__ void __launch_bounds__(kTaylorThreads)
taylor_kernel(const float* __restrict__ spec, long long Nf, int dmin, int dmax,
              float* __restrict__ fdr) {
  using S = TaylorShape<NT>;
  extern __shared__ float sm[];
  float* x = sm;                 // staged input, NT rows
  float* a = sm + NT * S::WS;
  float* b = sm + 2 * NT * S::WS;
  const long long n0 = (long long)blockIdx.x * S::C;
  // every thread stages at most two channels, the same for every step; their wrapped
  // indices are formed once, then the loads of 8 steps are issued together
  const int w0 = threadIdx.x, w1 = threadIdx.x + kTaylorThreads;
  const bool h0 = w0 < S::W, h1 = w1 < S::W;
  long long c0 = n0 - S::H + w0, c1 = n0 - S::H + w1;
  while (c0 < 0) c0 += Nf;  // a few steps at most: n0 - H + w lies within W of [0, Nf)
  while (c0 >= Nf) c0 -= Nf;
  while (c1 < 0) c1 += Nf;
  while (c1 >= Nf) c1 -= Nf;
#pragma unroll
  for (int t0 = 0; t0 < NT; t0 += 8) {
    float v0[8], v1[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const long long row = (long long)(t0 + u) * Nf;
      const bool in = t0 + u < NT;
      v0[u] = (in && h0) ? __ldg(spec + row + c0) : 0.f;
      v1[u] = (in && h1) ? __ldg(spec + row + c1) : 0.f;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      if (t0 + u < NT) {
        if (h0) x[(t0 + u) * S::WS + S::PAD + w0] = v0[u];
        if (h1) x[(t0 + u) * S::WS + S::PAD + w1] = v1[u];
      }
    }
  }
  __syncthreads();
  for (int pass = 0; pass < 2; ++pass) {
    const int sgn = pass == 0 ? +1 : -1;
    if ((sgn > 0 && dmax < 0) || (sgn < 0 && dmin > 0)) continue;
    const float* res = sgn > 0 ? taylor_stages<+1, NT, 1>(x, a, b) : taylor_stages<-1, NT, 1>(x, a, b);
    // column d of the result (row |d| of the final stage), channels H .. H+C-1 of the tile
    const int lo = sgn > 0 ? max(dmin, 0) : dmin;
    const int hi = sgn > 0 ? dmax : min(dmax, -1);
    for (int d = lo; d <= hi; ++d) {
      const int r = d >= 0 ? d : -d;
      float* col = fdr + (long long)(d - dmin) * Nf;
      for (int w = threadIdx.x; w < S::C; w += kTaylorThreads) {
        const long long n = n0 + w;
        if (n < Nf) col[n] = res[r * S::WS + S::PAD + S::H + w];
      }
    }
    __syncthreads();  // a and b are free for the other sign
  }
}

}  // namespace fdr

using namespace fdr;

extern "C" {

int fdr_taylor_tree(const float* spectrogram, int64_t Nf, int64_t Nt, int dmin, int dmax, float* fdr,
                    fdr_stream_t stream) {
  FDR_CHECK_ARG(spectrogram != nullptr && fdr != nullptr, "taylor_tree: NULL argument");
  FDR_CHECK_ARG(Nt >= 2 && Nt <= 64 && (Nt & (Nt - 1)) == 0,
                "taylor_tree: Nt must be a power of two in [2, 64] (got %lld)", (long long)Nt);
  FDR_CHECK_ARG(Nf >= 1, "taylor_tree: Nf must be positive");
  FDR_CHECK_ARG(dmin <= dmax && dmin >= -(Nt - 1) && dmax <= Nt - 1,
                "taylor_tree: drifts must satisfy -(Nt-1) <= dmin <= dmax <= Nt-1");
  static bool attr_done[64] = {false};
  int dev = 0;
  FDR_CUDA(cudaGetDevice(&dev));
  if (dev < 64 && !attr_done[dev]) {
#define FDR_TAYLOR_ATTR(NT)                                                                    \
    FDR_CUDA(cudaFuncSetAttribute(taylor_kernel<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                  (int)TaylorShape<NT>::SMEM));
    FDR_TAYLOR_ATTR(2) FDR_TAYLOR_ATTR(4) FDR_TAYLOR_ATTR(8) FDR_TAYLOR_ATTR(16) FDR_TAYLOR_ATTR(32)
    FDR_TAYLOR_ATTR(64)
#undef FDR_TAYLOR_ATTR
    attr_done[dev] = true;
  }
  cudaStream_t s = (cudaStream_t)stream;
  switch (Nt) {
#define FDR_TAYLOR_CASE(NT)                                                                    \
    case NT: {                                                                                 \
      const long long grid = cdiv(Nf, TaylorShape<NT>::C);                                     \
      FDR_CHECK_ARG(grid <= 0x7fffffffLL, "taylor_tree: Nf too large");                       \
      taylor_kernel<NT><<<(unsigned)grid, kTaylorThreads, TaylorShape<NT>::SMEM, s>>>(         \
          spectrogram, Nf, dmin, dmax, fdr);                                                   \
      break;                                                                                   \
    }
    FDR_TAYLOR_CASE(2) FDR_TAYLOR_CASE(4) FDR_TAYLOR_CASE(8) FDR_TAYLOR_CASE(16) FDR_TAYLOR_CASE(32)
    FDR_TAYLOR_CASE(64)
#undef FDR_TAYLOR_CASE
  }
  FDR_LAUNCH_CHECK("taylor_kernel");
  return FDR_OK;
}

}  // extern "C"
