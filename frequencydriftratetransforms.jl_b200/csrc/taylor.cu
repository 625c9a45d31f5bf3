// Taylor-tree integer FDR (fdr_taylor_tree).
//
// The reference computes integer-shift FDRs by brute force (intfdr, intfdr.jl:34-45) and
// notes that "the Taylor Tree algorithm" would remove the redundant additions but is not
// included (README.md:88-92).  This is that algorithm for Nt = 2^m time steps: FDR column d
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
// steps, are staged in shared memory; the m stages run in place between two buffers; the
// positive and the negative trees are formed one after the other from the same staged
// input.  Additions are float32, in a fixed order, so the result is deterministic.
#include "fdr_internal.cuh"

namespace fdr {

constexpr int kTaylorThreads = 256;

// buffers: 2 x Nt rows of W floats; row r = block*L + drift at the stage with block length L
template <int SIGN>
__device__ void taylor_tree_tile(float* a, float* b, int Nt, int W, float** out_buf) {
  for (int L = 1; L < Nt; L *= 2) {
    const int nout = Nt * W;
    for (int e = threadIdx.x; e < nout; e += blockDim.x) {
      const int r = e / W, w = e - r * W;
      const int B = r / (2 * L), d = r - B * 2 * L;
      const int top = 2 * B * L + d / 2, bot = (2 * B + 1) * L + d / 2;
      const int wb = w + SIGN * ((d + 1) / 2);
      const float vb = (wb >= 0 && wb < W) ? a[bot * W + wb] : 0.f;
      b[r * W + w] = a[top * W + w] + vb;
    }
    __syncthreads();
    float* t = a;
    a = b;
    b = t;
  }
  *out_buf = a;
}

__global__ void __launch_bounds__(kTaylorThreads)
taylor_kernel(const float* __restrict__ spec, long long Nf, int Nt, int C, int dmin, int dmax,
              float* __restrict__ fdr) {
  extern __shared__ float sm[];
  const int H = Nt - 1;       // halo channels on each side
  const int W = C + 2 * H;
  float* a = sm;
  float* b = sm + Nt * W;
  const long long n0 = (long long)blockIdx.x * C;
  const int ncols = dmax - dmin + 1;
  for (int pass = 0; pass < 2; ++pass) {
    const int sgn = pass == 0 ? +1 : -1;
    if ((sgn > 0 && dmax < 0) || (sgn < 0 && dmin > 0)) continue;
    __syncthreads();  // the buffers are free
    for (int e = threadIdx.x; e < Nt * W; e += blockDim.x) {
      const int t = e / W, w = e - t * W;
      long long n = (n0 - H + w) % Nf;
      if (n < 0) n += Nf;
      a[t * W + w] = __ldg(spec + (long long)t * Nf + n);
    }
    __syncthreads();
    float* res = nullptr;
    if (sgn > 0) taylor_tree_tile<+1>(a, b, Nt, W, &res);
    else taylor_tree_tile<-1>(a, b, Nt, W, &res);
    // column d of the result (row |d| of the final stage), channels H .. H+C-1 of the tile
    const int lo = sgn > 0 ? max(dmin, 0) : dmin;
    const int hi = sgn > 0 ? dmax : min(dmax, -1);
    for (int d = lo; d <= hi; ++d) {
      const int r = d >= 0 ? d : -d;
      float* col = fdr + (long long)(d - dmin) * Nf;
      for (int w = threadIdx.x; w < C; w += blockDim.x) {
        const long long n = n0 + w;
        if (n < Nf) col[n] = res[r * W + H + w];
      }
    }
    (void)ncols;
  }
}

static int taylor_tile(int Nt) { return Nt <= 32 ? 256 : 128; }

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
  const int C = taylor_tile((int)Nt);
  const int W = C + 2 * ((int)Nt - 1);
  const size_t sm = sizeof(float) * 2 * (size_t)Nt * W;
  static bool attr_done[64] = {false};
  int dev = 0;
  FDR_CUDA(cudaGetDevice(&dev));
  if (dev < 64 && !attr_done[dev]) {
    FDR_CUDA(cudaFuncSetAttribute(taylor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
    attr_done[dev] = true;
  }
  const long long grid = cdiv(Nf, C);
  FDR_CHECK_ARG(grid <= 0x7fffffffLL, "taylor_tree: Nf too large");
  taylor_kernel<<<(unsigned)grid, kTaylorThreads, sm, (cudaStream_t)stream>>>(spectrogram, Nf, (int)Nt, C,
                                                                           dmin, dmax, fdr);
  FDR_LAUNCH_CHECK("taylor_kernel");
  return FDR_OK;
}

}  // extern "C"
