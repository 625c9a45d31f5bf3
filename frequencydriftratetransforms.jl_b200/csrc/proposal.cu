// Learned drift-rate window proposal: a small 1-D convolutional network that reads the
// 256-channel-summed power of a coarse channel (nbins x Nt) and predicts which of `nwin`
// drift-rate windows hold proto-hits, so that zdtfdr! runs only over those windows
// (rate batches through the r0 iterator, zdtfdr.jl:354).  The reference has no learned
// component; this is the training/serving extension of its batched-rate search
// (batchrates.jl:22-60).
//
// Network (all convolutions along the bin axis, zero padded to keep the length):
//   x [B][Nt][X] -> conv(Nt->C, K) ReLU -> conv(C->C, K) ReLU -> conv(C->C, K) ReLU
//                -> conv(C->nwin, 1) -> max over bins -> logits [B][nwin]
// Loss: mean binary cross-entropy with logits.  Optimiser: Adam on float32 master weights;
// the forward pass uses their float16 rounding ("FP16 weights").  Every reduction runs in a
// fixed order (per-block partial sums, then an ordered sum), so results are deterministic
// and a resumed training run matches an uninterrupted one bit for bit.
#include <cuda_fp16.h>
#include <math.h>
#include <string.h>

#include "fdr_internal.cuh"

namespace fdr {

constexpr int kConvTile = 256;  // bins per CTA

struct Layer {
  int cin, cout, k;
  int64_t woff, boff;  // offsets (floats) into the parameter vector
};

}  // namespace fdr

struct fdr_propose_net {
  int nbins, nt, width, ksize, nwin;
  fdr::Layer L[4];
  int64_t nparams = 0;
  float* params = nullptr;   // float32 master weights (w then b per layer)
  __half* wh = nullptr;      // float16 copy used by the forward pass
  float* m = nullptr;        // Adam moments
  float* v = nullptr;
  float* grad = nullptr;
  int64_t step = 0;
  uint64_t seed = 0;
  // activations for backward (allocated for max batch)
  int maxb = 0;
  float* act[4] = {nullptr, nullptr, nullptr, nullptr};  // outputs of layers 1..4
  int* argmax = nullptr;
  float* dact[2] = {nullptr, nullptr};                    // ping-pong gradient buffers
  float* partial = nullptr;                               // per-block weight-grad partials
  int64_t partial_elems = 0;
  float* loss = nullptr;                                  // device scalar
};

namespace fdr {

// --------------------------------------------------------------------------------------
// Network input, one pass over the spectrogram.  For bin b (channels n = b*factor + i,
// i < factor) and x = s - 1 (zero mean for an exponential(1) background):
//   power[t][b] = sum_i x[n, t] / sqrt(factor)
//   lag[l + ML][b] = sum_i sum_{t < Nt-1} x[n, t] * x[(n + l) mod Nf, t+1] / sqrt(factor*(Nt-1))
// each optionally compressed to sign(v)*log1p(|v|).  One CTA of 256 threads per bin; the
// bin's channels plus a halo of ML either side are staged in shared memory for `chunk`+1
// steps at a time (all loads of a chunk in flight together); every block reduction runs in
// a fixed order.
// --------------------------------------------------------------------------------------
constexpr int kFeatThreads = 256;
constexpr int kFeatMaxNt = 64;

__device__ __forceinline__ float compress_value(float v, int compress) {
  return compress ? copysignf(log1pf(fabsf(v)), v) : v;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

template <int ML>
__global__ void __launch_bounds__(kFeatThreads)
proposal_input_kernel(const float* __restrict__ spec, long long Nf, int Nt, int factor, int nbins,
                      int chunk, float pscale, float lscale, int compress,
                      float* __restrict__ pow_out, float* __restrict__ lag_out) {
  constexpr int NL = 2 * ML + 1;
  constexpr int NW = kFeatThreads / 32;
  extern __shared__ float tile[];  // (chunk + 1) rows of W floats
  __shared__ float red_p[kFeatMaxNt][NW];
  __shared__ float red_l[NL][NW];
  const int W = factor + 2 * ML;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int bin = blockIdx.x;
  const long long n0 = (long long)bin * factor;
  float lacc[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) lacc[l] = 0.f;
  for (int t0 = 0; t0 < Nt; t0 += chunk) {
    const int tc = min(chunk, Nt - t0);       // steps summed in this chunk
    const int rows = min(tc + 1, Nt - t0);    // plus the next step for the lag products
    __syncthreads();                          // the tile is free
    for (int r = 0; r < rows; ++r) {
      const float* col = spec + (long long)(t0 + r) * Nf;
      for (int i = tid; i < W; i += kFeatThreads) {
        long long n = n0 - ML + i;
        n = n < 0 ? n + Nf : (n >= Nf ? n - Nf : n);
        tile[r * W + i] = __ldg(col + n) - 1.f;
      }
    }
    __syncthreads();
    for (int r = 0; r < tc; ++r) {
      const float* xr = tile + r * W + ML;
      if (pow_out) {
        float ps = 0.f;
        for (int i = tid; i < factor; i += kFeatThreads) ps += xr[i];
        ps = warp_sum(ps);
        if (lane == 0) red_p[t0 + r][warp] = ps;
      }
      if (lag_out && r + 1 < rows) {
        const float* xn = tile + (r + 1) * W;  // channel n0 - ML + i of step t+1
        for (int i = tid; i < factor; i += kFeatThreads) {
          const float a = xr[i];
#pragma unroll
          for (int l = 0; l < NL; ++l) lacc[l] = fmaf(a, xn[i + l], lacc[l]);
        }
      }
    }
  }
  if (lag_out) {
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      const float v = warp_sum(lacc[l]);
      if (lane == 0) red_l[l][warp] = v;
    }
  }
  __syncthreads();
  if (pow_out && tid < Nt) {
    float v = 0.f;
    for (int w = 0; w < NW; ++w) v += red_p[tid][w];
    pow_out[(long long)tid * nbins + bin] = compress_value(v * pscale, compress);
  }
  if (lag_out && tid < NL) {
    float v = 0.f;
    for (int w = 0; w < NW; ++w) v += red_l[tid][w];
    lag_out[(long long)tid * nbins + bin] = compress_value(v * lscale, compress);
  }
}

static int launch_input(const float* spec, int64_t Nf, int64_t Nt, int factor, int maxlag,
                        int compress, float* pow_out, float* lag_out, cudaStream_t s,
                        const char* who) {
  FDR_CHECK_ARG(spec != nullptr && (pow_out || lag_out), "%s: NULL argument", who);
  FDR_CHECK_ARG(maxlag == 8, "%s: this build supports maxlag 8", who);
  FDR_CHECK_ARG(factor >= 1 && factor <= 4096 && Nf % factor == 0 && Nf >= 2 * maxlag + 1 &&
                Nf / factor <= 0x7fffffff,
                "%s: Nf must be a multiple of factor (<= 4096) and >= %d", who, 2 * maxlag + 1);
  FDR_CHECK_ARG(Nt >= 1 && Nt <= kFeatMaxNt && (lag_out == nullptr || Nt >= 2),
                "%s: Nt must be in [1, %d] (>= 2 for lag products)", who, kFeatMaxNt);
  const int nbins = (int)(Nf / factor);
  const int W = factor + 2 * maxlag;
  const int chunk = std::max(1, std::min(16, (int)((48 * 1024 / sizeof(float)) / W) - 1));
  const size_t sm = sizeof(float) * (size_t)(chunk + 1) * W;
  const float pscale = 1.f / sqrtf((float)factor);
  const float lscale = Nt >= 2 ? 1.f / sqrtf((float)factor * (float)(Nt - 1)) : 0.f;
  proposal_input_kernel<8><<<nbins, kFeatThreads, sm, s>>>(spec, Nf, (int)Nt, factor, nbins, chunk,
                                                           pscale, lscale, compress, pow_out, lag_out);
  FDR_LAUNCH_CHECK("proposal_input_kernel");
  return FDR_OK;
}

// --------------------------------------------------------------------------------------
// Convolution forward: y[b][co][x] = b[co] + sum_{ci,k} w[co][ci][k] * in[b][ci][x+k-pad]
// grid (X/kConvTile, B), block kConvTile threads (one bin each, all output channels).
// --------------------------------------------------------------------------------------
template <int COUT, int KS>
__global__ void __launch_bounds__(kConvTile)
conv_fwd_kernel(const float* __restrict__ in, int cin, int X, const __half* __restrict__ w,
                const float* __restrict__ bias, int relu, float* __restrict__ out) {
  extern __shared__ float sm[];
  const int pad = KS / 2;
  const int TW = kConvTile + KS - 1;
  float* xs = sm;                 // cin * TW
  float* wsm = sm + cin * TW;     // COUT * cin * KS
  const int b = blockIdx.y, x0 = blockIdx.x * kConvTile;
  const float* inb = in + (long long)b * cin * X;
  for (int i = threadIdx.x; i < cin * TW; i += blockDim.x) {
    const int ci = i / TW, xx = x0 - pad + (i - ci * TW);
    xs[i] = (xx >= 0 && xx < X) ? inb[(long long)ci * X + xx] : 0.f;
  }
  for (int i = threadIdx.x; i < COUT * cin * KS; i += blockDim.x) wsm[i] = __half2float(w[i]);
  __syncthreads();
  const int x = x0 + threadIdx.x;
  if (x >= X) return;
  float acc[COUT];
#pragma unroll
  for (int co = 0; co < COUT; ++co) acc[co] = bias[co];
  for (int ci = 0; ci < cin; ++ci) {
#pragma unroll
    for (int k = 0; k < KS; ++k) {
      const float v = xs[ci * TW + threadIdx.x + k];
#pragma unroll
      for (int co = 0; co < COUT; ++co) acc[co] = fmaf(wsm[(co * cin + ci) * KS + k], v, acc[co]);
    }
  }
  float* ob = out + (long long)b * COUT * X;
#pragma unroll
  for (int co = 0; co < COUT; ++co) ob[(long long)co * X + x] = relu ? fmaxf(acc[co], 0.f) : acc[co];
}

// logits[b][w] = max_x y[b][w][x] (first maximum), argmax kept for the backward pass.
__global__ void maxpool_kernel(const float* __restrict__ y, int nw, int X, float* __restrict__ logits,
                               int* __restrict__ argmax) {
  const int b = blockIdx.y, w = blockIdx.x;
  const float* r = y + ((long long)b * nw + w) * X;
  float best = -INFINITY;
  int bi = 0;
  for (int x = threadIdx.x; x < X; x += blockDim.x) {
    const float v = r[x];
    if (v > best) { best = v; bi = x; }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const float ov = __shfl_down_sync(0xffffffffu, best, o);
    const int oi = __shfl_down_sync(0xffffffffu, bi, o);
    if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
  }
  __shared__ float sv[32];
  __shared__ int si[32];
  if ((threadIdx.x & 31) == 0) { sv[threadIdx.x >> 5] = best; si[threadIdx.x >> 5] = bi; }
  __syncthreads();
  if (threadIdx.x == 0) {
    float bv = sv[0];
    int bix = si[0];
    for (int i = 1; i < (int)(blockDim.x + 31) / 32; ++i)
      if (sv[i] > bv || (sv[i] == bv && si[i] < bix)) { bv = sv[i]; bix = si[i]; }
    logits[(long long)b * nw + w] = bv;
    argmax[(long long)b * nw + w] = bix;
  }
}

// Mean BCE with logits (single block, fixed order) and its gradient scattered to the
// argmax bins of dy (dy must be zero on entry).
__global__ void bce_kernel(const float* __restrict__ logits, const float* __restrict__ labels,
                           const int* __restrict__ argmax, int n, int nw, int X,
                           float* __restrict__ dy, float* __restrict__ loss) {
  __shared__ float part[256];
  float s = 0.f;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float z = logits[i], y = labels[i];
    s += fmaxf(z, 0.f) - z * y + log1pf(expf(-fabsf(z)));
    if (dy) {
      const float p = 1.f / (1.f + expf(-z));
      const int b = i / nw, w = i - b * nw;
      dy[((long long)b * nw + w) * X + argmax[i]] = (p - y) / (float)n;
    }
  }
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int i = 0; i < blockDim.x; ++i) t += part[i];
    *loss = t / (float)n;
  }
}

// d_in[b][ci][x] = sum_{co,k} w[co][ci][k] * g[b][co][x-k+pad],
// g = d_out masked by the ReLU of the layer output (when relu_out != NULL).
__global__ void __launch_bounds__(kConvTile)
conv_bwd_data_kernel(const float* __restrict__ dout, const float* __restrict__ relu_out, int cout,
                     int cin, int ks, int X, const __half* __restrict__ w, float* __restrict__ din) {
  extern __shared__ float sm[];
  const int pad = ks / 2;
  const int TW = kConvTile + ks - 1;
  float* gs = sm;                  // cout * TW
  float* wsm = sm + cout * TW;     // cout * cin * ks
  const int b = blockIdx.y, x0 = blockIdx.x * kConvTile;
  for (int i = threadIdx.x; i < cout * TW; i += blockDim.x) {
    const int co = i / TW, xx = x0 + pad - (ks - 1) + (i - co * TW);  // covers x - k + pad
    float g = 0.f;
    if (xx >= 0 && xx < X) {
      const long long idx = ((long long)b * cout + co) * X + xx;
      g = dout[idx];
      if (relu_out && relu_out[idx] <= 0.f) g = 0.f;
    }
    gs[i] = g;
  }
  for (int i = threadIdx.x; i < cout * cin * ks; i += blockDim.x) wsm[i] = __half2float(w[i]);
  __syncthreads();
  const int x = x0 + threadIdx.x;
  if (x >= X) return;
  for (int ci = 0; ci < cin; ++ci) {
    float acc = 0.f;
    for (int co = 0; co < cout; ++co)
      for (int k = 0; k < ks; ++k)
        acc = fmaf(wsm[(co * cin + ci) * ks + k], gs[co * TW + threadIdx.x + (ks - 1) - k], acc);
    din[((long long)b * cin + ci) * X + x] = acc;
  }
}

// Per-block partial weight / bias gradients: partial[blk][co][ci][k] and [blk][bias co],
// blk = (b, x-tile).  grid (X/kConvTile, B), block kConvTile.
__global__ void __launch_bounds__(kConvTile)
conv_bwd_weight_kernel(const float* __restrict__ dout, const float* __restrict__ relu_out,
                       const float* __restrict__ in, int cout, int cin, int ks, int X,
                       float* __restrict__ partial) {
  extern __shared__ float sm[];
  const int pad = ks / 2;
  const int TW = kConvTile + ks - 1;
  float* xs = sm;                       // cin * TW
  float* gs = sm + cin * TW;            // cout * kConvTile
  const int b = blockIdx.y, x0 = blockIdx.x * kConvTile;
  for (int i = threadIdx.x; i < cin * TW; i += blockDim.x) {
    const int ci = i / TW, xx = x0 - pad + (i - ci * TW);
    xs[i] = (xx >= 0 && xx < X) ? in[((long long)b * cin + ci) * X + xx] : 0.f;
  }
  for (int i = threadIdx.x; i < cout * kConvTile; i += blockDim.x) {
    const int co = i / kConvTile, xx = x0 + (i - co * kConvTile);
    float g = 0.f;
    if (xx < X) {
      const long long idx = ((long long)b * cout + co) * X + xx;
      g = dout[idx];
      if (relu_out && relu_out[idx] <= 0.f) g = 0.f;
    }
    gs[i] = g;
  }
  __syncthreads();
  const int nw = cout * cin * ks;
  const long long blk = (long long)blockIdx.y * gridDim.x + blockIdx.x;
  float* pb = partial + blk * (nw + cout);
  for (int i = threadIdx.x; i < nw + cout; i += blockDim.x) {
    float acc = 0.f;
    if (i < nw) {
      const int co = i / (cin * ks), r = i - co * cin * ks, ci = r / ks, k = r - ci * ks;
      for (int x = 0; x < kConvTile; ++x) acc = fmaf(gs[co * kConvTile + x], xs[ci * TW + x + k], acc);
    } else {
      const int co = i - nw;
      for (int x = 0; x < kConvTile; ++x) acc += gs[co * kConvTile + x];
    }
    pb[i] = acc;
  }
}

// grad[off + i] = sum over blocks (in order) of partial[blk][i]
__global__ void reduce_partials_kernel(const float* __restrict__ partial, int nblk, int n,
                                       float* __restrict__ gw, float* __restrict__ gb, int nw) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float s = 0.f;
  for (int k = 0; k < nblk; ++k) s += partial[(long long)k * n + i];
  if (i < nw) gw[i] = s; else gb[i - nw] = s;
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, __half* __restrict__ wh, long long n, float lr,
                            float b1, float b2, float eps, float c1, float c2) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  p[i] = pi;
  wh[i] = __float2half_rn(pi);
}

__global__ void to_half_kernel(const float* __restrict__ p, __half* __restrict__ wh, long long n) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) wh[i] = __float2half_rn(p[i]);
}

// ---- host helpers ---------------------------------------------------------------------
static uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

static int set_attrs() {
  static bool done[64] = {false};
  int dev = 0;
  FDR_CUDA(cudaGetDevice(&dev));
  if (dev < 64 && done[dev]) return FDR_OK;
  const int big = 160 * 1024;  // conv layers with up to 64 input channels need <= 107 KB
  FDR_CUDA(cudaFuncSetAttribute(conv_fwd_kernel<32, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  FDR_CUDA(cudaFuncSetAttribute(conv_fwd_kernel<16, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  FDR_CUDA(cudaFuncSetAttribute(conv_bwd_data_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  FDR_CUDA(cudaFuncSetAttribute(conv_bwd_weight_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  if (dev < 64) done[dev] = true;
  return FDR_OK;
}

static int conv_forward(const fdr_propose_net* n, int li, const float* in, int B, float* out,
                        cudaStream_t s) {
  const Layer& L = n->L[li];
  const int X = n->nbins;
  const int TW = kConvTile + L.k - 1;
  const size_t sm = sizeof(float) * (L.cin * TW + L.cout * L.cin * L.k);
  dim3 grid((unsigned)cdiv(X, kConvTile), (unsigned)B);
  const int relu = li < 3;
  const __half* w = n->wh + L.woff;
  const float* bias = n->params + L.boff;
  if (L.cout == 32 && L.k == 5) {
    conv_fwd_kernel<32, 5><<<grid, kConvTile, sm, s>>>(in, L.cin, X, w, bias, relu, out);
  } else if (L.cout == 16 && L.k == 1) {
    conv_fwd_kernel<16, 1><<<grid, kConvTile, sm, s>>>(in, L.cin, X, w, bias, relu, out);
  } else {
    set_error(FDR_ERR_INVALID_ARGUMENT, "proposal net: unsupported layer shape");
    return FDR_ERR_INVALID_ARGUMENT;
  }
  FDR_LAUNCH_CHECK("conv_fwd_kernel");
  return FDR_OK;
}

static int net_forward(fdr_propose_net* n, const float* x, int B, float* logits, cudaStream_t s) {
  FDR_CHECK_ARG(B >= 1 && B <= n->maxb, "proposal net: batch %d exceeds the maximum %d", B, n->maxb);
  const float* in = x;
  for (int li = 0; li < 4; ++li) {
    FDR_TRY(conv_forward(n, li, in, B, n->act[li], s));
    in = n->act[li];
  }
  maxpool_kernel<<<dim3(n->nwin, B), 256, 0, s>>>(n->act[3], n->nwin, n->nbins, logits, n->argmax);
  FDR_LAUNCH_CHECK("maxpool_kernel");
  return FDR_OK;
}

// Forward + loss + backward into n->grad.  logits: device [B][nwin] scratch.
static int net_grad(fdr_propose_net* n, const float* x, const float* labels, int B, float* logits,
                    cudaStream_t s) {
  FDR_TRY(net_forward(n, x, B, logits, s));
  const int X = n->nbins;
  float* dy = n->dact[0];
  FDR_CUDA(cudaMemsetAsync(dy, 0, sizeof(float) * (size_t)B * n->nwin * X, s));
  bce_kernel<<<1, 256, 0, s>>>(logits, labels, n->argmax, B * n->nwin, n->nwin, X, dy, n->loss);
  FDR_LAUNCH_CHECK("bce_kernel");
  for (int li = 3; li >= 0; --li) {
    const Layer& L = n->L[li];
    const float* layer_in = li == 0 ? x : n->act[li - 1];
    const float* relu_out = li < 3 ? n->act[li] : nullptr;
    const int TW = kConvTile + L.k - 1;
    dim3 grid((unsigned)cdiv(X, kConvTile), (unsigned)B);
    const int nblk = grid.x * grid.y;
    const int nwp = L.cout * L.cin * L.k + L.cout;
    size_t smw = sizeof(float) * (L.cin * TW + L.cout * kConvTile);
    conv_bwd_weight_kernel<<<grid, kConvTile, smw, s>>>(dy, relu_out, layer_in, L.cout, L.cin, L.k,
                                                        X, n->partial);
    FDR_LAUNCH_CHECK("conv_bwd_weight_kernel");
    reduce_partials_kernel<<<(unsigned)cdiv(nwp, 256), 256, 0, s>>>(
        n->partial, nblk, nwp, n->grad + L.woff, n->grad + L.boff, L.cout * L.cin * L.k);
    FDR_LAUNCH_CHECK("reduce_partials_kernel");
    if (li > 0) {
      float* din = (dy == n->dact[0]) ? n->dact[1] : n->dact[0];
      size_t smd = sizeof(float) * (L.cout * TW + L.cout * L.cin * L.k);
      conv_bwd_data_kernel<<<grid, kConvTile, smd, s>>>(dy, relu_out, L.cout, L.cin, L.k, X,
                                                        n->wh + L.woff, din);
      FDR_LAUNCH_CHECK("conv_bwd_data_kernel");
      dy = din;
    }
  }
  return FDR_OK;
}

static void net_release(fdr_propose_net* n) {
  if (!n) return;
  cudaFree(n->params);
  cudaFree(n->wh);
  cudaFree(n->m);
  cudaFree(n->v);
  cudaFree(n->grad);
  for (auto* a : n->act) cudaFree(a);
  cudaFree(n->argmax);
  for (auto* a : n->dact) cudaFree(a);
  cudaFree(n->partial);
  cudaFree(n->loss);
  delete n;
}

}  // namespace fdr

using namespace fdr;

extern "C" {

int fdr_propose_create(fdr_propose_net** out, int nbins, int nt, int width, int ksize, int nwin,
                       int max_batch, uint64_t seed) {
  FDR_CHECK_ARG(out != nullptr, "fdr_propose_create: NULL handle");
  FDR_CHECK_ARG(nbins >= 1 && nt >= 1 && nt <= 64 && nwin >= 1 && max_batch >= 1,
                "fdr_propose_create: bad sizes");
  FDR_CHECK_ARG(width == 32 && ksize == 5 && nwin == 16,
                "fdr_propose_create: this build supports width 32, kernel 5, 16 windows");
  *out = nullptr;
  FDR_TRY(set_attrs());
  fdr_propose_net* n = new fdr_propose_net();
  n->nbins = nbins; n->nt = nt; n->width = width; n->ksize = ksize; n->nwin = nwin;
  n->maxb = max_batch;
  n->seed = seed;
  const int cins[4] = {nt, width, width, width}, couts[4] = {width, width, width, nwin};
  const int ks[4] = {ksize, ksize, ksize, 1};
  int64_t off = 0;
  for (int i = 0; i < 4; ++i) {
    n->L[i] = {cins[i], couts[i], ks[i], off, off + (int64_t)couts[i] * cins[i] * ks[i]};
    off = n->L[i].boff + couts[i];
  }
  n->nparams = off;
  // He-uniform initialisation from a seeded splitmix64 stream; zero biases.
  std::vector<float> h((size_t)off, 0.f);
  uint64_t st = seed;
  for (int i = 0; i < 4; ++i) {
    const float bound = sqrtf(6.f / (float)(n->L[i].cin * n->L[i].k));
    for (int64_t j = 0; j < (int64_t)n->L[i].cout * n->L[i].cin * n->L[i].k; ++j) {
      const double u = (double)(splitmix(st) >> 11) * (1.0 / 9007199254740992.0);
      h[(size_t)(n->L[i].woff + j)] = (float)((2.0 * u - 1.0) * bound);
    }
  }
  const size_t act_elems = (size_t)max_batch * width * nbins;
  int64_t maxblk = cdiv(nbins, kConvTile) * max_batch, maxw = 0;
  for (int i = 0; i < 4; ++i) maxw = std::max<int64_t>(maxw, (int64_t)couts[i] * cins[i] * ks[i] + couts[i]);
  n->partial_elems = maxblk * maxw;
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = cudaMalloc(&n->params, sizeof(float) * off);
  if (e == cudaSuccess) e = cudaMalloc(&n->wh, sizeof(__half) * off);
  if (e == cudaSuccess) e = cudaMalloc(&n->m, sizeof(float) * off);
  if (e == cudaSuccess) e = cudaMalloc(&n->v, sizeof(float) * off);
  if (e == cudaSuccess) e = cudaMalloc(&n->grad, sizeof(float) * off);
  for (int i = 0; i < 4 && e == cudaSuccess; ++i) e = cudaMalloc(&n->act[i], sizeof(float) * act_elems);
  for (int i = 0; i < 2 && e == cudaSuccess; ++i) e = cudaMalloc(&n->dact[i], sizeof(float) * act_elems);
  if (e == cudaSuccess) e = cudaMalloc(&n->argmax, sizeof(int) * (size_t)max_batch * nwin);
  if (e == cudaSuccess) e = cudaMalloc(&n->partial, sizeof(float) * n->partial_elems);
  if (e == cudaSuccess) e = cudaMalloc(&n->loss, sizeof(float));
  if (e == cudaSuccess) e = cudaMemcpy(n->params, h.data(), sizeof(float) * off, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(n->m, 0, sizeof(float) * off);
  if (e == cudaSuccess) e = cudaMemset(n->v, 0, sizeof(float) * off);
  if (e != cudaSuccess) {
    int st2 = cuda_status(e, "fdr_propose_create");
    net_release(n);
    return st2;
  }
  to_half_kernel<<<(unsigned)cdiv(off, 256), 256>>>(n->params, n->wh, off);
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) { int st2 = cuda_status(e, "fdr_propose_create"); net_release(n); return st2; }
  count_launch();
  *out = n;
  return FDR_OK;
}

int fdr_propose_destroy(fdr_propose_net* n) {
  if (n) { cudaDeviceSynchronize(); net_release(n); }
  return FDR_OK;
}

int fdr_propose_num_params(const fdr_propose_net* n, int64_t* count) {
  FDR_CHECK_ARG(n && count, "NULL argument");
  *count = n->nparams;
  return FDR_OK;
}

int fdr_propose_features(const float* spec, int64_t Nf, int64_t Nt, int factor, int compress,
                         float* out, fdr_stream_t stream) {
  return launch_input(spec, Nf, Nt, factor, 8, compress, out, nullptr, (cudaStream_t)stream,
                      "fdr_propose_features");
}

int fdr_propose_lag_features(const float* spec, int64_t Nf, int64_t Nt, int factor, int maxlag,
                             int compress, float* out, fdr_stream_t stream) {
  return launch_input(spec, Nf, Nt, factor, maxlag, compress, nullptr, out, (cudaStream_t)stream,
                      "fdr_propose_lag_features");
}

int fdr_propose_input(const float* spec, int64_t Nf, int64_t Nt, int factor, int maxlag,
                      int compress, float* out, fdr_stream_t stream) {
  FDR_CHECK_ARG(out != nullptr, "fdr_propose_input: NULL argument");
  return launch_input(spec, Nf, Nt, factor, maxlag, compress, out,
                      out + Nt * (Nf / std::max(factor, 1)), (cudaStream_t)stream, "fdr_propose_input");
}

int fdr_propose_forward(fdr_propose_net* n, const float* x, int batch, float* logits,
                        fdr_stream_t stream) {
  FDR_CHECK_ARG(n && x && logits, "fdr_propose_forward: NULL argument");
  return net_forward(n, x, batch, logits, (cudaStream_t)stream);
}

int fdr_propose_gradients(fdr_propose_net* n, const float* x, const float* labels, int batch,
                          float* logits, float* grad_out, float* loss_out, fdr_stream_t stream) {
  FDR_CHECK_ARG(n && x && labels && logits, "fdr_propose_gradients: NULL argument");
  cudaStream_t s = (cudaStream_t)stream;
  FDR_TRY(net_grad(n, x, labels, batch, logits, s));
  if (grad_out) FDR_CUDA(cudaMemcpyAsync(grad_out, n->grad, sizeof(float) * n->nparams, cudaMemcpyDeviceToDevice, s));
  if (loss_out) FDR_CUDA(cudaMemcpyAsync(loss_out, n->loss, sizeof(float), cudaMemcpyDeviceToDevice, s));
  return FDR_OK;
}

int fdr_propose_train_step(fdr_propose_net* n, const float* x, const float* labels, int batch,
                           float lr, float* logits, float* loss_out, fdr_stream_t stream) {
  FDR_CHECK_ARG(n && x && labels && logits, "fdr_propose_train_step: NULL argument");
  cudaStream_t s = (cudaStream_t)stream;
  FDR_TRY(net_grad(n, x, labels, batch, logits, s));
  n->step += 1;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float c1 = 1.f - powf(b1, (float)n->step), c2 = 1.f - powf(b2, (float)n->step);
  adam_kernel<<<(unsigned)cdiv(n->nparams, 256), 256, 0, s>>>(n->params, n->grad, n->m, n->v, n->wh,
                                                               n->nparams, lr, b1, b2, eps, c1, c2);
  FDR_LAUNCH_CHECK("adam_kernel");
  if (loss_out) FDR_CUDA(cudaMemcpyAsync(loss_out, n->loss, sizeof(float), cudaMemcpyDeviceToDevice, s));
  return FDR_OK;
}

// Checkpoint state: params, m, v (host float arrays of num_params) and the step count.
int fdr_propose_get_state(fdr_propose_net* n, float* params, float* m, float* v, int64_t* step) {
  FDR_CHECK_ARG(n != nullptr, "NULL net");
  FDR_CUDA(cudaDeviceSynchronize());
  if (params) FDR_CUDA(cudaMemcpy(params, n->params, sizeof(float) * n->nparams, cudaMemcpyDeviceToHost));
  if (m) FDR_CUDA(cudaMemcpy(m, n->m, sizeof(float) * n->nparams, cudaMemcpyDeviceToHost));
  if (v) FDR_CUDA(cudaMemcpy(v, n->v, sizeof(float) * n->nparams, cudaMemcpyDeviceToHost));
  if (step) *step = n->step;
  return FDR_OK;
}

int fdr_propose_set_state(fdr_propose_net* n, const float* params, const float* m, const float* v,
                          int64_t step) {
  FDR_CHECK_ARG(n && params, "NULL argument");
  FDR_CUDA(cudaDeviceSynchronize());
  FDR_CUDA(cudaMemcpy(n->params, params, sizeof(float) * n->nparams, cudaMemcpyHostToDevice));
  if (m) FDR_CUDA(cudaMemcpy(n->m, m, sizeof(float) * n->nparams, cudaMemcpyHostToDevice));
  if (v) FDR_CUDA(cudaMemcpy(n->v, v, sizeof(float) * n->nparams, cudaMemcpyHostToDevice));
  n->step = step;
  to_half_kernel<<<(unsigned)cdiv(n->nparams, 256), 256>>>(n->params, n->wh, n->nparams);
  FDR_LAUNCH_CHECK("to_half_kernel");
  FDR_CUDA(cudaDeviceSynchronize());
  return FDR_OK;
}

}  // extern "C"
