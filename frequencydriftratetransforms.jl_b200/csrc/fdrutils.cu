// FDR statistics, normalisation and proto-hit search (src/fdrutils.jl of
// FrequencyDriftRateTransforms.jl): fdrstats (:39-50), fdrnormalize! (:70-90),
// fdrdenormalize (:104-119), findprotohits (:148-169).
#include <math.h>
#include <string.h>

#define FDR_TU_ID 4
#include "fdr_internal.cuh"

namespace fdr {

constexpr int kRedThreads = 256;
constexpr int kHitThreads = 256;
constexpr int kHitRounds = 16;
constexpr long long kHitTile = (long long)kHitThreads * kHitRounds;  // elements per tile

// ------------------------------------------------------------------------------------
// fdrstats in the reference's Float32 arithmetic.
//
// m = mean(fdr[:,1]) and s = minimum(std(fdr, dims=1)) (fdrutils.jl:39-50) reduce each
// column with Julia's pairwise mapreduce (Base.mapreduce_impl, block size 1024): a range of
// at most 1024 elements (a leaf) is summed sequentially, ((f(a1) + f(a2)) + f(a3)) + ...,
// and a longer range [lo, hi] splits at mid = lo + (hi - lo) >> 1, its value being
// left + right.  mean = sum / Float32(n); Statistics.varm! scales the pairwise sum of
// abs2(x - mean) by Float32(1 // (n - 1)); std = sqrt of that, all in Float32.
//
// With D the smallest depth at which every node of the recursion has at most 1024
// elements (node lengths at depth d are ceil(n/2^d) or floor(n/2^d)), every node above
// depth D-1 is internal and every node at depth D-1 (a "unit", M = 2^(D-1) of them) is one
// leaf or two.  A unit's range follows from its index: from the root, bit b of the index
// (most significant first) picks the left part (the first ceil(len/2) elements) or the
// right part.  Units are summed by threads, and combined in order up a perfect binary tree:
// within a thread (G consecutive units), across the CTA (T threads) and across the S CTAs of
// a column (S partials, combined by the next kernel).
// ------------------------------------------------------------------------------------
constexpr int kPwThreads = 256;
constexpr long long kPwLeaf = 1024;

__device__ __forceinline__ const float* pw_column(const float* const* mats, const float* base,
                                                  long long Nf, long long Nrb, long long col) {
  if (mats) {
    const long long b = col / Nrb;
    return mats[b] + (col - b * Nrb) * Nf;
  }
  return base + col * Nf;
}

// f(x) of the reduction: x (sum) or abs2(x - m) (centralised sum of squares), rounded as
// Julia's Float32 operations, never fused into a multiply-add.
template <bool SQ>
__device__ __forceinline__ float pw_f(float x, float m) {
  if (SQ) {
    const float d = __fsub_rn(x, m);
    return __fmul_rn(d, d);
  }
  return x;
}

// v + f(a.x) + f(a.y) + f(a.z) + f(a.w) in order; the plain-sum pass (!SQ) also keeps the
// running maximum mx of the values (fmaxf: a NaN never becomes the maximum).
template <bool SQ>
__device__ __forceinline__ float pw_add4(float v, float4 a, float m, float& mx) {
  if (!SQ) mx = fmaxf(mx, fmaxf(fmaxf(a.x, a.y), fmaxf(a.z, a.w)));
  v = __fadd_rn(v, pw_f<SQ>(a.x, m));
  v = __fadd_rn(v, pw_f<SQ>(a.y, m));
  v = __fadd_rn(v, pw_f<SQ>(a.z, m));
  return __fadd_rn(v, pw_f<SQ>(a.w, m));
}

// Sequential sum of one leaf of len >= 1 elements (and, for !SQ, its maximum in mx, which
// starts at -inf).  The 16-byte loads run one batch of four ahead of the adds that consume
// them (software pipelining), so each thread keeps up to eight loads in flight while its
// dependent chain of adds proceeds in order.
template <bool SQ>
__device__ float pw_leaf(const float* __restrict__ p, long long len, float m, float& mx) {
  float v;
  long long i;
  if ((reinterpret_cast<uintptr_t>(p) & 15) == 0 && len >= 4) {
    const float4* q = reinterpret_cast<const float4*>(p);
    const long long nq = len >> 2;
    const float4 a = __ldg(q);
    if (!SQ) mx = fmaxf(mx, fmaxf(fmaxf(a.x, a.y), fmaxf(a.z, a.w)));
    v = pw_f<SQ>(a.x, m);
    v = __fadd_rn(v, pw_f<SQ>(a.y, m));
    v = __fadd_rn(v, pw_f<SQ>(a.z, m));
    v = __fadd_rn(v, pw_f<SQ>(a.w, m));
    long long k = 1;
    if (k + 4 <= nq) {
      float4 cur[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) cur[u] = __ldg(q + k + u);
      k += 4;
      for (; k + 4 <= nq; k += 4) {
        float4 nxt[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) nxt[u] = __ldg(q + k + u);
#pragma unroll
        for (int u = 0; u < 4; ++u) v = pw_add4<SQ>(v, cur[u], m, mx);
#pragma unroll
        for (int u = 0; u < 4; ++u) cur[u] = nxt[u];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) v = pw_add4<SQ>(v, cur[u], m, mx);
    }
    for (; k < nq; ++k) v = pw_add4<SQ>(v, __ldg(q + k), m, mx);
    i = nq << 2;
  } else {
    const float a = __ldg(p);
    if (!SQ) mx = fmaxf(mx, a);
    v = pw_f<SQ>(a, m);
    i = 1;
  }
  for (; i < len; ++i) {
    const float a = __ldg(p + i);
    if (!SQ) mx = fmaxf(mx, a);
    v = __fadd_rn(v, pw_f<SQ>(a, m));
  }
  return v;
}

// Coalesced form for columns whose leaves are all exactly 1024 elements (n a power of two,
// n >= 2^15, 16-byte aligned columns): leaf i of the column is elements [1024 i, 1024 i +
// 1024).  The 32 lanes of a warp own 32 leaves; in each of 32 rounds the warp reads 32
// elements of every one of them with 16-byte loads (four leaves per load instruction, one
// whole 128-byte line each) into shared memory, then each lane adds its leaf's 32 elements
// in order.  stage: 32 rows of 33 floats (lane L reading row L, element e, hits bank
// (L + e) mod 32).
template <bool SQ>
__device__ float pw_leaf_warp(const float* __restrict__ x, long long my_leaf, float m,
                              float* __restrict__ stage, float& mx) {
  const int lane = threadIdx.x & 31;
  const int g = lane >> 3, q = lane & 7;
  long long slot_leaf[8];  // load i: lanes 8g..8g+7 fetch the leaf of lane 4i + g
#pragma unroll
  for (int i = 0; i < 8; ++i) slot_leaf[i] = __shfl_sync(0xffffffffu, my_leaf, 4 * i + g);
  float v = 0.f;
  for (int r = 0; r < 32; ++r) {
    float4 t[8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
      t[i] = __ldg(reinterpret_cast<const float4*>(x + slot_leaf[i] * 1024 + 32 * r) + q);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      float* d = stage + (4 * i + g) * 33 + 4 * q;
      d[0] = t[i].x; d[1] = t[i].y; d[2] = t[i].z; d[3] = t[i].w;
    }
    __syncwarp();
    const float* src = stage + lane * 33;
    int e0 = 0;
    if (r == 0) { v = pw_f<SQ>(src[0], m); e0 = 1; }
#pragma unroll 8
    for (int e = e0; e < 32; ++e) v = __fadd_rn(v, pw_f<SQ>(src[e], m));
    if (!SQ) {
#pragma unroll 8
      for (int e = 0; e < 32; ++e) mx = fmaxf(mx, src[e]);
    }
    __syncwarp();
  }
  return v;
}

// Range [lo, lo + len) of unit u (the depth-`bits` node) of a column of n elements.
__device__ __forceinline__ void pw_unit_range(long long n, int bits, long long u, long long& lo,
                                              long long& len) {
  lo = 0;
  len = n;
  for (int b = bits - 1; b >= 0; --b) {
    const long long c = (len + 1) >> 1;
    if ((u >> b) & 1) { lo += c; len -= c; } else { len = c; }
  }
}

// Pairwise (perfect binary tree, left + right) combination of S values, S a power of two.
__device__ __forceinline__ float pw_tree(const float* __restrict__ v, int S) {
  float stk[32];
  for (int k = 0; k < S; ++k) {
    float a = v[k];
    int lev = 0;
    while ((k >> lev) & 1) { a = __fadd_rn(stk[lev], a); ++lev; }
    stk[lev] = a;
  }
  int top = 0;
  while ((1 << top) < S) ++top;
  return stk[top];
}

// grid (S, ncols), block max(2*T, 32) threads (T a power of two <= kPwThreads/2): CTA (s, col)
// combines the units [s*T*G, (s+1)*T*G) of column col into part[col*S + s].  Threads 2i and
// 2i+1 (adjacent lanes) take the first and second leaf of each of their G units and combine
// them with one shuffle.  With SQ, f(x) = abs2(x - mean of the column), the mean taken from
// the first pass's partials part_sum.  Without SQ and with leafmax set, the maximum of leaf
// slot (u, h) (the first or second leaf of unit u; -inf for the absent second leaf of a
// one-leaf unit) goes to leafmax[col * 2^(bits+1) + 2u + h].
template <bool SQ>
__global__ void __launch_bounds__(kPwThreads, 4)  // <= 64 registers: 8 CTAs of 128 threads per SM
pw_units_kernel(const float* const* __restrict__ mats, const float* __restrict__ base, long long Nf,
                long long Nrb, int bits, int T, long long G, int S, const float* __restrict__ part_sum,
                float* __restrict__ part, int leaves1024, float* __restrict__ leafmax) {
  const long long col = blockIdx.y;
  const float* x = pw_column(mats, base, Nf, Nrb, col);
  __shared__ float red[kPwThreads / 2];
  extern __shared__ float stage[];  // coalesced form: 32 x 33 floats per warp
  // the coalesced form needs every lane active and an aligned column (uniform per CTA)
  const bool warp_path = leaves1024 && (reinterpret_cast<uintptr_t>(x) & 15) == 0 &&
                         (int)blockDim.x == 2 * T;
  __shared__ float s_mean;
  float m = 0.f;
  if (SQ) {
    if (threadIdx.x == 0) s_mean = __fdiv_rn(pw_tree(part_sum + col * S, S), (float)Nf);
    __syncthreads();
    m = s_mean;
  }
  const int h = threadIdx.x & 1;
  const bool active = (int)(threadIdx.x >> 1) < T;  // a block of 32 threads may exceed 2T
  const long long u0 = ((long long)blockIdx.x * T + (threadIdx.x >> 1)) * G;
  float stk[40];
  for (long long k = 0; k < G; ++k) {
    long long lo = 0, len = 0;
    if (active) pw_unit_range(Nf, bits, u0 + k, lo, len);
    const bool two = len > kPwLeaf;
    const long long c = two ? (len + 1) >> 1 : len;
    const long long ln = h ? (two ? len - c : 0) : c;
    float v;
    float mx = -INFINITY;
    if (warp_path) {  // unit u = leaves 2u and 2u + 1 of 1024 elements
      const long long my = 2 * (u0 + k) + h;
      v = pw_leaf_warp<SQ>(x, FDR_DBG_OK(my * 1024 + 1024 <= Nf) ? my : 0, m,
                           stage + (threadIdx.x >> 5) * (32 * 33), mx);
    } else {
      v = (ln > 0 && FDR_DBG_OK(lo + (h ? c : 0) + ln <= Nf)) ? pw_leaf<SQ>(x + lo + (h ? c : 0), ln, m, mx) : 0.f;
    }
    if (!SQ && leafmax && active)
      leafmax[(col << (bits + 1)) + 2 * (u0 + k) + h] = mx;
    const float o = __shfl_xor_sync(0xffffffffu, v, 1);
    float a = h ? o : v;                    // the unit's first leaf
    if (two) a = __fadd_rn(a, h ? v : o);   // + its second leaf
    int lev = 0;
    while ((k >> lev) & 1) { a = __fadd_rn(stk[lev], a); ++lev; }
    stk[lev] = a;
  }
  int top = 0;
  while ((1LL << top) < G) ++top;
  if (h == 0 && active) red[threadIdx.x >> 1] = stk[top];
  __syncthreads();
  for (int w = T >> 1; w >= 1; w >>= 1) {
    float a = 0.f;
    if ((int)threadIdx.x < w) a = __fadd_rn(red[2 * threadIdx.x], red[2 * threadIdx.x + 1]);
    __syncthreads();
    if ((int)threadIdx.x < w) red[threadIdx.x] = a;
    __syncthreads();
  }
  if (threadIdx.x == 0) part[col * S + blockIdx.x] = red[0];
}

// m = mean of column 0, s = minimum std over the columns (NaN if any is NaN); ms[2] = the
// fdrdenormalize threshold snr*s + m in Float64 (FDR_SNR_F64) or Float32 (FDR_SNR_F32).
__global__ void pw_finalize_kernel(const float* __restrict__ part_sum, const float* __restrict__ part_sq,
                                   long long ncols, int S, long long Nf, int snr_mode, double snr,
                                   double* __restrict__ ms) {
  __shared__ float smin[256];
  __shared__ int snan[256];
  const float inv = __fdiv_rn(1.0f, (float)(Nf - 1));  // Float32(1 // (n-1))
  float best = INFINITY;
  int nan = 0;
  for (long long c = threadIdx.x; c < ncols; c += blockDim.x) {
    const float sd = __fsqrt_rn(__fmul_rn(pw_tree(part_sq + c * S, S), inv));
    if (isnan(sd)) nan = 1; else best = fminf(best, sd);
  }
  smin[threadIdx.x] = best;
  snan[threadIdx.x] = nan;
  __syncthreads();
  if (threadIdx.x == 0) {
    float b = INFINITY;
    int anynan = 0;
    for (int i = 0; i < (int)blockDim.x; ++i) { b = fminf(b, smin[i]); anynan |= snan[i]; }
    const float m = __fdiv_rn(pw_tree(part_sum, S), (float)Nf);
    const float s = anynan ? __int_as_float(0x7fc00000) : b;
    ms[0] = (double)m;
    ms[1] = (double)s;
    if (snr_mode == FDR_SNR_F32)
      ms[2] = (double)__fadd_rn(__fmul_rn((float)snr, s), m);
    else
      ms[2] = snr * (double)s + (double)m;
  }
}

struct PwShape {
  int bits;     // depth of the units
  long long M;  // units per column
  int T;        // threads per CTA
  int S;        // CTAs (partials) per column
  long long G;  // units per thread
};

static PwShape pw_shape(long long n, long long ncols, int smax) {
  int D = 0;
  while (cdiv(n, 1LL << D) > kPwLeaf) ++D;
  PwShape p;
  p.bits = D > 0 ? D - 1 : 0;
  p.M = 1LL << p.bits;
  p.T = (int)std::min<long long>(kPwThreads / 2, p.M);
  long long S = 1;
  // At least ~4 CTAs per SM: more CTAs per column first, then smaller CTAs (down to 32
  // unit pairs), which also spread more evenly over the SMs.
  const long long target = 4LL * sm_count();
  while (ncols * S < target && 2 * S <= smax) {
    if (2 * S * p.T <= p.M) S *= 2;
    else if (p.T > 32) { p.T /= 2; S *= 2; }
    else break;
  }
  p.S = (int)S;
  p.G = p.M / (S * p.T);
  return p;
}

int pairwise_stats_parts(long long Nf, long long ncols, int smax) { return pw_shape(Nf, ncols, smax).S; }

int pairwise_stats_launch(const float* const* d_mats, const float* base, long long nb, long long Nf,
                          long long Nrb, float* part, int smax, double* d_ms, int snr_mode,
                          double snr, cudaStream_t s, float* leafmax) {
  const long long ncols = nb * Nrb;
  FDR_CHECK_ARG(ncols <= 65535, "fdrstats: at most 65535 columns in total");
  FDR_CHECK_ARG(smax >= 1 && smax <= (1 << 20), "fdrstats: bad partial count");
  const PwShape p = pw_shape(Nf, ncols, smax);
  float* part_sum = part;
  float* part_sq = part + ncols * p.S;
  const dim3 grid((unsigned)p.S, (unsigned)ncols);
  const int threads = std::max(32, 2 * p.T);  // whole warps: the leaf exchange is a warp shuffle
  // leaves of exactly 1024 elements (n a power of two >= 2^15, at least 16 units per CTA)
  const int leaves1024 = (is_pow2(Nf) && Nf >= (1LL << 15) && p.T >= 16) ? 1 : 0;
  const size_t smem = leaves1024 ? sizeof(float) * (threads / 32) * 32 * 33 : 0;
  pw_units_kernel<false><<<grid, threads, smem, s>>>(d_mats, base, Nf, Nrb, p.bits, p.T, p.G, p.S, nullptr,
                                                    part_sum, leaves1024, leafmax);
  FDR_LAUNCH_CHECK("pw_units_kernel<sum>");
  pw_units_kernel<true><<<grid, threads, smem, s>>>(d_mats, base, Nf, Nrb, p.bits, p.T, p.G, p.S, part_sum,
                                                   part_sq, leaves1024, nullptr);
  FDR_LAUNCH_CHECK("pw_units_kernel<abs2>");
  pw_finalize_kernel<<<1, 256, 0, s>>>(part_sum, part_sq, ncols, p.S, Nf, snr_mode, snr, d_ms);
  FDR_LAUNCH_CHECK("pw_finalize_kernel");
  return FDR_OK;
}

// m = mean(column 0); s = min over columns of sqrt(corrected variance).
__global__ void stats_finalize_kernel(const double* __restrict__ acc, long long ncols,
                                      long long Nf, double* __restrict__ ms) {
  __shared__ double smin[256];
  double best = INFINITY;
  bool nan = false;
  for (long long c = threadIdx.x; c < ncols; c += blockDim.x) {
    const double s1 = acc[2 * c], s2 = acc[2 * c + 1];
    const double mean = s1 / (double)Nf;
    double var = (s2 - s1 * mean) / (double)(Nf - 1);
    if (var < 0) var = 0;
    const double sd = sqrt(var);
    if (isnan(sd)) nan = true;
    best = fmin(best, sd);
  }
  if (nan) best = NAN;
  smin[threadIdx.x] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = INFINITY;
    bool anynan = false;
    for (int i = 0; i < blockDim.x; ++i) {
      if (isnan(smin[i])) anynan = true;
      b = fmin(b, smin[i]);
    }
    ms[0] = acc[0] / (double)Nf;
    ms[1] = anynan ? NAN : b;
  }
}

__global__ void normalize_kernel(float* const* __restrict__ mats, long long Nf, long long Nrb,
                                 long long nb, float m, float s) {
  const long long per = Nf * Nrb;
  const long long total = per * nb;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long b = e / per, r = e - b * per;
    float* x = mats[b] + r;
    *x = __fdiv_rn(__fsub_rn(*x, m), s);
  }
}

// Ordered proto-hit compaction.  Tile t of matrix b covers linear (column-major)
// elements [t*kHitTile, (t+1)*kHitTile) of that matrix; tiles are numbered matrix-major.
// The threshold is thr_host, or *d_thr when d_thr is not NULL (computed on the device).

// Pass 1: counts[tile] = number of elements >= threshold (16-byte loads).
__global__ void __launch_bounds__(kHitThreads)
protohits_count_kernel(const float* const* __restrict__ mats, long long Nf, long long Nrb,
                       long long tiles_per_mat, double thr_host, const double* __restrict__ d_thr,
                       long long* __restrict__ counts) {
  const long long tile = blockIdx.x;
  const long long b = tile / tiles_per_mat, tt = tile - b * tiles_per_mat;
  const long long per = Nf * Nrb;
  const float* x = mats[b];
  const double thr = d_thr ? *d_thr : thr_host;
  const long long e0 = tt * kHitTile;
  int c = 0;
  const bool aligned = ((reinterpret_cast<uintptr_t>(x) & 15) == 0);
#pragma unroll
  for (int r = 0; r < kHitRounds / 4; ++r) {
    const long long e = e0 + 4 * ((long long)r * kHitThreads + threadIdx.x);
    if (aligned && e + 3 < per) {
      const float4 v = __ldcs(reinterpret_cast<const float4*>(x + e));
      c += ((double)v.x >= thr) + ((double)v.y >= thr) + ((double)v.z >= thr) + ((double)v.w >= thr);
    } else {
      for (int u = 0; u < 4; ++u)
        if (e + u < per) c += ((double)x[e + u] >= thr);
    }
  }
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  __shared__ int wc[kHitThreads / 32];
  if ((threadIdx.x & 31) == 0) wc[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long t = 0;
    for (int i = 0; i < kHitThreads / 32; ++i) t += wc[i];
    counts[tile] = t;
  }
}

// Pass 2: write the hits of each tile at offsets[tile], in column-major order.  Tiles
// without hits return at once, so this pass re-reads only the tiles that hold hits.  CTA 0
// also stores the total and the threshold in result[0..1] (mapped host memory).
__global__ void __launch_bounds__(kHitThreads)
protohits_write_kernel(const float* const* __restrict__ mats, long long Nf, long long Nrb,
                       long long tiles_per_mat, long long ntiles, double thr_host,
                       const double* __restrict__ d_thr, const long long* __restrict__ offsets,
                       long long* __restrict__ hits, long long cap, long long* __restrict__ result) {
  const long long tile = blockIdx.x;
  if (tile == 0 && threadIdx.x == 0) {  // the total and the threshold, for the host
    result[0] = offsets[ntiles];
    result[1] = __double_as_longlong(d_thr ? *d_thr : thr_host);
  }
  const long long start = offsets[tile];
  if (offsets[tile + 1] == start || start >= cap) return;  // uniform over the CTA
  const long long b = tile / tiles_per_mat, tt = tile - b * tiles_per_mat;
  const long long per = Nf * Nrb;
  const float* x = mats[b];
  const double thr = d_thr ? *d_thr : thr_host;
  const long long e0 = tt * kHitTile;
  __shared__ int wcount[kHitThreads / 32];
  __shared__ long long running;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) running = start;
  __syncthreads();
  for (int r = 0; r < kHitRounds; ++r) {
    const long long e = e0 + (long long)r * kHitThreads + threadIdx.x;
    const bool hit = (e < per) && ((double)x[e] >= thr);
    const unsigned bal = __ballot_sync(0xffffffffu, hit);
    if (lane == 0) wcount[w] = __popc(bal);
    __syncthreads();
    long long before = running;
    for (int i = 0; i < w; ++i) before += wcount[i];
    before += __popc(bal & ((1u << lane) - 1u));
    if (hit && before < cap && FDR_DBG_OK(before >= 0)) {
      const long long j = e / Nf, i = e - j * Nf;
      hits[2 * before] = i;
      hits[2 * before + 1] = b * Nrb + j;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      long long tot = 0;
      for (int i = 0; i < kHitThreads / 32; ++i) tot += wcount[i];
      running += tot;
    }
    __syncthreads();
  }
}

// fdrdenormalize (fdrutils.jl:104-107) from float64 moments: thr = snr*s + m with m and s
// rounded to Float32 (the reference's types), in Float64 (FDR_SNR_F64) or Float32
// (FDR_SNR_F32) arithmetic.
__global__ void threshold_kernel(const double* __restrict__ ms, int snr_mode, double snr,
                                 double* __restrict__ thr) {
  const float m = (float)ms[0], s = (float)ms[1];
  thr[0] = snr_mode == FDR_SNR_F32 ? (double)__fadd_rn(__fmul_rn((float)snr, s), m)
                                   : snr * (double)s + (double)m;
}

// Exclusive scan of counts (single CTA of whole warps); offsets[n] = total.  Each thread sums a
// contiguous chunk, the chunk sums are scanned with warp shuffles (within and then across the
// warps), and each thread writes its chunk's offsets.
__global__ void scan_counts_kernel(const long long* __restrict__ counts, long long n,
                                   long long* __restrict__ offsets) {
  __shared__ long long wsum[32];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5, nw = blockDim.x >> 5;
  const long long per = (n + blockDim.x - 1) / blockDim.x;
  const long long a = min(n, (long long)t * per), bnd = min(n, a + per);
  long long s = 0;
  for (long long i = a; i < bnd; ++i) s += counts[i];
  long long x = s;  // inclusive scan over the warp
  for (int o = 1; o < 32; o <<= 1) {
    const long long y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[w] = x;
  __syncthreads();
  if (w == 0) {
    long long y = lane < nw ? wsum[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const long long z = __shfl_up_sync(0xffffffffu, y, o);
      if (lane >= o) y += z;
    }
    wsum[lane] = y;
  }
  __syncthreads();
  long long run = x - s + (w > 0 ? wsum[w - 1] : 0);
  if (t == (int)blockDim.x - 1) offsets[n] = run + s;
  for (long long i = a; i < bnd; ++i) {
    offsets[i] = run;
    run += counts[i];
  }
}

static unsigned grid_1d(long long total) {
  long long b = cdiv(total, 256);
  long long cap = (long long)sm_count() * 16;
  return (unsigned)std::max(1LL, std::min(b, cap));
}

// Device copy of a host array of nb matrix pointers.
int upload_ptrs(const void* const* host, int64_t nb, void*** dev, cudaStream_t s) {
  FDR_TRY(scratch_alloc((void**)dev, sizeof(void*) * nb, s));
  const int st = upload_words(*dev, host, sizeof(void*) * nb, s);
  if (st != FDR_OK) scratch_free(*dev, s);
  return st;
}

// fdrstats in Float32 pairwise order into the device array ms[3] = (m, s, threshold) (no host
// synchronisation); the threshold is fdrdenormalize(snr, m, s) for snr_mode FDR_SNR_F64 /
// FDR_SNR_F32 (unused otherwise).
int stats_device(const float* const* d_mats, int64_t nb, int64_t Nf, int64_t Nrb, double* d_ms,
                 int snr_mode, double snr, cudaStream_t s) {
  const long long ncols = nb * Nrb;
  const int smax = 256;
  const int S = pairwise_stats_parts(Nf, ncols, smax);
  float* part = nullptr;
  FDR_TRY(scratch_alloc((void**)&part, sizeof(float) * 2 * ncols * S, s));
  const int st = pairwise_stats_launch(d_mats, nullptr, nb, Nf, Nrb, part, smax, d_ms, snr_mode, snr, s);
  scratch_free(part, s);
  return st;
}

// Per-column float64 sum and sum of squares of one Nf x ncols matrix, added into acc.
__global__ void __launch_bounds__(kRedThreads)
moments_accumulate_kernel(const float* __restrict__ x, long long Nf, double* __restrict__ acc) {
  const long long col = blockIdx.y;
  const float* c = x + col * Nf;
  double s1 = 0.0, s2 = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < Nf;
       i += (long long)gridDim.x * blockDim.x) {
    const double v = (double)c[i];
    s1 += v;
    s2 += v * v;
  }
  for (int o = 16; o > 0; o >>= 1) {
    s1 += __shfl_down_sync(0xffffffffu, s1, o);
    s2 += __shfl_down_sync(0xffffffffu, s2, o);
  }
  __shared__ double r1[kRedThreads / 32], r2[kRedThreads / 32];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { r1[w] = s1; r2[w] = s2; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int i = 0; i < kRedThreads / 32; ++i) { a += r1[i]; b += r2[i]; }
    atomicAdd(acc + 2 * col, a);
    atomicAdd(acc + 2 * col + 1, b);
  }
}

int moments_accumulate(const float* x, long long Nf, long long ncols, double* acc, cudaStream_t s) {
  FDR_CHECK_ARG(ncols <= 65535, "statistics: at most 65535 columns");
  const long long rows_blocks = std::max<long long>(1, std::min<long long>(cdiv(Nf, kRedThreads * 8),
      std::max<long long>(1, (long long)sm_count() * 8 / std::max<long long>(1, ncols))));
  moments_accumulate_kernel<<<dim3((unsigned)rows_blocks, (unsigned)ncols), kRedThreads, 0, s>>>(x, Nf, acc);
  FDR_LAUNCH_CHECK("moments_accumulate_kernel");
  return FDR_OK;
}

int stats_finalize_launch(const double* acc, long long ncols, long long Nf, double* d_ms,
                          cudaStream_t s) {
  stats_finalize_kernel<<<1, 256, 0, s>>>(acc, ncols, Nf, d_ms);
  FDR_LAUNCH_CHECK("stats_finalize_kernel");
  return FDR_OK;
}

int threshold_launch(const double* d_ms, int snr_mode, double snr, double* d_thr, cudaStream_t s) {
  threshold_kernel<<<1, 1, 0, s>>>(d_ms, snr_mode, snr, d_thr);
  FDR_LAUNCH_CHECK("threshold_kernel");
  return FDR_OK;
}

// Common end of the proto-hit searches: checks the launches, waits for the stream and reads
// the total and the threshold that the write kernel stored in the mapped words `h`, frees
// the scratch block and reports capacity.
static int hits_finish(const volatile long long* h, bool has_thr, double thr_host, int64_t capacity,
                       int64_t* count, double* thr_used, void* scratch, cudaStream_t s) {
  int st = FDR_OK;
  cudaError_t e = cudaPeekAtLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) st = cuda_status(e, "findprotohits");
  scratch_free(scratch, s);
  if (st != FDR_OK) return st;
  const long long total = h[0];
  double thr = thr_host;
  if (has_thr) {
    const long long bits = h[1];
    memcpy(&thr, &bits, sizeof(double));
  }
  *count = total;
  if (thr_used) *thr_used = thr;
  if (total > capacity) {
    set_error(FDR_ERR_CAPACITY, "findprotohits: %lld hits exceed capacity %lld", total,
              (long long)capacity);
    return FDR_ERR_CAPACITY;
  }
  return FDR_OK;
}

// Count, scan and ordered write of the proto-hits of nb device matrices (d_mats: device
// array of pointers).  Synchronises s; *count receives the total.  *thr_used receives the
// threshold (read back from d_thr when given).
int hits_run(const float* const* d_mats, int64_t nb, int64_t Nf, int64_t Nrb, double thr_host,
             const double* d_thr, int64_t* hits, int64_t capacity, int64_t* count,
             double* thr_used, cudaStream_t s) {
  const long long per = Nf * Nrb;
  const long long tiles_per_mat = cdiv(per, kHitTile);
  const long long ntiles = tiles_per_mat * nb;
  FDR_CHECK_ARG(ntiles < (1LL << 31), "findprotohits: too many elements");
  if (capacity > 0) FDR_TRY(device_view(hits, (void**)&hits, "findprotohits: hit buffer"));
  void *res_host = nullptr, *res_dev = nullptr;
  FDR_TRY(pinned_staging(2 * sizeof(long long), &res_host, &res_dev));
  long long* counts = nullptr;  // ntiles counts, ntiles+1 offsets, then the threshold copy
  FDR_TRY(scratch_alloc((void**)&counts, sizeof(long long) * (2 * ntiles + 2), s));
  long long* offsets = counts + ntiles;
  protohits_count_kernel<<<(unsigned)ntiles, kHitThreads, 0, s>>>(d_mats, Nf, Nrb, tiles_per_mat,
                                                                 thr_host, d_thr, counts);
  scan_counts_kernel<<<1, 1024, 0, s>>>(counts, ntiles, offsets);
  protohits_write_kernel<<<(unsigned)ntiles, kHitThreads, 0, s>>>(
      d_mats, Nf, Nrb, tiles_per_mat, ntiles, thr_host, d_thr, offsets, (long long*)hits, capacity,
      static_cast<long long*>(res_dev));
  count_launch(3);
  return hits_finish(static_cast<const volatile long long*>(res_host), d_thr != nullptr, thr_host,
                     capacity, count, thr_used, counts, s);
}

// ------------------------------------------------------------------------------------
// Proto-hits after fdrstats (the snr path): the first statistics pass leaves the maximum of
// every pairwise leaf, so once the threshold is known only the leaves whose maximum reaches
// it are read again.  Leaf slots are numbered column by column, and within a column in
// element order (unit u's first leaf is slot 2u, its second 2u + 1), so writing the hits of
// the slots in slot order gives findall's column-major order.
// ------------------------------------------------------------------------------------
constexpr int kSlotThreads = 256;

// Element range [lo, lo + len) of leaf slot `slot` (2u + h) of a column of n elements.
__device__ __forceinline__ void pw_slot_range(long long n, int bits, long long slot, long long& lo,
                                              long long& len) {
  long long ulo, ulen;
  pw_unit_range(n, bits, slot >> 1, ulo, ulen);
  const bool two = ulen > kPwLeaf;
  const long long c = two ? (ulen + 1) >> 1 : ulen;
  if ((slot & 1) == 0) { lo = ulo; len = c; }
  else { lo = ulo + c; len = two ? ulen - c : 0; }
}

// The elements of a leaf slot (at most 1024) into the lanes' registers: v[i] = x[lane + 32 i].
// All 32 loads of a lane are issued before any is used, so a slot costs one memory latency.
__device__ __forceinline__ void slot_load(const float* __restrict__ x, long long lo, long long len,
                                          long long Nf, int lane, float (&v)[32]) {
#pragma unroll
  for (int i = 0; i < 32; ++i) {
    const long long e = lane + 32 * i;
    v[i] = (e < len && FDR_DBG_OK(lo + e < Nf)) ? __ldg(x + e) : 0.f;
  }
}

// One thread per leaf slot: slot_count = hits in the slot (0 without reading it when its
// maximum is below the threshold); block_total[block] = the CTA's sum.  The CTA's gated
// slots are listed in shared memory and dealt out to its warps, one slot per warp at a time.
__global__ void __launch_bounds__(kSlotThreads)
protohits_slot_count_kernel(const float* const* __restrict__ mats, long long Nf, long long Nrb, int bits,
                            long long nslots, const double* __restrict__ d_thr,
                            const float* __restrict__ leafmax, int* __restrict__ slot_count,
                            long long* __restrict__ block_total) {
  __shared__ int list[kSlotThreads];
  __shared__ int nlist, total;
  const long long slot0 = (long long)blockIdx.x * kSlotThreads;
  const long long slot = slot0 + threadIdx.x;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const double thr = *d_thr;
  if (threadIdx.x == 0) nlist = total = 0;
  __syncthreads();
  const bool gate = slot < nslots && (double)leafmax[slot] >= thr;
  if (gate) list[atomicAdd(&nlist, 1)] = threadIdx.x;
  else if (slot < nslots) slot_count[slot] = 0;
  __syncthreads();
  for (int k = w; k < nlist; k += kSlotThreads / 32) {
    const long long sl = slot0 + list[k];
    const long long col = sl >> (bits + 1);
    long long lo, len;
    pw_slot_range(Nf, bits, sl - (col << (bits + 1)), lo, len);
    float v[32];
    slot_load(pw_column(mats, nullptr, Nf, Nrb, col) + lo, lo, len, Nf, lane, v);
    int c = 0;
#pragma unroll
    for (int i = 0; i < 32; ++i) c += (lane + 32 * i < len) && ((double)v[i] >= thr);
    c = (int)__reduce_add_sync(0xffffffffu, (unsigned)c);
    if (lane == 0) {
      slot_count[sl] = c;
      atomicAdd(&total, c);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) block_total[blockIdx.x] = total;
}

// Writes the hits of each slot with slot_count > 0 at block_off[block] + the exclusive sum of
// the CTA's earlier slot counts, in element order within the slot (a warp ballot per 32
// elements), one 16-byte (i, j) store per hit when the buffer allows (consecutive hits of a
// ballot land in one contiguous run, which also suits a buffer in mapped host memory).  The
// CTA's slots with hits are dealt out to its warps.  CTAs without hits, or starting past the
// capacity, return at once; CTA 0 first stores the total and the threshold in result[0..1].
__global__ void __launch_bounds__(kSlotThreads)
protohits_slot_write_kernel(const float* const* __restrict__ mats, long long Nf, long long Nrb, int bits,
                            long long nslots, long long nblk, const double* __restrict__ d_thr,
                            const int* __restrict__ slot_count, const long long* __restrict__ block_off,
                            long long* __restrict__ hits, long long cap, long long* __restrict__ result) {
  const double thr = *d_thr;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    result[0] = block_off[nblk];
    result[1] = __double_as_longlong(thr);
  }
  const long long start = block_off[blockIdx.x];
  if (block_off[blockIdx.x + 1] == start || start >= cap) return;  // uniform over the CTA
  __shared__ int wtot[kSlotThreads / 32];
  __shared__ int list[kSlotThreads];
  __shared__ long long offs[kSlotThreads];
  __shared__ int nlist;
  const long long slot0 = (long long)blockIdx.x * kSlotThreads;
  const long long slot = slot0 + threadIdx.x;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int cnt = slot < nslots ? slot_count[slot] : 0;
  int incl = cnt;  // inclusive scan over the warp
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) wtot[w] = incl;
  if (threadIdx.x == 0) nlist = 0;
  __syncthreads();
  long long my_off = start + incl - cnt;
  for (int i = 0; i < w; ++i) my_off += wtot[i];
  if (cnt > 0) {
    const int k = atomicAdd(&nlist, 1);
    list[k] = threadIdx.x;
    offs[k] = my_off;
  }
  __syncthreads();
  const bool vec = (reinterpret_cast<uintptr_t>(hits) & 15) == 0;
  for (int k = w; k < nlist; k += kSlotThreads / 32) {
    const long long sl = slot0 + list[k];
    long long base = offs[k];
    if (base >= cap) continue;  // uniform over the warp
    const long long col = sl >> (bits + 1);
    long long lo, len;
    pw_slot_range(Nf, bits, sl - (col << (bits + 1)), lo, len);
    float v[32];
    slot_load(pw_column(mats, nullptr, Nf, Nrb, col) + lo, lo, len, Nf, lane, v);
#pragma unroll
    for (int i = 0; i < 32; ++i) {
      const long long e = lane + 32 * i;
      const bool hit = e < len && (double)v[i] >= thr;
      const unsigned bal = __ballot_sync(0xffffffffu, hit);
      if (bal == 0u) continue;  // uniform over the warp
      const long long pos = base + __popc(bal & ((1u << lane) - 1u));
      if (hit && pos < cap && FDR_DBG_OK(pos >= 0)) {
        if (vec) {
          *reinterpret_cast<longlong2*>(hits + 2 * pos) = make_longlong2(lo + e, col);
        } else {
          hits[2 * pos] = lo + e;
          hits[2 * pos + 1] = col;
        }
      }
      base += __popc(bal);
    }
  }
}

// fdrstats (Float32 pairwise) into d_ms = (m, s, threshold), the threshold fdrdenormalize(snr,
// m, s) in snr_mode's type, then the proto-hits at or above it through the leaf gate.
// Synchronises s; returns like hits_run.
int snr_protohits_run(const float* const* d_mats, int64_t nb, int64_t Nf, int64_t Nrb, double* d_ms,
                      int snr_mode, double snr, int64_t* hits, int64_t capacity, int64_t* count,
                      double* thr_used, cudaStream_t s) {
  const long long ncols = nb * Nrb;
  FDR_CHECK_ARG(ncols <= 65535, "fdrstats: at most 65535 columns in total");
  const int smax = 256;
  const PwShape p = pw_shape(Nf, ncols, smax);
  const long long nslots = ncols * 2 * p.M;
  const long long nblk = cdiv(nslots, kSlotThreads);
  FDR_CHECK_ARG(nblk < (1LL << 31), "findprotohits: too many leaves");
  if (capacity > 0) FDR_TRY(device_view(hits, (void**)&hits, "findprotohits: hit buffer"));
  void *res_host = nullptr, *res_dev = nullptr;
  FDR_TRY(pinned_staging(2 * sizeof(long long), &res_host, &res_dev));
  // one scratch block: block totals and offsets (int64), partial sums, leaf maxima, slot counts
  const size_t b_tot = sizeof(long long) * (2 * nblk + 1);
  const size_t b_part = sizeof(float) * 2 * ncols * p.S;
  const size_t b_max = sizeof(float) * nslots;
  const size_t b_cnt = sizeof(int) * nslots;
  char* buf = nullptr;
  FDR_TRY(scratch_alloc((void**)&buf, b_tot + b_part + b_max + b_cnt + 64, s));
  long long* block_total = reinterpret_cast<long long*>(buf);
  long long* block_off = block_total + nblk;
  float* part = reinterpret_cast<float*>(buf + ((b_tot + 15) & ~size_t(15)));
  float* leafmax = part + 2 * ncols * p.S;
  int* slot_count = reinterpret_cast<int*>(leafmax + nslots);
  int st = pairwise_stats_launch(d_mats, nullptr, nb, Nf, Nrb, part, smax, d_ms, snr_mode, snr, s,
                                 leafmax);
  if (st != FDR_OK) { scratch_free(buf, s); return st; }
  const double* d_thr = d_ms + 2;
  protohits_slot_count_kernel<<<(unsigned)nblk, kSlotThreads, 0, s>>>(
      d_mats, Nf, Nrb, p.bits, nslots, d_thr, leafmax, slot_count, block_total);
  scan_counts_kernel<<<1, 1024, 0, s>>>(block_total, nblk, block_off);
  protohits_slot_write_kernel<<<(unsigned)nblk, kSlotThreads, 0, s>>>(
      d_mats, Nf, Nrb, p.bits, nslots, nblk, d_thr, slot_count, block_off, (long long*)hits, capacity,
      static_cast<long long*>(res_dev));
  count_launch(3);
  return hits_finish(static_cast<const volatile long long*>(res_host), true, snr, capacity, count,
                     thr_used, buf, s);
}

}  // namespace fdr

using namespace fdr;

extern "C" {

int fdr_stats(const float* const* fdrs, int64_t nb, int64_t Nf, int64_t Nrb, double* m,
              double* s_out, fdr_stream_t stream) {
  FDR_CHECK_ARG(fdrs && m && s_out, "fdrstats: NULL argument");
  FDR_CHECK_ARG(nb >= 1 && Nf >= 1 && Nrb >= 1, "fdrstats: bad sizes");
  for (int64_t b = 0; b < nb; ++b) FDR_CHECK_ARG(fdrs[b] != nullptr, "fdrstats: matrix %lld is NULL", (long long)b);
  cudaStream_t s = (cudaStream_t)stream;
  // The finalize kernel writes (m, s) straight into mapped pinned words: no device-to-host
  // copy that would queue behind the copy engine's other work.
  void *ms_host = nullptr, *ms_dev = nullptr;
  FDR_TRY(pinned_staging(3 * sizeof(double), &ms_host, &ms_dev));
  void** d_mats = nullptr;
  FDR_TRY(upload_ptrs((const void* const*)fdrs, nb, &d_mats, s));
  int st = stats_device((const float* const*)d_mats, nb, Nf, Nrb, static_cast<double*>(ms_dev), 0,
                        0.0, s);
  if (st == FDR_OK) {
    const cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = cuda_status(e, "fdrstats");
  }
  scratch_free(d_mats, s);
  const volatile double* h = static_cast<const volatile double*>(ms_host);
  *m = st == FDR_OK ? h[0] : 0.0;
  *s_out = st == FDR_OK ? h[1] : 0.0;
  return st;
}

int fdr_normalize(float* const* fdrs, int64_t nb, int64_t Nf, int64_t Nrb, float m, float s_,
                  fdr_stream_t stream) {
  FDR_CHECK_ARG(fdrs != nullptr, "fdrnormalize!: NULL argument");
  FDR_CHECK_ARG(nb >= 1 && Nf >= 1 && Nrb >= 1, "fdrnormalize!: bad sizes");
  cudaStream_t s = (cudaStream_t)stream;
  void** d_mats = nullptr;
  FDR_TRY(upload_ptrs((const void* const*)fdrs, nb, &d_mats, s));
  normalize_kernel<<<grid_1d(nb * Nf * Nrb), 256, 0, s>>>((float* const*)d_mats, Nf, Nrb, nb, m, s_);
  FDR_LAUNCH_CHECK("normalize_kernel");
  scratch_free(d_mats, s);
  return FDR_OK;
}

int fdr_findprotohits(const float* const* fdrs, int64_t nb, int64_t Nf, int64_t Nrb,
                      double threshold, int snr, int64_t* hits, int64_t capacity,
                      int64_t* count, double* threshold_used, fdr_stream_t stream) {
  FDR_CHECK_ARG(fdrs && count, "findprotohits: NULL argument");
  FDR_CHECK_ARG(nb >= 1 && Nf >= 1 && Nrb >= 1, "findprotohits: bad sizes");
  FDR_CHECK_ARG(capacity >= 0 && (capacity == 0 || hits != nullptr), "findprotohits: bad hit buffer");
  FDR_CHECK_ARG(snr == 0 || snr == FDR_SNR_F64 || snr == FDR_SNR_F32,
                "findprotohits: snr must be 0, FDR_SNR_F64 or FDR_SNR_F32 (got %d)", snr);
  for (int64_t b = 0; b < nb; ++b) FDR_CHECK_ARG(fdrs[b] != nullptr, "findprotohits: matrix %lld is NULL", (long long)b);
  cudaStream_t s = (cudaStream_t)stream;
  *count = 0;
  void** d_mats = nullptr;
  double* d_ms = nullptr;  // m, s, threshold
  FDR_TRY(upload_ptrs((const void* const*)fdrs, nb, &d_mats, s));
  int st = FDR_OK;
  if (snr) {
    // fdrdenormalize(snr, fdrs) = snr*s + m with the reference's Float32 m and s
    st = scratch_alloc((void**)&d_ms, 3 * sizeof(double), s);
    if (st == FDR_OK)
      st = snr_protohits_run((const float* const*)d_mats, nb, Nf, Nrb, d_ms, snr, threshold, hits,
                             capacity, count, threshold_used, s);
  } else {
    st = hits_run((const float* const*)d_mats, nb, Nf, Nrb, threshold, nullptr, hits, capacity,
                  count, threshold_used, s);
  }
  scratch_free(d_ms, s);
  scratch_free(d_mats, s);
  return st;
}

}  // extern "C"
