// FDR statistics, normalisation and proto-hit search (src/fdrutils.jl of
// FrequencyDriftRateTransforms.jl): fdrstats (:39-50), fdrnormalize! (:70-90),
// fdrdenormalize (:104-119), findprotohits (:148-169).
#include <math.h>
#include <string.h>

#include "fdr_internal.cuh"

namespace fdr {

constexpr int kRedThreads = 256;
constexpr int kHitThreads = 256;
constexpr int kHitRounds = 16;
constexpr long long kHitTile = (long long)kHitThreads * kHitRounds;  // elements per tile

// Per-column sum and sum of squares in float64.  grid.x: chunks of rows; grid.y: columns.
__global__ void __launch_bounds__(kRedThreads)
column_moments_kernel(const float* const* __restrict__ mats, long long Nf, long long Nrb,
                      double* __restrict__ acc /* [col][2] */) {
  const long long col = blockIdx.y;             // global column (matrix-major)
  const long long b = col / Nrb, j = col - b * Nrb;
  const float* x = mats[b] + j * Nf;
  double s1 = 0.0, s2 = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < Nf;
       i += (long long)gridDim.x * blockDim.x) {
    double v = (double)x[i];
    s1 += v;
    s2 += v * v;
  }
  __shared__ double r1[kRedThreads / 32], r2[kRedThreads / 32];
  for (int o = 16; o > 0; o >>= 1) {
    s1 += __shfl_down_sync(0xffffffffu, s1, o);
    s2 += __shfl_down_sync(0xffffffffu, s2, o);
  }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { r1[w] = s1; r2[w] = s2; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, c = 0.0;
    for (int i = 0; i < kRedThreads / 32; ++i) { a += r1[i]; c += r2[i]; }
    atomicAdd(acc + 2 * col, a);
    atomicAdd(acc + 2 * col + 1, c);
  }
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
// without hits return at once, so this pass re-reads only the tiles that hold hits.
__global__ void __launch_bounds__(kHitThreads)
protohits_write_kernel(const float* const* __restrict__ mats, long long Nf, long long Nrb,
                       long long tiles_per_mat, double thr_host, const double* __restrict__ d_thr,
                       const long long* __restrict__ offsets, long long* __restrict__ hits,
                       long long cap) {
  const long long tile = blockIdx.x;
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
    if (hit && before < cap) {
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

// thr = snr * Float32(s) + Float32(m)   (fdrdenormalize with the reference's Float32 m, s)
__global__ void threshold_kernel(const double* __restrict__ ms, double snr, double* __restrict__ thr) {
  thr[0] = snr * (double)(float)ms[1] + (double)(float)ms[0];
}

// Exclusive scan of counts (single CTA); offsets[n] = total.
__global__ void scan_counts_kernel(const long long* __restrict__ counts, long long n,
                                   long long* __restrict__ offsets) {
  __shared__ long long part[1024];
  const long long per = (n + blockDim.x - 1) / blockDim.x;
  const long long a = threadIdx.x * per, bnd = min(n, a + per);
  long long s = 0;
  for (long long i = a; i < bnd; ++i) s += counts[i];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long run = 0;
    for (int i = 0; i < blockDim.x; ++i) { long long v = part[i]; part[i] = run; run += v; }
    offsets[n] = run;
  }
  __syncthreads();
  long long run = part[threadIdx.x];
  for (long long i = a; i < bnd; ++i) { offsets[i] = run; run += counts[i]; }
}

static unsigned grid_1d(long long total) {
  long long b = cdiv(total, 256);
  long long cap = (long long)sm_count() * 16;
  return (unsigned)std::max(1LL, std::min(b, cap));
}

// Device copy of a host array of nb matrix pointers.
int upload_ptrs(const void* const* host, int64_t nb, void*** dev, cudaStream_t s) {
  FDR_TRY(scratch_alloc((void**)dev, sizeof(void*) * nb, s));
  FDR_CUDA(cudaMemcpyAsync(*dev, host, sizeof(void*) * nb, cudaMemcpyHostToDevice, s));
  return FDR_OK;
}

// Stats into a device array ms[2] (no host synchronisation).
int stats_device(const float* const* d_mats, int64_t nb, int64_t Nf, int64_t Nrb,
                        double* d_ms, cudaStream_t s) {
  const long long ncols = nb * Nrb;
  double* acc = nullptr;
  FDR_TRY(scratch_alloc((void**)&acc, sizeof(double) * 2 * ncols, s));
  FDR_CUDA(cudaMemsetAsync(acc, 0, sizeof(double) * 2 * ncols, s));
  const long long rows_blocks = std::max<long long>(1, std::min<long long>(cdiv(Nf, kRedThreads * 8),
      std::max<long long>(1, (long long)sm_count() * 8 / std::max<long long>(1, ncols))));
  FDR_CHECK_ARG(ncols <= 65535, "fdrstats: at most 65535 columns in total");
  column_moments_kernel<<<dim3((unsigned)rows_blocks, (unsigned)ncols), kRedThreads, 0, s>>>(
      d_mats, Nf, Nrb, acc);
  FDR_LAUNCH_CHECK("column_moments_kernel");
  stats_finalize_kernel<<<1, 256, 0, s>>>(acc, ncols, Nf, d_ms);
  FDR_LAUNCH_CHECK("stats_finalize_kernel");
  scratch_free(acc, s);
  return FDR_OK;
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

int threshold_launch(const double* d_ms, double snr, double* d_thr, cudaStream_t s) {
  threshold_kernel<<<1, 1, 0, s>>>(d_ms, snr, d_thr);
  FDR_LAUNCH_CHECK("threshold_kernel");
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
  long long* counts = nullptr;  // ntiles counts, ntiles+1 offsets, then the threshold copy
  FDR_TRY(scratch_alloc((void**)&counts, sizeof(long long) * (2 * ntiles + 2), s));
  long long* offsets = counts + ntiles;
  protohits_count_kernel<<<(unsigned)ntiles, kHitThreads, 0, s>>>(d_mats, Nf, Nrb, tiles_per_mat,
                                                                 thr_host, d_thr, counts);
  scan_counts_kernel<<<1, 1024, 0, s>>>(counts, ntiles, offsets);
  protohits_write_kernel<<<(unsigned)ntiles, kHitThreads, 0, s>>>(
      d_mats, Nf, Nrb, tiles_per_mat, thr_host, d_thr, offsets, (long long*)hits, capacity);
  count_launch(3);
  int st = FDR_OK;
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) st = cuda_status(e, "protohits kernels");
  long long total = 0;
  double thr = thr_host;
  if (st == FDR_OK) {
    e = cudaMemcpyAsync(&total, offsets + ntiles, sizeof(long long), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && d_thr)
      e = cudaMemcpyAsync(&thr, d_thr, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = cuda_status(e, "findprotohits count");
  }
  scratch_free(counts, s);
  if (st != FDR_OK) return st;
  *count = total;
  if (thr_used) *thr_used = thr;
  if (total > capacity) {
    set_error(FDR_ERR_CAPACITY, "findprotohits: %lld hits exceed capacity %lld", total,
              (long long)capacity);
    return FDR_ERR_CAPACITY;
  }
  return FDR_OK;
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
  void** d_mats = nullptr;
  double* d_ms = nullptr;
  FDR_TRY(upload_ptrs((const void* const*)fdrs, nb, &d_mats, s));
  FDR_TRY(scratch_alloc((void**)&d_ms, 2 * sizeof(double), s));
  int st = stats_device((const float* const*)d_mats, nb, Nf, Nrb, d_ms, s);
  double h[2] = {0, 0};
  if (st == FDR_OK) {
    cudaError_t e = cudaMemcpyAsync(h, d_ms, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = cuda_status(e, "fdrstats copy");
  }
  scratch_free(d_ms, s);
  scratch_free(d_mats, s);
  *m = h[0];
  *s_out = h[1];
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
  for (int64_t b = 0; b < nb; ++b) FDR_CHECK_ARG(fdrs[b] != nullptr, "findprotohits: matrix %lld is NULL", (long long)b);
  cudaStream_t s = (cudaStream_t)stream;
  *count = 0;
  void** d_mats = nullptr;
  double* d_ms = nullptr;  // m, s, threshold
  FDR_TRY(upload_ptrs((const void* const*)fdrs, nb, &d_mats, s));
  int st = FDR_OK;
  if (snr) {
    st = scratch_alloc((void**)&d_ms, 3 * sizeof(double), s);
    // fdrdenormalize(snr, fdrs) = snr*s + m with the reference's Float32 m and s
    if (st == FDR_OK) st = stats_device((const float* const*)d_mats, nb, Nf, Nrb, d_ms, s);
    if (st == FDR_OK) st = threshold_launch(d_ms, threshold, d_ms + 2, s);
  }
  if (st == FDR_OK)
    st = hits_run((const float* const*)d_mats, nb, Nf, Nrb, threshold, snr ? d_ms + 2 : nullptr,
                  hits, capacity, count, threshold_used, s);
  scratch_free(d_ms, s);
  scratch_free(d_mats, s);
  return st;
}

}  // extern "C"
