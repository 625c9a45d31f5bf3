// Clustering of proto-hits into hits (fdr_cluster_protohits).
//
// findprotohits (fdrutils.jl:148-169) returns every FDR cell above threshold; one drifting
// signal is seen at several neighbouring (frequency, drift rate) cells, and the step after
// it, "detection of unique signals ... within the proto-hits" (the reference's README.md:57-66), lives
// outside the reference (DopplerDriftSearchTools.jl).  This is that step on the device:
// the connected components of the proto-hits under a (di, dj) neighbourhood (|Δi| <= di
// channels, |Δj| <= dj drift-rate columns, no wrap-around), with per-cluster counts,
// bounding boxes and the peak cell.
//
// Hits arrive as findprotohits writes them: zero-based (i, j) pairs in column-major order,
// i.e. sorted by key = j*Nf + i.  Union-find over hit indices: each hit looks up its
// forward neighbours (later keys) by binary search in the sorted keys and links the two
// roots, always hooking the larger index under the smaller, so every parent pointer points
// to a smaller index and every component's root is its first hit in column-major order.
// Cluster numbers follow that order; all per-cluster reductions are integer atomics
// (min, max, add, and max over (value, -index) packed into 64 bits), so the result does not
// depend on scheduling.
#include <climits>

#include "fdr_internal.cuh"

namespace fdr {

constexpr int kCluThreads = 256;
constexpr int kCasLimit = 1 << 20;  // retries of one link before reporting failure

__device__ __forceinline__ long long hit_key(const long long* hits, long long h, long long Nf) {
  return hits[2 * h + 1] * Nf + hits[2 * h];
}

__global__ void check_sorted_kernel(const long long* __restrict__ hits, long long n, long long Nf,
                                    long long Nj, int* __restrict__ err) {
  const long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (h >= n) return;
  const long long i = hits[2 * h], j = hits[2 * h + 1];
  if (i < 0 || i >= Nf || j < 0 || j >= Nj) atomicOr(err, 1);
  if (h > 0 && hit_key(hits, h - 1, Nf) >= j * Nf + i) atomicOr(err, 2);
}

__device__ __forceinline__ int uf_find(const volatile int* parent, int x) {
  // parent[x] < x for every non-root, so this walk ends after at most x steps
  int p = parent[x];
  while (p != x) {
    x = p;
    p = parent[x];
  }
  return x;
}

__global__ void init_parent_kernel(int* __restrict__ parent, long long n) {
  const long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (h < n) parent[h] = (int)h;
}

// Link hit h with every later hit within (di, dj).
__global__ void link_kernel(const long long* __restrict__ hits, long long n, long long Nf, int di,
                            int dj, int* parent, int* __restrict__ err) {
  const long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (h >= n) return;
  const long long i = hits[2 * h], j = hits[2 * h + 1];
  for (int dc = 0; dc <= dj; ++dc) {
    const long long lo_i = dc == 0 ? i + 1 : (i - di < 0 ? 0 : i - di);
    const long long hi_i = (i + di >= Nf) ? Nf - 1 : i + di;
    if (lo_i > hi_i) continue;
    const long long klo = (j + dc) * Nf + lo_i, khi = (j + dc) * Nf + hi_i;
    // first index g > h with key >= klo
    long long a = h + 1, b = n;
    while (a < b) {
      const long long m = (a + b) >> 1;
      if (hit_key(hits, m, Nf) < klo) a = m + 1; else b = m;
    }
    for (long long g = a; g < n && hit_key(hits, g, Nf) <= khi; ++g) {
      int x = (int)h, y = (int)g;
      int it = 0;
      for (; it < kCasLimit; ++it) {
        x = uf_find(parent, x);
        y = uf_find(parent, y);
        if (x == y) break;
        if (x > y) { const int t = x; x = y; y = t; }
        const int old = atomicCAS(parent + y, y, x);  // hook root y under the smaller root x
        if (old == y) break;
        y = old;
      }
      if (it == kCasLimit) atomicOr(err, 4);
    }
  }
}

// root[h]; flag[h] = 1 for roots.
__global__ void flatten_kernel(const int* __restrict__ parent, long long n, int* __restrict__ root,
                               int* __restrict__ flag) {
  const long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (h >= n) return;
  int x = (int)h;
  while (parent[x] != x) x = parent[x];
  root[h] = x;
  flag[h] = (x == (int)h);
}

// Exclusive scan of flag (n < 2^31) in three steps: per-block sums, a scan of those in one
// CTA, then per-block scans with the block offset.
__global__ void block_sums_kernel(const int* __restrict__ flag, long long n, int* __restrict__ bsum) {
  __shared__ int s[kCluThreads / 32];
  const long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  int v = h < n ? flag[h] : 0;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < kCluThreads / 32; ++w) t += s[w];
    bsum[blockIdx.x] = t;
  }
}

// result[0] receives the cluster total and result[1] the error flags that the earlier kernels
// of the stream left in *err (result is a mapped host word pair, read after the stream syncs).
__global__ void scan_bsums_kernel(int* __restrict__ bsum, long long nb, const int* __restrict__ err,
                                  long long* __restrict__ result) {
  // one CTA of kCluThreads threads; each thread scans a contiguous chunk
  __shared__ long long part[kCluThreads];
  const long long per = (nb + kCluThreads - 1) / kCluThreads;
  const long long a = threadIdx.x * per, b = min(nb, a + per);
  long long s = 0;
  for (long long k = a; k < b; ++k) s += bsum[k];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long run = 0;
    for (int k = 0; k < kCluThreads; ++k) { const long long v = part[k]; part[k] = run; run += v; }
    result[0] = run;
    result[1] = *err;
  }
  __syncthreads();
  long long run = part[threadIdx.x];
  for (long long k = a; k < b; ++k) { const int v = bsum[k]; bsum[k] = (int)run; run += v; }
}

__global__ void block_scan_kernel(const int* __restrict__ flag, long long n, const int* __restrict__ boff,
                                  int* __restrict__ cid) {
  __shared__ int s[kCluThreads / 32];
  const long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int v = h < n ? flag[h] : 0;
  int x = v;  // inclusive warp scan
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s[w] = x;
  __syncthreads();
  int before = 0;
  for (int k = 0; k < w; ++k) before += s[k];
  if (h < n) cid[h] = boff[blockIdx.x] + before + x - v;  // exclusive
}

__global__ void init_clusters_kernel(fdr_hit_cluster* __restrict__ cl, unsigned long long* __restrict__ peak,
                                     long long nc) {
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= nc) return;
  fdr_hit_cluster z;
  z.peak_i = z.peak_j = -1;
  z.peak_value = 0.f;
  z.reserved = 0;
  z.count = 0;
  z.i_min = z.j_min = LLONG_MAX;
  z.i_max = z.j_max = -1;
  z.first = -1;
  cl[c] = z;
  peak[c] = 0ull;
}

// Order-preserving map of a float to an unsigned 32-bit integer (NaN sorts above +inf).
__device__ __forceinline__ unsigned int ordered_bits(float v) {
  const unsigned int u = __float_as_uint(v);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__global__ void summarise_kernel(const long long* __restrict__ hits, long long n, long long Nf,
                                 const int* __restrict__ root, const int* __restrict__ cid,
                                 const float* const* __restrict__ fdrs, long long Nrb,
                                 long long capacity, long long* __restrict__ labels,
                                 fdr_hit_cluster* __restrict__ cl, unsigned long long* __restrict__ peak) {
  const long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (h >= n) return;
  const int r = root[h];
  const long long c = cid[r];
  if (labels) labels[h] = c;
  if (c >= capacity) return;
  const long long i = hits[2 * h], j = hits[2 * h + 1];
  fdr_hit_cluster* k = cl + c;
  atomicAdd((unsigned long long*)&k->count, 1ull);
  atomicMin((long long*)&k->i_min, i);
  atomicMax((long long*)&k->i_max, i);
  atomicMin((long long*)&k->j_min, j);
  atomicMax((long long*)&k->j_max, j);
  if (r == (int)h) k->first = h;
  float v = 0.f;
  if (fdrs) {
    const long long b = j / Nrb, jj = j - b * Nrb;
    v = fdrs[b][jj * Nf + i];
  }
  // larger value first; on ties the smaller hit index (earlier in column-major order)
  const unsigned long long key = ((unsigned long long)ordered_bits(v) << 32) |
                                 (unsigned long long)(0xFFFFFFFFu - (unsigned int)h);
  atomicMax(peak + c, key);
}

__global__ void finish_clusters_kernel(const long long* __restrict__ hits, long long nc,
                                       const unsigned long long* __restrict__ peak,
                                       const float* const* __restrict__ fdrs, long long Nf,
                                       long long Nrb, fdr_hit_cluster* __restrict__ cl) {
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const long long h = (long long)(0xFFFFFFFFu - (unsigned int)(peak[c] & 0xFFFFFFFFull));
  const long long i = hits[2 * h], j = hits[2 * h + 1];
  cl[c].peak_i = i;
  cl[c].peak_j = j;
  if (fdrs) {
    const long long b = j / Nrb, jj = j - b * Nrb;
    cl[c].peak_value = fdrs[b][jj * Nf + i];
  } else {
    cl[c].peak_value = __int_as_float(0x7fc00000);  // NaN: no FDR given
  }
}

}  // namespace fdr

using namespace fdr;

extern "C" {

int fdr_cluster_protohits(const int64_t* hits, int64_t nhits, int64_t Nf, int64_t Nj, int di, int dj,
                          const float* const* fdrs, int64_t nb, int64_t Nrb, int64_t* labels,
                          fdr_hit_cluster* clusters, int64_t capacity, int64_t* nclusters,
                          fdr_stream_t stream) {
  FDR_CHECK_ARG(nclusters != nullptr, "cluster_protohits: NULL count");
  *nclusters = 0;
  FDR_CHECK_ARG(nhits >= 0 && nhits < (1LL << 31), "cluster_protohits: nhits out of range");
  FDR_CHECK_ARG(nhits == 0 || hits != nullptr, "cluster_protohits: NULL hits");
  FDR_CHECK_ARG(Nf >= 1 && Nj >= 1 && Nj <= (INT64_MAX / Nf), "cluster_protohits: bad FDR size");
  FDR_CHECK_ARG(di >= 0 && dj >= 0, "cluster_protohits: negative neighbourhood");
  FDR_CHECK_ARG(capacity >= 0 && (capacity == 0 || clusters != nullptr), "cluster_protohits: bad cluster buffer");
  FDR_CHECK_ARG(fdrs == nullptr || (nb >= 1 && Nrb >= 1 && nb * Nrb == Nj),
                "cluster_protohits: the FDR matrices must cover the Nj drift-rate columns");
  if (fdrs)
    for (int64_t b = 0; b < nb; ++b)
      FDR_CHECK_ARG(fdrs[b] != nullptr, "cluster_protohits: matrix %lld is NULL", (long long)b);
  if (nhits == 0) return FDR_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const long long n = nhits;
  const unsigned grid = (unsigned)cdiv(n, kCluThreads);
  // scratch: parent, root, flag, cid (n ints each), block sums, then the error flags; the
  // total and the flags come back through mapped pinned words, not a device-to-host copy
  const size_t ints = 4 * (size_t)n + grid + 1;
  void *res_host = nullptr, *res_dev = nullptr;
  FDR_TRY(pinned_staging(2 * sizeof(long long), &res_host, &res_dev));
  int* w = nullptr;
  FDR_TRY(scratch_alloc((void**)&w, sizeof(int) * ints, s));
  int *parent = w, *root = w + n, *flag = w + 2 * n, *cid = w + 3 * n, *bsum = w + 4 * n;
  int* err = bsum + grid;
  int st = FDR_OK;
  void** d_mats = nullptr;
  unsigned long long* peak = nullptr;
  long long h_total = 0;
  int h_err = 0;
  cudaError_t e = cudaMemsetAsync(err, 0, sizeof(int), s);
  if (e != cudaSuccess) st = cuda_status(e, "cluster scratch");
  if (st == FDR_OK && fdrs) st = upload_ptrs((const void* const*)fdrs, nb, &d_mats, s);
  if (st == FDR_OK) {
    check_sorted_kernel<<<grid, kCluThreads, 0, s>>>((const long long*)hits, n, Nf, Nj, err);
    init_parent_kernel<<<grid, kCluThreads, 0, s>>>(parent, n);
    link_kernel<<<grid, kCluThreads, 0, s>>>((const long long*)hits, n, Nf, di, dj, parent, err);
    flatten_kernel<<<grid, kCluThreads, 0, s>>>(parent, n, root, flag);
    block_sums_kernel<<<grid, kCluThreads, 0, s>>>(flag, n, bsum);
    scan_bsums_kernel<<<1, kCluThreads, 0, s>>>(bsum, grid, err, static_cast<long long*>(res_dev));
    block_scan_kernel<<<grid, kCluThreads, 0, s>>>(flag, n, bsum, cid);
    count_launch(7);
    e = cudaPeekAtLastError();
    if (e != cudaSuccess) st = cuda_status(e, "cluster kernels");
  }
  if (st == FDR_OK) {
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = cuda_status(e, "cluster count");
  }
  if (st == FDR_OK) {
    const volatile long long* r = static_cast<const volatile long long*>(res_host);
    h_total = r[0];
    h_err = (int)r[1];
  }
  if (st == FDR_OK && (h_err & 3)) {
    set_error(FDR_ERR_INVALID_ARGUMENT, "cluster_protohits: hits must be in range and in column-major "
              "order without repeats (as findprotohits returns them)");
    st = FDR_ERR_INVALID_ARGUMENT;
  }
  if (st == FDR_OK && (h_err & 4)) {
    set_error(FDR_ERR_CUDA, "cluster_protohits: union-find did not settle");
    st = FDR_ERR_CUDA;
  }
  const long long nc = h_total;
  const long long keep = std::min<long long>(nc, capacity);
  if (st == FDR_OK && keep > 0)
    st = scratch_alloc((void**)&peak, sizeof(unsigned long long) * keep, s);
  if (st == FDR_OK) {
    if (keep > 0) {
      init_clusters_kernel<<<(unsigned)cdiv(keep, kCluThreads), kCluThreads, 0, s>>>(clusters, peak, keep);
      count_launch();
    }
    summarise_kernel<<<grid, kCluThreads, 0, s>>>((const long long*)hits, n, Nf, root, cid,
                                                  (const float* const*)d_mats, Nrb, keep,
                                                  (long long*)labels, clusters, peak);
    count_launch();
    if (keep > 0) {
      finish_clusters_kernel<<<(unsigned)cdiv(keep, kCluThreads), kCluThreads, 0, s>>>(
          (const long long*)hits, keep, peak, (const float* const*)d_mats, Nf, Nrb, clusters);
      count_launch();
    }
    e = cudaPeekAtLastError();
    if (e != cudaSuccess) st = cuda_status(e, "cluster summaries");
  }
  scratch_free(peak, s);
  scratch_free(d_mats, s);
  scratch_free(w, s);
  if (st != FDR_OK) return st;
  *nclusters = nc;
  if (nc > capacity) {
    set_error(FDR_ERR_CAPACITY, "cluster_protohits: %lld clusters exceed capacity %lld", nc,
              (long long)capacity);
    return FDR_ERR_CAPACITY;
  }
  return FDR_OK;
}

}  // extern "C"
