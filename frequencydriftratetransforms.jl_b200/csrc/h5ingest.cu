// Decoding of bitshuffle/LZ4-filtered HDF5 chunks: the storage of rawspec's HDF5
// filterbank products, which test/heavytests.jl:11-14 of FrequencyDriftRateTransforms.jl
// reads through HDF5.jl and H5Zbitshuffle.jl (HDF5 filter 32008).
//
// A chunk filtered by bitshuffle with LZ4 compression is
//   8 bytes  big-endian: uncompressed chunk size in bytes
//   4 bytes  big-endian: block size in bytes (a multiple of 8 elements)
//   per block of block-size bytes (the last block holds the remaining whole groups of 8
//   elements): 4 bytes big-endian compressed size, then one LZ4 block
//   the remaining (elements mod 8) elements, stored raw.
// Each decompressed block holds its n elements bit-transposed: bit k of byte j of element e
// is bit (e mod 8) of byte (8 j + k) * (n / 8) + e / 8 of the block (byte j = 0 is the least
// significant byte of the little-endian element, bit k = 0 its least significant bit).
//
// The host functions here decompress (LZ4 block format: sequences of a token, literal bytes
// and a back-reference of at least 4 bytes with a 16-bit little-endian offset); the bit
// transpose back to elements runs on the device (fdr_bitunshuffle).
#include <string.h>

#define FDR_TU_ID 5
#include "fdr_internal.cuh"

namespace fdr {

static inline uint64_t read_be64(const uint8_t* p) {
  uint64_t v = 0;
  for (int i = 0; i < 8; ++i) v = (v << 8) | p[i];
  return v;
}
static inline uint32_t read_be32(const uint8_t* p) {
  return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3];
}
static inline void write_be32(uint8_t* p, uint32_t v) {
  p[0] = (uint8_t)(v >> 24); p[1] = (uint8_t)(v >> 16); p[2] = (uint8_t)(v >> 8); p[3] = (uint8_t)v;
}
static inline void write_be64(uint8_t* p, uint64_t v) {
  for (int i = 7; i >= 0; --i) { p[i] = (uint8_t)v; v >>= 8; }
}

// One LZ4 block into dst[0, cap).  Returns the decoded size, or -1 on a malformed block
// (truncated input, an offset of 0 or before the start, output beyond cap).
static int64_t lz4_block_decode(const uint8_t* src, int64_t n, uint8_t* dst, int64_t cap) {
  int64_t ip = 0, op = 0;
  while (ip < n) {
    const uint8_t token = src[ip++];
    int64_t lit = token >> 4;
    if (lit == 15) {
      uint8_t b;
      do {
        if (ip >= n) return -1;
        b = src[ip++];
        lit += b;
      } while (b == 255);
    }
    if (lit > n - ip || lit > cap - op) return -1;
    memcpy(dst + op, src + ip, (size_t)lit);
    ip += lit;
    op += lit;
    if (ip == n) break;  // the last sequence ends after its literals
    if (n - ip < 2) return -1;
    const int64_t off = (int64_t)src[ip] | ((int64_t)src[ip + 1] << 8);
    ip += 2;
    if (off == 0 || off > op) return -1;
    int64_t ml = token & 15;
    if (ml == 15) {
      uint8_t b;
      do {
        if (ip >= n) return -1;
        b = src[ip++];
        ml += b;
      } while (b == 255);
    }
    ml += 4;
    if (ml > cap - op) return -1;
    const uint8_t* from = dst + op - off;
    for (int64_t i = 0; i < ml; ++i) dst[op + i] = from[i];  // overlapping copies repeat
    op += ml;
  }
  return op;
}

static void put_len(uint8_t* dst, int64_t& op, int64_t extra) {
  while (extra >= 255) { dst[op++] = 255; extra -= 255; }
  dst[op++] = (uint8_t)extra;
}

// Greedy LZ4 block encoder (hash of 4-byte sequences, matches of at least 4 bytes, the last
// 5 bytes always literals and no match starting in the last 12 bytes, as the format
// requires).  dst needs n + n/255 + 16 bytes.  Returns the encoded size.
static int64_t lz4_block_encode(const uint8_t* src, int64_t n, uint8_t* dst) {
  constexpr int kHashLog = 14;
  constexpr int64_t kMfLimit = 12, kLastLiterals = 5;
  static thread_local int64_t table[1 << kHashLog];
  for (int i = 0; i < (1 << kHashLog); ++i) table[i] = -1;
  int64_t ip = 0, anchor = 0, op = 0;
  auto rd32 = [&](int64_t p) { uint32_t v; memcpy(&v, src + p, 4); return v; };
  auto emit = [&](int64_t lit_end, int64_t off, int64_t ml) {
    const int64_t lit = lit_end - anchor;
    const int64_t mcode = ml - 4;
    uint8_t& tok = dst[op++];
    tok = (uint8_t)((lit >= 15 ? 15 : lit) << 4);
    if (lit >= 15) put_len(dst, op, lit - 15);
    memcpy(dst + op, src + anchor, (size_t)lit);
    op += lit;
    if (ml > 0) {
      tok |= (uint8_t)(mcode >= 15 ? 15 : mcode);
      dst[op++] = (uint8_t)(off & 0xff);
      dst[op++] = (uint8_t)(off >> 8);
      if (mcode >= 15) put_len(dst, op, mcode - 15);
    }
  };
  while (n >= kMfLimit + 1 && ip + kMfLimit < n) {
    const uint32_t seq = rd32(ip);
    const uint32_t h = (seq * 2654435761u) >> (32 - kHashLog);
    const int64_t ref = table[h];
    table[h] = ip;
    if (ref >= 0 && ip - ref <= 65535 && rd32(ref) == seq) {
      int64_t ml = 4;
      while (ip + ml < n - kLastLiterals && src[ref + ml] == src[ip + ml]) ++ml;
      emit(ip, ip - ref, ml);
      ip += ml;
      anchor = ip;
    } else {
      ++ip;
    }
  }
  emit(n, 0, 0);  // last literals
  return op;
}

// 8 x 8 bit transpose of the bytes of x (byte i bit j <-> byte j bit i), by three rounds of
// exchanging the off-diagonal 1x1, 2x2 and 4x4 bit blocks.
__host__ __device__ __forceinline__ uint64_t bit_transpose8(uint64_t x) {
  uint64_t t;
  t = (x ^ (x >> 7)) & 0x00AA00AA00AA00AAull;
  x ^= t ^ (t << 7);
  t = (x ^ (x >> 14)) & 0x0000CCCC0000CCCCull;
  x ^= t ^ (t << 14);
  t = (x ^ (x >> 28)) & 0x00000000F0F0F0F0ull;
  x ^= t ^ (t << 28);
  return x;
}

// One thread per group of 8 elements of a block: gathers its elem_size*8 bit-row bytes,
// transposes each byte plane and writes its 8 elements.  Blocks of block_elems elements,
// the last holding the whole groups that remain; the final (nelem mod 8) elements are raw.
template <int ES>
__global__ void bitunshuffle_kernel(const uint8_t* __restrict__ in, long long nelem,
                                    long long block_elems, uint8_t* __restrict__ out) {
  const long long ngroups = nelem / 8;
  const long long gpb = block_elems / 8;  // groups per full block
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < ngroups;
       g += (long long)gridDim.x * blockDim.x) {
    const long long blk = g / gpb;
    const long long gi = g - blk * gpb;               // group within its block
    const long long b0 = blk * gpb;                    // first group of the block
    const long long bg = min(gpb, ngroups - b0);      // groups in this block
    const uint8_t* src = in + b0 * 8 * ES;             // the block's bytes
    uint8_t res[8 * ES];
#pragma unroll
    for (int j = 0; j < ES; ++j) {
      uint64_t x = 0;
#pragma unroll
      for (int k = 0; k < 8; ++k)
        if (FDR_DBG_OK(b0 * 8 * ES + (8 * j + k) * bg + gi < nelem * ES))
          x |= (uint64_t)src[(8 * j + k) * bg + gi] << (8 * k);
      x = bit_transpose8(x);  // now byte e = the 8 bits k of element e's byte j
#pragma unroll
      for (int e = 0; e < 8; ++e) res[e * ES + j] = (uint8_t)(x >> (8 * e));
    }
    uint8_t* dst = out + g * 8 * ES;
#pragma unroll
    for (int i = 0; i < 8 * ES; ++i) dst[i] = res[i];
  }
  // the raw tail
  const long long tail0 = ngroups * 8 * ES, tail = nelem * ES - tail0;
  if (blockIdx.x == 0)
    for (long long i = threadIdx.x; i < tail; i += blockDim.x) out[tail0 + i] = in[tail0 + i];
}

}  // namespace fdr

using namespace fdr;

extern "C" {

int fdr_lz4_decompress(const uint8_t* src, int64_t src_size, uint8_t* dst, int64_t dst_capacity,
                       int64_t* dst_size) {
  FDR_CHECK_ARG(src && dst && dst_size && src_size >= 0 && dst_capacity >= 0, "lz4: bad arguments");
  const int64_t r = lz4_block_decode(src, src_size, dst, dst_capacity);
  FDR_CHECK_ARG(r >= 0, "lz4: malformed block or output beyond %lld bytes", (long long)dst_capacity);
  *dst_size = r;
  return FDR_OK;
}

int fdr_lz4_compress(const uint8_t* src, int64_t src_size, uint8_t* dst, int64_t dst_capacity,
                     int64_t* dst_size) {
  FDR_CHECK_ARG(src && dst && dst_size && src_size >= 0, "lz4: bad arguments");
  FDR_CHECK_ARG(dst_capacity >= src_size + src_size / 255 + 16, "lz4: output capacity too small");
  *dst_size = lz4_block_encode(src, src_size, dst);
  return FDR_OK;
}

int fdr_bitshuffle_lz4_decode(const uint8_t* chunk, int64_t chunk_size, int elem_size, uint8_t* out,
                              int64_t out_capacity, int64_t* nbytes, int64_t* block_elems) {
  FDR_CHECK_ARG(chunk && out && nbytes && block_elems, "bitshuffle: NULL argument");
  FDR_CHECK_ARG(elem_size >= 1 && elem_size <= 8, "bitshuffle: element size %d", elem_size);
  FDR_CHECK_ARG(chunk_size >= 12, "bitshuffle: chunk of %lld bytes has no header", (long long)chunk_size);
  const uint64_t total = read_be64(chunk);
  const uint32_t bbytes = read_be32(chunk + 8);
  FDR_CHECK_ARG(total % (uint64_t)elem_size == 0 && (int64_t)total <= out_capacity,
                "bitshuffle: %llu uncompressed bytes (capacity %lld, element size %d)",
                (unsigned long long)total, (long long)out_capacity, elem_size);
  FDR_CHECK_ARG(bbytes > 0 && bbytes % (8u * (uint32_t)elem_size) == 0,
                "bitshuffle: block size %u is not a multiple of 8 elements", bbytes);
  const int64_t nelem = (int64_t)(total / (uint64_t)elem_size);
  const int64_t bel = bbytes / elem_size;
  int64_t ip = 12, op = 0;
  const int64_t whole = nelem - nelem % 8;
  for (int64_t e0 = 0; e0 < whole; e0 += bel) {
    const int64_t ne = std::min(bel, whole - e0);
    FDR_CHECK_ARG(chunk_size - ip >= 4, "bitshuffle: truncated block header");
    const int64_t csz = read_be32(chunk + ip);
    ip += 4;
    FDR_CHECK_ARG(csz <= chunk_size - ip, "bitshuffle: truncated block");
    const int64_t r = lz4_block_decode(chunk + ip, csz, out + op, ne * elem_size);
    FDR_CHECK_ARG(r == ne * elem_size, "bitshuffle: block decoded to %lld bytes, expected %lld",
                  (long long)r, (long long)(ne * elem_size));
    ip += csz;
    op += r;
  }
  const int64_t tail = (nelem - whole) * elem_size;
  FDR_CHECK_ARG(chunk_size - ip >= tail, "bitshuffle: truncated raw tail");
  memcpy(out + op, chunk + ip, (size_t)tail);
  *nbytes = op + tail;
  *block_elems = bel;
  return FDR_OK;
}

int fdr_bitshuffle_lz4_encode(const uint8_t* shuffled, int64_t nbytes, int elem_size,
                              int64_t block_elems, uint8_t* out, int64_t out_capacity,
                              int64_t* out_size) {
  FDR_CHECK_ARG(shuffled && out && out_size, "bitshuffle: NULL argument");
  FDR_CHECK_ARG(elem_size >= 1 && elem_size <= 8 && nbytes % elem_size == 0, "bitshuffle: bad sizes");
  FDR_CHECK_ARG(block_elems > 0 && block_elems % 8 == 0, "bitshuffle: block of %lld elements",
                (long long)block_elems);
  const int64_t nelem = nbytes / elem_size;
  const int64_t whole = nelem - nelem % 8;
  const int64_t nblocks = (whole + block_elems - 1) / block_elems;
  const int64_t bb = block_elems * elem_size;
  FDR_CHECK_ARG(out_capacity >= 12 + nblocks * (4 + bb + bb / 255 + 16) + elem_size * 8,
                "bitshuffle: output capacity too small");
  write_be64(out, (uint64_t)nbytes);
  write_be32(out + 8, (uint32_t)bb);
  int64_t op = 12;
  for (int64_t e0 = 0; e0 < whole; e0 += block_elems) {
    const int64_t ne = std::min(block_elems, whole - e0);
    const int64_t c = lz4_block_encode(shuffled + e0 * elem_size, ne * elem_size, out + op + 4);
    write_be32(out + op, (uint32_t)c);
    op += 4 + c;
  }
  memcpy(out + op, shuffled + whole * elem_size, (size_t)((nelem - whole) * elem_size));
  *out_size = op + (nelem - whole) * elem_size;
  return FDR_OK;
}

int fdr_bitunshuffle(const uint8_t* in, int64_t nelem, int elem_size, int64_t block_elems,
                     uint8_t* out, fdr_stream_t stream) {
  FDR_CHECK_ARG(in && out && nelem >= 0, "bitunshuffle: bad arguments");
  FDR_CHECK_ARG(block_elems > 0 && block_elems % 8 == 0, "bitunshuffle: block of %lld elements",
                (long long)block_elems);
  cudaStream_t s = (cudaStream_t)stream;
  const long long ngroups = nelem / 8;
  const unsigned grid = (unsigned)std::max<long long>(1, std::min<long long>(cdiv(ngroups, 256), 16LL * sm_count()));
  switch (elem_size) {
    case 1: bitunshuffle_kernel<1><<<grid, 256, 0, s>>>(in, nelem, block_elems, out); break;
    case 2: bitunshuffle_kernel<2><<<grid, 256, 0, s>>>(in, nelem, block_elems, out); break;
    case 4: bitunshuffle_kernel<4><<<grid, 256, 0, s>>>(in, nelem, block_elems, out); break;
    case 8: bitunshuffle_kernel<8><<<grid, 256, 0, s>>>(in, nelem, block_elems, out); break;
    default:
      set_error(FDR_ERR_INVALID_ARGUMENT, "bitunshuffle: element size %d (1, 2, 4 or 8)", elem_size);
      return FDR_ERR_INVALID_ARGUMENT;
  }
  FDR_LAUNCH_CHECK("bitunshuffle_kernel");
  return FDR_OK;
}

}  // extern "C"
