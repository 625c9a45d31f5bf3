// Generic batched FFT engine (any length whose prime factors are <= 64).
//
// This is the library's own FFT: mixed-radix Stockham stages in shared memory (radix 2, 3,
// 4, 5, 8 specialised, other primes up to 64 by direct DFT), one pass per transform when
// the length fits a CTA (<= kMaxCtaElems points) and the four-step split into two such
// passes otherwise.  Real transforms use the two-for-one packing (two real columns in one
// complex transform).  The reference gets these transforms from FFTW / cuFFT
// (zdtfdr.jl:119-123, ext/CUDAFrequencyDriftRateTransformsExt.jl:59-79).
#pragma once
#include "fdr_internal.cuh"

namespace fdr {

constexpr int kMaxCtaElems = 8192;   // complex points held by one CTA (double-buffered)
constexpr int kMaxRadixPrime = 64;   // largest prime factor handled by a direct-DFT stage
constexpr int kMaxStages = 24;

// One pass: transforms of length L along axis l of a 3-D view; element (b0, b1, l) of the
// input is at in[b0*is0 + b1*is1 + l*isl] (complex units), output likewise.
struct PassDesc {
  const float2* in;
  float2* out;
  const float2* mul;  // optional pointwise multiplier addressed like the output (or NULL)
  long long is0, is1, isl, os0, os1, osl, ms0, ms1, msl;
  long long nb0, nb1;
  long long tw_n;     // 0: none; else output l of batch b is multiplied by exp(sign*2*pi*i*l*b/tw_n)
  const float2* roots;  // exp(-2*pi*i*m/L), m < L
  int L, nst;
  int radix[kMaxStages];
  int sign;           // -1: forward (exp(-...)), +1: backward
  float scale;
  int tw_dim;         // batch dimension (0 or 1) whose index enters the four-step twiddle
  int bpc;            // transforms per CTA (consecutive along b1)
  int ld_b1_fast;     // load with b1 fastest across threads (else l fastest)
  int st_b1_fast;     // store with b1 fastest across threads
};

// Builds the radix list for L; false if L has a prime factor > kMaxRadixPrime.
bool plan_radices(long long L, int* radix, int* nst);

// Shared roots table exp(-2*pi*i*m/L), m < L, for the current device (cached).
int get_roots(long long L, const float2** roots);

// Launch one pass (fills the plan fields of d from L).
int launch_pass(PassDesc d, cudaStream_t s);

// Transform along a strided axis: element (b, l) at buf[b*sb + l*sl] for b < nb, l < L
// (b is the fast, coalesced index), in place, L <= kMaxCtaElems.  Optional pointwise
// multiply by mul (same addressing) after the transform.
int fft_strided_inplace(float2* buf, long long L, long long sl, long long nb, long long sb,
                        int sign, float scale, const float2* mul, cudaStream_t s);

// Transforms of length N along the contiguous axis of ncol columns (column stride ld):
// in -> out, with tmp an N*ncol scratch used by the four-step split (may be NULL when
// N <= kMaxCtaElems).  in may equal out only when N <= kMaxCtaElems.
int fft_contig(const float2* in, long long ldin, float2* out, long long ldout, long long N,
               long long ncol, int sign, float scale, float2* tmp, cudaStream_t s);

// Scratch (complex elements) needed by rfft_columns / irfft_columns per column pair.
long long real_fft_scratch_per_pair(long long N);

// R2C of ncol real columns (length N, stride ldin) into F (K = N/2+1 rows, stride ldF).
// scratch: real_fft_scratch_per_pair(N) * pairs_per_chunk complex elements.
int rfft_columns(const float* in, long long ldin, long long ncol, long long N, float2* F,
                 long long ldF, float2* scratch, long long pairs_per_chunk, cudaStream_t s);

// C2R (normalised by 1/N) of ncol half spectra (K rows, stride ldS) into real columns of
// length N (stride ldout).  The imaginary parts of bin 0 and, for even N, bin N/2 are
// ignored, as FFTW's and cuFFT's c2r do.
int irfft_columns(const float2* S, long long ldS, long long ncol, long long N, float* out,
                  long long ldout, float2* scratch, long long pairs_per_chunk, cudaStream_t s);

}  // namespace fdr
