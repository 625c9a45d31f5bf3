// Fused ZDT path for power-of-two Nf (2^12 .. 2^22) and Nt <= 16.
//
// The reference computes zdtfdr! as rfft -> prephase -> FFT_l -> .*V -> IFFT_l ->
// postphase -> irfft (zdtfdr.jl:349-362), materialising F, Y (K x Nl) and V (K x Nl) in
// device memory.  Mathematically the chirp-Z stage evaluates, for every frequency bin k
// and drift rate r_j = r0 + j*dr,
//     S_j[k] = sum_t F[k, t] * exp(2*pi*i * k * t * r_j / Nf)
// (the fftfdr.jl phasor form; Bluestein's convolution computes exactly this).  For the
// small Nt of this path the direct evaluation per bin (Horner's rule in t) costs about
// the same arithmetic as three length-Nl FFTs and needs neither V nor Y, so this path
// keeps F on chip and never writes the K x Nl intermediates:
//
//   kernel A (zdtf_input):  four-step pass 1 of the forward FFT of two real columns packed
//                           as one complex column (t pairs): DFT_P over n_b, twiddle.
//   kernel B (zdtf_czt):    per pair of bin residues {k1, P-k1}: forward DFT_Q (pass 2) and
//                           two-for-one unpack into F[k, t] held in registers; then, per
//                           block of drift rates, S_j[k] by Horner's rule with exact
//                           integer phase reduction, the window, two-for-one packing of
//                           rate pairs, inverse DFT_Q (pass 1 of the output FFT) and the
//                           inter-pass twiddle (with the 1/Nf scale).
//   kernel C (zdtf_output): inverse DFT_P (pass 2), real/imaginary parts to the two
//                           output columns of each rate pair.
//
// Nf = P*Q; bin k = k1 + P*k2, channel n = na + Q*nb.  Phases: r0 and dr are float32,
// hence dyadic, so k*r_j/Nf is an exact fraction m / 2^bits with m computed in 64-bit
// integer arithmetic modulo 2^bits; only the final conversion to a float in [-1, 1)
// half-turns rounds.
#define FDR_TU_ID 1  // index violations of the debug build report this file as unit 1
#include <cuda.h>  // CUtensorMap (the encode entry point is fetched from the runtime)
#include <cooperative_groups.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>
#include <math.h>
#include <string.h>

#include "fft_device.cuh"
#include "fft_engine.cuh"
#include "umma.cuh"
#include "zdt_ws.cuh"

namespace cg = cooperative_groups;

namespace fdr {

constexpr int kFusedMinLog2 = 12;
constexpr int kFusedMaxLog2 = 22;
constexpr int kFusedMaxNt = 16;      // F in registers
constexpr int kFusedMaxNtSmem = 64;  // F in shared memory
constexpr int kRatesPerBlock = 8;  // 4 rate pairs (8 sequences) per inverse-FFT block in kernel B
constexpr int kHorner = 4;         // rates evaluated together by one thread (a half block)

// Shared-memory stride of one FFT sequence of kernels A and C (TILE sequences per CTA):
// padded length plus an offset that spreads the TILE sequences over distinct banks.
template <int P, int TILE>
__host__ __device__ constexpr int ac_stride() { return padlen(P) + 16 / TILE; }
template <int Q>
__host__ __device__ constexpr int b_stride() { return padlen(Q) + 1; }

struct PhaseInt {
  unsigned long long R0, Rd, mask;
  int bits;
  float scale;  // 2^(1-bits): converts a signed residue to half-turns
};

struct FusedTables {
  const float2* rootsP;  // exp(-2 pi i m / P), m < P
  const float2* twP;     // Stockham pass twiddles of length P (tw_offset layout)
  const float2* twQ;     // Stockham pass twiddles of length Q
  const float2* tw_lo;   // exp(-2 pi i m / N), m < 2^B
  const float2* tw_hi;   // exp(-2 pi i m 2^B / N), m < N / 2^B
  int B;
};

// exp(-2 pi i m / N) for 0 <= m < N (two-level table product).
__device__ __forceinline__ float2 tw_fwd(const FusedTables& t, long long m) {
  return cmul(__ldg(t.tw_hi + (m >> t.B)), __ldg(t.tw_lo + (m & ((1LL << t.B) - 1))));
}

// exp(2 pi i ph / 2^bits) for a residue 0 <= ph < 2^bits.
__device__ __forceinline__ float2 cis_phase(unsigned long long ph, const PhaseInt& p) {
  long long sp = (long long)ph;
  if ((ph >> (p.bits - 1)) & 1ULL) sp -= (long long)(1ULL << p.bits);
  return cispif(__ll2float_rn(sp) * p.scale);
}

// ------------------------------------------------------------------------------------
// Kernel A: forward four-step pass 1.  grid (Q/TA, NP); A[p][k1][na].
// ------------------------------------------------------------------------------------
template <int P, int TA, int T>
__global__ void __launch_bounds__(T)
zdtf_input_kernel(const float* __restrict__ spec, long long N, int Nt, int Q,
                  float2* __restrict__ A, FusedTables tab) {
  constexpr int SS = ac_stride<P, TA>();
  constexpr int TP = TA / 2;  // sequence pairs: each thread moves two adjacent channels
  extern __shared__ float2 sm[];
  float2* buf = sm;
  float2* twt = sm + TA * SS;
  const int na0 = blockIdx.x * TA;
  const int p = blockIdx.y;
  for (int i = threadIdx.x; i < tw_size(P); i += T) twt[i] = __ldg(tab.twP + i);
  const float* c0 = spec + (long long)(2 * p) * N;
  const bool has1 = (2 * p + 1) < Nt;
  const float* c1 = spec + (long long)(2 * p + 1) * N;
  static_assert((TP * P) % T == 0, "tile must divide evenly");
  constexpr int NL = TP * P / T;  // loads per thread: all issued before any is consumed
  {
    float2 a[NL], b[NL];
#pragma unroll
    for (int i = 0; i < NL; ++i) {
      const int e = threadIdx.x + i * T;
      const int sp = e % TP, nb = e / TP;
      const long long n = (long long)(na0 + 2 * sp) + (long long)Q * nb;
      a[i] = FDR_DBG_OK(n + 2 <= N) ? __ldcs(reinterpret_cast<const float2*>(c0 + n)) : make_float2(0.f, 0.f);
      b[i] = (has1 && FDR_DBG_OK(n + 2 <= N)) ? __ldcs(reinterpret_cast<const float2*>(c1 + n))
                                               : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int i = 0; i < NL; ++i) {
      const int e = threadIdx.x + i * T;
      const int sp = e % TP, nb = e / TP;
      buf[(2 * sp) * SS + pidx(nb)] = make_float2(a[i].x, b[i].x);
      buf[(2 * sp + 1) * SS + pidx(nb)] = make_float2(a[i].y, b[i].y);
    }
  }
  __syncthreads();
  smem_fft<P, TA, SS, T, -1>(buf, twt);
  for (int e = threadIdx.x; e < TP * P; e += T) {
    const int sp = e % TP, k1 = e / TP;
    const int na = na0 + 2 * sp;
    const float2 v0 = cmul(buf[(2 * sp) * SS + pidx(k1)], tw_fwd(tab, (long long)k1 * na));
    const float2 v1 = cmul(buf[(2 * sp + 1) * SS + pidx(k1)], tw_fwd(tab, (long long)k1 * (na + 1)));
    if (FDR_DBG_OK(((long long)p * P + k1) * Q + na + 2 <= (long long)gridDim.y * P * Q))
      *reinterpret_cast<float4*>(A + ((long long)p * P + k1) * Q + na) = make_float4(v0.x, v0.y, v1.x, v1.y);
  }
}

// Kernel A for P = 2048 = 64 x 32: two register passes with one shared-memory transpose (the
// forward-sign mirror of zdtf_output_tma64_kernel).  nb = nb1 + 64*nb2, k1 = k1b + 32*k1a:
//   X[k1b + 32 k1a] = sum_nb1 w64^(k1a nb1) [w^(k1b nb1) sum_nb2 x[nb1 + 64 nb2] w32^(k1b nb2)]
// with w = exp(-2 pi i / P).  Thread (seq, nb1) loads its 32 values of the two packed time
// steps straight from the spectrogram and transforms them over nb2; lanes h and h + 16 then
// share the 64-point DFT over nb1 (decimation in time: lane h takes nb1 = 2k + h, lane 1
// applies w64^n, one shuffle exchange), and A is stored with the inter-pass twiddle
// exp(-2 pi i k1 n_a / Nf) from a two-level table in shared memory.  Shared-memory strides
// as in the output kernel (S1 = 33, SSEQ = 2 mod 16): conflict-free transposes.
struct In64Shape {
  static constexpr int P1 = 64, P2 = 32, P = P1 * P2, TS = 8, T = 64 * TS;
  static constexpr int S1 = P2 + 1;
  static constexpr int SSEQ = ((P1 * S1 + 15) / 16) * 16 + 16 / TS;
  static constexpr size_t REGION = sizeof(float2) * TS * SSEQ;
  static constexpr int TW1 = P1 * S1;  // tw1[nb1][k] = w^(nb1 k), rows S1 apart
  static constexpr size_t smem(int B, long long N) {
    return REGION + sizeof(float2) * (TW1 + P1 / 2 + (1LL << B) + (N >> B));
  }
};

__global__ void __launch_bounds__(In64Shape::T, 1)
zdtf_input64_kernel(const float* __restrict__ spec, long long N, int Nt, int Q,
                    float2* __restrict__ A, FusedTables tab) {
  using SH = In64Shape;
  constexpr int P = SH::P, P1 = SH::P1, P2 = SH::P2, TS = SH::TS, S1 = SH::S1, SSEQ = SH::SSEQ;
  extern __shared__ float2 sm[];
  float2* region = sm;           // TS * SSEQ: the transpose
  float2* tw1 = sm + TS * SSEQ;  // w^(nb1 k): P1 rows of S1
  float2* tw2 = tw1 + SH::TW1;   // w64^n, n < P1 / 2
  const int nlo = 1 << tab.B, nhi = (int)(N >> tab.B);
  float2* tlo = tw2 + P1 / 2;  // exp(-2 pi i m / N), m < 2^B
  float2* thi = tlo + nlo;     // exp(-2 pi i m 2^B / N), m < N / 2^B
  const int tid = threadIdx.x;
  for (int i = tid; i < P; i += SH::T)
    tw1[(i / P2) * S1 + i % P2] = __ldg(tab.rootsP + (((i / P2) * (i % P2)) & (P - 1)));
  for (int i = tid; i < P1 / 2; i += SH::T) tw2[i] = __ldg(tab.rootsP + i * (P / P1));
  for (int i = tid; i < nlo; i += SH::T) tlo[i] = __ldg(tab.tw_lo + i);
  for (int i = tid; i < nhi; i += SH::T) thi[i] = __ldg(tab.tw_hi + i);
  const int na0 = blockIdx.x * TS;
  const int p = blockIdx.y;
  const float* c0 = spec + (long long)(2 * p) * N;
  const bool has1 = (2 * p + 1) < Nt;
  const float* c1 = spec + (long long)(2 * p + 1) * N;
  // pass 1: thread (seq, nb1), all 32 loads of each column issued before any is used
  const int seq1 = tid % TS, nb1 = tid / TS;
  float2 v[P2];
  {
    const long long n0 = (long long)(na0 + seq1) + (long long)Q * nb1;
    const long long st = (long long)Q * P1;
#pragma unroll
    for (int m = 0; m < P2; ++m) v[m].x = FDR_DBG_OK(n0 + st * m < N) ? __ldcs(c0 + n0 + st * m) : 0.f;
#pragma unroll
    for (int m = 0; m < P2; ++m) v[m].y = (has1 && FDR_DBG_OK(n0 + st * m < N)) ? __ldcs(c1 + n0 + st * m) : 0.f;
  }
  __syncthreads();  // the tables are in shared memory
  Dft<P2>::run(v, -1);
  {
    float2* b = region + seq1 * SSEQ + nb1 * S1;
    const float2* t1 = tw1 + nb1 * S1;
#pragma unroll
    for (int k = 0; k < P2; ++k) b[k] = cmul(v[k], t1[k]);
  }
  __syncthreads();
  // pass 2: lane = seq + TS * (k1b mod (16 / TS)) + 16 * h
  const int lane = tid & 31;
  const int seq2 = lane % TS, h = lane >> 4;
  const int k1b = ((lane / TS) % (16 / TS)) + (16 / TS) * (tid >> 5);
  {
    const float2* b = region + seq2 * SSEQ + h * S1 + k1b;
#pragma unroll
    for (int k = 0; k < P1 / 2; ++k) v[k] = b[2 * k * S1];
  }
  Dft<P1 / 2>::run(v, -1);  // E (h = 0) or O (h = 1) at n mod 32
  // lane 0-half keeps E[0..15] and receives O[0..15]; lane 1-half keeps O[16..31] and
  // receives E[16..31]; each applies w64^n to its 16 O values:
  // X[n] = E[n] + w64^n O[n], X[n + 32] = E[n] - w64^n O[n]
#pragma unroll
  for (int i = 0; i < P1 / 4; ++i) {
    const float2 s = h ? v[i] : v[i + P1 / 4];
    float2 o;
    o.x = __shfl_xor_sync(0xffffffffu, s.x, 16);
    o.y = __shfl_xor_sync(0xffffffffu, s.y, 16);
    const float2 e = h ? o : v[i];
    const float2 w = cmul(h ? v[i + P1 / 4] : o, tw2[i + (P1 / 4) * h]);
    v[i] = cadd(e, w);           // k1a = i + 16h
    v[i + P1 / 4] = csub(e, w);  // k1a = i + 16h + 32
  }
  const int na = na0 + seq2;
  float2* a0 = A + (long long)p * P * Q + na;
#pragma unroll
  for (int i = 0; i < P1 / 2; ++i) {
    const int k1a = (i & (P1 / 4 - 1)) + 16 * h + (i >= P1 / 4 ? P1 / 2 : 0);
    const int k1 = k1b + P2 * k1a;
    const long long m = (long long)k1 * na;
    const float2 t = cmul(thi[m >> tab.B], tlo[m & (nlo - 1)]);
    if (FDR_DBG_OK((long long)p * P * Q + na + (long long)k1 * Q < (long long)gridDim.y * P * Q))
      a0[(long long)k1 * Q] = cmul(v[i], t);
  }
}
// ------------------------------------------------------------------------------------
// Kernel B helpers
// ------------------------------------------------------------------------------------
struct CztArgs {
  const float2* A;
  float2* W;          // [pair][k1][na] for pairs [0, npairs)
  float2* F;          // A->F mode output (K x Nt) or NULL
  const double* wk;   // custom window values (K) or NULL
  const int* blk_base;  // rate index (on the r0 + j*dr grid) of each 8-rate block's first
                        // rate, or NULL for 8*block (the contiguous rates 0..Nr-1)
  long long N;
  int P, Nt, NP, Nr, npairs, pairs_per_group, window;
  PhaseInt ph;
  FusedTables tab;
};

// Position (side, k2) of the bin N - k for the base at (side, k2) of CTA c.
__device__ __forceinline__ void mirror_of(int c, int side, int k2, int Q, int* ms, int* mk2) {
  if (c == 0 && side == 0) { *ms = 0; *mk2 = (Q - k2) & (Q - 1); }
  else if (c == 0) { *ms = 1; *mk2 = Q - 1 - k2; }
  else { *ms = 1 - side; *mk2 = Q - 1 - k2; }
}

// Forward pass 2 + two-for-one unpack: G[b][t] = F[k_b, t] for the two bases of this
// thread (b = side, k2 = threadIdx.x); CTA 0's thread 0 also stores the Nyquist bin's
// F[N/2, t] into gnyq (shared memory).  buf holds 8 sequences of stride b_stride<Q>().
template <int Q, int NTR>
__device__ __forceinline__ void czt_forward(const CztArgs& a, int c, const int* k1s, float2* buf,
                                            const float2* twt, float2* gnyq,
                                            float2 (&G)[2][NTR]) {
  constexpr int T = Q / 2;
  constexpr int SS = b_stride<Q>();
  constexpr int PC = 4;  // t pairs per chunk (8 sequences: 4 pairs x 2 sides)
  const int tid = threadIdx.x;
#pragma unroll
  for (int b = 0; b < 2; ++b)
#pragma unroll
    for (int t = 0; t < NTR; ++t) G[b][t] = make_float2(0.f, 0.f);
  // Only thread 0 of CTA 0 touches gnyq; t-pairs beyond Nt are never loaded, so clear all.
  if (c == 0 && tid == 0)
    for (int t = 0; t < NTR; ++t) gnyq[t] = make_float2(0.f, 0.f);
#pragma unroll
  for (int p0 = 0; p0 < NTR / 2; p0 += PC) {
    if (p0 < a.NP) {
      __syncthreads();
      {
        constexpr int NL = 2 * PC * Q / T;  // loads per thread, issued before any is stored
        float2 v[NL];
#pragma unroll
        for (int i = 0; i < NL; ++i) {
          const int e = tid + i * T;
          const int seq = e / Q, na = e - seq * Q;
          const int pp = p0 + (seq >> 1), side = seq & 1;
          v[i] = (pp < a.NP && FDR_DBG_OK(((long long)pp * a.P + k1s[side]) * Q + na < (long long)a.NP * a.P * Q))
                     ? __ldcs(a.A + ((long long)pp * a.P + k1s[side]) * Q + na)
                             : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int i = 0; i < NL; ++i) {
          const int e = tid + i * T;
          const int seq = e / Q, na = e - seq * Q;
          buf[seq * SS + pidx(na)] = v[i];
        }
      }
      __syncthreads();
      smem_fft<Q, 2 * PC, SS, T, -1>(buf, twt);
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        int ms, mk2;
        mirror_of(c, b, tid, Q, &ms, &mk2);
#pragma unroll
        for (int u = 0; u < PC; ++u) {
          if (2 * (p0 + u) + 1 < NTR) {
            const float2 zk = buf[(2 * u + b) * SS + pidx(tid)];
            const float2 zm = cconj(buf[(2 * u + ms) * SS + pidx(mk2)]);
            const float2 sm_ = cadd(zk, zm), d = csub(zk, zm);
            G[b][2 * (p0 + u)] = make_float2(0.5f * sm_.x, 0.5f * sm_.y);
            G[b][2 * (p0 + u) + 1] = make_float2(0.5f * d.y, -0.5f * d.x);
          }
        }
      }
      if (c == 0 && tid == 0) {
#pragma unroll
        for (int u = 0; u < PC; ++u) {
          if (2 * (p0 + u) + 1 < NTR) {
            const float2 z = buf[(2 * u) * SS + pidx(Q / 2)];
            gnyq[2 * (p0 + u)] = make_float2(z.x, 0.f);
            gnyq[2 * (p0 + u) + 1] = make_float2(z.y, 0.f);
          }
        }
      }
    }
  }
  __syncthreads();
}

template <int NTR>
__device__ __forceinline__ float2 horner(const float2 (&G)[NTR], float2 w) {
  float2 s = G[NTR - 1];
#pragma unroll
  for (int t = NTR - 2; t >= 0; --t) {
    s = make_float2(fmaf(s.x, w.x, fmaf(-s.y, w.y, G[t].x)), fmaf(s.x, w.y, fmaf(s.y, w.x, G[t].y)));
  }
  return s;
}

// Packed-FP32 helpers (sm_100 FFMA2 / FMUL2): lane 0 and lane 1 carry two independent
// evaluations, each lane performing exactly the scalar operation sequence.
__device__ __forceinline__ float2 pk_fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 pk_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 pk_neg(float2 a) { return __fmul2_rn(a, make_float2(-1.f, -1.f)); }

// horner() for the two bins of a thread at once: (Gx[t], Gy[t]) hold the real and imaginary
// parts of F[k_b, t] for b = 0, 1 in the two lanes; (wx, wy) the two multipliers.
template <int NTR>
__device__ __forceinline__ void horner_pk(const float2 (&Gx)[NTR], const float2 (&Gy)[NTR], float2 wx,
                                          float2 wy, float2& sx, float2& sy) {
  const float2 nwy = pk_neg(wy);
  sx = Gx[NTR - 1];
  sy = Gy[NTR - 1];
#pragma unroll
  for (int t = NTR - 2; t >= 0; --t) {
    const float2 tx = pk_fma(sx, wx, pk_fma(sy, nwy, Gx[t]));
    const float2 ty = pk_fma(sx, wy, pk_fma(sy, wx, Gy[t]));
    sx = tx;
    sy = ty;
  }
}

__device__ __forceinline__ float window_value(const CztArgs& a, long long k) {
  if (a.window == FDR_WINDOW_HAMMING) return (float)(0.53836 + 0.46164 * cospi(2.0 * (double)k / (double)a.N));
  if (a.window == FDR_WINDOW_CUSTOM) return (float)a.wk[k];
  return 1.f;
}

// ------------------------------------------------------------------------------------
// Kernel B: grid (P/2, rate groups), Q/2 threads.
// ------------------------------------------------------------------------------------
// WINDOWED = false: the rectangular window (weights 1, skipped: the same FDR bit for bit).
template <int Q, int NTR, bool WINDOWED>
__global__ void __launch_bounds__(Q / 2, (Q <= 512 ? 2 : 1)) zdtf_czt_kernel(CztArgs a) {
  constexpr int T = Q / 2;
  constexpr int SS = b_stride<Q>();
  extern __shared__ float2 sm[];
  float2* buf = sm;                           // kRatesPerBlock * SS
  float2* twt = buf + kRatesPerBlock * SS;    // tw_size(Q)
  float2* twr = twt + tw_size(Q);             // 2 * Q
  float2* gnyq = twr + 2 * Q;                 // NTR
  float2* buf2 = gnyq + NTR;                  // kRatesPerBlock * SS
  // the thread's phase residues alpha_b, beta_b (kept in shared memory, not registers)
  unsigned long long* phs = reinterpret_cast<unsigned long long*>(buf2 + kRatesPerBlock * SS);
  const int tid = threadIdx.x;
  const int c = blockIdx.x;
  const int P = a.P;
  const int k1s[2] = {c == 0 ? 0 : c, c == 0 ? P / 2 : P - c};
  const float invN = 1.0f / (float)a.N;
  for (int i = tid; i < tw_size(Q); i += T) twt[i] = __ldg(a.tab.twQ + i);
  for (int i = tid; i < 2 * Q; i += T) {
    const int side = i / Q, na = i - side * Q;
    twr[i] = cscale(cconj(tw_fwd(a.tab, (long long)k1s[side] * na)), invN);
  }
  float2 Gx[NTR], Gy[NTR];  // lanes = the thread's two bins
  {
    float2 G[2][NTR];
    czt_forward<Q, NTR>(a, c, k1s, buf, twt, gnyq, G);
#pragma unroll
    for (int t = 0; t < NTR; ++t) {
      Gx[t] = make_float2(G[0][t].x, G[1][t].x);
      Gy[t] = make_float2(G[0][t].y, G[1][t].y);
    }
  }

  // Per-base phase state: w_{k,j} = exp(2 pi i (alpha + j*beta) / 2^bits); rates are taken
  // kHorner at a time, w = w(first rate of the group, exact) * pw[jr] (exact).
  const unsigned long long mask = a.ph.mask;
  // PWx/PWy[i - 1] = exact w(k_b, i*dr) for i = 1..kHorner (lanes = b; w(k_b, 0) = 1)
  float2 PWx[kHorner], PWy[kHorner];
  float2 WIN;
#pragma unroll
  for (int b = 0; b < 2; ++b) {
    const unsigned long long k = (unsigned long long)k1s[b] + (unsigned long long)P * tid;
    const unsigned long long beta = (k * a.ph.Rd) & mask;
    phs[(2 * b) * T + tid] = (k * a.ph.R0) & mask;
    phs[(2 * b + 1) * T + tid] = beta;
#pragma unroll
    for (int i = 1; i <= kHorner; ++i) {
      const float2 p = cis_phase(((unsigned long long)i * beta) & mask, a.ph);
      if (b == 0) { PWx[i - 1].x = p.x; PWy[i - 1].x = p.y; } else { PWx[i - 1].y = p.x; PWy[i - 1].y = p.y; }
    }
    const float wv = window_value(a, (long long)k);
    if (b == 0) WIN.x = wv; else WIN.y = wv;
  }
  // Nyquist bin (CTA 0, thread 0)
  const unsigned long long kny = (unsigned long long)(a.N / 2);

  int ms[2], mk2[2];
#pragma unroll
  for (int b = 0; b < 2; ++b) mirror_of(c, b, tid, Q, &ms[b], &mk2[b]);
  const bool dc = (c == 0 && tid == 0);

  // Rate blocks alternate between buf2 and buf (the forward pass used buf): the inverse
  // DFT_Q ping-pongs between the two, and the buffer a block's Horner sums go to was last
  // read before the previous block's final barrier, so no barrier precedes the writes.
  constexpr bool kFlip = (passes_before_emit(Q) % 2) == 0;
  float2* hb = buf2;
  float2* ob = buf;
  const int q_begin = blockIdx.y * a.pairs_per_group;
  const int q_end = min(a.npairs, q_begin + a.pairs_per_group);
  for (int q0 = q_begin; q0 < q_end; q0 += kRatesPerBlock / 2) {
    const int j0 = 2 * q0;
    const long long jg = a.blk_base ? (long long)__ldg(a.blk_base + (q0 >> 2)) : (long long)j0;
    // exact phase of the block's first rate; the second half starts at w0 * w(k, 4*dr)
    float2 Wbx, Wby;
    {
      const float2 w0 = cis_phase((phs[tid] + (unsigned long long)jg * phs[T + tid]) & mask, a.ph);
      const float2 w1 = cis_phase((phs[2 * T + tid] + (unsigned long long)jg * phs[3 * T + tid]) & mask, a.ph);
      Wbx = make_float2(w0.x, w1.x);
      Wby = make_float2(w0.y, w1.y);
    }
#pragma unroll
    for (int h = 0; h < kRatesPerBlock / kHorner; ++h) {
      const int jh = j0 + h * kHorner;
      float2 S[2][kHorner];
      float2 W0x = Wbx, W0y = Wby;
      if (h > 0) {  // w(first rate of the half) = wb * w(k, kHorner*dr)
        W0x = pk_fma(Wbx, PWx[kHorner - 1], pk_mul(pk_neg(Wby), PWy[kHorner - 1]));
        W0y = pk_fma(Wbx, PWy[kHorner - 1], pk_mul(Wby, PWx[kHorner - 1]));
      }
      const float2 NW0y = pk_neg(W0y);
      if (jh < a.Nr) {
#pragma unroll
        for (int jr = 0; jr < kHorner; ++jr) {
          float2 wx = W0x, wy = W0y;  // jr = 0: w(k, 0) = 1
          if (jr > 0) {
            wx = pk_fma(W0x, PWx[jr - 1], pk_mul(NW0y, PWy[jr - 1]));
            wy = pk_fma(W0x, PWy[jr - 1], pk_mul(W0y, PWx[jr - 1]));
          }
          float2 sx, sy;
          horner_pk<NTR>(Gx, Gy, wx, wy, sx, sy);
          if (WINDOWED) {
            sx = pk_mul(sx, WIN);
            sy = pk_mul(sy, WIN);
          }
          S[0][jr] = make_float2(sx.x, sy.x);
          S[1][jr] = make_float2(sx.y, sy.y);
        }
        if (jh + kHorner > a.Nr) {  // rates past the grid's last (uniform over the CTA): zero
#pragma unroll
          for (int jr = 0; jr < kHorner; ++jr)
            if (jh + jr >= a.Nr) S[0][jr] = S[1][jr] = make_float2(0.f, 0.f);
        }
      } else {  // a half block past the last rate (uniform over the CTA): no sums
#pragma unroll
        for (int jr = 0; jr < kHorner; ++jr) S[0][jr] = S[1][jr] = make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int b = 0; b < 2; ++b) {
#pragma unroll
        for (int u2 = 0; u2 < kHorner / 2; ++u2) {
          const int u = h * (kHorner / 2) + u2;  // rate pair within the block
          const float2 sa = S[b][2 * u2], sb = S[b][2 * u2 + 1];
          if (dc && b == 0) {
            hb[(2 * u) * SS + pidx(0)] = make_float2(sa.x, sb.x);  // real-only DC bin
          } else {
            hb[(2 * u + b) * SS + pidx(tid)] = make_float2(sa.x - sb.y, sa.y + sb.x);          // sa + i sb
            hb[(2 * u + ms[b]) * SS + pidx(mk2[b])] = make_float2(sa.x + sb.y, sb.x - sa.y);  // conj(sa) + i conj(sb)
          }
        }
      }
    }
    if (c == 0 && tid == 0) {
      float2 Gn[NTR];
#pragma unroll
      for (int t = 0; t < NTR; ++t) Gn[t] = gnyq[t];
      const float wn = window_value(a, (long long)kny);
      for (int u = 0; u < kRatesPerBlock / 2; ++u) {
        float v[2];
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
          const int j = j0 + 2 * u + hh;
          const unsigned long long alpha_n = (kny * a.ph.R0) & mask, beta_n = (kny * a.ph.Rd) & mask;
          const float2 w = cis_phase((alpha_n + (unsigned long long)(jg + 2 * u + hh) * beta_n) & mask, a.ph);
          const float2 sv = horner<NTR>(Gn, w);
          v[hh] = (j < a.Nr) ? sv.x * wn : 0.f;  // real-only Nyquist bin
        }
        hb[(2 * u) * SS + pidx(Q / 2)] = make_float2(v[0], v[1]);
      }
    }
    __syncthreads();
    // inverse DFT_Q; its last pass writes W (with the inter-pass twiddle and 1/Nf) directly.
    // Row (q0 + p, k1) of W starts at Wq + (p*P + k1)*Q: a 32-bit offset (p < 4; the fused
    // path has P*Q = Nf <= 2^22).
    float2* const Wq = a.W + (long long)q0 * P * Q;
    const int k1a = k1s[0], k1b = k1s[1];
    stockham_passes_emit_pp<Q, kRatesPerBlock, SS, T, +1, 1>(hb, ob, twt, [&](int seq, int na, float2 v) {
      const int p = seq >> 1, side = seq & 1;
      const unsigned off = (unsigned)((p * P + (side ? k1b : k1a)) * Q + na);
      if (q0 + p < q_end && FDR_DBG_OK((long long)q0 * P * Q + off < (long long)a.npairs * P * Q))
        Wq[off] = cmul(v, twr[side * Q + na]);
    });
    if (kFlip) {
      float2* t = hb;
      hb = ob;
      ob = t;
    }
  }
}

// ------------------------------------------------------------------------------------
// Kernel B for 16 < Nt <= NT (32 or 64): F[k, t] of the CTA's Q bases lives in shared
// memory, t-major with the bases in adjacent pairs interleaved by component: float4
// gs4[t*(Q/2) + b/2] = {Re F[b0], Re F[b1], Im F[b0], Im F[b1]} for b0 = b & ~1, b1 = b0 + 1,
// so one 16-byte load gives the packed-FP32 operands (Re, Re) and (Im, Im) of a base pair.
// T = Q*G threads, G = threads per base pair and rate half; each thread evaluates RT = 4/G
// rates of every 8-rate block for its two bases, lanes = bases.  Base b (0 <= b < Q) is side
// b/(Q/2), k2 = b % (Q/2) (a pair never straddles the sides: Q/2 is even).
// ------------------------------------------------------------------------------------
template <int Q>
struct CztSmemShape {
  static constexpr int G = Q >= 512 ? 1 : 2;
  static constexpr int T = Q * G;
  static constexpr int RT = 4 / G;
  // gs starts on a 16-byte boundary (an even float2 offset)
  static constexpr int GS_OFF = (kRatesPerBlock * b_stride<Q>() + tw_size(Q) + 2 * Q + 1) & ~1;
  template <int NT>
  static constexpr size_t smem() {
    return sizeof(float2) * (GS_OFF + NT * Q + NT);
  }
};

// F[b, t] in the base-pair interleaved layout of gs (see CztSmemShape).
__device__ __forceinline__ void gs_put(float2* gs, int Q, int t, int b, float2 v) {
  float* f = reinterpret_cast<float*>(gs) + ((t * (Q / 2) + (b >> 1)) << 2) + (b & 1);
  f[0] = v.x;
  f[2] = v.y;
}
__device__ __forceinline__ float2 gs_get(const float2* gs, int Q, int t, int b) {
  const float* f = reinterpret_cast<const float*>(gs) + ((t * (Q / 2) + (b >> 1)) << 2) + (b & 1);
  return make_float2(f[0], f[2]);
}

// Forward DFT_Q of the CTA's A rows for all t into gs (pair-interleaved F), by all T
// threads of the block.  HALF: keep only the bins of side own_side (Q/2 bins per row of gs;
// the DFTs of both sides are still computed, the two-for-one unpacking needs both).
template <int Q, int NT, int T = CztSmemShape<Q>::T, bool HALF = false>
__device__ __forceinline__ void czt_forward_smem(const CztArgs& a, int c, const int* k1s,
                                                 float2* buf, const float2* twt, float2* gs,
                                                 float2* gnyq, int own_side = 0) {
  constexpr int SS = b_stride<Q>();
  constexpr int PC = 4;
  constexpr int QROW = HALF ? Q / 2 : Q;  // bins per row of gs
  const int tid = threadIdx.x;
  for (int i = tid; i < NT * QROW; i += T) gs[i] = make_float2(0.f, 0.f);
  if (c == 0 && tid == 0)
    for (int t = 0; t < NT; ++t) gnyq[t] = make_float2(0.f, 0.f);
  // A rows of chunk p0 (PC t pairs x 2 sides) into registers; the next chunk's loads are
  // issued before the current chunk's FFT, so their latency overlaps it
  constexpr int NE = 2 * PC * Q;  // elements per chunk
  constexpr int NL = (NE + T - 1) / T;
  float2 v[NL];
  auto load_chunk = [&](int p0) {
#pragma unroll
    for (int i = 0; i < NL; ++i) {
      const int e = tid + i * T;
      const int seq = e / Q, na = e - seq * Q;
      const int pp = p0 + (seq >> 1), side = seq & 1;
      v[i] = ((NE % T == 0 || e < NE) && pp < a.NP &&
              FDR_DBG_OK(((long long)pp * a.P + k1s[side]) * Q + na < (long long)a.NP * a.P * Q))
                 ? __ldcs(a.A + ((long long)pp * a.P + k1s[side]) * Q + na)
                 : make_float2(0.f, 0.f);
    }
  };
  load_chunk(0);
  for (int p0 = 0; p0 < a.NP; p0 += PC) {
    __syncthreads();
#pragma unroll
    for (int i = 0; i < NL; ++i) {
      const int e = tid + i * T;
      const int seq = e / Q, na = e - seq * Q;
      if (NE % T == 0 || e < NE) buf[seq * SS + pidx(na)] = v[i];
    }
    if (p0 + PC < a.NP) load_chunk(p0 + PC);
    __syncthreads();
    smem_fft<Q, 2 * PC, SS, T, -1>(buf, twt);
    for (int e = tid; e < PC * QROW; e += T) {
      const int u = e / QROW;
      const int b = e - u * QROW + (HALF ? own_side * (Q / 2) : 0);
      if (p0 + u >= a.NP) continue;
      const int side = b / (Q / 2), k2 = b - side * (Q / 2);
      int ms, mk2;
      mirror_of(c, side, k2, Q, &ms, &mk2);
      const float2 zk = buf[(2 * u + side) * SS + pidx(k2)];
      const float2 zm = cconj(buf[(2 * u + ms) * SS + pidx(mk2)]);
      const float2 sm_ = cadd(zk, zm), d = csub(zk, zm);
      const int t0 = 2 * (p0 + u);
      const int bg = HALF ? k2 : b;  // bin within gs's row
      gs_put(gs, QROW, t0, bg, make_float2(0.5f * sm_.x, 0.5f * sm_.y));
      if (t0 + 1 < NT) gs_put(gs, QROW, t0 + 1, bg, make_float2(0.5f * d.y, -0.5f * d.x));
    }
    if (c == 0 && tid == 0) {
      for (int u = 0; u < PC && p0 + u < a.NP; ++u) {
        const float2 z = buf[(2 * u) * SS + pidx(Q / 2)];
        const int t0 = 2 * (p0 + u);
        gnyq[t0] = make_float2(z.x, 0.f);
        if (t0 + 1 < NT) gnyq[t0 + 1] = make_float2(z.y, 0.f);
      }
    }
  }
  __syncthreads();
}

template <int Q, int NT>
__global__ void __launch_bounds__(CztSmemShape<Q>::T, 1) zdtf_czt_smem_kernel(CztArgs a) {
  using SH = CztSmemShape<Q>;
  constexpr int T = SH::T, RT = SH::RT;
  constexpr int SS = b_stride<Q>();
  extern __shared__ float2 sm[];
  float2* buf = sm;
  float2* twt = buf + kRatesPerBlock * SS;
  float2* twr = twt + tw_size(Q);
  float2* gs = sm + SH::GS_OFF;
  float2* gnyq = gs + NT * Q;
  const int tid = threadIdx.x;
  const int c = blockIdx.x;
  const int P = a.P;
  const int k1s[2] = {c == 0 ? 0 : c, c == 0 ? P / 2 : P - c};
  const float invN = 1.0f / (float)a.N;
  for (int i = tid; i < tw_size(Q); i += T) twt[i] = __ldg(a.tab.twQ + i);
  for (int i = tid; i < 2 * Q; i += T) {
    const int side = i / Q, na = i - side * Q;
    twr[i] = cscale(cconj(tw_fwd(a.tab, (long long)k1s[side] * na)), invN);
  }
  czt_forward_smem<Q, NT>(a, c, k1s, buf, twt, gs, gnyq);

  // thread -> (base pair bp, rate group rg): bases b0 = 2 bp and b0 + 1 (the two lanes of
  // every packed operation), rates rg*RT .. rg*RT + RT - 1 of each 8-rate block
  const int bp = tid % (Q / 2), rg = tid / (Q / 2);
  const int b0 = 2 * bp;
  const int side = b0 / (Q / 2), k20 = b0 - side * (Q / 2);
  int ms[2], mk2[2];
  mirror_of(c, side, k20, Q, &ms[0], &mk2[0]);
  mirror_of(c, side, k20 + 1, Q, &ms[1], &mk2[1]);
  const bool dc = (c == 0 && side == 0 && k20 == 0);  // lane 0 is the DC bin
  const unsigned long long mask = a.ph.mask;
  unsigned long long alpha[2], beta[2];
  float2 pwx[RT], pwy[RT];  // pw[i] = exact w(k_lane, i*dr), lanes = the two bases
  float2 win;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const unsigned long long k = (unsigned long long)k1s[side] + (unsigned long long)P * (k20 + h);
    alpha[h] = (k * a.ph.R0) & mask;
    beta[h] = (k * a.ph.Rd) & mask;
#pragma unroll
    for (int i = 0; i < RT; ++i) {
      const float2 p = cis_phase(((unsigned long long)i * beta[h]) & mask, a.ph);
      if (h == 0) { pwx[i].x = p.x; pwy[i].x = p.y; } else { pwx[i].y = p.x; pwy[i].y = p.y; }
    }
    const float wv = window_value(a, (long long)k);
    if (h == 0) win.x = wv; else win.y = wv;
  }
  const unsigned long long kny = (unsigned long long)(a.N / 2);
  const unsigned long long alpha_n = (kny * a.ph.R0) & mask, beta_n = (kny * a.ph.Rd) & mask;
  const int Nt = a.Nt;
  const float4* gs4 = reinterpret_cast<const float4*>(gs);

  const int q_begin = blockIdx.y * a.pairs_per_group;
  const int q_end = min(a.npairs, q_begin + a.pairs_per_group);
  for (int q0 = q_begin; q0 < q_end; q0 += kRatesPerBlock / 2) {
    const int j0 = 2 * q0 + rg * RT;  // this thread's first rate of the block
    const long long jb = a.blk_base ? (long long)__ldg(a.blk_base + (q0 >> 2)) : (long long)(2 * q0);
    // w(k_lane, first rate) exact; the thread's other rates = that * pw[i] (exact pw)
    float2 W0x, W0y;
    {
      const unsigned long long jj = (unsigned long long)(jb + rg * RT);
      const float2 w0 = cis_phase((alpha[0] + jj * beta[0]) & mask, a.ph);
      const float2 w1 = cis_phase((alpha[1] + jj * beta[1]) & mask, a.ph);
      W0x = make_float2(w0.x, w1.x);
      W0y = make_float2(w0.y, w1.y);
    }
    float2 Wx[RT], Wy[RT], NWy[RT], Sx[RT], Sy[RT];
    {
      const float2 NW0y = pk_neg(W0y);
      const float4 gl = gs4[(Nt - 1) * (Q / 2) + bp];
#pragma unroll
      for (int r = 0; r < RT; ++r) {
        if (r == 0) {
          Wx[r] = W0x;
          Wy[r] = W0y;
        } else {
          Wx[r] = pk_fma(W0x, pwx[r], pk_mul(NW0y, pwy[r]));
          Wy[r] = pk_fma(W0x, pwy[r], pk_mul(W0y, pwx[r]));
        }
        NWy[r] = pk_neg(Wy[r]);
        Sx[r] = make_float2(gl.x, gl.y);
        Sy[r] = make_float2(gl.z, gl.w);
      }
    }
    // Horner's rule over t for the thread's RT rates, both bases in the packed lanes
#pragma unroll 4
    for (int t = Nt - 2; t >= 0; --t) {
      const float4 gt = gs4[t * (Q / 2) + bp];
      const float2 gx = make_float2(gt.x, gt.y), gy = make_float2(gt.z, gt.w);
#pragma unroll
      for (int r = 0; r < RT; ++r) {
        const float2 tx = pk_fma(Sx[r], Wx[r], pk_fma(Sy[r], NWy[r], gx));
        const float2 ty = pk_fma(Sx[r], Wy[r], pk_fma(Sy[r], Wx[r], gy));
        Sx[r] = tx;
        Sy[r] = ty;
      }
    }
    __syncthreads();  // buf is free
#pragma unroll
    for (int up = 0; up < RT / 2; ++up) {
      const int u = rg * (RT / 2) + up;  // rate pair within the block
      const bool ok_a = j0 + 2 * up < a.Nr, ok_b = j0 + 2 * up + 1 < a.Nr;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const float wh = h ? win.y : win.x;
        const float2 sa = ok_a ? cscale(make_float2(h ? Sx[2 * up].y : Sx[2 * up].x,
                                                    h ? Sy[2 * up].y : Sy[2 * up].x), wh)
                               : make_float2(0.f, 0.f);
        const float2 sb = ok_b ? cscale(make_float2(h ? Sx[2 * up + 1].y : Sx[2 * up + 1].x,
                                                    h ? Sy[2 * up + 1].y : Sy[2 * up + 1].x), wh)
                               : make_float2(0.f, 0.f);
        if (dc && h == 0) {
          buf[(2 * u) * SS + pidx(0)] = make_float2(sa.x, sb.x);
        } else {
          buf[(2 * u + side) * SS + pidx(k20 + h)] = make_float2(sa.x - sb.y, sa.y + sb.x);
          buf[(2 * u + ms[h]) * SS + pidx(mk2[h])] = make_float2(sa.x + sb.y, sb.x - sa.y);
        }
      }
    }
    if (c == 0 && tid == 0) {
      const float wn = window_value(a, (long long)kny);
      for (int u = 0; u < kRatesPerBlock / 2; ++u) {
        float v[2];
        for (int hh = 0; hh < 2; ++hh) {
          const int j = 2 * q0 + 2 * u + hh;
          const float2 wv = cis_phase((alpha_n + (unsigned long long)(jb + 2 * u + hh) * beta_n) & mask, a.ph);
          float2 sv = gnyq[Nt - 1];
          for (int t = Nt - 2; t >= 0; --t)
            sv = make_float2(fmaf(sv.x, wv.x, fmaf(-sv.y, wv.y, gnyq[t].x)),
                             fmaf(sv.x, wv.y, fmaf(sv.y, wv.x, gnyq[t].y)));
          v[hh] = (j < a.Nr) ? sv.x * wn : 0.f;
        }
        buf[(2 * u) * SS + pidx(Q / 2)] = make_float2(v[0], v[1]);
      }
    }
    __syncthreads();
    float2* const W = a.W;
    const int k1a = k1s[0], k1b = k1s[1];
    smem_fft_emit<Q, kRatesPerBlock, SS, T, +1>(buf, twt, [&](int seq, int na, float2 v) {
      const int q = q0 + (seq >> 1), sd = seq & 1;
      if (q < q_end && FDR_DBG_OK(((long long)q * P + (sd ? k1b : k1a)) * Q + na < (long long)a.npairs * P * Q))
        W[((long long)q * P + (sd ? k1b : k1a)) * Q + na] = cmul(v, twr[sd * Q + na]);
    });
  }
}

// ------------------------------------------------------------------------------------
// Kernel B, warp-specialised (Q = 256 or 512, Nt <= NT): F of the CTA's Q bases in shared
// memory (pair-interleaved as for zdtf_czt_smem_kernel).  H = 256 Horner threads (one base
// pair each, RT = 8 or 4 rates of every 8-rate block, two bases per packed-FP32 lane pair)
// fill one of two rate-block buffers while the I = Q/2 FFT threads run the inverse DFT_Q of
// the other and write W.  The hand-over uses hardware named barriers (bar.sync / bar.arrive
// with thread counts, no polling):
//   FULL(i mod 2):  the Horner threads arrive once block i is in buffer i mod 2; the FFT
//                   threads wait on it before transforming block i;
//   EMPTY(i mod 2): the FFT threads arrive once they have read block i (when block i + 2
//                   exists); the Horner threads wait on it before writing block i + 2.
// The FFT phase (shared-memory latency and its own barriers) thus runs under the Horner phase
// instead of after it: measured 6-9% faster than zdtf_czt_smem_kernel at Nt = 32 and 64.
// (The Horner phase itself stays latency-bound; 512 Horner threads, or loads of F issued two
// steps ahead, measured no faster.)
// ------------------------------------------------------------------------------------
template <int Q>
struct CztWsShape {
  static constexpr int H = 256;                   // Horner threads
  static constexpr int RG = 2 * H / Q;            // rate groups: 1 (Q = 512) or 2 (Q = 256)
  static constexpr int RT = kRatesPerBlock / RG;  // rates of a block per Horner thread
  static constexpr int C = RT < 4 ? RT : 4;       // rates evaluated together
  static constexpr int I = Q / 2;                 // FFT threads
  static constexpr int T = H + I;
  static constexpr int SS = b_stride<Q>();
  static constexpr int BUF1 = kRatesPerBlock * SS;       // second rate-block buffer
  static constexpr int TWT = 2 * kRatesPerBlock * SS;    // DFT_Q twiddles (tw_size(Q))
  static constexpr int TWR = TWT + tw_size(Q);           // W twiddles (2 Q)
  static constexpr int GS_OFF = (TWR + 2 * Q + 1) & ~1;  // F, on a 16-byte boundary
  template <int NT>
  static constexpr size_t smem() { return sizeof(float2) * (GS_OFF + NT * Q + NT); }
};
constexpr int kBarFull = 1, kBarEmpty = 3, kBarFft = 5;

template <int Q, int NT>
__global__ void __launch_bounds__(CztWsShape<Q>::T, 1) zdtf_czt_ws_kernel(CztArgs a) {
  using SH = CztWsShape<Q>;
  constexpr int T = SH::T, H = SH::H, I = SH::I, RT = SH::RT, C = SH::C, SS = SH::SS;
  static_assert(RT % C == 0 && C % 2 == 0 && (Q / 2) % 32 == 0, "rate pairs; warp-uniform rate groups");
  extern __shared__ float2 sm[];
  float2* const buf0 = sm;
  float2* const buf1 = sm + SH::BUF1;
  float2* const twt = sm + SH::TWT;
  float2* const twr = sm + SH::TWR;
  float2* const gs = sm + SH::GS_OFF;
  float2* const gnyq = gs + NT * Q;
  const int tid = threadIdx.x;
  const int c = blockIdx.x;
  const int P = a.P;
  const int k1s[2] = {c == 0 ? 0 : c, c == 0 ? P / 2 : P - c};
  const float invN = 1.0f / (float)a.N;
  for (int i = tid; i < tw_size(Q); i += T) twt[i] = __ldg(a.tab.twQ + i);
  for (int i = tid; i < 2 * Q; i += T) {
    const int side = i / Q, na = i - side * Q;
    twr[i] = cscale(cconj(tw_fwd(a.tab, (long long)k1s[side] * na)), invN);
  }
  czt_forward_smem<Q, NT, T>(a, c, k1s, buf0, twt, gs, gnyq);  // ends with a barrier

  const int q_begin = blockIdx.y * a.pairs_per_group;
  const int q_end = min(a.npairs, q_begin + a.pairs_per_group);
  const int nblk = q_end > q_begin ? (q_end - q_begin + kRatesPerBlock / 2 - 1) / (kRatesPerBlock / 2) : 0;

  if (tid < H) {
    // ---------------- Horner threads ----------------
    const int bp = tid % (Q / 2), rg = tid / (Q / 2);
    const int b0 = 2 * bp;
    const int side = b0 / (Q / 2), k20 = b0 - side * (Q / 2);
    int ms[2], mk2[2];
    mirror_of(c, side, k20, Q, &ms[0], &mk2[0]);
    mirror_of(c, side, k20 + 1, Q, &ms[1], &mk2[1]);
    const bool dc = (c == 0 && side == 0 && k20 == 0);  // lane 0 is the DC bin
    const unsigned long long mask = a.ph.mask;
    unsigned long long alpha[2], beta[2];
    float2 pwx[C], pwy[C];  // exact w(k_lane, i*dr) for i = 1..C (lanes = the two bases)
    float2 win;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const unsigned long long k = (unsigned long long)k1s[side] + (unsigned long long)P * (k20 + h);
      alpha[h] = (k * a.ph.R0) & mask;
      beta[h] = (k * a.ph.Rd) & mask;
#pragma unroll
      for (int i = 1; i <= C; ++i) {
        const float2 p = cis_phase(((unsigned long long)i * beta[h]) & mask, a.ph);
        if (h == 0) { pwx[i - 1].x = p.x; pwy[i - 1].x = p.y; } else { pwx[i - 1].y = p.x; pwy[i - 1].y = p.y; }
      }
      const float wv = window_value(a, (long long)k);
      if (h == 0) win.x = wv; else win.y = wv;
    }
    const unsigned long long kny = (unsigned long long)(a.N / 2);
    const unsigned long long alpha_n = (kny * a.ph.R0) & mask, beta_n = (kny * a.ph.Rd) & mask;
    const int Nt = a.Nt;
    const float4* gs4 = reinterpret_cast<const float4*>(gs);
    for (int ib = 0; ib < nblk; ++ib) {
      const int q0 = q_begin + ib * (kRatesPerBlock / 2);
      float2* const hb = (ib & 1) ? buf1 : buf0;
      const int j0 = 2 * q0 + rg * RT;  // this thread's first rate of the block
      const long long jb = a.blk_base ? (long long)__ldg(a.blk_base + (q0 >> 2)) : (long long)(2 * q0);
      float2 Wbx, Wby;  // exact w(k_lane, first rate of the thread)
      {
        const unsigned long long jj = (unsigned long long)(jb + rg * RT);
        const float2 w0 = cis_phase((alpha[0] + jj * beta[0]) & mask, a.ph);
        const float2 w1 = cis_phase((alpha[1] + jj * beta[1]) & mask, a.ph);
        Wbx = make_float2(w0.x, w1.x);
        Wby = make_float2(w0.y, w1.y);
      }
#pragma unroll
      for (int ch = 0; ch < RT / C; ++ch) {  // chunks of C rates
        float2 Sx[C], Sy[C];
        const bool live = j0 + C * ch < a.Nr;  // uniform over the warp (rg is)
        if (live) {
          float2 W0x = Wbx, W0y = Wby;
          if (ch > 0) {  // w(first rate of the chunk) = wb * w(k, C*dr) (ch = 1 only: RT <= 2C)
            W0x = pk_fma(Wbx, pwx[C - 1], pk_mul(pk_neg(Wby), pwy[C - 1]));
            W0y = pk_fma(Wbx, pwy[C - 1], pk_mul(Wby, pwx[C - 1]));
          }
          const float2 NW0y = pk_neg(W0y);
          float2 Wx[C], Wy[C], NWy[C];
          const float4 gl = gs4[(Nt - 1) * (Q / 2) + bp];
#pragma unroll
          for (int r = 0; r < C; ++r) {
            if (r == 0) {
              Wx[r] = W0x;
              Wy[r] = W0y;
            } else {
              Wx[r] = pk_fma(W0x, pwx[r - 1], pk_mul(NW0y, pwy[r - 1]));
              Wy[r] = pk_fma(W0x, pwy[r - 1], pk_mul(W0y, pwx[r - 1]));
            }
            NWy[r] = pk_neg(Wy[r]);
            Sx[r] = make_float2(gl.x, gl.y);
            Sy[r] = make_float2(gl.z, gl.w);
          }
#pragma unroll 4
          for (int t = Nt - 2; t >= 0; --t) {
            const float4 gt = gs4[t * (Q / 2) + bp];
            const float2 gx = make_float2(gt.x, gt.y), gy = make_float2(gt.z, gt.w);
#pragma unroll
            for (int r = 0; r < C; ++r) {
              const float2 tx = pk_fma(Sx[r], Wx[r], pk_fma(Sy[r], NWy[r], gx));
              const float2 ty = pk_fma(Sx[r], Wy[r], pk_fma(Sy[r], Wx[r], gy));
              Sx[r] = tx;
              Sy[r] = ty;
            }
          }
        } else {
#pragma unroll
          for (int r = 0; r < C; ++r) Sx[r] = Sy[r] = make_float2(0.f, 0.f);
        }
        if (ch == 0 && ib >= 2) {  // the FFT threads have read this buffer's previous block
          if (ib & 1) named_sync<kBarEmpty + 1, T>(); else named_sync<kBarEmpty, T>();
        }
#pragma unroll
        for (int up = 0; up < C / 2; ++up) {
          const int u = rg * (RT / 2) + ch * (C / 2) + up;  // rate pair within the block
          const int ja = j0 + C * ch + 2 * up;
          const bool ok_a = ja < a.Nr, ok_b = ja + 1 < a.Nr;
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const float wh = h ? win.y : win.x;
            const float2 sa = ok_a ? cscale(make_float2(h ? Sx[2 * up].y : Sx[2 * up].x,
                                                        h ? Sy[2 * up].y : Sy[2 * up].x), wh)
                                   : make_float2(0.f, 0.f);
            const float2 sb = ok_b ? cscale(make_float2(h ? Sx[2 * up + 1].y : Sx[2 * up + 1].x,
                                                        h ? Sy[2 * up + 1].y : Sy[2 * up + 1].x), wh)
                                   : make_float2(0.f, 0.f);
            if (dc && h == 0) {
              hb[(2 * u) * SS + pidx(0)] = make_float2(sa.x, sb.x);
            } else {
              hb[(2 * u + side) * SS + pidx(k20 + h)] = make_float2(sa.x - sb.y, sa.y + sb.x);
              hb[(2 * u + ms[h]) * SS + pidx(mk2[h])] = make_float2(sa.x + sb.y, sb.x - sa.y);
            }
          }
        }
      }
      if (c == 0 && tid == 0) {  // the real-only Nyquist bin of every rate of the block
        const float wn = window_value(a, (long long)kny);
        for (int u = 0; u < kRatesPerBlock / 2; ++u) {
          float v[2];
          for (int hh = 0; hh < 2; ++hh) {
            const int j = 2 * q0 + 2 * u + hh;
            const float2 wv = cis_phase((alpha_n + (unsigned long long)(jb + 2 * u + hh) * beta_n) & mask, a.ph);
            float2 sv = gnyq[Nt - 1];
            for (int t = Nt - 2; t >= 0; --t)
              sv = make_float2(fmaf(sv.x, wv.x, fmaf(-sv.y, wv.y, gnyq[t].x)),
                               fmaf(sv.x, wv.y, fmaf(sv.y, wv.x, gnyq[t].y)));
            v[hh] = (j < a.Nr) ? sv.x * wn : 0.f;
          }
          hb[(2 * u) * SS + pidx(Q / 2)] = make_float2(v[0], v[1]);
        }
      }
      if (ib & 1) named_arrive<kBarFull + 1, T>(); else named_arrive<kBarFull, T>();
    }
  } else {
    // ---------------- FFT threads ----------------
    const int ltid = tid - H;
    const int k1a = k1s[0], k1b = k1s[1];
    for (int ib = 0; ib < nblk; ++ib) {
      const int q0 = q_begin + ib * (kRatesPerBlock / 2);
      float2* const hb = (ib & 1) ? buf1 : buf0;
      float2* const Wq = a.W + (long long)q0 * P * Q;  // 32-bit offsets below (Nf <= 2^22)
      if (ib & 1) named_sync<kBarFull + 1, T>(); else named_sync<kBarFull, T>();
      group_fft_emit<Q, kRatesPerBlock, SS, I, +1, kBarFft, 1>(hb, twt, ltid, [&](int seq, int na, float2 v) {
        const int p = seq >> 1, sd = seq & 1;
        const unsigned off = (unsigned)((p * P + (sd ? k1b : k1a)) * Q + na);
        if (q0 + p < q_end && FDR_DBG_OK((long long)q0 * P * Q + off < (long long)a.npairs * P * Q))
          Wq[off] = cmul(v, twr[sd * Q + na]);
      });
      if (ib + 2 < nblk) {
        if (ib & 1) named_arrive<kBarEmpty + 1, T>(); else named_arrive<kBarEmpty, T>();
      }
    }
  }
}

// ------------------------------------------------------------------------------------
// Kernel B for 32 < Nt <= 64 with 512 bins per residue pair (the split 2048 x 512 at Nf =
// 2^20 and 4096 x 512 at 2^21, instead of 4096 x 256 / 8192 x 256): F of 64 steps for 512
// bins (256 KB) does not fit one CTA, so a cluster of two CTAs shares the residue pair.  CTA
// rank s keeps F of side s (residue k1 or P - k1: 256 bins, 128 KB) and evaluates Horner's
// rule for them.  Each rate pair of a block has an owner (pairs 0 and 1: rank 0; 2 and 3:
// rank 1); every CTA writes its sums, at the direct and the mirror positions, into the
// owner's rate-block buffer through distributed shared memory.  One cluster barrier per
// block makes them visible, then each CTA runs the inverse DFT_Q of its own two rate pairs
// (4 sequences) and writes W.  The two rate-block buffers alternate, so a CTA may write into
// its peer's buffer for block i + 1 while the peer still transforms block i.
// ------------------------------------------------------------------------------------
// Forward DFT_Q for a two-CTA cluster (zdtf_czt_cl_kernel): CTA `rank` transforms only the A
// rows of its own side (PC = 8 t pairs per chunk, 8 sequences in buf) and takes the mirror
// values of the two-for-one unpacking from the CTA that holds the mirror side (itself for
// residue pair 0), through distributed shared memory.  Two cluster barriers per chunk: the
// peer's transforms are complete before they are read, and read before they are replaced.
template <int Q, int NT, int T>
__device__ __forceinline__ void czt_forward_cluster(const CztArgs& a, int c, const int* k1s, float2* buf,
                                                    const float2* twt, float2* gs, float2* gnyq,
                                                    int rank, cg::cluster_group& cluster) {
  constexpr int SS = b_stride<Q>();
  constexpr int PC = 8, QH = Q / 2;
  constexpr int NE = PC * Q, NL = (NE + T - 1) / T;
  const int tid = threadIdx.x;
  for (int i = tid; i < NT * QH; i += T) gs[i] = make_float2(0.f, 0.f);
  if (c == 0 && rank == 0 && tid == 0)
    for (int t = 0; t < NT; ++t) gnyq[t] = make_float2(0.f, 0.f);
  const long long k1 = k1s[rank];
  float2 v[NL];
  auto load_chunk = [&](int p0) {
#pragma unroll
    for (int i = 0; i < NL; ++i) {
      const int e = tid + i * T;
      const int u = e / Q, na = e - u * Q;
      const int pp = p0 + u;
      v[i] = ((NE % T == 0 || e < NE) && pp < a.NP &&
              FDR_DBG_OK(((long long)pp * a.P + k1) * Q + na < (long long)a.NP * a.P * Q))
                 ? __ldcs(a.A + ((long long)pp * a.P + k1) * Q + na)
                 : make_float2(0.f, 0.f);
    }
  };
  load_chunk(0);
  for (int p0 = 0; p0 < a.NP; p0 += PC) {
    if (p0 > 0) cluster.sync();  // the peer has read this buffer's previous chunk
#pragma unroll
    for (int i = 0; i < NL; ++i) {
      const int e = tid + i * T;
      const int u = e / Q, na = e - u * Q;
      if (NE % T == 0 || e < NE) buf[u * SS + pidx(na)] = v[i];
    }
    if (p0 + PC < a.NP) load_chunk(p0 + PC);
    __syncthreads();
    smem_fft<Q, PC, SS, T, -1>(buf, twt);
    cluster.sync();  // both sides' transforms of this chunk are complete
    for (int e = tid; e < PC * QH; e += T) {
      const int u = e / QH, k2 = e - u * QH;
      if (p0 + u >= a.NP) continue;
      int ms, mk2;
      mirror_of(c, rank, k2, Q, &ms, &mk2);
      const float2* src = ms == rank ? buf : cluster.map_shared_rank(buf, ms);
      const float2 zk = buf[u * SS + pidx(k2)];
      const float2 zm = cconj(src[u * SS + pidx(mk2)]);
      const float2 sm_ = cadd(zk, zm), d = csub(zk, zm);
      const int t0 = 2 * (p0 + u);
      gs_put(gs, QH, t0, k2, make_float2(0.5f * sm_.x, 0.5f * sm_.y));
      if (t0 + 1 < NT) gs_put(gs, QH, t0 + 1, k2, make_float2(0.5f * d.y, -0.5f * d.x));
    }
    if (c == 0 && rank == 0 && tid == 0) {
      for (int u = 0; u < PC && p0 + u < a.NP; ++u) {
        const float2 z = buf[u * SS + pidx(Q / 2)];
        const int t0 = 2 * (p0 + u);
        gnyq[t0] = make_float2(z.x, 0.f);
        if (t0 + 1 < NT) gnyq[t0 + 1] = make_float2(z.y, 0.f);
      }
    }
  }
  cluster.sync();  // every read of either buffer is done: they become rate-block buffers
}

struct CztClShape {
  static constexpr int Q = 512, NT = 64, T = 512;
  static constexpr int QH = Q / 2;                    // bins of one side (one CTA)
  static constexpr int RG = 2 * T / QH;               // rate groups: 4 (128 bin pairs)
  static constexpr int RT = kRatesPerBlock / RG;      // 2 rates (one rate pair) per thread
  static constexpr int SS = b_stride<Q>();
  static constexpr int TWT = 2 * kRatesPerBlock * SS;  // after two 8-sequence buffers
  static constexpr int TWR = TWT + tw_size(Q);
  static constexpr int GS_OFF = (TWR + 2 * Q + 1) & ~1;
  static constexpr size_t SMEM = sizeof(float2) * (GS_OFF + NT * QH + NT);
};

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(CztClShape::T, 1)
zdtf_czt_cl_kernel(CztArgs a) {
  using SH = CztClShape;
  constexpr int Q = SH::Q, NT = SH::NT, T = SH::T, QH = SH::QH, RT = SH::RT, SS = SH::SS;
  static_assert(RT == 2, "one rate pair per thread");
  cg::cluster_group cluster = cg::this_cluster();
  extern __shared__ float2 sm[];
  float2* const buf = sm;  // forward pass: 8 sequences; then two buffers of 8 (two rate blocks)
  float2* const twt = sm + SH::TWT;
  float2* const twr = sm + SH::TWR;
  float2* const gs = sm + SH::GS_OFF;
  float2* const gnyq = gs + NT * QH;
  const int tid = threadIdx.x;
  const int rank = (int)cluster.block_rank();  // the side this CTA holds
  const int c = blockIdx.x >> 1;                // residue pair
  const int P = a.P;
  const int k1s[2] = {c == 0 ? 0 : c, c == 0 ? P / 2 : P - c};
  const float invN = 1.0f / (float)a.N;
  for (int i = tid; i < tw_size(Q); i += T) twt[i] = __ldg(a.tab.twQ + i);
  for (int i = tid; i < 2 * Q; i += T) {
    const int sd = i / Q, na = i - sd * Q;
    twr[i] = cscale(cconj(tw_fwd(a.tab, (long long)k1s[sd] * na)), invN);
  }
  czt_forward_cluster<Q, NT, T>(a, c, k1s, buf, twt, gs, gnyq, rank, cluster);

  // thread -> (bin pair bp of this side, rate pair rg of every block)
  const int bp = tid % (QH / 2), rg = tid / (QH / 2);
  const int side = rank, k20 = 2 * bp;
  int ms[2], mk2[2];
  mirror_of(c, side, k20, Q, &ms[0], &mk2[0]);
  mirror_of(c, side, k20 + 1, Q, &ms[1], &mk2[1]);
  const bool dc = (c == 0 && side == 0 && k20 == 0);  // lane 0 is the DC bin
  const unsigned long long mask = a.ph.mask;
  unsigned long long alpha[2], beta[2];
  float2 pwx, pwy;  // exact w(k_lane, dr) (lanes = the two bins)
  float2 win;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const unsigned long long k = (unsigned long long)k1s[side] + (unsigned long long)P * (k20 + h);
    alpha[h] = (k * a.ph.R0) & mask;
    beta[h] = (k * a.ph.Rd) & mask;
    const float2 p = cis_phase(beta[h] & mask, a.ph);
    if (h == 0) { pwx.x = p.x; pwy.x = p.y; } else { pwx.y = p.x; pwy.y = p.y; }
    const float wv = window_value(a, (long long)k);
    if (h == 0) win.x = wv; else win.y = wv;
  }
  const unsigned long long kny = (unsigned long long)(a.N / 2);
  const unsigned long long alpha_n = (kny * a.ph.R0) & mask, beta_n = (kny * a.ph.Rd) & mask;
  const int Nt = a.Nt;
  const float4* gs4 = reinterpret_cast<const float4*>(gs);
  const int owner = rg >> 1, ul = rg & 1;  // this thread's rate pair: owner CTA, pair there
  const int k1a = k1s[0], k1b = k1s[1];

  const int q_begin = blockIdx.y * a.pairs_per_group;
  const int q_end = min(a.npairs, q_begin + a.pairs_per_group);
  const int nblk = q_end > q_begin ? (q_end - q_begin + kRatesPerBlock / 2 - 1) / (kRatesPerBlock / 2) : 0;
  // two rate blocks per cluster barrier: 8 sequences per buffer ([block 0: 4][block 1: 4])
  const int nsb = (nblk + 1) / 2;
  for (int isb = 0; isb < nsb; ++isb) {
    float2* const hb_local = buf + (isb & 1) * kRatesPerBlock * SS;  // 8 sequences
    float2* const hb_owner = owner == rank ? hb_local : cluster.map_shared_rank(hb_local, owner);
#pragma unroll 1
    for (int bb = 0; bb < 2; ++bb) {
      const int ib = 2 * isb + bb;
      const bool live = ib < nblk;  // an odd last block leaves the second half unused
      const int q0 = q_begin + ib * (kRatesPerBlock / 2);
      float2* const hb = hb_owner + bb * 4 * SS;
      const int j0 = 2 * q0 + rg * RT;  // this thread's first rate of the block
      const long long jb = !live ? 0 : a.blk_base ? (long long)__ldg(a.blk_base + (q0 >> 2)) : (long long)(2 * q0);
      float2 Sx[2], Sy[2];
      if (live && j0 < a.Nr) {  // uniform over the warp (rg is)
        float2 W0x, W0y;
        {
          const unsigned long long jj = (unsigned long long)(jb + rg * RT);
          const float2 w0 = cis_phase((alpha[0] + jj * beta[0]) & mask, a.ph);
          const float2 w1 = cis_phase((alpha[1] + jj * beta[1]) & mask, a.ph);
          W0x = make_float2(w0.x, w1.x);
          W0y = make_float2(w0.y, w1.y);
        }
        const float2 NW0y = pk_neg(W0y);
        float2 Wx[2], Wy[2], NWy[2];
        Wx[0] = W0x;
        Wy[0] = W0y;
        Wx[1] = pk_fma(W0x, pwx, pk_mul(NW0y, pwy));
        Wy[1] = pk_fma(W0x, pwy, pk_mul(W0y, pwx));
        NWy[0] = NW0y;
        NWy[1] = pk_neg(Wy[1]);
        const float4 gl = gs4[(Nt - 1) * (QH / 2) + bp];
#pragma unroll
        for (int r = 0; r < 2; ++r) {
          Sx[r] = make_float2(gl.x, gl.y);
          Sy[r] = make_float2(gl.z, gl.w);
        }
#pragma unroll 4
        for (int t = Nt - 2; t >= 0; --t) {
          const float4 gt = gs4[t * (QH / 2) + bp];
          const float2 gx = make_float2(gt.x, gt.y), gy = make_float2(gt.z, gt.w);
#pragma unroll
          for (int r = 0; r < 2; ++r) {
            const float2 tx = pk_fma(Sx[r], Wx[r], pk_fma(Sy[r], NWy[r], gx));
            const float2 ty = pk_fma(Sx[r], Wy[r], pk_fma(Sy[r], Wx[r], gy));
            Sx[r] = tx;
            Sy[r] = ty;
          }
        }
      } else {
        Sx[0] = Sx[1] = Sy[0] = Sy[1] = make_float2(0.f, 0.f);
      }
      const bool ok_a = live && j0 < a.Nr, ok_b = live && j0 + 1 < a.Nr;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const float wh = h ? win.y : win.x;
        const float2 sa = ok_a ? cscale(make_float2(h ? Sx[0].y : Sx[0].x, h ? Sy[0].y : Sy[0].x), wh)
                               : make_float2(0.f, 0.f);
        const float2 sb = ok_b ? cscale(make_float2(h ? Sx[1].y : Sx[1].x, h ? Sy[1].y : Sy[1].x), wh)
                               : make_float2(0.f, 0.f);
        if (dc && h == 0) {
          hb[(2 * ul) * SS + pidx(0)] = make_float2(sa.x, sb.x);
        } else {
          hb[(2 * ul + side) * SS + pidx(k20 + h)] = make_float2(sa.x - sb.y, sa.y + sb.x);
          hb[(2 * ul + ms[h]) * SS + pidx(mk2[h])] = make_float2(sa.x + sb.y, sb.x - sa.y);
        }
      }
      if (c == 0 && rank == 0 && tid == 0) {  // the real-only Nyquist bin of every rate of the block
        const float wn = window_value(a, (long long)kny);
        for (int u = 0; u < kRatesPerBlock / 2; ++u) {
          float v[2];
          for (int hh = 0; hh < 2; ++hh) {
            const int j = 2 * q0 + 2 * u + hh;
            float2 sv = make_float2(0.f, 0.f);
            if (live) {
              const float2 wv = cis_phase((alpha_n + (unsigned long long)(jb + 2 * u + hh) * beta_n) & mask, a.ph);
              sv = gnyq[Nt - 1];
              for (int t = Nt - 2; t >= 0; --t)
                sv = make_float2(fmaf(sv.x, wv.x, fmaf(-sv.y, wv.y, gnyq[t].x)),
                                 fmaf(sv.x, wv.y, fmaf(sv.y, wv.x, gnyq[t].y)));
            }
            v[hh] = (live && j < a.Nr) ? sv.x * wn : 0.f;
          }
          float2* const hbo = ((u >> 1) == rank ? hb_local : cluster.map_shared_rank(hb_local, u >> 1)) + bb * 4 * SS;
          hbo[(2 * (u & 1)) * SS + pidx(Q / 2)] = make_float2(v[0], v[1]);
        }
      }
    }
    cluster.sync();  // both blocks' sums, local and remote, are in the owners' buffers
    // the inverse DFT_Q of this CTA's rate pairs 2*rank, 2*rank + 1 of both blocks (8
    // sequences); the last pass writes W
    smem_fft_emit<Q, 2 * kRatesPerBlock / 2, SS, T, +1>(hb_local, twt, [&](int ls, int na, float2 v) {
      const int bb = ls >> 2, lq = ls & 3;
      const int q0 = q_begin + (2 * isb + bb) * (kRatesPerBlock / 2);
      const int p = 2 * rank + (lq >> 1), sd = lq & 1;
      const unsigned off = (unsigned)((p * P + (sd ? k1b : k1a)) * Q + na);
      if (q0 + p < q_end && FDR_DBG_OK((long long)q0 * P * Q + off < (long long)a.npairs * P * Q))
        a.W[(long long)q0 * P * Q + off] = cmul(v, twr[sd * Q + na]);
    });
  }
}

// A -> F (reference layout K x Nt) for the split of zdtf_czt_cl_kernel: CTA 2c + s writes the
// F of side s of residue pair c (no cluster: the two sides are independent here).
__global__ void __launch_bounds__(CztClShape::T, 1) zdtf_a2f_half_kernel(CztArgs a) {
  using SH = CztClShape;
  constexpr int Q = SH::Q, NT = SH::NT, T = SH::T, QH = SH::QH;
  extern __shared__ float2 sm[];
  float2* const buf = sm;
  float2* const twt = sm + SH::TWT;
  float2* const gs = sm + SH::GS_OFF;
  float2* const gnyq = gs + NT * QH;
  const int tid = threadIdx.x;
  const int side = blockIdx.x & 1, c = blockIdx.x >> 1;
  const int P = a.P;
  const int k1s[2] = {c == 0 ? 0 : c, c == 0 ? P / 2 : P - c};
  for (int i = tid; i < tw_size(Q); i += T) twt[i] = __ldg(a.tab.twQ + i);
  czt_forward_smem<Q, NT, T, true>(a, c, k1s, buf, twt, gs, gnyq, side);
  const long long K = a.N / 2 + 1;
  for (int e = tid; e < QH * a.Nt; e += T) {
    const int t = e / QH, k2 = e - t * QH;
    if (FDR_DBG_OK((long long)k1s[side] + (long long)P * k2 + t * K < K * a.Nt))
      a.F[(long long)k1s[side] + (long long)P * k2 + t * K] = gs_get(gs, QH, t, k2);
  }
  if (c == 0 && side == 0 && tid == 0)
    for (int t = 0; t < a.Nt; ++t) a.F[a.N / 2 + t * K] = gnyq[t];
}

template <int Q, int NT>
__global__ void __launch_bounds__(CztSmemShape<Q>::T, 1) zdtf_a2f_smem_kernel(CztArgs a) {
  using SH = CztSmemShape<Q>;
  constexpr int T = SH::T;
  constexpr int SS = b_stride<Q>();
  extern __shared__ float2 sm[];
  float2* buf = sm;
  float2* twt = buf + kRatesPerBlock * SS;
  float2* twr = twt + tw_size(Q);
  float2* gs = sm + SH::GS_OFF;
  float2* gnyq = gs + NT * Q;
  const int tid = threadIdx.x;
  const int c = blockIdx.x;
  const int P = a.P;
  const int k1s[2] = {c == 0 ? 0 : c, c == 0 ? P / 2 : P - c};
  for (int i = tid; i < tw_size(Q); i += T) twt[i] = __ldg(a.tab.twQ + i);
  czt_forward_smem<Q, NT>(a, c, k1s, buf, twt, gs, gnyq);
  const long long K = a.N / 2 + 1;
  for (int e = tid; e < Q * a.Nt; e += T) {
    const int t = e / Q, b = e - t * Q;
    const int side = b / (Q / 2), k2 = b - side * (Q / 2);
    if (FDR_DBG_OK((long long)k1s[side] + (long long)P * k2 + t * K < K * a.Nt))
      a.F[(long long)k1s[side] + (long long)P * k2 + t * K] = gs_get(gs, Q, t, b);
  }
  if (c == 0 && tid == 0)
    for (int t = 0; t < a.Nt; ++t) a.F[a.N / 2 + t * K] = gnyq[t];
}

// A -> F (reference layout K x Nt) for the staged stages after a fused input!.
template <int Q, int NTR>
__global__ void __launch_bounds__(Q / 2, 1) zdtf_a2f_kernel(CztArgs a) {
  constexpr int T = Q / 2;
  constexpr int SS = b_stride<Q>();
  extern __shared__ float2 sm[];
  float2* buf = sm;
  float2* twt = buf + kRatesPerBlock * SS;
  float2* twr = twt + tw_size(Q);
  float2* gnyq = twr + 2 * Q;
  const int tid = threadIdx.x;
  const int c = blockIdx.x;
  const int P = a.P;
  const int k1s[2] = {c == 0 ? 0 : c, c == 0 ? P / 2 : P - c};
  for (int i = tid; i < tw_size(Q); i += T) twt[i] = __ldg(a.tab.twQ + i);
  float2 G[2][NTR];
  czt_forward<Q, NTR>(a, c, k1s, buf, twt, gnyq, G);
  const long long K = a.N / 2 + 1;
#pragma unroll
  for (int b = 0; b < 2; ++b) {
    const long long k = (long long)k1s[b] + (long long)P * tid;
#pragma unroll
    for (int t = 0; t < NTR; ++t)
      if (t < a.Nt) a.F[k + t * K] = G[b][t];
  }
  if (c == 0 && tid == 0) {
    for (int t = 0; t < a.Nt; ++t) a.F[a.N / 2 + t * K] = gnyq[t];
  }
}

// ------------------------------------------------------------------------------------
// Kernel C: inverse four-step pass 2.  grid (Q/TC, pairs).
// ------------------------------------------------------------------------------------
template <int P, int TC, int T>
__global__ void __launch_bounds__(T)
zdtf_output_kernel(const float2* __restrict__ W, long long N, int Q, int Nr, float* __restrict__ dest,
                   FusedTables tab, double* __restrict__ acc) {
  constexpr int SS = ac_stride<P, TC>();
  constexpr int TP = TC / 2;
  extern __shared__ float2 sm[];
  float2* buf = sm;
  float2* twt = sm + TC * SS;
  const int na0 = blockIdx.x * TC;
  const int q = blockIdx.y;
  for (int i = threadIdx.x; i < tw_size(P); i += T) twt[i] = __ldg(tab.twP + i);
  const float2* w = W + (long long)q * P * Q;
  static_assert((TP * P) % T == 0, "tile must divide evenly");
  constexpr int NL = TP * P / T;  // loads per thread: all issued before any is consumed
  {
    float4 v[NL];
#pragma unroll
    for (int i = 0; i < NL; ++i) {
      const int e = threadIdx.x + i * T;
      const int sp = e % TP, k1 = e / TP;
      v[i] = __ldcs(reinterpret_cast<const float4*>(w + (long long)k1 * Q + na0 + 2 * sp));
    }
#pragma unroll
    for (int i = 0; i < NL; ++i) {
      const int e = threadIdx.x + i * T;
      const int sp = e % TP, k1 = e / TP;
      buf[(2 * sp) * SS + pidx(k1)] = make_float2(v[i].x, v[i].y);
      buf[(2 * sp + 1) * SS + pidx(k1)] = make_float2(v[i].z, v[i].w);
    }
  }
  __syncthreads();
  smem_fft<P, TC, SS, T, +1>(buf, twt);
  const int j = 2 * q;
  float* d0 = dest + (long long)j * N;
  float* d1 = dest + (long long)(j + 1) * N;
  const bool has1 = (j + 1) < Nr;
  double m[4] = {0.0, 0.0, 0.0, 0.0};
  for (int e = threadIdx.x; e < TP * P; e += T) {
    const int sp = e % TP, nb = e / TP;
    const long long n = (long long)(na0 + 2 * sp) + (long long)Q * nb;
    const float2 v0 = buf[(2 * sp) * SS + pidx(nb)];
    const float2 v1 = buf[(2 * sp + 1) * SS + pidx(nb)];
    if (FDR_DBG_OK(n + 2 <= N && j < Nr)) __stcs(reinterpret_cast<float2*>(d0 + n), make_float2(v0.x, v1.x));
    if (has1 && FDR_DBG_OK(n + 2 <= N)) __stcs(reinterpret_cast<float2*>(d1 + n), make_float2(v0.y, v1.y));
    if (acc) {
      m[0] += (double)v0.x + (double)v1.x;
      m[1] += (double)v0.x * v0.x + (double)v1.x * v1.x;
      if (has1) {
        m[2] += (double)v0.y + (double)v1.y;
        m[3] += (double)v0.y * v0.y + (double)v1.y * v1.y;
      }
    }
  }
  if (acc) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
      for (int o = 16; o > 0; o >>= 1) m[i] += __shfl_down_sync(0xffffffffu, m[i], o);
    __shared__ double red[4][T / 32];
    const int wid = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0)
      for (int i = 0; i < 4; ++i) red[i][wid] = m[i];
    __syncthreads();
    if (threadIdx.x < 4) {
      double t = 0.0;
      for (int i = 0; i < T / 32; ++i) t += red[threadIdx.x][i];
      if (threadIdx.x < 2 || has1) atomicAdd(acc + 2 * j + threadIdx.x, t);
    }
  }
}

// Kernel C for P = P1 * P2 (P1, P2 in {8, 16, 32}): two register passes with one
// shared-memory transpose.  k1 = k1a + P1*k1b, nb = nb_b + P2*nb_a:
//   z[nb_b + P2*nb_a] = sum_k1a w_P1^(k1a*nb_a) * w_P^(k1a*nb_b) * sum_k1b X[k1a + P1*k1b] w_P2^(k1b*nb_b)
// Thread (seq, k1a) loads its P2 inputs straight from W, transforms them in registers,
// applies the twiddle and writes them transposed; thread (seq, nb_b) then transforms over
// k1a and writes its P1 outputs (two rates of the pair) to the FDR columns.
template <int P1, int P2, int TS>
struct Out2Shape {
  static constexpr int P = P1 * P2;
  static constexpr int T = TS * (P1 > P2 ? P1 : P2);
  static constexpr int S1 = P2 + 1;                       // k1a stride (float2)
  static constexpr int SSEQ = ((P1 * S1 + 15) / 16) * 16 + 2;  // sequence stride, = 2 mod 16
  static constexpr size_t SMEM = sizeof(float2) * (TS * SSEQ + P);
};

template <int P1, int P2, int TS>
__global__ void __launch_bounds__(Out2Shape<P1, P2, TS>::T)
zdtf_output2_kernel(const float2* __restrict__ W, long long N, int Q, int Nr,
                    float* __restrict__ dest, const float2* __restrict__ rootsP,
                    double* __restrict__ acc) {
  using SH = Out2Shape<P1, P2, TS>;
  constexpr int P = SH::P, S1 = SH::S1, SSEQ = SH::SSEQ;
  extern __shared__ float2 sm[];
  float2* buf = sm;
  float2* roots = sm + TS * SSEQ;  // exp(-2 pi i m / P)
  const int na0 = blockIdx.x * TS;
  const int q = blockIdx.y;
  for (int i = threadIdx.x; i < P; i += SH::T) roots[i] = __ldg(rootsP + i);
  const int seq = threadIdx.x % TS;
  const int r = threadIdx.x / TS;  // k1a in pass 1, nb_b in pass 2
  const float2* w = W + (long long)q * P * Q + na0 + seq;
  __syncthreads();
  if (r < P1) {
    float2 v[P2];
#pragma unroll
    for (int m = 0; m < P2; ++m) v[m] = __ldcs(w + (long long)(r + P1 * m) * Q);
    Dft<P2>::run(v, +1);
    float2* b = buf + seq * SSEQ + r * S1;
#pragma unroll
    for (int nbb = 0; nbb < P2; ++nbb) {
      const float2 t = roots[(r * nbb) & (P - 1)];
      b[nbb] = cmul(v[nbb], make_float2(t.x, -t.y));
    }
  }
  __syncthreads();
  const int j = 2 * q;
  const bool has1 = (j + 1) < Nr;
  double m[4] = {0.0, 0.0, 0.0, 0.0};  // sum and sum of squares of the two columns
  if (r < P2) {
    float2 v[P1];
    const float2* b = buf + seq * SSEQ + r;
#pragma unroll
    for (int k1a = 0; k1a < P1; ++k1a) v[k1a] = b[k1a * S1];
    Dft<P1>::run(v, +1);
    float* d0 = dest + (long long)j * N + na0 + seq + (long long)Q * r;
    float* d1 = d0 + N;
#pragma unroll
    for (int nba = 0; nba < P1; ++nba) {
      const long long off = (long long)Q * P2 * nba;
      if (FDR_DBG_OK(na0 + seq + (long long)Q * r + off < N && j < Nr)) __stcs(d0 + off, v[nba].x);
      if (has1 && FDR_DBG_OK(na0 + seq + (long long)Q * r + off < N)) __stcs(d1 + off, v[nba].y);
    }
    if (acc) {
#pragma unroll
      for (int nba = 0; nba < P1; ++nba) {
        const double x = v[nba].x, y = has1 ? v[nba].y : 0.f;
        m[0] += x; m[1] += x * x; m[2] += y; m[3] += y * y;
      }
    }
  }
  if (acc) {  // block reduction of the column moments, then one atomic add per value
#pragma unroll
    for (int i = 0; i < 4; ++i)
      for (int o = 16; o > 0; o >>= 1) m[i] += __shfl_down_sync(0xffffffffu, m[i], o);
    __shared__ double red[4][SH::T / 32];
    const int wid = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0)
      for (int i = 0; i < 4; ++i) red[i][wid] = m[i];
    __syncthreads();
    if (threadIdx.x < 4) {
      double t = 0.0;
      for (int i = 0; i < SH::T / 32; ++i) t += red[threadIdx.x][i];
      if (threadIdx.x < 2 || has1) atomicAdd(acc + 2 * j + threadIdx.x, t);
    }
  }
}

// ------------------------------------------------------------------------------------
// Output pass with TMA (P = P1*P2 = 1024, split as in zdtf_output2_kernel): a persistent
// grid, two CTAs per SM, walks the (rate pair, 8-residue) tiles; each tile's W (1024 k1
// rows x 8 complex, 64 KB) is fetched by the tensor-memory accelerator as four 256-row
// boxes completing on an mbarrier.  Waits on the mbarrier are bounded by kTmaWaitNs of
// %globaltimer; a wait that runs out sets g_fused_fault and the CTA returns (reported by
// fdr_synchronize).
// ------------------------------------------------------------------------------------
__device__ int g_fused_fault;
constexpr unsigned long long kTmaWaitNs = 1000000000ull;  // 1 s

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity,
                                                  unsigned long long limit_ns = kTmaWaitNs) {
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait(bar, parity))
    if (global_ns() - t0 > limit_ns) return false;
  return true;
}

// Self-test of the bounded wait: one CTA waits on an mbarrier that nothing completes, gives
// up after limit_ns and raises the fault flag exactly as the TMA kernels do.
__global__ void bounded_wait_selftest_kernel(unsigned long long limit_ns) {
  __shared__ unsigned long long bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const bool ok = mbar_wait_bounded(&bar, 0u, limit_ns);
  if (__syncthreads_or(!ok) && threadIdx.x == 0) atomicOr(&g_fused_fault, 8);
}
// FDR store of one row of a rate pair through lane pairs: v = (rate j, rate j + 1) values of
// this lane's channel; lanes 2s and 2s + 1 hold adjacent channels, so the even lane writes
// both channels of rate j and the odd lane both of rate j + 1 as one 8-byte streaming store
// each (half the store instructions of per-lane scalar stores).  Every lane of the warp
// must call it; d0 is this lane's element of rate j, d1 = d0 + Nf.
__device__ __forceinline__ void store_rate_pair(float* d0, float* d1, float2 v, bool odd, bool has1,
                                                const float* dlo, const float* dhi) {
  const float recv = __shfl_xor_sync(0xffffffffu, odd ? v.x : v.y, 1);
  if (!odd) {
    if (FDR_DBG_OK(d0 >= dlo && d0 + 2 <= dhi)) __stcs(reinterpret_cast<float2*>(d0), make_float2(v.x, recv));
  } else if (has1) {
    if (FDR_DBG_OK(d1 - 1 >= dlo && d1 + 1 <= dhi)) __stcs(reinterpret_cast<float2*>(d1 - 1), make_float2(recv, v.y));
  }
}

// 2-D tiled TMA load (no multicast) of box {x .. x+15 floats, y .. y+255 rows} into dst.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      ::"r"(smem_addr(dst)), "l"((unsigned long long)map), "r"(x), "r"(y), "r"(smem_addr(bar))
      : "memory");
}

// 3-D tiled TMA load (no multicast) of box {x .. x+15 floats, y .. y+31, z .. z+31} into dst.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(smem_addr(dst)), "l"((unsigned long long)map), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
      : "memory");
}

// The W tile lands (TMA) in a region that pass 1 then overwrites with its transposed
// output, so a CTA needs ~76 KB and two fit per SM; the next tile's fetch is issued as soon
// as pass 2 has read the region, overlapping pass 2's DFTs and FDR stores (and the other
// CTA's work).
template <int P1, int P2, int TS>
struct OutTmaShape {
  static constexpr int P = P1 * P2;
  static constexpr int T = TS * (P1 > P2 ? P1 : P2);
  static constexpr int S1 = P2 + 1;
  static constexpr int SSEQ = ((P1 * S1 + 15) / 16) * 16 + 2;
  static constexpr int BOXR = 256;
  static constexpr int NBOX = P / BOXR;
  static constexpr unsigned TILEB = sizeof(float2) * P * TS;
  static constexpr size_t REGION = sizeof(float2) * TS * SSEQ > TILEB ? sizeof(float2) * TS * SSEQ : TILEB;
  static constexpr size_t SMEM = 128 + ((REGION + 127) / 128) * 128 + sizeof(float2) * P + 16;
  static constexpr int MINB = 2;  // CTAs per SM
};

template <int P1, int P2, int TS>
__global__ void __launch_bounds__(OutTmaShape<P1, P2, TS>::T, OutTmaShape<P1, P2, TS>::MINB)
zdtf_output_tma_kernel(const __grid_constant__ CUtensorMap wmap, long long N, int Q, int Nr,
                        int npairs, float* __restrict__ dest, const float2* __restrict__ rootsP,
                        double* __restrict__ acc) {
  using SH = OutTmaShape<P1, P2, TS>;
  constexpr int P = SH::P, S1 = SH::S1, SSEQ = SH::SSEQ;
  extern __shared__ unsigned char smraw[];
  const uintptr_t base = ((uintptr_t)smraw + 127) & ~(uintptr_t)127;
  float2* region = (float2*)base;
  float2* roots = (float2*)(base + ((SH::REGION + 127) / 128) * 128);
  unsigned long long* bar = (unsigned long long*)(roots + P);
  const int tid = threadIdx.x;
  const int ntna = Q / TS;
  const long long ntiles = (long long)ntna * npairs;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int i = tid; i < P; i += SH::T) roots[i] = __ldg(rootsP + i);
  __syncthreads();
  auto issue = [&](long long tile) {  // thread 0 only
    const int q = (int)(tile / ntna), nat = (int)(tile - (long long)q * ntna);
    mbar_expect_tx(&bar[0], SH::TILEB);
#pragma unroll
    for (int b = 0; b < SH::NBOX; ++b)
      tma_load_2d(region + b * SH::BOXR * TS, &wmap, 2 * TS * nat, q * P + b * SH::BOXR, &bar[0]);
  };
  const long long first = blockIdx.x, stride = gridDim.x;
  if (tid == 0 && first < ntiles) issue(first);
  const int seq = tid % TS;
  const int r = tid / TS;
  int it = 0;
  for (long long tile = first; tile < ntiles; tile += stride, ++it) {
    const bool ok = mbar_wait_bounded(&bar[0], (unsigned)(it & 1));
    if (__syncthreads_or(!ok)) {
      if (tid == 0) atomicOr(&g_fused_fault, 1);
      return;
    }
    const int q = (int)(tile / ntna), nat = (int)(tile - (long long)q * ntna);
    const int na0 = nat * TS;
    float2 v[P2];
    if (r < P1) {
#pragma unroll
      for (int m = 0; m < P2; ++m) v[m] = region[(r + P1 * m) * TS + seq];
    }
    __syncthreads();  // the tile is in registers: the region takes the transpose
    if (r < P1) {
      Dft<P2>::run(v, +1);
      float2* b = region + seq * SSEQ + r * S1;
#pragma unroll
      for (int nbb = 0; nbb < P2; ++nbb) {
        const float2 t = roots[(r * nbb) & (P - 1)];
        b[nbb] = cmul(v[nbb], make_float2(t.x, -t.y));
      }
    }
    __syncthreads();
    const int j = 2 * q;
    const bool has1 = (j + 1) < Nr;
    float2 w[P1];
    if (r < P2) {
      const float2* b = region + seq * SSEQ + r;
#pragma unroll
      for (int k1a = 0; k1a < P1; ++k1a) w[k1a] = b[k1a * S1];
    }
    __syncthreads();  // the region is read: fetch the next tile into it
    if (tid == 0 && tile + stride < ntiles) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(tile + stride);
    }
    double m[4] = {0.0, 0.0, 0.0, 0.0};
    static_assert(SH::T == TS * P2 && TS % 2 == 0, "every lane stores, channel pairs in lane pairs");
    if (r < P2) {
      Dft<P1>::run(w, +1);
      float* d0 = dest + (long long)j * N + na0 + seq + (long long)Q * r;
      float* d1 = d0 + N;
#pragma unroll
      for (int nba = 0; nba < P1; ++nba) {
        const long long off = (long long)Q * P2 * nba;
        store_rate_pair(d0 + off, d1 + off, w[nba], seq & 1, has1, dest, dest + N * (long long)Nr);
      }
      if (acc) {
#pragma unroll
        for (int nba = 0; nba < P1; ++nba) {
          const double x = w[nba].x, y = has1 ? w[nba].y : 0.f;
          m[0] += x; m[1] += x * x; m[2] += y; m[3] += y * y;
        }
      }
    }
    if (acc) {
#pragma unroll
      for (int i = 0; i < 4; ++i)
        for (int o = 16; o > 0; o >>= 1) m[i] += __shfl_down_sync(0xffffffffu, m[i], o);
      __shared__ double red[4][SH::T / 32];
      const int wid = tid >> 5;
      if ((tid & 31) == 0)
        for (int i = 0; i < 4; ++i) red[i][wid] = m[i];
      __syncthreads();
      if (tid < 4) {
        double t = 0.0;
        for (int i = 0; i < SH::T / 32; ++i) t += red[tid][i];
        if (tid < 2 || has1) atomicAdd(acc + 2 * j + tid, t);
      }
      __syncthreads();  // red is free for the next tile
    }
  }
}

// ------------------------------------------------------------------------------------
// Output pass with TMA for P = 2048 = 64 x 32 (the four-step split of Nf = 2^20 with 512
// bins per czt CTA).  As zdtf_output_tma_kernel, with 8 residues per tile (2048 rows x
// 64 B = 128 KB, one CTA of 512 threads per SM; tiles of 4 residues, 32-byte rows, two
// CTAs per SM, measured 4x slower).  Pass 1: thread (seq, k1a < 64) transforms its 32
// values over k1b.  Pass 2 (the 64-point DFT over k1a) is split between lanes h = 0, 1 of a
// warp (decimation in time): lane h transforms the 32 values k1a = 2k + h, lane 1 applies
// w_64^n, and the two exchange half of their results by shuffles, so every lane ends with
// 32 of the 64 outputs.
// Shared-memory strides: S1 = 33 (odd) and SSEQ = 16/TS (mod 16) keep the transposed
// writes of pass 1 (TS seq x 16/TS k1a per half-warp) and the reads of pass 2 (TS seq x
// 16/TS nb_b per half-warp, h fixed) on distinct bank pairs.
// ------------------------------------------------------------------------------------
template <int TS_>
struct OutTma64Shape {
  static constexpr int P1 = 64, P2 = 32, P = P1 * P2, TS = TS_, T = 64 * TS;
  static constexpr int S1 = P2 + 1;
  static constexpr int SSEQ = ((P1 * S1 + 15) / 16) * 16 + 16 / TS;
  static constexpr int BOXR = 256;
  static constexpr int NBOX = P / BOXR;
  static constexpr unsigned TILEB = sizeof(float2) * P * TS;
  static constexpr size_t REGION = sizeof(float2) * TS * SSEQ > TILEB ? sizeof(float2) * TS * SSEQ : TILEB;
  // tables: tw1[k1a][n] = conj w^(k1a n) (pass 1: one row per thread, rows S1 apart so the
  // two rows a half-warp reads sit in different banks), tw2[n] = conj w64^n
  static constexpr int TW1 = P1 * S1;
  static constexpr size_t SMEM = 128 + ((REGION + 127) / 128) * 128 + sizeof(float2) * (TW1 + P1 / 2) + 16;
  static constexpr int MINB = TS <= 4 ? 2 : 1;
};

template <int TS_>
__global__ void __launch_bounds__(OutTma64Shape<TS_>::T, OutTma64Shape<TS_>::MINB)
zdtf_output_tma64_kernel(const __grid_constant__ CUtensorMap wmap, long long N, int Q, int Nr,
                         int npairs, float* __restrict__ dest, const float2* __restrict__ rootsP,
                         double* __restrict__ acc) {
  using SH = OutTma64Shape<TS_>;
  constexpr int P = SH::P, P1 = SH::P1, P2 = SH::P2, TS = SH::TS, S1 = SH::S1, SSEQ = SH::SSEQ;
  extern __shared__ unsigned char smraw[];
  const uintptr_t base = ((uintptr_t)smraw + 127) & ~(uintptr_t)127;
  float2* region = (float2*)base;
  float2* tw1 = (float2*)(base + ((SH::REGION + 127) / 128) * 128);  // P1 rows of S1
  float2* tw2 = tw1 + SH::TW1;                                          // P1 / 2
  unsigned long long* bar = (unsigned long long*)(tw2 + P1 / 2);
  const int tid = threadIdx.x;
  const int ntna = Q / TS;
  const long long ntiles = (long long)ntna * npairs;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int i = tid; i < P; i += SH::T)
    tw1[(i / P2) * S1 + i % P2] = cconj(__ldg(rootsP + (((i / P2) * (i % P2)) & (P - 1))));
  for (int i = tid; i < P1 / 2; i += SH::T) tw2[i] = cconj(__ldg(rootsP + i * (P / P1)));
  __syncthreads();
  auto issue = [&](long long tile) {  // thread 0 only
    const int q = (int)(tile / ntna), nat = (int)(tile - (long long)q * ntna);
    mbar_expect_tx(&bar[0], SH::TILEB);
#pragma unroll
    for (int b = 0; b < SH::NBOX; ++b)
      tma_load_2d(region + b * SH::BOXR * TS, &wmap, 2 * TS * nat, q * P + b * SH::BOXR, &bar[0]);
  };
  const long long first = blockIdx.x, stride = gridDim.x;
  if (tid == 0 && first < ntiles) issue(first);
  // pass 1 roles
  const int seq1 = tid % TS, r = tid / TS;  // r = k1a < 64
  // pass 2 roles: lane = seq + TS * (nb_b mod (16 / TS)) + 16 * h
  const int lane = tid & 31;
  const int seq2 = lane % TS, h = lane >> 4;
  const int nbb = ((lane / TS) % (16 / TS)) + (16 / TS) * (tid >> 5);
  int it = 0;
  for (long long tile = first; tile < ntiles; tile += stride, ++it) {
    const bool ok = mbar_wait_bounded(&bar[0], (unsigned)(it & 1));
    if (__syncthreads_or(!ok)) {
      if (tid == 0) atomicOr(&g_fused_fault, 1);
      return;
    }
    const int q = (int)(tile / ntna), nat = (int)(tile - (long long)q * ntna);
    const int na0 = nat * TS;
    float2 v[P2];
#pragma unroll
    for (int m = 0; m < P2; ++m) v[m] = region[(r + P1 * m) * TS + seq1];
    __syncthreads();  // the tile is in registers: the region takes the transpose
    Dft<P2>::run(v, +1);
    {
      float2* b = region + seq1 * SSEQ + r * S1;
      const float2* t1 = tw1 + r * S1;
#pragma unroll
      for (int n = 0; n < P2; ++n) b[n] = cmul(v[n], t1[n]);
    }
    __syncthreads();
    {
      const float2* b = region + seq2 * SSEQ + h * S1 + nbb;
#pragma unroll
      for (int k = 0; k < P1 / 2; ++k) v[k] = b[2 * k * S1];
    }
    __syncthreads();  // the region is read: fetch the next tile into it
    if (tid == 0 && tile + stride < ntiles) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(tile + stride);
    }
    Dft<P1 / 2>::run(v, +1);  // E (h = 0) or O (h = 1) at n mod 32
    // lane 0-half keeps E[0..15] and receives O[0..15]; lane 1-half keeps O[16..31] and
    // receives E[16..31]; each applies w^n to its 16 O values:
    // z[n] = E[n] + w^n O[n], z[n + 32] = E[n] - w^n O[n]
#pragma unroll
    for (int i = 0; i < P1 / 4; ++i) {
      const float2 s = h ? v[i] : v[i + P1 / 4];
      float2 o;
      o.x = __shfl_xor_sync(0xffffffffu, s.x, 16);
      o.y = __shfl_xor_sync(0xffffffffu, s.y, 16);
      const float2 e = h ? o : v[i];
      const float2 w = cmul(h ? v[i + P1 / 4] : o, tw2[i + (P1 / 4) * h]);
      v[i] = cadd(e, w);             // z[i + 16h]
      v[i + P1 / 4] = csub(e, w);    // z[i + 16h + 32]
    }
    const int j = 2 * q;
    const bool has1 = (j + 1) < Nr;
    double m[4] = {0.0, 0.0, 0.0, 0.0};
    {
      float* d0 = dest + (long long)j * N + na0 + seq2 + (long long)Q * nbb;
      float* d1 = d0 + N;
#pragma unroll
      for (int i = 0; i < P1 / 2; ++i) {
        const int nba = (i & (P1 / 4 - 1)) + 16 * h + (i >= P1 / 4 ? P1 / 2 : 0);
        const long long off = (long long)Q * P2 * nba;
        store_rate_pair(d0 + off, d1 + off, v[i], seq2 & 1, has1, dest, dest + N * (long long)Nr);
      }
      if (acc) {
#pragma unroll
        for (int i = 0; i < P1 / 2; ++i) {
          const double x = v[i].x, y = has1 ? v[i].y : 0.f;
          m[0] += x; m[1] += x * x; m[2] += y; m[3] += y * y;
        }
      }
    }
    if (acc) {
#pragma unroll
      for (int i = 0; i < 4; ++i)
        for (int o = 16; o > 0; o >>= 1) m[i] += __shfl_down_sync(0xffffffffu, m[i], o);
      __shared__ double red[4][SH::T / 32];
      const int wid = tid >> 5;
      if ((tid & 31) == 0)
        for (int i = 0; i < 4; ++i) red[i][wid] = m[i];
      __syncthreads();
      if (tid < 4) {
        double t = 0.0;
        for (int i = 0; i < SH::T / 32; ++i) t += red[tid][i];
        if (tid < 2 || has1) atomicAdd(acc + 2 * j + tid, t);
      }
      __syncthreads();  // red is free for the next tile
    }
  }
}

// ------------------------------------------------------------------------------------
// Mixed-precision output pass (workspace flag FDR_ZDT_MIXED_PRECISION; P = 1024 = 32 x 32).
// Both radix-32 stages of the inverse DFT_P run as tensor-core contractions: per tile
// (rate pair, 8 residues) C (64 x 256) = A (64 x 64) * B (64 x 256), where A is the real
// embedding [[Re D, -Im D], [Im D, Re D]] of the 32-point inverse DFT matrix D and B holds
// the real and imaginary parts of the 256 sequences (32 values each).  Operands are split
// into bfloat16 pairs x = hi + lo (hi = bf16(x), lo = bf16(x - hi)) and C accumulates
// hi*hi + hi*lo + lo*hi in float32 with mma.sync m16n8k16 (the lo*lo term, ~2^-16 relative,
// is dropped).  The inter-stage twiddles, the statistics and the stores stay in float32 /
// float64.  W tiles arrive by TMA into a double buffer as in zdtf_output_tma_kernel.
// ------------------------------------------------------------------------------------
struct OutMmaShape {
  static constexpr int P = 1024, TS = 8, T = 256;
  static constexpr unsigned STAGE = sizeof(float2) * P * TS;            // 64 KB
  static constexpr int NFRAG = 16;                                      // 4 M-tiles x 4 K-tiles
  static constexpr size_t AFRAG = (size_t)NFRAG * 32 * 2 * sizeof(uint4);  // hi + lo per lane
  static constexpr size_t SMEM = 1024 + 2 * (size_t)STAGE + AFRAG + sizeof(float2) * (P + 32) + 16;
};

__device__ __forceinline__ unsigned bf16_pair(float a, float b) {  // a in the low half
  __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<unsigned*>(&v);
}
__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], const uint4& a, unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a.x), "r"(a.y), "r"(a.z), "r"(a.w), "r"(b0), "r"(b1));
}

// Element (i, k) of the 64 x 64 real embedding of D[a][b] = exp(+2 pi i a b / 32).
__device__ __forceinline__ float dft32_embed(int i, int k, const float2* cs) {
  const float2 e = cs[((i & 31) * (k & 31)) & 31];  // (cos, sin)
  if (i < 32) return k < 32 ? e.x : -e.y;
  return k < 32 ? e.y : e.x;
}

// B fragments (hi, lo) of this warp's 4 column tiles for all 4 K-tiles, from a [32][256]
// complex matrix in shared memory (real K rows 0..31 = real parts, 32..63 = imaginary).
__device__ __forceinline__ void load_b_frags(const float2* src, int col0, int g, int t,
                                             unsigned (&bh)[4][4][2], unsigned (&bl)[4][4][2]) {
#pragma unroll
  for (int kt = 0; kt < 2; ++kt) {
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      const int c = col0 + nt * 8 + g;
      const float2 v0 = src[(kt * 16 + 2 * t) * 256 + c];
      const float2 v1 = src[(kt * 16 + 2 * t + 1) * 256 + c];
      const float2 v8 = src[(kt * 16 + 2 * t + 8) * 256 + c];
      const float2 v9 = src[(kt * 16 + 2 * t + 9) * 256 + c];
      // real parts -> K-tile kt, imaginary parts -> K-tile kt + 2
      float h0 = bf16_round(v0.x), h1 = bf16_round(v1.x), h8 = bf16_round(v8.x), h9 = bf16_round(v9.x);
      bh[kt][nt][0] = bf16_pair(h0, h1);
      bh[kt][nt][1] = bf16_pair(h8, h9);
      bl[kt][nt][0] = bf16_pair(v0.x - h0, v1.x - h1);
      bl[kt][nt][1] = bf16_pair(v8.x - h8, v9.x - h9);
      h0 = bf16_round(v0.y); h1 = bf16_round(v1.y); h8 = bf16_round(v8.y); h9 = bf16_round(v9.y);
      bh[kt + 2][nt][0] = bf16_pair(h0, h1);
      bh[kt + 2][nt][1] = bf16_pair(h8, h9);
      bl[kt + 2][nt][0] = bf16_pair(v0.y - h0, v1.y - h1);
      bl[kt + 2][nt][1] = bf16_pair(v8.y - h8, v9.y - h9);
    }
  }
}

// C[mt][nt] = A * B over the 4 K-tiles, three split products each.
__device__ __forceinline__ void mma_pass(const uint4* afrag, int lane, const unsigned (&bh)[4][4][2],
                                         const unsigned (&bl)[4][4][2], float (&c)[4][4][4]) {
#pragma unroll
  for (int mt = 0; mt < 4; ++mt) {
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int e = 0; e < 4; ++e) c[mt][nt][e] = 0.f;
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) {
      const uint4 ah = afrag[((mt * 4 + kt) * 32 + lane) * 2];
      const uint4 al = afrag[((mt * 4 + kt) * 32 + lane) * 2 + 1];
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        mma_bf16_16816(c[mt][nt], al, bh[kt][nt][0], bh[kt][nt][1]);
        mma_bf16_16816(c[mt][nt], ah, bl[kt][nt][0], bl[kt][nt][1]);
        mma_bf16_16816(c[mt][nt], ah, bh[kt][nt][0], bh[kt][nt][1]);
      }
    }
  }
}

__global__ void __launch_bounds__(OutMmaShape::T, 1)
zdtf_output_mma_kernel(const __grid_constant__ CUtensorMap wmap, long long N, int Q, int Nr, int npairs,
                       float* __restrict__ dest, const float2* __restrict__ rootsP,
                       double* __restrict__ acc) {
  using SH = OutMmaShape;
  constexpr int P = SH::P, TS = SH::TS;
  extern __shared__ unsigned char smraw[];
  const uintptr_t base = ((uintptr_t)smraw + 1023) & ~(uintptr_t)1023;
  float2* stage0 = (float2*)base;
  float2* stage1 = (float2*)(base + SH::STAGE);
  uint4* afrag = (uint4*)(base + 2 * (size_t)SH::STAGE);
  float2* roots = (float2*)(base + 2 * (size_t)SH::STAGE + SH::AFRAG);  // exp(-2 pi i m / P)
  float2* cs = roots + P;                                                // cos, sin of 2 pi m / 32
  unsigned long long* bar = (unsigned long long*)(cs + 32);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int ntna = Q / TS;
  const long long ntiles = (long long)ntna * npairs;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int i = tid; i < P; i += SH::T) roots[i] = __ldg(rootsP + i);
  if (tid < 32) {
    float sn, cn;
    sincospif((float)tid / 16.f, &sn, &cn);
    cs[tid] = make_float2(cn, sn);
  }
  __syncthreads();
  // A fragments of the 16 (M-tile, K-tile) blocks, hi and lo, in the mma.sync m16n8k16 layout
  for (int e = tid; e < SH::NFRAG * 32; e += SH::T) {
    const int f = e >> 5, ln = e & 31, mt = f >> 2, kt = f & 3;
    const int gg = ln >> 2, tt = ln & 3;
    float v[8];
    const int rows[8] = {gg, gg, gg + 8, gg + 8, gg, gg, gg + 8, gg + 8};
    const int cols[8] = {2 * tt, 2 * tt + 1, 2 * tt, 2 * tt + 1, 2 * tt + 8, 2 * tt + 9, 2 * tt + 8, 2 * tt + 9};
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = dft32_embed(mt * 16 + rows[q], kt * 16 + cols[q], cs);
    float h[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) h[q] = bf16_round(v[q]);
    afrag[e * 2] = make_uint4(bf16_pair(h[0], h[1]), bf16_pair(h[2], h[3]), bf16_pair(h[4], h[5]),
                              bf16_pair(h[6], h[7]));
    afrag[e * 2 + 1] = make_uint4(bf16_pair(v[0] - h[0], v[1] - h[1]), bf16_pair(v[2] - h[2], v[3] - h[3]),
                                  bf16_pair(v[4] - h[4], v[5] - h[5]), bf16_pair(v[6] - h[6], v[7] - h[7]));
  }
  __syncthreads();
  auto issue = [&](long long tile, int st) {  // thread 0 only
    const int q = (int)(tile / ntna), nat = (int)(tile - (long long)q * ntna);
    float2* dst = st ? stage1 : stage0;
    mbar_expect_tx(&bar[st], SH::STAGE);
#pragma unroll
    for (int b = 0; b < P / 256; ++b)
      tma_load_2d(dst + b * 256 * TS, &wmap, 2 * TS * nat, q * P + b * 256, &bar[st]);
  };
  const long long first = blockIdx.x, stride = gridDim.x;
  if (tid == 0) {
    if (first < ntiles) issue(first, 0);
    if (first + stride < ntiles) issue(first + stride, 1);
  }
  const int col0 = warp * 32;
  int it = 0;
  for (long long tile = first; tile < ntiles; tile += stride, ++it) {
    const int st = it & 1;
    const bool ok = mbar_wait_bounded(&bar[st], (unsigned)((it >> 1) & 1));
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicOr(&g_fused_fault, 4);
        if (tile + stride < ntiles) (void)mbar_wait_bounded(&bar[st ^ 1], (unsigned)(((it + 1) >> 1) & 1));
      }
      return;
    }
    float2* stg = st ? stage1 : stage0;
    const int q = (int)(tile / ntna), nat = (int)(tile - (long long)q * ntna);
    const int na0 = nat * TS;
    unsigned bh[4][4][2], bl[4][4][2];
    float c[4][4][4];
    // pass 1: sequences (r = k1 mod 32, seq) over m = k1 / 32; column c = r*8 + seq, row m
    load_b_frags(stg, col0, g, t, bh, bl);
    __syncthreads();  // the tile is in registers: the stage takes the transposed result
    mma_pass(afrag, lane, bh, bl, c);
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int nt = 0; nt < 4; ++nt)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int nbb = mt * 16 + g + (e >= 2 ? 8 : 0);
          const int col = col0 + nt * 8 + 2 * t + (e & 1);
          const int r = col >> 3, seq = col & 7;
          const float re = c[mt][nt][e], im = c[mt + 2][nt][e];
          const float2 w = roots[(r * nbb) & (P - 1)];  // multiply by conj(w) = exp(+2 pi i r nbb / P)
          stg[r * 256 + nbb * 8 + seq] = make_float2(re * w.x + im * w.y, im * w.x - re * w.y);
        }
    __syncthreads();
    // pass 2: sequences (nbb, seq) over k1a = r; column c = nbb*8 + seq, row r
    load_b_frags(stg, col0, g, t, bh, bl);
    __syncthreads();  // the stage is read: refill it with the tile after next
    if (tid == 0 && tile + 2 * stride < ntiles) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(tile + 2 * stride, st);
    }
    mma_pass(afrag, lane, bh, bl, c);
    const int j = 2 * q;
    const bool has1 = (j + 1) < Nr;
    double m[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int nt = 0; nt < 4; ++nt)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int nba = mt * 16 + g + 8 * h;
          const int col = col0 + nt * 8 + 2 * t;
          const int nbb = col >> 3, seq = col & 7;
          const long long n = (long long)(na0 + seq) + (long long)Q * (nbb + 32 * nba);
          const float x0 = c[mt][nt][2 * h], x1 = c[mt][nt][2 * h + 1];
          const float y0 = c[mt + 2][nt][2 * h], y1 = c[mt + 2][nt][2 * h + 1];
          if (FDR_DBG_OK(n + 2 <= N && j < Nr))
            __stcs(reinterpret_cast<float2*>(dest + (long long)j * N + n), make_float2(x0, x1));
          if (has1 && FDR_DBG_OK(n + 2 <= N))
            __stcs(reinterpret_cast<float2*>(dest + (long long)(j + 1) * N + n), make_float2(y0, y1));
          if (acc) {
            m[0] += (double)x0 + (double)x1;
            m[1] += (double)x0 * x0 + (double)x1 * x1;
            if (has1) {
              m[2] += (double)y0 + (double)y1;
              m[3] += (double)y0 * y0 + (double)y1 * y1;
            }
          }
        }
    if (acc) {
#pragma unroll
      for (int i = 0; i < 4; ++i)
        for (int o = 16; o > 0; o >>= 1) m[i] += __shfl_down_sync(0xffffffffu, m[i], o);
      __shared__ double red[4][SH::T / 32];
      if (lane == 0)
        for (int i = 0; i < 4; ++i) red[i][warp] = m[i];
      __syncthreads();
      if (tid < 4) {
        double tt2 = 0.0;
        for (int i = 0; i < SH::T / 32; ++i) tt2 += red[tid][i];
        if (tid < 2 || has1) atomicAdd(acc + 2 * j + tid, tt2);
      }
      __syncthreads();
    }
  }
}

// ------------------------------------------------------------------------------------
// Mixed-precision output pass for P = 2048 = 32 x 64 on the fifth-generation tensor cores
// (tcgen05, accumulators in tensor memory).  Per tile (rate pair q, 8 residues) the inverse
// DFT_P of sequence s,
//   z[s][n + 32 c] = sum_r e^(2 pi i r c / 64) e^(2 pi i r n / 2048) sum_m e^(2 pi i m n / 32) x[s][r + 64 m],
// runs as two real-embedded contractions with bfloat16 split operands (v = hi + lo, hi =
// bf16(v), lo = bf16(v - hi); hi*hi + hi*lo + lo*hi accumulated in float32, the lo*lo term,
// ~2^-16 relative, dropped):
//   pass 1: D1 (512 x 64)  = X (512 x 64) * E32 (64 x 64)    rows (s, r), K (m, re/im), N (n, re/im)
//   pass 2: D2 (128 x 256) = E64 (128 x 128) * Y (128 x 256) rows (re/im, c), K (r, re/im), N (s, n)
// The tile is fetched (TMA, 3-D tensor map) as two 64 KB halves, r < 32 and r >= 32, and
// processed as a pipeline over the halves: half h is converted in place to its 256 rows of
// X (K-major) while the MMAs of the other half run; pass 1's epilogue for half h writes, in
// place again, the 64 K rows of Y (MN-major, no transpose between the passes) that pass 2
// consumes as its K steps 4h .. 4h + 3; and half h is refilled with the next tile as soon as
// those MMAs have read it, so the fetch overlaps the rest of the tile and the FDR stores.
// Pass 2's rows are the pair's two rates (real parts: rate j, imaginary parts: rate j + 1);
// each epilogue lane holds 8 residues of one rate per output channel, and lane pairs store
// whole 32-byte sectors.  Every mbarrier wait is bounded (kTmaWaitNs); tensor memory is
// freed on all paths.
// ------------------------------------------------------------------------------------
struct OutUmmaShape {
  static constexpr int P = 2048, P1 = 64, P2 = 32, TS = 8, T = 512;
  static constexpr unsigned HALF = 65536;  // one half tile: 8 residues x 32 r x 32 m
  // byte layouts of the operands (core matrices of 8 rows x 16 bytes; umma.cuh); X and Y
  // of half h live in region half h, hi then lo
  static constexpr unsigned X_SBO = 1024, X_LBO = 128, X_PART = 32768;  // K-major, 256 rows
  static constexpr unsigned Y_SBO = 128, Y_LBO = 4096, Y_PART = 32768;  // MN-major, 64 K rows
  static constexpr unsigned E32_SBO = 1024, E32_LBO = 128, E32_PART = 8192;
  static constexpr unsigned E64_SBO = 2048, E64_LBO = 128, E64_PART = 32768;
  static constexpr int S1 = P2 + 1;  // twiddle table rows
  static constexpr unsigned OFF_E32 = 2 * HALF;
  static constexpr unsigned OFF_E64 = OFF_E32 + 2 * E32_PART;
  static constexpr unsigned OFF_TW = OFF_E64 + 2 * E64_PART;
  static constexpr unsigned OFF_BAR = OFF_TW + sizeof(float2) * P1 * S1;
  static constexpr size_t SMEM = 1024 + OFF_BAR + 64;
  static constexpr unsigned TMEM_COLS = 512;  // D1: 4 blocks x 64 columns; D2: 256 columns
  static constexpr unsigned D2_COL = 256;
};
static_assert(OutUmmaShape::SMEM <= 232448, "zdtf_output_umma_kernel: shared memory");
static_assert(OutUmmaShape::OFF_BAR % 8 == 0, "zdtf_output_umma_kernel: mbarrier alignment");

// Row of X (and lane of D1) of sequence (s, r); block r / 16, so half h holds rows
// 256 h .. 256 h + 255.  16-byte shared-memory accesses are served per 8 lanes, which must
// hit 8 different 16-byte bank slots: the 8 converting lanes of one r (s = lane mod 8)
// write rows with 8 different (row mod 8), and the 8 epilogue lanes of one 8-row group
// hold 8 different r mod 8, i.e. the 8 K rows of one core matrix of Y.
__device__ __forceinline__ int umma_xrow(int s, int r) {
  return ((r + s) & 7) + 8 * s + 64 * (r >> 3);
}
// Byte offset of element (row, k) of a K-major operand (K chunks 128 bytes apart).
__device__ __forceinline__ unsigned umma_kmaj(int row, int k, unsigned sbo) {
  return (unsigned)(row >> 3) * sbo + (unsigned)(k >> 3) * 128u + (unsigned)(row & 7) * 16u +
         (unsigned)(k & 7) * 2u;
}
// a = hi + lo, b = hi' + lo' in bfloat16, packed two per word (a in the low half).
__device__ __forceinline__ void umma_split2(float a, float b, unsigned& hi, unsigned& lo) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  const float2 hf = __bfloat1622float2(h);
  const __nv_bfloat162 l = __floats2bfloat162_rn(a - hf.x, b - hf.y);
  hi = *reinterpret_cast<const unsigned*>(&h);
  lo = *reinterpret_cast<const unsigned*>(&l);
}

__global__ void __launch_bounds__(OutUmmaShape::T, 1)
zdtf_output_umma_kernel(const __grid_constant__ CUtensorMap wmap, long long N, int Q, int Nr,
                        int npairs, float* __restrict__ dest, const float2* __restrict__ rootsP,
                        double* __restrict__ acc) {
  using SH = OutUmmaShape;
  constexpr int P = SH::P, P1 = SH::P1, P2 = SH::P2, TS = SH::TS;
  extern __shared__ unsigned char smraw[];
  unsigned char* sm = (unsigned char*)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
  unsigned char* e32 = sm + SH::OFF_E32;
  unsigned char* e64 = sm + SH::OFF_E64;
  float2* tw = (float2*)(sm + SH::OFF_TW);
  // mbarriers: [0], [1] the two halves' fetches; [2], [3] pass 1 of half 0, 1; [4], [5]
  // pass 2's K steps of half 0, 1.  Each completes once per tile.
  unsigned long long* bar = (unsigned long long*)(sm + SH::OFF_BAR);
  unsigned* tslot = (unsigned*)(bar + 6);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ntna = Q / TS;
  const long long ntiles = (long long)ntna * npairs;
  if (tid == 0) {
    for (int i = 0; i < 6; ++i) mbar_init(&bar[i], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    umma::tmem_alloc(tslot, SH::TMEM_COLS);
    umma::tmem_relinquish();
  }
  // E32 (B of pass 1, K-major): row nu = 2 n + re/im of the output, K pair (Re, Im) of x_m
  for (int e = tid; e < 64 * 32; e += SH::T) {
    const int nu = e >> 5, m = e & 31, n = nu >> 1, co = nu & 1;
    const float2 w = cconj(__ldg(rootsP + ((64 * m * n) & (P - 1))));  // e^(2 pi i m n / 32)
    unsigned h, l;
    umma_split2(co ? w.y : w.x, co ? w.x : -w.y, h, l);
    const unsigned off = umma_kmaj(nu, 2 * m, SH::E32_SBO);
    *reinterpret_cast<unsigned*>(e32 + off) = h;
    *reinterpret_cast<unsigned*>(e32 + SH::E32_PART + off) = l;
  }
  // E64 (A of pass 2, K-major): row 64 re/im + c; K 64 h + 32 re/im + (r mod 32) for
  // r = 32 h + (r mod 32), so that K steps 4h .. 4h + 3 are half h's; pairs (r, r + 1)
  for (int e = tid; e < 128 * 64; e += SH::T) {
    const int row = e >> 6, k0 = 2 * (e & 63);
    const int co = row >> 6, c = row & 63, ci = (k0 >> 5) & 1, r0 = 32 * (k0 >> 6) + (k0 & 31);
    float v[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const float2 w = cconj(__ldg(rootsP + ((32 * (r0 + u) * c) & (P - 1))));  // e^(2 pi i r c / 64)
      v[u] = co == ci ? w.x : (co == 0 ? -w.y : w.y);
    }
    unsigned h, l;
    umma_split2(v[0], v[1], h, l);
    const unsigned off = umma_kmaj(row, k0, SH::E64_SBO);
    *reinterpret_cast<unsigned*>(e64 + off) = h;
    *reinterpret_cast<unsigned*>(e64 + SH::E64_PART + off) = l;
  }
  for (int i = tid; i < P1 * P2; i += SH::T)
    tw[(i / P2) * SH::S1 + i % P2] = cconj(__ldg(rootsP + (((i / P2) * (i % P2)) & (P - 1))));
  umma::fence_smem_to_async();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const unsigned tbase = *tslot;
  const unsigned sb = umma::smem_u32(sm);
  auto issue = [&](long long tile, int h) {  // thread 0 only: half h of a tile
    const int q = (int)(tile / ntna), nat = (int)(tile - (long long)q * ntna);
    mbar_expect_tx(&bar[h], SH::HALF);
    tma_load_3d(sm + h * SH::HALF, &wmap, 2 * TS * nat, 32 * h, 32 * q, &bar[h]);
  };
  const long long first = blockIdx.x, stride = gridDim.x;
  if (tid == 0 && first < ntiles) {
    issue(first, 0);
    issue(first, 1);
  }
  constexpr unsigned idesc1 = umma::idesc_bf16_f32(128, 64, false, false);
  constexpr unsigned idesc2 = umma::idesc_bf16_f32(128, 256, false, true);
  const unsigned lane_base = (unsigned)(32 * (warp & 3)) << 16;
  // converting role (per half): sequence (s, r = 32 h + cl), values m = 16 cm .. 16 cm + 15
  const int cs = tid & 7, cl = (tid >> 3) & 31, cm = tid >> 8;
  // pass-1 epilogue role (per half): block 2 h + eb, lanes of quarter warp mod 4, columns
  // 32 ec .. 32 ec + 31 (channels n = 16 ec .. 16 ec + 15)
  const int eb = (warp >> 2) & 1, ec = warp >> 3;
  const int erow = 128 * eb + 32 * (warp & 3) + lane;  // row within the half
  const int es = (erow >> 3) & 7;
  const int erl = (((erow & 7) - es) & 7) + 8 * (erow >> 6);  // r mod 32
  unsigned pend = 0;  // MMA groups committed and not yet waited for (bit k: bar[2 + k])
  bool fail = false;
  int it = 0;

  auto convert = [&](int h) {  // half h of the W tile, in place, to its rows of X (hi, lo)
    const float2* src = (const float2*)(sm + h * SH::HALF);
    float2 v[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = src[((16 * cm + i) * 32 + cl) * TS + cs];
    __syncthreads();
    const int row = umma_xrow(cs, 32 * h + cl) - 256 * h;
    unsigned char* xr = sm + h * SH::HALF + (unsigned)(row >> 3) * SH::X_SBO + (unsigned)(row & 7) * 16u;
#pragma unroll
    for (int c4 = 0; c4 < 4; ++c4) {  // K chunk 4 cm + c4: x_m for m = 4 (4 cm + c4) .. + 3
      uint4 hv, lv;
      umma_split2(v[4 * c4].x, v[4 * c4].y, hv.x, lv.x);
      umma_split2(v[4 * c4 + 1].x, v[4 * c4 + 1].y, hv.y, lv.y);
      umma_split2(v[4 * c4 + 2].x, v[4 * c4 + 2].y, hv.z, lv.z);
      umma_split2(v[4 * c4 + 3].x, v[4 * c4 + 3].y, hv.w, lv.w);
      const unsigned kc = (unsigned)(4 * cm + c4) * 128u;
      *reinterpret_cast<uint4*>(xr + kc) = hv;
      *reinterpret_cast<uint4*>(xr + SH::X_PART + kc) = lv;
    }
    umma::fence_smem_to_async();
    umma::fence_before_sync();
    __syncthreads();
  };
  auto pass1 = [&](int h) {  // thread 0: blocks 2h, 2h + 1 x 4 K steps x 3 products
    umma::fence_after_sync();
#pragma unroll 1
    for (int bb = 0; bb < 2; ++bb) {
      const unsigned d = tbase + 64u * (unsigned)(2 * h + bb);
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const unsigned xa = sb + h * SH::HALF + (unsigned)bb * 16u * SH::X_SBO + (unsigned)t * 256u;
        const unsigned ea = sb + SH::OFF_E32 + (unsigned)t * 256u;
        const uint64_t xh = umma::sdesc(xa, SH::X_LBO, SH::X_SBO);
        const uint64_t xl = umma::sdesc(xa + SH::X_PART, SH::X_LBO, SH::X_SBO);
        const uint64_t eh = umma::sdesc(ea, SH::E32_LBO, SH::E32_SBO);
        const uint64_t el = umma::sdesc(ea + SH::E32_PART, SH::E32_LBO, SH::E32_SBO);
        umma::mma_bf16(d, xh, eh, idesc1, t > 0);
        umma::mma_bf16(d, xh, el, idesc1, true);
        umma::mma_bf16(d, xl, eh, idesc1, true);
      }
    }
    umma::commit(&bar[2 + h]);
  };
  auto epilogue1 = [&](int h) {  // D1 rows of half h times the twiddle, to its K rows of Y
    float d[32];
    umma::ld32_wait(tbase + lane_base + 64u * (unsigned)(2 * h + eb) + 32u * (unsigned)ec, d);
    const float2* twr = tw + (32 * h + erl) * SH::S1 + 16 * ec;
    unsigned char* yre = sm + h * SH::HALF + (unsigned)(erl >> 3) * SH::Y_LBO + (unsigned)(erl & 7) * 16u;
    unsigned char* yim = yre + 4u * SH::Y_LBO;  // K row 32 + (r mod 32)
#pragma unroll
    for (int g = 0; g < 2; ++g) {  // channels n = 16 ec + 8 g .. + 7
      unsigned rh[4], rl[4], ih[4], il[4];
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        const int n0 = 8 * g + 2 * p;
        const float2 y0 = cmul(make_float2(d[2 * n0], d[2 * n0 + 1]), twr[n0]);
        const float2 y1 = cmul(make_float2(d[2 * n0 + 2], d[2 * n0 + 3]), twr[n0 + 1]);
        umma_split2(y0.x, y1.x, rh[p], rl[p]);
        umma_split2(y0.y, y1.y, ih[p], il[p]);
      }
      const unsigned nofs = (unsigned)(4 * es + 2 * ec + g) * SH::Y_SBO;  // N group (32 s + n) / 8
      *reinterpret_cast<uint4*>(yre + nofs) = make_uint4(rh[0], rh[1], rh[2], rh[3]);
      *reinterpret_cast<uint4*>(yre + SH::Y_PART + nofs) = make_uint4(rl[0], rl[1], rl[2], rl[3]);
      *reinterpret_cast<uint4*>(yim + nofs) = make_uint4(ih[0], ih[1], ih[2], ih[3]);
      *reinterpret_cast<uint4*>(yim + SH::Y_PART + nofs) = make_uint4(il[0], il[1], il[2], il[3]);
    }
    umma::fence_smem_to_async();
    umma::fence_before_sync();
    __syncthreads();
  };
  auto pass2 = [&](int h) {  // thread 0: K steps 4h .. 4h + 3 x 3 products into D2
    umma::fence_after_sync();
#pragma unroll
    for (int t4 = 0; t4 < 4; ++t4) {
      const int t = 4 * h + t4;
      const unsigned ea = sb + SH::OFF_E64 + (unsigned)t * 256u;
      const unsigned ya = sb + h * SH::HALF + (unsigned)(2 * t4) * SH::Y_LBO;
      const uint64_t eh = umma::sdesc(ea, SH::E64_LBO, SH::E64_SBO);
      const uint64_t el = umma::sdesc(ea + SH::E64_PART, SH::E64_LBO, SH::E64_SBO);
      const uint64_t yh = umma::sdesc(ya, SH::Y_LBO, SH::Y_SBO);
      const uint64_t yl = umma::sdesc(ya + SH::Y_PART, SH::Y_LBO, SH::Y_SBO);
      umma::mma_bf16(tbase + SH::D2_COL, eh, yh, idesc2, t > 0);
      umma::mma_bf16(tbase + SH::D2_COL, eh, yl, idesc2, true);
      umma::mma_bf16(tbase + SH::D2_COL, el, yh, idesc2, true);
    }
    umma::commit(&bar[4 + h]);
  };
  // waits for MMA group k (bar[2 + k]) of this tile; false if the wait ran out
  auto mma_wait = [&](int k) {
    const bool ok = mbar_wait_bounded(&bar[2 + k], (unsigned)(it & 1));
    if (__syncthreads_or(!ok)) return false;
    pend &= ~(1u << k);
    umma::fence_after_sync();
    return true;
  };

  for (long long tile = first; tile < ntiles; tile += stride, ++it) {
    const int q = (int)(tile / ntna), nat = (int)(tile - (long long)q * ntna);
    const int na0 = nat * TS;
    const bool more = tile + stride < ntiles;
    bool ok = mbar_wait_bounded(&bar[0], (unsigned)(it & 1));
    if (__syncthreads_or(!ok)) { fail = true; break; }
    convert(0);
    if (tid == 0) pass1(0);
    pend |= 1u;
    ok = mbar_wait_bounded(&bar[1], (unsigned)(it & 1));
    if (__syncthreads_or(!ok)) { fail = true; break; }
    convert(1);  // overlaps pass 1 of half 0
    if (tid == 0) pass1(1);
    pend |= 2u;
    if (!mma_wait(0)) { fail = true; break; }
    epilogue1(0);  // overlaps pass 1 of half 1
    if (tid == 0) pass2(0);
    pend |= 4u;
    if (!mma_wait(1)) { fail = true; break; }
    epilogue1(1);  // overlaps pass 2 of half 0
    if (tid == 0) pass2(1);
    pend |= 8u;
    if (!mma_wait(2)) { fail = true; break; }
    if (tid == 0 && more) {  // half 0 is read: refill it with the next tile's
      umma::fence_smem_to_async();
      issue(tile + stride, 0);
    }
    if (!mma_wait(3)) { fail = true; break; }
    if (tid == 0 && more) {
      umma::fence_smem_to_async();
      issue(tile + stride, 1);
    }
    {  // pass-2 epilogue: lane (re/im, c) of D2, channels n = 8 (warp / 4) .. + 7, 8 residues
      const int co = (warp & 3) >> 1, c = 32 * (warp & 1) + lane, ng = warp >> 2;
      const int j = 2 * q;
      float z[64];  // z[8 s + i]: channel 8 ng + i of residue s
      umma::ld8x8_wait<32>(tbase + SH::D2_COL + lane_base + 8u * (unsigned)ng, z);
      if (co == 0 || j + 1 < Nr) {
        // The 8 residues of one (rate, channel) are one 32-byte sector.  Lanes 2k and 2k + 1
        // (channels c, c + 1) write both halves of one sector per instruction: the even
        // lane passes residues 4-7 of its channel to the odd lane, the odd lane residues
        // 0-3 of its channel to the even lane, so each store instruction fills 16 sectors.
        const bool odd = lane & 1;
        float* col = dest + (long long)(j + co) * N + na0;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const float4 lo = make_float4(z[i], z[8 + i], z[16 + i], z[24 + i]);
          const float4 hi = make_float4(z[32 + i], z[40 + i], z[48 + i], z[56 + i]);
          const float4 snd = odd ? lo : hi;
          float4 rcv;
          rcv.x = __shfl_xor_sync(0xffffffffu, snd.x, 1);
          rcv.y = __shfl_xor_sync(0xffffffffu, snd.y, 1);
          rcv.z = __shfl_xor_sync(0xffffffffu, snd.z, 1);
          rcv.w = __shfl_xor_sync(0xffffffffu, snd.w, 1);
          float* pe = col + (long long)Q * (8 * ng + i + 32 * (c & ~1));  // even channel's sector
          float* po = pe + (long long)Q * 32;                             // odd channel's sector
          float* da = odd ? pe + 4 : pe;
          float* db = odd ? po + 4 : po;
          if (FDR_DBG_OK(da >= dest && da + 4 <= dest + N * (long long)Nr))
            __stcs(reinterpret_cast<float4*>(da), odd ? rcv : lo);
          if (FDR_DBG_OK(db >= dest && db + 4 <= dest + N * (long long)Nr))
            __stcs(reinterpret_cast<float4*>(db), odd ? hi : rcv);
        }
        if (acc) {
          double s1 = 0.0, s2 = 0.0;
#pragma unroll
          for (int e = 0; e < 64; ++e) {
            const double x = z[e];
            s1 += x;
            s2 += x * x;
          }
          for (int o = 16; o > 0; o >>= 1) {
            s1 += __shfl_down_sync(0xffffffffu, s1, o);
            s2 += __shfl_down_sync(0xffffffffu, s2, o);
          }
          if (lane == 0) {
            atomicAdd(acc + 2 * (j + co), s1);
            atomicAdd(acc + 2 * (j + co) + 1, s2);
          }
        }
      }
    }
    umma::fence_before_sync();
  }
  if (fail) {
    if (tid == 0) atomicOr(&g_fused_fault, 16);
    // MMA groups still outstanding get one more bounded wait each before their tensor
    // memory is freed
    for (int k = 0; k < 4; ++k)
      if (pend & (1u << k)) (void)mbar_wait_bounded(&bar[2 + k], (unsigned)(it & 1));
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    umma::fence_after_sync();
    umma::tmem_dealloc(tbase, SH::TMEM_COLS);
  }
}

// ------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------
// Tile (sequences per CTA) and block size of kernels A and C for a given P: one radix-16
// butterfly per thread per pass, about 75 KB of shared memory, two CTAs per SM.
template <int P>
struct AcShape {
  static constexpr int TILE = P >= 4096 ? 4 : 8;
  static constexpr int T = (TILE * P / 16 > 512) ? 512 : (TILE * P / 16 < 32 ? 32 : TILE * P / 16);
  static constexpr size_t SMEM = sizeof(float2) * (TILE * ac_stride<P, TILE>() + tw_size(P));
};

template <int Q>
struct CztShape {  // buf | twt | twr | gnyq | buf2 (the second rate-block buffer) | phase residues
  static constexpr size_t SMEM =
      sizeof(float2) * (2 * kRatesPerBlock * b_stride<Q>() + tw_size(Q) + 2 * Q + kFusedMaxNt) +
      sizeof(unsigned long long) * 4 * (Q / 2);
};

// log2 of the four-step factor Q for Nf = 2^L and Nt time steps.  With F in registers
// (Nt <= 16): 512 bins per CTA up to Nf = 2^20 (256 threads, two CTAs per SM, so one CTA's
// barriers overlap the other's Horner sums; P <= 2048 keeps the TMA output passes), 1024
// above; with F in shared memory 512 (Nt <= 32) and 256 (Nt <= 64).  Mixed-precision
// workspaces split the same way (their tensor-core output passes cover P = 1024 and 2048).
static int fused_qlog(int L, int64_t Nt) {
  // 32 < Nt <= 64 at Nf = 2^20, 2^21: 512 bins per residue pair, F split over a cluster of two
  // CTAs (zdtf_czt_cl_kernel), so that P stays 2048 / 4096
  const int cap = Nt <= 16 ? (L <= 20 ? 9 : 10)
                           : (Nt <= 32 ? 9 : ((L == 20 || L == 21) ? 9 : 8));
  return std::min(cap, (L + 1) / 2);
}

void fused_split_log2(int64_t Nf, int64_t Nt, int* Plog, int* Qlog) {
  const int L = ilog2(Nf);
  *Qlog = fused_qlog(L, Nt);
  *Plog = L - *Qlog;
}

bool zdt_fused_eligible(int64_t Nf, int64_t Nt, int64_t Nr) {
  if (!is_pow2(Nf) || Nt > kFusedMaxNtSmem || Nt < 1 || Nr < 1) return false;
  const int L = ilog2(Nf);
  if (L < kFusedMinLog2 || L > kFusedMaxLog2) return false;
  return (L - fused_qlog(L, Nt)) <= 12;  // P <= 4096
}

static void float_parts(float x, long long* m, int* e) {
  if (x == 0.f) { *m = 0; *e = 0; return; }
  int ex = 0;
  const float f = frexpf(x, &ex);
  long long mm = (long long)ldexpf(f, 24);
  int ee = ex - 24;
  while (mm != 0 && (mm % 2) == 0) { mm /= 2; ++ee; }
  *m = mm;
  *e = ee;
}

static bool make_phase(float r0, float dr, int L, PhaseInt* ph) {
  if (!isfinite(r0) || !isfinite(dr)) return false;
  long long m0, md;
  int e0, ed;
  float_parts(r0, &m0, &e0);
  float_parts(dr, &md, &ed);
  int s = 0;
  if (m0 != 0 && -e0 > s) s = -e0;
  if (md != 0 && -ed > s) s = -ed;
  const int bits = L + s;
  if (bits > 62) return false;
  const unsigned long long mask = (1ULL << bits) - 1ULL;
  auto part = [&](long long m, int e) -> unsigned long long {
    if (m == 0) return 0ULL;
    const int sh = e + s;  // >= 0
    if (sh >= bits) return 0ULL;
    return (((unsigned long long)m) << sh) & mask;  // two's complement wrap is exact mod 2^bits
  };
  ph->R0 = part(m0, e0);
  ph->Rd = part(md, ed);
  ph->mask = mask;
  ph->bits = bits;
  ph->scale = ldexpf(1.0f, 1 - bits);
  return true;
}

// Sizes and twiddle tables of the fused kernels for one (Nf, Nt, Nr); shared by the ZDT
// workspace and by batches of channels with the same shape.
struct FusedPlan {
  int64_t N = 0, Nt = 0, Nr = 0;
  int L = 0, B = 0, P = 0, Q = 0;
  float2* tables = nullptr;  // twP | twQ | tw_lo | tw_hi | rootsP
  FusedTables tab;
  int64_t NP = 0, npairs = 0;
};

static std::vector<float2> roots_table(long long n, long long N, long long count) {
  // exp(-2 pi i m n / N) for m < count, angle reduced exactly in integers
  std::vector<float2> h((size_t)count);
  for (long long m = 0; m < count; ++m) {
    const long long r = (m * n) % N;
    const double a = -2.0 * (double)r / (double)N;  // half-turns in (-2, 0]
    h[(size_t)m] = make_float2((float)cos(M_PI * a), (float)sin(M_PI * a));
  }
  return h;
}

// Stockham pass twiddles for length len in the tw_offset layout.
static std::vector<float2> pass_twiddles(int len) {
  std::vector<float2> h((size_t)tw_size(len));
  int ns = 1;
  while (ns < len) {
    const int R = plan_radix(len / ns);
    if (ns > 1) {
      const int off = tw_offset(len, ns);
      for (int r = 1; r < R; ++r)
        for (int k = 0; k < ns; ++k) {
          const long long m = (long long)r * k, M = (long long)ns * R;
          const double a = -2.0 * (double)(m % M) / (double)M;
          h[(size_t)(off + (r - 1) * ns + k)] = make_float2((float)cos(M_PI * a), (float)sin(M_PI * a));
        }
    }
    ns *= R;
  }
  return h;
}

#define FDR_FOR_P(X) X(64) X(128) X(256) X(512) X(1024) X(2048) X(4096)
#define FDR_FOR_Q(X) X(64) X(128) X(256) X(512) X(1024)

static int set_smem_attrs() {
  static bool done[64] = {false};
  int dev = 0;
  FDR_CUDA(cudaGetDevice(&dev));
  if (dev < 64 && done[dev]) return FDR_OK;
#define SET_AC(P)                                                                              \
  FDR_CUDA(cudaFuncSetAttribute(zdtf_input_kernel<P, AcShape<P>::TILE, AcShape<P>::T>,         \
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)AcShape<P>::SMEM)); \
  FDR_CUDA(cudaFuncSetAttribute(zdtf_output_kernel<P, AcShape<P>::TILE, AcShape<P>::T>,        \
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)AcShape<P>::SMEM));
  FDR_FOR_P(SET_AC)
#undef SET_AC
#define SET_C2(P1, P2)                                                                         \
  FDR_CUDA(cudaFuncSetAttribute(zdtf_output2_kernel<P1, P2, 8>,                                \
                                cudaFuncAttributeMaxDynamicSharedMemorySize,                   \
                                (int)Out2Shape<P1, P2, 8>::SMEM));
  SET_C2(8, 8) SET_C2(8, 16) SET_C2(16, 16) SET_C2(16, 32) SET_C2(32, 32)
#undef SET_C2
  FDR_CUDA(cudaFuncSetAttribute(zdtf_output_mma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)OutMmaShape::SMEM));
  FDR_CUDA(cudaFuncSetAttribute(zdtf_output_umma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)OutUmmaShape::SMEM));
  FDR_CUDA(cudaFuncSetAttribute(zdtf_output_tma_kernel<32, 32, 8>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)OutTmaShape<32, 32, 8>::SMEM));
  FDR_CUDA(cudaFuncSetAttribute(zdtf_output_tma64_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)OutTma64Shape<8>::SMEM));
  // P = 2048 input: Nf = 2^20 or 2^21, table split B = 10 or 11
  FDR_CUDA(cudaFuncSetAttribute(zdtf_input64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)In64Shape::smem(11, 1LL << 21)));
#define SET_B(Q)                                                                               \
  FDR_CUDA(cudaFuncSetAttribute(zdtf_czt_kernel<Q, kFusedMaxNt, false>,                        \
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CztShape<Q>::SMEM)); \
  FDR_CUDA(cudaFuncSetAttribute(zdtf_czt_kernel<Q, kFusedMaxNt, true>,                         \
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CztShape<Q>::SMEM)); \
  FDR_CUDA(cudaFuncSetAttribute(zdtf_a2f_kernel<Q, kFusedMaxNt>,                               \
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CztShape<Q>::SMEM));
  FDR_FOR_Q(SET_B)
#undef SET_B
#define SET_BS(Q, NT)                                                                          \
  FDR_CUDA(cudaFuncSetAttribute(zdtf_czt_smem_kernel<Q, NT>,                                   \
                                cudaFuncAttributeMaxDynamicSharedMemorySize,                   \
                                (int)CztSmemShape<Q>::template smem<NT>()));                   \
  FDR_CUDA(cudaFuncSetAttribute(zdtf_a2f_smem_kernel<Q, NT>,                                   \
                                cudaFuncAttributeMaxDynamicSharedMemorySize,                   \
                                (int)CztSmemShape<Q>::template smem<NT>()));
  SET_BS(64, 32) SET_BS(128, 32) SET_BS(256, 32) SET_BS(512, 32)
  SET_BS(64, 64) SET_BS(128, 64) SET_BS(256, 64)
#undef SET_BS
#define SET_WS(Q, NT)                                                                          \
  FDR_CUDA(cudaFuncSetAttribute(zdtf_czt_ws_kernel<Q, NT>,                                     \
                                cudaFuncAttributeMaxDynamicSharedMemorySize,                   \
                                (int)CztWsShape<Q>::template smem<NT>()));
  SET_WS(512, 32) SET_WS(256, 32) SET_WS(256, 64)
#undef SET_WS
  FDR_CUDA(cudaFuncSetAttribute(zdtf_czt_cl_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)CztClShape::SMEM));
  FDR_CUDA(cudaFuncSetAttribute(zdtf_a2f_half_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)CztClShape::SMEM));
  if (dev < 64) done[dev] = true;
  return FDR_OK;
}

int fused_plan_create(FusedPlan** out, int64_t N, int64_t Nt, int64_t Nr) {
  *out = nullptr;
  if (!zdt_fused_eligible(N, Nt, Nr)) {
    set_error(FDR_ERR_UNSUPPORTED_SIZE, "fused plan: Nf=%lld Nt=%lld not supported",
              (long long)N, (long long)Nt);
    return FDR_ERR_UNSUPPORTED_SIZE;
  }
  FDR_TRY(set_smem_attrs());
  FusedPlan* st = new FusedPlan();
  st->N = N; st->Nt = Nt; st->Nr = Nr;
  st->L = ilog2(N);
  const int Qlog = fused_qlog(st->L, Nt);
  st->Q = 1 << Qlog;
  st->P = (int)(N >> Qlog);
  st->B = (st->L + 1) / 2;
  st->NP = cdiv(Nt, 2);
  st->npairs = cdiv(Nr, 2);
  const long long P = st->P, Q = st->Q;
  const long long nlo = 1LL << st->B, nhi = N >> st->B;
  const long long ntwP = tw_size((int)P), ntwQ = tw_size((int)Q);
  const long long ntab = ntwP + ntwQ + nlo + nhi + P;
  cudaError_t e = cudaMalloc(&st->tables, sizeof(float2) * ntab);
  if (e != cudaSuccess) { delete st; return cuda_status(e, "cudaMalloc(fused tables)"); }
  std::vector<float2> h;
  auto append = [&](const std::vector<float2>& v) { h.insert(h.end(), v.begin(), v.end()); };
  append(pass_twiddles((int)P));
  append(pass_twiddles((int)Q));
  append(roots_table(1, N, nlo));
  append(roots_table(nlo, N, nhi));
  append(roots_table(1, P, P));
  e = cudaMemcpy(st->tables, h.data(), sizeof(float2) * ntab, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) { cudaFree(st->tables); delete st; return cuda_status(e, "upload fused tables"); }
  st->tab.twP = st->tables;
  st->tab.twQ = st->tables + ntwP;
  st->tab.tw_lo = st->tables + ntwP + ntwQ;
  st->tab.tw_hi = st->tables + ntwP + ntwQ + nlo;
  st->tab.rootsP = st->tables + ntwP + ntwQ + nlo + nhi;
  st->tab.B = st->B;
  *out = st;
  return FDR_OK;
}

void fused_plan_destroy(FusedPlan* st) {
  if (!st) return;
  cudaFree(st->tables);
  delete st;
}

int64_t fused_plan_table_bytes(const FusedPlan* st) {
  return (int64_t)sizeof(float2) * (tw_size(st->P) + tw_size(st->Q) + (1LL << st->B) + (st->N >> st->B) + st->P);
}
int64_t fused_A_elems(const FusedPlan* st) { return st->N * st->NP; }
int64_t fused_W_elems(const FusedPlan* st) { return st->N * st->npairs; }

int fused_input(const FusedPlan* st, const float* spec, float2* A, cudaStream_t s) {
  const int P = st->P, Q = st->Q;
  if (P == 2048 && Q >= In64Shape::TS) {
    zdtf_input64_kernel<<<dim3(Q / In64Shape::TS, (unsigned)st->NP), In64Shape::T,
                          In64Shape::smem(st->B, st->N), s>>>(spec, st->N, (int)st->Nt, Q, A, st->tab);
    FDR_LAUNCH_CHECK("zdtf_input64_kernel");
    return FDR_OK;
  }
#define LAUNCH_A(PP)                                                                           \
  if (P == PP) {                                                                               \
    constexpr int TA = AcShape<PP>::TILE, T = AcShape<PP>::T;                                  \
    zdtf_input_kernel<PP, TA, T><<<dim3(Q / TA, (unsigned)st->NP), T, AcShape<PP>::SMEM, s>>>( \
        spec, st->N, (int)st->Nt, Q, A, st->tab);                                              \
    FDR_LAUNCH_CHECK("zdtf_input_kernel");                                                     \
    return FDR_OK;                                                                             \
  }
  FDR_FOR_P(LAUNCH_A)
#undef LAUNCH_A
  set_error(FDR_ERR_UNSUPPORTED_SIZE, "fused input: P=%d", P);
  return FDR_ERR_UNSUPPORTED_SIZE;
}

static CztArgs czt_args(const FusedPlan* st, const float2* A, float2* W) {
  CztArgs a;
  memset(&a, 0, sizeof(a));
  a.A = A;
  a.W = W;
  a.N = st->N;
  a.P = st->P;
  a.Nt = (int)st->Nt;
  a.NP = (int)st->NP;
  a.Nr = (int)st->Nr;
  a.npairs = (int)st->npairs;
  a.tab = st->tab;
  return a;
}

int fused_a2f(const FusedPlan* st, const float2* A, float2* F, cudaStream_t s) {
  CztArgs a = czt_args(st, A, nullptr);
  a.F = F;
  const int Q = st->Q, ctas = st->P / 2;
  if (st->Nt > 32 && Q == CztClShape::Q) {
    zdtf_a2f_half_kernel<<<2 * ctas, CztClShape::T, CztClShape::SMEM, s>>>(a);
    FDR_LAUNCH_CHECK("zdtf_a2f_half_kernel");
    return FDR_OK;
  }
  if (st->Nt > kFusedMaxNt) {
    const int NT = st->Nt <= 32 ? 32 : 64;
#define LAUNCH_A2FS(QQ, NN)                                                                    \
    if (Q == QQ && NT == NN) {                                                                 \
      zdtf_a2f_smem_kernel<QQ, NN><<<ctas, CztSmemShape<QQ>::T,                                \
                                     CztSmemShape<QQ>::template smem<NN>(), s>>>(a);           \
      FDR_LAUNCH_CHECK("zdtf_a2f_smem_kernel");                                                \
      return FDR_OK;                                                                           \
    }
    LAUNCH_A2FS(64, 32) LAUNCH_A2FS(128, 32) LAUNCH_A2FS(256, 32) LAUNCH_A2FS(512, 32)
    LAUNCH_A2FS(64, 64) LAUNCH_A2FS(128, 64) LAUNCH_A2FS(256, 64)
#undef LAUNCH_A2FS
    set_error(FDR_ERR_UNSUPPORTED_SIZE, "fused A->F: Q=%d Nt=%lld", Q, (long long)st->Nt);
    return FDR_ERR_UNSUPPORTED_SIZE;
  }
#define LAUNCH_A2F(QQ)                                                                         \
  if (Q == QQ) {                                                                               \
    zdtf_a2f_kernel<QQ, kFusedMaxNt><<<ctas, QQ / 2, CztShape<QQ>::SMEM, s>>>(a);              \
    FDR_LAUNCH_CHECK("zdtf_a2f_kernel");                                                       \
    return FDR_OK;                                                                             \
  }
  FDR_FOR_Q(LAUNCH_A2F)
#undef LAUNCH_A2F
  set_error(FDR_ERR_UNSUPPORTED_SIZE, "fused A->F: Q=%d", Q);
  return FDR_ERR_UNSUPPORTED_SIZE;
}

bool fused_phase_ok(const FusedPlan* st, float r0, float dr) {
  PhaseInt ph;
  return make_phase(r0, dr, st->L, &ph);
}

// Rate groups (grid.y of the czt kernel) by default: about four waves of one CTA per SM.
int fused_default_groups(const FusedPlan* st) {
  const int ctas = st->P / 2;
  return std::max(1, std::min<int>((int)cdiv(4 * sm_count(), ctas),
                                   (int)cdiv(st->npairs, kRatesPerBlock / 2)));
}

int fused_czt(const FusedPlan* st, const float2* A, float2* W, float r0, float dr, int window,
              const double* wk, int groups, cudaStream_t s) {
  return fused_czt_blocks(st, A, W, r0, dr, window, wk, nullptr, groups, s);
}

int fused_czt_blocks(const FusedPlan* st, const float2* A, float2* W, float r0, float dr,
                     int window, const double* wk, const int* blk_base, int groups,
                     cudaStream_t s) {
  PhaseInt ph;
  if (!make_phase(r0, dr, st->L, &ph)) {
    set_error(FDR_ERR_UNSUPPORTED_SIZE, "fused czt: rates need more than 62 phase bits");
    return FDR_ERR_UNSUPPORTED_SIZE;
  }
  CztArgs a = czt_args(st, A, W);
  a.ph = ph;
  a.window = window;
  a.wk = wk;
  a.blk_base = blk_base;
  const int Q = st->Q, ctas = st->P / 2;
  if (groups <= 0) groups = fused_default_groups(st);
  int ppg = (int)cdiv(st->npairs, groups);
  ppg = (int)cdiv(ppg, kRatesPerBlock / 2) * (kRatesPerBlock / 2);
  groups = (int)cdiv(st->npairs, ppg);
  a.pairs_per_group = ppg;
  if (st->Nt > 32 && Q == CztClShape::Q) {  // F of 64 steps for 512 bins: two-CTA cluster
    zdtf_czt_cl_kernel<<<dim3(2 * ctas, groups), CztClShape::T, CztClShape::SMEM, s>>>(a);
    FDR_LAUNCH_CHECK("zdtf_czt_cl_kernel");
    return FDR_OK;
  }
  // 16 < Nt <= 64 with 256 or 512 bins per CTA: the warp-specialised kernel (measured 6-9%
  // faster than zdtf_czt_smem_kernel at Nf = 2^19..2^20); Nt <= 16 keeps F in registers.
  if (st->Nt > kFusedMaxNt && ((Q == 512 && st->Nt <= 32) || (Q == 256 && st->Nt <= 64))) {
    const int NT = st->Nt <= 32 ? 32 : 64;
#define LAUNCH_WS(QQ, NN)                                                                      \
    if (Q == QQ && NT == NN) {                                                                 \
      zdtf_czt_ws_kernel<QQ, NN><<<dim3(ctas, groups), CztWsShape<QQ>::T,                      \
                                   CztWsShape<QQ>::template smem<NN>(), s>>>(a);               \
      FDR_LAUNCH_CHECK("zdtf_czt_ws_kernel");                                                  \
      return FDR_OK;                                                                           \
    }
    LAUNCH_WS(512, 32) LAUNCH_WS(256, 32) LAUNCH_WS(256, 64)
#undef LAUNCH_WS
  }
  if (st->Nt > kFusedMaxNt) {
    const int NT = st->Nt <= 32 ? 32 : 64;
#define LAUNCH_BS(QQ, NN)                                                                      \
    if (Q == QQ && NT == NN) {                                                                 \
      zdtf_czt_smem_kernel<QQ, NN><<<dim3(ctas, groups), CztSmemShape<QQ>::T,                  \
                                     CztSmemShape<QQ>::template smem<NN>(), s>>>(a);           \
      FDR_LAUNCH_CHECK("zdtf_czt_smem_kernel");                                                \
      return FDR_OK;                                                                           \
    }
    LAUNCH_BS(64, 32) LAUNCH_BS(128, 32) LAUNCH_BS(256, 32) LAUNCH_BS(512, 32)
    LAUNCH_BS(64, 64) LAUNCH_BS(128, 64) LAUNCH_BS(256, 64)
#undef LAUNCH_BS
  } else {
#define LAUNCH_B(QQ)                                                                           \
    if (Q == QQ) {                                                                             \
      if (window == FDR_WINDOW_RECT)                                                           \
        zdtf_czt_kernel<QQ, kFusedMaxNt, false><<<dim3(ctas, groups), QQ / 2, CztShape<QQ>::SMEM, s>>>(a); \
      else                                                                                     \
        zdtf_czt_kernel<QQ, kFusedMaxNt, true><<<dim3(ctas, groups), QQ / 2, CztShape<QQ>::SMEM, s>>>(a); \
      FDR_LAUNCH_CHECK("zdtf_czt_kernel");                                                     \
      return FDR_OK;                                                                           \
    }
    FDR_FOR_Q(LAUNCH_B)
#undef LAUNCH_B
  }
  set_error(FDR_ERR_UNSUPPORTED_SIZE, "fused czt: Q=%d Nt=%lld", Q, (long long)st->Nt);
  return FDR_ERR_UNSUPPORTED_SIZE;
}

// cuTensorMapEncodeTiled from the driver, through the runtime (no link against libcuda);
// looked up once per process (thread-safe static initialisation).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = []() -> PFN_cuTensorMapEncodeTiled_v12000 {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess && q == cudaDriverEntryPointSuccess)
      return (PFN_cuTensorMapEncodeTiled_v12000)p;
    (void)cudaGetLastError();
    return nullptr;
  }();
  return fn;
}

int bounded_wait_selftest(unsigned long long limit_ns, cudaStream_t s) {
  bounded_wait_selftest_kernel<<<1, 32, 0, s>>>(limit_ns);
  FDR_LAUNCH_CHECK("bounded_wait_selftest_kernel");
  return FDR_OK;
}

// Tensor map of W as a 2-D float32 array: rows (rate pair, k1) of 2*Q floats, 16 x 256 boxes.
static bool w_tensor_map(CUtensorMap* map, const float2* W, int64_t Q, int64_t rows, int ts) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc || ((uintptr_t)W & 15) != 0) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)(2 * Q), (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)(2 * Q * sizeof(float))};
  const cuuint32_t box[2] = {(cuuint32_t)(2 * ts), 256u};
  const cuuint32_t estr[2] = {1u, 1u};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void*)W, dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tensor map of W for P = 2048 as a 3-D float32 array (2 Q floats, r < 64, 32 * pair + m):
// row k1 = r + 64 m of rate pair q is (r, 32 q + m).  Box {16 floats, 32 r, 32 m}: 8 residues
// of one half (r < 32 or r >= 32) of a tile, 64 KB.
static bool w_tensor_map_halves(CUtensorMap* map, const float2* W, int64_t Q, int64_t npairs) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc || ((uintptr_t)W & 15) != 0) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)(2 * Q), 64u, (cuuint64_t)(32 * npairs)};
  const cuuint64_t strides[2] = {(cuuint64_t)(2 * Q * sizeof(float)),
                                 (cuuint64_t)(64 * 2 * Q * sizeof(float))};
  const cuuint32_t box[3] = {16u, 32u, 32u};
  const cuuint32_t estr[3] = {1u, 1u, 1u};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void*)W, dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// FDR_NO_TMA=1 in the environment selects the register-load output kernel instead.
static bool tma_output_enabled() {
  const char* e = getenv("FDR_NO_TMA");
  return !(e && e[0] == '1');
}

int fused_take_fault() {
  int h = 0;
  if (cudaMemcpyFromSymbol(&h, g_fused_fault, sizeof(int)) != cudaSuccess) {
    (void)cudaGetLastError();
    return FDR_OK;
  }
  if (h) {
    const int z = 0;
    (void)cudaMemcpyToSymbol(g_fused_fault, &z, sizeof(int));
    set_error(FDR_ERR_CUDA, "a bounded TMA/mbarrier wait timed out (flags 0x%x; the FDR of that "
              "call is incomplete)", h);
    return FDR_ERR_CUDA;
  }
  return FDR_OK;
}

// The output pass with the split-bfloat16 tensor-core DFTs: tcgen05 for P = 2048, mma.sync
// for P = 1024 (other shapes, an unaligned destination and a failed tensor-map encode use
// the float32 kernels).
int fused_output_mixed(const FusedPlan* st, const float2* W, float* dest, double* acc, cudaStream_t s) {
  if (st->P == 2048 && st->Q >= 8 && ((uintptr_t)dest & 15) == 0) {
    CUtensorMap map;
    using SH = OutUmmaShape;
    if (w_tensor_map_halves(&map, W, st->Q, st->npairs)) {
      const long long ntiles = (long long)(st->Q / SH::TS) * st->npairs;
      const int grid = (int)std::min<long long>(ntiles, sm_count());
      zdtf_output_umma_kernel<<<grid, SH::T, SH::SMEM, s>>>(
          map, st->N, st->Q, (int)st->Nr, (int)st->npairs, dest, st->tab.rootsP, acc);
      FDR_LAUNCH_CHECK("zdtf_output_umma_kernel");
      return FDR_OK;
    }
  }
  if (st->P == 1024 && st->Q >= 8) {
    CUtensorMap map;
    if (w_tensor_map(&map, W, st->Q, st->npairs * (int64_t)st->P, 8)) {
      const long long ntiles = (long long)(st->Q / 8) * st->npairs;
      const int grid = (int)std::min<long long>(ntiles, sm_count());
      zdtf_output_mma_kernel<<<grid, OutMmaShape::T, OutMmaShape::SMEM, s>>>(
          map, st->N, st->Q, (int)st->Nr, (int)st->npairs, dest, st->tab.rootsP, acc);
      FDR_LAUNCH_CHECK("zdtf_output_mma_kernel");
      return FDR_OK;
    }
  }
  return fused_output(st, W, dest, acc, s);
}

int fused_output(const FusedPlan* st, const float2* W, float* dest, double* acc, cudaStream_t s) {
  const int P = st->P, Q = st->Q;
  if (P == 1024 && Q >= 8 && tma_output_enabled()) {
    CUtensorMap map;
    if (w_tensor_map(&map, W, Q, st->npairs * (int64_t)P, 8)) {
      const long long ntiles = (long long)(Q / 8) * st->npairs;
      using SH = OutTmaShape<32, 32, 8>;
      const int grid = (int)std::min<long long>(ntiles, (long long)SH::MINB * sm_count());
      zdtf_output_tma_kernel<32, 32, 8><<<grid, SH::T, SH::SMEM, s>>>(
          map, st->N, Q, (int)st->Nr, (int)st->npairs, dest, st->tab.rootsP, acc);
      FDR_LAUNCH_CHECK("zdtf_output_tma_kernel");
      return FDR_OK;
    }
  }
  if (P == 2048 && Q >= 8 && tma_output_enabled()) {
    CUtensorMap map;
    using SH = OutTma64Shape<8>;
    if (w_tensor_map(&map, W, Q, st->npairs * (int64_t)P, SH::TS)) {
      const long long ntiles = (long long)(Q / SH::TS) * st->npairs;
      const int grid = (int)std::min<long long>(ntiles, (long long)SH::MINB * sm_count());
      zdtf_output_tma64_kernel<8><<<grid, SH::T, SH::SMEM, s>>>(
          map, st->N, Q, (int)st->Nr, (int)st->npairs, dest, st->tab.rootsP, acc);
      FDR_LAUNCH_CHECK("zdtf_output_tma64_kernel");
      return FDR_OK;
    }
  }
#define LAUNCH_C2(PP, P1, P2)                                                                  \
  if (P == PP) {                                                                               \
    using SH = Out2Shape<P1, P2, 8>;                                                           \
    zdtf_output2_kernel<P1, P2, 8><<<dim3(Q / 8, (unsigned)st->npairs), SH::T, SH::SMEM, s>>>( \
        W, st->N, Q, (int)st->Nr, dest, st->tab.rootsP, acc);                                  \
    FDR_LAUNCH_CHECK("zdtf_output2_kernel");                                                   \
    return FDR_OK;                                                                             \
  }
  LAUNCH_C2(64, 8, 8)
  LAUNCH_C2(128, 8, 16)
  LAUNCH_C2(256, 16, 16)
  LAUNCH_C2(512, 16, 32)
  LAUNCH_C2(1024, 32, 32)
#undef LAUNCH_C2
#define LAUNCH_C(PP)                                                                           \
  if (P == PP) {                                                                               \
    constexpr int TC = AcShape<PP>::TILE, T = AcShape<PP>::T;                                  \
    zdtf_output_kernel<PP, TC, T><<<dim3(Q / TC, (unsigned)st->npairs), T, AcShape<PP>::SMEM, s>>>( \
        W, st->N, Q, (int)st->Nr, dest, st->tab, acc);                                         \
    FDR_LAUNCH_CHECK("zdtf_output_kernel");                                                    \
    return FDR_OK;                                                                             \
  }
  FDR_FOR_P(LAUNCH_C)
#undef LAUNCH_C
  set_error(FDR_ERR_UNSUPPORTED_SIZE, "fused output: P=%d", P);
  return FDR_ERR_UNSUPPORTED_SIZE;
}

// ---- workspace wrappers ----------------------------------------------------------------
static FusedPlan* st_of(fdr_zdt* ws) { return reinterpret_cast<FusedPlan*>(ws->fstate); }

int zdt_fused_setup(fdr_zdt* ws) {
  FusedPlan* st = nullptr;
  FDR_TRY(fused_plan_create(&st, ws->Nf, ws->Nt, ws->Nr));
  ws->fstate = st;
  ws->fP = st->P;
  ws->fQ = st->Q;
  cudaError_t e;
  if ((e = cudaMalloc(&ws->A, sizeof(float2) * fused_A_elems(st))) != cudaSuccess) return cuda_status(e, "cudaMalloc(A)");
  ws->W_pairs = st->npairs;
  if ((e = cudaMalloc(&ws->W, sizeof(float2) * fused_W_elems(st))) != cudaSuccess) return cuda_status(e, "cudaMalloc(W)");
  ws->bytes += fused_plan_table_bytes(st) + (int64_t)sizeof(float2) * (fused_A_elems(st) + fused_W_elems(st));
  ws->fused = true;
  return FDR_OK;
}

void zdt_fused_release(fdr_zdt* ws) {
  fused_plan_destroy(st_of(ws));
  ws->fstate = nullptr;
  cudaFree(ws->A);
  cudaFree(ws->W);
  ws->A = ws->W = nullptr;
}

int zdt_fused_input(fdr_zdt* ws, const float* spec, cudaStream_t s) {
  return fused_input(st_of(ws), spec, ws->A, s);
}

int zdt_fused_A_to_F(fdr_zdt* ws, cudaStream_t s) { return fused_a2f(st_of(ws), ws->A, ws->F, s); }

int zdt_fused_run(fdr_zdt* ws, float r0, float* dest, int window, const double* wk,
                  double* acc, cudaStream_t s) {
  FusedPlan* st = st_of(ws);
  if (!ws->A_valid || !fused_phase_ok(st, r0, ws->dr)) {
    // No fused input stage to start from (F was set by other means) or rates whose exact
    // phase does not fit 62 bits: run the staged stages.
    return zdt_staged_run(ws, r0, dest, window, wk, acc, s);
  }
  FDR_TRY(fused_czt(st, ws->A, ws->W, r0, ws->dr, window, wk, 0, s));
  zdt_mark(ws, "czt", s);
  if (ws->flags & FDR_ZDT_MIXED_PRECISION) FDR_TRY(fused_output_mixed(st, ws->W, dest, acc, s));
  else FDR_TRY(fused_output(st, ws->W, dest, acc, s));
  zdt_mark(ws, "output", s);
  return FDR_OK;
}

// A subset of the workspace's rates: nblocks blocks of 8 consecutive rates, block i starting
// at rate index blk_base[i] (device) of the r0 + j*dr grid; the FDR columns 8i..8i+7 of dest.
// The plan's tables are shared; only the rate count differs.
int zdt_fused_run_blocks(fdr_zdt* ws, const int* blk_base, int64_t nblocks, float* dest,
                         int window, const double* wk, double* acc, cudaStream_t s) {
  const FusedPlan* st = st_of(ws);
  FDR_CHECK_ARG(ws->A_valid, "zdtfdr blocks: the workspace holds no fused input stage");
  FDR_CHECK_ARG(fused_phase_ok(st, ws->r0, ws->dr), "zdtfdr blocks: rates need more than 62 phase bits");
  FDR_CHECK_ARG(nblocks >= 1 && 4 * nblocks <= ws->W_pairs,
                "zdtfdr blocks: %lld blocks exceed the workspace's %lld rates", (long long)nblocks,
                (long long)(2 * ws->W_pairs));
  FusedPlan sub = *st;
  sub.Nr = 8 * nblocks;
  sub.npairs = 4 * nblocks;
  FDR_TRY(fused_czt_blocks(&sub, ws->A, ws->W, ws->r0, ws->dr, window, wk, blk_base, 0, s));
  zdt_mark(ws, "czt", s);
  if (ws->flags & FDR_ZDT_MIXED_PRECISION) FDR_TRY(fused_output_mixed(&sub, ws->W, dest, acc, s));
  else FDR_TRY(fused_output(&sub, ws->W, dest, acc, s));
  zdt_mark(ws, "output", s);
  return FDR_OK;
}

}  // namespace fdr
