// Device-side FFT building blocks shared by the generic engine and the fused ZDT kernels:
// small DFTs on register arrays and an in-place Stockham FFT of power-of-two length over
// several sequences held in shared memory.
#pragma once
#include "fdr_internal.cuh"

namespace fdr {

// DFT of R points in registers; sign -1 forward (exp(-2 pi i ...)), +1 backward.
template <int R>
struct Dft;

template <>
struct Dft<2> {
  __device__ __forceinline__ static void run(float2* v, int) {
    float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <>
struct Dft<4> {
  __device__ __forceinline__ static void run(float2* v, int sign) {
    float2 a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
    float2 c = cadd(v[1], v[3]), d = csub(v[1], v[3]);
    float2 di = cmul_i(d, sign);  // sign*i*d
    v[0] = cadd(a, c);
    v[2] = csub(a, c);
    v[1] = cadd(b, di);
    v[3] = csub(b, di);
  }
};

template <>
struct Dft<8> {
  __device__ __forceinline__ static void run(float2* v, int sign) {
    const float h = 0.70710678118654752440f;
    float2 a[4], b[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      a[r] = cadd(v[r], v[r + 4]);
      b[r] = csub(v[r], v[r + 4]);
    }
    // b[r] *= exp(sign*2*pi*i*r/8)
    const float s = (float)sign;
    b[1] = make_float2(h * (b[1].x - s * b[1].y), h * (b[1].y + s * b[1].x));
    b[2] = cmul_i(b[2], sign);
    b[3] = make_float2(h * (-b[3].x - s * b[3].y), h * (-b[3].y + s * b[3].x));
    Dft<4>::run(a, sign);
    Dft<4>::run(b, sign);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      v[2 * m] = a[m];
      v[2 * m + 1] = b[m];
    }
  }
};

template <>
struct Dft<16> {
  // 4 x 4 decomposition: r = r1 + 4*r2, m = m2 + 4*m1
  __device__ __forceinline__ static void run(float2* v, int sign) {
    // cos / sin of 2*pi*e/16, e = 0..9
    const float C[10] = {1.f, 0.92387953251128675613f, 0.70710678118654752440f,
                         0.38268343236508977173f, 0.f, -0.38268343236508977173f,
                         -0.70710678118654752440f, -0.92387953251128675613f, -1.f,
                         -0.92387953251128675613f};
    const float S[10] = {0.f, 0.38268343236508977173f, 0.70710678118654752440f,
                         0.92387953251128675613f, 1.f, 0.92387953251128675613f,
                         0.70710678118654752440f, 0.38268343236508977173f, 0.f,
                         -0.38268343236508977173f};
    float2 y[4][4];
#pragma unroll
    for (int r1 = 0; r1 < 4; ++r1) {
      float2 t[4] = {v[r1], v[r1 + 4], v[r1 + 8], v[r1 + 12]};
      Dft<4>::run(t, sign);
#pragma unroll
      for (int m2 = 0; m2 < 4; ++m2) y[r1][m2] = t[m2];
    }
#pragma unroll
    for (int r1 = 1; r1 < 4; ++r1)
#pragma unroll
      for (int m2 = 1; m2 < 4; ++m2) {
        const int e = r1 * m2;
        y[r1][m2] = cmul(y[r1][m2], make_float2(C[e], sign * S[e]));
      }
#pragma unroll
    for (int m2 = 0; m2 < 4; ++m2) {
      float2 t[4] = {y[0][m2], y[1][m2], y[2][m2], y[3][m2]};
      Dft<4>::run(t, sign);
#pragma unroll
      for (int m1 = 0; m1 < 4; ++m1) v[m2 + 4 * m1] = t[m1];
    }
  }
};

template <>
struct Dft<32> {
  // radix-2 split into even / odd halves, each a 16-point DFT
  __device__ __forceinline__ static void run(float2* v, int sign) {
    // cos / sin of 2*pi*m/32, m = 0..15
    const float C[16] = {1.f, 0.98078528040323044913f, 0.92387953251128675613f,
                         0.83146961230254523708f, 0.70710678118654752440f,
                         0.55557023301960222474f, 0.38268343236508977173f,
                         0.19509032201612826785f, 0.f, -0.19509032201612826785f,
                         -0.38268343236508977173f, -0.55557023301960222474f,
                         -0.70710678118654752440f, -0.83146961230254523708f,
                         -0.92387953251128675613f, -0.98078528040323044913f};
    const float S[16] = {0.f, 0.19509032201612826785f, 0.38268343236508977173f,
                         0.55557023301960222474f, 0.70710678118654752440f,
                         0.83146961230254523708f, 0.92387953251128675613f,
                         0.98078528040323044913f, 1.f, 0.98078528040323044913f,
                         0.92387953251128675613f, 0.83146961230254523708f,
                         0.70710678118654752440f, 0.55557023301960222474f,
                         0.38268343236508977173f, 0.19509032201612826785f};
    float2 e[16], o[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      e[i] = v[2 * i];
      o[i] = v[2 * i + 1];
    }
    Dft<16>::run(e, sign);
    Dft<16>::run(o, sign);
#pragma unroll
    for (int m = 0; m < 16; ++m) {
      const float2 t = (m == 0) ? o[0] : cmul(o[m], make_float2(C[m], sign * S[m]));
      v[m] = cadd(e[m], t);
      v[m + 16] = csub(e[m], t);
    }
  }
};

template <>
struct Dft<3> {
  __device__ __forceinline__ static void run(float2* v, int sign) {
    const float c = -0.5f, sn = 0.86602540378443864676f;
    float2 t1 = cadd(v[1], v[2]);
    float2 t2 = make_float2(v[0].x + c * t1.x, v[0].y + c * t1.y);
    float2 d = csub(v[1], v[2]);
    float2 t3 = cmul_i(cscale(d, sn), sign);
    v[0] = cadd(v[0], t1);
    v[1] = cadd(t2, t3);
    v[2] = csub(t2, t3);
  }
};

template <>
struct Dft<5> {
  __device__ __forceinline__ static void run(float2* v, int sign) {
    const float c1 = 0.30901699437494742410f, c2 = -0.80901699437494742410f;
    const float s1 = 0.95105651629515357212f, s2 = 0.58778525229247312917f;
    float2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
    float2 t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
    float2 v0 = v[0];
    float2 a1 = make_float2(v0.x + c1 * t1.x + c2 * t2.x, v0.y + c1 * t1.y + c2 * t2.y);
    float2 a2 = make_float2(v0.x + c2 * t1.x + c1 * t2.x, v0.y + c2 * t1.y + c1 * t2.y);
    float2 b1 = cmul_i(make_float2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y), sign);
    float2 b2 = cmul_i(make_float2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y), sign);
    v[0] = cadd(v0, cadd(t1, t2));
    v[1] = cadd(a1, b1);
    v[4] = csub(a1, b1);
    v[2] = cadd(a2, b2);
    v[3] = csub(a2, b2);
  }
};

// Shared-memory layout of an FFT sequence: element i is stored at pidx(i) = i + i/16
// within a sequence of padded stride padlen(LEN).  With the radix plan below every
// half-warp of a Stockham pass then reads and writes 16 distinct 8-byte bank pairs.
__host__ __device__ constexpr int padlen(int len) { return len + len / 16; }
__device__ __forceinline__ int pidx(int i) { return i + (i >> 4); }

// Radix of the pass that starts with NS (= product of the earlier radices) for length LEN.
__host__ __device__ constexpr int plan_radix(int rem) {
  return (rem % 16 == 0 && rem != 32) ? 16 : ((rem % 8 == 0) ? 8 : ((rem % 4 == 0) ? 4 : 2));
}
// Offset, in a per-length twiddle table, of the pass that starts at NS.  The table holds,
// for each pass with NS > 1, exp(-2*pi*i*r*k/(NS*R)) at [(r-1)*NS + k] (r in [1,R), k < NS),
// so that threads with consecutive k read consecutive entries.
__host__ __device__ constexpr int tw_offset(int len, int ns_target) {
  int off = 0, ns = 1;
  while (ns < ns_target) {
    const int R = plan_radix(len / ns);
    if (ns > 1) off += (R - 1) * ns;
    ns *= R;
  }
  return off;
}
__host__ __device__ constexpr int tw_size(int len) { return tw_offset(len, len); }

// One radix-R Stockham pass over NSEQ power-of-two sequences of length LEN stored at
// buf[seq*SSTRIDE + pidx(i)], in place: every thread first reads the inputs of its
// butterflies into registers, the block synchronises, then the outputs are written.
// twt is the per-length twiddle table (tw_offset layout, forward sign).
template <int LEN, int NSEQ, int SSTRIDE, int T, int SIGN, int NS, int R>
__device__ __forceinline__ void stockham_pass(float2* buf, const float2* twt) {
  constexpr int NBF = LEN / R;             // butterflies per sequence
  constexpr int NB = NBF * NSEQ;           // butterflies in total
  constexpr int PER = (NB + T - 1) / T;    // per thread
  const float2* tw = twt + tw_offset(LEN, NS);
  float2 v[PER][R];
#pragma unroll
  for (int i = 0; i < PER; ++i) {
    const int j = threadIdx.x + i * T;
    if (NB % T == 0 || j < NB) {
      const int seq = j / NBF, jj = j - seq * NBF;
      const float2* a = buf + seq * SSTRIDE;
#pragma unroll
      for (int r = 0; r < R; ++r) v[i][r] = a[pidx(jj + r * NBF)];
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < PER; ++i) {
    const int j = threadIdx.x + i * T;
    if (NB % T == 0 || j < NB) {
      const int seq = j / NBF, jj = j - seq * NBF;
      const int k = jj % NS;
      if (NS > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          float2 w = tw[(r - 1) * NS + k];
          if (SIGN > 0) w.y = -w.y;
          v[i][r] = cmul(v[i][r], w);
        }
      }
      Dft<R>::run(v[i], SIGN);
      float2* b = buf + seq * SSTRIDE;
      const int base = (jj / NS) * NS * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) b[pidx(base + r * NS)] = v[i][r];
    }
  }
  __syncthreads();
}

// One radix-R Stockham pass from src to dst (same layout, distinct buffers): each thread
// transforms its butterflies one at a time; ends with a barrier.
template <int LEN, int NSEQ, int SSTRIDE, int T, int SIGN, int NS, int R>
__device__ __forceinline__ void stockham_pass_oop(const float2* src, float2* dst, const float2* twt) {
  constexpr int NBF = LEN / R;
  constexpr int NB = NBF * NSEQ;
  constexpr int PER = (NB + T - 1) / T;
  const float2* tw = twt + tw_offset(LEN, NS);
#pragma unroll
  for (int i = 0; i < PER; ++i) {
    const int j = threadIdx.x + i * T;
    if (NB % T == 0 || j < NB) {
      const int seq = j / NBF, jj = j - seq * NBF;
      const int k = jj % NS;
      float2 v[R];
      const float2* a = src + seq * SSTRIDE;
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = a[pidx(jj + r * NBF)];
      if (NS > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          float2 w = tw[(r - 1) * NS + k];
          if (SIGN > 0) w.y = -w.y;
          v[r] = cmul(v[r], w);
        }
      }
      Dft<R>::run(v, SIGN);
      float2* b = dst + seq * SSTRIDE;
      const int base = (jj / NS) * NS * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) b[pidx(base + r * NS)] = v[r];
    }
  }
  __syncthreads();
}

// The last pass of an in-place Stockham FFT whose outputs go to emit(seq, i, value)
// instead of shared memory (natural order i).  Ends with a barrier if SYNC.
template <int LEN, int NSEQ, int SSTRIDE, int T, int SIGN, int NS, int R, class Emit, bool SYNC = true>
__device__ __forceinline__ void stockham_last_pass_emit(float2* buf, const float2* twt, Emit emit) {
  constexpr int NBF = LEN / R;
  constexpr int NB = NBF * NSEQ;
  constexpr int PER = (NB + T - 1) / T;
  const float2* tw = twt + tw_offset(LEN, NS);
#pragma unroll
  for (int i = 0; i < PER; ++i) {
    const int j = threadIdx.x + i * T;
    if (NB % T == 0 || j < NB) {
      const int seq = j / NBF, jj = j - seq * NBF;
      const int k = jj % NS;
      float2 v[R];
      const float2* a = buf + seq * SSTRIDE;
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = a[pidx(jj + r * NBF)];
      if (NS > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          float2 w = tw[(r - 1) * NS + k];
          if (SIGN > 0) w.y = -w.y;
          v[r] = cmul(v[r], w);
        }
      }
      Dft<R>::run(v, SIGN);
      const int base = (jj / NS) * NS * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) emit(seq, base + r * NS, v[r]);
    }
  }
  if (SYNC) __syncthreads();
}

template <int LEN, int NSEQ, int SSTRIDE, int T, int SIGN, int NS, class Emit>
__device__ __forceinline__ void stockham_passes_emit(float2* buf, const float2* twt, Emit emit) {
  constexpr int R = plan_radix(LEN / NS);
  if constexpr (NS * R < LEN) {
    stockham_pass<LEN, NSEQ, SSTRIDE, T, SIGN, NS, R>(buf, twt);
    stockham_passes_emit<LEN, NSEQ, SSTRIDE, T, SIGN, NS * R>(buf, twt, emit);
  } else {
    stockham_last_pass_emit<LEN, NSEQ, SSTRIDE, T, SIGN, NS, R>(buf, twt, emit);
  }
}

// Ping-pong form of stockham_passes_emit: the passes alternate between buffers a and b
// (a holds the input), the last pass reads whichever holds the data and hands its outputs
// to emit; no barrier after it.  The buffer that the last pass does NOT read was last read
// before the final barrier, so the caller may refill it at once.
template <int LEN, int NSEQ, int SSTRIDE, int T, int SIGN, int NS, class Emit>
__device__ __forceinline__ void stockham_passes_emit_pp(float2* a, float2* b, const float2* twt, Emit emit) {
  constexpr int R = plan_radix(LEN / NS);
  if constexpr (NS * R < LEN) {
    stockham_pass_oop<LEN, NSEQ, SSTRIDE, T, SIGN, NS, R>(a, b, twt);
    stockham_passes_emit_pp<LEN, NSEQ, SSTRIDE, T, SIGN, NS * R>(b, a, twt, emit);
  } else {
    stockham_last_pass_emit<LEN, NSEQ, SSTRIDE, T, SIGN, NS, R, Emit, false>(a, twt, emit);
  }
}

// Number of shared-memory passes before the emitting pass of a length-LEN FFT.
__host__ __device__ constexpr int passes_before_emit(int len) {
  int n = 0, ns = 1;
  while (ns * plan_radix(len / ns) < len) {
    ns *= plan_radix(len / ns);
    ++n;
  }
  return n;
}

// smem_fft whose final pass hands each output to emit(seq, i, value) (no shared store).
template <int LEN, int NSEQ, int SSTRIDE, int T, int SIGN, class Emit>
__device__ __forceinline__ void smem_fft_emit(float2* buf, const float2* twt, Emit emit) {
  static_assert((LEN & (LEN - 1)) == 0, "power-of-two length");
  static_assert(SSTRIDE >= padlen(LEN), "sequence stride too small");
  stockham_passes_emit<LEN, NSEQ, SSTRIDE, T, SIGN, 1>(buf, twt, emit);
}

// ------------------------------------------------------------------------------------
// FFTs by a group of whole warps of a block (warp-specialised kernels): the group's T
// threads, numbered ltid = 0..T-1, synchronise on hardware named barrier BAR (bar.sync with
// a thread count: no other warp of the block takes part).
// ------------------------------------------------------------------------------------
template <int ID, int NTHR>
__device__ __forceinline__ void named_sync() {
  asm volatile("bar.sync %0, %1;" ::"n"(ID), "n"(NTHR) : "memory");
}
template <int ID, int NTHR>
__device__ __forceinline__ void named_arrive() {
  asm volatile("bar.arrive %0, %1;" ::"n"(ID), "n"(NTHR) : "memory");
}

// In-place Stockham FFT of NSEQ sequences (layout as smem_fft) by a group of T threads whose
// last pass hands each output to emit(seq, i, value); the inputs must be visible to the group
// when it is called.  Every pass but the last reads its butterflies into registers, waits for
// the group, writes, and waits again; the last pass only reads, so the buffer may be reused
// once every thread of the group has returned.
template <int LEN, int NSEQ, int SSTRIDE, int T, int SIGN, int BAR, int NS, class Emit>
__device__ __forceinline__ void group_fft_emit(float2* buf, const float2* twt, int ltid, Emit emit) {
  constexpr int R = plan_radix(LEN / NS);
  constexpr int NBF = LEN / R;
  constexpr int NB = NBF * NSEQ;
  constexpr int PER = (NB + T - 1) / T;
  const float2* tw = twt + tw_offset(LEN, NS);
  float2 v[PER][R];
#pragma unroll
  for (int i = 0; i < PER; ++i) {
    const int j = ltid + i * T;
    if (NB % T == 0 || j < NB) {
      const int seq = j / NBF, jj = j - seq * NBF;
      const float2* a = buf + seq * SSTRIDE;
#pragma unroll
      for (int r = 0; r < R; ++r) v[i][r] = a[pidx(jj + r * NBF)];
    }
  }
  if constexpr (NS * R < LEN) named_sync<BAR, T>();  // every input read before any write
#pragma unroll
  for (int i = 0; i < PER; ++i) {
    const int j = ltid + i * T;
    if (NB % T == 0 || j < NB) {
      const int seq = j / NBF, jj = j - seq * NBF;
      const int k = jj % NS;
      if (NS > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          float2 w = tw[(r - 1) * NS + k];
          if (SIGN > 0) w.y = -w.y;
          v[i][r] = cmul(v[i][r], w);
        }
      }
      Dft<R>::run(v[i], SIGN);
      const int base = (jj / NS) * NS * R + k;
      if constexpr (NS * R < LEN) {
        float2* b = buf + seq * SSTRIDE;
#pragma unroll
        for (int r = 0; r < R; ++r) b[pidx(base + r * NS)] = v[i][r];
      } else {
#pragma unroll
        for (int r = 0; r < R; ++r) emit(seq, base + r * NS, v[i][r]);
      }
    }
  }
  if constexpr (NS * R < LEN) {
    named_sync<BAR, T>();  // the pass's outputs are visible to the group
    group_fft_emit<LEN, NSEQ, SSTRIDE, T, SIGN, BAR, NS * R>(buf, twt, ltid, emit);
  }
}

template <int LEN, int NSEQ, int SSTRIDE, int T, int SIGN, int NS>
__device__ __forceinline__ void stockham_passes(float2* buf, const float2* twt) {
  if constexpr (NS < LEN) {
    constexpr int R = plan_radix(LEN / NS);
    stockham_pass<LEN, NSEQ, SSTRIDE, T, SIGN, NS, R>(buf, twt);
    stockham_passes<LEN, NSEQ, SSTRIDE, T, SIGN, NS * R>(buf, twt);
  }
}

// In-place FFT (natural order in and out) of NSEQ sequences of power-of-two length LEN
// held at buf[seq*SSTRIDE + pidx(i)] (SSTRIDE >= padlen(LEN)).  twt: the length's
// twiddle table (tw_size(LEN) entries, see tw_offset).  Must be called by all T threads of
// the block; the caller synchronises before (the inputs are visible); the function ends
// with a barrier.
template <int LEN, int NSEQ, int SSTRIDE, int T, int SIGN>
__device__ __forceinline__ void smem_fft(float2* buf, const float2* twt) {
  static_assert((LEN & (LEN - 1)) == 0, "power-of-two length");
  static_assert(SSTRIDE >= padlen(LEN), "sequence stride too small");
  stockham_passes<LEN, NSEQ, SSTRIDE, T, SIGN, 1>(buf, twt);
}

}  // namespace fdr
