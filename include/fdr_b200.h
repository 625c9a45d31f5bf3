/*
 * fdr_b200.h -- C ABI of the B200-native frequency-drift-rate (FDR) transform library
 * (libfdrb200.so).
 *
 * This is the drop-in boundary for FrequencyDriftRateTransforms.jl's GPU path: the
 * reference specialises three generics for CuArrays in
 * ext/CUDAFrequencyDriftRateTransformsExt.jl (plan_ffts! :50-82, output! :94-103,
 * fdrsynchronize :26-28) and runs every other stage as CUDA.jl broadcasts.  A Julia
 * extension that ccalls this library replaces all of them; each entry point below names
 * the reference function it stands in for.
 *
 * Conventions
 *  - Every function returns an fdr_status (0 = FDR_OK).  On failure,
 *    fdr_last_error_string() describes the last error of the calling host thread.
 *    Nonzero statuses correspond to the reference's thrown errors (@assert, error(...)).
 *  - Arrays are Julia column-major: an Nf x Nt spectrogram has channel (frequency) index
 *    fastest; element (n, t) of a matrix with leading dimension ld is at p[n + t*ld].
 *    Complex arrays are interleaved float pairs (ComplexF32).
 *  - Array arguments are DEVICE pointers unless the parameter says "host".  On the fused
 *    ZDT path (zdtfdr!, its rate blocks, the fused proto-hit scan and the batch) the
 *    spectrogram and the FDR destinations must be 8-byte aligned (cudaMalloc'd and CuArray
 *    storage, and its columns for even Nf, are); other pointers are rejected with
 *    FDR_ERR_INVALID_ARGUMENT before any kernel runs.
 *  - Work is ordered on the given CUDA stream (NULL = the legacy default stream) and is
 *    asynchronous unless the function says it synchronises (those that return values
 *    computed on the device to host variables).
 *  - Element type is Float32 (the reference is generic over Real element types; this
 *    library implements Float32 only).
 *  - Indices returned to the caller are ZERO-based (the Julia shim adds 1).
 */
#ifndef FDR_B200_H
#define FDR_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* cudaStream_t-compatible handle. */
typedef struct CUstream_st* fdr_stream_t;

typedef enum fdr_status {
  FDR_OK = 0,
  FDR_ERR_INVALID_ARGUMENT = 1,   /* @assert / error() in the reference */
  FDR_ERR_UNSUPPORTED_SIZE = 2,   /* FFT length with a prime factor > 64, or beyond limits */
  FDR_ERR_UNSUPPORTED_WINDOW = 3, /* zdtfdr.jl:311-313 "unsupported window type" */
  FDR_ERR_OUT_OF_MEMORY = 4,
  FDR_ERR_CUDA = 5,               /* a CUDA runtime call failed */
  FDR_ERR_CAPACITY = 6,           /* more proto-hits than the caller's capacity */
  FDR_ERR_NO_DEVICE = 7
} fdr_status;

typedef enum fdr_window {
  FDR_WINDOW_RECT = 0,    /* zdtfdr.jl:307-309 (default) */
  FDR_WINDOW_HAMMING = 1, /* zdtfdr.jl:303-305: 0.53836 + 0.46164*cospi(2k/Nf) */
  FDR_WINDOW_CUSTOM = 2   /* w(k, Nf) evaluated by the caller: K = Nf/2+1 float64 values */
} fdr_window;

/* Workspace flags (fdr_zdt_create). */
#define FDR_ZDT_OUTPUT_ALIGNED 0x1u /* accepted for API parity (FFTW planner hint); no effect */
#define FDR_ZDT_EXACT_PHASE 0x2u    /* staged stages reduce chirp phases exactly (default:
                                       the reference's Float32 phase arguments) */
#define FDR_ZDT_STAGED_ONLY 0x4u    /* fdr_zdt_execute always runs the staged kernels */
#define FDR_ZDT_MIXED_PRECISION 0x8u /* fused path with P = 2048 (tcgen05, tensor-memory
                                       accumulators; e.g. Nf = 2^20 and 2^21 with Nt <= 16) or
                                       P = 1024 (mma.sync; e.g. Nf = 2^19): the inverse DFT_P
                                       runs as split-bfloat16 tensor-core contractions with
                                       float32 accumulation (relative error ~1e-5 of the FDR's
                                       peak instead of ~1e-6; same split as without the flag;
                                       no counterpart in the reference) */

#define FDR_ZDT_FAST_STATS 0x10u     /* the snr statistics of the fused proto-hit scan
                                       (fdr_zdtfdr_protohits) come from float64 column moments
                                       accumulated while the FDR is written: two fewer reads
                                       of the FDR, but m and s may differ from the reference's
                                       Float32 pairwise values in the last bits (default: the
                                       Float32 pairwise values of fdr_stats) */

/* `snr` argument of the proto-hit searches: 0 = `threshold` is the threshold itself;
   otherwise findprotohits(...; snr=true) computes fdrdenormalize(threshold, fdrs) =
   threshold*s + m (fdrutils.jl:104-107) in Julia's promoted type of `threshold`:
   FDR_SNR_F64 for a Float64 snr (Float64 arithmetic and comparison), FDR_SNR_F32 for an
   Int or Float32 snr (Float32 arithmetic: Float32(snr)*s rounded, + m rounded; Float32
   comparison). */
#define FDR_SNR_F64 1
#define FDR_SNR_F32 2

/* Rate arithmetic for intshift/intfdr (round(rate*(t-1)) in the rate's element type). */
#define FDR_RATES_F64 0
#define FDR_RATES_F32 1

/* ---------------------------------------------------------------------------------- */
/* Library information                                                                 */
/* ---------------------------------------------------------------------------------- */
const char* fdr_version(void);
const char* fdr_last_error_string(void);
const char* fdr_status_string(int status);
/* Number of CUDA kernels this library has launched in the process (a diagnostic with no
   counterpart in the reference; used to count device launches in benchmarks). */
int64_t fdr_kernel_launches(void);
/* fdrsynchronize (fdrutils.jl:129-130; CuArray method ext:26-28): synchronise `stream`
   (NULL: the whole device).  Also reports, once, a bounded wait of the TMA-fed kernels that
   ran out since the last call (FDR_ERR_CUDA; that call's FDR is incomplete). */
int fdr_synchronize(fdr_stream_t stream);
/* Debug build (no counterpart in the reference): libfdrb200_debug.so is compiled with
   FDR_DEBUG, in which the kernels check their global-memory indices against the buffers'
   extents; a failed check skips the access and records the first violation per source
   unit (unit id and line), which fdr_synchronize reports as FDR_ERR_CUDA.
   fdr_debug_build() is 1 in that library, 0 in libfdrb200.so.  fdr_debug_fault synchronises
   `stream` (NULL: the device) and returns, then clears, the first recorded violation in
   *word (bit 63 set, unit id in bits 32..62, line in bits 0..31; 0 if none or in the
   normal build). */
int fdr_debug_build(void);
int fdr_debug_fault(uint64_t* word, fdr_stream_t stream);
/* Self-test of that failure path (no counterpart in the reference): launches one CTA that
   waits on an mbarrier nothing completes, gives up after limit_ns (<= 1 s) and raises the
   fault flag, so that the next fdr_synchronize returns FDR_ERR_CUDA.  No GPU fault. */
int fdr_selftest_bounded_wait(int64_t limit_ns, fdr_stream_t stream);

/* ---------------------------------------------------------------------------------- */
/* zdtutils.jl                                                                         */
/* ---------------------------------------------------------------------------------- */
/* calcNl (zdtutils.jl:7-9): smallest n >= Nt+Nr-1 whose prime factors are in `factors`
   (host array; NULL -> (2,3,5)).  Returns -1 on invalid input. */
int64_t fdr_calc_nl(int64_t Nt, int64_t Nr, const int64_t* factors, int nfactors);
/* growNr (zdtutils.jl:17-19). */
int64_t fdr_grow_nr(int64_t Nt, int64_t Nr, const int64_t* factors, int nfactors);
/* estimate_memory (zdtutils.jl:35-53): the reference's formula, in bytes. */
int64_t fdr_estimate_memory(int64_t Nf, int64_t Nt, int64_t Nr, int64_t Ni, int64_t No,
                            const int64_t* factors, int nfactors);

/* ---------------------------------------------------------------------------------- */
/* ZDT workspace and stages (zdtfdr.jl)                                                */
/* ---------------------------------------------------------------------------------- */
typedef struct fdr_zdt fdr_zdt;

typedef struct fdr_zdt_info {
  int64_t Nf, Nt, Nr, Nl, K; /* K = Nf/2 + 1 */
  float r0, dr;
  uint32_t flags;
  int32_t fused;             /* 1 if fdr_zdt_execute uses the fused kernels */
  int64_t bytes;             /* device bytes owned by the workspace */
  int32_t nfactors;
  int64_t factors[8];
} fdr_zdt_info;

/* ZDTWorkspace(spectrogram, r0, dr, Nr, factors; output_aligned) (zdtfdr.jl:37-87 and
   plan_ffts! ext:50-82): allocates F (K x Nt), Y (K x Nl), V (K x Nl) and FFT scratch,
   runs input!(spectrogram) when `spectrogram` is non-NULL, computes V (computeV!,
   zdtfdr.jl:173-187) and synchronises `stream` (zdtfdr.jl:72). */
int fdr_zdt_create(fdr_zdt** ws, const float* spectrogram, int64_t Nf, int64_t Nt,
                   float r0, float dr, int64_t Nr, const int64_t* factors, int nfactors,
                   uint32_t flags, fdr_stream_t stream);
int fdr_zdt_destroy(fdr_zdt* ws);
/* show / sizeof / driftrates (zdtfdr.jl:89-103, zdtutils.jl:62-64). */
int fdr_zdt_get_info(const fdr_zdt* ws, fdr_zdt_info* info);
/* No reference counterpart: the four-step split Nf = P x Q that the fused path of a
   workspace with these sizes and flags uses (P residues in the input and output passes, Q
   bins per czt CTA).  FDR_ERR_UNSUPPORTED_SIZE when the fused path does not apply (the
   staged kernels run).  Host arithmetic only: touches no device. */
int fdr_zdt_fused_split(int64_t Nf, int64_t Nt, int64_t Nr, uint32_t flags, int64_t* P, int64_t* Q);
/* Field access to ws.F, ws.Y (Yf and Ys are its first Nt / Nr columns) and ws.V. */
int fdr_zdt_buffers(fdr_zdt* ws, void** F, void** Y, void** V);
/* input! (zdtfdr.jl:209-212): F = rfft(spectrogram, dims=1). */
int fdr_zdt_input(fdr_zdt* ws, const float* spectrogram, fdr_stream_t stream);
/* preprocess! (zdtfdr.jl:221-239): Yf = F .* prephase(r0); Y[:, Nt+1:end] = 0. */
int fdr_zdt_preprocess(fdr_zdt* ws, float r0, fdr_stream_t stream);
/* convolve! (zdtfdr.jl:249-253): Y = ifft_l(fft_l(Y) .* V) (normalised). */
int fdr_zdt_convolve(fdr_zdt* ws, fdr_stream_t stream);
/* postprocess! (zdtfdr.jl:297-321): Ys .*= postphase .* w(k, Nf).  `custom_window` is a
   device array of K float64 values for FDR_WINDOW_CUSTOM, else ignored. */
int fdr_zdt_postprocess(fdr_zdt* ws, int window, const double* custom_window,
                        fdr_stream_t stream);
/* output! (zdtfdr.jl:328-331; CuArray method ext:94-103): dest (Nf x Nr, leading
   dimension Nf) = irfft(Ys, Nf) (normalised).  Like the reference's CuArray method it may
   clobber Ys, so call it once per ZDT. */
int fdr_zdt_output(fdr_zdt* ws, float* dest, fdr_stream_t stream);
/* zdtfdr!([w,] dests, ws[, spectrogram]; r0) (zdtfdr.jl:349-378): if `spectrogram` is
   non-NULL runs input!, then for b in 0..nbatch-1 computes the FDR for rates
   r0s[b] + j*dr (j < Nr) into dests[b] (Nf x Nr).  `r0s` and `dests` are HOST arrays of
   nbatch entries; r0s == NULL uses the workspace's r0 for every batch.  Uses the fused
   kernels when available (power-of-two Nf >= 4096 and FDR_ZDT_STAGED_ONLY not set),
   else the staged stages.  After a fused call the contents of Y are unspecified. */
int fdr_zdt_execute(fdr_zdt* ws, const float* spectrogram, const float* r0s, int64_t nbatch,
                    float* const* dests, int window, const double* custom_window,
                    fdr_stream_t stream);
/* The fused threshold/proto-hit scan: zdtfdr!(dests, ws[, spectrogram]; r0) followed by
   findprotohits(dests, threshold; snr) (zdtfdr.jl:349-378, fdrutils.jl:148-169).  With snr,
   the statistics are fdr_stats's Float32 pairwise values over the dests (two reads of the
   FDR; the first also keeps each pairwise leaf's maximum, so that only leaves that can hold
   a hit are read again for the proto-hits), or, for a workspace created with
   FDR_ZDT_FAST_STATS, float64 column moments accumulated while the FDR columns are written
   (no extra read; the FDR is then read once more to count the proto-hits).  Hits, count and
   threshold as in fdr_findprotohits (the batches are the hcat'd matrices).  Synchronises
   `stream`. */
int fdr_zdtfdr_protohits(fdr_zdt* ws, const float* spectrogram, const float* r0s, int64_t nbatch,
                         float* const* dests, int window, const double* custom_window,
                         double threshold, int snr, int64_t* hits, int64_t capacity,
                         int64_t* count, double* threshold_used, fdr_stream_t stream);
/* zdtfdr! over a subset of the workspace's drift rates in one pass: nblocks blocks of 8
   consecutive rates, block i covering rates r0 + (8*blocks[i] + u)*dr (u < 8, host array,
   8*(blocks[i]+1) <= Nr, 8*nblocks <= Nr rounded up to even), written to the FDR columns
   8i..8i+7 of dest (device, Nf x 8*nblocks column-major).  One input stage and one pass of
   the fused kernels for all blocks, so a sparse set of rate windows costs in proportion to
   its size (the r0 iterator of zdtfdr!, zdtfdr.jl:354, pays a full pass per r0).  No
   counterpart in the reference; fused workspaces only (FDR_ERR_UNSUPPORTED_SIZE else). */
int fdr_zdt_execute_blocks(fdr_zdt* ws, const float* spectrogram, const int32_t* blocks,
                           int64_t nblocks, float* dest, int window, const double* custom_window,
                           fdr_stream_t stream);
/* fdr_zdt_execute_blocks followed by the fused threshold/proto-hit scan of its dest, as
   fdr_zdtfdr_protohits (statistics over the computed columns; hit j is the dest column). */
int fdr_zdtfdr_blocks_protohits(fdr_zdt* ws, const float* spectrogram, const int32_t* blocks,
                                int64_t nblocks, float* dest, int window, const double* custom_window,
                                double threshold, int snr, int64_t* hits, int64_t capacity,
                                int64_t* count, double* threshold_used, fdr_stream_t stream);
/* Per-stage device time of the last fdr_zdt_execute call (enable with
   fdr_zdt_set_timing(ws, 1)); times[i] in milliseconds, names via stage_names. */
int fdr_zdt_set_timing(fdr_zdt* ws, int enable);
int fdr_zdt_stage_times(fdr_zdt* ws, float* times_ms, int max_stages, int* nstages,
                        const char** stage_names);

/* ---------------------------------------------------------------------------------- */
/* Batches of coarse channels (no single reference function: the reference runs one      */
/* zdtfdr! per spectrogram; pipelines loop over coarse channels, its README.md:57-71)     */
/* ---------------------------------------------------------------------------------- */
typedef struct fdr_batch fdr_batch;
typedef struct fdr_batch_channel {
  int64_t Nf, Nt, Nr;        /* spectrogram Nf x Nt; rates r0 + j*dr, j < Nr */
  float r0, dr;
  const float* spectrogram;  /* device, Nf x Nt column-major */
  float* fdr;                /* device, Nf x Nr column-major (written by each launch) */
} fdr_batch_channel;
/* Plan nch channels of any shapes over `slots` streams (1..16): channels of equal
   (Nf, Nt, Nr) share one fused plan; each slot owns intermediates sized for the largest
   channel.  The channel array (host) is copied; the device arrays must outlive the batch. */
int fdr_batch_create(fdr_batch** batch, const fdr_batch_channel* channels, int64_t nch,
                     int slots, fdr_stream_t stream);
/* Autotuner: per distinct shape, the czt kernel's rate-group split (timed over 1, 2, 4, 8),
   then the number of active slots (timed over powers of two up to `slots`); cached per shape
   for the process.  Call before fdr_batch_capture.  Synchronises `stream`. */
int fdr_batch_autotune(fdr_batch* batch, fdr_stream_t stream);
/* Records the whole batch (forked over the active slot streams) into one CUDA graph;
   `stream` must not be the legacy default stream.  Runs the batch once eagerly first. */
int fdr_batch_capture(fdr_batch* batch, fdr_stream_t stream);
/* Computes every channel's FDR: one cudaGraphLaunch when captured, else eager launches. */
int fdr_batch_launch(fdr_batch* batch, fdr_stream_t stream);
int fdr_batch_get_tuning(const fdr_batch* batch, int* groups, int ngroups, int* nplans,
                         int* active_slots);
int fdr_batch_info(const fdr_batch* batch, int64_t* nchannels, int64_t* nfused, int64_t* bytes,
                   int* captured);
int fdr_batch_destroy(fdr_batch* batch);

/* ---------------------------------------------------------------------------------- */
/* Learned drift-rate window proposal (no reference counterpart: a training/serving     */
/* extension of the batched rate search, batchrates.jl:22-60, zdtfdr.jl:354)             */
/* ---------------------------------------------------------------------------------- */
typedef struct fdr_propose_net fdr_propose_net;
/* 4-layer 1-D conv net over nbins coarse bins with nt input channels (nt <= 64): three k=5 layers of
   `width` channels with ReLU, a 1x1 layer to nwin window logits, max over bins.  This build
   supports width 32, ksize 5, nwin 16.  Weights: seeded He-uniform, float32 master copy,
   float16 copy used by the forward pass.  max_batch bounds the batch of every call. */
int fdr_propose_create(fdr_propose_net** net, int nbins, int nt, int width, int ksize, int nwin,
                       int max_batch, uint64_t seed);
int fdr_propose_destroy(fdr_propose_net* net);
int fdr_propose_num_params(const fdr_propose_net* net, int64_t* count);
/* Network input of one spectrogram (Nf x Nt): out[t][bin] = (sum of `factor` consecutive
   channels - factor) / sqrt(factor), bin < Nf/factor (device, Nt x Nf/factor row-major);
   with compress != 0 each value v is replaced by sign(v) * log1p(|v|).  Nt <= 64. */
int fdr_propose_features(const float* spectrogram, int64_t Nf, int64_t Nt, int factor,
                         int compress, float* out, fdr_stream_t stream);
/* Drift evidence of one spectrogram: out[l + maxlag][bin] = sum over the `factor` channels n
   of the bin and over t < Nt-1 of (s[n,t] - 1) * (s[(n + l) mod Nf, t+1] - 1), divided by
   sqrt(factor * (Nt - 1)), for lags l in [-maxlag, maxlag] (maxlag 8, factor <= 4096; device,
   (2*maxlag+1) x Nf/factor row-major).  Zero mean, unit variance for an exponential(1)
   background; a tone drifting r channels per step shows up at lags floor(r) and ceil(r).
   compress as for fdr_propose_features. */
int fdr_propose_lag_features(const float* spectrogram, int64_t Nf, int64_t Nt, int factor,
                             int maxlag, int compress, float* out, fdr_stream_t stream);
/* Both in one pass: out rows 0..Nt-1 as fdr_propose_features, rows Nt..Nt+2*maxlag as
   fdr_propose_lag_features (the input of a network with nt = Nt + 2*maxlag + 1). */
int fdr_propose_input(const float* spectrogram, int64_t Nf, int64_t Nt, int factor, int maxlag,
                      int compress, float* out, fdr_stream_t stream);
/* logits[b][w] (device) for x[b][t][bin] (device), b < batch. */
int fdr_propose_forward(fdr_propose_net* net, const float* x, int batch, float* logits,
                        fdr_stream_t stream);
/* Mean binary cross-entropy with labels[b][w] in {0,1}; gradient of every parameter into
   grad_out (device, num_params floats; may be NULL) and the loss into loss_out (device). */
int fdr_propose_gradients(fdr_propose_net* net, const float* x, const float* labels, int batch,
                          float* logits, float* grad_out, float* loss_out, fdr_stream_t stream);
/* One Adam step (beta 0.9/0.999, eps 1e-8) at learning rate lr; deterministic. */
int fdr_propose_train_step(fdr_propose_net* net, const float* x, const float* labels, int batch,
                           float lr, float* logits, float* loss_out, fdr_stream_t stream);
/* Checkpoint state (HOST arrays of num_params floats): weights, Adam moments, step count. */
int fdr_propose_get_state(fdr_propose_net* net, float* params, float* m, float* v, int64_t* step);
int fdr_propose_set_state(fdr_propose_net* net, const float* params, const float* m, const float* v,
                          int64_t step);

/* ---------------------------------------------------------------------------------- */
/* intfdr.jl                                                                           */
/* ---------------------------------------------------------------------------------- */
/* intshift! (intfdr.jl:7-14): dout[:, t] = circshift(din[:, t], -round(rate*t)). */
int fdr_intshift(const float* din, int64_t Nf, int64_t Nt, double rate, int rate_type,
                 float* dout, fdr_stream_t stream);
/* intfdr! (intfdr.jl:34-45): fdr[n, j] = sum over t = 0..Nt-1, in t order from +0.0f, of
   spec[(n + round(rates[j]*t)) mod Nf, t].  `rates` is a HOST array of Nr values; the
   product rates[j]*t is formed in float64 (FDR_RATES_F64) or float32 (FDR_RATES_F32) and
   rounded to nearest, ties to even, as Julia's round does.  Bit-exact with the
   reference's CPU intfdr. */
int fdr_intfdr(const float* spec, int64_t Nf, int64_t Nt, const double* rates, int64_t Nr,
               int rate_type, float* fdr, fdr_stream_t stream);
/* intfdr! with caller-computed integer shifts: `shifts` is a HOST array of Nr*Nt int64
   (shift of rate j at time t at shifts[j*Nt + t]). */
int fdr_intfdr_shifts(const float* spec, int64_t Nf, int64_t Nt, const int64_t* shifts,
                      int64_t Nr, float* fdr, fdr_stream_t stream);
/* Taylor-tree integer FDR (the faster intfdr variant the reference's README.md:88-92
   mentions; no counterpart in the reference code).  Nt a power of two in [2, 64]; column d - dmin of
   fdr (device, Nf x (dmax-dmin+1) column-major) for each integer total drift d in
   [dmin, dmax] (|d| <= Nt-1, rate d/(Nt-1) channels per step) sums
   spec[(n + p_d(t)) mod Nf, t] along the tree path p_d: p_d = 0 for Nt = 1, and over 2L
   steps the path of drift floor(|d|/2) over the first L steps followed by the same path
   over the last L steps offset by ceil(|d|/2) (negated for d < 0).  d = 0 and |d| = Nt-1
   equal intfdr at rates 0 and +-1; float32 pairwise additions in a fixed order. */
int fdr_taylor_tree(const float* spectrogram, int64_t Nf, int64_t Nt, int dmin, int dmax,
                    float* fdr, fdr_stream_t stream);

/* ---------------------------------------------------------------------------------- */
/* fftfdr.jl                                                                           */
/* ---------------------------------------------------------------------------------- */
typedef struct fdr_fft_ws fdr_fft_ws;
/* fftfdr_workspace(spectrogram) (fftfdr.jl:39-59): holds rfft(spectrogram) (K x Nt). */
int fdr_fftfdr_workspace(fdr_fft_ws** ws, const float* spectrogram, int64_t Nf, int64_t Nt,
                         fdr_stream_t stream);
/* fftfdr_workspace! (fftfdr.jl:69-84): re-FFT a same-size spectrogram into ws. */
int fdr_fftfdr_workspace_update(fdr_fft_ws* ws, const float* spectrogram, int64_t Nf,
                                int64_t Nt, fdr_stream_t stream);
int fdr_fftfdr_destroy(fdr_fft_ws* ws);
/* Device pointer of ws.dest_rfft (K x Nt complex). */
int fdr_fftfdr_rfft_buffer(fdr_fft_ws* ws, void** F);
/* fdshiftsum! (fftfdr.jl:86-96): dest (Nf) = irfft(sum_t F .* phasor(rate)). */
int fdr_fdshiftsum(fdr_fft_ws* ws, float rate, float* dest, fdr_stream_t stream);
/* fdshift! (fftfdr.jl:104-111): de-Dopplered spectrogram dest (Nf x Nt). */
int fdr_fdshift(fdr_fft_ws* ws, float rate, float* dest, fdr_stream_t stream);
/* fftfdr! (fftfdr.jl:126-134): fdr[:, j] = fdshiftsum(rates[j]) for a HOST array of Nr
   float32 rates; fdr has leading dimension Nf. */
int fdr_fftfdr(fdr_fft_ws* ws, const float* rates, int64_t Nr, float* fdr,
               fdr_stream_t stream);

/* ---------------------------------------------------------------------------------- */
/* fdrutils.jl                                                                         */
/* ---------------------------------------------------------------------------------- */
/* fdrstats (fdrutils.jl:39-50) over nb matrices (HOST array of nb device pointers), each
   Nf x Nrb with leading dimension Nf: m = mean of column 1 of the first matrix,
   s = minimum over all columns of the corrected standard deviation (NaN if any is NaN).
   Computed in Float32 in the order of Julia's CPU code: each column is reduced by Base's
   pairwise mapreduce (blocks of at most 1024 elements summed sequentially, combined
   pairwise), mean = sum / Float32(Nf), variance = pairwise sum of abs2(x - mean) times
   Float32(1 // (Nf - 1)) (Statistics.varm!), std = sqrt.  Deterministic.  Julia's @simd
   block loop may reassociate on its host, so the reference's own last bits of m and s can
   differ from these on some CPUs.  Synchronises `stream` and writes the Float32 values as
   host doubles. */
int fdr_stats(const float* const* fdrs, int64_t nb, int64_t Nf, int64_t Nrb, double* m,
              double* s, fdr_stream_t stream);
/* fdrstats of a single FDR matrix without allocating device memory.  This entry point has
   no counterpart in the reference; it serves callers that must not allocate once they are
   running -- e.g. a real-time pipeline (an allocation can stall on the device or fail when
   memory is short) or a host whose device memory is entirely held by its own pool
   allocator.  Same results as fdr_stats for nb = 1, bit for bit (the same Float32 pairwise
   kernels).  Its scratch space is a fixed file-scope device array sized for at most
   FDR_STATS_NOALLOC_MAX_COLUMNS columns (16 bytes per column plus 32), which every GPU that
   loads the library keeps until the process exits; larger Nr is rejected with
   FDR_ERR_INVALID_ARGUMENT.  Every call writes all the scratch it reads, so no state carries
   over from the previous call.  All calls share that array: any two calls on one device
   whose work may interleave race -- calls on different streams, and calls that two host
   threads enqueue on the same stream -- so serialise the calls on the host.  The first call
   on a device (and CUDA context) looks up the array's device address
   (cudaGetSymbolAddress) with that device current; make that first call before any stream
   capture begins.  Synchronises `stream` and writes host doubles. */
#define FDR_STATS_NOALLOC_MAX_COLUMNS 8192
int fdr_stats_noalloc(const float* fdr, int64_t Nf, int64_t Nr, double* m, double* s,
                      fdr_stream_t stream);
/* fdrnormalize! (fdrutils.jl:70-90): x = (x - m) / s in float32 for nb matrices. */
int fdr_normalize(float* const* fdrs, int64_t nb, int64_t Nf, int64_t Nrb, float m, float s,
                  fdr_stream_t stream);
/* findprotohits (fdrutils.jl:148-169) over nb matrices treated as hcat'd: every (i, j)
   with fdr[i, j] >= threshold, in column-major (findall) order, written as ZERO-based
   int64 pairs hits[2*h] = i, hits[2*h+1] = j (buffer of 2*capacity int64: device memory,
   or mapped pinned host memory, which the kernels then write directly, with no copy;
   other host memory is rejected with FDR_ERR_INVALID_ARGUMENT).
   Each float32 element is compared with the float64 threshold (Julia promotes the
   Float32 element for `>=(threshold)` with a Float64 threshold).  snr = FDR_SNR_F64 or
   FDR_SNR_F32 replaces `threshold` by fdrdenormalize(threshold, fdrs) = threshold*s + m
   with fdr_stats's m and s, in Float64 or Float32 arithmetic as Julia promotes a Float64
   or an Int/Float32 snr.  Synchronises `stream`; *count (host) receives the
   total number of hits; if it exceeds `capacity`, the first `capacity` hits are written
   and FDR_ERR_CAPACITY is returned.  *threshold_used (host, may be NULL) receives the
   threshold compared against. */
int fdr_findprotohits(const float* const* fdrs, int64_t nb, int64_t Nf, int64_t Nrb,
                      double threshold, int snr, int64_t* hits, int64_t capacity,
                      int64_t* count, double* threshold_used, fdr_stream_t stream);

/* ---------------------------------------------------------------------------------- */
/* Proto-hits -> hits.  No counterpart in the reference: it is the step after           */
/* findprotohits that its README.md:57-66 places in DopplerDriftSearchTools.jl.           */
/* ---------------------------------------------------------------------------------- */
typedef struct fdr_hit_cluster {
  int64_t peak_i, peak_j; /* zero-based cell of the largest FDR value (first in column-major
                             order on ties; the first hit when no FDR is given) */
  float peak_value;       /* FDR value there (NaN when no FDR is given) */
  int32_t reserved;
  int64_t count;          /* proto-hits in the cluster */
  int64_t i_min, i_max, j_min, j_max; /* bounding box */
  int64_t first;          /* index into the hit list of the cluster's first hit */
} fdr_hit_cluster;

/* Connected components of the proto-hits `hits` (device, nhits (i, j) int64 pairs in the
   column-major order findprotohits returns; i < Nf, j < Nj) where two proto-hits touch
   when |i - i'| <= di and |j - j'| <= dj (no wrap-around).  Clusters are numbered in the
   order of their first proto-hit; labels (device, nhits int64, may be NULL) receive each
   proto-hit's cluster; clusters (device, capacity entries) their summaries, with peak
   values read from the FDR matrices fdrs[0..nb) of Nrb columns each (host array of device
   pointers, nb*Nrb == Nj; may be NULL).  Synchronises `stream`; *nclusters (host) receives
   the number of clusters; more than `capacity` returns FDR_ERR_CAPACITY (labels are still
   complete).  Unsorted or out-of-range hits return FDR_ERR_INVALID_ARGUMENT. */
int fdr_cluster_protohits(const int64_t* hits, int64_t nhits, int64_t Nf, int64_t Nj, int di,
                          int dj, const float* const* fdrs, int64_t nb, int64_t Nrb,
                          int64_t* labels, fdr_hit_cluster* clusters, int64_t capacity,
                          int64_t* nclusters, fdr_stream_t stream);

/* ---------------------------------------------------------------------------------- */
/* HDF5 filterbank ingest: rawspec's products store the (time, IF, channel) float32       */
/* dataset "data" in chunks filtered by bitshuffle with LZ4 (HDF5 filter 32008), which   */
/* test/heavytests.jl:11-14 reads through HDF5.jl + H5Zbitshuffle.jl.  These decode such  */
/* chunks; the HDF5 structure itself is parsed by the host binding.                       */
/* ---------------------------------------------------------------------------------- */
/* One LZ4 block (the LZ4 block format, no frame) from host src into host dst.  Malformed
   input (truncated sequences, offsets of 0 or before the start) or more than dst_capacity
   bytes of output return FDR_ERR_INVALID_ARGUMENT. */
int fdr_lz4_decompress(const uint8_t* src, int64_t src_size, uint8_t* dst, int64_t dst_capacity,
                       int64_t* dst_size);
/* Greedy LZ4 block encoder (host); dst_capacity >= src_size + src_size/255 + 16. */
int fdr_lz4_compress(const uint8_t* src, int64_t src_size, uint8_t* dst, int64_t dst_capacity,
                     int64_t* dst_size);
/* A bitshuffle+LZ4 chunk (host): its 12-byte header (big-endian uncompressed bytes and block
   bytes), the LZ4 blocks decompressed into out, which then holds each block's elements still
   bit-transposed, followed by the raw (elements mod 8) tail; *nbytes receives the
   uncompressed size, *block_elems the block length in elements (fdr_bitunshuffle's input). */
int fdr_bitshuffle_lz4_decode(const uint8_t* chunk, int64_t chunk_size, int elem_size, uint8_t* out,
                              int64_t out_capacity, int64_t* nbytes, int64_t* block_elems);
/* The inverse (host): bit-transposed blocks of block_elems elements (shuffled, nbytes) into a
   bitshuffle+LZ4 chunk. */
int fdr_bitshuffle_lz4_encode(const uint8_t* shuffled, int64_t nbytes, int elem_size,
                              int64_t block_elems, uint8_t* out, int64_t out_capacity,
                              int64_t* out_size);
/* Device: the bit transpose back to elements of nelem elements of elem_size bytes (1, 2, 4
   or 8) in blocks of block_elems (a multiple of 8; the last block holds the remaining whole
   groups of 8, the final nelem mod 8 elements are copied raw).  in and out are device
   buffers of nelem*elem_size bytes. */
int fdr_bitunshuffle(const uint8_t* in, int64_t nelem, int elem_size, int64_t block_elems,
                     uint8_t* out, fdr_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* FDR_B200_H */
