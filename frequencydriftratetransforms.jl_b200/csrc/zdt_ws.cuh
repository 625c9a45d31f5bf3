// ZDT workspace layout shared by the staged (zdt.cu) and fused (zdt_fused.cu) paths.
#pragma once
#include "fdr_internal.cuh"

struct fdr_zdt {
  int64_t Nf = 0, Nt = 0, Nr = 0, Nl = 0, K = 0;
  float r0 = 0.f, dr = 0.f;
  uint32_t flags = 0;
  std::vector<int64_t> factors;
  int device = 0;

  // Reference buffers (zdtfdr.jl:44-66): F is K x Nt, Y and V are K x Nl, column-major.
  float2* F = nullptr;
  float2* Y = nullptr;
  float2* V = nullptr;
  // Scratch for the real FFTs of the staged path.
  float2* rscratch = nullptr;
  int64_t rscratch_pairs = 0;

  // Fused path state (power-of-two Nf): see zdt_fused.cu.
  bool fused = false;
  int fP = 0, fQ = 0;            // Nf = fP * fQ four-step split
  float2* A = nullptr;           // input-stage intermediate, (Nt/2 rounded up) x fP x fQ
  float2* W = nullptr;           // inverse-stage intermediate for one chunk of rate pairs
  int64_t W_pairs = 0;           // rate pairs held by W
  void* fstate = nullptr;        // fused-path tables and sizes (zdt_fused.cu)
  bool A_valid = false;          // A holds the spectrogram last given to input!
  bool F_valid = false;          // F holds rfft of that spectrogram

  // Optional per-stage device timing of fdr_zdt_execute.
  bool timing = false;
  std::vector<cudaEvent_t> events;
  std::vector<const char*> ev_names;
  std::vector<float> stage_ms;
  std::vector<const char*> stage_names;

  int64_t bytes = 0;
};

namespace fdr {
// Staged stages (zdt.cu)
int zdt_stage_input(fdr_zdt* ws, const float* spec, cudaStream_t s);
int zdt_ensure_F(fdr_zdt* ws, cudaStream_t s);
// Fused path (zdt_fused.cu)
bool zdt_fused_eligible(int64_t Nf, int64_t Nt, int64_t Nr);
// log2 of P and Q of the fused split (Nf a power of two, zdt_fused_eligible true).
void fused_split_log2(int64_t Nf, int64_t Nt, int* Plog, int* Qlog);
int zdt_fused_setup(fdr_zdt* ws);
int zdt_fused_input(fdr_zdt* ws, const float* spec, cudaStream_t s);
int zdt_fused_A_to_F(fdr_zdt* ws, cudaStream_t s);
// acc (may be NULL): per-column float64 sum and sum of squares of dest are added into
// acc[2*j], acc[2*j+1] while dest is written.
int zdt_fused_run(fdr_zdt* ws, float r0, float* dest, int window, const double* custom_window,
                  double* acc, cudaStream_t s);
int zdt_staged_run(fdr_zdt* ws, float r0, float* dest, int window, const double* wk, double* acc,
                   cudaStream_t s);
void zdt_fused_release(fdr_zdt* ws);

// Fused kernels for one (Nf, Nt, Nr) shape with caller-owned intermediates (zdt_fused.cu).
struct FusedPlan;
int fused_plan_create(FusedPlan** out, int64_t N, int64_t Nt, int64_t Nr);
void fused_plan_destroy(FusedPlan* st);
int64_t fused_plan_table_bytes(const FusedPlan* st);
int64_t fused_A_elems(const FusedPlan* st);
int64_t fused_W_elems(const FusedPlan* st);
bool fused_phase_ok(const FusedPlan* st, float r0, float dr);
int fused_default_groups(const FusedPlan* st);
int fused_input(const FusedPlan* st, const float* spec, float2* A, cudaStream_t s);
int fused_a2f(const FusedPlan* st, const float2* A, float2* F, cudaStream_t s);
int fused_czt(const FusedPlan* st, const float2* A, float2* W, float r0, float dr, int window,
              const double* wk, int groups, cudaStream_t s);
int fused_czt_blocks(const FusedPlan* st, const float2* A, float2* W, float r0, float dr,
                     int window, const double* wk, const int* blk_base, int groups,
                     cudaStream_t s);
int fused_output(const FusedPlan* st, const float2* W, float* dest, double* acc, cudaStream_t s);
int fused_output_mixed(const FusedPlan* st, const float2* W, float* dest, double* acc, cudaStream_t s);
// Reads and clears the fused kernels' fault flag (a bounded TMA wait that ran out).
int fused_take_fault();
int bounded_wait_selftest(unsigned long long limit_ns, cudaStream_t s);
int zdt_fused_run_blocks(fdr_zdt* ws, const int* blk_base, int64_t nblocks, float* dest,
                         int window, const double* wk, double* acc, cudaStream_t s);
// timing helpers
void zdt_mark(fdr_zdt* ws, const char* name, cudaStream_t s);
}  // namespace fdr
