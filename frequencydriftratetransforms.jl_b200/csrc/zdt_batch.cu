// Batched ZDT over many coarse channels of uneven shape (Nf, Nt, rates) in one CUDA-graph
// launch.  The reference processes one spectrogram per zdtfdr! call; a pipeline such as
// DopplerDriftSearchPipeline.jl loops over coarse channels (the reference's README.md:57-71).  Here the
// loop is captured once: channels are spread over `slots` streams forked from the caller's
// stream, each slot owning the fused path's intermediates (A, W) sized for the largest
// channel, channels of equal (Nf, Nt, Nr) share one FusedPlan (twiddle tables), and the
// whole batch replays with a single cudaGraphLaunch.  Channels the fused kernels do not
// cover (non-power-of-two Nf, Nt > 64, phases beyond 62 bits) run the staged kernels of a
// private workspace inside the same graph.
//
// Autotuning: for every distinct shape the czt kernel's rate-group split (grid.y) is timed
// over {1, 2, 4, 8} groups on that shape's first channel, then the number of active slots
// is timed over {1, 2, ..., slots} on the whole batch.  Results are cached per shape
// signature for the process.
#include <functional>
#include <map>
#include <mutex>
#include <string.h>
#include <tuple>

#include "zdt_ws.cuh"

using namespace fdr;

struct fdr_batch {
  struct Chan {
    fdr_batch_channel c;
    int plan = -1;            // index into plans, or -1 for the staged path
    fdr_zdt* staged = nullptr;
  };
  std::vector<Chan> ch;
  std::vector<FusedPlan*> plans;
  std::vector<std::tuple<int64_t, int64_t, int64_t>> plan_keys;  // (Nf, Nt, Nr) of each plan
  std::vector<int> groups;    // czt rate groups per plan (0: default)
  int nslots = 1, active = 1;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> joins;
  cudaEvent_t fork = nullptr;
  std::vector<float2*> A, W;
  int64_t maxA = 0, maxW = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int64_t bytes = 0;
  int device = 0;
};

namespace fdr {

using Sig = std::tuple<int, int64_t, int64_t, int64_t>;  // device, Nf, Nt, Nr
static std::mutex g_tune_mu;
static std::map<Sig, int> g_tuned_groups;

static void batch_release(fdr_batch* b) {
  if (!b) return;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (auto& c : b->ch)
    if (c.staged) fdr_zdt_destroy(c.staged);
  for (auto* p : b->plans) fused_plan_destroy(p);
  for (auto* a : b->A) cudaFree(a);
  for (auto* w : b->W) cudaFree(w);
  for (auto e : b->joins) cudaEventDestroy(e);
  if (b->fork) cudaEventDestroy(b->fork);
  for (auto s : b->streams) cudaStreamDestroy(s);
  delete b;
}

// Enqueue channel i on stream s (slot buffers of `slot`).
static int enqueue_channel(fdr_batch* b, size_t i, int slot, cudaStream_t s) {
  auto& c = b->ch[i];
  if (c.plan >= 0) {
    const FusedPlan* p = b->plans[c.plan];
    FDR_TRY(fused_input(p, c.c.spectrogram, b->A[slot], s));
    FDR_TRY(fused_czt(p, b->A[slot], b->W[slot], c.c.r0, c.c.dr, FDR_WINDOW_RECT, nullptr,
                      b->groups[c.plan], s));
    FDR_TRY(fused_output(p, b->W[slot], c.c.fdr, nullptr, s));
    return FDR_OK;
  }
  float* dest = c.c.fdr;
  return fdr_zdt_execute(c.staged, c.c.spectrogram, &c.c.r0, 1, &dest, FDR_WINDOW_RECT, nullptr,
                         (fdr_stream_t)s);
}

// Fork the active slot streams from s, enqueue every channel round-robin, join back into s.
static int enqueue_all(fdr_batch* b, cudaStream_t s) {
  const int k = std::max(1, std::min(b->active, b->nslots));
  FDR_CUDA(cudaEventRecord(b->fork, s));
  for (int j = 0; j < k; ++j) FDR_CUDA(cudaStreamWaitEvent(b->streams[j], b->fork, 0));
  for (size_t i = 0; i < b->ch.size(); ++i) {
    const int slot = (int)(i % k);
    FDR_TRY(enqueue_channel(b, i, slot, b->streams[slot]));
  }
  for (int j = 0; j < k; ++j) {
    FDR_CUDA(cudaEventRecord(b->joins[j], b->streams[j]));
    FDR_CUDA(cudaStreamWaitEvent(s, b->joins[j], 0));
  }
  return FDR_OK;
}

static int time_ms(cudaStream_t s, float* ms, const std::function<int()>& fn, int reps) {
  cudaEvent_t e0, e1;
  FDR_CUDA(cudaEventCreate(&e0));
  FDR_CUDA(cudaEventCreate(&e1));
  int st = fn();  // warm-up
  if (st == FDR_OK) {
    cudaEventRecord(e0, s);
    for (int r = 0; r < reps && st == FDR_OK; ++r) st = fn();
    cudaEventRecord(e1, s);
    cudaError_t e = cudaEventSynchronize(e1);
    if (e != cudaSuccess) st = cuda_status(e, "autotune timing");
    if (st == FDR_OK) {
      cudaEventElapsedTime(ms, e0, e1);
      *ms /= reps;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return st;
}

}  // namespace fdr

extern "C" {

int fdr_batch_create(fdr_batch** out, const fdr_batch_channel* channels, int64_t nch,
                     int slots, fdr_stream_t stream) {
  FDR_CHECK_ARG(out && channels && nch >= 1, "fdr_batch_create: bad arguments");
  FDR_CHECK_ARG(slots >= 1 && slots <= 16, "fdr_batch_create: slots must be 1..16");
  *out = nullptr;
  for (int64_t i = 0; i < nch; ++i) {
    const auto& c = channels[i];
    FDR_CHECK_ARG(c.spectrogram && c.fdr && c.Nf >= 1 && c.Nt >= 1 && c.Nr >= 1,
                  "fdr_batch_create: channel %lld is invalid", (long long)i);
    // the fused kernels move the spectrogram and the FDR in 8-byte pairs of floats
    FDR_CHECK_ARG(((reinterpret_cast<uintptr_t>(c.spectrogram) | reinterpret_cast<uintptr_t>(c.fdr)) & 7) == 0,
                  "fdr_batch_create: channel %lld: spectrogram and fdr must be 8-byte aligned",
                  (long long)i);
  }
  fdr_batch* b = new fdr_batch();
  cudaGetDevice(&b->device);
  b->nslots = b->active = slots;
  auto fail = [&](int st) { batch_release(b); return st; };
  std::map<std::tuple<int64_t, int64_t, int64_t>, int> plan_of;
  for (int64_t i = 0; i < nch; ++i) {
    fdr_batch::Chan c;
    c.c = channels[i];
    if (zdt_fused_eligible(c.c.Nf, c.c.Nt, c.c.Nr)) {
      auto key = std::make_tuple(c.c.Nf, c.c.Nt, c.c.Nr);
      auto it = plan_of.find(key);
      if (it == plan_of.end()) {
        FusedPlan* p = nullptr;
        int st = fused_plan_create(&p, c.c.Nf, c.c.Nt, c.c.Nr);
        if (st != FDR_OK) return fail(st);
        b->plans.push_back(p);
        b->plan_keys.push_back(key);
        b->groups.push_back(0);
        b->bytes += fused_plan_table_bytes(p);
        it = plan_of.emplace(key, (int)b->plans.size() - 1).first;
      }
      if (fused_phase_ok(b->plans[it->second], c.c.r0, c.c.dr)) {
        c.plan = it->second;
        b->maxA = std::max(b->maxA, fused_A_elems(b->plans[c.plan]));
        b->maxW = std::max(b->maxW, fused_W_elems(b->plans[c.plan]));
      }
    }
    if (c.plan < 0) {
      int st = fdr_zdt_create(&c.staged, nullptr, c.c.Nf, c.c.Nt, c.c.r0, c.c.dr, c.c.Nr, nullptr,
                              0, FDR_ZDT_STAGED_ONLY, stream);
      if (st != FDR_OK) return fail(st);
      fdr_zdt_info info;
      fdr_zdt_get_info(c.staged, &info);
      b->bytes += info.bytes;
    }
    b->ch.push_back(c);
  }
  cudaError_t e;
  if ((e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming)) != cudaSuccess)
    return fail(cuda_status(e, "cudaEventCreate"));
  for (int j = 0; j < slots; ++j) {
    cudaStream_t s;
    cudaEvent_t ev;
    if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) != cudaSuccess)
      return fail(cuda_status(e, "cudaStreamCreate"));
    b->streams.push_back(s);
    if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess)
      return fail(cuda_status(e, "cudaEventCreate"));
    b->joins.push_back(ev);
    float2 *A = nullptr, *W = nullptr;
    if (b->maxA > 0) {
      if ((e = cudaMalloc(&A, sizeof(float2) * b->maxA)) != cudaSuccess) return fail(cuda_status(e, "cudaMalloc(A)"));
      b->A.push_back(A);
      if ((e = cudaMalloc(&W, sizeof(float2) * b->maxW)) != cudaSuccess) return fail(cuda_status(e, "cudaMalloc(W)"));
      b->W.push_back(W);
      b->bytes += (int64_t)sizeof(float2) * (b->maxA + b->maxW);
    } else {
      b->A.push_back(nullptr);
      b->W.push_back(nullptr);
    }
  }
  // Cached tuning for known shapes.
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    for (size_t p = 0; p < b->plans.size(); ++p) {
      const auto& k = b->plan_keys[p];
      auto it = g_tuned_groups.find(Sig(b->device, std::get<0>(k), std::get<1>(k), std::get<2>(k)));
      if (it != g_tuned_groups.end()) b->groups[p] = it->second;
    }
  }
  *out = b;
  return FDR_OK;
}

int fdr_batch_destroy(fdr_batch* b) {
  if (b) {
    cudaDeviceSynchronize();
    batch_release(b);
  }
  return FDR_OK;
}

int fdr_batch_autotune(fdr_batch* b, fdr_stream_t stream) {
  FDR_CHECK_ARG(b != nullptr, "fdr_batch_autotune: NULL batch");
  cudaStream_t s = (cudaStream_t)stream;
  FDR_CHECK_ARG(b->exec == nullptr, "fdr_batch_autotune: tune before capturing");
  // 1. per shape: czt rate groups
  for (size_t p = 0; p < b->plans.size(); ++p) {
    size_t i0 = 0;
    while (i0 < b->ch.size() && b->ch[i0].plan != (int)p) ++i0;
    if (i0 == b->ch.size()) continue;
    const auto& c = b->ch[i0];
    const FusedPlan* plan = b->plans[p];
    FDR_TRY(fused_input(plan, c.c.spectrogram, b->A[0], s));
    int best = 0;
    float best_ms = 1e30f;
    const int cand[4] = {1, 2, 4, 8};
    for (int g : cand) {
      if (g > 1 && g > (int)cdiv(cdiv(c.c.Nr, 2), 4)) break;  // fewer than 4 pairs per group
      float ms = 0.f;
      FDR_TRY(time_ms(s, &ms, [&]() {
        return fused_czt(plan, b->A[0], b->W[0], c.c.r0, c.c.dr, FDR_WINDOW_RECT, nullptr, g, s);
      }, 3));
      if (ms < best_ms) { best_ms = ms; best = g; }
    }
    b->groups[p] = best;
    std::lock_guard<std::mutex> lock(g_tune_mu);
    const auto& key = b->plan_keys[p];
    g_tuned_groups[Sig(b->device, std::get<0>(key), std::get<1>(key), std::get<2>(key))] = best;
  }
  // 2. active slots
  int best_k = b->nslots;
  float best_ms = 1e30f;
  for (int k = 1; k <= b->nslots; k *= 2) {
    b->active = k;
    float ms = 0.f;
    FDR_TRY(time_ms(s, &ms, [&]() { return enqueue_all(b, s); }, 2));
    if (ms < best_ms) { best_ms = ms; best_k = k; }
  }
  b->active = best_k;
  return FDR_OK;
}

int fdr_batch_get_tuning(const fdr_batch* b, int* groups, int ngroups, int* nplans, int* active_slots) {
  FDR_CHECK_ARG(b != nullptr, "fdr_batch_get_tuning: NULL batch");
  if (nplans) *nplans = (int)b->plans.size();
  if (groups)
    for (int i = 0; i < ngroups && i < (int)b->groups.size(); ++i)
      groups[i] = b->groups[i] > 0 ? b->groups[i] : fused_default_groups(b->plans[i]);
  if (active_slots) *active_slots = b->active;
  return FDR_OK;
}

int fdr_batch_capture(fdr_batch* b, fdr_stream_t stream) {
  FDR_CHECK_ARG(b != nullptr, "fdr_batch_capture: NULL batch");
  FDR_CHECK_ARG(stream != nullptr, "fdr_batch_capture: capture needs a non-default stream");
  cudaStream_t s = (cudaStream_t)stream;
  if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
  if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
  // One eager pass first: first-use set-up (tables, attributes) must not happen in capture.
  FDR_TRY(enqueue_all(b, s));
  FDR_CUDA(cudaStreamSynchronize(s));
  FDR_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  int st = enqueue_all(b, s);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(s, &g);
  if (st != FDR_OK) { if (g) cudaGraphDestroy(g); return st; }
  if (e != cudaSuccess) return cuda_status(e, "cudaStreamEndCapture");
  b->graph = g;
  FDR_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
  return FDR_OK;
}

int fdr_batch_launch(fdr_batch* b, fdr_stream_t stream) {
  FDR_CHECK_ARG(b != nullptr, "fdr_batch_launch: NULL batch");
  cudaStream_t s = (cudaStream_t)stream;
  if (b->exec) {
    FDR_CUDA(cudaGraphLaunch(b->exec, s));
    return FDR_OK;
  }
  return enqueue_all(b, s);
}

int fdr_batch_info(const fdr_batch* b, int64_t* nchannels, int64_t* nfused, int64_t* bytes,
                   int* captured) {
  FDR_CHECK_ARG(b != nullptr, "fdr_batch_info: NULL batch");
  int64_t nf = 0;
  for (auto& c : b->ch) nf += (c.plan >= 0);
  if (nchannels) *nchannels = (int64_t)b->ch.size();
  if (nfused) *nfused = nf;
  if (bytes) *bytes = b->bytes;
  if (captured) *captured = b->exec != nullptr;
  return FDR_OK;
}

}  // extern "C"
