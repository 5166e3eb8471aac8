// Batched grids, grid plans (CUDA graphs) and the grid autotuner.  None of
// these has a counterpart in the reference, which computes one grid per call
// (generate/grid.rs:265-378); they exist so many (mesh, grid) requests share
// one persistent propagation launch instead of paying its fixed cost —
// rounds that each end in a grid-wide barrier — once per grid.
//
// A job (GridJob) computes several grids in one set of launches.  Every
// grid's states are relaxed in the rounds of their own distance buckets
// whatever else is in the job, so each grid's output is bit-identical to
// computing it alone; a job takes as many rounds as its slowest grid.
//
// A batch runs as waves: jobs of at most wave_cells cells (128M by default; a
// larger grid alone), packed largest grid first.  Grids that share a job
// share its rounds and barriers, so the more a job holds the fewer rounds the
// batch pays for, until a job's keys and lists outgrow the L2 cache so far
// that each round's accesses slow down (256 grids, 547M cells: 64M-cell waves
// 306 ms, 128M 297 ms, 256M 321 ms, one job 438 ms), while a plan's
// autotuning, which times one wave per class, grows (6.5 s at 64M, 11.6 s at
// 128M).
//
// A plan captures every wave's whole pipeline (memsets, seeding, collection,
// the cooperative propagation kernel, rays, finalisation) into one CUDA graph
// once and replays it.  Its workspace is allocated on a stream the plan owns
// and kept until the plan is freed.
//
// The autotuner times a plan at several cooperative grid sizes — the one knob
// that moves propagation time most: more blocks relax big buckets faster, but
// every round ends in a barrier whose cost grows with the block count — and
// keeps the fastest, timing one wave per class of waves (device, sign, one
// grid or several, log2 of the cell count).  The choice is cached per class
// and reused by later plans.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "m2s_internal.cuh"

using namespace m2s;

namespace {

int read_grids(uint32_t n, const float* first, const float* size, const uint64_t* count, std::vector<GridDesc>* out) {
  if (!first || !size || !count) return M2S_ERR_INVALID_ARGUMENT;
  out->resize(n);
  for (uint32_t k = 0; k < n; ++k) {
    GridDesc& g = (*out)[k];
    for (int d = 0; d < 3; ++d) {
      g.first[d] = first[3 * k + d];
      g.size[d] = size[3 * k + d];
      g.n[d] = count[3 * k + d];
    }
    int st = check_grid(g);
    if (st) {
      set_error("grid " + std::to_string(k) + ": cell counts must be non-zero and give fewer than 2^32 - 1 cells");
      return st;
    }
  }
  return M2S_OK;
}

int read_meshes(const m2s_mesh* const* meshes, uint32_t n, std::vector<MeshView>* out) {
  if (!meshes) return M2S_ERR_INVALID_ARGUMENT;
  int dev = 0;
  cudaGetDevice(&dev);
  out->resize(n);
  for (uint32_t k = 0; k < n; ++k) {
    if (!meshes[k]) return M2S_ERR_INVALID_ARGUMENT;
    if (meshes[k]->device != dev) {
      set_error("mesh " + std::to_string(k) + " lives on another device");
      return M2S_ERR_INVALID_ARGUMENT;
    }
    (*out)[k] = meshes[k]->mesh.view();
  }
  return M2S_OK;
}

std::mutex g_tune_mu;
std::map<uint64_t, unsigned> g_tuned_blocks;

uint64_t tune_key(const GridJob& job) {
  int dev = 0;
  cudaGetDevice(&dev);
  uint64_t lg = 0;
  while ((1ull << lg) < job.cells()) ++lg;
  return ((uint64_t)dev << 32) | ((uint64_t)job.sign() << 16) | ((uint64_t)(job.grids() > 1) << 8) | lg;
}

}  // namespace

struct m2s_grid_plan {
  int device = 0;
  cudaStream_t own = nullptr;  // allocation and capture stream
  std::vector<std::unique_ptr<GridJob>> jobs;  // one per wave
  cudaGraphExec_t exec = nullptr;
  uint64_t stats[kGridStats] = {};
  uint32_t restarts = 0;

  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
  }
  // Records every job's pipeline, one after the other, into one executable graph.
  int capture() {
    drop_graph();
    M2S_CUDA(cudaStreamBeginCapture(own, cudaStreamCaptureModeThreadLocal));
    int st = M2S_OK;
    for (auto& j : jobs)
      if ((st = j->enqueue(own, nullptr))) break;
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(own, &g);
    if (st) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    const cudaError_t ei = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
      exec = nullptr;
      return cuda_fail(ei, "cudaGraphInstantiate");
    }
    return M2S_OK;
  }
  // Launches the graph; if a job's lists overflowed, doubles them, re-captures
  // and launches again (every job starts from scratch, so results are unaffected).
  int run(cudaStream_t s) {
    int st;
    for (uint32_t attempt = 0;; ++attempt) {
      if (!exec && (st = capture())) return st;
      M2S_CUDA(cudaGraphLaunch(exec, s));
      uint64_t sum[kGridStats] = {};
      bool again = false;
      for (auto& j : jobs) {
        GridRunInfo info;
        if ((st = j->read_state(s, &info))) return st;
        sum[0] += info.seeds;
        sum[1] += info.rounds;
        sum[2] += info.entries;
        sum[3] += info.evals;
        sum[4] += info.ray_hits;
        sum[6] += info.launches;
        sum[7] += info.far_phases;
        sum[8] += info.solo_rounds;
        sum[9] = std::max<uint64_t>(sum[9], info.max_list);
        sum[10] += info.filter_same;
        sum[11] += info.filter_bound;
        for (int a = 0; a < 7; ++a) sum[12 + a] += info.audit[a];
        if (!info.overflow) continue;
        if (attempt >= 6 || j->capacity() >= 0x40000000u) {
          set_error("grid propagation lists overflowed at the largest capacity");
          return M2S_ERR_LIMIT;
        }
        j->set_capacity(j->capacity() * 2);
        if ((st = j->alloc_lists(own))) return st;
        again = true;
      }
      if (!again) {
        sum[5] = restarts;
        for (int i = 0; i < kGridStats; ++i) stats[i] = sum[i];
        return M2S_OK;
      }
      M2S_CUDA(cudaStreamSynchronize(own));
      drop_graph();
      ++restarts;
    }
  }
  ~m2s_grid_plan() {
    drop_graph();
    cudaDeviceSynchronize();  // replays on other streams may still read the workspace
  }
};

extern "C" {

int m2s_grid_sdf_batch_device(const m2s_mesh* const* meshes, uint32_t n_grids, const float* first_cells,
                              const float* cell_sizes, const uint64_t* cell_counts, int sign, float* d_out,
                              uint32_t* d_status, void* stream) {
  if (sign < 0 || sign > 1) return M2S_ERR_INVALID_ARGUMENT;
  if (n_grids == 0) return M2S_OK;
  int st;
  if ((st = require_device())) return st;
  std::vector<GridDesc> grids;
  std::vector<MeshView> views;
  if ((st = read_grids(n_grids, first_cells, cell_sizes, cell_counts, &grids))) return st;
  if ((st = read_meshes(meshes, n_grids, &views))) return st;
  if (!d_out) return M2S_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  DevBuf<uint32_t> own;
  if (!d_status) {
    if ((st = own.alloc(1, s))) return st;
    M2S_CUDA(cudaMemsetAsync(own.p, 0, 4, s));
    d_status = own.p;
  }
  uint64_t stats[kGridStats] = {};
  st = grid_sdf_batch(views.data(), n_grids, grids.data(), sign, d_out, d_status, s, stats, grid_phase_slot(),
                      grid_tuning());
  record_grid_stats(stats);
  return st;
}

int m2s_grid_plan_create(const m2s_mesh* const* meshes, uint32_t n_grids, const float* first_cells,
                         const float* cell_sizes, const uint64_t* cell_counts, int sign, float* d_out,
                         uint32_t* d_status, void* stream, m2s_grid_plan** out_plan) {
  (void)stream;
  if (!out_plan) return M2S_ERR_INVALID_ARGUMENT;
  *out_plan = nullptr;
  if (sign < 0 || sign > 1 || n_grids == 0 || !d_out || !d_status) return M2S_ERR_INVALID_ARGUMENT;
  int st;
  if ((st = require_device())) return st;
  std::vector<GridDesc> grids;
  std::vector<MeshView> views;
  if ((st = read_grids(n_grids, first_cells, cell_sizes, cell_counts, &grids))) return st;
  if ((st = read_meshes(meshes, n_grids, &views))) return st;
  m2s_grid_plan* P = new m2s_grid_plan();
  cudaGetDevice(&P->device);
  cudaError_t e = cudaStreamCreateWithFlags(&P->own, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete P;
    return cuda_fail(e, "cudaStreamCreateWithFlags");
  }
  auto fail = [&](int code) {
    cudaStream_t own = P->own;
    delete P;  // frees the workspace on `own`
    cudaStreamSynchronize(own);
    cudaStreamDestroy(own);
    return code;
  };
  if ((st = prepare_waves(views.data(), n_grids, grids.data(), sign, d_out, d_status, P->own, grid_tuning(),
                          &P->jobs)))
    return fail(st);
  for (auto& j : P->jobs) {
    if ((st = j->alloc_lists(P->own))) return fail(st);
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tuned_blocks.find(tune_key(*j));
    if (it != g_tuned_blocks.end()) j->set_cooperative_blocks(it->second);
  }
  e = cudaStreamSynchronize(P->own);
  if (e != cudaSuccess) return fail(cuda_fail(e, "cudaStreamSynchronize"));
  if ((st = P->capture())) return fail(st);
  *out_plan = P;
  return M2S_OK;
}

int m2s_grid_plan_run(m2s_grid_plan* plan, void* stream) {
  if (!plan) return M2S_ERR_INVALID_ARGUMENT;
  int st;
  if ((st = require_device())) return st;
  st = plan->run((cudaStream_t)stream);
  record_grid_stats(plan->stats);
  return st;
}

int m2s_grid_plan_autotune(m2s_grid_plan* plan, void* stream, uint32_t* out_blocks) {
  if (!plan) return M2S_ERR_INVALID_ARGUMENT;
  int st;
  if ((st = require_device())) return st;
  cudaStream_t s = (cudaStream_t)stream;
  if ((st = plan->run(s))) return st;  // settles every job's list capacity
  int dev = 0, sms = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaEvent_t e0, e1;
  M2S_CUDA(cudaEventCreate(&e0));
  M2S_CUDA(cudaEventCreate(&e1));
  struct EvFree {
    cudaEvent_t a, b;
    ~EvFree() {
      cudaEventDestroy(a);
      cudaEventDestroy(b);
    }
  } evf{e0, e1};
  // One job per class is timed (launched directly, not from the graph); the
  // choice applies to every job of the class and to later plans.
  std::map<uint64_t, unsigned> chosen;
  for (auto& jp : plan->jobs) {
    GridJob& job = *jp;
    const uint64_t key = tune_key(job);
    if (chosen.count(key)) continue;
    const unsigned most = job.max_cooperative_blocks();
    std::vector<unsigned> cand = {job.cooperative_blocks(), 16, 32, 64, (unsigned)sms / 2, (unsigned)sms,
                                  2u * sms, 3u * sms, most};
    std::sort(cand.begin(), cand.end());
    cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
    float best_ms = INFINITY;
    unsigned best = job.cooperative_blocks();
    for (unsigned c : cand) {
      if (c < 1 || c > most) continue;
      job.set_cooperative_blocks(c);
      if ((st = job.enqueue(s, nullptr))) return st;  // warm-up
      M2S_CUDA(cudaEventRecord(e0, s));
      for (int rep = 0; rep < 2; ++rep)
        if ((st = job.enqueue(s, nullptr))) return st;
      M2S_CUDA(cudaEventRecord(e1, s));
      M2S_CUDA(cudaEventSynchronize(e1));
      float ms = 0.0f;
      M2S_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (ms < best_ms) {
        best_ms = ms;
        best = c;
      }
    }
    chosen[key] = best;
  }
  for (auto& jp : plan->jobs) jp->set_cooperative_blocks(chosen[tune_key(*jp)]);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (auto& kv : chosen) g_tuned_blocks[kv.first] = kv.second;
  }
  plan->drop_graph();
  if ((st = plan->run(s))) return st;  // re-captures with the chosen shapes
  if (out_blocks) *out_blocks = plan->jobs.front()->cooperative_blocks();
  return M2S_OK;
}

uint64_t m2s_grid_plan_cells(const m2s_grid_plan* plan) {
  uint64_t n = 0;
  if (plan)
    for (auto& j : plan->jobs) n += j->cells();
  return n;
}
uint64_t m2s_grid_plan_device_bytes(const m2s_grid_plan* plan) {
  uint64_t n = 0;
  if (plan)
    for (auto& j : plan->jobs) n += j->device_bytes();
  return n;
}
uint32_t m2s_grid_plan_blocks(const m2s_grid_plan* plan) {
  return plan && !plan->jobs.empty() ? plan->jobs.front()->cooperative_blocks() : 0;
}
uint32_t m2s_grid_plan_waves(const m2s_grid_plan* plan) { return plan ? (uint32_t)plan->jobs.size() : 0; }

void m2s_grid_plan_free(m2s_grid_plan* plan) {
  if (!plan) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(plan->device);
  cudaStream_t own = plan->own;
  delete plan;
  cudaStreamSynchronize(own);
  cudaStreamDestroy(own);
  cudaSetDevice(prev);
}

void m2s_set_grid_tuning(int blocks_per_sm, uint32_t cells_per_block, uint64_t wave_cells, int solo_max) {
  GridTuning t = grid_tuning();
  t.blocks_per_sm = blocks_per_sm > 0 ? blocks_per_sm : 0;
  t.cells_per_block = cells_per_block ? cells_per_block : 1024;
  t.wave_cells = wave_cells ? wave_cells : (1ull << 27);
  t.solo_max = solo_max < 0 ? 64u : (uint32_t)solo_max;
  set_grid_tuning(t);
}

void m2s_set_fp64_audit(int enable) {
  GridTuning t = grid_tuning();
  t.fp64_audit = enable != 0;
  set_grid_tuning(t);
}

void m2s_set_grid_bound_filter(int enable) {
  GridTuning t = grid_tuning();
  t.bound_filter = enable != 0;
  set_grid_tuning(t);
}

void m2s_clear_grid_autotune(void) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tuned_blocks.clear();
}

}  // extern "C"
