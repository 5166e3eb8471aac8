// Serving loop: resident meshes, HBM-budget admission and continuous batching
// of point and grid requests.  No counterpart in the reference, whose
// resident-structure API (build_sdf_acceleration / query_sdf, lib.rs:410-485)
// answers one call at a time on the caller's thread; this file is the server
// a caller would otherwise write around that API.
//
// Three worker threads, each on its own CUDA stream(s), so a slow step of one
// kind never holds up the others:
//  * uploads: copy a mesh, build its triangle records and LBVH on the device
//    and make it resident under a mesh id;
//  * points: each request is copied in, queried and copied out on one of a
//    pool of streams, so requests on different meshes overlap on the device;
//    completions are picked up from CUDA events;
//  * grids: kGridLanes lanes (a thread and a stream each) form waves from
//    the head of the grid queue: whenever a lane is free it takes the
//    waiting requests in arrival order, up to a wave's worth of cells (a
//    larger grid alone), and computes them as one batched job.  A request is
//    therefore admitted at the next wave boundary of any lane, and two waves
//    run on the device at once, each a persistent launch sized so that both
//    fit.  A grid's values in a wave are bit-identical to computing it alone,
//    and a point request runs exactly the kernels of m2s_query_sdf, so every
//    result is the same alone and in the mix.
//
// Admission: every request reserves an estimate of the device memory it will
// hold (workspace and outputs; a mesh's resident structure for an upload)
// against the server's budget and waits, in arrival order per kind, until the
// reservation fits.  A request that could never fit is refused with
// M2S_ERR_OUT_OF_MEMORY.  An upload that does not fit first evicts resident
// meshes that no queued or running request uses, least recently used first.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "m2s_internal.cuh"

using namespace m2s;

namespace {

using Clock = std::chrono::steady_clock;

enum Kind { kUpload = 0, kPoints = 1, kGrid = 2 };

struct Request {
  uint64_t ticket = 0;
  int kind = 0;
  uint32_t mesh_id = 0;
  uint64_t need = 0;  // reserved device bytes
  // upload
  std::vector<float> verts;
  std::vector<uint8_t> idx;
  uint64_t nv = 0, ni = 0;
  int bits = 0, topo = 0, accel = 0, sign = 0;
  // points
  const float* q = nullptr;
  uint64_t nq = 0;
  // grid
  GridDesc grid{};
  int grid_sign = 0;
  float* out = nullptr;
  uint64_t cells = 0;
  Clock::time_point t_submit, t_done;
  int status = -1;  // -1 while pending
};
using RequestP = std::shared_ptr<Request>;

struct MeshEntry {
  m2s_mesh* mesh = nullptr;  // null while its upload is pending
  uint64_t bytes = 0;
  uint64_t last_use = 0;
  int users = 0;  // queued or running requests
  bool failed = false;
};

// Device bytes a resident mesh holds: triangle records in both orders (48 B
// each) and 64-byte LBVH nodes; the build needs about as much again for a
// moment (vertices, indices, Morton keys, sort buffers).
uint64_t mesh_bytes(uint64_t tris, int accel) {
  return accel == M2S_ACCEL_NONE ? 48 * tris : 160 * tris;
}
uint64_t upload_bytes(uint64_t tris, uint64_t nv, uint64_t ni, int bits, int accel) {
  return 2 * mesh_bytes(tris, accel) + 12 * nv + ni * (bits / 8) + (1u << 20);
}
// A point request: queries in and results out (16 B), Morton keys and order
// with their sort buffers, and the continuation list of the two-pass query.
uint64_t point_bytes(uint64_t nq) { return 64 * nq + (1u << 20); }

// The serving wave size, and the lanes that run waves side by side.
constexpr uint64_t kServeWaveCells = 4ull << 20;
constexpr int kGridLanes = 2;
// Unless the tuning names a count, each lane's waves run fit / lanes
// propagation blocks per SM, where `fit` is how many fit on one SM, so the
// lanes' persistent launches fit on the device together.  A cooperative
// launch starts only once all of its blocks can be resident, so a wave that
// does not fit yet waits for room; it never runs partly resident.  Measured
// on B200 (C5 mix, 64 resident meshes, 200 requests per rate), 2 blocks per
// SM per lane against 1 (which kept room for point kernels): p50 / p99 at
// 100, 400 and 1,600 requests/s 2.0 / 13.8, 2.4 / 17.5, 16.8 / 173 ms against
// 2.6 / 22.0, 2.7 / 27.2, 19.1 / 247 ms, and at 1,600 requests/s 1,192
// against 959 M grid cells/s.
int serve_blocks_per_sm(int sign) { return std::max(1, propagate_blocks_per_sm(sign) / kGridLanes); }
// A wave that starts while every other lane is idle and no grid request
// waits runs on all but kAloneSpare of the blocks that fit per SM: at low
// rates most waves run alone, and a large grid then finishes about as fast
// as a plain call while the spare room keeps point kernels running beside
// it.  Measured (C5 mix, 200 requests per rate) p99 at 50 / 100 / 200 / 400
// requests/s: 11.1 / 10.0 / 17.3 / 28.4 ms, against 11.7 / 11.6 / 17.6 / 28.3
// with half-width lanes always and 10.2 / 12.2 / 16.8 / 28.5 with no spare
// block — differences near the noise of a 200-request p99.
constexpr int kAloneSpare = 1;
int alone_blocks_per_sm(int sign) {
  return std::max(serve_blocks_per_sm(sign), propagate_blocks_per_sm(sign) - kAloneSpare);
}

}  // namespace

struct m2s_server {
  int device = 0;
  uint64_t budget = 0;
  uint32_t n_streams = 4;

  std::mutex mu;
  std::condition_variable cv_work;   // a queue got work, or memory was released
  std::condition_variable cv_done;   // a request completed
  bool stop = false;
  uint64_t next_ticket = 1;
  uint32_t next_mesh = 1;
  uint64_t reserved = 0, peak = 0, clock = 0;
  std::map<uint64_t, RequestP> tickets;
  std::map<uint32_t, MeshEntry> meshes;
  std::deque<RequestP> q[3];
  // counters
  uint64_t completed[3] = {0, 0, 0}, failed = 0, grid_batches = 0, grid_batched = 0, max_batch = 0, evictions = 0;

  cudaStream_t s_upload = nullptr, s_grid[kGridLanes] = {};
  std::vector<cudaStream_t> s_points;
  std::thread th[2 + kGridLanes];  // uploads, points, grid lanes
  bool lane_busy[kGridLanes] = {};  // a lane runs a wave

  // ---- helpers (mu held) ----
  bool fits(uint64_t need) const { return reserved + need <= budget; }
  // The head of queue k can be taken now: its mesh is gone or failed (it
  // completes with an error), or its mesh is resident and it fits.
  bool head_ready(int k) const {
    if (q[k].empty()) return false;
    const RequestP& r = q[k].front();
    auto it = meshes.find(r->mesh_id);
    return it == meshes.end() || it->second.failed || (it->second.mesh && fits(r->need));
  }
  void reserve(uint64_t need) {
    reserved += need;
    peak = std::max(peak, reserved);
  }
  void finish(const RequestP& r, int status) {
    r->status = status;
    r->t_done = Clock::now();
    reserved -= r->need;
    r->need = 0;
    if (r->kind != kUpload) {
      auto it = meshes.find(r->mesh_id);
      if (it != meshes.end()) it->second.users--;
    }
    if (status == M2S_OK) completed[r->kind]++;
    else failed++;
    cv_done.notify_all();
    cv_work.notify_all();
  }
  // Frees idle meshes, least recently used first, until `need` more bytes fit.
  void evict_for(uint64_t need) {
    while (!fits(need)) {
      uint32_t victim = 0;
      uint64_t oldest = UINT64_MAX;
      for (auto& kv : meshes)
        if (kv.second.mesh && kv.second.users == 0 && kv.second.last_use < oldest) {
          oldest = kv.second.last_use;
          victim = kv.first;
        }
      if (!victim) return;
      MeshEntry e = meshes[victim];
      meshes.erase(victim);
      reserved -= e.bytes;
      delete e.mesh;  // nothing queued or running uses it; its buffers go back on the upload stream
      ++evictions;
    }
  }

  void upload_loop();
  void points_loop();
  void grid_loop(int lane);
};

void m2s_server::upload_loop() {
  cudaSetDevice(device);
  for (;;) {
    RequestP r;
    {
      std::unique_lock<std::mutex> lk(mu);
      cv_work.wait(lk, [&] { return stop || !q[kUpload].empty(); });
      if (stop) return;
      r = q[kUpload].front();
      q[kUpload].pop_front();
      // Make room from idle meshes; otherwise wait for running requests to
      // release memory (the request fits the budget, checked at submit).
      for (;;) {
        evict_for(r->need);
        if (fits(r->need) || stop) break;
        cv_work.wait(lk);
      }
      if (stop) return;
      reserve(r->need);
    }
    m2s_mesh* h = nullptr;
    int st = m2s_build_sdf_acceleration(r->verts.data(), r->nv, r->idx.empty() ? nullptr : r->idx.data(), r->ni,
                                        r->bits, r->topo, r->accel, r->sign, &h, s_upload);
    if (st == M2S_OK && !h) st = M2S_ERR_EMPTY_MESH;  // RtreeBvh on an empty mesh has no structure
    std::vector<float>().swap(r->verts);
    std::vector<uint8_t>().swap(r->idx);
    std::lock_guard<std::mutex> lk(mu);
    MeshEntry& e = meshes[r->mesh_id];
    if (st == M2S_OK) {
      e.mesh = h;
      e.bytes = mesh_bytes(h->mesh.n_tris, r->accel);
      e.last_use = ++clock;
      reserved += e.bytes;  // the mesh stays resident; the build reservation ends below
      peak = std::max(peak, reserved);
    } else {
      e.failed = true;
    }
    finish(r, st);
  }
}

namespace {
struct InFlight {
  RequestP r;
  DevBuf<float> dq, dout;
  cudaEvent_t ev = nullptr;
  uint32_t slot = 0;
};
}  // namespace

void m2s_server::points_loop() {
  cudaSetDevice(device);
  constexpr uint32_t kSlots = 4096;
  uint32_t* h_status = nullptr;
  uint32_t* d_status = nullptr;
  if (cudaHostAlloc((void**)&h_status, kSlots * 4, cudaHostAllocPortable) != cudaSuccess ||
      cudaMalloc((void**)&d_status, kSlots * 4) != cudaSuccess) {
    cudaGetLastError();
    if (h_status) cudaFreeHost(h_status);
    std::lock_guard<std::mutex> lk(mu);
    stop = true;
    cv_work.notify_all();
    return;
  }
  std::vector<cudaEvent_t> free_events;
  std::deque<std::unique_ptr<InFlight>> flying;
  uint32_t next_stream = 0, next_slot = 0;
  for (;;) {
    std::vector<std::pair<RequestP, m2s_mesh*>> go;
    {
      std::unique_lock<std::mutex> lk(mu);
      if (flying.empty()) cv_work.wait(lk, [&] { return stop || head_ready(kPoints); });
      if (stop) break;
      // Admit in arrival order; a request whose mesh is still uploading, or
      // that does not fit yet, waits and so do the ones behind it.
      while (!q[kPoints].empty() && flying.size() + go.size() < kSlots) {
        RequestP r = q[kPoints].front();
        auto it = meshes.find(r->mesh_id);
        if (it == meshes.end() || it->second.failed) {
          q[kPoints].pop_front();
          finish(r, M2S_ERR_INVALID_ARGUMENT);
          continue;
        }
        if (!it->second.mesh || !fits(r->need)) break;
        q[kPoints].pop_front();
        reserve(r->need);
        it->second.last_use = ++clock;
        go.emplace_back(r, it->second.mesh);
      }
    }
    for (auto& g : go) {
      RequestP r = g.first;
      m2s_mesh* m = g.second;
      int st = M2S_OK;
      if (m->mesh.n_tris == 0 && m->accel != M2S_ACCEL_NONE) st = M2S_ERR_EMPTY_MESH;  // rtree.rs:148
      if (st) {
        std::lock_guard<std::mutex> lk(mu);
        finish(r, st);
        continue;
      }
      auto f = std::make_unique<InFlight>();
      f->r = r;
      f->slot = next_slot++ % kSlots;
      cudaStream_t s = s_points[next_stream++ % s_points.size()];
      if (free_events.empty()) {
        cudaEvent_t e;
        cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
        free_events.push_back(e);
      }
      f->ev = free_events.back();
      free_events.pop_back();
      st = f->dq.alloc(3 * r->nq, s);
      if (!st) st = f->dout.alloc(r->nq, s);
      if (!st && cudaMemsetAsync(d_status + f->slot, 0, 4, s) != cudaSuccess) st = M2S_ERR_CUDA;
      if (!st && cudaMemcpyAsync(f->dq.p, r->q, 12 * r->nq, cudaMemcpyHostToDevice, s) != cudaSuccess) st = M2S_ERR_CUDA;
      if (!st)
        st = query_points(m->mesh.view(), m->accel, m->sign, f->dq.p, r->nq, f->dout.p, nullptr, nullptr,
                          d_status + f->slot, s);
      if (!st && cudaMemcpyAsync(r->out, f->dout.p, 4 * r->nq, cudaMemcpyDeviceToHost, s) != cudaSuccess) st = M2S_ERR_CUDA;
      if (!st && cudaMemcpyAsync(h_status + f->slot, d_status + f->slot, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess)
        st = M2S_ERR_CUDA;
      if (!st && cudaEventRecord(f->ev, s) != cudaSuccess) st = M2S_ERR_CUDA;
      if (st) {
        cudaStreamSynchronize(s);
        free_events.push_back(f->ev);
        std::lock_guard<std::mutex> lk(mu);
        finish(r, st);
        continue;
      }
      flying.push_back(std::move(f));
    }
    // Completions, in any order.
    bool any = false;
    for (auto it = flying.begin(); it != flying.end();) {
      cudaError_t e = cudaEventQuery((*it)->ev);
      if (e == cudaErrorNotReady) {
        ++it;
        continue;
      }
      const int st = e == cudaSuccess ? status_from_bits(h_status[(*it)->slot]) : cuda_fail(e, "point request");
      free_events.push_back((*it)->ev);
      RequestP r = (*it)->r;
      it = flying.erase(it);  // frees the request's buffers on its stream
      std::lock_guard<std::mutex> lk(mu);
      finish(r, st);
      any = true;
    }
    if (!flying.empty() && !any && go.empty()) std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
  for (auto& f : flying) cudaEventSynchronize(f->ev);
  flying.clear();
  cudaDeviceSynchronize();
  for (auto e : free_events) cudaEventDestroy(e);
  cudaFreeHost(h_status);
  cudaFree(d_status);
}

void m2s_server::grid_loop(int lane) {
  cudaSetDevice(device);
  cudaStream_t s = s_grid[lane];
  uint32_t* h_status = nullptr;
  cudaHostAlloc((void**)&h_status, 4, cudaHostAllocPortable);
  for (;;) {
    std::vector<RequestP> wave;
    std::vector<MeshView> views;
    GridTuning tune = grid_tuning();
    tune.wave_cells = std::min<uint64_t>(tune.wave_cells ? tune.wave_cells : kServeWaveCells, kServeWaveCells);
    uint64_t cells = 0;
    bool alone = false;
    {
      std::unique_lock<std::mutex> lk(mu);
      cv_work.wait(lk, [&] { return stop || head_ready(kGrid); });
      if (stop) break;
      // The waiting requests join this wave in arrival order, up to a
      // wave's worth of cells (a larger grid alone); later ones wait for
      // the next free lane.
      while (!q[kGrid].empty()) {
        RequestP r = q[kGrid].front();
        auto it = meshes.find(r->mesh_id);
        if (it == meshes.end() || it->second.failed) {
          q[kGrid].pop_front();
          finish(r, M2S_ERR_INVALID_ARGUMENT);
          continue;
        }
        if (!it->second.mesh || !fits(r->need)) break;
        if (!wave.empty() && r->grid_sign != wave.front()->grid_sign) break;  // one sign per wave
        if (!wave.empty() && cells + r->cells > tune.wave_cells) break;
        q[kGrid].pop_front();
        reserve(r->need);
        it->second.last_use = ++clock;
        wave.push_back(r);
        views.push_back(it->second.mesh->mesh.view());
        cells += r->cells;
      }
      if (!wave.empty()) {
        alone = q[kGrid].empty();
        for (int l = 0; l < kGridLanes; ++l)
          if (l != lane && lane_busy[l]) alone = false;
        lane_busy[lane] = true;
        ++grid_batches;
        grid_batched += wave.size();
        max_batch = std::max<uint64_t>(max_batch, wave.size());
      }
    }
    if (wave.empty()) continue;
    if (tune.blocks_per_sm <= 0)
      tune.blocks_per_sm = alone ? alone_blocks_per_sm(wave.front()->grid_sign) : serve_blocks_per_sm(wave.front()->grid_sign);
    std::vector<GridDesc> grids;
    for (auto& r : wave) grids.push_back(r->grid);
    tune.wave_cells = std::max<uint64_t>(cells, 1);  // the whole wave is one job
    int st = M2S_OK;
    {
      DevBuf<float> dout;
      DevBuf<uint32_t> dst;
      if (!(st = dout.alloc(cells, s)) && !(st = dst.alloc(1, s))) {
        if (cudaMemsetAsync(dst.p, 0, 4, s) != cudaSuccess) st = M2S_ERR_CUDA;
        if (!st)
          st = grid_sdf_batch(views.data(), (uint32_t)wave.size(), grids.data(), wave.front()->grid_sign, dout.p,
                              dst.p, s, nullptr, nullptr, tune);
        uint64_t off = 0;
        for (const RequestP& r : wave) {
          if (!st && cudaMemcpyAsync(r->out, dout.p + off, 4 * r->cells, cudaMemcpyDeviceToHost, s) != cudaSuccess)
            st = M2S_ERR_CUDA;
          off += r->cells;
        }
        if (!st && cudaMemcpyAsync(h_status, dst.p, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess) st = M2S_ERR_CUDA;
        if (cudaStreamSynchronize(s) != cudaSuccess && !st) st = M2S_ERR_CUDA;
        if (!st) st = status_from_bits(*h_status);
      }
    }
    std::lock_guard<std::mutex> lk(mu);
    lane_busy[lane] = false;
    for (const RequestP& r : wave) finish(r, st);
  }
  cudaStreamSynchronize(s);
  cudaFreeHost(h_status);
}

namespace {

// Device bytes of a grid request: its share of the batch output (4 B/cell)
// and the workspace of a job of its own size (keys, bucket lists, touched
// lists, ray bits).  A wave's workspace never exceeds the sum of these over
// its grids (list capacity grows at most linearly with the cells), and waves
// run one at a time, so the sum over a batch bounds what the batch holds.
uint64_t grid_bytes(uint64_t cells) { return 4 * cells + grid_job_bytes(cells); }

int submit(m2s_server* S, RequestP r, uint64_t* ticket) {
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->stop) return M2S_ERR_INVALID_ARGUMENT;
  if (r->need > S->budget) {
    set_error("the request needs more device memory than the server's whole budget");
    return M2S_ERR_OUT_OF_MEMORY;
  }
  r->ticket = S->next_ticket++;
  r->t_submit = Clock::now();
  if (r->kind != kUpload) {
    auto it = S->meshes.find(r->mesh_id);
    if (it == S->meshes.end() || it->second.failed) return M2S_ERR_INVALID_ARGUMENT;
    it->second.users++;
  }
  S->tickets[r->ticket] = r;
  S->q[r->kind].push_back(r);
  *ticket = r->ticket;
  S->cv_work.notify_all();
  return M2S_OK;
}

}  // namespace

extern "C" {

int m2s_server_create(uint64_t hbm_budget_bytes, uint32_t point_streams, m2s_server** out) {
  if (!out) return M2S_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int st;
  if ((st = require_device())) return st;
  m2s_server* S = new m2s_server();
  cudaGetDevice(&S->device);
  S->budget = hbm_budget_bytes;
  S->n_streams = std::max<uint32_t>(1, std::min<uint32_t>(point_streams ? point_streams : 4, 32));
  bool ok = cudaStreamCreateWithFlags(&S->s_upload, cudaStreamNonBlocking) == cudaSuccess;
  for (int l = 0; ok && l < kGridLanes; ++l)
    ok = cudaStreamCreateWithFlags(&S->s_grid[l], cudaStreamNonBlocking) == cudaSuccess;
  for (uint32_t i = 0; ok && i < S->n_streams; ++i) {
    cudaStream_t s;
    ok = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess;
    if (ok) S->s_points.push_back(s);
  }
  if (!ok) {
    st = cuda_fail(cudaGetLastError(), "cudaStreamCreateWithFlags");
    for (auto s : S->s_points) cudaStreamDestroy(s);
    if (S->s_upload) cudaStreamDestroy(S->s_upload);
    for (auto g : S->s_grid)
      if (g) cudaStreamDestroy(g);
    delete S;
    return st;
  }
  {
    // Grow the device memory pool once, up front: growing it while requests
    // run (new physical memory for a larger working set) stalled every worker
    // for tens to hundreds of milliseconds now and then.  The pool keeps what
    // it reserved, so later allocations are carved from this.
    const uint64_t reserve = std::min<uint64_t>(hbm_budget_bytes / 2, 16ull << 30);
    void* p = nullptr;
    if (reserve && dev_alloc(&p, reserve, S->s_upload) == M2S_OK) {
      dev_free(p, S->s_upload);
      cudaStreamSynchronize(S->s_upload);
    }
  }
  S->th[kUpload] = std::thread([S] { S->upload_loop(); });
  S->th[kPoints] = std::thread([S] { S->points_loop(); });
  for (int l = 0; l < kGridLanes; ++l) S->th[2 + l] = std::thread([S, l] { S->grid_loop(l); });
  *out = S;
  return M2S_OK;
}

void m2s_server_free(m2s_server* S) {
  if (!S) return;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
    S->cv_work.notify_all();
  }
  for (auto& t : S->th)
    if (t.joinable()) t.join();
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(S->device);
  cudaDeviceSynchronize();
  for (auto& kv : S->meshes) delete kv.second.mesh;
  S->meshes.clear();
  cudaStreamSynchronize(S->s_upload);
  for (auto s : S->s_points) cudaStreamDestroy(s);
  cudaStreamDestroy(S->s_upload);
  for (auto g : S->s_grid) cudaStreamDestroy(g);
  cudaSetDevice(prev);
  delete S;
}

int m2s_server_submit_upload(m2s_server* S, const float* vertices, uint64_t nv, const void* indices, uint64_t ni,
                             int bits, int topo, int accel, int sign, uint32_t* mesh_id, uint64_t* ticket) {
  if (!S || !mesh_id || !ticket) return M2S_ERR_INVALID_ARGUMENT;
  if (accel < M2S_ACCEL_NONE || accel > M2S_ACCEL_RTREE_BVH || sign < 0 || sign > 1) return M2S_ERR_INVALID_ARGUMENT;
  if (bits != M2S_INDEX_NONE && bits != M2S_INDEX_U16 && bits != M2S_INDEX_U32) return M2S_ERR_INVALID_ARGUMENT;
  if (topo != M2S_TOPOLOGY_TRIANGLE_LIST && topo != M2S_TOPOLOGY_TRIANGLE_STRIP) return M2S_ERR_INVALID_ARGUMENT;
  if ((nv && !vertices) || (bits != M2S_INDEX_NONE && ni && !indices)) return M2S_ERR_INVALID_ARGUMENT;
  const uint64_t n = bits == M2S_INDEX_NONE ? nv : ni;
  if (topo == M2S_TOPOLOGY_TRIANGLE_LIST && n % 3) return M2S_ERR_INDEX_COUNT;  // lib.rs:203, lib.rs:207
  const uint64_t tris = topo == M2S_TOPOLOGY_TRIANGLE_LIST ? n / 3 : (n >= 3 ? n - 2 : 0);
  auto r = std::make_shared<Request>();
  r->kind = kUpload;
  r->verts.assign(vertices, vertices + 3 * nv);
  if (bits != M2S_INDEX_NONE && ni) {
    const uint8_t* p = (const uint8_t*)indices;
    r->idx.assign(p, p + ni * (bits / 8));
  }
  r->nv = nv;
  r->ni = ni;
  r->bits = bits;
  r->topo = topo;
  r->accel = accel;
  r->sign = sign;
  r->need = upload_bytes(tris, nv, ni, bits, accel);
  {
    std::lock_guard<std::mutex> lk(S->mu);
    r->mesh_id = S->next_mesh++;
    S->meshes[r->mesh_id] = MeshEntry{};
  }
  *mesh_id = r->mesh_id;
  int st = submit(S, r, ticket);
  if (st) {
    std::lock_guard<std::mutex> lk(S->mu);
    S->meshes.erase(r->mesh_id);
  }
  return st;
}

int m2s_server_submit_points(m2s_server* S, uint32_t mesh_id, const float* q, uint64_t nq, float* out,
                             uint64_t* ticket) {
  if (!S || !ticket || (nq && (!q || !out))) return M2S_ERR_INVALID_ARGUMENT;
  if (nq > 0xFFFFFFFFull) return M2S_ERR_INVALID_ARGUMENT;
  for (uint64_t i = 0; i < 3 * nq; ++i)
    if (!std::isfinite(q[i])) return M2S_ERR_NONFINITE_QUERY;  // lib.rs:374-376
  auto r = std::make_shared<Request>();
  r->kind = kPoints;
  r->mesh_id = mesh_id;
  r->q = q;
  r->nq = nq;
  r->out = out;
  r->need = point_bytes(nq);
  return submit(S, r, ticket);
}

int m2s_server_submit_grid(m2s_server* S, uint32_t mesh_id, const float first_cell[3], const float cell_size[3],
                           const uint64_t cell_count[3], int sign, float* out, uint64_t* ticket) {
  if (!S || !ticket || !first_cell || !cell_size || !cell_count || !out || sign < 0 || sign > 1)
    return M2S_ERR_INVALID_ARGUMENT;
  auto r = std::make_shared<Request>();
  r->kind = kGrid;
  r->mesh_id = mesh_id;
  for (int d = 0; d < 3; ++d) {
    r->grid.first[d] = first_cell[d];
    r->grid.size[d] = cell_size[d];
    r->grid.n[d] = cell_count[d];
  }
  int st = check_grid(r->grid);
  if (st) return st;
  r->grid_sign = sign;
  r->out = out;
  r->cells = r->grid.cells();
  r->need = grid_bytes(r->cells);
  return submit(S, r, ticket);
}

int m2s_server_wait(m2s_server* S, uint64_t ticket, double timeout_s, int* status, double* latency_s) {
  if (!S) return M2S_ERR_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->tickets.find(ticket);
  if (it == S->tickets.end()) return M2S_ERR_INVALID_ARGUMENT;
  RequestP r = it->second;
  auto done = [&] { return r->status >= 0; };
  if (timeout_s < 0) {
    S->cv_done.wait(lk, done);
  } else if (!S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done)) {
    return M2S_ERR_LIMIT;  // still pending; the ticket stays valid
  }
  if (status) *status = r->status;
  if (latency_s) *latency_s = std::chrono::duration<double>(r->t_done - r->t_submit).count();
  S->tickets.erase(it);
  return M2S_OK;
}

int m2s_server_remove_mesh(m2s_server* S, uint32_t mesh_id) {
  if (!S) return M2S_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->meshes.find(mesh_id);
  if (it == S->meshes.end() || !it->second.mesh || it->second.users) return M2S_ERR_INVALID_ARGUMENT;
  S->reserved -= it->second.bytes;
  delete it->second.mesh;
  S->meshes.erase(it);
  S->cv_work.notify_all();
  return M2S_OK;
}

int m2s_server_stats(m2s_server* S, uint64_t out[12]) {
  if (!S || !out) return M2S_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(S->mu);
  uint64_t resident = 0, queued = 0;
  for (auto& kv : S->meshes) resident += kv.second.mesh ? 1 : 0;
  for (auto& qq : S->q) queued += qq.size();
  const uint64_t v[12] = {S->completed[kUpload], S->completed[kPoints], S->completed[kGrid], S->failed,
                          S->grid_batches,       S->grid_batched,       S->max_batch,        S->reserved,
                          S->peak,               resident,              queued,              S->evictions};
  for (int i = 0; i < 12; ++i) out[i] = v[i];
  return M2S_OK;
}

}  // extern "C"
