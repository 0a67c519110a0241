// bhr_engine.cpp -- many solves on one device, advanced together.
//
// The reference runs one solve per process (HighOrder/main.c:50-55 loops the
// m modes; TD_GPU_code/run.sh submits one job per trajectory).  The engine
// keeps every admitted solve's fields and tables resident, admits queued
// requests while the HBM budget allows, and advances all running solves with
// one launch per RK stage over a work-list of (solve, tile) pairs (one
// launch per group of up to kGroupSolves solves, whose stage arguments
// travel in the launch's parameters), captured as a CUDA graph.  Requests
// arriving while others run join at the next step boundary (continuous
// batching); finished solves leave with their waveform.  Each tile is
// computed by the same code as a lone solve, so a request's result does not
// depend on what it shares the GPU with.
//
// Host work per request (grid, tables, initial data, trajectory records,
// device allocations; waveform readback and release at the end) runs on a
// worker thread with its own streams and stream-ordered allocations, so the
// stepping thread only swaps prepared solves in and finished ones out.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "bhr.h"
#include "bhr_host.h"
#include "bhr_internal.h"
#include "bhr_solver_impl.h"

using namespace bhr;

namespace {

struct Request {
  int64_t id;
  bhr_params p;
  std::vector<double> traj;
  double t_submit;
};

struct Running {
  int64_t id;
  bhr_solver *s;
  double t_submit, t_start;
  int remaining;
};

struct Finished {
  int state = 3;  // 3 done, 4 failed
  int status = BHR_OK;
  std::string error;
  double t_submit = 0, t_start = 0, t_finish = 0;
  int steps = 0;
  std::vector<double> t, h, dedt;
};

double now_s() {
  using clk = std::chrono::steady_clock;
  static const clk::time_point t0 = clk::now();
  return std::chrono::duration<double>(clk::now() - t0).count();
}

// Device bytes a solve will hold (states, coefficient planes, tables, rows,
// source records), estimated before creating it.
size_t solve_bytes(const bhr_params &p, int traj_rows) {
  const size_t NM = static_cast<size_t>(p.N) * p.M;
  size_t b = NM * 8 * (12 + 1);  // u0, u1, u2 (4 planes each), bb
  if (p.precision == BHR_MIXED) b += NM * 4 * (4 + 4 + 4);  // delta1, eps2, FP32 coefficient planes
  b += static_cast<size_t>(CF_COUNT + 2) * p.N * 8 + static_cast<size_t>(RF_COUNT + 12) * p.M * 8;
  b += static_cast<size_t>(4) * p.PTSX * p.PTSY * 8;  // two source patch buffers
  if (traj_rows > 0 && p.dt > 0) b += static_cast<size_t>(p.T / p.dt + 2) * sizeof(StepRec);
  if (p.dt > 0 && p.Fr > 0) b += static_cast<size_t>(p.T / p.dt / p.Fr + 2) * (16 + 2 * p.M) * 8;  // rows, psi samples
  return b + (1 << 20);
}

}  // namespace

struct bhr_engine {
  int device = 0;
  size_t budget = 0;
  int tiling = kTilingBlock8n;  // stage tiling of the FP64 kernels (bhr_tiling values)
  int rows = 8;              // its tile height: every solve's tensor maps use it
  cudaStream_t stream = nullptr;
  // Requests and the worker (lock wmu): the queue, solves being prepared,
  // prepared solves waiting to join, finished solves waiting to be
  // released, and the bytes all of these and the running solves hold.
  std::mutex wmu;
  std::condition_variable wcv;   // worker: work arrived
  std::condition_variable rcv;   // stepping thread: a prepared solve arrived
  std::deque<Request> queue;
  std::unordered_set<int64_t> preparing;
  std::vector<Running> ready;
  std::vector<Running> to_release;
  int releasing = 0;  // finished solves being read back and released
  size_t used = 0;
  int64_t head_id = -1;   // the oldest queued request when it last did not fit
  int head_bypassed = 0;  // later requests prepared ahead of it since
  int64_t next_id = 1;
  bool stop = false;
  std::thread worker;
  // Results (lock dmu).
  std::mutex dmu;
  std::unordered_map<int64_t, Finished> done;
  int finished = 0;
  // Stepping state (lock mu).
  std::mutex mu;
  std::vector<Running> active;
  BatchSolve *d_solves = nullptr;
  ExtractArgs *d_ext = nullptr;
  SourceArgs *d_src = nullptr;
  MixedBatch *d_mixed = nullptr;  // mixed-precision solves' stage 2/3 tables
  int cap_solves = 0, ntiles = 0, nsrc = 0, max_ptsx = 1, max_ptsy = 1;
  // The work-lists, as launch groups: for FP64 stage s, groups64[s - 1]
  // (stage 1: every solve, FP64 solves first; stages 2 and 3: the FP64
  // solves); for the FP32 stages 2 and 3 of mixed solves, mixgroups[s - 2]
  // (kMixTileRows-high tiles).  ntiles counts every stage's tiles.
  std::vector<BatchGroup> groups64[3];
  std::vector<MixedGroup> mixgroups[2];
  int *d_err = nullptr;     // BHR_TIMEOUT from a bounded wait in a stage kernel
  cudaGraphExec_t graph = nullptr;  // one batch step
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool dirty = true;
  long long batch_steps = 0;
  double point_updates = 0.0;
  double device_ms = 0.0;
};

namespace {

int set_fail(int status, const std::string &msg) {
  set_error(msg);
  return status;
}

void release_tables(bhr_engine *e) {
  if (e->graph) cudaGraphExecDestroy(e->graph);
  e->graph = nullptr;
  for (void *q : {static_cast<void *>(e->d_solves), static_cast<void *>(e->d_ext), static_cast<void *>(e->d_src),
                  static_cast<void *>(e->d_mixed)})
    if (q) cudaFreeAsync(q, e->stream);
  e->d_solves = nullptr;
  e->d_ext = nullptr;
  e->d_src = nullptr;
  e->d_mixed = nullptr;
  e->cap_solves = 0;
}

// One batch step: sources of the sourced solves, three stages over the
// work-list, extraction of every solve.
int enqueue_batch_step(bhr_engine *e) {
  const int n = static_cast<int>(e->active.size());
  if (e->nsrc > 0) {
    cudaError_t err = launch_source_batch(e->d_src, e->nsrc, e->max_ptsy, e->max_ptsx, e->stream);
    if (err != cudaSuccess) return set_fail(BHR_CUDA_ERROR, std::string("source batch: ") + cudaGetErrorString(err));
  }
  // Stage 1 is FP64 for every solve; stages 2 and 3 run FP64 solves'
  // tiles through the FP64 kernels and mixed solves' tiles through the
  // FP32 ones.
  for (int stage = 1; stage <= 3; stage++) {
    cudaError_t err = cudaSuccess;
    for (const BatchGroup &g : e->groups64[stage - 1])
      if (err == cudaSuccess) err = launch_stage_batch(stage, e->tiling, e->d_solves, g, e->d_err, e->stream);
    if (stage > 1)
      for (const MixedGroup &g : e->mixgroups[stage - 2])
        if (err == cudaSuccess) err = launch_mixed_batch(stage, e->d_mixed, g, e->stream);
    if (err != cudaSuccess) return set_fail(BHR_CUDA_ERROR, std::string("stage batch: ") + cudaGetErrorString(err));
  }
  cudaError_t err = launch_extract_batch(e->d_ext, n, e->stream);
  if (err != cudaSuccess) return set_fail(BHR_CUDA_ERROR, std::string("extract batch: ") + cudaGetErrorString(err));
  return BHR_OK;
}

// Rebuilds the solve table, the work-list and the step graph after the set
// of running solves changed.
int rebuild(bhr_engine *e) {
  const int n = static_cast<int>(e->active.size());
  if (e->graph) {
    cudaGraphExecDestroy(e->graph);
    e->graph = nullptr;
  }
  e->dirty = false;
  if (n == 0) {
    e->ntiles = 0;
    for (auto &g : e->groups64) g.clear();
    for (auto &g : e->mixgroups) g.clear();
    return BHR_OK;
  }
  std::vector<BatchSolve> solves(n);
  std::vector<ExtractArgs> ext(n);
  std::vector<SourceArgs> src;
  std::vector<MixedBatch> mixed;
  std::vector<int> fp64, mix, mix_index(n, -1);
  e->max_ptsx = 1;
  e->max_ptsy = 1;
  for (int i = 0; i < n; i++) {
    bhr_solver *s = e->active[i].s;
    BatchSolve &B = solves[i];
    double *vin[3] = {s->u0, s->u1, s->u2}, *out[3] = {s->u1, s->u2, s->u0};
    for (int k = 0; k < 3; k++) {
      B.maps[k] = s->maps[k];
      B.args[k] = solver_stage_args(s);
      B.args[k].vin = vin[k];
      B.args[k].un = s->u0;
      B.args[k].out = out[k];
    }
    if (s->mixed) {
      B.args[0].dout = s->d1f;
      MixedBatch X{};
      X.maps[0] = s->mmaps[0];
      X.maps[1] = s->mmaps[1];
      X.args[0] = X.args[1] = solver_mixed_args(s);
      X.args[0].e_out = s->e2f;
      X.args[1].u_out = s->u0;
      mix_index[i] = static_cast<int>(mixed.size());
      mixed.push_back(X);
      mix.push_back(i);
    } else {
      fp64.push_back(i);
    }
    ext[i] = solver_extract_args(s);
    ext[i].set_ks = 1;  // stages and extraction run in sequence here
    if (s->has_source) {
      src.push_back(solver_source_args(s));
      e->max_ptsx = std::max(e->max_ptsx, s->p.PTSX);
      e->max_ptsy = std::max(e->max_ptsy, s->p.PTSY);
    }
  }
  // The launch groups: blocks are ordered solve by solve, row band by row
  // band; stage 1 takes the FP64 solves, then the mixed ones.
  auto add = [](auto &groups, int row, int N, int M, int rows, const auto &args) {
    if (groups.empty() || groups.back().nsolves == kGroupSolves) {
      groups.emplace_back();
      std::memset(&groups.back(), 0, sizeof(groups.back()));
    }
    auto &g = groups.back();
    const int j = g.nsolves++;
    g.first[j] = g.ntiles;
    g.tiles_x[j] = N / TC;
    g.solve[j] = row;
    g.args[j] = args;
    g.ntiles += (N / TC) * (M / rows);
    g.first[j + 1] = g.ntiles;
  };
  std::vector<int> order1 = fp64;
  order1.insert(order1.end(), mix.begin(), mix.end());
  e->ntiles = 0;
  for (int stage = 1; stage <= 3; stage++) {
    std::vector<BatchGroup> &G = e->groups64[stage - 1];
    G.clear();
    for (int i : stage == 1 ? order1 : fp64) {
      const bhr_params &p = e->active[i].s->p;
      add(G, i, p.N, p.M, e->rows, solves[i].args[stage - 1]);
      if (stage == 1) e->ntiles += (p.N / TC) * (p.M / e->rows);
    }
  }
  for (int stage = 2; stage <= 3; stage++) {
    std::vector<MixedGroup> &G = e->mixgroups[stage - 2];
    G.clear();
    for (int i : mix) {
      const bhr_params &p = e->active[i].s->p;
      add(G, mix_index[i], p.N, p.M, kMixTileRows, mixed[mix_index[i]].args[stage - 2]);
      if (stage == 2) e->ntiles += (p.N / TC) * (p.M / kMixTileRows);
    }
  }
  e->nsrc = static_cast<int>(src.size());
  // The per-solve tables share one capacity.
  cudaError_t err = cudaSuccess;
  if (n > e->cap_solves) {
    const int c = std::max(n, 2 * e->cap_solves);
    if (e->d_solves) cudaFreeAsync(e->d_solves, e->stream);
    if (e->d_ext) cudaFreeAsync(e->d_ext, e->stream);
    if (e->d_src) cudaFreeAsync(e->d_src, e->stream);
    if (e->d_mixed) cudaFreeAsync(e->d_mixed, e->stream);
    e->d_solves = nullptr;
    e->d_ext = nullptr;
    e->d_src = nullptr;
    e->d_mixed = nullptr;
    e->cap_solves = 0;
    if ((err = cudaMallocAsync(&e->d_solves, sizeof(BatchSolve) * c, e->stream)) ||
        (err = cudaMallocAsync(&e->d_ext, sizeof(ExtractArgs) * c, e->stream)) || (err = cudaMallocAsync(&e->d_src, sizeof(SourceArgs) * c, e->stream)) ||
        (err = cudaMallocAsync(&e->d_mixed, sizeof(MixedBatch) * c, e->stream)))
      return set_fail(BHR_OUT_OF_MEMORY, std::string("engine tables: ") + cudaGetErrorString(err));
    e->cap_solves = c;
  }
  if ((err = cudaMemcpyAsync(e->d_solves, solves.data(), sizeof(BatchSolve) * n, cudaMemcpyHostToDevice, e->stream)) ||
      (err = cudaMemcpyAsync(e->d_ext, ext.data(), sizeof(ExtractArgs) * n, cudaMemcpyHostToDevice, e->stream)) ||
      (e->nsrc > 0 && (err = cudaMemcpyAsync(e->d_src, src.data(), sizeof(SourceArgs) * e->nsrc,
                                             cudaMemcpyHostToDevice, e->stream))) ||
      (!mixed.empty() && (err = cudaMemcpyAsync(e->d_mixed, mixed.data(), sizeof(MixedBatch) * mixed.size(),
                                                cudaMemcpyHostToDevice, e->stream))) ||
      (err = cudaStreamSynchronize(e->stream)))
    return set_fail(BHR_CUDA_ERROR, std::string("engine upload: ") + cudaGetErrorString(err));
  // Capture one batch step.
  cudaGraph_t g = nullptr;
  if ((err = cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal)))
    return set_fail(BHR_CUDA_ERROR, std::string("capture: ") + cudaGetErrorString(err));
  const int st = enqueue_batch_step(e);
  err = cudaStreamEndCapture(e->stream, &g);
  if (st != BHR_OK) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  if (err != cudaSuccess) return set_fail(BHR_CUDA_ERROR, std::string("capture: ") + cudaGetErrorString(err));
  err = cudaGraphInstantiate(&e->graph, g, 0);
  cudaGraphDestroy(g);
  if (err != cudaSuccess) return set_fail(BHR_CUDA_ERROR, std::string("instantiate: ") + cudaGetErrorString(err));
  return BHR_OK;
}

// Reads back a finished solve's waveform and releases it.
Finished finish(bhr_solver *s, const Running &R) {
  Finished f;
  f.t_submit = R.t_submit;
  f.t_start = R.t_start;
  f.steps = s->nt;
  bhr_info inf{};
  bhr_solver_info(s, &inf);
  f.t.resize(inf.rows_done);
  f.h.resize(static_cast<size_t>(inf.rows_done) * 14);
  f.dedt.resize(inf.rows_done);
  int nrows = 0;
  f.status = bhr_solver_waveform(s, f.t.data(), f.h.data(), f.dedt.data(), inf.rows_done, &nrows);
  if (f.status == BHR_OK) {
    RunState rs{};
    if (cudaMemcpy(&rs, s->rs, sizeof(rs), cudaMemcpyDeviceToHost) != cudaSuccess)
      f.status = BHR_CUDA_ERROR;
    else if (rs.err)
      f.status = rs.err;
  }
  f.state = f.status == BHR_OK ? 3 : 4;
  if (f.status != BHR_OK) f.error = bhr_last_error_string();
  f.t_finish = now_s();
  bhr_solver_destroy(s);
  return f;
}

// Later requests prepared ahead of the oldest queued one while it does not
// fit the budget, before admission waits for it (so it is not starved).
constexpr int kMaxBypass = 64;

// The worker: releases finished solves, then prepares queued requests in
// arrival order while their estimated bytes fit the budget (one always
// when nothing else holds memory).  When the oldest does not fit, the
// first later one that does goes ahead of it, up to kMaxBypass of them.
void worker_loop(bhr_engine *e) {
  cudaSetDevice(e->device);
  std::unique_lock<std::mutex> lock(e->wmu);
  for (;;) {
    // index in the queue of the request to prepare next, or -1
    auto pick = [&]() -> int {
      if (e->queue.empty()) return -1;
      auto fits = [&](const Request &r) {
        return e->used == 0 || e->used + solve_bytes(r.p, static_cast<int>(r.traj.size() / 10)) <= e->budget;
      };
      if (fits(e->queue.front())) return 0;
      if (e->queue.front().id != e->head_id) {
        e->head_id = e->queue.front().id;
        e->head_bypassed = 0;
      }
      if (e->head_bypassed >= kMaxBypass) return -1;
      for (size_t i = 1; i < e->queue.size(); i++)
        if (fits(e->queue[i])) return static_cast<int>(i);
      return -1;
    };
    e->wcv.wait(lock, [&] { return e->stop || !e->to_release.empty() || pick() >= 0; });
    if (e->stop) return;
    if (!e->to_release.empty()) {
      std::vector<Running> rel;
      rel.swap(e->to_release);
      e->releasing += static_cast<int>(rel.size());
      lock.unlock();
      for (Running &R : rel) {
        const size_t bytes = R.s->bytes;
        Finished f = finish(R.s, R);
        {
          std::lock_guard<std::mutex> dl(e->dmu);
          e->done[R.id] = std::move(f);
          e->finished++;
        }
        lock.lock();
        e->used -= std::min(e->used, bytes);
        e->releasing--;
        e->rcv.notify_all();
        lock.unlock();
      }
      lock.lock();
      continue;
    }
    const int at = pick();
    Request r = std::move(e->queue[static_cast<size_t>(at)]);
    e->queue.erase(e->queue.begin() + at);
    if (at > 0) e->head_bypassed++;
    const size_t need = solve_bytes(r.p, static_cast<int>(r.traj.size() / 10));
    e->used += need;
    e->preparing.insert(r.id);
    lock.unlock();
    r.p.device = e->device;
    bhr_solver *s = nullptr;
    int st = solver_create(&r.p, e->rows, &s);
    if (st == BHR_OK && !r.traj.empty()) {
      st = bhr_solver_set_trajectory(s, r.traj.data(), static_cast<int>(r.traj.size() / 10));
      // batch steps read every step's record without waiting: all of them first
      if (st == BHR_OK) st = solver_wait_records(s, s->nt);
    }
    std::string msg;
    if (st != BHR_OK) {
      msg = bhr_last_error_string();
      if (s) bhr_solver_destroy(s);
      s = nullptr;
      Finished f;
      f.state = 4;
      f.status = st;
      f.error = msg;
      f.t_submit = r.t_submit;
      f.t_start = f.t_finish = now_s();
      std::lock_guard<std::mutex> dl(e->dmu);
      e->done[r.id] = std::move(f);
    }
    lock.lock();
    e->preparing.erase(r.id);
    e->used -= std::min(e->used, need);
    if (s) {
      e->used += s->bytes;
      e->ready.push_back({r.id, s, r.t_submit, now_s(), s->nt - s->steps_done});
    }
    e->rcv.notify_all();
  }
}

// Moves prepared solves into the running set (mu held).  When none is
// running but some are being prepared, waits a little for them.
void join_ready(bhr_engine *e) {
  std::unique_lock<std::mutex> lock(e->wmu);
  if (e->active.empty() && e->ready.empty() &&
      (!e->preparing.empty() || !e->queue.empty() || !e->to_release.empty() || e->releasing > 0))
    e->rcv.wait_for(lock, std::chrono::milliseconds(200), [&] { return !e->ready.empty(); });
  if (e->ready.empty()) return;
  for (Running &R : e->ready) {
    R.t_start = now_s();
    e->active.push_back(R);
  }
  e->ready.clear();
  e->dirty = true;
}

// Hands solves whose last step has run to the worker (mu held).
void hand_off_finished(bhr_engine *e) {
  std::vector<Running> fin;
  for (size_t i = 0; i < e->active.size();) {
    if (e->active[i].remaining > 0) {
      i++;
      continue;
    }
    fin.push_back(e->active[i]);
    e->active.erase(e->active.begin() + static_cast<long>(i));
    e->dirty = true;
  }
  if (fin.empty()) return;
  std::lock_guard<std::mutex> lock(e->wmu);
  e->to_release.insert(e->to_release.end(), fin.begin(), fin.end());
  e->wcv.notify_all();
}

}  // namespace

extern "C" {

int bhr_engine_create(int device, size_t hbm_budget_bytes, bhr_engine **out) {
  if (!out) return set_fail(BHR_INVALID_ARG, "null argument");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
    cudaGetLastError();
    return set_fail(BHR_NO_DEVICE, "no CUDA device");
  }
  if (device < 0 || device >= ndev) return set_fail(BHR_INVALID_ARG, "device ordinal out of range");
  auto *e = new bhr_engine();
  e->device = device;
  e->budget = hbm_budget_bytes;
  if (cudaSetDevice(device) != cudaSuccess || prepare_kernels() != cudaSuccess ||
      prepare_mixed_kernels() != cudaSuccess ||
      cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&e->ev0) != cudaSuccess || cudaEventCreate(&e->ev1) != cudaSuccess ||
      cudaMalloc(&e->d_err, sizeof(int)) != cudaSuccess || cudaMemset(e->d_err, 0, sizeof(int)) != cudaSuccess) {
    delete e;
    return set_fail(BHR_CUDA_ERROR, "engine set-up failed");
  }
  // BHR_ENGINE_TILING=block8|block16|persistent|block8n|ring selects the
  // FP64 stage kernels over the work-list (default block8n: 8-row tiles on
  // 128-thread blocks, each prefetching the work item two SM-counts ahead).
  if (const char *v = std::getenv("BHR_ENGINE_TILING")) {
    static const char *names[] = {"block8", "block16", "persistent", "block8n", "ring"};
    for (int t = 0; t < 5; t++)
      if (!std::strcmp(v, names[t])) e->tiling = t;
  }
  e->rows = tiling_rows(e->tiling);
  e->worker = std::thread(worker_loop, e);
  *out = e;
  return BHR_OK;
}

void bhr_engine_destroy(bhr_engine *e) {
  if (!e) return;
  {
    std::lock_guard<std::mutex> lock(e->wmu);
    e->stop = true;
    e->wcv.notify_all();
  }
  if (e->worker.joinable()) e->worker.join();
  std::lock_guard<std::mutex> lock(e->mu);
  cudaSetDevice(e->device);
  cudaStreamSynchronize(e->stream);
  for (auto &R : e->active) bhr_solver_destroy(R.s);
  for (auto &R : e->ready) bhr_solver_destroy(R.s);
  for (auto &R : e->to_release) bhr_solver_destroy(R.s);
  e->active.clear();
  release_tables(e);
  cudaStreamSynchronize(e->stream);
  if (e->ev0) cudaEventDestroy(e->ev0);
  if (e->ev1) cudaEventDestroy(e->ev1);
  if (e->d_err) cudaFree(e->d_err);
  cudaStreamDestroy(e->stream);
  delete e;
}

int bhr_engine_submit(bhr_engine *e, const bhr_params *p, const double *traj_rows, int nrows, int64_t *id) {
  if (!e || !p || !id || (traj_rows && nrows < 2)) return set_fail(BHR_INVALID_ARG, "bad submit arguments");
  if (p->integrator != BHR_SSPRK3) return set_fail(BHR_INVALID_ARG, "the batch engine steps BHR_SSPRK3 solves only");
  Request r;
  r.p = *p;
  if (traj_rows) r.traj.assign(traj_rows, traj_rows + static_cast<size_t>(nrows) * 10);
  r.t_submit = now_s();
  std::lock_guard<std::mutex> lock(e->wmu);
  r.id = e->next_id++;
  *id = r.id;
  e->queue.push_back(std::move(r));
  e->wcv.notify_all();
  return BHR_OK;
}

int bhr_engine_step(bhr_engine *e, int max_steps, int *running) {
  NvtxRange range("bhr_engine_step");
  if (!e || max_steps < 0) return set_fail(BHR_INVALID_ARG, "bad step arguments");
  std::lock_guard<std::mutex> lock(e->mu);
  if (cudaSetDevice(e->device) != cudaSuccess) return set_fail(BHR_CUDA_ERROR, "cudaSetDevice failed");
  join_ready(e);
  if (e->dirty)
    if (int st = rebuild(e)) return st;
  int n = max_steps;
  for (auto &R : e->active) n = std::min(n, R.remaining);
  if (!e->active.empty() && n > 0) {
    cudaError_t err = cudaEventRecord(e->ev0, e->stream);
    for (int i = 0; i < n && err == cudaSuccess; i++) err = cudaGraphLaunch(e->graph, e->stream);
    if (err == cudaSuccess) err = cudaEventRecord(e->ev1, e->stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
    if (err != cudaSuccess) return set_fail(BHR_CUDA_ERROR, std::string("engine step: ") + cudaGetErrorString(err));
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, e->ev0, e->ev1) == cudaSuccess) e->device_ms += ms;
    int derr = 0;
    if (cudaMemcpy(&derr, e->d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess || derr != 0)
      return set_fail(BHR_TIMEOUT, "engine step: a bounded device wait gave up");
    double pts = 0.0;
    for (auto &R : e->active) {
      R.remaining -= n;
      R.s->steps_done += n;
      pts += static_cast<double>(R.s->p.N) * R.s->p.M;
    }
    e->batch_steps += n;
    e->point_updates += pts * n;
  }
  hand_off_finished(e);
  if (running) {
    std::lock_guard<std::mutex> wl(e->wmu);
    *running = static_cast<int>(e->active.size() + e->ready.size() + e->preparing.size() + e->to_release.size() +
                                e->releasing);
  }
  return BHR_OK;
}

int bhr_engine_poll(bhr_engine *e, int64_t id, bhr_request_info *info) {
  if (!e || !info) return set_fail(BHR_INVALID_ARG, "bad poll arguments");
  std::memset(info, 0, sizeof(*info));
  {
    std::lock_guard<std::mutex> lock(e->wmu);
    for (auto &r : e->queue)
      if (r.id == id) {
        info->state = 1;
        info->submit_s = r.t_submit;
        return BHR_OK;
      }
    if (e->preparing.count(id)) {
      info->state = 1;
      return BHR_OK;
    }
    for (auto &R : e->ready)
      if (R.id == id) {
        info->state = 2;
        info->steps_total = R.s->nt;
        info->submit_s = R.t_submit;
        return BHR_OK;
      }
  }
  {
    std::lock_guard<std::mutex> lock(e->mu);
    for (auto &R : e->active)
      if (R.id == id) {
        info->state = 2;
        info->steps_total = R.s->nt;
        info->steps_done = R.s->steps_done;
        info->submit_s = R.t_submit;
        info->start_s = R.t_start;
        return BHR_OK;
      }
  }
  std::lock_guard<std::mutex> lock(e->dmu);
  auto it = e->done.find(id);
  if (it == e->done.end()) {
    // finished but not yet released by the worker: still reported running
    std::lock_guard<std::mutex> wl(e->wmu);
    for (auto &R : e->to_release)
      if (R.id == id) {
        info->state = 2;
        info->steps_total = info->steps_done = R.s->nt;
        info->submit_s = R.t_submit;
        info->start_s = R.t_start;
      }
    return BHR_OK;
  }
  const Finished &f = it->second;
  info->state = f.state;
  info->status = f.status;
  info->nrows = static_cast<int>(f.t.size());
  info->steps_total = info->steps_done = f.steps;
  info->submit_s = f.t_submit;
  info->start_s = f.t_start;
  info->finish_s = f.t_finish;
  return BHR_OK;
}

int bhr_engine_result(bhr_engine *e, int64_t id, double *t, double *h, double *dedt, int max_rows, int *nrows) {
  if (!e) return set_fail(BHR_INVALID_ARG, "null engine");
  std::lock_guard<std::mutex> lock(e->dmu);
  auto it = e->done.find(id);
  if (it == e->done.end()) return set_fail(BHR_INVALID_ARG, "request not finished");
  const Finished &f = it->second;
  if (f.state != 3) return set_fail(f.status ? f.status : BHR_INVALID_ARG, "request failed: " + f.error);
  const int n = std::min(static_cast<int>(f.t.size()), std::max(0, max_rows));
  if (t) std::memcpy(t, f.t.data(), sizeof(double) * n);
  if (h) std::memcpy(h, f.h.data(), sizeof(double) * 14 * n);
  if (dedt) std::memcpy(dedt, f.dedt.data(), sizeof(double) * n);
  if (nrows) *nrows = n;
  return BHR_OK;
}

int bhr_engine_stats(bhr_engine *e, bhr_engine_counters *st) {
  if (!e || !st) return set_fail(BHR_INVALID_ARG, "bad stats arguments");
  std::memset(st, 0, sizeof(*st));
  {
    std::lock_guard<std::mutex> lock(e->wmu);
    st->queued = static_cast<int>(e->queue.size() + e->preparing.size());
    st->running = static_cast<int>(e->ready.size() + e->to_release.size() + e->releasing);
    st->bytes_in_use = e->used;
  }
  {
    std::lock_guard<std::mutex> lock(e->dmu);
    st->finished = e->finished;
  }
  std::lock_guard<std::mutex> lock(e->mu);
  st->running += static_cast<int>(e->active.size());
  st->batch_steps = e->batch_steps;
  st->point_updates = e->point_updates;
  st->device_ms = e->device_ms;
  st->budget = e->budget;
  st->tiles = e->ntiles;
  return BHR_OK;
}

}  // extern "C"
