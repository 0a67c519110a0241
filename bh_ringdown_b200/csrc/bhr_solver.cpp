// bhr_solver.cpp -- the C ABI of include/bhr.h: one solve on one device.
//
// Replaces body() of HighOrder/body.cu:25-225.  Differences in structure:
// all state is per solve (no __device__ globals), the trajectory is read
// once into memory and turned into per-step source records before the
// loop, the extraction integrals and the projection stay on the device, and
// a step is five kernel launches on one stream with no host round trip.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <array>
#include <atomic>
#include <thread>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "bhr.h"
#include "bhr_host.h"
#include "bhr_internal.h"
#include "bhr_solver_impl.h"

namespace bhr {

static thread_local std::string g_err;
void set_error(const std::string &msg) { g_err = msg; }

#define BHR_CUDA_TRY(call)                                                                \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) {                                                              \
      set_error(std::string(#call) + ": " + cudaGetErrorString(e_));                      \
      return BHR_CUDA_ERROR;                                                              \
    }                                                                                     \
  } while (0)

}  // namespace bhr

using namespace bhr;

static constexpr int kGraphBatch = 16;

namespace {

int validate(const bhr_params &p) {
  if (p.N < 64 || p.N % TC != 0) {
    set_error("N must be a positive multiple of 64");
    return BHR_INVALID_ARG;
  }
  if (p.M < 16 || p.M % TR != 0) {
    set_error("M must be a multiple of 16 and >= 16");
    return BHR_INVALID_ARG;
  }
  if (!(p.Xmax > p.Xmin) || !(p.mass > 0.0) || !(std::fabs(p.a) < p.mass) || !(p.T > 0.0)) {
    set_error("need Xmax > Xmin, mass > 0, |a| < mass, T > 0");
    return BHR_INVALID_ARG;
  }
  if (p.m != std::floor(p.m)) {
    set_error("m must be an integer");
    return BHR_INVALID_ARG;
  }
  if (p.PTSX < 1 || p.PTSX > 1024 || p.PTSY < 1 || p.PTSY > 65535) {
    set_error("PTSX in [1,1024], PTSY >= 1");
    return BHR_INVALID_ARG;
  }
  if ((p.precision != BHR_FP64 && p.precision != BHR_MIXED) || (p.integrator != BHR_SSPRK3 && p.integrator != BHR_RK4)) {
    set_error("precision must be BHR_FP64 or BHR_MIXED and the integrator BHR_SSPRK3 or BHR_RK4");
    return BHR_INVALID_ARG;
  }
  if (p.integrator == BHR_RK4 && p.precision != BHR_FP64) {
    set_error("BHR_RK4 runs in BHR_FP64 only");
    return BHR_INVALID_ARG;
  }
  return BHR_OK;
}

template <class T>
int dalloc(bhr_solver *s, T **ptr, size_t count) {
  const size_t nbytes = sizeof(T) * (count ? count : 1);
  // Stream-ordered allocation from the device's pool: neither this nor the
  // matching cudaFreeAsync synchronizes the device, so solves can be
  // created and destroyed while others are stepping.
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void **>(ptr), nbytes, s->stream);
  if (e != cudaSuccess) {
    set_error(std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? BHR_OUT_OF_MEMORY : BHR_CUDA_ERROR;
  }
  s->bytes += nbytes;
  return BHR_OK;
}

void free_all(bhr_solver *s) {
  if (s->rec_thread.joinable()) {  // it writes into s->recs
    s->rec_stop = true;
    s->rec_thread.join();
  }
  void *ptrs[] = {s->u0,    s->u1,   s->u2,     s->u3,     s->coltab, s->rowtab, s->ctab,   s->rc,     s->th,
                  s->src,   s->ext,  s->integ,  s->wproj,  s->wdedt,  s->rows,   s->recs,   s->rs,  s->psirows,
                  s->d1f,   s->e2f,  s->colf32, s->rowf32, s->bbf};
  for (void *q : ptrs)
    if (q) cudaFreeAsync(q, s->stream);
  if (s->g1) cudaGraphExecDestroy(s->g1);
  if (s->gb) cudaGraphExecDestroy(s->gb);
  s->g1 = s->gb = nullptr;
  if (s->stream) {
    cudaStreamSynchronize(s->stream);
    cudaStreamDestroy(s->stream);
  }
  if (s->side) {
    cudaStreamSynchronize(s->side);
    cudaStreamDestroy(s->side);
  }
  if (s->fork) cudaEventDestroy(s->fork);
  if (s->join) cudaEventDestroy(s->join);
  if (s->fork2) cudaEventDestroy(s->fork2);
  s->stream = s->side = nullptr;
  s->fork = s->join = s->fork2 = nullptr;
}

// The device's default memory pool keeps freed blocks for reuse instead of
// returning them to the driver at each synchronization (once per device
// per process).
int keep_pool_memory(int device) {
  static std::mutex mu;
  static bool done[64] = {false};
  std::lock_guard<std::mutex> lock(mu);
  if (device < 0 || device >= 64 || done[device]) return 0;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) != cudaSuccess) return 1;
  uint64_t keep = UINT64_MAX;
  if (cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess) return 1;
  done[device] = true;
  return 0;
}

// Kerr tortoise coordinate as the source placement uses it
// (HighOrder/kern.cu:1194-1199).
double tortoise(double r, double a, double rpl, double rmn) {
  return r + (rpl * rpl + a * a) / (rpl - rmn) * std::log(r / rpl - 1.0) -
         (rmn * rmn + a * a) / (rpl - rmn) * std::log(r / rmn - 1.0);
}

}  // namespace

static int autotune_rows(bhr_solver *s);
static int flush_extract(bhr_solver *s);


extern "C" {

int bhr_abi_version(void) { return BHR_ABI_VERSION; }

int bhr_selftest_bounded_wait(int device, int *device_status) {
  if (!device_status) return BHR_INVALID_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    set_error("no CUDA device");
    return BHR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) return BHR_INVALID_ARG;
  BHR_CUDA_TRY(cudaSetDevice(device));
  cudaStream_t st = nullptr;
  int *d = nullptr;
  BHR_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void **>(&d), sizeof(int), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(d, 0, sizeof(int), st);
  if (e == cudaSuccess) e = launch_wait_selftest(d, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(device_status, d, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (d) cudaFreeAsync(d, st);
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  if (e != cudaSuccess) {
    set_error(std::string("wait self-check: ") + cudaGetErrorString(e));
    return BHR_CUDA_ERROR;
  }
  return BHR_OK;
}
int bhr_selftest_math(int device, const double *x, int n, double *out) {
  if (!x || !out || n <= 0) return BHR_INVALID_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    set_error("no CUDA device");
    return BHR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) return BHR_INVALID_ARG;
  BHR_CUDA_TRY(cudaSetDevice(device));
  cudaStream_t st = nullptr;
  double *d = nullptr;
  BHR_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  const size_t bytes = sizeof(double) * static_cast<size_t>(n);
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void **>(&d), 5 * bytes, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d, x, bytes, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = launch_math_selftest(d, n, d + n, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, d + n, 4 * bytes, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (d) cudaFreeAsync(d, st);
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  if (e != cudaSuccess) {
    set_error(std::string("math self-check: ") + cudaGetErrorString(e));
    return BHR_CUDA_ERROR;
  }
  return BHR_OK;
}
const char *bhr_last_error_string(void) { return g_err.c_str(); }
double bhr_swsh(double ell, double m, double theta) { return swsh(ell, m, theta); }

int bhr_params_default(bhr_params *p) {
  if (!p) return BHR_INVALID_ARG;
  std::memset(p, 0, sizeof(*p));
  p->N = 16000;
  p->M = 256;
  p->Xmin = -50.0;
  p->Xmax = 50.0;
  p->mass = 1.0;
  p->a = 1e-8;
  p->m = 2.0;
  p->dt = 0.002;
  p->courant = 0.25;
  p->out_every = 0.0;
  p->T = 1500.0;
  p->Fr = 50;
  p->out_start = p->Xmax + 200.0;
  p->ext_col = -1;
  p->PTSX = 128;
  p->PTSY = 128;
  p->wr_fac = 2.0;
  p->wt_fac = 6.0;
  p->integrator = BHR_SSPRK3;
  p->precision = BHR_FP64;
  p->init_kind = BHR_INIT_ZERO;
  p->init_center = 20.0;
  p->init_width = 2.0;
  p->init_ell = 2.0;
  p->device = 0;
  return BHR_OK;
}

int bhr_grid(const bhr_params *p, double *x_c, double *r_c, double *theta) {
  if (!p) return BHR_INVALID_ARG;
  if (int st = validate(*p)) return st;
  Grid g = make_grid(*p);
  if (x_c) std::memcpy(x_c, g.x_c.data(), sizeof(double) * p->N);
  if (r_c) std::memcpy(r_c, g.r_c.data(), sizeof(double) * p->N);
  if (theta) std::memcpy(theta, g.theta.data(), sizeof(double) * p->M);
  return BHR_OK;
}

int bhr_solver_create(const bhr_params *pin, bhr_solver **out) { return bhr::solver_create(pin, 0, out); }

}  // extern "C"

static int encode_maps(bhr_solver *s, int rows);

int bhr::solver_create(const bhr_params *pin, int tile_rows, bhr_solver **out) {
  NvtxRange range("bhr_solver_create");
  if (!pin || !out) {
    set_error("null argument");
    return BHR_INVALID_ARG;
  }
  *out = nullptr;
  if (int st = validate(*pin)) return st;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
    cudaGetLastError();
    set_error("no CUDA device");
    return BHR_NO_DEVICE;
  }
  if (pin->device < 0 || pin->device >= ndev) {
    set_error("device ordinal out of range");
    return BHR_INVALID_ARG;
  }
  auto *s = new bhr_solver();
  s->p = *pin;
  bhr_params &p = s->p;
  s->g = make_grid(p);
  const Grid &g = s->g;
  if (!(p.dt > 0.0)) {
    double dt = p.courant * std::fmin(g.dx, g.r_c[0] * g.dtheta);
    if (p.out_every > 0.0) {
      const double k = std::ceil(p.out_every / dt);
      dt = p.out_every / k;
      if (p.Fr <= 0) p.Fr = static_cast<int>(k);
    }
    p.dt = dt;
  }
  if (p.Fr <= 0) p.Fr = (p.out_every > 0.0) ? std::max(1, static_cast<int>(std::lround(p.out_every / p.dt))) : 1;
  s->Fr = p.Fr;
  s->ext_col = (p.ext_col < 0 || p.ext_col >= p.N) ? p.N - 1 : p.ext_col;
  s->even_m = (static_cast<int>(p.m) % 2) == 0;
  // HighOrder/body.cu:56-59 for rank 0 of p = 1.
  const double endtime = (p.T - p.Xmax - 200.0) / 1 * (0 + 1) + p.Xmax + 200.0;
  s->nt = static_cast<int>((endtime - 0.0) / p.dt);
  s->max_rows = s->nt / s->Fr + 2;

  const size_t NM = static_cast<size_t>(p.N) * p.M;
  int st = BHR_OK;
  // The side stream (source, extraction: a few blocks beside the stages)
  // gets the device's highest priority, so its blocks take the first SM
  // slots that free up.
  int hi_prio = 0;
  if (cudaSetDevice(p.device) != cudaSuccess || prepare_kernels() != cudaSuccess || keep_pool_memory(p.device) ||
      cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaDeviceGetStreamPriorityRange(nullptr, &hi_prio) != cudaSuccess ||
      cudaStreamCreateWithPriority(&s->side, cudaStreamNonBlocking, hi_prio) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->join, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->fork2, cudaEventDisableTiming) != cudaSuccess) {
    set_error("cannot set device / create stream");
    delete s;
    return BHR_CUDA_ERROR;
  }
  if ((st = dalloc(s, &s->u0, 4 * NM)) || (st = dalloc(s, &s->u1, 4 * NM)) || (st = dalloc(s, &s->u2, 4 * NM)) ||
      (st = dalloc(s, &s->coltab, static_cast<size_t>(CF_COUNT) * p.N)) ||
      (st = dalloc(s, &s->rowtab, static_cast<size_t>(RF_COUNT) * p.M)) || (st = dalloc(s, &s->ctab, NM)) ||
      (st = dalloc(s, &s->rc, p.N)) ||
      (st = dalloc(s, &s->th, p.M)) || (st = dalloc(s, &s->src, 4 * static_cast<size_t>(p.PTSX) * p.PTSY)) ||
      (st = dalloc(s, &s->ext, 2 * static_cast<size_t>(p.M))) || (st = dalloc(s, &s->integ, 4 * static_cast<size_t>(p.M))) ||
      (st = dalloc(s, &s->wproj, 7 * static_cast<size_t>(p.M))) || (st = dalloc(s, &s->wdedt, p.M)) ||
      (st = dalloc(s, &s->rows, 16 * static_cast<size_t>(s->max_rows))) ||
      (st = dalloc(s, &s->psirows, 2 * static_cast<size_t>(p.M) * s->max_rows)) || (st = dalloc(s, &s->rs, 1))) {
    free_all(s);
    delete s;
    return st;
  }
  std::vector<double> coltab, rowtab, w7, we, fa, gb;
  make_tables(p, g, coltab, rowtab);
  make_projection_weights(p, g, w7);
  make_dedt_weights(p, g, we);
  make_initial_factors(p, g, fa, gb);
  double *dfac = nullptr;  // fa then gb, freed once the product is formed
  if (!fa.empty() && cudaMallocAsync(reinterpret_cast<void **>(&dfac), (fa.size() + gb.size()) * 8, s->stream) !=
                         cudaSuccess) {
    set_error("cudaMallocAsync failed (initial data factors)");
    free_all(s);
    delete s;
    return BHR_OUT_OF_MEMORY;
  }
  auto up = [&](void *dst, const void *srcp, size_t n) { return cudaMemcpyAsync(dst, srcp, n, cudaMemcpyHostToDevice, s->stream); };
  cudaError_t e = cudaSuccess;
  if ((e = up(s->coltab, coltab.data(), coltab.size() * 8)) || (e = up(s->rowtab, rowtab.data(), rowtab.size() * 8)) ||
      (e = up(s->rc, g.r_c.data(), g.r_c.size() * 8)) || (e = up(s->th, g.theta.data(), g.theta.size() * 8)) ||
      (e = up(s->wproj, w7.data(), w7.size() * 8)) || (e = up(s->wdedt, we.data(), we.size() * 8)) ||
      (e = cudaMemsetAsync(s->u0, 0, 4 * NM * 8, s->stream)) ||
      (e = launch_coef_tables(s->coltab, s->rowtab, s->ctab, p.N, p.M, s->stream)) ||
      (e = cudaMemsetAsync(s->u1, 0, 4 * NM * 8, s->stream)) || (e = cudaMemsetAsync(s->u2, 0, 4 * NM * 8, s->stream)) ||
      (e = cudaMemsetAsync(s->integ, 0, 4 * p.M * 8, s->stream)) || (e = cudaMemsetAsync(s->ext, 0, 2 * p.M * 8, s->stream)) ||
      (e = cudaMemsetAsync(s->src, 0, 4 * static_cast<size_t>(p.PTSX) * p.PTSY * 8, s->stream)) ||
      (e = cudaMemsetAsync(s->rs, 0, sizeof(RunState), s->stream)) || (e = cudaStreamSynchronize(s->stream))) {
    set_error(std::string("upload: ") + cudaGetErrorString(e));
    if (dfac) cudaFreeAsync(dfac, s->stream);
    free_all(s);
    delete s;
    return BHR_CUDA_ERROR;
  }
  if (dfac) {  // Gaussian initial data: the products formed on the device
    if ((e = up(dfac, fa.data(), fa.size() * 8)) == cudaSuccess &&
        (e = up(dfac + fa.size(), gb.data(), gb.size() * 8)) == cudaSuccess)
      e = launch_init_product(s->u0, dfac, dfac + fa.size(), p.N, p.M, s->stream);
    cudaFreeAsync(dfac, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) {
      set_error(std::string("initial data: ") + cudaGetErrorString(e));
      free_all(s);
      delete s;
      return BHR_CUDA_ERROR;
    }
  }
  // BHR_STAGE_TILING=block8|block16|persistent|block8n|ring fixes the stage
  // tiling of solves whose tiling is not fixed by the caller.
  if (tile_rows == 0) {
    if (const char *v = std::getenv("BHR_STAGE_TILING")) {
      if (!std::strcmp(v, "block8")) tile_rows = 8;
      if (!std::strcmp(v, "block16")) tile_rows = 16;
      if (!std::strcmp(v, "persistent")) {
        tile_rows = 16;
        s->persist = 1;
      }
      if (!std::strcmp(v, "block8n")) {
        tile_rows = 8;
        s->narrow = 1;
      }
      if (!std::strcmp(v, "ring")) {
        tile_rows = 8;
        s->ring = 1;
      }
      if (!std::strcmp(v, "strip12")) {  // FP64 SSP-RK3 only; otherwise block8n
        tile_rows = 8;
        s->narrow = 1;
        s->strip12 = (p.precision == BHR_FP64 && p.integrator == BHR_SSPRK3) ? 1 : 0;
      }
    }
  }
  if (p.integrator == BHR_RK4) {
    s->rk4 = true;
    if ((st = dalloc(s, &s->u3, 4 * NM))) {
      free_all(s);
      delete s;
      return st;
    }
    if ((e = cudaMemsetAsync(s->u3, 0, 4 * NM * 8, s->stream)) || (e = cudaStreamSynchronize(s->stream))) {
      set_error(std::string("upload: ") + cudaGetErrorString(e));
      free_all(s);
      delete s;
      return BHR_CUDA_ERROR;
    }
  }
  if (p.precision == BHR_MIXED) {
    s->mixed = true;
    const size_t nc = static_cast<size_t>(CF_COUNT) * p.N, nr = static_cast<size_t>(RF_COUNT) * p.M;
    cudaError_t e2 = cudaSuccess;
    if ((st = dalloc(s, &s->d1f, 4 * NM)) || (st = dalloc(s, &s->e2f, 4 * NM)) || (st = dalloc(s, &s->colf32, nc)) ||
        (st = dalloc(s, &s->rowf32, nr)) || (st = dalloc(s, &s->bbf, 4 * NM))) {
      free_all(s);
      delete s;
      return st;
    }
    if ((e2 = prepare_mixed_kernels()) || (e2 = launch_to_float(s->coltab, s->colf32, nc, s->stream)) ||
        (e2 = launch_to_float(s->rowtab, s->rowf32, nr, s->stream)) ||
        (e2 = launch_mixed_coef(s->coltab, s->rowtab, s->ctab, s->bbf, p.N, p.M, 0.016666666666667 / g.dx,
                                s->stream)) ||
        (e2 = cudaMemsetAsync(s->d1f, 0, 4 * NM * sizeof(float), s->stream)) ||
        (e2 = cudaMemsetAsync(s->e2f, 0, 4 * NM * sizeof(float), s->stream)) ||
        (e2 = encode_mixed_maps(s->d1f, s->bbf, s->colf32, s->rowf32, nullptr, p.N, p.M, &s->mmaps[0])) ||
        (e2 = encode_mixed_maps(s->e2f, s->bbf, s->colf32, s->rowf32, s->u1, p.N, p.M, &s->mmaps[1])) ||
        (e2 = cudaStreamSynchronize(s->stream))) {
      set_error(std::string("mixed-precision set-up: ") + cudaGetErrorString(e2));
      free_all(s);
      delete s;
      return BHR_CUDA_ERROR;
    }
  }
  if (int rc = (tile_rows == 8 || tile_rows == 16) ? encode_maps(s, tile_rows) : autotune_rows(s)) {
    free_all(s);
    delete s;
    return rc;
  }
  *out = s;
  return BHR_OK;
}

extern "C" {

void bhr_solver_destroy(bhr_solver *s) {
  if (!s) return;
  cudaSetDevice(s->p.device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  free_all(s);
  delete s;
}

int bhr_solver_info(const bhr_solver *s, bhr_info *info) {
  if (!s || !info) return BHR_INVALID_ARG;
  info->N = s->p.N;
  info->M = s->p.M;
  info->dx = s->g.dx;
  info->dtheta = s->g.dtheta;
  info->dt = s->p.dt;
  info->nt = s->nt;
  info->Fr = s->Fr;
  info->steps_done = s->steps_done;
  // Reading the row count completes the last step's extraction first.
  if (int st = flush_extract(const_cast<bhr_solver *>(s))) return st;
  RunState rs{};
  BHR_CUDA_TRY(cudaMemcpyAsync(&rs, s->rs, sizeof(rs), cudaMemcpyDeviceToHost, s->stream));
  BHR_CUDA_TRY(cudaStreamSynchronize(s->stream));
  info->rows_done = rs.nrow;
  info->has_source = s->has_source ? 1 : 0;
  info->r_plus = s->g.r_plus;
  info->device_bytes = s->bytes;
  info->tile_rows = s->tile_rows;
  info->persistent = s->persist || s->ring;
  info->prefetch_ahead = (s->persist || s->ring) ? 0 : stage_prefetch_ahead(s->ahead);
  info->tiling = s->strip12 ? BHR_TILING_STRIP12
                 : s->ring ? BHR_TILING_RING
                 : s->narrow ? BHR_TILING_BLOCK8N
                 : s->persist ? BHR_TILING_PERSISTENT
                 : s->tile_rows == 8 ? BHR_TILING_BLOCK8 : BHR_TILING_BLOCK16;
  return BHR_OK;
}

}  // extern "C"

// Steps whose source records set_trajectory builds before it returns; the
// rest follow in chunks of kRecordChunk on a host thread.
static constexpr int kFirstRecords = 8192;
static constexpr int kRecordChunk = 16384;

// HighOrder/body.cu:97-124 as a resumable cursor over a copy of the
// trajectory rows: the pre-loop reads one line and then lines until
// ptime >= timer; each step reads two lines and uses the second; a read
// past the end leaves the particle variables unchanged; rp gets +1e-6 every
// step; the second time derivatives are backward differences of the first
// over dt (zero history at step 0); third derivatives are 0.  fill() must be
// called for consecutive step ranges.
struct RecordJob {
  bhr_params p;
  double dx, dtheta, rpl, rmn;
  std::vector<double> rows;
  int nrows = 0, cursor = 0;
  double row[10] = {0};
  double rp = 0, tmp11 = 0, tmp22 = 0, tmp33 = 0, timer = 0, start = 0;

  void read() {
    if (cursor < nrows) {
      std::memcpy(row, rows.data() + static_cast<size_t>(10) * cursor, sizeof(row));
      cursor++;
    }
  }
  void begin() {
    timer = 0.0;
    start = timer;
    read();
    do {
      read();
    } while (row[0] < timer && cursor < nrows);
    rp = row[1];
  }
  // Particle state and turn-on factor of the next n steps.
  void fill(int n, bhr_particle *pts, double *turn) {
    for (int i = 0; i < n; i++) {
      const int c0 = cursor;
      read();
      read();
      if (cursor != c0) rp = row[1];
      rp = rp + 1e-6;
      bhr_particle &pt = pts[i];
      pt = bhr_particle{};
      pt.rp = rp;
      pt.tp = row[2];
      pt.phip = row[6];
      pt.E = row[7];
      pt.lz = row[8];
      pt.Q = row[9];
      pt.drdt = row[3];
      pt.d2rdt2 = (row[3] - tmp11) / p.dt;
      pt.dthdt = row[4];
      pt.d2thdt2 = (row[4] - tmp22) / p.dt;
      pt.dphidt = row[5];
      pt.d2phidt2 = (row[5] - tmp33) / p.dt;
      tmp11 = row[3];
      tmp22 = row[4];
      tmp33 = row[5];
      turn[i] = std::pow(1.0 - std::exp(-(timer - start) / 25.0), 4);
      timer += p.dt;
    }
  }
};

// Records of steps [k0, k1) into out[0 .. k1-k0) on all host threads, from
// those steps' particle states and turn-on factors (pts, turn, indexed from
// k0): source coefficients times the turn-on window, radial width and patch
// origin.  Returns the first step whose particle is off the grid, inside
// the horizon or on a pole (its status in *bad_status), or -1.
static int build_records(const RecordJob &J, int k0, int k1, const bhr_particle *pts, const double *turn,
                         StepRec *out, int *bad_status) {
  const bhr_params &p = J.p;
  std::mutex bad_mu;
  int first_bad = -1, status = BHR_OK;
  auto work = [&](int a0, int a1) {
    for (int k = a0; k < a1; k++) {
      const bhr_particle &pt = pts[k - k0];
      StepRec &R = out[k - k0];
      double cr[6], ci[6];
      const int st = bhr_source_coefficients(&pt, p.a, p.mass, p.m, cr, ci);
      const double xp = tortoise(pt.rp, p.a, J.rpl, J.rmn);
      const double ipd = (xp - p.Xmin) / J.dx, itd = pt.tp / J.dtheta;
      if (st != BHR_OK || !std::isfinite(ipd) || !std::isfinite(itd) || std::fabs(ipd) > 1e9 ||
          std::fabs(itd) > 1e9) {
        std::lock_guard<std::mutex> lock(bad_mu);  // keep the earliest bad step
        if (first_bad < 0 || k < first_bad) {
          first_bad = k;
          status = st != BHR_OK ? st : BHR_INVALID_ARG;
        }
        return;
      }
      for (int i = 0; i < 6; i++) {
        R.c_re[i] = cr[i] * turn[k - k0];
        R.c_im[i] = ci[i] * turn[k - k0];
      }
      R.rp = pt.rp;
      R.tp = pt.tp;
      R.wr = p.wr_fac * J.dx * (1.0 - J.rpl / pt.rp);
      R.col0 = static_cast<int>(ipd) - p.PTSX / 2;
      R.row0 = static_cast<int>(itd) - p.PTSY / 2;
    }
  };
  const int n = k1 - k0;
  const int nth = std::max(1, std::min(64, static_cast<int>(std::thread::hardware_concurrency())));
  if (n < 2048 || nth == 1) {
    work(k0, k1);
  } else {
    std::vector<std::thread> pool;
    const int chunk = (n + nth - 1) / nth;
    for (int t = 0; t < nth; t++) {
      const int a0 = k0 + t * chunk, a1 = std::min(k1, a0 + chunk);
      if (a0 < a1) pool.emplace_back(work, a0, a1);
    }
    for (auto &th : pool) th.join();
  }
  *bad_status = status;
  return first_bad;
}

// Host thread: records of steps [k_from, nt) chunk by chunk, each uploaded
// (on its own stream, waited for) before it is published to stepping.
static void record_worker(bhr_solver *s, std::shared_ptr<RecordJob> job, int k_from) {
  cudaSetDevice(job->p.device);
  cudaStream_t up = nullptr;
  const bool ok_stream = cudaStreamCreateWithFlags(&up, cudaStreamNonBlocking) == cudaSuccess;
  std::vector<StepRec> buf(kRecordChunk);
  std::vector<bhr_particle> pts(kRecordChunk);
  std::vector<double> turn(kRecordChunk);
  for (int k0 = k_from; k0 < s->nt && !s->rec_stop.load(); k0 += kRecordChunk) {
    const int k1 = std::min(s->nt, k0 + kRecordChunk);
    job->fill(k1 - k0, pts.data(), turn.data());
    int status = BHR_OK;
    int bad = build_records(*job, k0, k1, pts.data(), turn.data(), buf.data(), &status);
    if (bad < 0 && (!ok_stream ||
                    cudaMemcpyAsync(s->recs + k0, buf.data(), sizeof(StepRec) * (k1 - k0), cudaMemcpyHostToDevice,
                                    up) != cudaSuccess ||
                    cudaStreamSynchronize(up) != cudaSuccess)) {
      bad = k0;
      status = BHR_CUDA_ERROR;
    }
    std::lock_guard<std::mutex> lock(s->rec_mu);
    if (bad >= 0) {
      s->rec_bad = bad;
      s->rec_status = status;
      s->rec_cv.notify_all();
      break;
    }
    s->rec_ready = k1;
    s->rec_cv.notify_all();
  }
  if (up) cudaStreamDestroy(up);
  // Stepping waits only while a thread may still publish the records it needs.
  std::lock_guard<std::mutex> lock(s->rec_mu);
  s->rec_running = false;
  s->rec_cv.notify_all();
}

// Stops and joins a record thread (before its records are freed or replaced).
static void stop_records(bhr_solver *s) {
  if (!s->rec_thread.joinable()) return;
  s->rec_stop = true;
  s->rec_thread.join();
  s->rec_stop = false;
}

int bhr::solver_wait_records(bhr_solver *s, int upto) {
  if (!s->has_source) return BHR_OK;
  upto = std::min(upto, s->nt);
  std::unique_lock<std::mutex> lock(s->rec_mu);
  if (s->rec_unusable) {
    set_error("the last trajectory set on this solve failed; set one before stepping");
    return BHR_INVALID_ARG;
  }
  s->rec_cv.wait(lock, [&] {
    return s->rec_ready >= upto || (s->rec_bad >= 0 && s->rec_bad < upto) || !s->rec_running;
  });
  if (s->rec_bad >= 0 && s->rec_bad < upto) {
    set_error("trajectory step " + std::to_string(s->rec_bad) +
              (s->rec_status == BHR_CUDA_ERROR ? ": record upload failed"
                                               : ": particle off the grid, inside the horizon or on a pole"));
    return s->rec_status;
  }
  if (s->rec_ready < upto) {
    set_error("trajectory records end at step " + std::to_string(s->rec_ready));
    return BHR_INVALID_ARG;
  }
  return BHR_OK;
}

extern "C" {

// The trajectory cursor of HighOrder/body.cu:97-124 (RecordJob above)
// feeds the per-step source records.
int bhr_solver_set_trajectory(bhr_solver *s, const double *rows, int nrows) {
  NvtxRange range("bhr_solver_set_trajectory");
  if (!s || !rows || nrows < 2) {
    set_error("trajectory needs at least two rows");
    return BHR_INVALID_ARG;
  }
  cudaSetDevice(s->p.device);
  if (int st = flush_extract(s)) return st;
  stop_records(s);
  {
    // Until this call succeeds the solve has no usable records: a sourced
    // solve whose trajectory change fails reports it at its next step.
    std::lock_guard<std::mutex> lock(s->rec_mu);
    s->rec_unusable = s->has_source;
    s->rec_running = false;
  }
  const bhr_params &p = s->p;
  const double a = p.a, mass = p.mass;
  const double rpl = mass + std::sqrt(mass * mass - a * a), rmn = mass - std::sqrt(mass * mass - a * a);
  // Per step: particle state (a sequential cursor), then source
  // coefficients, width and patch origin (independent, on all host
  // threads).  The first chunk of steps is built here; the rest on a host
  // thread while the device steps (solver_wait_records holds stepping back
  // until the records it reaches are uploaded).
  auto job = std::make_shared<RecordJob>();
  job->p = p;
  job->dx = s->g.dx;
  job->dtheta = s->g.dtheta;
  job->rpl = rpl;
  job->rmn = rmn;
  job->rows.assign(rows, rows + static_cast<size_t>(10) * nrows);
  job->nrows = nrows;
  job->begin();
  const int k_first = std::min(s->nt, kFirstRecords);
  std::vector<StepRec> recs(static_cast<size_t>(std::max(1, k_first)));
  std::vector<bhr_particle> pts(static_cast<size_t>(std::max(1, k_first)));
  std::vector<double> turn(static_cast<size_t>(std::max(1, k_first)));
  job->fill(k_first, pts.data(), turn.data());
  int bad_status = BHR_OK;
  const int bad = build_records(*job, 0, k_first, pts.data(), turn.data(), recs.data(), &bad_status);
  if (bad >= 0) {
    set_error("trajectory step " + std::to_string(bad) + ": particle off the grid, inside the horizon or on a pole");
    return bad_status;
  }
  cudaSetDevice(p.device);
  if (s->recs) cudaFreeAsync(s->recs, s->stream), s->bytes -= sizeof(StepRec) * static_cast<size_t>(s->nt ? s->nt : 1);
  s->recs = nullptr;
  if (int st = dalloc(s, &s->recs, static_cast<size_t>(s->nt))) return st;
  BHR_CUDA_TRY(cudaMemcpyAsync(s->recs, recs.data(), sizeof(StepRec) * k_first, cudaMemcpyHostToDevice, s->stream));
  BHR_CUDA_TRY(cudaStreamSynchronize(s->stream));
  {
    std::lock_guard<std::mutex> lock(s->rec_mu);
    s->rec_ready = k_first;
    s->rec_bad = -1;
    s->rec_status = BHR_OK;
    s->rec_unusable = false;
    s->rec_running = k_first < s->nt;
  }
  s->has_source = true;
  if (k_first < s->nt) {
    try {
      s->rec_thread = std::thread(record_worker, s, job, k_first);
    } catch (const std::exception &) {
      std::lock_guard<std::mutex> lock(s->rec_mu);
      s->rec_running = false;
      s->rec_unusable = true;
      set_error("could not start the trajectory record thread");
      return BHR_OUT_OF_MEMORY;
    }
  }
  // The patch of the current step (later patches are built one step ahead).
  BHR_CUDA_TRY(launch_source(solver_source_args(s), s->stream));
  BHR_CUDA_TRY(cudaStreamSynchronize(s->stream));
  // The launch arguments now carry the source and the new records: step
  // graphs captured before (steps taken without a trajectory) are rebuilt.
  if (s->g1) cudaGraphExecDestroy(s->g1);
  if (s->gb) cudaGraphExecDestroy(s->gb);
  s->g1 = s->gb = nullptr;
  return BHR_OK;
}

int bhr_solver_load_trajectory(bhr_solver *s, const char *path) {
  if (!s || !path) return BHR_INVALID_ARG;
  std::ifstream f(path);
  if (!f) {
    set_error(std::string("cannot open ") + path);
    return BHR_IO_ERROR;
  }
  std::vector<double> rows;
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream is(line);
    double v[10];
    int n = 0;
    while (n < 10 && (is >> v[n])) n++;
    if (n == 0) continue;
    if (n != 10) {
      set_error("malformed .traj row (need 10 columns)");
      return BHR_IO_ERROR;
    }
    rows.insert(rows.end(), v, v + 10);
  }
  return bhr_solver_set_trajectory(s, rows.data(), static_cast<int>(rows.size() / 10));
}

}  // extern "C"

static int encode_maps(bhr_solver *s, int rows) {
  const bhr_params &p = s->p;
  // {stage input, u^n slot, output}: SSP-RK3 stages 0..2, RK4 extras 3, 4
  double *const plan[5][3] = {{s->u0, s->u0, s->u1}, {s->u1, s->u0, s->u2}, {s->u2, s->u0, s->u0},
                              {s->u2, s->u0, s->u1}, {s->u1, s->u3, s->u0}};
  for (int i = 0; i < (s->rk4 ? 5 : 3); i++) {
    StageMaps &m = s->maps[i];
    CUtensorMap unused_q, unused_p;
    if (encode_state_maps(plan[i][1], p.N, p.M, rows, &unused_q, &unused_p, &m.u) != cudaSuccess ||
        encode_state_maps(plan[i][2], p.N, p.M, rows, &unused_q, &unused_p, &m.o) != cudaSuccess ||
        encode_state_maps(plan[i][0], p.N, p.M, rows, &m.q, &m.p, nullptr) != cudaSuccess ||
        encode_coef_maps(s->ctab, s->coltab, s->rowtab, p.N, p.M, rows, &m) != cudaSuccess) {
      set_error("cuTensorMapEncodeTiled failed");
      return BHR_CUDA_ERROR;
    }
  }
  if (s->strip12 && encode_strip_maps(s->u0, s->ctab, p.N, p.M, &s->smaps) != cudaSuccess) {
    set_error("cuTensorMapEncodeTiled failed (strip maps)");
    return BHR_CUDA_ERROR;
  }
  s->tile_rows = rows;
  return BHR_OK;
}


// Stage tiling autotuner: per (device, N, M) the stage kernels are timed
// on stages 1 and 2 (which write only the solve's scratch stages u1, u2):
// 8-row tiles on 128-thread blocks with the L2 prefetch one, two or four
// SM-counts ahead or none (the staging depth), 8- and 16-row tiles one per
// 256-thread block, the persistent 16-row kernels, the 8-row ring, and
// stages 1 and 2 fused in one launch (FP64 SSP-RK3 solves only); the
// fastest is kept for the process.
static int autotune_rows(bhr_solver *s) {
  static std::mutex mu;
  // device, N, M, FP64 SSP-RK3, rows, persist, narrow, ring, strip12, ahead
  static std::vector<std::array<int, 10>> cache;
  const bhr_params &p = s->p;
  const int fused_ok = (!s->mixed && !s->rk4) ? 1 : 0;
  {
    std::lock_guard<std::mutex> lock(mu);
    for (auto &c : cache)
      if (c[0] == p.device && c[1] == p.N && c[2] == p.M && c[3] == fused_ok) {
        s->persist = c[5];
        s->narrow = c[6];
        s->ring = c[7];
        s->strip12 = c[8];
        s->ahead = c[9];
        return encode_maps(s, c[4]);
      }
  }
  // rows, persist, narrow, ring, strip12 (stages 1 and 2 in one launch: only
  // FP64 SSP-RK3 solves; its stage 3 is block8n), prefetch distance in SM
  // counts (-1: none)
  static const int cands[9][6] = {{8, 0, 1, 0, 0, 2}, {8, 0, 1, 0, 0, 1}, {8, 0, 1, 0, 0, 4}, {8, 0, 1, 0, 0, -1},
                                  {8, 0, 0, 0, 0, 2}, {16, 0, 0, 0, 0, 2}, {16, 1, 0, 0, 0, 0},
                                  {8, 0, 0, 1, 0, 0}, {8, 0, 1, 0, 1, 2}};
  const int ncand = fused_ok ? 9 : 8;
  const int nsm = device_sm_count();
  double best_ms = 1e30;
  int best = 0;
  cudaEvent_t e0, e1;
  BHR_CUDA_TRY(cudaEventCreate(&e0));
  BHR_CUDA_TRY(cudaEventCreate(&e1));
  // Stages 1 and 2 (they write only the solve's scratch stages u1, u2) of
  // each candidate, or the fused launch that replaces them.
  auto ahead_of = [&](int c) { return cands[c][5] < 0 ? 0 : cands[c][5] * nsm; };
  for (int c = 0; c < ncand; c++) {
    s->persist = cands[c][1];
    s->narrow = cands[c][2];
    s->ring = cands[c][3];
    s->strip12 = cands[c][4];
    s->ahead = ahead_of(c);
    if (int st = encode_maps(s, cands[c][0])) return st;
    StageArgs A = solver_stage_args(s);
    A.src = nullptr;
    for (int rep = 0; rep < 6; rep++) {
      if (rep == 2) BHR_CUDA_TRY(cudaEventRecord(e0, s->stream));
      if (s->strip12) {
        A.vin = s->u0; A.un = s->u0; A.out = s->u2;
        BHR_CUDA_TRY(launch_stage12_strip(s->smaps, A, s->stream));
        continue;
      }
      A.vin = s->u0; A.un = s->u0; A.out = s->u1;
      BHR_CUDA_TRY(launch_stage(1, s->maps[0], A, s->stream));
      A.vin = s->u1; A.un = s->u0; A.out = s->u2;
      BHR_CUDA_TRY(launch_stage(2, s->maps[1], A, s->stream));
    }
    BHR_CUDA_TRY(cudaEventRecord(e1, s->stream));
    BHR_CUDA_TRY(cudaEventSynchronize(e1));
    float ms = 0.f;
    BHR_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
    if (ms < best_ms) {
      best_ms = ms;
      best = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  {
    std::lock_guard<std::mutex> lock(mu);
    cache.push_back({p.device, p.N, p.M, fused_ok, cands[best][0], cands[best][1], cands[best][2], cands[best][3],
                     cands[best][4], ahead_of(best)});
  }
  s->persist = cands[best][1];
  s->narrow = cands[best][2];
  s->ring = cands[best][3];
  s->strip12 = cands[best][4];
  s->ahead = ahead_of(best);
  return encode_maps(s, cands[best][0]);
}

StageArgs bhr::solver_stage_args(bhr_solver *s) {
  const bhr_params &p = s->p;
  const double odx = 1.0 / s->g.dx, odth = 1.0 / s->g.dtheta, odt = 1.0 / p.dt;
  const double third = 0.33333333333333333;
  StageArgs A{};
  A.coltab = s->coltab;
  A.rowtab = s->rowtab;
  A.src = s->has_source ? s->src : nullptr;
  A.recs = s->recs;
  A.rs = s->rs;
  A.err = &s->rs->err;
  A.N = p.N;
  A.M = p.M;
  A.PTSX = p.PTSX;
  A.PTSY = p.PTSY;
  A.even_m = s->even_m ? 1 : 0;
  A.rows = s->tile_rows;
  A.persist = s->persist;
  A.narrow = s->narrow;
  A.ring = s->ring;
  A.ahead = s->ahead;
  A.dt = p.dt;
  A.cx = 0.016666666666667 * odx;
  A.cy = 0.05 * third * odth;
  A.cyy = 0.05 * third * third * odth * odth;
  A.cko = 0.1 * 0.0625 * odt;
  A.a2 = p.a * p.a;
  A.m4a = -4.0 * p.a;
  return A;
}

MixedArgs bhr::solver_mixed_args(bhr_solver *s) {
  const StageArgs A = solver_stage_args(s);
  MixedArgs X{};
  X.err = A.err;
  X.N = A.N;
  X.M = A.M;
  X.even_m = A.even_m;
  X.dt = static_cast<float>(A.dt);
  X.cx = static_cast<float>(A.cx);
  X.cy = static_cast<float>(A.cy);
  X.cyy = static_cast<float>(A.cyy);
  X.cko = static_cast<float>(A.cko);
  return X;
}

SourceArgs bhr::solver_source_args(bhr_solver *s) {
  const bhr_params &p = s->p;
  SourceArgs S{};
  S.src = s->src;
  S.recs = s->recs;
  S.rs = s->rs;
  S.r_c = s->rc;
  S.theta = s->th;
  S.N = p.N;
  S.M = p.M;
  S.PTSX = p.PTSX;
  S.PTSY = p.PTSY;
  S.lookahead = 0;
  S.nrecs = s->nt;
  S.a = p.a;
  S.mass = p.mass;
  S.m = p.m;
  S.wt = p.wt_fac * s->g.dtheta;
  return S;
}

ExtractArgs bhr::solver_extract_args(bhr_solver *s) {
  const bhr_params &p = s->p;
  ExtractArgs E{};
  E.u = s->u0;
  E.ext = s->ext;
  E.integ = s->integ;
  E.wproj = s->wproj;
  E.wdedt = s->wdedt;
  E.rows = s->rows;
  E.psirows = s->psirows;
  E.rs = s->rs;
  E.N = p.N;
  E.M = p.M;
  E.ext_col = s->ext_col;
  E.Fr = s->Fr;
  E.max_rows = s->max_rows;
  E.even_m = s->even_m ? 1 : 0;
  E.dt = p.dt;
  E.out_start = p.out_start;
  E.Xmax = p.Xmax;
  return E;
}

// One step.  On the side stream, beside stage 1, the particle source of the
// next step is built (into the patch buffer this step does not read; its
// record is selected by the stage step clock, which the previous step
// advanced), and beside stage 2 (RK4: stages 2-3) the previous step's
// extraction runs when it is pending: it reads only u^n, which the stages
// before the last only read, and its own accumulators.  The side branch
// joins before the final stage, which overwrites u^n; a one-thread kernel
// then advances the stage step clock.  This step's extraction is left
// pending (flush_extract launches it, or the next step).  `ev` (10 events):
// 0..5 on the main stream (1..4 around the stages, the final stage between
// 3 and 4), 6..7 around the extraction and 8..9 around the source on the
// side stream.
static int launch_step(bhr_solver *s, cudaEvent_t *ev = nullptr) {
  auto mark = [&](int i) { return ev ? cudaEventRecord(ev[i], s->stream) : cudaSuccess; };
  auto side_mark = [&](int i) { return ev ? cudaEventRecord(ev[i], s->side) : cudaSuccess; };
  BHR_CUDA_TRY(mark(0));
  if (s->has_source) {
    BHR_CUDA_TRY(cudaEventRecord(s->fork, s->stream));
    BHR_CUDA_TRY(cudaStreamWaitEvent(s->side, s->fork, 0));
    SourceArgs S = solver_source_args(s);
    S.lookahead = 1;
    BHR_CUDA_TRY(side_mark(8));
    BHR_CUDA_TRY(launch_source(S, s->side));
    BHR_CUDA_TRY(side_mark(9));
  }
  const bool extract = s->pending_extract;
  const bool side = extract || s->has_source;
  auto fork_extract = [&]() -> cudaError_t {
    if (!extract) return side ? cudaEventRecord(s->join, s->side) : cudaSuccess;
    cudaError_t e;
    if ((e = cudaEventRecord(s->fork2, s->stream)) || (e = cudaStreamWaitEvent(s->side, s->fork2, 0)) ||
        (e = side_mark(6)) || (e = launch_extract(solver_extract_args(s), s->side)) || (e = side_mark(7)))
      return e;
    return cudaEventRecord(s->join, s->side);
  };
  auto join = [&]() { return side ? cudaStreamWaitEvent(s->stream, s->join, 0) : cudaSuccess; };
  StageArgs A = solver_stage_args(s);
  BHR_CUDA_TRY(mark(1));
  A.vin = s->u0; A.un = s->u0; A.out = s->u1;
  if (s->mixed) {
    // u1 in FP64 and delta1 in FP32, then the FP32 stages 2 and 3.
    A.dout = s->d1f;
    BHR_CUDA_TRY(launch_stage(1, s->maps[0], A, s->stream));
    BHR_CUDA_TRY(mark(2));
    BHR_CUDA_TRY(fork_extract());
    MixedArgs X = solver_mixed_args(s);
    X.e_out = s->e2f;
    BHR_CUDA_TRY(launch_mixed_stage(2, s->mmaps[0], X, s->stream));
    BHR_CUDA_TRY(mark(3));
    BHR_CUDA_TRY(join());
    X.e_out = nullptr;
    X.u_out = s->u0;
    BHR_CUDA_TRY(launch_mixed_stage(3, s->mmaps[1], X, s->stream));
  } else if (s->rk4) {
    // Classical RK4, the step's source held fixed in all four stages:
    // y1 = u + dt/2 L(u); y2 = u + dt/2 L(y1), z = (y1 + 2 y2 - u)/3;
    // y3 = u + dt L(y2); u <- z + y3/3 + dt/6 L(y3).
    const double dt = A.dt;
    A.dt = 0.5 * dt;
    BHR_CUDA_TRY(launch_stage(1, s->maps[0], A, s->stream));
    BHR_CUDA_TRY(mark(2));
    BHR_CUDA_TRY(fork_extract());
    A.vin = s->u1; A.un = s->u0; A.out = s->u2; A.zout = s->u3;
    BHR_CUDA_TRY(launch_stage(4, s->maps[1], A, s->stream));
    A.vin = s->u2; A.un = s->u0; A.out = s->u1; A.zout = nullptr; A.dt = dt;
    BHR_CUDA_TRY(launch_stage(4, s->maps[3], A, s->stream));
    BHR_CUDA_TRY(mark(3));
    BHR_CUDA_TRY(join());
    A.vin = s->u1; A.un = s->u3; A.out = s->u0; A.dt = dt / 6.0;
    BHR_CUDA_TRY(launch_stage(5, s->maps[4], A, s->stream));
  } else if (s->strip12) {
    // Stages 1 and 2 in one launch (u1 stays on chip), beside the previous
    // step's extraction, which reads only u^n.
    BHR_CUDA_TRY(fork_extract());
    A.vin = s->u0; A.un = s->u0; A.out = s->u2;
    BHR_CUDA_TRY(launch_stage12_strip(s->smaps, A, s->stream));
    BHR_CUDA_TRY(mark(2));
    BHR_CUDA_TRY(mark(3));
    BHR_CUDA_TRY(join());
    A.vin = s->u2; A.un = s->u0; A.out = s->u0;
    BHR_CUDA_TRY(launch_stage(3, s->maps[2], A, s->stream));
  } else {
    BHR_CUDA_TRY(launch_stage(1, s->maps[0], A, s->stream));
    BHR_CUDA_TRY(mark(2));
    BHR_CUDA_TRY(fork_extract());
    A.vin = s->u1; A.un = s->u0; A.out = s->u2;
    BHR_CUDA_TRY(launch_stage(2, s->maps[1], A, s->stream));
    BHR_CUDA_TRY(mark(3));
    BHR_CUDA_TRY(join());
    A.vin = s->u2; A.un = s->u0; A.out = s->u0;
    BHR_CUDA_TRY(launch_stage(3, s->maps[2], A, s->stream));
  }
  BHR_CUDA_TRY(mark(4));
  BHR_CUDA_TRY(launch_step_clock(s->rs, s->stream));
  BHR_CUDA_TRY(mark(5));
  s->pending_extract = true;
  return BHR_OK;
}

// The last step's extraction, before anything reads the waveform, the
// extraction buffers or the run counters, or replaces the state.
static int flush_extract(bhr_solver *s) {
  if (!s->pending_extract) return BHR_OK;
  BHR_CUDA_TRY(launch_extract(solver_extract_args(s), s->stream));
  s->pending_extract = false;
  return BHR_OK;
}

static int check_run_state(bhr_solver *s) {
  RunState rs{};
  BHR_CUDA_TRY(cudaMemcpyAsync(&rs, s->rs, sizeof(rs), cudaMemcpyDeviceToHost, s->stream));
  BHR_CUDA_TRY(cudaStreamSynchronize(s->stream));
  if (rs.err == BHR_NAN_DETECTED) {
    set_error("non-finite value in the extracted waveform");
    return BHR_NAN_DETECTED;
  }
  if (rs.err == BHR_TIMEOUT) {
    set_error("a bounded device wait gave up");
    return BHR_TIMEOUT;
  }
  return BHR_OK;
}

// Captures `count` steps of launch_step into an executable graph.  Every
// launch argument is fixed per solve; what changes from step to step (the
// step clocks, the timer, the source record) is read on the device from
// RunState, so one captured graph replays any step.  A graph starts and ends
// with an extraction pending: it extracts the step before it and leaves its
// own last step's extraction to what follows.
static int capture_steps(bhr_solver *s, int count, cudaGraphExec_t *out) {
  cudaGraph_t g = nullptr;
  const bool pending = s->pending_extract;
  s->pending_extract = true;
  BHR_CUDA_TRY(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
  int st = BHR_OK;
  for (int i = 0; i < count && st == BHR_OK; i++) st = launch_step(s);
  cudaError_t e = cudaStreamEndCapture(s->stream, &g);
  s->pending_extract = pending;
  if (st != BHR_OK) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  if (e != cudaSuccess) {
    set_error(std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
    return BHR_CUDA_ERROR;
  }
  e = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    set_error(std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    return BHR_CUDA_ERROR;
  }
  return BHR_OK;
}

static int enqueue_steps(bhr_solver *s, int nsteps) {
  if (nsteps <= 0) return BHR_OK;
  if (!s->g1)
    if (int st = capture_steps(s, 1, &s->g1)) return st;
  if (nsteps >= kGraphBatch && !s->gb)
    if (int st = capture_steps(s, kGraphBatch, &s->gb)) return st;
  int left = nsteps;
  if (!s->pending_extract) {  // the graphs start with an extraction pending
    if (int st = launch_step(s)) return st;
    left--;
  }
  while (left >= kGraphBatch) {
    BHR_CUDA_TRY(cudaGraphLaunch(s->gb, s->stream));
    left -= kGraphBatch;
  }
  while (left-- > 0) BHR_CUDA_TRY(cudaGraphLaunch(s->g1, s->stream));
  s->steps_done += nsteps;
  return BHR_OK;
}

extern "C" {

int bhr_solver_step(bhr_solver *s, int nsteps) {
  NvtxRange range("bhr_solver_step");
  if (!s || nsteps < 0) return BHR_INVALID_ARG;
  BHR_CUDA_TRY(cudaSetDevice(s->p.device));
  if (s->steps_done + nsteps > s->nt && s->has_source) {
    set_error("stepping past the end of the trajectory records");
    return BHR_INVALID_ARG;
  }
  if (int st = solver_wait_records(s, s->steps_done + nsteps + 1)) return st;
  if (int st = enqueue_steps(s, nsteps)) return st;
  return check_run_state(s);
}

int bhr_solver_time_steps(bhr_solver *s, int nsteps, double *ms) {
  NvtxRange range("bhr_solver_time_steps");
  if (!s || nsteps < 0 || !ms) return BHR_INVALID_ARG;
  BHR_CUDA_TRY(cudaSetDevice(s->p.device));
  if (s->steps_done + nsteps > s->nt && s->has_source) {
    set_error("stepping past the end of the trajectory records");
    return BHR_INVALID_ARG;
  }
  if (int st = solver_wait_records(s, s->steps_done + nsteps + 1)) return st;
  if (!s->g1)
    if (int st = capture_steps(s, 1, &s->g1)) return st;
  if (nsteps >= kGraphBatch && !s->gb)
    if (int st = capture_steps(s, kGraphBatch, &s->gb)) return st;
  cudaEvent_t e0, e1;
  BHR_CUDA_TRY(cudaEventCreate(&e0));
  BHR_CUDA_TRY(cudaEventCreate(&e1));
  BHR_CUDA_TRY(cudaEventRecord(e0, s->stream));
  const int st = enqueue_steps(s, nsteps);
  BHR_CUDA_TRY(cudaEventRecord(e1, s->stream));
  BHR_CUDA_TRY(cudaEventSynchronize(e1));
  float f = 0.f;
  BHR_CUDA_TRY(cudaEventElapsedTime(&f, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = f;
  if (st) return st;
  return check_run_state(s);
}

int bhr_solver_waveform(bhr_solver *s, double *t, double *h, double *dedt, int max_rows, int *nrows) {
  if (!s) return BHR_INVALID_ARG;
  BHR_CUDA_TRY(cudaSetDevice(s->p.device));
  if (int st = flush_extract(s)) return st;
  RunState rs{};
  BHR_CUDA_TRY(cudaMemcpyAsync(&rs, s->rs, sizeof(rs), cudaMemcpyDeviceToHost, s->stream));
  BHR_CUDA_TRY(cudaStreamSynchronize(s->stream));
  const int n = std::min(rs.nrow, std::max(0, max_rows));
  std::vector<double> buf(static_cast<size_t>(n) * 16);
  if (n > 0) {
    BHR_CUDA_TRY(cudaMemcpyAsync(buf.data(), s->rows, buf.size() * 8, cudaMemcpyDeviceToHost, s->stream));
    BHR_CUDA_TRY(cudaStreamSynchronize(s->stream));
  }
  for (int r = 0; r < n; r++) {
    if (t) t[r] = buf[16 * r];
    if (h)
      for (int i = 0; i < 14; i++) h[14 * r + i] = buf[16 * r + 1 + i];
    if (dedt) dedt[r] = buf[16 * r + 15];
  }
  if (nrows) *nrows = n;
  return BHR_OK;
}

int bhr_solver_run(bhr_solver *s, const char *out_dir, const char *name) {
  NvtxRange range("bhr_solver_run");
  if (!s) return BHR_INVALID_ARG;
  const int remaining = s->nt - s->steps_done;
  const int chunk = 1000;
  for (int done = 0; done < remaining; done += chunk) {
    if (int st = bhr_solver_step(s, std::min(chunk, remaining - done))) return st;
  }
  if (int st = flush_extract(s)) return st;
  if (int st = check_run_state(s)) return st;
  if (!out_dir || !name) return BHR_OK;
  RunState rs{};
  BHR_CUDA_TRY(cudaMemcpyAsync(&rs, s->rs, sizeof(rs), cudaMemcpyDeviceToHost, s->stream));
  BHR_CUDA_TRY(cudaStreamSynchronize(s->stream));
  std::vector<double> t(rs.nrow), h(static_cast<size_t>(rs.nrow) * 14), e(rs.nrow);
  int n = 0;
  if (int st = bhr_solver_waveform(s, t.data(), h.data(), e.data(), rs.nrow, &n)) return st;
  return bhr_write_waveform(out_dir, name, s->p.m, t.data(), h.data(), e.data(), n);
}

int bhr_write_waveform(const char *out_dir, const char *name, double m, const double *t, const double *h,
                       const double *dedt, int nrows) {
  if (!out_dir || !name || nrows < 0 || (nrows > 0 && (!t || !h))) {
    set_error("bad waveform arguments");
    return BHR_INVALID_ARG;
  }
  // File naming as QNM_Extraction's loadwaveforms expects
  // (QNM_Extraction/Library/ringdownlib.py:49-84): hm<m>_ for m >= 0 and
  // hmm<|m|>_ for m < 0.
  const int mi = static_cast<int>(m);
  char fname[4096];
  std::snprintf(fname, sizeof(fname), "%s/%s%d_%s.dat", out_dir, mi < 0 ? "hmm" : "hm", std::abs(mi), name);
  FILE *f = std::fopen(fname, "w");
  std::string full = std::string(fname) + ".full";
  FILE *g = std::fopen(full.c_str(), "w");
  if (!f || !g) {
    if (f) std::fclose(f);
    if (g) std::fclose(g);
    set_error(std::string("cannot write ") + fname);
    return BHR_IO_ERROR;
  }
  for (int r = 0; r < nrows; r++) {
    // HighOrder/body.cu:208: "%lf" time then 14 "%g" values.
    std::fprintf(f, "%lf", t[r]);
    for (int i = 0; i < 14; i++) std::fprintf(f, " %g", h[14 * r + i]);
    std::fprintf(f, "\n");
    std::fprintf(g, "%.17g", t[r]);
    for (int i = 0; i < 14; i++) std::fprintf(g, " %.17g", h[14 * r + i]);
    std::fprintf(g, " %.17g\n", dedt ? dedt[r] : 0.0);
  }
  std::fclose(f);
  std::fclose(g);
  return BHR_OK;
}

int bhr_solver_get_state(bhr_solver *s, double *qre, double *qim, double *pre, double *pim) {
  if (!s) return BHR_INVALID_ARG;
  BHR_CUDA_TRY(cudaSetDevice(s->p.device));
  if (int st = flush_extract(s)) return st;
  const size_t NM = static_cast<size_t>(s->p.N) * s->p.M;
  BHR_CUDA_TRY(launch_closure(s->u0, s->p.N, s->p.M, s->even_m ? 1 : 0, s->stream));
  double *outs[4] = {qre, qim, pre, pim};
  for (int f = 0; f < 4; f++)
    if (outs[f]) BHR_CUDA_TRY(cudaMemcpyAsync(outs[f], s->u0 + f * NM, NM * 8, cudaMemcpyDeviceToHost, s->stream));
  BHR_CUDA_TRY(cudaStreamSynchronize(s->stream));
  return BHR_OK;
}

int bhr_solver_set_state(bhr_solver *s, const double *qre, const double *qim, const double *pre, const double *pim) {
  if (!s) return BHR_INVALID_ARG;
  BHR_CUDA_TRY(cudaSetDevice(s->p.device));
  if (int st = flush_extract(s)) return st;
  const size_t NM = static_cast<size_t>(s->p.N) * s->p.M;
  const double *ins[4] = {qre, qim, pre, pim};
  for (int f = 0; f < 4; f++) {
    if (ins[f]) BHR_CUDA_TRY(cudaMemcpyAsync(s->u0 + f * NM, ins[f], NM * 8, cudaMemcpyHostToDevice, s->stream));
    else BHR_CUDA_TRY(cudaMemsetAsync(s->u0 + f * NM, 0, NM * 8, s->stream));
  }
  BHR_CUDA_TRY(cudaStreamSynchronize(s->stream));
  return BHR_OK;
}

int bhr_solver_get_extraction(bhr_solver *s, double *psi_re, double *psi_im, double *int_re, double *int_im,
                              double *dint_re, double *dint_im) {
  if (!s) return BHR_INVALID_ARG;
  BHR_CUDA_TRY(cudaSetDevice(s->p.device));
  if (int st = flush_extract(s)) return st;
  const int M = s->p.M;
  std::vector<double> e(2 * M), in(4 * M);
  BHR_CUDA_TRY(cudaMemcpyAsync(e.data(), s->ext, e.size() * 8, cudaMemcpyDeviceToHost, s->stream));
  BHR_CUDA_TRY(cudaMemcpyAsync(in.data(), s->integ, in.size() * 8, cudaMemcpyDeviceToHost, s->stream));
  BHR_CUDA_TRY(cudaStreamSynchronize(s->stream));
  double *outs[6] = {psi_re, psi_im, int_re, int_im, dint_re, dint_im};
  const double *srcs[6] = {e.data(), e.data() + M, in.data(), in.data() + M, in.data() + 2 * M, in.data() + 3 * M};
  for (int i = 0; i < 6; i++)
    if (outs[i]) std::memcpy(outs[i], srcs[i], M * 8);
  return BHR_OK;
}

}  // extern "C"

namespace {
// Layout of a checkpoint: this header, then the four state planes (4 N M),
// ext (2 M), integ (4 M), nrow waveform rows (16 doubles each) and their
// psi samples (2 M each).
struct CheckpointHeader {
  char magic[8];  // "BHRCKPT1"
  int N, M, nt, max_rows, steps_done, has_source;
  RunState rs;
  double dt, a, m;
};
constexpr char kCkptMagic[8] = {'B', 'H', 'R', 'C', 'K', 'P', 'T', '1'};

size_t checkpoint_bytes(const bhr_solver *s, int nrow) {
  const size_t NM = static_cast<size_t>(s->p.N) * s->p.M;
  return sizeof(CheckpointHeader) +
         8 * (4 * NM + 6 * static_cast<size_t>(s->p.M) + (16 + 2 * static_cast<size_t>(s->p.M)) * nrow);
}
}  // namespace

extern "C" {

int bhr_solver_psi_samples(bhr_solver *s, double *psi_re, double *psi_im, int max_rows, int *nrows) {
  if (!s) return BHR_INVALID_ARG;
  BHR_CUDA_TRY(cudaSetDevice(s->p.device));
  if (int st = flush_extract(s)) return st;
  RunState rs{};
  BHR_CUDA_TRY(cudaMemcpyAsync(&rs, s->rs, sizeof(rs), cudaMemcpyDeviceToHost, s->stream));
  BHR_CUDA_TRY(cudaStreamSynchronize(s->stream));
  const int n = std::min(rs.nrow, std::max(0, max_rows));
  const size_t M = s->p.M;
  std::vector<double> buf(2 * M * static_cast<size_t>(n));
  if (n > 0) {
    BHR_CUDA_TRY(cudaMemcpyAsync(buf.data(), s->psirows, buf.size() * 8, cudaMemcpyDeviceToHost, s->stream));
    BHR_CUDA_TRY(cudaStreamSynchronize(s->stream));
  }
  for (int r = 0; r < n; r++) {
    if (psi_re) std::memcpy(psi_re + r * M, buf.data() + 2 * M * r, M * 8);
    if (psi_im) std::memcpy(psi_im + r * M, buf.data() + 2 * M * r + M, M * 8);
  }
  if (nrows) *nrows = n;
  return BHR_OK;
}

size_t bhr_solver_checkpoint_size(bhr_solver *s) {
  if (!s) return 0;
  cudaSetDevice(s->p.device);
  if (flush_extract(s)) return 0;
  RunState rs{};
  if (cudaMemcpyAsync(&rs, s->rs, sizeof(rs), cudaMemcpyDeviceToHost, s->stream) != cudaSuccess ||
      cudaStreamSynchronize(s->stream) != cudaSuccess)
    return 0;
  return checkpoint_bytes(s, rs.nrow);
}

int bhr_solver_checkpoint(bhr_solver *s, void *buf, size_t size) {
  NvtxRange range("bhr_solver_checkpoint");
  if (!s || !buf) return BHR_INVALID_ARG;
  BHR_CUDA_TRY(cudaSetDevice(s->p.device));
  if (int st = flush_extract(s)) return st;
  CheckpointHeader h{};
  std::memcpy(h.magic, kCkptMagic, sizeof(h.magic));
  BHR_CUDA_TRY(cudaMemcpyAsync(&h.rs, s->rs, sizeof(RunState), cudaMemcpyDeviceToHost, s->stream));
  BHR_CUDA_TRY(cudaStreamSynchronize(s->stream));
  if (size < checkpoint_bytes(s, h.rs.nrow)) {
    set_error("checkpoint buffer too small (bhr_solver_checkpoint_size gives the size)");
    return BHR_INVALID_ARG;
  }
  h.N = s->p.N;
  h.M = s->p.M;
  h.nt = s->nt;
  h.max_rows = s->max_rows;
  h.steps_done = s->steps_done;
  h.has_source = s->has_source ? 1 : 0;
  h.dt = s->p.dt;
  h.a = s->p.a;
  h.m = s->p.m;
  const size_t NM = static_cast<size_t>(s->p.N) * s->p.M, M = s->p.M;
  char *out = static_cast<char *>(buf);
  std::memcpy(out, &h, sizeof(h));
  double *d = reinterpret_cast<double *>(out + sizeof(h));
  BHR_CUDA_TRY(cudaMemcpyAsync(d, s->u0, 4 * NM * 8, cudaMemcpyDeviceToHost, s->stream));
  BHR_CUDA_TRY(cudaMemcpyAsync(d + 4 * NM, s->ext, 2 * M * 8, cudaMemcpyDeviceToHost, s->stream));
  BHR_CUDA_TRY(cudaMemcpyAsync(d + 4 * NM + 2 * M, s->integ, 4 * M * 8, cudaMemcpyDeviceToHost, s->stream));
  if (h.rs.nrow > 0) {
    BHR_CUDA_TRY(cudaMemcpyAsync(d + 4 * NM + 6 * M, s->rows, 16 * static_cast<size_t>(h.rs.nrow) * 8,
                                 cudaMemcpyDeviceToHost, s->stream));
    BHR_CUDA_TRY(cudaMemcpyAsync(d + 4 * NM + 6 * M + 16 * static_cast<size_t>(h.rs.nrow), s->psirows,
                                 2 * M * static_cast<size_t>(h.rs.nrow) * 8, cudaMemcpyDeviceToHost, s->stream));
  }
  BHR_CUDA_TRY(cudaStreamSynchronize(s->stream));
  return BHR_OK;
}

int bhr_solver_restore(bhr_solver *s, const void *buf, size_t size) {
  NvtxRange range("bhr_solver_restore");
  if (!s || !buf || size < sizeof(CheckpointHeader)) return BHR_INVALID_ARG;
  BHR_CUDA_TRY(cudaSetDevice(s->p.device));
  CheckpointHeader h;
  std::memcpy(&h, buf, sizeof(h));
  if (std::memcmp(h.magic, kCkptMagic, sizeof(h.magic)) != 0 || h.N != s->p.N || h.M != s->p.M || h.nt != s->nt ||
      h.max_rows != s->max_rows || h.dt != s->p.dt || h.a != s->p.a || h.m != s->p.m ||
      h.has_source != (s->has_source ? 1 : 0) || h.rs.nrow < 0 || h.rs.nrow > s->max_rows ||
      size < checkpoint_bytes(s, h.rs.nrow)) {
    set_error("checkpoint does not match this solve (grid, spin, m, dt, length or trajectory)");
    return BHR_INVALID_ARG;
  }
  if (int st = flush_extract(s)) return st;
  if (s->has_source)
    if (int st = solver_wait_records(s, h.rs.ks + 1)) return st;
  const size_t NM = static_cast<size_t>(s->p.N) * s->p.M, M = s->p.M;
  const double *d = reinterpret_cast<const double *>(static_cast<const char *>(buf) + sizeof(h));
  BHR_CUDA_TRY(cudaMemcpyAsync(s->u0, d, 4 * NM * 8, cudaMemcpyHostToDevice, s->stream));
  BHR_CUDA_TRY(cudaMemcpyAsync(s->ext, d + 4 * NM, 2 * M * 8, cudaMemcpyHostToDevice, s->stream));
  BHR_CUDA_TRY(cudaMemcpyAsync(s->integ, d + 4 * NM + 2 * M, 4 * M * 8, cudaMemcpyHostToDevice, s->stream));
  if (h.rs.nrow > 0) {
    BHR_CUDA_TRY(cudaMemcpyAsync(s->rows, d + 4 * NM + 6 * M, 16 * static_cast<size_t>(h.rs.nrow) * 8,
                                 cudaMemcpyHostToDevice, s->stream));
    BHR_CUDA_TRY(cudaMemcpyAsync(s->psirows, d + 4 * NM + 6 * M + 16 * static_cast<size_t>(h.rs.nrow),
                                 2 * M * static_cast<size_t>(h.rs.nrow) * 8, cudaMemcpyHostToDevice, s->stream));
  }
  BHR_CUDA_TRY(cudaMemcpyAsync(s->rs, &h.rs, sizeof(RunState), cudaMemcpyHostToDevice, s->stream));
  // The patch of the step the solve resumes at (later ones are built ahead).
  if (s->has_source) BHR_CUDA_TRY(launch_source(solver_source_args(s), s->stream));
  BHR_CUDA_TRY(cudaStreamSynchronize(s->stream));
  s->steps_done = h.steps_done;
  return BHR_OK;
}

int bhr_solver_get_source(bhr_solver *s, double *tre, double *tim) {
  if (!s || !tre || !tim) return BHR_INVALID_ARG;
  BHR_CUDA_TRY(cudaSetDevice(s->p.device));
  const bhr_params &p = s->p;
  const size_t NM = static_cast<size_t>(p.N) * p.M;
  std::memset(tre, 0, NM * 8);
  std::memset(tim, 0, NM * 8);
  if (!s->has_source) return BHR_OK;
  RunState rs{};
  BHR_CUDA_TRY(cudaMemcpyAsync(&rs, s->rs, sizeof(rs), cudaMemcpyDeviceToHost, s->stream));
  BHR_CUDA_TRY(cudaStreamSynchronize(s->stream));
  if (rs.ks <= 0) return BHR_OK;
  StepRec rec{};
  std::vector<double> patch(2 * static_cast<size_t>(p.PTSX) * p.PTSY);
  BHR_CUDA_TRY(cudaMemcpyAsync(&rec, s->recs + (rs.ks - 1), sizeof(rec), cudaMemcpyDeviceToHost, s->stream));
  BHR_CUDA_TRY(cudaMemcpyAsync(patch.data(), s->src + ((rs.ks - 1) & 1) * patch.size(), patch.size() * 8,
                               cudaMemcpyDeviceToHost, s->stream));
  BHR_CUDA_TRY(cudaStreamSynchronize(s->stream));
  for (int j = 0; j < p.PTSY; j++) {
    const int row = rec.row0 + j;
    if (row < 0 || row >= p.M) continue;
    for (int k = 0; k < p.PTSX; k++) {
      const int col = rec.col0 + k;
      if (col < 0 || col >= p.N) continue;
      tre[static_cast<size_t>(row) * p.N + col] = patch[static_cast<size_t>(j) * p.PTSX + k];
      tim[static_cast<size_t>(row) * p.N + col] = patch[static_cast<size_t>(p.PTSY + j) * p.PTSX + k];
    }
  }
  return BHR_OK;
}

void *bhr_solver_stream(bhr_solver *s) { return s ? static_cast<void *>(s->stream) : nullptr; }

int bhr_solver_profile(bhr_solver *s, int nsteps, double *avg_ms5, double *total_ms) {
  NvtxRange range("bhr_solver_profile");
  if (!s || nsteps <= 0) return BHR_INVALID_ARG;
  BHR_CUDA_TRY(cudaSetDevice(s->p.device));
  if (s->has_source && s->steps_done + nsteps > s->nt) {
    set_error("profiling past the end of the trajectory records");
    return BHR_INVALID_ARG;
  }
  if (int st = solver_wait_records(s, s->steps_done + nsteps + 1)) return st;
  // Events bracket each launch of launch_step; the extraction and the
  // source run on the side stream beside the stages.
  std::vector<cudaEvent_t> ev(10 * static_cast<size_t>(nsteps));
  for (auto &e : ev) BHR_CUDA_TRY(cudaEventCreate(&e));
  std::vector<char> had_extract(nsteps);
  double sums[5] = {0, 0, 0, 0, 0};
  int nextract = 0;
  cudaEvent_t t0, t1;
  BHR_CUDA_TRY(cudaEventCreate(&t0));
  BHR_CUDA_TRY(cudaEventCreate(&t1));
  BHR_CUDA_TRY(cudaEventRecord(t0, s->stream));
  for (int i = 0; i < nsteps; i++) {
    had_extract[i] = s->pending_extract;
    if (int st = launch_step(s, &ev[10 * static_cast<size_t>(i)])) return st;
    s->steps_done++;
  }
  BHR_CUDA_TRY(cudaEventRecord(t1, s->stream));
  BHR_CUDA_TRY(cudaStreamSynchronize(s->stream));
  BHR_CUDA_TRY(cudaStreamSynchronize(s->side));
  for (int i = 0; i < nsteps; i++) {
    cudaEvent_t *e = &ev[10 * static_cast<size_t>(i)];
    float ms = 0.f;
    if (s->has_source) {
      BHR_CUDA_TRY(cudaEventElapsedTime(&ms, e[8], e[9]));
      sums[0] += ms;
    }
    for (int j = 1; j < 4; j++) {
      BHR_CUDA_TRY(cudaEventElapsedTime(&ms, e[j], e[j + 1]));
      sums[j] += ms;
    }
    if (had_extract[i]) {
      BHR_CUDA_TRY(cudaEventElapsedTime(&ms, e[6], e[7]));
      sums[4] += ms;
      nextract++;
    }
  }
  float tot = 0.f;
  BHR_CUDA_TRY(cudaEventElapsedTime(&tot, t0, t1));
  for (auto &e : ev) cudaEventDestroy(e);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  if (avg_ms5) {
    for (int j = 0; j < 4; j++) avg_ms5[j] = sums[j] / nsteps;
    avg_ms5[4] = nextract ? sums[4] / nextract : 0.0;
  }
  if (total_ms) *total_ms = tot;
  return check_run_state(s);
}

}  // extern "C"
