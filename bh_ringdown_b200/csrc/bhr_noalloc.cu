// bhr_noalloc.cu -- source-free SSP-RK3 steps on a caller's state without
// allocating anything.
//
// Some callers cannot call cudaMalloc: a host framework that reserves the
// device memory up front and hands out pieces of it (a cudaMalloc from
// inside the solver would fail or break its budget), or a latency-critical
// loop where cudaMalloc's implicit device synchronisation is not allowed.
// bhr_step_noalloc serves them: the caller passes the state in device
// memory it already owns, and the two intermediate SSP-RK3 stages plus the
// coefficient tables live in one file-scope __device__ array of fixed size
// below (every GPU that loads the library holds it until the process
// exits).  The stage kernels are the same ones bhr_solver_step launches.
#include <cmath>
#include <cstring>
#include <mutex>

#include "bhr.h"
#include "bhr_host.h"
#include "bhr_internal.h"

namespace bhr {
namespace {

// Largest grid the fixed scratch holds.
constexpr int kNoAllocMaxPoints = 131072;  // N*M
constexpr int kNoAllocMaxN = 16384;
constexpr int kNoAllocMaxM = 1024;
constexpr size_t kStageDoubles = 4 * static_cast<size_t>(kNoAllocMaxPoints);
constexpr size_t kCoefOff = 2 * kStageDoubles;  // per-point coefficient plane bb
constexpr size_t kColOff = kCoefOff + static_cast<size_t>(kNoAllocMaxPoints);
constexpr size_t kRowOff = kColOff + static_cast<size_t>(CF_COUNT) * kNoAllocMaxN;
constexpr size_t kFlagOff = kRowOff + static_cast<size_t>(RF_COUNT) * kNoAllocMaxM;
constexpr size_t kScratchDoubles = kFlagOff + 32;  // about 11.2 MB in all

// Scratch: [u1 | u2 | coefficient plane bb | column tables | row tables | error flag].  In host code
// this name is only a stand-in for the device symbol; the device address
// comes from cudaGetSymbolAddress below.
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;

// What one device's scratch holds: the parameters its tables were built
// for and the tensor maps over the last state it stepped.  Rebuilding the
// grid (a Newton solve per column) and the tables costs host time on every
// call, so a call with the same parameters and state reuses them.
struct DeviceScratch {
  double *base = nullptr;  // device address of g_noalloc_scratch on this device
  bool tables_valid = false;
  int N = 0, M = 0;
  double Xmin = 0, Xmax = 0, mass = 0, a = 0, m = 0, dt = 0;
  double *state = nullptr;
  StageMaps maps[3];
};

std::mutex g_mu;
DeviceScratch g_dev[kMaxDevices];
// Host staging for the grid and the tables (fixed size, no heap).
double h_x[kNoAllocMaxN], h_r[kNoAllocMaxN], h_tx[kNoAllocMaxN], h_th[kNoAllocMaxM];
double h_col[CF_COUNT * kNoAllocMaxN], h_row[RF_COUNT * kNoAllocMaxM];

int fail(int status, const char *msg) {
  set_error(msg);
  return status;
}

// Restores the calling thread's current device on every return path.
struct DeviceGuard {
  int prev = -1;
  DeviceGuard() {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

bool same_tables(const DeviceScratch &d, const bhr_params &p) {
  return d.tables_valid && d.N == p.N && d.M == p.M && d.Xmin == p.Xmin && d.Xmax == p.Xmax && d.mass == p.mass &&
         d.a == p.a && d.m == p.m && d.dt == p.dt;
}

}  // namespace
}  // namespace bhr

using namespace bhr;

extern "C" int bhr_step_noalloc(const bhr_params *p, double *state, int nsteps, void *stream) {
  if (!p || !state || nsteps < 0) return fail(BHR_INVALID_ARG, "bhr_step_noalloc: null argument or nsteps < 0");
  if (p->N < 64 || p->N % TC != 0 || p->M < 16 || p->M % TR != 0)
    return fail(BHR_INVALID_ARG, "bhr_step_noalloc: N must be a multiple of 64 and M a multiple of 16 (>= 16)");
  if (static_cast<long long>(p->N) * p->M > kNoAllocMaxPoints || p->N > kNoAllocMaxN || p->M > kNoAllocMaxM)
    return fail(BHR_INVALID_ARG,
                "bhr_step_noalloc: grid larger than the fixed scratch (N*M <= 131072, N <= 16384, M <= 1024)");
  if (!(p->Xmax > p->Xmin) || !(p->mass > 0.0) || !(std::fabs(p->a) < p->mass) || !(p->dt > 0.0) ||
      p->m != std::floor(p->m) || p->precision != BHR_FP64 || p->integrator != BHR_SSPRK3)
    return fail(BHR_INVALID_ARG, "bhr_step_noalloc: need Xmax > Xmin, |a| < mass, dt > 0, integer m, FP64 SSP-RK3");
  if (p->device < 0 || p->device >= kMaxDevices) return fail(BHR_INVALID_ARG, "bhr_step_noalloc: bad device");
  if (reinterpret_cast<uintptr_t>(state) % 16 != 0)
    return fail(BHR_INVALID_ARG, "bhr_step_noalloc: state must be 16-byte aligned");

  std::lock_guard<std::mutex> lock(g_mu);
  DeviceGuard guard;
  if (cudaSetDevice(p->device) != cudaSuccess) return fail(BHR_CUDA_ERROR, "bhr_step_noalloc: cudaSetDevice failed");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (st != nullptr) {
    int sdev = -1;
    if (cudaStreamGetDevice(st, &sdev) != cudaSuccess)
      return fail(BHR_INVALID_ARG, "bhr_step_noalloc: the stream is not a valid CUDA stream");
    if (sdev != p->device) return fail(BHR_INVALID_ARG, "bhr_step_noalloc: the stream belongs to another device");
  }
  DeviceScratch &D = g_dev[p->device];
  // Set-up, once per device, with that device current.
  if (!D.base) {
    double *ptr = nullptr;
    if (cudaGetSymbolAddress(reinterpret_cast<void **>(&ptr), g_noalloc_scratch) != cudaSuccess || !ptr)
      return fail(BHR_CUDA_ERROR, "bhr_step_noalloc: cudaGetSymbolAddress of the scratch failed");
    if (prepare_kernels() != cudaSuccess)
      return fail(BHR_CUDA_ERROR, "bhr_step_noalloc: setting the stage kernels' shared-memory size failed");
    D.base = ptr;
  }
  double *scr = D.base;
  double *u1 = scr, *u2 = scr + kStageDoubles;
  double *coltab = scr + kColOff, *rowtab = scr + kRowOff, *ctab = scr + kCoefOff;
  int *flag = reinterpret_cast<int *>(scr + kFlagOff);

  const int N = p->N, M = p->M;
  const double dx = (p->Xmax - p->Xmin) / N, dth = kPiParm / M;
  const bool rebuild = !same_tables(D, *p);
  if (rebuild || D.state != state) {
    for (int i = 0; i < 3; i++) {
      double *bufs[3] = {state, u1, u2};
      StageMaps &mp = D.maps[i];
      CUtensorMap unused_q, unused_p;
      if (encode_state_maps(state, N, M, TR, &unused_q, &unused_p, &mp.u) != cudaSuccess ||
          encode_state_maps(bufs[(i + 1) % 3], N, M, TR, &unused_q, &unused_p, &mp.o) != cudaSuccess ||
          encode_state_maps(bufs[i], N, M, TR, &mp.q, &mp.p, nullptr) != cudaSuccess ||
          encode_coef_maps(ctab, coltab, rowtab, N, M, TR, &mp) != cudaSuccess) {
        D.state = nullptr;
        return fail(BHR_CUDA_ERROR, "bhr_step_noalloc: cuTensorMapEncodeTiled failed");
      }
    }
    D.state = state;
  }
  if (rebuild) {
    // The tables are rewritten while no kernel of an earlier call may still
    // read them: every call ends with its stream drained.
    D.tables_valid = false;
    double r_plus = 0.0, r_minus = 0.0;
    fill_grid(*p, h_x, h_r, h_th, h_tx, &r_plus, &r_minus);
    fill_tables(*p, dx, h_r, h_th, h_col, h_row);
    if (cudaMemcpyAsync(coltab, h_col, sizeof(double) * CF_COUNT * N, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(rowtab, h_row, sizeof(double) * RF_COUNT * M, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        launch_coef_tables(coltab, rowtab, ctab, N, M, st) != cudaSuccess) {
      cudaStreamSynchronize(st);
      return fail(BHR_CUDA_ERROR, "bhr_step_noalloc: table upload failed");
    }
    D.N = N;
    D.M = M;
    D.Xmin = p->Xmin;
    D.Xmax = p->Xmax;
    D.mass = p->mass;
    D.a = p->a;
    D.m = p->m;
    D.dt = p->dt;
    D.tables_valid = true;
  }
  // The flag must start at zero on every call.
  if (cudaMemsetAsync(flag, 0, sizeof(int), st) != cudaSuccess) {
    cudaStreamSynchronize(st);
    return fail(BHR_CUDA_ERROR, "bhr_step_noalloc: clearing the error flag failed");
  }

  const double third = 0.33333333333333333;
  StageArgs A{};
  A.ahead = -1;  // the default L2 prefetch distance
  A.coltab = coltab;
  A.rowtab = rowtab;
  A.src = nullptr;
  A.recs = nullptr;
  A.rs = nullptr;
  A.err = flag;
  A.N = N;
  A.M = M;
  A.PTSX = p->PTSX;
  A.PTSY = p->PTSY;
  A.even_m = (static_cast<int>(p->m) % 2) == 0 ? 1 : 0;
  A.rows = TR;
  A.dt = p->dt;
  A.cx = 0.016666666666667 * (1.0 / dx);
  A.cy = 0.05 * third * (1.0 / dth);
  A.cyy = 0.05 * third * third * (1.0 / dth) * (1.0 / dth);
  A.cko = 0.1 * 0.0625 * (1.0 / p->dt);
  A.a2 = p->a * p->a;
  A.m4a = -4.0 * p->a;
  // The stage kernels request the coefficient tiles before their grid-
  // dependency wait, so the first one of the call is launched without
  // programmatic serialisation: it starts after the table build and the
  // flag reset have completed.  The later ones overlap as in the solver.
  const char *failed = nullptr;
  for (int k = 0; k < nsteps && !failed; k++) {
    A.vin = state; A.un = state; A.out = u1;
    if (launch_stage(1, D.maps[0], A, st, /*pdl=*/k > 0) != cudaSuccess) { failed = "stage 1 launch failed"; break; }
    A.vin = u1; A.un = state; A.out = u2;
    if (launch_stage(2, D.maps[1], A, st) != cudaSuccess) { failed = "stage 2 launch failed"; break; }
    A.vin = u2; A.un = state; A.out = state;
    if (launch_stage(3, D.maps[2], A, st) != cudaSuccess) { failed = "stage 3 launch failed"; break; }
  }
  if (!failed && launch_closure(state, N, M, A.even_m, st) != cudaSuccess) failed = "closure launch failed";
  if (failed) {
    // Let what was launched finish before the lock is released: a later
    // call may rewrite the tables these kernels read.
    cudaStreamSynchronize(st);
    cudaGetLastError();
    return fail(BHR_CUDA_ERROR, failed);
  }
  int h_flag = 0;
  const cudaError_t e1 = cudaMemcpyAsync(&h_flag, flag, sizeof(int), cudaMemcpyDeviceToHost, st);
  const cudaError_t e2 = cudaStreamSynchronize(st);
  if (e1 != cudaSuccess || e2 != cudaSuccess) {
    D.tables_valid = false;
    return fail(BHR_CUDA_ERROR, "bhr_step_noalloc: stream failed");
  }
  if (h_flag == BHR_TIMEOUT) return fail(BHR_TIMEOUT, "bhr_step_noalloc: a bounded device wait gave up");
  return BHR_OK;
}
