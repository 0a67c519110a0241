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
std::mutex g_mu;
double *g_scratch[kMaxDevices] = {nullptr};
// Host staging for the grid and the tables (fixed size, no heap).
double h_x[kNoAllocMaxN], h_r[kNoAllocMaxN], h_tx[kNoAllocMaxN], h_th[kNoAllocMaxM];
double h_col[CF_COUNT * kNoAllocMaxN], h_row[RF_COUNT * kNoAllocMaxM];

int fail(int status, const char *msg) {
  set_error(msg);
  return status;
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

  std::lock_guard<std::mutex> lock(g_mu);
  if (cudaSetDevice(p->device) != cudaSuccess) return fail(BHR_CUDA_ERROR, "bhr_step_noalloc: cudaSetDevice failed");
  // Set-up, once per device, with that device current.
  if (!g_scratch[p->device]) {
    double *ptr = nullptr;
    if (cudaGetSymbolAddress(reinterpret_cast<void **>(&ptr), g_noalloc_scratch) != cudaSuccess || !ptr)
      return fail(BHR_CUDA_ERROR, "bhr_step_noalloc: cudaGetSymbolAddress of the scratch failed");
    if (prepare_kernels() != cudaSuccess)
      return fail(BHR_CUDA_ERROR, "bhr_step_noalloc: setting the stage kernels' shared-memory size failed");
    g_scratch[p->device] = ptr;
  }
  double *scr = g_scratch[p->device];
  double *u1 = scr, *u2 = scr + kStageDoubles;
  double *coltab = scr + kColOff, *rowtab = scr + kRowOff, *ctab = scr + kCoefOff;
  int *flag = reinterpret_cast<int *>(scr + kFlagOff);
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  const int N = p->N, M = p->M;
  double r_plus = 0.0, r_minus = 0.0;
  fill_grid(*p, h_x, h_r, h_th, h_tx, &r_plus, &r_minus);
  const double dx = (p->Xmax - p->Xmin) / N, dth = kPiParm / M;
  fill_tables(*p, dx, h_r, h_th, h_col, h_row);

  StageMaps maps[3];
  double *bufs[3] = {state, u1, u2};
  for (int i = 0; i < 3; i++) {
    CUtensorMap unused_q, unused_p;
    if (encode_state_maps(state, N, M, TR, &unused_q, &unused_p, &maps[i].u) != cudaSuccess ||
        encode_state_maps(bufs[(i + 1) % 3], N, M, TR, &unused_q, &unused_p, &maps[i].o) != cudaSuccess ||
        encode_state_maps(bufs[i], N, M, TR, &maps[i].q, &maps[i].p, nullptr) != cudaSuccess ||
        encode_coef_maps(ctab, coltab, rowtab, N, M, TR, &maps[i]) != cudaSuccess)
      return fail(BHR_CUDA_ERROR, "bhr_step_noalloc: cuTensorMapEncodeTiled failed (state must be 16-byte aligned)");
  }
  // The tables must be current for this call; the flag must start at zero.
  if (cudaMemcpyAsync(coltab, h_col, sizeof(double) * CF_COUNT * N, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(rowtab, h_row, sizeof(double) * RF_COUNT * M, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemsetAsync(flag, 0, sizeof(int), st) != cudaSuccess ||
      launch_coef_tables(coltab, rowtab, ctab, N, M, st) != cudaSuccess)
    return fail(BHR_CUDA_ERROR, "bhr_step_noalloc: table upload failed");

  const double third = 0.33333333333333333;
  StageArgs A{};
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
  for (int k = 0; k < nsteps; k++) {
    A.vin = state; A.un = state; A.out = u1;
    if (launch_stage(1, maps[0], A, st) != cudaSuccess) return fail(BHR_CUDA_ERROR, "stage 1 launch failed");
    A.vin = u1; A.un = state; A.out = u2;
    if (launch_stage(2, maps[1], A, st) != cudaSuccess) return fail(BHR_CUDA_ERROR, "stage 2 launch failed");
    A.vin = u2; A.un = state; A.out = state;
    if (launch_stage(3, maps[2], A, st) != cudaSuccess) return fail(BHR_CUDA_ERROR, "stage 3 launch failed");
  }
  if (launch_closure(state, N, M, A.even_m, st) != cudaSuccess) return fail(BHR_CUDA_ERROR, "closure launch failed");
  int h_flag = 0;
  if (cudaMemcpyAsync(&h_flag, flag, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return fail(BHR_CUDA_ERROR, "bhr_step_noalloc: stream failed");
  if (h_flag == BHR_TIMEOUT) return fail(BHR_TIMEOUT, "bhr_step_noalloc: a bounded device wait gave up");
  return BHR_OK;
}
