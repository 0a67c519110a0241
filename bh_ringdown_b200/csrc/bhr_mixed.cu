// bhr_mixed.cu -- FP32 stages 2 and 3 of the mixed-precision (BHR_MIXED)
// SSP-RK3 step.
//
// Stage 1 is the FP64 stage kernel, which also stores delta1 = dt L(u^n) in
// FP32.  These kernels apply the homogeneous operator L0 (the right-hand
// side of HighOrder/kern.cu:171-299 without the source) in FP32 to fields of
// size O(dt |u|) and O(dt^2 |u|):
//   stage 2: eps2 = dt/4 L0(delta1)
//   stage 3: u^{n+1} = u1 + (double)(2 eps2 + 2/3 dt L0(eps2))
// The stencils are written on differences (f[+k] - f[0]) + (f[-k] - f[0]),
// which are exact or nearly so in FP32 for smooth fields, instead of on
// the raw values, whose sum cancels by three orders of magnitude in the
// 6th-order second derivative and the Kreiss-Oliger term.  Tiles are 64
// columns by 16 rows, one per block, loaded by TMA into shared memory with
// the closure rebuilt there, as in the FP64 kernels.
#include "bhr_device.cuh"
#include "bhr_internal.h"

#include <cudaTypedefs.h>

#include <cstddef>
#include <type_traits>

namespace bhr {
namespace {

constexpr int kMixRows = kMixTileRows;
constexpr int kMixThreads = 256;
// Blocks per SM: stage 2 fits in 64 registers a thread and ~50 KB of shared
// memory, so four; stage 3 (80 registers, its FP64 u1 tile: ~74 KB) three.
template <int STAGE>
constexpr int mix_blocks_per_sm() {
  return STAGE == 2 ? 4 : 3;
}

// Every TMA destination starts on a 128-byte boundary.
template <int STAGE>
struct __align__(128) MixSmem {
  alignas(128) float q[2][kMixRows + 6][WC];  // TMA box {WC, 22, 2}: q_re, q_im of the input with halo
  alignas(128) float p[2][kMixRows][WC];      // TMA box {WC, 16, 2}: p_re, p_im with column halo
  alignas(128) float kc[4][kMixRows][TC];     // TMA box {TC, 16, 4}: bb, ee, d_re, d_im formed in FP64 at set-up
  alignas(128) float cf[CF_COUNT][TC];        // TMA box {TC, CF_COUNT}
  alignas(128) float rf[RF_COUNT][kMixRows];  // TMA box {16, RF_COUNT}
  alignas(128) double u1[STAGE == 3 ? 4 : 1][kMixRows][TC];  // stage 3: TMA box {TC, 16, 4}
  uint64_t bar;
};
#define BHR_TMA_ALIGNED(T, m) static_assert(offsetof(T, m) % 128 == 0, "TMA destination " #m " not 128-byte aligned")
BHR_TMA_ALIGNED(MixSmem<2>, q);
BHR_TMA_ALIGNED(MixSmem<2>, p);
BHR_TMA_ALIGNED(MixSmem<2>, kc);
BHR_TMA_ALIGNED(MixSmem<2>, cf);
BHR_TMA_ALIGNED(MixSmem<2>, rf);
BHR_TMA_ALIGNED(MixSmem<3>, q);
BHR_TMA_ALIGNED(MixSmem<3>, p);
BHR_TMA_ALIGNED(MixSmem<3>, kc);
BHR_TMA_ALIGNED(MixSmem<3>, cf);
BHR_TMA_ALIGNED(MixSmem<3>, rf);
BHR_TMA_ALIGNED(MixSmem<3>, u1);

__device__ __forceinline__ float d1f(const float *v, int c) {
  return 45.0f * (v[c + 1] - v[c - 1]) - 9.0f * (v[c + 2] - v[c - 2]) + (v[c + 3] - v[c - 3]);
}
// (f[c+k] - f[c]) + (f[c-k] - f[c])
__device__ __forceinline__ float skf(const float *v, int c, int k) { return (v[c + k] - v[c]) + (v[c - k] - v[c]); }
// Kreiss-Oliger sum (f4 - 8 f3 + 28 f2 - 56 f1 + 70 f0 over both sides) on differences.
__device__ __forceinline__ float ko8f(const float *v, int c) {
  return skf(v, c, 4) - 8.0f * skf(v, c, 3) + 28.0f * skf(v, c, 2) - 56.0f * skf(v, c, 1);
}

// Single solve: the tile `n` places after this block's in launch order
// (n = 0: none).
struct MixGridAhead {
  const MixedMaps *T;
  int n;
  __device__ __forceinline__ bool operator()(const MixedMaps *&pm, int &c0, int &b0) const {
    const int L = blockIdx.y * gridDim.x + blockIdx.x + n;
    if (n <= 0 || L >= static_cast<int>(gridDim.x * gridDim.y)) return false;
    pm = T;
    c0 = (L % gridDim.x) * TC;
    b0 = (L / gridDim.x) * kMixRows;
    return true;
  }
};
// Batch: the work item `n` places later in the launch group.
template <int STAGE>
struct MixGroupAhead {
  const MixedBatch *solves;
  const MixedGroup *G;
  int n;
  __device__ __forceinline__ bool operator()(const MixedMaps *&pm, int &c0, int &b0) const {
    const int L = blockIdx.x + n;
    if (n <= 0 || L >= G->ntiles) return false;
    pm = &solves[G->solve[group_item(*G, L, kMixRows, c0, b0)]].maps[STAGE - 2];
    return true;
  }
};
// One 64 x 16 tile (columns c0.., rows b0..) of stage 2 or 3.  Thread 0
// prefetches into L2 the input of the later tile `ahead` names, so that the
// block which takes it finds its loads there.
template <int STAGE, class Ahead>
__device__ __forceinline__ void mixed_tile(const MixedMaps &T, const MixedArgs &A, const int c0, const int b0,
                                           const Ahead ahead) {
  constexpr int ROWS = kMixRows, RPT = ROWS / (kMixThreads / 32);
  extern __shared__ unsigned char smem_raw[];
  MixSmem<STAGE> &S = *reinterpret_cast<MixSmem<STAGE> *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~static_cast<uintptr_t>(127));
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
  const int N = A.N, M = A.M;
  const size_t NM = static_cast<size_t>(N) * M;

  if (tid == 0) {
    mbar_init(&S.bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  if (tid == 0) {
    const uint32_t bytes = static_cast<uint32_t>(sizeof(S.q) + sizeof(S.p) + sizeof(S.kc) + sizeof(S.cf) +
                                                 sizeof(S.rf) + (STAGE == 3 ? sizeof(S.u1) : 0));
    mbar_expect_tx(&S.bar, bytes);
    tma_load_3d(&S.kc[0][0][0], &T.bb, c0, b0, 0, &S.bar);
    tma_load_2d(&S.cf[0][0], &T.colf, c0, 0, &S.bar);
    tma_load_2d(&S.rf[0][0], &T.rowf, b0, 0, &S.bar);
  }
  grid_dependency_wait();
  launch_dependents();
  if (tid == 0) {
    tma_load_3d(&S.q[0][0][0], &T.q, c0 - 4, b0 - 3, 0, &S.bar);
    tma_load_3d(&S.p[0][0][0], &T.p, c0 - 4, b0, 2, &S.bar);
    if (STAGE == 3) tma_load_3d(&S.u1[0][0][0], &T.u1, c0, b0, 0, &S.bar);
    const MixedMaps *pm;
    int pc0, pb0;
    if (ahead(pm, pc0, pb0)) {
      tma_prefetch_3d(&pm->q, pc0 - 4, pb0 - 3, 0);
      tma_prefetch_3d(&pm->p, pc0 - 4, pb0, 2);
      tma_prefetch_3d(&pm->bb, pc0, pb0, 0);
      if (STAGE == 3) tma_prefetch_3d(&pm->u1, pc0, pb0, 0);
    }
  }
  const bool ok = mbar_wait_bounded(&S.bar, 0);
  if (!__syncthreads_and(ok)) {
    if (tid == 0) atomicCAS(A.err, 0, 5 /* BHR_TIMEOUT */);
    mbar_wait_bounded(&S.bar, 0);
    return;
  }

  // Closure of the input (linear, so the same extrapolation as for u):
  // poles on q (HighOrder/kern.cu:320-409), radial ends on all planes
  // (HighOrder/kern.cu:412-449).
  const float third = static_cast<float>(kThird);
  const bool lo_rows = (b0 == 0), hi_rows = (b0 + ROWS + 3 > M - 3);
  if (lo_rows || hi_rows) {
    for (int i = tid; i < 2 * WC; i += kMixThreads) {
      const int pl = i / WC, w = i - pl * WC;
      const int a = c0 - 4 + w;
      if (a < 3 || a >= N - 3) continue;
      float(*q)[WC] = S.q[pl];
      const int o = 3 - b0;
      if (lo_rows) {
        if (A.even_m) {
          q[2 + o][w] = (4.0f * q[3 + o][w] - q[4 + o][w]) * third;
          q[1 + o][w] = (4.0f * q[2 + o][w] - q[3 + o][w]) * third;
          q[0 + o][w] = (4.0f * q[1 + o][w] - q[2 + o][w]) * third;
        } else {
          q[2 + o][w] = 0.0f; q[1 + o][w] = 0.0f; q[0 + o][w] = 0.0f;
        }
      }
      if (hi_rows) {
        if (A.even_m) {
          q[M - 3 + o][w] = (4.0f * q[M - 4 + o][w] - q[M - 5 + o][w]) * third;
          q[M - 2 + o][w] = (4.0f * q[M - 3 + o][w] - q[M - 4 + o][w]) * third;
          q[M - 1 + o][w] = (4.0f * q[M - 2 + o][w] - q[M - 3 + o][w]) * third;
        } else {
          q[M - 3 + o][w] = 0.0f; q[M - 2 + o][w] = 0.0f; q[M - 1 + o][w] = 0.0f;
        }
      }
    }
  }
  const bool lo_cols = (c0 == 0), hi_cols = (c0 + TC + 4 > N - 3);
  if (lo_cols || hi_cols) {
    for (int i = tid; i < 4 * ROWS; i += kMixThreads) {
      const int pl = i / ROWS, r = i - pl * ROWS;
      const int b = b0 + r;
      if (b < 3 || b >= M - 3) continue;
      float *row = pl < 2 ? &S.q[pl][r + 3][0] : &S.p[pl - 2][r][0];
      const int o = 4 - c0;
      if (lo_cols) {
        row[2 + o] = (4.0f * row[3 + o] - row[4 + o]) * third;
        row[1 + o] = (4.0f * row[2 + o] - row[3 + o]) * third;
        row[0 + o] = (4.0f * row[1 + o] - row[2 + o]) * third;
      }
      if (hi_cols) {
        row[N - 3 + o] = (4.0f * row[N - 4 + o] - row[N - 5 + o]) * third;
        row[N - 2 + o] = (4.0f * row[N - 3 + o] - row[N - 4 + o]) * third;
        row[N - 1 + o] = (4.0f * row[N - 2 + o] - row[N - 3 + o]) * third;
      }
    }
  }
  __syncthreads();

  const int a0 = c0 + 2 * tx;
  const int w0 = 2 * tx + 4;
  const float dt = A.dt;
  auto rows = [&](auto inner_tag) {
    constexpr bool inner = decltype(inner_tag)::value;
#pragma unroll 1
    for (int rr = 0; rr < RPT; rr++) {
      const int r = RPT * ty + rr;
      const int b = b0 + r;
      if (b < 3 || b >= M - 3) continue;
      if (!inner && (a0 + 1 < 3 || a0 >= N - 3)) continue;

      // Theta derivatives of q.
      const float ctan_cy = S.rf[RF_CTAN][r] * A.cy;
      float ll[2][2];
#pragma unroll
      for (int pl = 0; pl < 2; pl++) {
        float f[7][2];
#pragma unroll
        for (int j = 0; j < 7; j++) {
          const float2 t = *reinterpret_cast<const float2 *>(&S.q[pl][r + j][w0]);
          f[j][0] = t.x;
          f[j][1] = t.y;
        }
#pragma unroll
        for (int c = 0; c < 2; c++) {
          const float y1 = (f[6][c] - f[0][c]) - 9.0f * (f[5][c] - f[1][c]) + 45.0f * (f[4][c] - f[2][c]);
          const float s1 = (f[4][c] - f[3][c]) + (f[2][c] - f[3][c]);
          const float s2 = (f[5][c] - f[3][c]) + (f[1][c] - f[3][c]);
          const float s3 = (f[6][c] - f[3][c]) + (f[0][c] - f[3][c]);
          const float y2 = 2.0f * s3 - 27.0f * s2 + 270.0f * s1;
          ll[pl][c] = y2 * A.cyy + ctan_cy * y1;
        }
      }

      // Coefficients (HighOrder/kern.cu:132-158, 192-197): bb, ee, d_re and
      // d_im, whose formulas cancel, were formed in FP64 at set-up; the
      // others are products of column and row factors, formed here in FP32.
      const float cs = S.rf[RF_COS][r], gth = S.rf[RF_G][r], s2r = S.rf[RF_S2][r];
      float kbb[2], kee[2], kdre[2], kdim[2], kare[2], kaim[2], kvre[2], kvim[2];
      float res[4][2];
#pragma unroll
      for (int c = 0; c < 2; c++) {
        const int w = 2 * tx + c;
        const float ib = 1.0f / fmaf(S.cf[CF_B1][w], s2r, S.cf[CF_B0][w]);
        const float cc = S.cf[CF_CCN][w] * ib;
        const float btr = S.cf[CF_XR][w] * ib;
        const float bti = (S.cf[CF_BI0][w] + S.cf[CF_BI1][w] * cs) * ib;
        kbb[c] = S.kc[0][r][w];
        kee[c] = S.kc[1][r][w];
        kdre[c] = S.kc[2][r][w];
        kdim[c] = S.kc[3][r][w];
        kvre[c] = -(S.cf[CF_CR0][w] + S.cf[CF_CR1][w] * gth) * ib;
        kvim[c] = -S.cf[CF_CIN][w] * ib;
        kare[c] = -btr;
        kaim[c] = -bti;
        res[0][c] = 0.0f;
        res[1][c] = 0.0f;
        res[2][c] = cc * ll[0][c];
        res[3][c] = cc * ll[1][c];
      }

      // Radial derivatives, dissipation and the right-hand side, plane by plane.
      float fc[4][2];
#pragma unroll
      for (int pl = 0; pl < 4; pl++) {
        const float *row = pl < 2 ? &S.q[pl][r + 3][0] : &S.p[pl - 2][r][0];
        float v[10];
#pragma unroll
        for (int j = 0; j < 5; j++) {
          const float2 t = *reinterpret_cast<const float2 *>(row + w0 - 4 + 2 * j);
          v[2 * j] = t.x;
          v[2 * j + 1] = t.y;
        }
#pragma unroll
        for (int c = 0; c < 2; c++) {
          const int a = a0 + c;
          const float f0 = v[4 + c];
          const float fx = d1f(v, 4 + c) * A.cx;
          const float fk = (inner || (a >= 4 && a < N - 4)) ? ko8f(v, 4 + c) * A.cko : 0.0f;
          fc[pl][c] = f0;
          if (pl == 0) {
            res[0][c] += fmaf(-kbb[c], fx, -fk);
            res[2][c] += fmaf(kdre[c], fx, -kvre[c] * f0);
            res[3][c] += fmaf(kdim[c], fx, -kvim[c] * f0);
          } else if (pl == 1) {
            res[1][c] += fmaf(-kbb[c], fx, -fk);
            res[2][c] += fmaf(-kdim[c], fx, kvim[c] * f0);
            res[3][c] += fmaf(kdre[c], fx, -kvre[c] * f0);
          } else if (pl == 2) {
            res[0][c] += f0;
            res[2][c] += fmaf(kee[c], fx, fmaf(-kare[c], f0, -fk));
            res[3][c] += -kaim[c] * f0;
          } else {
            res[1][c] += f0;
            res[2][c] += kaim[c] * f0;
            res[3][c] += fmaf(kee[c], fx, fmaf(-kare[c], f0, -fk));
          }
        }
      }

      const size_t base = static_cast<size_t>(b) * N + a0;
      const bool both = inner || ((a0 >= 3) && (a0 + 1 < N - 3));
      const bool ok0 = inner || (a0 >= 3 && a0 < N - 3), ok1 = inner || (a0 + 1 >= 3 && a0 + 1 < N - 3);
#pragma unroll
      for (int pl = 0; pl < 4; pl++) {
        if (STAGE == 2) {
          const float e0 = 0.25f * dt * res[pl][0], e1 = 0.25f * dt * res[pl][1];
          float *dst = A.e_out + pl * NM + base;
          if (both) {
            *reinterpret_cast<float2 *>(dst) = make_float2(e0, e1);
          } else {
            if (ok0) dst[0] = e0;
            if (ok1) dst[1] = e1;
          }
        } else {
          const double2 u = *reinterpret_cast<const double2 *>(&S.u1[pl][r][2 * tx]);
          const float i0 = fmaf(2.0f / 3.0f * dt, res[pl][0], 2.0f * fc[pl][0]);
          const float i1 = fmaf(2.0f / 3.0f * dt, res[pl][1], 2.0f * fc[pl][1]);
          const double o0 = u.x + static_cast<double>(i0), o1 = u.y + static_cast<double>(i1);
          double *dst = A.u_out + pl * NM + base;
          if (both) {
            *reinterpret_cast<double2 *>(dst) = make_double2(o0, o1);
          } else {
            if (ok0) dst[0] = o0;
            if (ok1) dst[1] = o1;
          }
        }
      }
    }
  };
  if (!lo_cols && !hi_cols) rows(std::true_type{});
  else rows(std::false_type{});
}

template <int STAGE>
__global__ void __launch_bounds__(kMixThreads, mix_blocks_per_sm<STAGE>())
    mixed_stage_kernel(const __grid_constant__ MixedMaps T, const MixedArgs A, int ahead) {
  mixed_tile<STAGE>(T, A, blockIdx.x * TC, blockIdx.y * kMixRows, MixGridAhead{&T, ahead});
}

// Mixed-precision solves of a batch: block -> (solve, tile), work item
// blockIdx.x of the launch group (its `solve` entries index the MixedBatch
// array).
template <int STAGE>
__global__ void __launch_bounds__(kMixThreads, mix_blocks_per_sm<STAGE>())
    mixed_batch_kernel(const MixedBatch *solves, const __grid_constant__ MixedGroup G, int ahead) {
  int c0, b0;
  const int i = group_item(G, blockIdx.x, kMixRows, c0, b0);
  mixed_tile<STAGE>(solves[G.solve[i]].maps[STAGE - 2], G.args[i], c0, b0, MixGroupAhead<STAGE>{solves, &G, ahead});
}

// bb, ee = Ataurho + bb, d_re = (Brho_re - bb Btau_re) - bb' ee and
// d_im = Brho_im - bb Btau_im of HighOrder/kern.cu:132-158, 192-197 in FP64
// with the FP64 stage kernels' arithmetic, stored in FP32 (planes of kc).
__global__ void mixed_coef_kernel(const double *coltab, const double *rowtab, const double *bbt, float *kc, int N,
                                  int M, double cx) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y;
  if (a >= N) return;
  const size_t NM = static_cast<size_t>(N) * M, id = static_cast<size_t>(b) * N + a;
  float out[4] = {0.f, 0.f, 0.f, 0.f};
  if (b >= 3 && b < M - 3 && a >= 3 && a < N - 3) {
    const double bb = bbt[id];
    const double ib = inv_bir(coltab[CF_B0 * N + a], coltab[CF_B1 * N + a], rowtab[RF_S2 * M + b]);
    const double ee = coltab[CF_ATN * N + a] * ib + bb;
    const double dbdx = d1c(bbt + id, 0) * cx;
    const double btr = coltab[CF_XR * N + a] * ib, brr = coltab[CF_YR * N + a] * ib;
    const double bti = (coltab[CF_BI0 * N + a] + coltab[CF_BI1 * N + a] * rowtab[RF_COS * M + b]) * ib;
    out[0] = static_cast<float>(bb);
    out[1] = static_cast<float>(ee);
    out[2] = static_cast<float>((brr - bb * btr) - dbdx * ee);
    out[3] = static_cast<float>(coltab[CF_BRI * N + a] * ib - bb * bti);
  }
  for (int k = 0; k < 4; k++) kc[k * NM + id] = out[k];
}

__global__ void to_float_kernel(const double *src, float *dst, size_t n) {
  const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = static_cast<float>(src[i]);
}

template <int STAGE>
size_t mix_smem_bytes() {
  return sizeof(MixSmem<STAGE>) + 128;
}

PFN_cuTensorMapEncodeTiled_v12000 mix_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    cudaDriverEntryPointQueryResult qr;
    void *fn = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &qr) != cudaSuccess ||
        qr != cudaDriverEntryPointSuccess || !fn)
      return nullptr;
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  return encode;
}

}  // namespace

cudaError_t encode_mixed_maps(const float *in, const float *bbf, const float *colf, const float *rowf,
                              const double *u1, int N, int M, MixedMaps *maps) {
  auto encode = mix_encoder();
  if (!encode) return cudaErrorNotSupported;
  const cuuint32_t estr[3] = {1, 1, 1};
  const cuuint64_t dims[3] = {static_cast<cuuint64_t>(N), static_cast<cuuint64_t>(M), 4};
  const cuuint64_t fstr[2] = {static_cast<cuuint64_t>(N) * 4, static_cast<cuuint64_t>(N) * M * 4};
  const cuuint64_t dstr[2] = {static_cast<cuuint64_t>(N) * 8, static_cast<cuuint64_t>(N) * M * 8};
  const cuuint32_t box_q[3] = {WC, kMixRows + 6, 2}, box_p[3] = {WC, kMixRows, 2}, box_u[3] = {TC, kMixRows, 4};
  const cuuint32_t box_kc[3] = {TC, kMixRows, 4};
  const cuuint64_t cdims[2] = {static_cast<cuuint64_t>(N), CF_COUNT};
  const cuuint64_t cstr[1] = {static_cast<cuuint64_t>(N) * 4};
  const cuuint32_t box_cf[2] = {TC, CF_COUNT};
  const cuuint64_t rdims[2] = {static_cast<cuuint64_t>(M), RF_COUNT};
  const cuuint64_t rstr[1] = {static_cast<cuuint64_t>(M) * 4};
  const cuuint32_t box_rf[2] = {kMixRows, RF_COUNT};
  const auto F32 = CU_TENSOR_MAP_DATA_TYPE_FLOAT32, F64 = CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
  const auto IL = CU_TENSOR_MAP_INTERLEAVE_NONE;
  const auto SW = CU_TENSOR_MAP_SWIZZLE_NONE;
  const auto L2 = CU_TENSOR_MAP_L2_PROMOTION_L2_256B;
  const auto OOB = CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE;
  CUresult r[6];
  r[0] = encode(&maps->q, F32, 3, const_cast<float *>(in), dims, fstr, box_q, estr, IL, SW, L2, OOB);
  r[1] = encode(&maps->p, F32, 3, const_cast<float *>(in), dims, fstr, box_p, estr, IL, SW, L2, OOB);
  r[2] = encode(&maps->bb, F32, 3, const_cast<float *>(bbf), dims, fstr, box_kc, estr, IL, SW, L2, OOB);
  r[3] = encode(&maps->colf, F32, 2, const_cast<float *>(colf), cdims, cstr, box_cf, estr, IL, SW, L2, OOB);
  r[4] = encode(&maps->rowf, F32, 2, const_cast<float *>(rowf), rdims, rstr, box_rf, estr, IL, SW, L2, OOB);
  r[5] = u1 ? encode(&maps->u1, F64, 3, const_cast<double *>(u1), dims, dstr, box_u, estr, IL, SW, L2, OOB)
            : CUDA_SUCCESS;
  for (CUresult x : r)
    if (x != CUDA_SUCCESS) return cudaErrorInvalidValue;
  return cudaSuccess;
}

cudaError_t prepare_mixed_kernels() {
  cudaError_t e;
  const int s2 = static_cast<int>(mix_smem_bytes<2>()), s3 = static_cast<int>(mix_smem_bytes<3>());
  if ((e = cudaFuncSetAttribute(mixed_stage_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, s2)) ||
      (e = cudaFuncSetAttribute(mixed_stage_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, s3)) ||
      (e = cudaFuncSetAttribute(mixed_batch_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, s2)) ||
      (e = cudaFuncSetAttribute(mixed_batch_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, s3)))
    return e;
  return cudaSuccess;
}

cudaError_t launch_mixed_stage(int stage, const MixedMaps &maps, const MixedArgs &a, cudaStream_t st) {
  const dim3 grid(a.N / TC, a.M / kMixRows), block(32, kMixThreads / 32);
  const int ahead = stage_prefetch_ahead();
  if (stage == 2) return launch_pdl(mixed_stage_kernel<2>, grid, block, mix_smem_bytes<2>(), st, maps, a, ahead);
  return launch_pdl(mixed_stage_kernel<3>, grid, block, mix_smem_bytes<3>(), st, maps, a, ahead);
}

cudaError_t launch_mixed_batch(int stage, const MixedBatch *solves, const MixedGroup &g, cudaStream_t st) {
  if (g.ntiles <= 0) return cudaSuccess;
  const dim3 grid(g.ntiles), block(32, kMixThreads / 32);
  const int ahead = stage_prefetch_ahead();
  if (stage == 2) return launch_pdl(mixed_batch_kernel<2>, grid, block, mix_smem_bytes<2>(), st, solves, g, ahead);
  return launch_pdl(mixed_batch_kernel<3>, grid, block, mix_smem_bytes<3>(), st, solves, g, ahead);
}

cudaError_t launch_mixed_coef(const double *coltab, const double *rowtab, const double *bbt, float *kc, int N, int M,
                              double cx, cudaStream_t st) {
  mixed_coef_kernel<<<dim3((N + 255) / 256, M), 256, 0, st>>>(coltab, rowtab, bbt, kc, N, M, cx);
  return cudaGetLastError();
}

cudaError_t launch_to_float(const double *src, float *dst, size_t n, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  to_float_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(src, dst, n);
  return cudaGetLastError();
}

}  // namespace bhr
