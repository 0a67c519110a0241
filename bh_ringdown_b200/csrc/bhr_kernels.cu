// bhr_kernels.cu -- sm_100a kernels of the FP64 Teukolsky step.
//
// The kernels of one time step (the solver runs the source of the next step
// and the extraction of the previous one on a side stream beside stages 1
// and 2, and advances the stage step clock after the final stage):
//   source_patch  the Gaussian-smeared particle source on its PTSX x PTSY patch
//                 (HighOrder/kern.cu:755-768 reset + 1185-2683 deposit)
//   stage<1,2,3>  one SSP-RK3 stage each (classical RK4: stages 1, 4, 4, 5,
//                 four launches): TMA stages a (q, p) tile with its
//                 halo into shared memory, the pole and radial-end closures of
//                 the stage input are rebuilt there, then the 6th-order
//                 stencils, Kreiss-Oliger dissipation, coefficients, source
//                 and the stage combination are applied and the interior
//                 of the next stage is written once
//                 (HighOrder/kern.cu:171-753 as kernel_rhs*/update*/boundary*)
//   extract       psi at the extraction column, its two time integrals, and
//                 on output steps the swsh projection and dE/dt
//                 (HighOrder/body.cu:168-212, HighOrder/proj.c:37-75)
//   step_clock    one thread: the stage step clock of the next step
//
// Storage: each state is four planes (q_re, q_im, p_re, p_im) of M x N
// doubles, idx(b,a) = N*b + a.  Only interior points 3 <= b < M-3,
// 3 <= a < N-3 are stored; the boundary rows and columns of every stage are
// the reference's extrapolation closure of the interior and are rebuilt by
// whoever reads them.
#include "bhr_device.cuh"
#include "bhr_internal.h"

#include <cudaTypedefs.h>

#include <algorithm>
#include <cstddef>
#include <cstdlib>
#include <type_traits>
#include <utility>

namespace bhr {

namespace {

// Constants, PTX helpers, stencils: bhr_device.cuh.

// Shared memory of one tile of ROWS theta rows (8 or 16).
template <int ROWS>
struct __align__(128) StageSmem {
  // Every TMA destination (and TMA store source) starts on a 128-byte boundary.
  alignas(128) double q[2][ROWS + 6][WC];    // TMA box {WC, ROWS+6, 2}: planes q_re, q_im with halo
  alignas(128) double p[2][ROWS][WC];        // TMA box {WC, ROWS, 2}: planes p_re, p_im with column halo
  alignas(128) double bb[ROWS][WC];          // TMA box {WC, ROWS, 1}: bb on the window columns
  alignas(128) double cf[CF_TILE][TC];       // TMA box {TC, CF_TILE}: column factors of the tile columns
  alignas(128) double un[4][ROWS][TC];       // TMA box {TC, ROWS, 4}: u^n (RK4 stage 5: z), stages > 1
  alignas(128) double rf[RF_COUNT][ROWS];    // TMA box {ROWS, RF_COUNT}: row factors of the tile rows
  uint64_t bar;
  int src_c0, src_r0;           // source patch corner of this step
  int src_buf;                  // source patch buffer of this step (k % 2)
  int done;                     // persistent kernels: warps done with this buffer's tile
  int issued;                   // persistent kernels: load phases issued into this buffer
  int abort;                    // persistent kernels (buffer 0): a bounded wait gave up
};
#define BHR_TMA_ALIGNED(T, m) static_assert(offsetof(T, m) % 128 == 0, "TMA destination " #m " not 128-byte aligned")
BHR_TMA_ALIGNED(StageSmem<8>, p);
BHR_TMA_ALIGNED(StageSmem<8>, bb);
BHR_TMA_ALIGNED(StageSmem<8>, cf);
BHR_TMA_ALIGNED(StageSmem<8>, un);
BHR_TMA_ALIGNED(StageSmem<8>, rf);
BHR_TMA_ALIGNED(StageSmem<16>, p);
BHR_TMA_ALIGNED(StageSmem<16>, bb);
BHR_TMA_ALIGNED(StageSmem<16>, cf);
BHR_TMA_ALIGNED(StageSmem<16>, un);
BHR_TMA_ALIGNED(StageSmem<16>, rf);
static_assert(sizeof(StageSmem<16>) % 128 == 0, "persistent buffers must stay 128-byte aligned");
static_assert(sizeof(StageSmem<8>) % 128 == 0, "ring buffers must stay 128-byte aligned");

// The time-independent per-point coefficient bb (HighOrder/kern.cu:141-147),
// which the stage kernels need on a stencil window, for the interior rows,
// once per solve.  1/bir and ee = Ataurho + bb are formed per point by the
// stage kernels from the column and row factors with the same arithmetic.
__global__ void coef_table_kernel(const double *coltab, const double *rowtab, double *ctab, int N, int M) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y;
  if (a >= N) return;
  const size_t id = static_cast<size_t>(b) * N + a;
  double bb = 0.0;
  if (b >= 3 && b < M - 3) {
    const double ib = inv_bir(coltab[CF_B0 * N + a], coltab[CF_B1 * N + a], rowtab[RF_S2 * M + b]);
    const double At = coltab[CF_ATN * N + a] * ib, Ar = coltab[CF_ARN * N + a] * ib;
    bb = -(At + sqrt_nr(fma(At, At, 4.0 * Ar))) * 0.5;
  }
  ctab[id] = bb;
}

// One tile (columns c0..c0+63, rows b0..b0+ROWS-1) of one Runge-Kutta stage
// (STAGE 1-3: SSP-RK3; classical RK4 runs stages 1, 4, 4, 5).
// A stage tile is processed in four steps, shared by the one-tile-per-block
// kernels and the persistent ones: thread 0 arms the tile's mbarrier and
// requests the set-up data, then (after the grid dependency) the stage
// input; all threads wait, rebuild the closure rows in shared memory and
// compute the tile's rows.

// Thread 0: arm the barrier for every byte of the tile and request the
// coefficient planes and column/row factors (written once, at set-up, so
// they may be requested before the previous kernel has finished).
template <int STAGE, int ROWS>
__device__ __forceinline__ void tile_issue_setup(StageSmem<ROWS> &S, const StageMaps &T, const int c0, const int b0) {
  const uint32_t bytes = static_cast<uint32_t>(sizeof(S.q) + sizeof(S.p) + sizeof(S.bb) + sizeof(S.cf) +
                                               sizeof(S.rf) + (STAGE == 1 ? 0 : sizeof(S.un)));
  mbar_expect_tx(&S.bar, bytes);
  tma_load_3d(&S.bb[0][0], &T.coef_bb, c0 - 4, b0, 0, &S.bar);
  tma_load_2d(&S.cf[0][0], &T.colf, c0, 0, &S.bar);
  tma_load_2d(&S.rf[0][0], &T.rowf, b0, 0, &S.bar);
}

// Thread 0, after the grid dependency (the stage step clock is advanced
// after the previous step's final stage, or by its extraction): this step's
// source patch corner and buffer.
// A block barrier publishes it to the other warps.
template <int ROWS>
__device__ __forceinline__ void tile_note_source(StageSmem<ROWS> &S, const StageArgs &A) {
  if (A.src != nullptr) {
    const int k = A.rs->ks;
    const StepRec &rec = A.recs[k];
    S.src_c0 = rec.col0;
    S.src_r0 = rec.row0;
    S.src_buf = k & 1;
  }
}

// Thread 0, after the grid dependency: request the stage input (and u^n).
template <int STAGE, int ROWS>
__device__ __forceinline__ void tile_issue_state(StageSmem<ROWS> &S, const StageMaps &T, const int c0, const int b0) {
  tma_load_3d(&S.q[0][0][0], &T.q, c0 - 4, b0 - 3, 0, &S.bar);
  tma_load_3d(&S.p[0][0][0], &T.p, c0 - 4, b0, 2, &S.bar);
  if (STAGE != 1) tma_load_3d(&S.un[0][0][0], &T.u, c0, b0, 0, &S.bar);
}

// All threads: the closure of the stage input, rebuilt in shared memory.
template <int ROWS, int THREADS>
__device__ __forceinline__ void tile_close(StageSmem<ROWS> &S, const StageArgs &A, const int c0, const int b0,
                                           const int tid) {
  constexpr int TR = ROWS;
  const int N = A.N, M = A.M;
  // Closure of the stage input rebuilt in shared memory.
  // Poles, q only (HighOrder/kern.cu:320-409): rows 2,1,0 from 3,4 and
  // M-3,M-2,M-1 from M-4,M-5 on columns 3..N-4; zero for odd m.
  const bool lo_rows = (b0 == 0), hi_rows = (b0 + TR + 3 > M - 3);
  if (lo_rows || hi_rows) {
    for (int i = tid; i < 2 * WC; i += THREADS) {
      const int pl = i / WC, w = i - pl * WC;
      const int a = c0 - 4 + w;
      if (a < 3 || a >= N - 3) continue;
      double(*q)[WC] = S.q[pl];
      const int o = 3 - b0;  // window row of global row g is g + o
      if (lo_rows) {
        if (A.even_m) {
          q[2 + o][w] = (4.0 * q[3 + o][w] - q[4 + o][w]) * kThird;
          q[1 + o][w] = (4.0 * q[2 + o][w] - q[3 + o][w]) * kThird;
          q[0 + o][w] = (4.0 * q[1 + o][w] - q[2 + o][w]) * kThird;
        } else {
          q[2 + o][w] = 0.0; q[1 + o][w] = 0.0; q[0 + o][w] = 0.0;
        }
      }
      if (hi_rows) {
        if (A.even_m) {
          q[M - 3 + o][w] = (4.0 * q[M - 4 + o][w] - q[M - 5 + o][w]) * kThird;
          q[M - 2 + o][w] = (4.0 * q[M - 3 + o][w] - q[M - 4 + o][w]) * kThird;
          q[M - 1 + o][w] = (4.0 * q[M - 2 + o][w] - q[M - 3 + o][w]) * kThird;
        } else {
          q[M - 3 + o][w] = 0.0; q[M - 2 + o][w] = 0.0; q[M - 1 + o][w] = 0.0;
        }
      }
    }
  }
  // Radial ends, all four planes, tile rows (HighOrder/kern.cu:412-449).
  const bool lo_cols = (c0 == 0), hi_cols = (c0 + TC + 4 > N - 3);
  if (lo_cols || hi_cols) {
    for (int i = tid; i < 4 * TR; i += THREADS) {
      const int pl = i / TR, r = i - pl * TR;
      const int b = b0 + r;
      if (b < 3 || b >= M - 3) continue;
      double *row = pl < 2 ? &S.q[pl][r + 3][0] : &S.p[pl - 2][r][0];
      const int o = 4 - c0;  // window column of global column a is a + o
      if (lo_cols) {
        row[2 + o] = (4.0 * row[3 + o] - row[4 + o]) * kThird;
        row[1 + o] = (4.0 * row[2 + o] - row[3 + o]) * kThird;
        row[0 + o] = (4.0 * row[1 + o] - row[2 + o]) * kThird;
      }
      if (hi_cols) {
        row[N - 3 + o] = (4.0 * row[N - 4 + o] - row[N - 5 + o]) * kThird;
        row[N - 2 + o] = (4.0 * row[N - 3 + o] - row[N - 4 + o]) * kThird;
        row[N - 1 + o] = (4.0 * row[N - 2 + o] - row[N - 3 + o]) * kThird;
      }
    }
  }
}

// Where the row work below puts a stage's output: global memory (the
// stage output planes), the tile's own u^n buffer (TMA-stored afterwards by
// the persistent kernels), or a shared-memory ring (the fused strip kernel).
enum OutMode { kOutGlobal = 0, kOutTile = 1, kOutRing = 2 };

// The source patch corner and buffer of the step a tile works on.
struct SrcNote {
  int c0, r0, buf;
};

// A tile's shared-memory inputs as the row work reads them.  Row pointers
// are indexed by window column (w = 0 is the tile's first column minus 4);
// cf(f) by 2 tx + the view's column offset; window row j of q is tile row
// j - 3.
template <int ROWS>
struct TileView {
  StageSmem<ROWS> &S;
  __device__ __forceinline__ const double *qwin(int pl, int j) const { return &S.q[pl][j][0]; }
  __device__ __forceinline__ const double *prow(int pl, int r) const { return &S.p[pl][r][0]; }
  __device__ __forceinline__ const double *bbrow(int r) const { return &S.bb[r][0]; }
  __device__ __forceinline__ const double *cf(int f) const { return S.cf[f]; }
  __device__ __forceinline__ double rf(int f, int r) const { return S.rf[f][r]; }
  __device__ __forceinline__ const double *unrow(int pl, int r) const { return &S.un[pl][r][0]; }
  __device__ __forceinline__ double *outrow(int pl, int r) const { return &S.un[pl][r][0]; }
};

// The right-hand side and the Shu-Osher combination of RPT rows of one
// 64-column row segment per warp (the thread's columns a0 = c0 + 2 tx and
// a0 + 1, window column w0 = woff + 2 tx + 4), written to the stage output.
// inner: every column of the segment is at least 4 from both radial ends
// (no per-column end checks).  Outputs are stored for columns in
// [st_lo, st_hi) (interior columns only); an inner segment stores all its
// columns unless MASKED.  nrows: the tile's rows (for the source patch
// overlap test).
// kOutTile: the outputs overwrite u^n in the tile buffer (each thread reads
// its u^n before writing there) for a TMA store of the whole tile.
// kOutRing: the outputs go to the view's output rows at window column w0.
template <int STAGE, int RPT, int OUT, bool MASKED, class View>
__device__ __forceinline__ void tile_rows(const View &V, const StageArgs &A, const int c0, const int b0,
                                          const int nrows, const int tx, const int ty, const int woff,
                                          const bool inner, const int st_lo, const int st_hi, const SrcNote note) {
  const int N = A.N, M = A.M;
  const size_t NM = static_cast<size_t>(N) * M;
  int src_c0 = 0, src_r0 = 0;
  bool tile_src = false;
  const double *srcp = A.src;
  if (A.src != nullptr) {
    src_c0 = note.c0;
    src_r0 = note.r0;
    srcp = A.src + static_cast<size_t>(note.buf) * 2 * A.PTSX * A.PTSY;
    tile_src = (src_c0 < c0 + TC) && (src_c0 + A.PTSX > c0) && (src_r0 < b0 + nrows) && (src_r0 + A.PTSY > b0);
  }

  const int a0 = c0 + 2 * tx;       // this thread's columns a0, a0+1
  const int w0 = woff + 2 * tx + 4;  // their window column
  const int cx0 = woff + 2 * tx;     // their index in the per-column arrays
  const double dt = A.dt;

  // Theta derivatives of q on all of this thread's rows
  // (HighOrder/kern.cu:206-226), from one pass over the RPT + 6 window rows
  // they reach: each row is read from shared memory once, not once per
  // output row (the shared-memory load pipe is the stage kernels' busiest
  // unit).
  double lla[RPT][2][2];
#pragma unroll
  for (int pl = 0; pl < 2; pl++) {
    double f[RPT + 6][2];
#pragma unroll
    for (int j = 0; j < RPT + 6; j++) {
      const double2 t = *reinterpret_cast<const double2 *>(V.qwin(pl, RPT * ty + j) + w0);
      f[j][0] = t.x;
      f[j][1] = t.y;
    }
#pragma unroll
    for (int rr = 0; rr < RPT; rr++) {
      const double ctan_cy = V.rf(RF_CTAN, RPT * ty + rr) * A.cy;
#pragma unroll
      for (int c = 0; c < 2; c++) {
        const double *g = &f[rr][0] + c;  // g[2 j] = row rr + j of column c
        const double y1 = (g[12] - g[0]) - 9.0 * (g[10] - g[2]) + 45.0 * (g[8] - g[4]);
        const double y2 = 2.0 * (g[12] + g[0]) - 27.0 * (g[10] + g[2]) + 270.0 * (g[8] + g[4]) - 490.0 * g[6];
        lla[rr][pl][c] = y2 * A.cyy + ctan_cy * y1;
      }
    }
  }

  // The row work, instantiated once for interior segments (no per-column
  // end checks) and once for segments at a radial end.
  auto rows = [&](auto inner_tag) {
  constexpr bool in = decltype(inner_tag)::value;
#pragma unroll 1
  for (int rr = 0; rr < RPT; rr++) {
    const int r = RPT * ty + rr;
    const int b = b0 + r;
    if (b < 3 || b >= M - 3) continue;
    if (!in && (a0 + 1 < 3 || a0 >= N - 3)) continue;
    double ll[2][2];
#pragma unroll
    for (int q = 0; q < RPT; q++)
      if (q == rr) {
        ll[0][0] = lla[q][0][0];
        ll[0][1] = lla[q][0][1];
        ll[1][0] = lla[q][1][0];
        ll[1][1] = lla[q][1][1];
      }

    // Coefficients at the two points (HighOrder/kern.cu:132-158, 192-197).
    const double cs = V.rf(RF_COS, r);
    const double gth = V.rf(RF_G, r);
    const double s2 = V.rf(RF_S2, r);
    double kbb[2], kee[2], kdre[2], kdim[2], kare[2], kaim[2], kvre[2], kvim[2];
    double res[4][2];
    // bb on columns a0-4 .. a0+5, and the per-column arrays, as 16-byte pairs
    double bw[10];
    const double *bbr = V.bbrow(r);
#pragma unroll
    for (int j = 0; j < 5; j++) {
      const double2 t = *reinterpret_cast<const double2 *>(bbr + w0 - 4 + 2 * j);
      bw[2 * j] = t.x;
      bw[2 * j + 1] = t.y;
    }
    auto pair = [&](const double *base) { return *reinterpret_cast<const double2 *>(base + cx0); };
    const double2 g0 = pair(V.cf(CF_B0)), gd = pair(V.cf(CF_DT)), g2 = pair(V.cf(CF_ATN));
    const double2 f1 = pair(V.cf(CF_XR)), f2 = pair(V.cf(CF_YR)), f3 = pair(V.cf(CF_BI0)), f5 = pair(V.cf(CF_BRI)),
                  f6 = pair(V.cf(CF_CR0)), f8 = pair(V.cf(CF_CIN));
#pragma unroll
    for (int c = 0; c < 2; c++) {
      const int a = a0 + c;
      auto pk = [&](double2 v) { return c ? v.y : v.x; };
      const double bb = bw[4 + c];
      // B1, CCN, CR1 and BI1 are Dt times a^2, -1, 1 and -4a: the same
      // products the column table holds, formed here to load 9 factors, not 12.
      const double Dt = pk(gd);
      const double ib = inv_bir(pk(g0), A.a2 * Dt, s2);
      const double ee = pk(g2) * ib + bb;  // Ataurho + bb
      const double dbdx = d1c(bw, 4 + c) * A.cx;
      const double cc = -Dt * ib;
      const double btr = pk(f1) * ib;
      const double brr = pk(f2) * ib;
      const double bti = (pk(f3) + (A.m4a * Dt) * cs) * ib;
      kbb[c] = bb;
      kee[c] = ee;
      kdim[c] = pk(f5) * ib - bb * bti;
      kvre[c] = -(pk(f6) + Dt * gth) * ib;
      kvim[c] = -pk(f8) * ib;
      kare[c] = -btr;
      kaim[c] = -bti;
      kdre[c] = (brr - bb * btr) - dbdx * ee;
      double sre = 0.0, sim = 0.0;
      if (tile_src) {
        const int sc = a - src_c0, sr = b - src_r0;
        if (sc >= 0 && sc < A.PTSX && sr >= 0 && sr < A.PTSY) {
          sre = srcp[static_cast<size_t>(sr) * A.PTSX + sc];
          sim = srcp[static_cast<size_t>(A.PTSY + sr) * A.PTSX + sc];
        }
      }
      res[2][c] = fma(cc, ll[0][c], sre);
      res[3][c] = fma(cc, ll[1][c], sim);
    }

    // Radial first derivative and dissipation plane by plane, each folded
    // into the right-hand side as soon as it is formed
    // (HighOrder/kern.cu:233-261, 281-296).
    double fc[4][2];
#pragma unroll
    for (int pl = 0; pl < 4; pl++) {
      const double *row = pl < 2 ? V.qwin(pl, r + 3) : V.prow(pl - 2, r);
      double v[10];
#pragma unroll
      for (int j = 0; j < 5; j++) {
        const double2 t = *reinterpret_cast<const double2 *>(row + w0 - 4 + 2 * j);
        v[2 * j] = t.x;
        v[2 * j + 1] = t.y;
      }
#pragma unroll
      for (int c = 0; c < 2; c++) {
        const int a = a0 + c;
        const double f0 = v[4 + c];
        const double fx = d1c(v, 4 + c) * A.cx;
        const double fk = (in || (a >= 4 && a < N - 4)) ? ko8c(v, 4 + c) * A.cko : 0.0;
        fc[pl][c] = f0;
        // each term folded into its accumulator by one FMA (res[0] and
        // res[1] start with the q planes' terms)
        if (pl == 0) {         // q_re
          res[0][c] = fma(-kbb[c], fx, -fk);
          res[2][c] = fma(kdre[c], fx, fma(-kvre[c], f0, res[2][c]));
          res[3][c] = fma(kdim[c], fx, fma(-kvim[c], f0, res[3][c]));
        } else if (pl == 1) {  // q_im
          res[1][c] = fma(-kbb[c], fx, -fk);
          res[2][c] = fma(-kdim[c], fx, fma(kvim[c], f0, res[2][c]));
          res[3][c] = fma(kdre[c], fx, fma(-kvre[c], f0, res[3][c]));
        } else if (pl == 2) {  // p_re
          res[0][c] += f0;
          res[2][c] = fma(kee[c], fx, fma(-kare[c], f0, res[2][c] - fk));
          res[3][c] = fma(-kaim[c], f0, res[3][c]);
        } else {               // p_im
          res[1][c] += f0;
          res[2][c] = fma(kaim[c], f0, res[2][c]);
          res[3][c] = fma(kee[c], fx, fma(-kare[c], f0, res[3][c] - fk));
        }
      }
    }

    // Stage combination: SSP-RK3 in Shu-Osher form (stages 1-3,
    // HighOrder/kern.cu:301-318, 582-620), or classical RK4 (stage 1 with
    // dt/2, then stages 4, 4 and 5).
    const size_t base = static_cast<size_t>(b) * N + a0;
    const bool both = (in && !MASKED) || ((a0 >= st_lo) && (a0 + 1 < st_hi));
    auto store2 = [&](double *dst, const double v0, const double v1) {
      if (both) {
        *reinterpret_cast<double2 *>(dst) = make_double2(v0, v1);
      } else {
        if (a0 >= st_lo && a0 < st_hi) dst[0] = v0;
        if (a0 + 1 >= st_lo && a0 + 1 < st_hi) dst[1] = v1;
      }
    };
#pragma unroll
    for (int pl = 0; pl < 4; pl++) {
      double o[2];
      if (STAGE == 1) {
        o[0] = fc[pl][0] + dt * res[pl][0];
        o[1] = fc[pl][1] + dt * res[pl][1];
        if (A.dout != nullptr) {  // mixed precision: delta1 in FP32
          const float d0 = static_cast<float>(dt * res[pl][0]), d1 = static_cast<float>(dt * res[pl][1]);
          float *fd = A.dout + pl * NM + base;
          if (both) {
            *reinterpret_cast<float2 *>(fd) = make_float2(d0, d1);
          } else {
            if (a0 >= st_lo && a0 < st_hi) fd[0] = d0;
            if (a0 + 1 >= st_lo && a0 + 1 < st_hi) fd[1] = d1;
          }
        }
      } else {
        const double2 u = *reinterpret_cast<const double2 *>(V.unrow(pl, r) + cx0);
        if (STAGE == 2) {
          o[0] = 0.25 * (3.0 * u.x + fc[pl][0] + dt * res[pl][0]);
          o[1] = 0.25 * (3.0 * u.y + fc[pl][1] + dt * res[pl][1]);
        } else if (STAGE == 3) {
          o[0] = kThird * (u.x + 2.0 * fc[pl][0] + 2.0 * dt * res[pl][0]);
          o[1] = kThird * (u.y + 2.0 * fc[pl][1] + 2.0 * dt * res[pl][1]);
        } else if (STAGE == 4) {
          // RK4 stages 2 and 3: y = u^n + h L(y'), h = dt/2 or dt.  Stage 2
          // also folds y1 (its input) and y2 into z = (y1 + 2 y2 - u^n)/3,
          // so the last stage needs z and y3 only.
          o[0] = u.x + dt * res[pl][0];
          o[1] = u.y + dt * res[pl][1];
          if (A.zout != nullptr)
            store2(A.zout + pl * NM + base, (fc[pl][0] + 2.0 * o[0] - u.x) * kThird,
                   (fc[pl][1] + 2.0 * o[1] - u.y) * kThird);
        } else {
          // RK4 stage 4 (u^n slot = z, h = dt/6):
          // u^{n+1} = z + y3/3 + dt/6 L(y3) = u^n + dt/6 (k1 + 2 k2 + 2 k3 + k4).
          o[0] = u.x + kThird * fc[pl][0] + dt * res[pl][0];
          o[1] = u.y + kThird * fc[pl][1] + dt * res[pl][1];
        }
      }
      if (OUT == kOutTile) {
        *reinterpret_cast<double2 *>(V.outrow(pl, r) + cx0) = make_double2(o[0], o[1]);
      } else if (OUT == kOutRing) {
        store2(V.outrow(pl, r) + w0, o[0], o[1]);
      } else {
        store2(A.out + pl * NM + base, o[0], o[1]);
      }
    }
  }
  };
  if (inner) rows(std::true_type{});
  else rows(std::false_type{});
}

// All threads: the right-hand side and the Shu-Osher combination of the
// tile's rows, written to the stage output (TO_SMEM: into the tile's u^n
// buffer, for tiles without closure points).
template <int STAGE, int ROWS, int THREADS, bool TO_SMEM>
__device__ __forceinline__ void tile_compute(StageSmem<ROWS> &S, const StageArgs &A, const int c0, const int b0,
                                             const int tx, const int ty) {
  const bool lo_cols = (c0 == 0), hi_cols = (c0 + TC + 4 > A.N - 3);
  const SrcNote note{S.src_c0, S.src_r0, S.src_buf};
  tile_rows<STAGE, ROWS / (THREADS / 32), TO_SMEM ? kOutTile : kOutGlobal, false>(
      TileView<ROWS>{S}, A, c0, b0, ROWS, tx, ty, 0, !lo_cols && !hi_cols, 3, A.N - 3, note);
}

// Thread 0: prefetch into L2 the stage input of a later tile (its maps
// and corner), so that the block which takes it, some microseconds on,
// finds its loads in L2 instead of waiting for HBM at the start of its life.
template <int STAGE>
__device__ __forceinline__ void tile_prefetch(const StageMaps &T, const int c0, const int b0) {
  tma_prefetch_3d(&T.q, c0 - 4, b0 - 3, 0);
  tma_prefetch_3d(&T.p, c0 - 4, b0, 2);
  tma_prefetch_3d(&T.coef_bb, c0 - 4, b0, 0);
  if (STAGE != 1) tma_prefetch_3d(&T.u, c0, b0, 0);
}

// Thread 0: prefetch into L2 what the next stage reads of a tile: this
// stage's output there (the next stage's input; its halo is the
// neighbouring tiles' outputs), u^n and the bb window.
__device__ __forceinline__ void tile_prefetch_next(const StageMaps &T, const int c0, const int b0) {
  tma_prefetch_3d(&T.o, c0, b0, 0);
  tma_prefetch_3d(&T.u, c0, b0, 0);
  tma_prefetch_3d(&T.coef_bb, c0 - 4, b0, 0);
}

// One tile per block (grid N/64 x M/ROWS, two blocks per SM).  Thread 0
// prefetches the tile `ahead` names, if any (after the grid dependency).
template <int STAGE, int ROWS, int THREADS, class Ahead>
__device__ __forceinline__ void stage_tile(const StageMaps &T, const StageArgs &A, const int c0, const int b0,
                                           const Ahead ahead) {
  extern __shared__ unsigned char smem_raw[];
  StageSmem<ROWS> &S = *reinterpret_cast<StageSmem<ROWS> *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~static_cast<uintptr_t>(127));
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
  if (tid == 0) {
    mbar_init(&S.bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  if (tid == 0) tile_issue_setup<STAGE>(S, T, c0, b0);
  // Everything below reads what the earlier kernels of the step wrote.
  grid_dependency_wait();
  launch_dependents();
  if (tid == 0) {
    tile_issue_state<STAGE>(S, T, c0, b0);
    tile_note_source(S, A);
    const StageMaps *pm;
    int pc0, pb0;
    const int kind = ahead(pm, pc0, pb0);
    if (kind == 1) tile_prefetch<STAGE>(*pm, pc0, pb0);
    if (kind == 2) tile_prefetch_next(*pm, pc0, pb0);
  }
  const bool ok = mbar_wait_bounded(&S.bar, 0);
  if (!__syncthreads_and(ok)) {
    if (tid == 0) atomicCAS(A.err, 0, 5 /* BHR_TIMEOUT */);
    mbar_wait_bounded(&S.bar, 0);
    return;
  }
  tile_close<ROWS, THREADS>(S, A, c0, b0, tid);
  __syncthreads();
  tile_compute<STAGE, ROWS, THREADS, false>(S, A, c0, b0, tx, ty);
}

// Single solve: the block's tile is blockIdx.y * gridDim.x + blockIdx.x in
// launch order; the tile `n` places later (kind 1; n = A.ahead, 0: none).
// The last n blocks name instead the next stage's first n tiles (kind 2):
// their input, this stage's output and u^n, was written long before and has
// left L2.
template <int ROWS>
struct GridAhead {
  const StageMaps *T;
  int n;
  __device__ __forceinline__ int operator()(const StageMaps *&pm, int &c0, int &b0) const {
    const int ntiles = static_cast<int>(gridDim.x * gridDim.y);
    int L = blockIdx.y * gridDim.x + blockIdx.x + n, kind = 1;
    if (n <= 0) return 0;
    if (L >= ntiles) {
      L -= ntiles;
      kind = 2;
      if (L >= n || L >= ntiles) return 0;
    }
    pm = T;
    c0 = (L % gridDim.x) * TC;
    b0 = (L / gridDim.x) * ROWS;
    return kind;
  }
};
// Batch: the work item `n` places later in the group.  (Prefetching the
// next stage's first items from the last blocks, as the single-solve
// kernels do, measured no gain here.)
template <int STAGE, int ROWS>
struct GroupAhead {
  const BatchSolve *solves;
  const BatchGroup *G;
  int n;
  __device__ __forceinline__ int operator()(const StageMaps *&pm, int &c0, int &b0) const {
    const int L = blockIdx.x + n;
    if (n <= 0 || L >= G->ntiles) return 0;
    pm = &solves[G->solve[group_item(*G, L, ROWS, c0, b0)]].maps[STAGE - 1];
    return 1;
  }
};

template <int STAGE, int ROWS>
__global__ void __launch_bounds__(STAGE_THREADS, 2)
    stage_kernel(const __grid_constant__ StageMaps T, const StageArgs A) {
  stage_tile<STAGE, ROWS, STAGE_THREADS>(T, A, blockIdx.x * TC, blockIdx.y * ROWS, GridAhead<ROWS>{&T, A.ahead});
}

// 8-row tiles on 128-thread blocks: four blocks (16 warps) per SM, so four
// tiles' loads and computations interleave instead of two.
constexpr int kNarrowThreads = 128;
template <int STAGE>
__global__ void __launch_bounds__(kNarrowThreads, 4)
    stage_narrow_kernel(const __grid_constant__ StageMaps T, const StageArgs A) {
  stage_tile<STAGE, 8, kNarrowThreads>(T, A, blockIdx.x * TC, blockIdx.y * 8, GridAhead<8>{&T, A.ahead});
}

// Several solves advanced together: block -> (solve, tile), work item
// blockIdx.x of the launch group.
template <int STAGE, int ROWS>
__global__ void __launch_bounds__(STAGE_THREADS, 2)
    stage_batch_kernel(const BatchSolve *solves, const __grid_constant__ BatchGroup G, int ahead) {
  int c0, b0;
  const int i = group_item(G, blockIdx.x, ROWS, c0, b0);
  stage_tile<STAGE, ROWS, STAGE_THREADS>(solves[G.solve[i]].maps[STAGE - 1], G.args[i], c0, b0,
                                        GroupAhead<STAGE, ROWS>{solves, &G, ahead});
}

// ---- persistent stage kernels -------------------------------------------
// One block per SM walks the tiles blockIdx.x, blockIdx.x + gridDim.x, ...
// through a ring of NBUF shared-memory tile buffers: the loads of tile
// i+NBUF are issued as soon as tile i is computed, so they run under the
// computation of the tiles between and the SM's share of HBM bandwidth is
// kept busy.  Tile work is the same code as the one-tile-per-block kernels.
// Two shapes:
//   persistent  16-row tiles, 512 threads, 2 buffers, interior tiles stored
//               by TMA from shared memory (also the batch engine's)
//   ring        8-row tiles, 256 threads, 2 buffers, two blocks per SM
//               (16 warps, four tiles resident), outputs stored from
//               registers
constexpr int kPersistThreads = 512;
constexpr int kPersistRows = 16;
constexpr int kRingThreads = 256;
constexpr int kRingRows = 8;
constexpr int kRingBufs = 2;
constexpr int kRingBlocksPerSM = 2;

// Work item i of this block: the solve's maps and arguments and the tile
// corner.  Single solve: tiles in row-major order over the N/64 x M/rows grid.
struct SingleWork {
  const StageMaps *T;
  const StageArgs *A;
  int ntiles, tiles_x, rows;
  __device__ __forceinline__ int count() const { return ntiles; }
  __device__ __forceinline__ void get(int t, const StageMaps *&tm, const StageArgs *&ta, int &c0, int &b0) const {
    tm = T;
    ta = A;
    c0 = (t % tiles_x) * TC;
    b0 = (t / tiles_x) * rows;
  }
};
// Batch: work item t of the launch group.
template <int STAGE, int ROWS>
struct GroupWork {
  const BatchSolve *solves;
  const BatchGroup *G;
  __device__ __forceinline__ int count() const { return G->ntiles; }
  __device__ __forceinline__ void get(int t, const StageMaps *&tm, const StageArgs *&ta, int &c0, int &b0) const {
    const int i = group_item(*G, t, ROWS, c0, b0);
    tm = &solves[G->solve[i]].maps[STAGE - 1];
    ta = &G->args[i];
  }
};

// Warps are not held together between tiles: each waits for the tile's
// data itself, and the last warp to finish a tile (a shared counter) stores
// it (TMA, for tiles without closure points) and refills the buffer with
// tile i+2.  Tiles with closure points rebuild them first, behind a named
// barrier all warps reach in the same order.  After a bounded wait gives up
// the block records BHR_TIMEOUT, issues nothing more and lets the loads in
// flight land before it exits.
template <int STAGE, int ROWS, int THREADS, int NBUF, bool TMA_STORE, class Work>
__device__ __forceinline__ void stage_persistent(const Work &W, int *err) {
  constexpr int NWARPS = THREADS / 32;
  extern __shared__ unsigned char smem_raw[];
  StageSmem<ROWS> *buf = reinterpret_cast<StageSmem<ROWS> *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~static_cast<uintptr_t>(127));
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
  const int ntiles = W.count(), stride = gridDim.x, first = blockIdx.x;
  volatile int *abort_flag = &buf[0].abort;
  if (tid == 0) {
    for (int j = 0; j < NBUF; j++) {
      mbar_init(&buf[j].bar, 1);
      buf[j].done = 0;
      buf[j].issued = 0;
    }
    buf[0].abort = 0;
    fence_barrier_init();
  }
  __syncthreads();
  const StageMaps *tm;
  const StageArgs *ta;
  int c0, b0;
  if (tid == 0) {
    for (int j = 0; j < NBUF; j++) {
      const int t = first + j * stride;
      if (t < ntiles) {
        W.get(t, tm, ta, c0, b0);
        tile_issue_setup<STAGE>(buf[j], *tm, c0, b0);
        buf[j].issued = 1;
      }
    }
  }
  grid_dependency_wait();
  launch_dependents();
  if (tid == 0) {
    for (int j = 0; j < NBUF; j++) {
      const int t = first + j * stride;
      if (t < ntiles) {
        W.get(t, tm, ta, c0, b0);
        tile_issue_state<STAGE>(buf[j], *tm, c0, b0);
        tile_note_source(buf[j], *ta);
      }
    }
  }
  __syncthreads();  // the first tiles' source notes
  int i = 0;
  for (int t = first; t < ntiles; t += stride, i++) {
    StageSmem<ROWS> &S = buf[i % NBUF];
    bool stop = *abort_flag != 0;
    if (!stop && !mbar_wait_bounded(&S.bar, (i / NBUF) & 1)) {
      if (tx == 0) {
        atomicExch(&buf[0].abort, 1);
        atomicCAS(err, 0, 5 /* BHR_TIMEOUT */);
      }
      stop = true;
    }
    stop = __any_sync(0xffffffffu, stop);
    W.get(t, tm, ta, c0, b0);
    const int N = ta->N, M = ta->M;
    const bool edge = (b0 == 0) || (b0 + ROWS + 3 > M - 3) || (c0 == 0) || (c0 + TC + 4 > N - 3);
    const bool full = (b0 >= 3) && (b0 + ROWS <= M - 3) && (c0 >= 3) && (c0 + TC <= N - 3);
    if (edge) {
      if (!stop) tile_close<ROWS, THREADS>(S, *ta, c0, b0, tid);
      named_barrier_sync(1, THREADS);
    }
    if (!stop) {
      if (TMA_STORE && full) {
        tile_compute<STAGE, ROWS, THREADS, true>(S, *ta, c0, b0, tx, ty);
        fence_proxy_async();  // this thread's outputs, for the TMA store
      } else {
        tile_compute<STAGE, ROWS, THREADS, false>(S, *ta, c0, b0, tx, ty);
      }
    }
    __syncwarp();
    if (tx == 0) {
      __threadfence_block();
      if (atomicAdd(&S.done, 1) == NWARPS - 1) {
        __threadfence_block();
        S.done = 0;
        const bool ab = *abort_flag != 0;
        if (TMA_STORE && full && !ab) {
          tma_store_3d(&tm->o, &S.un[0][0][0], c0, b0, 0);
          bulk_commit();
          bulk_wait_read();
        }
        const int tn = t + NBUF * stride;
        if (tn < ntiles && !ab) {
          fence_proxy_async();
          const StageMaps *tm2;
          const StageArgs *ta2;
          int c2, b2;
          W.get(tn, tm2, ta2, c2, b2);
          tile_note_source(S, *ta2);
          tile_issue_setup<STAGE>(S, *tm2, c2, b2);
          tile_issue_state<STAGE>(S, *tm2, c2, b2);
          S.issued += 1;
        }
      }
    }
  }
  // The TMA stores this thread issued, then (after a failure) the loads
  // still in flight.
  if (tx == 0) bulk_wait_all();
  __syncthreads();
  if (tid == 0 && *abort_flag != 0)
    for (int j = 0; j < NBUF; j++)
      if (buf[j].issued > 0) mbar_wait_bounded(&buf[j].bar, (buf[j].issued - 1) & 1);
}

template <int STAGE>
__global__ void __launch_bounds__(kPersistThreads, 1)
    stage_persistent_kernel(const __grid_constant__ StageMaps T, const __grid_constant__ StageArgs A) {
  SingleWork W{&T, &A, (A.N / TC) * (A.M / kPersistRows), A.N / TC, kPersistRows};
  stage_persistent<STAGE, kPersistRows, kPersistThreads, 2, true>(W, A.err);
}

template <int STAGE>
__global__ void __launch_bounds__(kRingThreads, kRingBlocksPerSM)
    stage_ring_kernel(const __grid_constant__ StageMaps T, const __grid_constant__ StageArgs A) {
  SingleWork W{&T, &A, (A.N / TC) * (A.M / kRingRows), A.N / TC, kRingRows};
  stage_persistent<STAGE, kRingRows, kRingThreads, kRingBufs, false>(W, A.err);
}

template <int STAGE>
__global__ void __launch_bounds__(kPersistThreads, 1)
    stage_persistent_batch_kernel(const BatchSolve *solves, const __grid_constant__ BatchGroup G, int *err) {
  GroupWork<STAGE, kPersistRows> W{solves, &G};
  stage_persistent<STAGE, kPersistRows, kPersistThreads, 2, true>(W, err);
}

// The 8-row tilings over a batch work-list (tiles of 8 rows).
template <int STAGE>
__global__ void __launch_bounds__(kRingThreads, kRingBlocksPerSM)
    stage_ring_batch_kernel(const BatchSolve *solves, const __grid_constant__ BatchGroup G, int *err) {
  GroupWork<STAGE, kRingRows> W{solves, &G};
  stage_persistent<STAGE, kRingRows, kRingThreads, kRingBufs, false>(W, err);
}

template <int STAGE>
__global__ void __launch_bounds__(kNarrowThreads, 4)
    stage_narrow_batch_kernel(const BatchSolve *solves, const __grid_constant__ BatchGroup G, int ahead) {
  int c0, b0;
  const int i = group_item(G, blockIdx.x, 8, c0, b0);
  stage_tile<STAGE, 8, kNarrowThreads>(solves[G.solve[i]].maps[STAGE - 1], G.args[i], c0, b0,
                                       GroupAhead<STAGE, 8>{solves, &G, ahead});
}

// ---- stages 1 and 2 fused over column strips (the strip12 tiling) --------
// One 512-thread block per SM walks work items (column strip, theta
// segment).  A strip computes both stages on kStripCols = 128 columns (two
// 64-column warp segments): stage 1 from u^n into a shared-memory ring that
// holds u1, stage 2 from that ring.  Stage 2's outputs are stored on the
// strip's middle kStripOut = 120 columns only (its outer 4 on each side read
// stage-1 values outside the computed columns), so strips overlap by 8
// columns and u1 never goes to HBM: per grid point the launch reads u^n and
// bb (40 B) and writes u2 (32 B), where separate stage-1 and stage-2
// launches move 64 + 96 B (+16 B of bb).
// Rows go down a segment in phases of kStripG = 4: in phase p warps 0-7
// compute stage 1 on rows [R, R + 4), R = s1_lo + 4 p, and warps 8-15
// compute stage 2 on rows [R - 7, R - 3), whose theta stencil reaches u1
// rows up to R - 1, finished in earlier phases; one warp per row segment.
// The u^n rows reach shared memory by TMA one phase ahead (q planes 7 rows
// ahead of stage 1's rows, p planes and bb 4 rows ahead); column factors and
// row factors are loaded once per item.  At the start of every phase the
// closures of what arrived (u^n) and of what stage 1 finished (u1) are
// rebuilt in the rings, with the extrapolation order of the other kernels
// (HighOrder/kern.cu:320-449): pole rows of the q planes on columns
// [3, N-3), radial ends of all planes on interior rows.  Every point is
// computed by the same row work (tile_rows) from the same values as in the
// separate stage kernels, so results agree with them to rounding (the
// compiler's fused multiply-add choices may differ between instantiations).
constexpr int kStripThreads = 512;
constexpr int kStripCols = 2 * TC;            // computed columns per strip
constexpr int kStripOut = kStripCols - 8;     // stage-2 output columns per strip
constexpr int kStripWin = kStripCols + 8;     // window columns (stencils reach +-4)
constexpr int kStripG = 4;                    // rows per phase
constexpr int kStripLag = kStripG + 3;        // stage 2 trails stage 1 by this many rows
constexpr int kQRing = 24;                    // u^n q rows held (six 4-row chunks)
constexpr int kPRing = 16;                    // u^n p and bb rows held, and u1 rows (four chunks)
constexpr int kStripMaxRows = 264;            // stage-1 rows of one item (row-factor buffer)

struct __align__(128) StripSmem {
  alignas(128) double qn[2][kQRing][kStripWin];  // TMA boxes {136, 4, 1}: u^n q_re, q_im
  alignas(128) double pn[2][kPRing][kStripWin];  // u^n p_re, p_im
  alignas(128) double bb[kPRing][kStripWin];     // bb
  alignas(128) double q1[2][kPRing][kStripWin];  // u1 q_re, q_im (stage 1 output)
  alignas(128) double p1[2][kPRing][kStripWin];  // u1 p_re, p_im
  alignas(16) double cf[CF_TILE][kStripCols];    // column factors of the computed columns
  alignas(16) double rf[RF_COUNT][kStripMaxRows];  // row factors of the item's rows
  uint64_t bar[2];                               // loads of even / odd phases
  int src_c0, src_r0, src_buf;
};
BHR_TMA_ALIGNED(StripSmem, qn);
BHR_TMA_ALIGNED(StripSmem, pn);
BHR_TMA_ALIGNED(StripSmem, bb);
static_assert((4 * kStripWin * 8) % 128 == 0, "4-row TMA chunks must keep 128-byte alignment");
static_assert(sizeof(StripSmem) + 128 <= 227 * 1024, "strip buffers exceed shared memory");

// One item: column strip `s` (stage-2 outputs on columns [120 s, 120 s + 120)),
// stage-2 rows [s2_lo, s2_hi), stage-1 rows [s1_lo, s1_hi).
struct StripItem {
  int cs;        // first computed column: 120 s - 4
  int s1_lo, s1_hi, s2_lo, s2_hi;
  int st_lo, st_hi;  // stage-2 output columns
};

__device__ __forceinline__ StripItem strip_item(const StripGeom &G, const int N, const int M, const int item) {
  const int s = item % G.nstrips, g = item / G.nstrips;
  StripItem it;
  it.cs = kStripOut * s - 4;
  it.s2_lo = 3 + g * G.seg_rows;
  it.s2_hi = min(M - 3, it.s2_lo + G.seg_rows);
  it.s1_lo = max(3, it.s2_lo - 3);
  it.s1_hi = min(M - 3, it.s2_hi + 3);
  it.st_lo = max(3, kStripOut * s);
  it.st_hi = min(N - 3, kStripOut * s + kStripOut);
  return it;
}

// Ring rows: u^n q rows by (r - s1_lo + 5) mod 24 (no q row below
// s1_lo - 5 is read), everything else by (r - s1_lo) mod 16 (no row below
// s1_lo - 10 is read).  The 4-row TMA chunks land on 4-row-aligned slots.
static_assert(kPRing == 16, "pslot masks with 15");
__device__ __forceinline__ int qslot(int r, int base) {
  return static_cast<int>(static_cast<unsigned>(r - base + 5) % kQRing);
}
__device__ __forceinline__ int pslot(int r, int base) { return (r - base + 32) & (kPRing - 1); }

// The views the row work reads: stage 1 (u^n rings in, u1 ring out) and
// stage 2 (u1 rings in, u^n as the u^n term, global out).
template <int STAGE>
struct StripView {
  StripSmem &S;
  int b0, base, rf0, woff;
  __device__ __forceinline__ const double *qwin(int pl, int j) const {
    const int r = b0 - 3 + j;
    return STAGE == 1 ? &S.qn[pl][qslot(r, base)][0] : &S.q1[pl][pslot(r, base)][0];
  }
  __device__ __forceinline__ const double *prow(int pl, int r) const {
    return STAGE == 1 ? &S.pn[pl][pslot(b0 + r, base)][0] : &S.p1[pl][pslot(b0 + r, base)][0];
  }
  __device__ __forceinline__ const double *bbrow(int r) const { return &S.bb[pslot(b0 + r, base)][0]; }
  __device__ __forceinline__ const double *cf(int f) const { return S.cf[f]; }
  __device__ __forceinline__ double rf(int f, int r) const { return S.rf[f][b0 + r - rf0]; }
  // u^n at row b0 + r, indexed by the per-column index (window column - 4)
  __device__ __forceinline__ const double *unrow(int pl, int r) const {
    return (pl < 2 ? &S.qn[pl][qslot(b0 + r, base)][0] : &S.pn[pl - 2][pslot(b0 + r, base)][0]) + 4;
  }
  __device__ __forceinline__ double *outrow(int pl, int r) const {
    return pl < 2 ? &S.q1[pl][pslot(b0 + r, base)][0] : &S.p1[pl - 2][pslot(b0 + r, base)][0];
  }
};

// Extrapolation closure of pole rows of one q plane in a ring, on window
// columns whose grid column is in [3, N-3): the top rows 2, 1, 0 from rows
// 3, 4, or those of the bottom rows M-3, M-2, M-1 (in that order, each
// from the two rows above it) that lie in [lo, hi) -- the rows a TMA chunk
// just brought, so no later load overwrites them.
__device__ __forceinline__ void ring_close_poles(double (*q)[kStripWin], const bool top, const int M, const int N,
                                                 const int cs, const int base, const int even_m, const int tid,
                                                 const bool qring, const int lo, const int hi) {
  auto row = [&](int r) { return q[qring ? qslot(r, base) : pslot(r, base)]; };
  for (int w = tid; w < kStripWin; w += kStripThreads) {
    const int a = cs - 4 + w;
    if (a < 3 || a >= N - 3) continue;
    if (top) {
      if (even_m) {
        row(2)[w] = (4.0 * row(3)[w] - row(4)[w]) * kThird;
        row(1)[w] = (4.0 * row(2)[w] - row(3)[w]) * kThird;
        row(0)[w] = (4.0 * row(1)[w] - row(2)[w]) * kThird;
      } else {
        row(2)[w] = 0.0; row(1)[w] = 0.0; row(0)[w] = 0.0;
      }
    } else {
      for (int r = M - 3; r < M; r++) {
        if (r < lo || r >= hi) continue;
        row(r)[w] = even_m ? (4.0 * row(r - 1)[w] - row(r - 2)[w]) * kThird : 0.0;
      }
    }
  }
}

__device__ __forceinline__ void close_end_row(double *row, const int N, const int cs) {
  const int o = 4 - cs;  // window column of grid column a is a + o
  if (cs - 4 < 3) {
    row[2 + o] = (4.0 * row[3 + o] - row[4 + o]) * kThird;
    row[1 + o] = (4.0 * row[2 + o] - row[3 + o]) * kThird;
    row[0 + o] = (4.0 * row[1 + o] - row[2 + o]) * kThird;
  }
  // high end: only the closure columns inside the window (the last of
  // them may lie beyond it, where no computed column's stencil reaches)
  if (cs - 4 + kStripWin > N - 3) {
    if (N - 3 + o < kStripWin) row[N - 3 + o] = (4.0 * row[N - 4 + o] - row[N - 5 + o]) * kThird;
    if (N - 2 + o < kStripWin) row[N - 2 + o] = (4.0 * row[N - 3 + o] - row[N - 4 + o]) * kThird;
    if (N - 1 + o < kStripWin) row[N - 1 + o] = (4.0 * row[N - 2 + o] - row[N - 3 + o]) * kThird;
  }
}

// Thread 0: the loads a phase needs beyond the earlier phases' (first == true:
// everything phase 0 needs), on that phase's barrier.  q planes: rows
// [R + 3, R + 7) (first: [R - 5, R + 7)); p planes and bb: rows [R, R + 4).
__device__ __forceinline__ void strip_issue(StripSmem &S, const StripMaps &T, const StripItem &it, const int R,
                                            const bool first, uint64_t *bar) {
  const uint32_t chunk = 4 * kStripWin * sizeof(double);
  const int nq = first ? 3 : 1;
  mbar_expect_tx(bar, chunk * (2 * nq + 2 + 1));
  const int x = it.cs - 4;
  for (int c = 0; c < nq; c++) {
    const int r = first ? R - 5 + 4 * c : R + 3;
    const int sl = qslot(r, it.s1_lo);
    tma_load_3d(&S.qn[0][sl][0], &T.st, x, r, 0, bar);
    tma_load_3d(&S.qn[1][sl][0], &T.st, x, r, 1, bar);
  }
  const int sl = pslot(R, it.s1_lo);
  tma_load_3d(&S.pn[0][sl][0], &T.st, x, R, 2, bar);
  tma_load_3d(&S.pn[1][sl][0], &T.st, x, R, 3, bar);
  tma_load_3d(&S.bb[sl][0], &T.bb, x, R, 0, bar);
}

__global__ void __launch_bounds__(kStripThreads, 1)
    stage12_strip_kernel(const __grid_constant__ StripMaps T, const __grid_constant__ StageArgs A, const StripGeom G) {
  extern __shared__ unsigned char smem_raw[];
  StripSmem &S = *reinterpret_cast<StripSmem *>((reinterpret_cast<uintptr_t>(smem_raw) + 127) &
                                                ~static_cast<uintptr_t>(127));
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
  const int N = A.N, M = A.M;
  const int nitems = G.nstrips * G.segs;
  // stage-1 warps 0-7, stage-2 warps 8-15: row ty % 8 / 2 of the phase, half ty % 2
  const int grp = ty >> 3, wrow = (ty & 7) >> 1, half = ty & 1;
  if (tid == 0) {
    mbar_init(&S.bar[0], 1);
    mbar_init(&S.bar[1], 1);
    fence_barrier_init();
  }
  // u1 rows outside the grid are never read for a stored output; start them finite
  static_assert(sizeof(S.q1) == sizeof(S.p1), "u1 rings of equal size");
  constexpr int kU1Ring = static_cast<int>(sizeof(S.q1) / sizeof(double));  // 2 planes x 16 rows x 136
  for (int i = tid; i < kU1Ring; i += kStripThreads) {
    (&S.q1[0][0][0])[i] = 0.0;
    (&S.p1[0][0][0])[i] = 0.0;
  }
  grid_dependency_wait();
  launch_dependents();
  if (tid == 0 && A.src != nullptr) {
    const int k = A.rs->ks;
    S.src_c0 = A.recs[k].col0;
    S.src_r0 = A.recs[k].row0;
    S.src_buf = k & 1;
  }
  __syncthreads();
  const SrcNote note{S.src_c0, S.src_r0, S.src_buf};
  int ph = 0;  // phases run by this block so far (barrier parity)
  for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
    const StripItem it = strip_item(G, N, M, item);
    if (it.s2_lo >= it.s2_hi) continue;  // uniform across the block
    // set-up data of the item: column factors of the computed columns, row factors of its rows
    for (int i = tid; i < CF_TILE * kStripCols; i += kStripThreads) {
      const int f = i / kStripCols, j = i - f * kStripCols, a = it.cs + j;
      S.cf[f][j] = (a >= 0 && a < N) ? A.coltab[static_cast<size_t>(f) * N + a] : 0.0;
    }
    const int nrows1 = it.s1_hi - it.s1_lo;
    for (int i = tid; i < RF_COUNT * nrows1; i += kStripThreads) {
      const int f = i / nrows1, r = i - f * nrows1;
      S.rf[f][r] = A.rowtab[static_cast<size_t>(f) * M + it.s1_lo + r];
    }
    const bool lo_edge = it.cs - 4 < 3, hi_edge = it.cs - 4 + kStripWin > N - 3;
    const int nph = (it.s2_hi + 3 - it.s1_lo + kStripG - 1) / kStripG + 1;
    if (tid == 0) {
      fence_proxy_async();  // earlier generic writes of the rings before the async-proxy loads
      strip_issue(S, T, it, it.s1_lo, true, &S.bar[ph & 1]);
    }
    bool aborted = false;
    for (int p = 0; p < nph; p++, ph++) {
      const int R = it.s1_lo + kStripG * p;
      const bool ok = mbar_wait_bounded(&S.bar[ph & 1], (ph >> 1) & 1);
      if (!__syncthreads_and(ok)) {
        if (tid == 0) atomicCAS(A.err, 0, 5 /* BHR_TIMEOUT */);
        mbar_wait_bounded(&S.bar[ph & 1], (ph >> 1) & 1);
        aborted = true;
        break;
      }
      // Closures of what arrived for this phase (u^n q rows: the prologue's
      // or [R + 3, R + 7); p rows [R, R + 4)) and of the u1 rows stage 1
      // finished in the previous phase ([R - 4, R)): radial ends on interior
      // rows, pole rows on interior columns -- disjoint points, one pass.
      const int q_lo = p == 0 ? R - 5 : R + 3, q_hi = R + 7;
      const bool un_top = (p == 0 && it.s1_lo < 6);  // stage 1's window reaches rows 0..2
      const bool un_bot = q_lo < M && M - 3 < q_hi;  // some of rows M-3..M-1 arrived
      const bool u1_top = (p > 0 && R - kStripG <= 4 && 4 < R && it.s1_lo == 3);
      const bool u1_bot = (p > 0 && R - kStripG <= M - 4 && M - 4 < R && it.s1_hi == M - 3);
      if (lo_edge || hi_edge || un_top || un_bot || u1_top || u1_bot) {
        if (lo_edge || hi_edge) {
          const int nq = 2 * (q_hi - q_lo);
          for (int i = tid; i < nq + 2 * kStripG + (p > 0 ? 4 * kStripG : 0); i += kStripThreads) {
            double *row = nullptr;
            int r;
            if (i < nq) {
              r = q_lo + i / 2;
              row = &S.qn[i & 1][qslot(r, it.s1_lo)][0];
            } else if (i < nq + 2 * kStripG) {
              const int j = i - nq;
              r = R + j / 2;
              row = &S.pn[j & 1][pslot(r, it.s1_lo)][0];
            } else {
              const int j = i - nq - 2 * kStripG, pl = j & 3;
              r = R - kStripG + j / 4;
              if (r < it.s1_lo || r >= it.s1_hi) continue;
              row = pl < 2 ? &S.q1[pl][pslot(r, it.s1_lo)][0] : &S.p1[pl - 2][pslot(r, it.s1_lo)][0];
            }
            if (r >= 3 && r < M - 3) close_end_row(row, N, it.cs);
          }
        }
        for (int pl = 0; pl < 2; pl++) {
          if (un_top) ring_close_poles(S.qn[pl], true, M, N, it.cs, it.s1_lo, A.even_m, tid, true, 0, 0);
          if (un_bot) ring_close_poles(S.qn[pl], false, M, N, it.cs, it.s1_lo, A.even_m, tid, true, q_lo, q_hi);
          if (u1_top) ring_close_poles(S.q1[pl], true, M, N, it.cs, it.s1_lo, A.even_m, tid, false, 0, 0);
          if (u1_bot) ring_close_poles(S.q1[pl], false, M, N, it.cs, it.s1_lo, A.even_m, tid, false, M - 3, M);
        }
        __syncthreads();
      }
      // the next phase's rows (their ring slots are not read in this one)
      if (tid == 0) {
        fence_proxy_async();
        if (p + 1 < nph) strip_issue(S, T, it, R + kStripG, false, &S.bar[(ph + 1) & 1]);
      }
      if (grp == 0) {
        const int b = R + wrow;
        if (b >= it.s1_lo && b < it.s1_hi) {
          StripView<1> V{S, R, it.s1_lo, it.s1_lo, half * TC};
          const int c0 = it.cs + half * TC;
          tile_rows<1, 1, kOutRing, false>(V, A, c0, R, kStripG, tx, wrow, half * TC,
                                           c0 >= 4 && c0 + TC <= N - 4, 3, N - 3, note);
        }
      } else {
        const int R2 = R - kStripLag;
        const int b = R2 + wrow;
        if (b >= it.s2_lo && b < it.s2_hi) {
          StripView<2> V{S, R2, it.s1_lo, it.s1_lo, half * TC};
          const int c0 = it.cs + half * TC;
          tile_rows<2, 1, kOutGlobal, true>(V, A, c0, R2, kStripG, tx, wrow, half * TC,
                                            c0 >= 4 && c0 + TC <= N - 4, it.st_lo, it.st_hi, note);
        }
      }
      __syncthreads();
    }
    if (aborted) return;
  }
}

// ---- closure of stored planes (HighOrder/kern.cu:622-753) ------------------
__device__ __forceinline__ double pole_val(const double *P, int N, int M, int even, int b, int a) {
  if (b >= 3 && b < M - 3) return P[static_cast<size_t>(b) * N + a];
  if (!even) return 0.0;
  if (b < 3) {
    const double f3 = P[static_cast<size_t>(3) * N + a], f4 = P[static_cast<size_t>(4) * N + a];
    const double f2 = (4.0 * f3 - f4) * kThird;
    if (b == 2) return f2;
    const double f1 = (4.0 * f2 - f3) * kThird;
    if (b == 1) return f1;
    return (4.0 * f1 - f2) * kThird;
  }
  const double g4 = P[static_cast<size_t>(M - 4) * N + a], g5 = P[static_cast<size_t>(M - 5) * N + a];
  const double g3 = (4.0 * g4 - g5) * kThird;
  if (b == M - 3) return g3;
  const double g2 = (4.0 * g3 - g4) * kThird;
  if (b == M - 2) return g2;
  return (4.0 * g2 - g3) * kThird;
}

__device__ __forceinline__ double closed_val(const double *P, int N, int M, int even, int b, int a) {
  if (a >= 3 && a < N - 3) return pole_val(P, N, M, even, b, a);
  if (a < 3) {
    const double f3 = pole_val(P, N, M, even, b, 3), f4 = pole_val(P, N, M, even, b, 4);
    const double f2 = (4.0 * f3 - f4) * kThird;
    if (a == 2) return f2;
    const double f1 = (4.0 * f2 - f3) * kThird;
    if (a == 1) return f1;
    return (4.0 * f1 - f2) * kThird;
  }
  const double g4 = pole_val(P, N, M, even, b, N - 4), g5 = pole_val(P, N, M, even, b, N - 5);
  const double g3 = (4.0 * g4 - g5) * kThird;
  if (a == N - 3) return g3;
  const double g2 = (4.0 * g3 - g4) * kThird;
  if (a == N - 2) return g2;
  return (4.0 * g2 - g3) * kThird;
}

__global__ void closure_poles_kernel(double *P, int N, int M, int even) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  const int pl = blockIdx.y;
  if (a < 3 || a >= N - 3) return;
  double *Q = P + static_cast<size_t>(pl) * N * M;
  const double v0 = pole_val(Q, N, M, even, 0, a), v1 = pole_val(Q, N, M, even, 1, a),
               v2 = pole_val(Q, N, M, even, 2, a);
  const double w3 = pole_val(Q, N, M, even, M - 3, a), w2 = pole_val(Q, N, M, even, M - 2, a),
               w1 = pole_val(Q, N, M, even, M - 1, a);
  Q[a] = v0;
  Q[static_cast<size_t>(N) + a] = v1;
  Q[static_cast<size_t>(2) * N + a] = v2;
  Q[static_cast<size_t>(M - 3) * N + a] = w3;
  Q[static_cast<size_t>(M - 2) * N + a] = w2;
  Q[static_cast<size_t>(M - 1) * N + a] = w1;
}

__global__ void closure_ends_kernel(double *P, int N, int M) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  const int pl = blockIdx.y;
  if (b >= M) return;
  double *row = P + static_cast<size_t>(pl) * N * M + static_cast<size_t>(b) * N;
  row[2] = (4.0 * row[3] - row[4]) * kThird;
  row[N - 3] = (4.0 * row[N - 4] - row[N - 5]) * kThird;
  row[1] = (4.0 * row[2] - row[3]) * kThird;
  row[N - 2] = (4.0 * row[N - 3] - row[N - 4]) * kThird;
  row[0] = (4.0 * row[1] - row[2]) * kThird;
  row[N - 1] = (4.0 * row[N - 2] - row[N - 3]) * kThird;
}

// ---- particle source patch (HighOrder/kern.cu:1185-1227, 2666-2683) ---------
// The smeared delta is separable: the radial Gaussian factors R0..R2, the
// tilde-phi phase and Delta depend on the column only, the angular factors
// T0..T2 on the row only.  A block takes kSrcRows patch rows: each thread
// forms its column's factors once, the first threads form the rows'
// factors, and the per-point work is the bilinear sum and the epilogue.
constexpr int kSrcRows = 4;

__device__ __forceinline__ void source_rows(const SourceArgs &A, const int j0, const int k) {
  __shared__ double rowf[kSrcRows][5];  // T0, T1, T2, cos theta, sin theta
  __shared__ int rok[kSrcRows];
  // The patch of step k goes to buffer k % 2; a lookahead past the last
  // record builds nothing.
  const int kstep = A.rs->ks + A.lookahead;
  if (kstep >= A.nrecs) return;  // uniform across the block
  // By value: the stores to the patch below must not force reloads.
  const StepRec rec = A.recs[kstep];
  double *__restrict__ src = A.src + static_cast<size_t>(kstep & 1) * 2 * A.PTSX * A.PTSY;
  const double a = A.a, mass = A.mass;
  if (k < kSrcRows) {
    const int row = j0 + k + rec.row0;
    const bool ok = (j0 + k < A.PTSY) && row > 0 && row < A.M;
    rok[k] = ok;
    if (ok) {
      const double g0 = 1.0 / sqrt(2.0 * kPie);
      const double th = A.theta[row], wt = A.wt;
      const double dth = th - rec.tp;
      const double T0 = g0 * exp(-dth * dth / (2.0 * wt * wt)) / wt;
      rowf[k][0] = T0;
      rowf[k][1] = -dth / (wt * wt) * T0;
      rowf[k][2] = (-1.0 / (wt * wt) + dth * dth / (wt * wt * wt * wt)) * T0;
      rowf[k][3] = cos(th);
      rowf[k][4] = sin(th);
    }
  }
  __syncthreads();
  if (k >= A.PTSX) return;
  const int col = k + rec.col0;
  const bool cok = col > 0 && col < A.N;
  double r = 0.0, R0 = 0.0, R1 = 0.0, R2 = 0.0, cph = 0.0, sph = 0.0, delta = 0.0, c8 = 0.0, ra2 = 0.0;
  if (cok) {
    const double rpl = mass + sqrt(mass * mass - a * a), rmn = mass - sqrt(mass * mass - a * a);
    const double g0 = 1.0 / sqrt(2.0 * kPie);
    const double wr = rec.wr;
    r = A.r_c[col];
    const double dr = r - rec.rp;
    R0 = g0 * exp(-dr * dr / (2.0 * wr * wr)) / wr;
    R1 = -dr / (wr * wr) * R0;
    R2 = (-1.0 / (wr * wr) + dr * dr / (wr * wr * wr * wr)) * R0;
    const double ph = -A.m * a / (rpl - rmn) * log((r - rpl) / (r - rmn));
    sincos(ph, &sph, &cph);
    delta = r * r + a * a - 2.0 * mass * r;
    c8 = 8.0 * kPie * delta / (r * r * r);  // 8 pi Delta / r^3
    ra2 = (r * r + a * a) * (r * r + a * a);
  }
#pragma unroll
  for (int jj = 0; jj < kSrcRows; jj++) {
    const int j = j0 + jj;
    if (j >= A.PTSY) break;
    double sre = 0.0, sim = 0.0;
    if (cok && rok[jj]) {
      const double T0 = rowf[jj][0], T1 = rowf[jj][1], T2 = rowf[jj][2], ctv = rowf[jj][3], st = rowf[jj][4];
      const double bas[6] = {R0 * T0, R0 * T1, R0 * T2, R1 * T0, R1 * T1, R2 * T0};
      double tr = 0.0, ti = 0.0;
#pragma unroll
      for (int i = 0; i < 6; i++) {
        tr += rec.c_re[i] * bas[i];
        ti += rec.c_im[i] * bas[i];
      }
      // TT = Sigma * t / rho^4 with rho = -1/(r - i a cos): 1/rho^4 = (r - i a cos)^4.
      const double x = r, y = -a * ctv;
      const double x2 = x * x - y * y, y2 = 2.0 * x * y;        // (x+iy)^2
      const double x4 = x2 * x2 - y2 * y2, y4 = 2.0 * x2 * y2;  // (x+iy)^4
      const double sig = r * r + a * a * ctv * ctv;
      const double Tr = sig * (tr * x4 - ti * y4), Ti = sig * (tr * y4 + ti * x4);
      const double Ur = Tr * cph - Ti * sph, Ui = Tr * sph + Ti * cph;
      // 8 pi Delta U / (((r^2+a^2)^2 - a^2 Delta sin^2) r^3)
      const double f = c8 / (ra2 - a * a * delta * st * st);
      sre = f * Ur;
      sim = f * Ui;
    }
    src[static_cast<size_t>(j) * A.PTSX + k] = sre;
    src[static_cast<size_t>(A.PTSY + j) * A.PTSX + k] = sim;
  }
}

__global__ void source_patch_kernel(const SourceArgs A) {
  grid_dependency_wait();
  launch_dependents();
  source_rows(A, blockIdx.x * kSrcRows, threadIdx.x);
}

// Sourced solves of a batch: blockIdx.y picks the solve.
__global__ void source_batch_kernel(const SourceArgs *args) {
  grid_dependency_wait();
  launch_dependents();
  const SourceArgs &A = args[blockIdx.y];
  if (static_cast<int>(blockIdx.x) * kSrcRows < A.PTSY) source_rows(A, blockIdx.x * kSrcRows, threadIdx.x);
}

// ---- extraction, integration, projection (HighOrder/body.cu:168-212) ------
constexpr int kExtractThreads = 256;
constexpr int kSums = 15;

// Every kernel calls griddepcontrol.wait before it lets its dependents
// start, and a solver's extraction is ordered after the previous one
// through the step's stage 3 (which waits for it), so when this kernel
// starts, the previous step's extraction (the only writer of integ, rows,
// k, nrow and timer) has completed: those, and the weights written at
// set-up, are read before the wait; only psi at the extraction column waits
// for stage 3.
__device__ __forceinline__ void extract_body(const ExtractArgs &A) {
  __shared__ double red[kExtractThreads / 32][kSums];
  const int tid = threadIdx.x;
  const int N = A.N, M = A.M;
  const size_t NM = static_cast<size_t>(N) * M;
  const int k = A.rs->k;
  const int nrow = A.rs->nrow;
  const double timer = A.rs->timer;
  const bool out_step = ((k % A.Fr) == 0) && (static_cast<double>(k) * A.dt >= A.out_start);
  int bad = 0;
  double acc[kSums];
#pragma unroll
  for (int i = 0; i < kSums; i++) acc[i] = 0.0;
  for (int b = tid; b < M; b += kExtractThreads) {
    double in[4], wl[7], we = 0.0;
#pragma unroll
    for (int i = 0; i < 4; i++) in[i] = A.integ[i * M + b];
#pragma unroll
    for (int l = 0; l < 7; l++) wl[l] = out_step ? A.wproj[l * M + b] : 0.0;
    if (out_step) we = A.wdedt[b];
    if (b == tid) {
      grid_dependency_wait();
      launch_dependents();
    }
    const double psr = closed_val(A.u, N, M, A.even_m, b, A.ext_col);
    const double psi = closed_val(A.u + NM, N, M, A.even_m, b, A.ext_col);
    if (!isfinite(psr) || !isfinite(psi)) bad = 1;
    A.ext[b] = psr;
    A.ext[M + b] = psi;
    if (out_step && nrow < A.max_rows && A.psirows != nullptr) {
      A.psirows[(2 * static_cast<size_t>(nrow)) * M + b] = psr;
      A.psirows[(2 * static_cast<size_t>(nrow) + 1) * M + b] = psi;
    }
    const double ir = in[0] + psr * A.dt;
    const double ii = in[1] + psi * A.dt;
    const double dr = in[2] + ir * A.dt;
    const double di = in[3] + ii * A.dt;
    A.integ[b] = ir;
    A.integ[M + b] = ii;
    A.integ[2 * M + b] = dr;
    A.integ[3 * M + b] = di;
    if (out_step) {
#pragma unroll
      for (int l = 0; l < 7; l++) {
        acc[2 * l] += wl[l] * dr;
        acc[2 * l + 1] -= wl[l] * di;
      }
      acc[14] += (ir * ir + ii * ii) * we;
    }
  }
  if (tid >= M) {  // threads without a row still wait before the block ends
    grid_dependency_wait();
    launch_dependents();
  }
  if (out_step) {
#pragma unroll
    for (int i = 0; i < kSums; i++) {
      double v = acc[i];
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
      if ((tid & 31) == 0) red[tid >> 5][i] = v;
    }
  }
  const int any_bad = __syncthreads_or(bad);
  if (tid == 0) {
    if (any_bad) atomicCAS(&A.rs->err, 0, 4 /* BHR_NAN_DETECTED */);
    if (out_step && nrow < A.max_rows) {
      double *row = A.rows + static_cast<size_t>(nrow) * 16;
      row[0] = timer - A.Xmax;
      for (int i = 0; i < kSums; i++) {
        double v = 0.0;
        for (int w = 0; w < kExtractThreads / 32; w++) v += red[w][i];
        row[1 + i] = v;
      }
      A.rs->nrow = nrow + 1;
    }
    A.rs->timer = timer + A.dt;
    A.rs->k = k + 1;
    if (A.set_ks) A.rs->ks = k + 1;
  }
}

__global__ void __launch_bounds__(kExtractThreads) extract_kernel(const ExtractArgs A) { extract_body(A); }

// After a solver step's final stage: advance the stage step clock.  Its own
// launch, because every block of the final stage reads the clock.
__global__ void step_clock_kernel(RunState *rs) {
  grid_dependency_wait();
  launch_dependents();
  if (threadIdx.x == 0) rs->ks += 1;
}

// One block per solve of a batch.
__global__ void __launch_bounds__(kExtractThreads) extract_batch_kernel(const ExtractArgs *args) {
  extract_body(args[blockIdx.x]);
}

}  // namespace

// ---- host launchers -------------------------------------------------------
size_t stage_smem_bytes() { return sizeof(StageSmem<16>) + 128; }

static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    cudaDriverEntryPointQueryResult qr;
    void *fn = nullptr;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &qr);
    if (e != cudaSuccess || qr != cudaDriverEntryPointSuccess || !fn) return nullptr;
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  return encode;
}

cudaError_t encode_coef_maps(double *ctab, const double *coltab, const double *rowtab, int N, int M, int rows,
                             StageMaps *maps) {
  const cuuint32_t TRb = static_cast<cuuint32_t>(rows);
  auto encode = tensor_map_encoder();
  if (!encode) return cudaErrorNotSupported;
  const cuuint64_t dims[3] = {static_cast<cuuint64_t>(N), static_cast<cuuint64_t>(M), 1};
  const cuuint64_t strides[2] = {static_cast<cuuint64_t>(N) * 8, static_cast<cuuint64_t>(N) * M * 8};
  const cuuint32_t estr[3] = {1, 1, 1};
  const cuuint32_t box_bb[3] = {WC, TRb, 1};
  const cuuint64_t cdims[2] = {static_cast<cuuint64_t>(N), CF_COUNT};
  const cuuint64_t cstrides[1] = {static_cast<cuuint64_t>(N) * 8};
  const cuuint32_t box_cf[2] = {TC, CF_TILE};
  CUresult r1 = encode(&maps->coef_bb, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, ctab, dims, strides, box_bb, estr,
                       CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  CUresult r3 = encode(&maps->colf, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double *>(coltab), cdims, cstrides,
                       box_cf, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                       CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  const cuuint64_t rdims[2] = {static_cast<cuuint64_t>(M), RF_COUNT};
  const cuuint64_t rstrides[1] = {static_cast<cuuint64_t>(M) * 8};
  const cuuint32_t box_rf[2] = {TRb, RF_COUNT};
  CUresult r4 = encode(&maps->rowf, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double *>(rowtab), rdims, rstrides,
                       box_rf, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                       CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return (r1 == CUDA_SUCCESS && r3 == CUDA_SUCCESS && r4 == CUDA_SUCCESS) ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t launch_coef_tables(const double *coltab, const double *rowtab, double *ctab, int N, int M,
                               cudaStream_t st) {
  coef_table_kernel<<<dim3((N + 255) / 256, M), 256, 0, st>>>(coltab, rowtab, ctab, N, M);
  return cudaGetLastError();
}

cudaError_t encode_state_maps(void *planes, int N, int M, int rows, CUtensorMap *tm_q, CUtensorMap *tm_p,
                              CUtensorMap *tm_u) {
  const cuuint32_t TRb = static_cast<cuuint32_t>(rows);
  auto encode = tensor_map_encoder();
  if (!encode) return cudaErrorNotSupported;
  const cuuint64_t dims[3] = {static_cast<cuuint64_t>(N), static_cast<cuuint64_t>(M), 4};
  const cuuint64_t strides[2] = {static_cast<cuuint64_t>(N) * 8, static_cast<cuuint64_t>(N) * M * 8};
  const cuuint32_t estr[3] = {1, 1, 1};
  const cuuint32_t box_q[3] = {WC, TRb + 6, 2};
  const cuuint32_t box_p[3] = {WC, TRb, 2};
  CUresult r1 = encode(tm_q, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, planes, dims, strides, box_q, estr,
                       CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  CUresult r2 = encode(tm_p, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, planes, dims, strides, box_p, estr,
                       CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  CUresult r3 = CUDA_SUCCESS;
  if (tm_u) {
    const cuuint32_t box_u[3] = {TC, TRb, 4};
    r3 = encode(tm_u, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, planes, dims, strides, box_u, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  }
  return (r1 == CUDA_SUCCESS && r2 == CUDA_SUCCESS && r3 == CUDA_SUCCESS) ? cudaSuccess : cudaErrorInvalidValue;
}


// Multiprocessors of the current device (cached per device).
static int sm_count() {
  static int counts[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (counts[dev] == 0) {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    counts[dev] = n > 0 ? n : 148;
  }
  return counts[dev];
}

static size_t persist_smem_bytes() { return 2 * sizeof(StageSmem<kPersistRows>) + 128; }
static size_t ring_smem_bytes() { return kRingBufs * sizeof(StageSmem<kRingRows>) + 128; }

// Runtime stage number -> kernel template argument.
template <class F>
static cudaError_t by_stage(const int stage, F &&f) {
  switch (stage) {
    case 1: return f(std::integral_constant<int, 1>{});
    case 2: return f(std::integral_constant<int, 2>{});
    case 3: return f(std::integral_constant<int, 3>{});
    case 4: return f(std::integral_constant<int, 4>{});
    case 5: return f(std::integral_constant<int, 5>{});
    default: return cudaErrorInvalidValue;
  }
}

// Blocks ahead (in launch order) whose stage input a one-tile-per-block
// stage kernel prefetches into L2: twice the SM count (half a wave of
// block8n's four blocks per SM, one wave of block8's two) unless the caller
// asks for another distance (the solver's autotuner times a few), or
// BHR_PREFETCH_AHEAD (0 turns the prefetch off).  Measured at 16384 x 256,
// block8n: 220 us per step without, 203 us with 259-333 blocks ahead, 210
// at 592, 246 at 1184 (prefetched lines evicted before use).
int stage_prefetch_ahead(const int requested) {
  static const int env = [] {
    const char *v = std::getenv("BHR_PREFETCH_AHEAD");
    return v ? std::max(0, std::atoi(v)) : -1;
  }();
  if (env >= 0) return env;
  return requested >= 0 ? requested : 2 * sm_count();
}
int device_sm_count() { return sm_count(); }

cudaError_t launch_stage(int stage, const StageMaps &maps, const StageArgs &a_in, cudaStream_t st, bool pdl) {
  StageArgs a = a_in;
  a.ahead = (a.persist || a.ring) ? 0 : stage_prefetch_ahead(a.ahead);
  return by_stage(stage, [&](auto sc) {
    constexpr int S = decltype(sc)::value;
    if (a.narrow) {
      const size_t smem = sizeof(StageSmem<8>) + 128;
      return launch_ex(pdl, stage_narrow_kernel<S>, dim3(a.N / TC, a.M / 8), dim3(32, kNarrowThreads / 32), smem, st,
                       maps, a);
    }
    if (a.ring) {
      const int ntiles = (a.N / TC) * (a.M / kRingRows);
      return launch_ex(pdl, stage_ring_kernel<S>, dim3(std::min(ntiles, kRingBlocksPerSM * sm_count())),
                       dim3(32, kRingThreads / 32), ring_smem_bytes(), st, maps, a);
    }
    if (a.persist) {
      const int ntiles = (a.N / TC) * (a.M / kPersistRows);
      return launch_ex(pdl, stage_persistent_kernel<S>, dim3(std::min(ntiles, sm_count())),
                       dim3(32, kPersistThreads / 32), persist_smem_bytes(), st, maps, a);
    }
    const dim3 block(32, STAGE_THREADS / 32);
    if (a.rows == 8)
      return launch_ex(pdl, stage_kernel<S, 8>, dim3(a.N / TC, a.M / 8), block, sizeof(StageSmem<8>) + 128, st, maps,
                       a);
    return launch_ex(pdl, stage_kernel<S, 16>, dim3(a.N / TC, a.M / 16), block, sizeof(StageSmem<16>) + 128, st, maps,
                     a);
  });
}

// Once per device (the attribute is per device context).
cudaError_t prepare_kernels() {
  const int s8 = static_cast<int>(sizeof(StageSmem<8>) + 128), s16 = static_cast<int>(sizeof(StageSmem<16>) + 128);
  const int sp = static_cast<int>(persist_smem_bytes()), sr = static_cast<int>(ring_smem_bytes());
  constexpr auto kSmem = cudaFuncAttributeMaxDynamicSharedMemorySize;
  if (cudaError_t r = cudaFuncSetAttribute(stage12_strip_kernel, kSmem, static_cast<int>(strip_smem_bytes()))) return r;
  for (int stage = 1; stage <= 5; stage++) {
    const cudaError_t e = by_stage(stage, [&](auto sc) {
      constexpr int S = decltype(sc)::value;
      cudaError_t r;
      if ((r = cudaFuncSetAttribute(stage_kernel<S, 8>, kSmem, s8)) ||
          (r = cudaFuncSetAttribute(stage_kernel<S, 16>, kSmem, s16)) ||
          (r = cudaFuncSetAttribute(stage_narrow_kernel<S>, kSmem, s8)) ||
          (r = cudaFuncSetAttribute(stage_persistent_kernel<S>, kSmem, sp)) ||
          (r = cudaFuncSetAttribute(stage_ring_kernel<S>, kSmem, sr)))
        return r;
      if constexpr (S <= 3) {  // the batch engine steps SSP-RK3 only
        if ((r = cudaFuncSetAttribute(stage_batch_kernel<S, 8>, kSmem, s8)) ||
            (r = cudaFuncSetAttribute(stage_batch_kernel<S, 16>, kSmem, s16)) ||
            (r = cudaFuncSetAttribute(stage_persistent_batch_kernel<S>, kSmem, sp)) ||
            (r = cudaFuncSetAttribute(stage_narrow_batch_kernel<S>, kSmem, s8)) ||
            (r = cudaFuncSetAttribute(stage_ring_batch_kernel<S>, kSmem, sr)))
          return r;
      }
      return cudaSuccess;
    });
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_stage_batch(int stage, int tiling, const BatchSolve *solves, const BatchGroup &g, int *err,
                               cudaStream_t st) {
  const int ntiles = g.ntiles;
  if (ntiles <= 0) return cudaSuccess;
  if (stage < 1 || stage > 3) return cudaErrorInvalidValue;
  return by_stage(stage, [&](auto sc) {
    constexpr int S = decltype(sc)::value < 4 ? decltype(sc)::value : 1;
    switch (tiling) {
      case kTilingPersistent:
        return launch_pdl(stage_persistent_batch_kernel<S>, dim3(std::min(ntiles, sm_count())),
                          dim3(32, kPersistThreads / 32), persist_smem_bytes(), st, solves, g, err);
      case kTilingRing:
        return launch_pdl(stage_ring_batch_kernel<S>, dim3(std::min(ntiles, kRingBlocksPerSM * sm_count())),
                          dim3(32, kRingThreads / 32), ring_smem_bytes(), st, solves, g, err);
      case kTilingBlock8n:
        return launch_pdl(stage_narrow_batch_kernel<S>, dim3(ntiles), dim3(32, kNarrowThreads / 32),
                          sizeof(StageSmem<8>) + 128, st, solves, g, stage_prefetch_ahead());
      case kTilingBlock8:
        return launch_pdl(stage_batch_kernel<S, 8>, dim3(ntiles), dim3(32, STAGE_THREADS / 32),
                          sizeof(StageSmem<8>) + 128, st, solves, g, stage_prefetch_ahead());
      default:
        return launch_pdl(stage_batch_kernel<S, 16>, dim3(ntiles), dim3(32, STAGE_THREADS / 32),
                          sizeof(StageSmem<16>) + 128, st, solves, g, stage_prefetch_ahead());
    }
  });
}

size_t strip_smem_bytes() { return sizeof(StripSmem) + 128; }

cudaError_t encode_strip_maps(double *state, double *ctab, int N, int M, StripMaps *maps) {
  auto encode = tensor_map_encoder();
  if (!encode) return cudaErrorNotSupported;
  const cuuint32_t estr[3] = {1, 1, 1};
  const cuuint32_t box[3] = {kStripWin, kStripG, 1};
  const cuuint64_t dims[3] = {static_cast<cuuint64_t>(N), static_cast<cuuint64_t>(M), 4};
  const cuuint64_t strides[2] = {static_cast<cuuint64_t>(N) * 8, static_cast<cuuint64_t>(N) * M * 8};
  const cuuint64_t bdims[3] = {static_cast<cuuint64_t>(N), static_cast<cuuint64_t>(M), 1};
  CUresult r1 = encode(&maps->st, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, state, dims, strides, box, estr,
                       CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  CUresult r2 = encode(&maps->bb, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, ctab, bdims, strides, box, estr,
                       CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return (r1 == CUDA_SUCCESS && r2 == CUDA_SUCCESS) ? cudaSuccess : cudaErrorInvalidValue;
}

StripGeom strip_geometry(int N, int M) {
  StripGeom G{};
  G.nstrips = (N - 3 + kStripOut - 1) / kStripOut;
  const int rows = M - 6;
  const int max_seg = kStripMaxRows - 6;
  G.segs = std::max(std::max(1, sm_count() / G.nstrips), (rows + max_seg - 1) / max_seg);
  G.seg_rows = (rows + G.segs - 1) / G.segs;
  return G;
}

cudaError_t launch_stage12_strip(const StripMaps &maps, const StageArgs &a, cudaStream_t st, bool pdl) {
  const StripGeom G = strip_geometry(a.N, a.M);
  const int nitems = G.nstrips * G.segs;
  return launch_ex(pdl, stage12_strip_kernel, dim3(std::min(nitems, sm_count())), dim3(32, kStripThreads / 32),
                   strip_smem_bytes(), st, maps, a, G);
}

cudaError_t launch_source_batch(const SourceArgs *args, int nsolves, int max_ptsy, int max_ptsx, cudaStream_t st) {
  if (nsolves <= 0) return cudaSuccess;
  return launch_pdl(source_batch_kernel, dim3((max_ptsy + kSrcRows - 1) / kSrcRows, nsolves),
                    dim3(std::max(max_ptsx, kSrcRows)), 0, st, args);
}

cudaError_t launch_extract_batch(const ExtractArgs *args, int nsolves, cudaStream_t st) {
  if (nsolves <= 0) return cudaSuccess;
  return launch_pdl(extract_batch_kernel, dim3(nsolves), dim3(kExtractThreads), 0, st, args);
}

cudaError_t launch_source(const SourceArgs &a, cudaStream_t st) {
  return launch_pdl(source_patch_kernel, dim3((a.PTSY + kSrcRows - 1) / kSrcRows), dim3(std::max(a.PTSX, kSrcRows)), 0,
                    st, a);
}

cudaError_t launch_step_clock(RunState *rs, cudaStream_t st) { return launch_pdl(step_clock_kernel, dim3(1), dim3(32), 0, st, rs); }

cudaError_t launch_extract(const ExtractArgs &a, cudaStream_t st) {
  return launch_pdl(extract_kernel, dim3(1), dim3(kExtractThreads), 0, st, a);
}

// Gaussian initial data on the interior: q_re = fa[a] * gb[b] (the product
// the host would form; the closure is rebuilt by every reader).
__global__ void init_product_kernel(double *q, const double *fa, const double *gb, int N, int M) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x, b = blockIdx.y;
  if (a >= 3 && a < N - 3 && b >= 3 && b < M - 3) q[static_cast<size_t>(b) * N + a] = fa[a] * gb[b];
}

cudaError_t launch_init_product(double *q, const double *fa, const double *gb, int N, int M, cudaStream_t st) {
  init_product_kernel<<<dim3((N + 255) / 256, M), 256, 0, st>>>(q, fa, gb, N, M);
  return cudaGetLastError();
}

// Self-check of the bounded barrier wait every stage kernel uses: one block
// waits on an mbarrier that nothing completes; the wait gives up after its
// iteration limit and the kernel returns BHR_TIMEOUT (5) in *status instead
// of spinning forever.
__global__ void wait_selftest_kernel(int *status) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  const bool ok = mbar_wait_bounded(&bar, 0);
  if (threadIdx.x == 0) *status = ok ? 0 : 5;
}

cudaError_t launch_wait_selftest(int *status, cudaStream_t st) {
  wait_selftest_kernel<<<1, 32, 0, st>>>(status);
  return cudaGetLastError();
}

// Self-check of the Newton-refined reciprocal and square root the stage and
// table kernels use, beside CUDA's own correctly rounded 1.0 / x and
// sqrt(x): out = [rcp_nr(x) | 1.0 / x | sqrt_nr(x) | sqrt(x)], n each.
__global__ void math_selftest_kernel(const double *x, int n, double *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double v = x[i];
  out[i] = rcp_nr(v);
  out[n + i] = 1.0 / v;
  out[2 * n + i] = sqrt_nr(v);
  out[3 * n + i] = sqrt(v);
}

cudaError_t launch_math_selftest(const double *x, int n, double *out, cudaStream_t st) {
  math_selftest_kernel<<<(n + 255) / 256, 256, 0, st>>>(x, n, out);
  return cudaGetLastError();
}

cudaError_t launch_closure(double *planes, int N, int M, int even_m, cudaStream_t st) {
  closure_poles_kernel<<<dim3((N + 127) / 128, 4), 128, 0, st>>>(planes, N, M, even_m);
  closure_ends_kernel<<<dim3((M + 127) / 128, 4), 128, 0, st>>>(planes, N, M);
  return cudaGetLastError();
}

}  // namespace bhr
