// bhr_internal.h -- shared definitions between the host code (bhr_solver.cpp)
// and the sm_100a kernels (bhr_kernels.cu).  Not part of the public ABI.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace bhr {

// Stage tile: TC radial columns x TR theta rows per CTA.  The loaded window
// adds 4 columns each side (the Kreiss-Oliger stencil reaches +-4,
// HighOrder/kern.cu:247-256) and 3 rows each side for q (the 6th-order
// theta stencils reach +-3, HighOrder/kern.cu:206-222).
constexpr int TC = 64;
constexpr int TR = 16;       // largest tile height; tiles are 8 or 16 rows
constexpr int WC = TC + 8;   // window columns
constexpr int STAGE_THREADS = 256;

// Per-column coefficient factors (host-built, FP64).  With bir = B0 +
// B1*sin^2(theta) every coefficient of HighOrder/kern.cu:132-158 is a
// per-column numerator, a per-row factor and 1/bir.
enum ColField {
  // The first CF_TILE factors are the ones every FP64 stage tile loads.
  CF_B0 = 0,   // -(2 cL - Om^2) Sg^2 / cL^2
  CF_DT,       // Dt; with the solve's a^2 and -4a it also gives B1, CCN,
               // CR1 and BI1 below, which the FP64 stage kernels form per point
  CF_ATN,      // 2 (cL - Om^2) Sg^2 / cL^2        Ataurho = ATN / bir
  CF_XR,       // BtauReal * bir
  CF_YR,       // BrhoReal * bir
  CF_CR0,      // CReal * bir, theta-free part
  CF_BI0,      // BtauImag * bir, theta-free part
  CF_BRI,      // BrhoImag * bir
  CF_CIN,      // CImag * bir
  CF_TILE,
  CF_ARN = CF_TILE,  // -Om^2 Sg^2 / cL^2          Arhorho = ARN / bir (the bb table only)
  CF_B1,       // a^2 Dt
  CF_CCN,      // -Dt                              Ayy     = CCN / bir
  CF_CR1,      // Dt: multiplies g(theta) = 4cot^2 - 4m cot csc + m^2 csc^2
  CF_BI1,      // -4 a Dt: multiplies cos(theta)
  CF_COUNT
};
enum RowField { RF_S2 = 0, RF_COS, RF_G, RF_CTAN, RF_COUNT };

// One step's particle source, prepared on the host from the trajectory.
struct StepRec {
  double c_re[6], c_im[6];  // bilinear coefficients times the turn-on window
  double rp, tp, wr;        // particle r, theta and the radial width
  int col0, row0;           // patch origin: ip - PTSX/2, it - PTSY/2
};

// Device-side run counters, advanced on the device so a captured step graph
// can be replayed.  Two step clocks: `ks` (steps whose stages are done; it
// selects the step's source record and patch buffer) is advanced by a
// one-thread kernel after a solver step's final stage, or by the extraction
// where stages and extraction run in sequence (batch engine); `k` (steps
// extracted; the waveform's clock) by the extraction kernel.  A solver runs
// the extraction of step n beside stage 2 of step n+1, so until it has run
// k == ks - 1.
struct RunState {
  int k;          // steps extracted
  int nrow;       // waveform rows written
  int err;        // bhr_status of the first device-detected failure
  int ks;         // steps whose stages are done
  double timer;   // accumulated as timer += dt (HighOrder/body.cu:214)
};

struct StageArgs {
  const double *vin;    // stage input planes (also the TMA source)
  const double *un;     // u^n planes (stages 2 and 3)
  double *out;          // output planes
  const double *coltab; // [CF_COUNT][N]
  const double *rowtab; // [RF_COUNT][M]
  const double *src;    // source patch buffers [2][2][PTSY][PTSX] (step k: buffer k % 2) or nullptr
  const StepRec *recs;  // per-step records or nullptr
  const RunState *rs;
  int *err;
  int N, M, PTSX, PTSY;
  int even_m;
  int rows;             // tile height: 8 or 16 theta rows
  int persist;          // 1: 16-row tiles walked by one persistent block per SM
  int narrow;           // 1: 8-row tiles on 128-thread blocks (four per SM)
  int ring;             // 1: 8-row tiles walked by two 256-thread blocks per SM, two buffers each
  int ahead;            // one-tile-per-block kernels: each block prefetches into L2 the stage
                        // input of the block this many places later in launch order (0: none,
                        // -1: stage_prefetch_ahead's default; launch_stage resolves it)
  float *dout;          // mixed precision, stage 1: delta1 = dt L(u^n) in FP32, or nullptr
  double *zout;         // RK4 stage 2: z = (y1 + 2 y2 - u^n)/3, or nullptr
  double dt;            // the stage's step in the combination (RK4: dt/2, dt, dt/6)
  double cx, cy, cyy, cko;
  double a2, m4a;       // a^2 and -4a: B1 = a2 Dt and BI1 = m4a Dt, the products the column table holds
};

struct SourceArgs {
  double *src;          // two patch buffers [2][2][PTSY][PTSX]: step k's patch in buffer k % 2
  const StepRec *recs;
  const RunState *rs;
  const double *r_c;    // [N]
  const double *theta;  // [M]
  int N, M, PTSX, PTSY;
  int lookahead;        // the patch built is for step rs->ks + lookahead (0 or 1)
  int nrecs;            // steps with a record; later steps are skipped
  double a, mass, m, wt;
};

struct ExtractArgs {
  const double *u;      // u^n planes after the step
  double *ext;          // [2][M] psi at ext_col
  double *integ;        // [4][M] int_re, int_im, dint_re, dint_im
  const double *wproj;  // [7][M] Boole x swsh projection weights
  const double *wdedt;  // [M]
  double *rows;         // [max_rows][16]: t, h+/hx x 7, dedt
  double *psirows;      // [max_rows][2][M]: psi at the extraction column on each row's step, or nullptr
  RunState *rs;
  int N, M, ext_col, Fr, max_rows, even_m;
  int set_ks;           // 1: also advance rs->ks (stages and extraction in sequence)
  double dt, out_start, Xmax;
};

// Launchers (bhr_kernels.cu).
// Tensor maps a stage kernel reads through: the input state (q with halo,
// p with column halo), u^n (bare tile, stages 2 and 3), the per-point
// coefficient planes (bb with column halo; 1/bir and ee) and the column
// factor table.
struct StageMaps {
  CUtensorMap q, p, u, coef_bb, colf, rowf;
  CUtensorMap o;  // stage output planes, box {TC, rows, 4} (TMA stores)
};

// One launch's share of a batch work-list: up to kGroupSolves solves whose
// tiles follow one another in launch order, each solve's row band by row
// band (TC columns by the kernel's tile height).  The stage arguments travel
// in the kernel's parameter space, where the stage kernels read them as
// they read a lone solve's (constant-bank operands, no loads from global
// memory in the row loops); each block finds its solve by a binary search
// over `first`.  The tensor maps stay in the batch's solve table.
constexpr int kGroupSolves = 112;
template <class Args>
struct WorkGroup {
  int nsolves, ntiles;
  int first[kGroupSolves + 1];  // each solve's first work item; first[nsolves] = ntiles
  int tiles_x[kGroupSolves];    // TC-column tiles per row band (N / TC)
  int solve[kGroupSolves];      // the solve's row in the batch's solve table
  Args args[kGroupSolves];
};
using BatchGroup = WorkGroup<StageArgs>;
static_assert(sizeof(BatchGroup) + 64 <= 32764, "a kernel's parameters are limited to 32764 bytes");

// Fused stages 1 and 2 over column strips (tiling kTilingStrip12): the state
// and bb planes read in 136-column x 4-row boxes.
struct StripMaps {
  CUtensorMap st, bb;
};
// Column strips of 120 output columns; theta segments of seg_rows stage-2
// rows; one work item per (strip, segment).
struct StripGeom {
  int nstrips, segs, seg_rows;
};
StripGeom strip_geometry(int N, int M);
size_t strip_smem_bytes();
cudaError_t encode_strip_maps(double *state, double *ctab, int N, int M, StripMaps *maps);
// Stages 1 and 2 of one SSP-RK3 step in one launch: reads u^n, writes u2
// (a.out) on the interior; u1 stays in shared memory.
cudaError_t launch_stage12_strip(const StripMaps &maps, const StageArgs &a, cudaStream_t st, bool pdl = true);

// Mixed precision (BHR_MIXED): SSP-RK3 rearranged so that FP32 carries only
// O(dt^2) corrections.  With delta1 = dt L(u^n) (L with the source) and L0
// the homogeneous operator,
//   u1      = u^n + delta1                       (FP64, the FP64 stage 1)
//   eps2    = dt/4 L0(delta1)                    (FP32 stage 2)
//   u^{n+1} = u1 + 2 eps2 + (2/3) dt L0(eps2)    (FP32 stage 3, FP64 sum)
// which is the Shu-Osher scheme exactly in exact arithmetic (L is affine).
struct MixedMaps {
  CUtensorMap q, p;     // FP32 input planes (delta1 or eps2), halo boxes
  CUtensorMap bb;       // FP32 planes bb, ee, d_re, d_im (tile box)
  CUtensorMap colf, rowf;  // FP32 column / row factor tables
  CUtensorMap u1;       // stage 3: FP64 u1 planes, tile box
};
struct MixedArgs {
  float *e_out;         // stage 2: eps2 planes
  double *u_out;        // stage 3: u^{n+1} planes
  int *err;
  int N, M, even_m;
  float dt, cx, cy, cyy, cko;
};
struct MixedBatch {
  MixedMaps maps[2];    // stages 2 and 3
  MixedArgs args[2];
};
using MixedGroup = WorkGroup<MixedArgs>;
static_assert(sizeof(MixedGroup) + 64 <= 32764, "a kernel's parameters are limited to 32764 bytes");
cudaError_t encode_mixed_maps(const float *in, const float *bbf, const float *colf, const float *rowf,
                              const double *u1, int N, int M, MixedMaps *maps);
cudaError_t launch_mixed_stage(int stage, const MixedMaps &maps, const MixedArgs &a, cudaStream_t st);
// One launch of a mixed stage over a group of mixed solves (16-row tiles).
cudaError_t launch_mixed_batch(int stage, const MixedBatch *solves, const MixedGroup &g, cudaStream_t st);
cudaError_t launch_to_float(const double *src, float *dst, size_t n, cudaStream_t st);
// kc[4][M][N] (FP32): bb, ee, d_re, d_im formed in FP64 from the tables.
cudaError_t launch_mixed_coef(const double *coltab, const double *rowtab, const double *bbt, float *kc, int N, int M,
                              double cx, cudaStream_t st);
cudaError_t prepare_mixed_kernels();

// A batch of solves advanced together: per solve, the tensor maps and
// arguments of its three stages (the arguments are copied into the launch
// groups).
struct BatchSolve {
  StageMaps maps[3];
  StageArgs args[3];
};

// Tensor maps of one state (four M x N planes): q planes with the +-3 row
// and +-4 column halo, p planes with the column halo, and (tm_u, may be
// null) the bare tile of all four planes for reading u^n.
cudaError_t encode_state_maps(void *planes, int N, int M, int rows, CUtensorMap *tm_q, CUtensorMap *tm_p,
                              CUtensorMap *tm_u);
// pdl = false launches without programmatic serialisation: the stage then
// starts only once everything before it on the stream has completed (for a
// first launch after tables were rewritten, which the stage kernels read
// before their grid-dependency wait).
cudaError_t launch_stage(int stage, const StageMaps &maps, const StageArgs &a, cudaStream_t st, bool pdl = true);
cudaError_t launch_step_clock(RunState *rs, cudaStream_t st);
// Per-point coefficient planes [bb | 1/bir | ee] (3 x M x N) from the tables,
// and the tensor maps over them and over the column table.
cudaError_t launch_coef_tables(const double *coltab, const double *rowtab, double *ctab, int N, int M,
                               cudaStream_t st);
cudaError_t encode_coef_maps(double *ctab, const double *coltab, const double *rowtab, int N, int M, int rows,
                             StageMaps *maps);
cudaError_t launch_source(const SourceArgs &a, cudaStream_t st);
// persist = 1 walks the work-list with one block per SM (16-row tiles);
// err receives BHR_TIMEOUT if a bounded wait gives up.
// Stage tilings (the values of bhr_tiling): kernels and tile heights.
enum StageTiling {
  kTilingBlock8 = 0,
  kTilingBlock16 = 1,
  kTilingPersistent = 2,
  kTilingBlock8n = 3,
  kTilingRing = 4,
  kTilingStrip12 = 5  // stages 1 and 2 fused (launch_stage12_strip), stage 3 as block8n
};
constexpr int tiling_rows(int tiling) {
  return (tiling == kTilingBlock8 || tiling == kTilingBlock8n || tiling == kTilingRing) ? 8 : 16;
}
// Tile height of the mixed-precision FP32 stage kernels.
constexpr int kMixTileRows = 16;
// One launch of an FP64 stage over a group of a batch's solves (tiles of the
// tiling's height).
cudaError_t launch_stage_batch(int stage, int tiling, const BatchSolve *solves, const BatchGroup &g, int *err,
                               cudaStream_t st);
cudaError_t launch_source_batch(const SourceArgs *args, int nsolves, int max_ptsy, int max_ptsx, cudaStream_t st);
cudaError_t launch_extract_batch(const ExtractArgs *args, int nsolves, cudaStream_t st);
cudaError_t launch_extract(const ExtractArgs &a, cudaStream_t st);
cudaError_t launch_closure(double *planes, int N, int M, int even_m, cudaStream_t st);
cudaError_t launch_wait_selftest(int *status, cudaStream_t st);
cudaError_t launch_math_selftest(const double *x, int n, double *out, cudaStream_t st);
cudaError_t launch_init_product(double *q, const double *fa, const double *gb, int N, int M, cudaStream_t st);
size_t stage_smem_bytes();
cudaError_t prepare_kernels();
// Blocks ahead (in launch order) whose input a one-tile-per-block stage
// kernel prefetches into L2: BHR_PREFETCH_AHEAD when set (0: no prefetch),
// else `requested` when >= 0, else twice the SM count.
int stage_prefetch_ahead(int requested = -1);
// The device's SM count (cached per device).
int device_sm_count();

}  // namespace bhr
