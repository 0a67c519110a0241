// bhr_solver_impl.h -- the solve object shared by the C ABI (bhr_solver.cpp)
// and the batch engine (bhr_engine.cpp).  Not part of the public ABI.
#pragma once

#include <atomic>
#include <condition_variable>
#include <mutex>
#include <thread>

#include "bhr.h"
#include "bhr_host.h"
#include "bhr_internal.h"

struct bhr_solver {
  bhr_params p{};
  bhr::Grid g;
  int nt = 0, Fr = 1, max_rows = 0, ext_col = 0;
  bool even_m = true;
  bool has_source = false;
  cudaStream_t stream = nullptr;
  // The particle source of step k+1 is built on `side` while step k's
  // stages run: forked after step k-1's extraction, joined into step k's.
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr, fork2 = nullptr;
  // device memory
  double *u0 = nullptr, *u1 = nullptr, *u2 = nullptr;
  // classical RK4 (BHR_RK4): u1 holds y1 then y3, u2 y2, u3 z = (y1 + 2 y2 - u^n)/3
  bool rk4 = false;
  double *u3 = nullptr;
  double *coltab = nullptr, *rowtab = nullptr, *ctab = nullptr, *rc = nullptr, *th = nullptr;
  double *src = nullptr, *ext = nullptr, *integ = nullptr, *wproj = nullptr, *wdedt = nullptr, *rows = nullptr;
  double *psirows = nullptr;  // psi(theta) at the extraction column per waveform row
  // mixed precision (BHR_MIXED): FP32 delta1 and eps2 planes, FP32 tables
  bool mixed = false;
  float *d1f = nullptr, *e2f = nullptr, *colf32 = nullptr, *rowf32 = nullptr, *bbf = nullptr;
  bhr::MixedMaps mmaps[2];  // stages 2 and 3
  bhr::StepRec *recs = nullptr;
  bhr::RunState *rs = nullptr;
  size_t bytes = 0;
  // Per stage: input state, u^n slot and TMA store target.  SSP-RK3 uses
  // 0..2 (u^n -> u1, u1 -> u2, u2 -> u^n); RK4 uses 0, 1, 3 (u2 -> u1) and
  // 4 (u1 with z -> u^n).
  bhr::StageMaps maps[5];
  int tile_rows = 16; // stage tile height chosen for this grid
  int persist = 0;     // 1: persistent stage kernels (16-row tiles, one block per SM)
  int narrow = 0;      // 1: 8-row tiles on 128-thread blocks (four per SM)
  int ahead = -1;      // L2 prefetch distance of the one-tile-per-block stage kernels (-1: default)
  int ring = 0;        // 1: 8-row tiles through 2-buffer rings, two 256-thread blocks per SM
  int strip12 = 0;     // 1: stages 1 and 2 in one launch over column strips (FP64 SSP-RK3; stage 3 block8n)
  bhr::StripMaps smaps;
  int steps_done = 0;
  // The extraction of the last step launched has not been launched yet: it
  // runs beside the next step's first stages, or before a host read.
  bool pending_extract = false;
  // Captured step graphs: one step, and kGraphBatch steps in one launch.
  cudaGraphExec_t g1 = nullptr, gb = nullptr;
  // Per-step source records past the first chunk are built and uploaded by
  // a host thread after set_trajectory returns; stepping waits for the
  // steps it reaches (lock rec_mu).
  std::thread rec_thread;
  std::mutex rec_mu;
  std::condition_variable rec_cv;
  std::atomic<bool> rec_stop{false};
  int rec_ready = 0;                // records on the device: steps [0, rec_ready)
  int rec_bad = -1;                 // first step whose record failed, or -1
  int rec_status = 0;               // its status
  bool rec_running = false;         // a record thread may still publish records
  bool rec_unusable = false;        // a trajectory change failed after the old records were dropped
};


namespace bhr {
// Creates a solve; tile_rows 0 lets the autotuner (or BHR_STAGE_TILING) pick
// the stage tiling, 8 or 16 fixes one-tile-per-block kernels of that height
// (the batch engine's choice, whose own kernels read the solve's maps).
int solver_create(const bhr_params *p, int tile_rows, bhr_solver **out);
// Launch arguments of the solve's kernels (stage pointers vin/un/out unset).
StageArgs solver_stage_args(bhr_solver *s);
SourceArgs solver_source_args(bhr_solver *s);
ExtractArgs solver_extract_args(bhr_solver *s);
MixedArgs solver_mixed_args(bhr_solver *s);
// Waits until the source records of steps [0, upto) are on the device
// (returns the status of a record that failed before upto).
int solver_wait_records(bhr_solver *s, int upto);
}  // namespace bhr
