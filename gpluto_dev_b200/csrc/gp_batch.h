// gp_batch.h -- device-side tables of the batched step (many independent
// grids advanced together by persistent launches).
//
// Each grid ("slot") keeps its own state in a region of one device pool, its
// own dt sequence and step budget.  An RK stage is two persistent launches
// over all slots: the sweep launch (register-heavy Riemann work, 3 blocks
// per SM) takes every sweep tile; the cell launch (edge EMFs and the stage
// finish, latency-bound, 8 blocks per SM) takes every EMF tile, then every
// finish tile.  A finish tile of slot s waits until every EMF tile of s has
// completed (per-slot counters).  Tiles are taken from an atomic queue head
// in table order, so a waiting tile only ever waits on tiles that running
// blocks have already taken: progress does not depend on how many blocks
// are resident.
#pragma once
#include <cstdint>

#include "gp_kernels.cuh"

namespace gp {

enum BatchPhase { BP_SWEEP_X = 0, BP_SWEEP_Y = 1, BP_SWEEP_Z = 2, BP_EMF = 3, BP_FINISH = 4 };
enum BatchGroup { BG_SWEEPS = 0, BG_EMF = 1, BG_FINISH = 2, BG_COUNT = 3 };

constexpr int BATCH_THREADS = SWEEP_THREADS;  // 4 warps per block, every phase
constexpr int BATCH_ROWS_PER_TILE = BATCH_THREADS / 32;

struct BatchTile {
  int slot;
  int phase;
  int idx;  // tile index within (slot, phase)
  int pad;
};

// Per-slot scalars, written by the device (the last finish tile of a step).
struct BatchScalars {
  double dt;                      // dt of the step about to run
  double dtdx[3];                 // dt / dx_d
  double invdt;                   // invDt_hyp of the last completed step
  unsigned long long invdt_bits;  // running max of C_dt over stage 1
  uint32_t err;                   // OR of error bits
  int bcur;                       // face buffer holding B^n
  int steps_left;                 // steps still to run (0: idle)
  int steps_done;
};

// Per-slot description (written by the host when the slot is admitted).
struct BatchSlot {
  int physics, ndim, precision, nvar;
  int nx, ny, nz;
  int seg;                 // pencil segment of the y/z sweeps
  int cpt;                 // cells per thread of the EMF and finish tiles
  int ntiles[5];           // tiles per phase
  int need[BG_COUNT];      // tiles per group
  long long n;
  double cfl, cfl_max_var;
  double dx[3];
  BatchScalars* sc;
  // StageArgs for [stage-1][bcur]; the dU, Cdt, UCT-data and EMF pointers
  // are float* in the mixed form (same layout: every member of
  // StageArgs<double> and StageArgs<float> has the same size and offset).
  StageArgs<double> sa[2][3];
};

static_assert(sizeof(StageArgs<double>) == sizeof(StageArgs<float>), "StageArgs layout");

// Tile table header: tiles [0, nsweep) are sweep tiles, [nsweep, ntiles)
// EMF then finish tiles.
struct BatchTableHeader {
  int nsweep;
  int ntiles;
  long long spin_limit;  // polls before a dependency wait gives up
  int bias_slot;         // fault injection (tests): this slot's EMF count
  int bias_need;         //   must reach need + bias_need; -1 / 0 = off
};

// Queue heads of the two launches and per-slot group counters; cleared
// before every stage.
struct BatchCounters {
  int head[2];
  int pad[30];
  int done[1];  // [max_slots][BG_COUNT]
};

// Tile dispatch, one per part and precision form (separate translation
// units of relocatable device code: the FP64 form is compiled without
// contraction so that it keeps the reference's rounding, the mixed form with
// it; the sweep part with the sweeps' register budget, the cell part with a
// small one).  Called by every thread of the block.
__device__ void batch_sweep_tile_fp64(const BatchSlot& s, const BatchTile& t, int stage,
                                      double* smem);
__device__ void batch_sweep_tile_mixed(const BatchSlot& s, const BatchTile& t, int stage,
                                       double* smem);
__device__ void batch_cell_tile_fp64(const BatchSlot& s, const BatchTile& t, int stage);
__device__ void batch_cell_tile_mixed(const BatchSlot& s, const BatchTile& t, int stage);

#ifndef GP_CELL_MINB
#define GP_CELL_MINB 8
#endif

// Shared memory a block needs (largest staging area of any phase).
constexpr int batch_smem_bytes() {
  return (int)sizeof(double) * sweep_x_stage_doubles<8>();
}

}  // namespace gp
