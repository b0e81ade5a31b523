// gp_batch_tiles.cu -- one tile of a batched stage: the same per-row,
// per-column and per-cell bodies as the single-grid kernels, applied to one
// slot's StageArgs.  Compiled four times as relocatable device code:
// GP_BATCH_PART=0 (sweep tiles) or 1 (EMF and finish tiles), each with
// GP_MIXED=0 (FP64, -fmad=false: bit-identical to the single-grid FP64 step)
// and GP_MIXED=1 (FP32 reconstruction/Riemann/EMF, contraction allowed).
//
// Schemes built for batches: ideal MHD with PLM-MC + HLLD + UCT_HLLD,
// relativistic MHD with PLM-MC + HLLD + UCT_HLL, and hydrodynamics with
// PLM-MC + HLLC, in 2-D and 3-D; the host refuses any other combination.
#include "gp_batch.h"

#ifndef GP_MIXED
#define GP_MIXED 0
#endif
#ifndef GP_BATCH_PART
#define GP_BATCH_PART 0
#endif

namespace gp {

#if GP_MIXED
using RT = float;
using CTT = float;
#if GP_BATCH_PART == 0
#define GP_BATCH_TILE batch_sweep_tile_mixed
#else
#define GP_BATCH_TILE batch_cell_tile_mixed
#endif
#else
using RT = double;
using CTT = double;
#if GP_BATCH_PART == 0
#define GP_BATCH_TILE batch_sweep_tile_fp64
#else
#define GP_BATCH_TILE batch_cell_tile_fp64
#endif
#endif

namespace {

// y/z sweep work item -> (x column, transverse index, segment); items run x
// fastest so that the threads of a block read contiguous cells.
template <int PHYS, int NV, int NDIM, int RS, int CT, int LIM, int DIR>
__device__ __forceinline__ void sweep_m_item(const StageArgs<CTT>& a, const Grid3& g, int S,
                                             long long item, double* smem, int tid) {
  const int nd = DIR == 1 ? g.ny : g.nz;
  const int ntr = DIR == 1 ? g.nz : g.ny;
  const int nseg = (nd + S - 1) / S;
  const long long items = (long long)g.nx * nseg * ntr;
  if (item >= items) return;
  const int i = (int)(item % g.nx);
  const long long r = item / g.nx;
  const int seg = (int)(r % nseg);
  const int t = (int)(r / nseg);
  sweep_m_col<PHYS, NV, NDIM, RS, CT, LIM, DIR, RT, CTT>(a, g, i, t, seg, S, smem, tid);
}

// One non-inlined function per (scheme, phase): each gets its own register
// allocation, as the single-grid kernels do, instead of one allocation over
// the union of every phase of every scheme.
template <int PHYS, int NV, int NDIM, int RS, int CT, int LIM>
__device__ __noinline__ void tile_sweep_x(const StageArgs<CTT>& a, Grid3 g, int idx,
                                          double* smem) {
  const int tid = threadIdx.x;
  sweep_x_row<PHYS, NV, NDIM, RS, CT, LIM, RT, CTT>(a, g, idx * BATCH_ROWS_PER_TILE + (tid >> 5),
                                                    smem, tid);
}

template <int PHYS, int NV, int NDIM, int RS, int CT, int LIM, int DIR>
__device__ __noinline__ void tile_sweep_m(const StageArgs<CTT>& a, Grid3 g, int seg, int idx,
                                          double* smem) {
  const int tid = threadIdx.x;
  sweep_m_item<PHYS, NV, NDIM, RS, CT, LIM, DIR>(a, g, seg, (long long)idx * BATCH_THREADS + tid,
                                                 smem, tid);
}

template <int NDIM, int LIM>
__device__ __noinline__ void tile_emf(const StageArgs<CTT>& a, Grid3 g, int cpt, int idx) {
  const long long c0 = (long long)idx * BATCH_THREADS * cpt + threadIdx.x;
  for (int q = 0; q < cpt; q++) emf_cell<NDIM, LIM, RT, CTT>(a, g, c0 + (long long)q * BATCH_THREADS);
}

template <int PHYS, int NV, int NDIM>
__device__ __noinline__ void tile_finish(const StageArgs<CTT>& a, Grid3 g, int cpt, int idx,
                                         int stage) {
  const long long c0 = (long long)idx * BATCH_THREADS * cpt + threadIdx.x;
  double mx = 0.0;
  for (int q = 0; q < cpt; q++) {
    const double cdt = finish_cell<PHYS, NV, NDIM, CTT>(a, g, c0 + (long long)q * BATCH_THREADS);
    mx = GP_MAX(mx, cdt);
  }
  if (stage == 1) warp_invdt_max(a.invdt_bits, mx, threadIdx.x & 31);
}

template <int PHYS, int NV, int NDIM, int RS, int CT, int LIM>
__device__ __forceinline__ void run_tile(const StageArgs<CTT>& a, const Grid3& g, int seg,
                                         int cpt, int phase, int idx, int stage, double* smem) {
  switch (phase) {
#if GP_BATCH_PART == 0
    case BP_SWEEP_X:
      tile_sweep_x<PHYS, NV, NDIM, RS, CT, LIM>(a, g, idx, smem);
      break;
    case BP_SWEEP_Y:
      tile_sweep_m<PHYS, NV, NDIM, RS, CT, LIM, 1>(a, g, seg, idx, smem);
      break;
    case BP_SWEEP_Z:
      if constexpr (NDIM == 3) tile_sweep_m<PHYS, NV, NDIM, RS, CT, LIM, 2>(a, g, seg, idx, smem);
      break;
#else
    case BP_EMF:
      if constexpr (PHYS != PHYS_HD) tile_emf<NDIM, LIM>(a, g, cpt, idx);
      break;
    case BP_FINISH:
      tile_finish<PHYS, NV, NDIM>(a, g, cpt, idx, stage);
      break;
#endif
    default:
      break;
  }
}

}  // namespace

static_assert(sizeof(StageArgs<CTT>) % 8 == 0, "StageArgs copied as 8-byte words");

#if GP_BATCH_PART == 0
__device__ void GP_BATCH_TILE(const BatchSlot& s, const BatchTile& t, int stage, double* smem) {
#else
__device__ void GP_BATCH_TILE(const BatchSlot& s, const BatchTile& t, int stage) {
  double* smem = nullptr;  // the cell bodies stage nothing
#endif
  // One copy of the slot's StageArgs per block, in shared memory: the bodies
  // store through the state pointers, and shared memory cannot alias them,
  // so the fields are read cheaply without a private copy per thread.
  __shared__ StageArgs<CTT> sa;
  {
    const unsigned long long* src =
        reinterpret_cast<const unsigned long long*>(&s.sa[stage - 1][s.sc->bcur]);
    unsigned long long* dst = reinterpret_cast<unsigned long long*>(&sa);
    constexpr int W = (int)(sizeof(StageArgs<CTT>) / 8);
    for (int w = threadIdx.x; w < W; w += blockDim.x) dst[w] = src[w];
  }
  __syncthreads();
  const StageArgs<CTT>& a = sa;
  const Grid3 g{s.nx, s.ny, s.nz, s.n};
  const int seg = s.seg, cpt = s.cpt;
  if (s.physics == PHYS_MHD) {
    if (s.ndim == 2)
      run_tile<PHYS_MHD, 8, 2, RS_HLLD, CT_UCT_HLLD, LIM_MC>(a, g, seg, cpt, t.phase, t.idx,
                                                             stage, smem);
    else
      run_tile<PHYS_MHD, 8, 3, RS_HLLD, CT_UCT_HLLD, LIM_MC>(a, g, seg, cpt, t.phase, t.idx,
                                                             stage, smem);
  } else if (s.physics == PHYS_RMHD) {
    if (s.ndim == 2)
      run_tile<PHYS_RMHD, 8, 2, RS_HLLD, CT_UCT_HLL, LIM_MC>(a, g, seg, cpt, t.phase, t.idx,
                                                            stage, smem);
    else
      run_tile<PHYS_RMHD, 8, 3, RS_HLLD, CT_UCT_HLL, LIM_MC>(a, g, seg, cpt, t.phase, t.idx,
                                                            stage, smem);
  } else {
    if (s.ndim == 2)
      run_tile<PHYS_HD, 5, 2, RS_HLLC, 0, LIM_MC>(a, g, seg, cpt, t.phase, t.idx, stage, smem);
    else
      run_tile<PHYS_HD, 5, 3, RS_HLLC, 0, LIM_MC>(a, g, seg, cpt, t.phase, t.idx, stage, smem);
  }
}

}  // namespace gp
