// gp_batch.cu -- batched step: one device pool, a slot table, a phase-ordered
// tile table and two persistent launches per RK stage over all slots; runs
// of steps captured as CUDA graphs (C ABI in include/gpluto_b200.h).
//
// In each launch every block repeatedly takes the next tile from an atomic
// queue head.  The sweep launch (168 registers, 3 blocks/SM) takes the sweep
// tiles of every slot; the cell launch (64 registers, 8 blocks/SM: the edge
// EMF and finish bodies are latency-bound and want the occupancy) takes the
// EMF tiles, then the finish tiles, and a finish tile of slot s first waits
// until all EMF tiles of s have completed.  Each wait is a bounded spin:
// after kSpinLimit polls the block records a batch error and skips, and once
// that error is set every later wait gives up at once, so a launch always
// ends.  The last finish tile of slot s in stage 2 evaluates NextTimeStep for
// s (the same arithmetic as the single-grid path), rotates its face buffers
// and counts the step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <new>
#include <vector>

#include "../../include/gpluto_b200.h"
#include "gp_batch.h"
#include "gp_launch.h"

namespace gp {

namespace {

constexpr long long kSpinLimit = 1LL << 22;  // ~0.3 us per poll: about a second
constexpr uint32_t kErrWaitRanOut = 1u;      // batch error word: a wait gave up

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) {
  return *reinterpret_cast<const volatile uint32_t*>(p);
}

// NextTimeStep of one slot (Src/update_stage.cpp:422-435 and
// Src/next_time_step.cpp:80,125) and the step bookkeeping.
__device__ void step_epilogue(const BatchSlot& s) {
  BatchScalars* sc = s.sc;
  const double mx = __longlong_as_double((long long)sc->invdt_bits);
  const double inv = mx / (double)s.ndim;
  const double dt = sc->dt;
  double dtn = s.cfl / inv;
  dtn = (dtn <= s.cfl_max_var * dt) ? dtn : s.cfl_max_var * dt;
  sc->invdt = inv;
  sc->dt = dtn;
  sc->dtdx[0] = dtn / s.dx[0];
  sc->dtdx[1] = dtn / s.dx[1];
  sc->dtdx[2] = dtn / s.dx[2];
  sc->invdt_bits = 0ull;
  sc->bcur = (sc->bcur + 2) % 3;
  sc->steps_done += 1;
  sc->steps_left -= 1;
  if (sc->err & ERR_QUIT) sc->steps_left = 0;
}

// Persistent loop of one launch: part 0 takes the sweep tiles [0, nsweep),
// part 1 the EMF and finish tiles [nsweep, ntiles).
template <int PART>
__device__ __forceinline__ void batch_loop(const BatchSlot* __restrict__ slots,
                                           const BatchTile* __restrict__ tiles,
                                           const BatchTableHeader* __restrict__ hdr,
                                           BatchCounters* ctr, int stage, uint32_t* batch_err,
                                           double* smem) {
  __shared__ int s_tile;
  __shared__ int s_go;
  const int t0 = PART == 0 ? 0 : hdr->nsweep;
  const int t1 = PART == 0 ? hdr->nsweep : hdr->ntiles;
  for (;;) {
    if (threadIdx.x == 0) s_tile = t0 + atomicAdd(&ctr->head[PART], 1);
    __syncthreads();
    const int ti = s_tile;
    if (ti >= t1) break;  // block-uniform
    const BatchTile t = tiles[ti];
    const BatchSlot& s = slots[t.slot];
    if (threadIdx.x == 0) {
      int go = s.sc->steps_left > 0 && ld_volatile(batch_err) == 0u;
      if (go && PART == 1 && t.phase == BP_FINISH && s.physics != PHYS_HD) {
        const int need = s.need[BG_EMF] + (t.slot == hdr->bias_slot ? hdr->bias_need : 0);
        const int* c = &ctr->done[t.slot * BG_COUNT + BG_EMF];
        const long long limit = hdr->spin_limit;
        long long it = 0;
        while (ld_acquire(c) < need) {
          if (ld_volatile(batch_err) != 0u) { go = 0; break; }
          if (++it > limit) {
            atomicOr(batch_err, kErrWaitRanOut);
            go = 0;
            break;
          }
          __nanosleep(128);
        }
      }
      s_go = go;
    }
    __syncthreads();
    const int go = s_go;
    if (go) {
      if constexpr (PART == 0) {
        if (s.precision == GP_MIXED) batch_sweep_tile_mixed(s, t, stage, smem);
        else batch_sweep_tile_fp64(s, t, stage, smem);
      } else {
        if (s.precision == GP_MIXED) batch_cell_tile_mixed(s, t, stage);
        else batch_cell_tile_fp64(s, t, stage);
      }
    }
    __syncthreads();  // the tile's writes are done; s_tile/s_go may be reused
    if (PART == 1 && threadIdx.x == 0 && go) {
      const int grp = t.phase == BP_EMF ? BG_EMF : BG_FINISH;
      __threadfence();
      const int old = atomicAdd(&ctr->done[t.slot * BG_COUNT + grp], 1);
      if (grp == BG_FINISH && stage == 2 && old == s.need[BG_FINISH] - 1) {
        __threadfence();
        step_epilogue(s);
      }
    }
  }
}

__global__ void __launch_bounds__(BATCH_THREADS, GP_SWEEP_MINB)
    batch_sweep_kernel(const BatchSlot* __restrict__ slots, const BatchTile* __restrict__ tiles,
                       const BatchTableHeader* __restrict__ hdr, BatchCounters* ctr, int stage,
                       uint32_t* batch_err) {
  extern __shared__ double smem[];
  batch_loop<0>(slots, tiles, hdr, ctr, stage, batch_err, smem);
}

__global__ void __launch_bounds__(BATCH_THREADS, GP_CELL_MINB)
    batch_cell_kernel(const BatchSlot* __restrict__ slots, const BatchTile* __restrict__ tiles,
                      const BatchTableHeader* __restrict__ hdr, BatchCounters* ctr, int stage,
                      uint32_t* batch_err) {
  batch_loop<1>(slots, tiles, hdr, ctr, stage, batch_err, nullptr);
}

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  return set_last_error(code, buf);
}

constexpr size_t kAlign = 256;

size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

struct SlotLayout {
  long long n;
  int nvar, ndim;
  bool mhd, mixed;
  size_t bytes;
};

// Region of one slot: U[2], V, dU, Cdt, Bs[3 buffers][ndim], ct[ndim][6],
// Ee, scalars.  Every array starts on a 256-byte boundary; dU, Cdt, ct and
// Ee hold floats in the mixed form.
SlotLayout slot_layout(const gp_grid_desc* g, const gp_scheme* sc) {
  SlotLayout L;
  L.ndim = g->ndim;
  const long long nz = g->ndim == 3 ? g->nint[2] : 1;
  L.n = (long long)g->nint[0] * g->nint[1] * nz;
  L.mhd = sc->physics != GP_HD;  // MHD and RMHD: staggered fields, UCT data, EMFs
  L.mixed = sc->precision == GP_MIXED;
  L.nvar = L.mhd ? 8 : 5;
  const size_t cell = sizeof(double) * (size_t)L.n;
  // flux differences, inverse-dt terms, UCT data, EMFs: float in the mixed form
  const size_t fcell = (L.mixed ? sizeof(float) : sizeof(double)) * (size_t)L.n;
  size_t b = 0;
  b += 2 * align_up(cell * L.nvar);           // U[0], U[1]
  b += align_up(cell * L.nvar);               // V
  b += align_up(fcell * L.nvar * L.ndim);     // dU
  b += align_up(fcell * L.ndim);              // Cdt
  if (L.mhd) {
    b += 3 * L.ndim * align_up(cell);         // face buffers
    b += L.ndim * 6 * align_up(fcell);        // UCT face data
    b += (L.ndim == 3 ? 3 : 1) * align_up(fcell);  // edge EMFs
  }
  b += align_up(sizeof(BatchScalars));
  L.bytes = b;
  return L;
}

bool scheme_built(const gp_scheme* sc) {
  if (sc->rk_stages != 2) return false;
  if (sc->limiter != GP_LIM_MC || sc->reconstruction != GP_REC_LINEAR) return false;
  if (sc->precision != GP_FP64 && sc->precision != GP_MIXED) return false;
  if (sc->physics == GP_MHD) return sc->riemann == GP_RS_HLLD && sc->ct_emf == GP_CT_UCT_HLLD;
  if (sc->physics == GP_RMHD) return sc->riemann == GP_RS_HLLD && sc->ct_emf == GP_CT_UCT_HLL;
  if (sc->physics == GP_HD) return sc->riemann == GP_RS_HLLC;
  return false;
}

}  // namespace
}  // namespace gp

using gp::BatchScalars;
using gp::BatchSlot;
using gp::BatchTile;

struct gp_batch {
  cudaStream_t stream;
  bool own_stream;
  int max_slots;
  int ctas;
  int ctas_full;  // blocks that fit on the device at once
  char* pool;
  size_t pool_bytes, pool_used;
  std::map<size_t, size_t> free_list;  // offset -> size
  std::vector<BatchSlot> slots;        // host copy of the slot table
  std::vector<char> used;
  std::vector<size_t> off, bytes;
  BatchSlot* slots_d;
  BatchTile* tiles_d;
  int tiles_cap;
  gp::BatchTableHeader* hdr_d;
  int cell_ctas;  // blocks of the cell launch
  gp::BatchCounters* ctr_d;
  size_t ctr_bytes;
  uint32_t* err_d;
  long long spin_limit;     // dependency-wait polls (kSpinLimit unless injected)
  int bias_slot, bias_need; // injected dependency fault (tests), -1 / 0 = none
  BatchScalars* sc_h;  // pinned copy of every slot's scalars
  bool dirty;
  std::map<int, cudaGraphExec_t> graphs;
};

namespace {

#define BATCH_CUDA(call)                                                                  \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return gp::fail(GP_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));       \
  } while (0)

bool pool_alloc(gp_batch* b, size_t bytes, size_t* off) {
  for (auto it = b->free_list.begin(); it != b->free_list.end(); ++it) {
    if (it->second >= bytes) {
      *off = it->first;
      const size_t rest = it->second - bytes;
      const size_t roff = it->first + bytes;
      b->free_list.erase(it);
      if (rest) b->free_list[roff] = rest;
      b->pool_used += bytes;
      return true;
    }
  }
  return false;
}

void pool_free(gp_batch* b, size_t off, size_t bytes) {
  auto it = b->free_list.emplace(off, bytes).first;
  auto nx = std::next(it);
  if (nx != b->free_list.end() && it->first + it->second == nx->first) {
    it->second += nx->second;
    b->free_list.erase(nx);
  }
  if (it != b->free_list.begin()) {
    auto pv = std::prev(it);
    if (pv->first + pv->second == it->first) {
      pv->second += it->second;
      b->free_list.erase(it);
    }
  }
  b->pool_used -= bytes;
}

void free_batch(gp_batch* b) {
  for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
  b->graphs.clear();
  cudaFree(b->pool);
  cudaFree(b->slots_d);
  cudaFree(b->tiles_d);
  cudaFree(b->hdr_d);
  cudaFree(b->ctr_d);
  cudaFree(b->err_d);
  cudaFreeHost(b->sc_h);
  if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
}

void apply_shape(BatchSlot& s, const gp_tile_shape* shape) {
  const int seg = shape && shape->seg > 0 ? shape->seg : 32;
  s.seg = std::min(seg, std::max(s.ny, s.nz));
  s.cpt = shape && shape->cells_per_thread > 0 ? std::min(shape->cells_per_thread, 64) : 2;
}

void tile_counts(BatchSlot& s) {
  const long long rows = (long long)s.ny * s.nz;
  s.ntiles[gp::BP_SWEEP_X] = (int)((rows + gp::BATCH_ROWS_PER_TILE - 1) / gp::BATCH_ROWS_PER_TILE);
  auto items = [&](int nd, int ntr) {
    const long long nseg = (nd + s.seg - 1) / s.seg;
    const long long it = (long long)s.nx * nseg * ntr;
    return (int)((it + gp::BATCH_THREADS - 1) / gp::BATCH_THREADS);
  };
  s.ntiles[gp::BP_SWEEP_Y] = items(s.ny, s.nz);
  s.ntiles[gp::BP_SWEEP_Z] = s.ndim == 3 ? items(s.nz, s.ny) : 0;
  const long long per = (long long)gp::BATCH_THREADS * s.cpt;
  const int cells = (int)((s.n + per - 1) / per);
  s.ntiles[gp::BP_EMF] = s.physics != gp::PHYS_HD ? cells : 0;
  s.ntiles[gp::BP_FINISH] = cells;
  s.need[gp::BG_SWEEPS] = s.ntiles[0] + s.ntiles[1] + s.ntiles[2];
  s.need[gp::BG_EMF] = s.ntiles[gp::BP_EMF];
  s.need[gp::BG_FINISH] = s.ntiles[gp::BP_FINISH];
}

// Phase-ordered tile table: all sweeps (the sweep launch), then all EMF
// tiles, then all finish tiles (the cell launch); slots from the largest
// grid down, so that the EMF tiles of the largest (longest) grids complete
// first.
int rebuild_tiles(gp_batch* b) {
  std::vector<int> order;
  for (int i = 0; i < b->max_slots; i++)
    if (b->used[i]) order.push_back(i);
  std::stable_sort(order.begin(), order.end(),
                   [&](int x, int y) { return b->slots[x].n > b->slots[y].n; });
  std::vector<BatchTile> t;
  // Sweep tiles: grouped by code path -- (precision, physics, dimensions,
  // direction) -- so that the blocks running at one time mostly execute the
  // same instructions; EMF and finish tiles: slot by slot.
  std::vector<std::pair<long long, BatchTile>> sw;
  for (int sidx : order) {
    const BatchSlot& s = b->slots[sidx];
    for (int ph = gp::BP_SWEEP_X; ph <= gp::BP_SWEEP_Z; ph++) {
      const long long key = ((long long)s.precision * 4 + s.physics) * 8 + s.ndim * 2 + 0;
      for (int k = 0; k < s.ntiles[ph]; k++)
        sw.push_back({key * 8 + ph, BatchTile{sidx, ph, k, 0}});
    }
  }
  std::stable_sort(sw.begin(), sw.end(),
                   [](const std::pair<long long, BatchTile>& x,
                      const std::pair<long long, BatchTile>& y) { return x.first < y.first; });
  for (auto& e : sw) t.push_back(e.second);
  const int nsweep = (int)t.size();
  for (int ph : {gp::BP_EMF, gp::BP_FINISH})
    for (int sidx : order)
      for (int k = 0; k < b->slots[sidx].ntiles[ph]; k++) t.push_back(BatchTile{sidx, ph, k, 0});
  const int nt = (int)t.size();
  if (nt > b->tiles_cap) {
    // captured graphs hold the old table's address: drop them
    for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
    b->graphs.clear();
    cudaFree(b->tiles_d);
    b->tiles_d = nullptr;
    const int cap = std::max(nt, 2 * b->tiles_cap);
    BATCH_CUDA(cudaMalloc((void**)&b->tiles_d, sizeof(BatchTile) * (size_t)cap));
    b->tiles_cap = cap;
  }
  if (nt) BATCH_CUDA(cudaMemcpy(b->tiles_d, t.data(), sizeof(BatchTile) * nt, cudaMemcpyHostToDevice));
  gp::BatchTableHeader h{nsweep, nt, b->spin_limit, b->bias_slot, b->bias_need};
  BATCH_CUDA(cudaMemcpy(b->hdr_d, &h, sizeof(h), cudaMemcpyHostToDevice));
  BATCH_CUDA(cudaMemcpy(b->slots_d, b->slots.data(), sizeof(BatchSlot) * b->max_slots,
                        cudaMemcpyHostToDevice));
  b->dirty = false;
  return GP_OK;
}

int capture(gp_batch* b, int nsteps, cudaGraphExec_t* out) {
  cudaGraph_t g = nullptr;
  BATCH_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  const int smem = gp::batch_smem_bytes();
  bool ok = true;
  for (int st = 0; st < nsteps && ok; st++)
    for (int stage = 1; stage <= 2 && ok; stage++) {
      if (cudaMemsetAsync(b->ctr_d, 0, b->ctr_bytes, b->stream) != cudaSuccess) ok = false;
      gp::batch_sweep_kernel<<<b->ctas, gp::BATCH_THREADS, smem, b->stream>>>(
          b->slots_d, b->tiles_d, b->hdr_d, b->ctr_d, stage, b->err_d);
      gp::batch_cell_kernel<<<b->cell_ctas, gp::BATCH_THREADS, 0, b->stream>>>(
          b->slots_d, b->tiles_d, b->hdr_d, b->ctr_d, stage, b->err_d);
      if (cudaGetLastError() != cudaSuccess) ok = false;
    }
  cudaError_t e = cudaStreamEndCapture(b->stream, &g);
  if (!ok || e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return gp::fail(GP_ERR_CUDA, "capturing the batched step failed");
  }
  e = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return gp::fail(GP_ERR_CUDA, "graph instantiation: %s", cudaGetErrorString(e));
  return GP_OK;
}

}  // namespace

extern "C" {

size_t gp_batch_slot_bytes(const gp_grid_desc* grid, const gp_scheme* scheme) {
  if (!grid || !scheme || (grid->ndim != 2 && grid->ndim != 3)) return 0;
  return gp::slot_layout(grid, scheme).bytes;
}

int gp_batch_create(size_t pool_bytes, int max_slots, int ctas, void* stream, gp_batch** out) {
  if (!out || max_slots < 1 || pool_bytes == 0 || ctas < 0)
    return gp::fail(GP_ERR_INVALID, "bad batch arguments");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return gp::fail(GP_ERR_NO_DEVICE, "no CUDA device: the batched step has no CPU path");
  }
  gp_batch* b = new (std::nothrow) gp_batch();
  if (!b) return gp::fail(GP_ERR_NOMEM, "host allocation");
  b->max_slots = max_slots;
  b->spin_limit = gp::kSpinLimit;
  b->bias_slot = -1;
  b->bias_need = 0;
  b->slots.assign(max_slots, BatchSlot{});
  b->used.assign(max_slots, 0);
  b->off.assign(max_slots, 0);
  b->bytes.assign(max_slots, 0);
  b->stream = static_cast<cudaStream_t>(stream);
  int rc = GP_OK;
  auto chk = [&](cudaError_t e, const char* what) {
    if (rc == GP_OK && e != cudaSuccess) {
      cudaGetLastError();
      rc = gp::fail(e == cudaErrorMemoryAllocation ? GP_ERR_NOMEM : GP_ERR_CUDA, "%s: %s", what,
                    cudaGetErrorString(e));
    }
  };
  if (!b->stream) {
    chk(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "stream");
    b->own_stream = rc == GP_OK;
  }
  b->pool_bytes = pool_bytes / gp::kAlign * gp::kAlign;
  chk(cudaMalloc((void**)&b->pool, b->pool_bytes), "device pool");
  b->free_list[0] = b->pool_bytes;
  chk(cudaMalloc((void**)&b->slots_d, sizeof(BatchSlot) * max_slots), "slot table");
  chk(cudaMalloc((void**)&b->hdr_d, sizeof(gp::BatchTableHeader)), "tile table header");
  b->ctr_bytes = sizeof(gp::BatchCounters) + sizeof(int) * (size_t)max_slots * gp::BG_COUNT;
  chk(cudaMalloc((void**)&b->ctr_d, b->ctr_bytes), "counters");
  chk(cudaMalloc((void**)&b->err_d, sizeof(uint32_t)), "error word");
  chk(cudaMallocHost((void**)&b->sc_h, sizeof(BatchScalars) * max_slots), "status mirror");
  if (rc == GP_OK) {
    chk(cudaMemset(b->slots_d, 0, sizeof(BatchSlot) * max_slots), "memset");
    chk(cudaMemset(b->hdr_d, 0, sizeof(gp::BatchTableHeader)), "memset");
    chk(cudaMemset(b->err_d, 0, sizeof(uint32_t)), "memset");
    std::memset(b->sc_h, 0, sizeof(BatchScalars) * max_slots);
    int per_sm = 0, nsm = 0, dev = 0;
    chk(cudaGetDevice(&dev), "device");
    chk(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev), "SM count");
    chk(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gp::batch_sweep_kernel,
                                                      gp::BATCH_THREADS, gp::batch_smem_bytes()),
        "occupancy");
    b->ctas_full = std::max(1, per_sm) * nsm;
    b->ctas = ctas > 0 ? ctas : b->ctas_full;
    int per_sm_cell = 0;
    chk(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_cell, gp::batch_cell_kernel,
                                                      gp::BATCH_THREADS, 0),
        "occupancy");
    b->cell_ctas = std::max(1, per_sm_cell) * nsm;
  }
  if (rc != GP_OK) {
    free_batch(b);
    delete b;
    return rc;
  }
  *out = b;
  return GP_OK;
}

int gp_batch_destroy(gp_batch* b) {
  if (!b) return GP_ERR_INVALID;
  if (b->stream) cudaStreamSynchronize(b->stream);
  free_batch(b);
  delete b;
  return GP_OK;
}

int gp_batch_add(gp_batch* b, const gp_grid_desc* grid, const gp_scheme* scheme,
                 const gp_tile_shape* shape, const double* Vc, const double* Vs0,
                 const double* Vs1, const double* Vs2, double dt0, int nsteps, int* slot) {
  if (!b || !grid || !scheme || !Vc || !slot) return gp::fail(GP_ERR_INVALID, "null argument");
  *slot = -1;
  if (grid->ndim != 2 && grid->ndim != 3) return gp::fail(GP_ERR_UNSUPPORTED, "ndim must be 2 or 3");
  if (!gp::scheme_built(scheme))
    return gp::fail(GP_ERR_UNSUPPORTED,
                    "batches are built for MHD PLM-MC/HLLD/UCT_HLLD, RMHD PLM-MC/HLLD/UCT_HLL "
                    "and HD PLM-MC/HLLC, RK2");
  for (int d = 0; d < grid->ndim; d++) {
    if (grid->nint[d] < 2) return gp::fail(GP_ERR_INVALID, "nint[%d] < 2", d);
    if (grid->lbound[d] != GP_BC_PERIODIC || grid->rbound[d] != GP_BC_PERIODIC)
      return gp::fail(GP_ERR_UNSUPPORTED, "only periodic boundaries are built");
  }
  if (!(dt0 > 0.0) || nsteps < 0) return gp::fail(GP_ERR_INVALID, "bad dt0 or nsteps");
  const bool mhd = scheme->physics != GP_HD;  // staggered fields (MHD, RMHD)
  if (mhd && (!Vs0 || !Vs1 || (grid->ndim == 3 && !Vs2)))
    return gp::fail(GP_ERR_INVALID, "face fields missing");
  int idx = -1;
  for (int i = 0; i < b->max_slots; i++)
    if (!b->used[i]) { idx = i; break; }
  if (idx < 0) return gp::fail(GP_ERR_NOMEM, "slot table full (%d slots)", b->max_slots);
  const gp::SlotLayout L = gp::slot_layout(grid, scheme);
  if (L.n >= (1LL << 31)) return gp::fail(GP_ERR_UNSUPPORTED, "grids are limited to fewer than 2^31 cells");
  size_t off = 0;
  if (!pool_alloc(b, L.bytes, &off))
    return gp::fail(GP_ERR_NOMEM, "pool full: %zu bytes requested, %zu of %zu in use", L.bytes,
                    b->pool_used, b->pool_bytes);
  // carve the region
  char* p = b->pool + off;
  auto take = [&](size_t bytes) { char* q = p; p += gp::align_up(bytes); return q; };
  const long long n = L.n;
  const size_t cell = sizeof(double) * (size_t)n;
  const size_t fcell = (L.mixed ? sizeof(float) : sizeof(double)) * (size_t)n;
  double* U0 = (double*)take(cell * L.nvar);
  double* U1 = (double*)take(cell * L.nvar);
  double* V = (double*)take(cell * L.nvar);
  double* dU = (double*)take(fcell * L.nvar * L.ndim);
  double* Cdt = (double*)take(fcell * L.ndim);
  double* B[3][3] = {};
  void* ct[3][6] = {};
  double* Ee[3] = {};
  if (mhd) {
    for (int k = 0; k < 3; k++)
      for (int d = 0; d < L.ndim; d++) B[k][d] = (double*)take(cell);
    for (int d = 0; d < L.ndim; d++)
      for (int r = 0; r < 6; r++) ct[d][r] = take(fcell);
    for (int d = 0; d < 3; d++)
      if (L.ndim == 3 || d == 2) Ee[d] = (double*)take(fcell);
  }
  BatchScalars* sc = (BatchScalars*)take(sizeof(BatchScalars));

  BatchSlot s;
  std::memset(&s, 0, sizeof(s));
  s.physics = scheme->physics;
  s.ndim = grid->ndim;
  s.precision = scheme->precision;
  s.nvar = L.nvar;
  s.nx = grid->nint[0];
  s.ny = grid->nint[1];
  s.nz = grid->ndim == 3 ? grid->nint[2] : 1;
  s.n = n;
  apply_shape(s, shape);
  s.cfl = scheme->cfl;
  s.cfl_max_var = scheme->cfl_max_var;
  for (int d = 0; d < 3; d++) {
    const int nn = d == 0 ? s.nx : d == 1 ? s.ny : s.nz;
    s.dx[d] = (grid->dx[d] && d < grid->ndim) ? grid->dx[d][0] : (grid->xend[d] - grid->xbeg[d]) / nn;
    if (!(s.dx[d] > 0.0)) s.dx[d] = 1.0;
  }
  s.sc = sc;
  tile_counts(s);
  for (int bc = 0; bc < 3; bc++) {
    const int b0 = bc, b1 = (bc + 1) % 3, b2 = (bc + 2) % 3;
    for (int stage = 1; stage <= 2; stage++) {
      gp::StageArgs<double>& a = s.sa[stage - 1][bc];
      a.V = V;
      a.Vout = V;
      a.dU = dU;
      a.Cdt = Cdt;
      a.U0 = U0;
      a.Uc = stage == 1 ? U0 : U1;
      a.Uout = stage == 1 ? U1 : U0;
      for (int q = 0; q < 3; q++) {
        const bool on = mhd && q < L.ndim;
        a.Bs[q] = on ? B[stage == 1 ? b0 : b1][q] : nullptr;
        a.Bs0[q] = on ? B[b0][q] : nullptr;
        a.Bsout[q] = on ? B[stage == 1 ? b1 : b2][q] : nullptr;
        a.Ee[q] = Ee[q];
        a.dx[q] = s.dx[q];
        for (int r = 0; r < 6; r++) a.ct[q][r] = static_cast<double*>(ct[q][r]);
      }
      a.dtdx = sc->dtdx;
      a.gamma = scheme->gamma;
      a.small_rho = scheme->small_rho;
      a.small_prs = scheme->small_prs;
      a.stage = stage;
      a.w0 = a.w1 = a.wr = 0.5;  // RK2 combine of stage 2 (Src/rk_step.cpp:30-35)
      a.invdt_bits = &sc->invdt_bits;
      a.err = &sc->err;
    }
  }
  // initial state: V and the faces from the host, U by the start-up map
  int rc = GP_OK;
  auto chk = [&](cudaError_t e, const char* what) {
    if (rc == GP_OK && e != cudaSuccess) {
      cudaGetLastError();
      rc = gp::fail(GP_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    }
  };
  chk(cudaMemcpyAsync(V, Vc, cell * L.nvar, cudaMemcpyHostToDevice, b->stream), "upload V");
  if (mhd) {
    const double* src[3] = {Vs0, Vs1, Vs2};
    for (int d = 0; d < L.ndim; d++)
      chk(cudaMemcpyAsync(B[0][d], src[d], cell, cudaMemcpyHostToDevice, b->stream), "upload Vs");
  }
  chk(cudaMemsetAsync(dU, 0, fcell * L.nvar * L.ndim, b->stream), "clear dU");
  if (rc == GP_OK && gp::launch_prim2cons(scheme->physics, V, U0, n, scheme->gamma, b->stream) != 0)
    rc = gp::fail(GP_ERR_UNSUPPORTED, "start-up map");
  BatchScalars hs;
  std::memset(&hs, 0, sizeof(hs));
  hs.dt = dt0;
  for (int d = 0; d < 3; d++) hs.dtdx[d] = dt0 / s.dx[d];
  hs.steps_left = nsteps;
  chk(cudaMemcpyAsync(sc, &hs, sizeof(hs), cudaMemcpyHostToDevice, b->stream), "scalars");
  chk(cudaStreamSynchronize(b->stream), "admission");
  if (rc != GP_OK) {
    pool_free(b, off, L.bytes);
    return rc;
  }
  b->slots[idx] = s;
  b->used[idx] = 1;
  b->off[idx] = off;
  b->bytes[idx] = L.bytes;
  b->sc_h[idx] = hs;
  b->dirty = true;
  *slot = idx;
  return GP_OK;
}

int gp_batch_set_shape(gp_batch* b, int slot, const gp_tile_shape* shape) {
  if (!b || slot < 0 || slot >= b->max_slots || !b->used[slot])
    return gp::fail(GP_ERR_INVALID, "no such slot");
  BatchSlot& s = b->slots[slot];
  apply_shape(s, shape);
  tile_counts(s);
  b->dirty = true;
  return GP_OK;
}

int gp_batch_set_ctas(gp_batch* b, int ctas) {
  if (!b || ctas < 0) return gp::fail(GP_ERR_INVALID, "bad arguments");
  BATCH_CUDA(cudaStreamSynchronize(b->stream));
  const int c = ctas > 0 ? ctas : b->ctas_full;
  if (c != b->ctas) {
    for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
    b->graphs.clear();
    b->ctas = c;
  }
  return GP_OK;
}

int gp_batch_remove(gp_batch* b, int slot) {
  if (!b || slot < 0 || slot >= b->max_slots || !b->used[slot])
    return gp::fail(GP_ERR_INVALID, "no such slot");
  BATCH_CUDA(cudaStreamSynchronize(b->stream));
  pool_free(b, b->off[slot], b->bytes[slot]);
  b->used[slot] = 0;
  std::memset(&b->slots[slot], 0, sizeof(BatchSlot));
  std::memset(&b->sc_h[slot], 0, sizeof(BatchScalars));
  b->dirty = true;
  return GP_OK;
}

int gp_batch_advance(gp_batch* b, int nsteps) {
  if (!b || nsteps < 1) return gp::fail(GP_ERR_INVALID, "bad arguments");
  if (b->dirty) {
    BATCH_CUDA(cudaStreamSynchronize(b->stream));
    int rc = rebuild_tiles(b);
    if (rc) return rc;
  }
  auto it = b->graphs.find(nsteps);
  if (it == b->graphs.end()) {
    cudaGraphExec_t ge = nullptr;
    int rc = capture(b, nsteps, &ge);
    if (rc) return rc;
    it = b->graphs.emplace(nsteps, ge).first;
  }
  BATCH_CUDA(cudaGraphLaunch(it->second, b->stream));
  return GP_OK;
}

int gp_batch_wait(gp_batch* b) {
  if (!b) return GP_ERR_INVALID;
  BATCH_CUDA(cudaStreamSynchronize(b->stream));
  uint32_t err = 0;
  BATCH_CUDA(cudaMemcpy(&err, b->err_d, sizeof(err), cudaMemcpyDeviceToHost));
  for (int i = 0; i < b->max_slots; i++)
    if (b->used[i])
      BATCH_CUDA(cudaMemcpyAsync(&b->sc_h[i], b->slots[i].sc, sizeof(BatchScalars),
                                 cudaMemcpyDeviceToHost, b->stream));
  BATCH_CUDA(cudaStreamSynchronize(b->stream));
  if (err) {
    // the report consumes the error word; the slots that were advancing when
    // a wait ran out hold a partly updated state (remove or re-admit them)
    BATCH_CUDA(cudaMemset(b->err_d, 0, sizeof(uint32_t)));
    return gp::fail(GP_ERR_TIMEOUT, "a batched stage gave up waiting on a dependency "
                    "(the EMF tiles of a slot did not complete within the wait limit)");
  }
  return GP_OK;
}

int gp_batch_inject_wait_fault(gp_batch* b, int slot, int extra_need, long long spin_limit) {
  if (!b || extra_need < 0 || spin_limit < 0 ||
      (extra_need > 0 && (slot < 0 || slot >= b->max_slots || !b->used[slot])))
    return gp::fail(GP_ERR_INVALID, "bad arguments");
  BATCH_CUDA(cudaStreamSynchronize(b->stream));
  b->bias_slot = extra_need > 0 ? slot : -1;
  b->bias_need = extra_need;
  b->spin_limit = spin_limit > 0 ? spin_limit : gp::kSpinLimit;
  b->dirty = true;  // the next advance rewrites the table header
  return GP_OK;
}

int gp_batch_slot_status(const gp_batch* b, int slot, gp_slot_status* st) {
  if (!b || !st || slot < 0 || slot >= b->max_slots || !b->used[slot])
    return gp::fail(GP_ERR_INVALID, "no such slot");
  const BatchScalars& s = b->sc_h[slot];
  st->steps_done = s.steps_done;
  st->steps_left = s.steps_left;
  st->err_bits = s.err;
  st->dt = s.dt;
  st->invDt_hyp = s.invdt;
  return GP_OK;
}

int gp_batch_download(gp_batch* b, int slot, double* Uc, double* Vc, double* Vs0, double* Vs1,
                      double* Vs2) {
  if (!b || slot < 0 || slot >= b->max_slots || !b->used[slot])
    return gp::fail(GP_ERR_INVALID, "no such slot");
  BATCH_CUDA(cudaStreamSynchronize(b->stream));
  const BatchSlot& s = b->slots[slot];
  BatchScalars hs;
  BATCH_CUDA(cudaMemcpy(&hs, s.sc, sizeof(hs), cudaMemcpyDeviceToHost));
  const size_t cell = sizeof(double) * (size_t)s.n;
  const gp::StageArgs<double>& a = s.sa[0][hs.bcur];  // stage-1 inputs = current state
  if (Uc) BATCH_CUDA(cudaMemcpy(Uc, a.U0, cell * s.nvar, cudaMemcpyDeviceToHost));
  if (Vc) BATCH_CUDA(cudaMemcpy(Vc, a.V, cell * s.nvar, cudaMemcpyDeviceToHost));
  double* dst[3] = {Vs0, Vs1, Vs2};
  for (int d = 0; d < 3; d++)
    if (dst[d] && a.Bs[d]) BATCH_CUDA(cudaMemcpy(dst[d], a.Bs[d], cell, cudaMemcpyDeviceToHost));
  return GP_OK;
}

int gp_batch_info(const gp_batch* b, size_t* pool_used, size_t* pool_bytes, int* slots,
                  int* ctas) {
  if (!b) return GP_ERR_INVALID;
  if (pool_used) *pool_used = b->pool_used;
  if (pool_bytes) *pool_bytes = b->pool_bytes;
  if (slots) {
    int c = 0;
    for (int i = 0; i < b->max_slots; i++) c += b->used[i] ? 1 : 0;
    *slots = c;
  }
  if (ctas) *ctas = b->ctas;
  return GP_OK;
}

}  // extern "C"
