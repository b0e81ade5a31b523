// gp_noalloc.cu -- one RK2 step that allocates no memory.
//
// Some callers cannot call cudaMalloc: hosts whose device memory is owned by
// another allocator or framework and must not change size once set up, and
// latency-critical loops that forbid allocation.  gp_advance_step_noalloc
// serves them: the caller passes the state arrays (device pointers it
// already owns) and every intermediate of the step (the stage-1 state, flux
// differences, inverse-dt terms, UCT face data, edge EMFs, face-field
// buffers, step scalars) lives in the file-scope device array
// g_noalloc_scratch below.
//
// That array is GP_NOALLOC_MAX_CELLS * GP_NOALLOC_DOUBLES_PER_CELL doubles
// plus a small header (~8 MB).  Every GPU that loads the library keeps it
// until the process exits.  All calls share it and it keeps the previous
// call's contents; the step scalars that must start at zero are cleared on
// every call.  Calls that overlap on the GPU (different streams, different
// threads) race on the array.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/gpluto_b200.h"
#include "gp_checks.h"
#include "gp_launch.h"

namespace {

constexpr long long kMaxCells = GP_NOALLOC_MAX_CELLS;
// per cell: U1 (8) + dU (3 x 8) + C_dt (3) + two face buffers (2 x 3)
// + UCT face data (3 x 6) + edge EMFs (3)
constexpr long long kDoublesPerCell = 8 + 24 + 3 + 6 + 18 + 3;
constexpr long long kHeader = 64;  // step scalars, 512 bytes

static_assert(kDoublesPerCell == GP_NOALLOC_DOUBLES_PER_CELL, "scratch layout");

__device__ __align__(256) double g_noalloc_scratch[kHeader + kMaxCells * kDoublesPerCell];

struct Scalars {  // first bytes of the scratch array
  double dt;
  double dtdx[3];
  unsigned long long invdt_bits;
  uint32_t err;
  uint32_t pad;
};

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device.  The host-side
// symbol is only a stand-in: a kernel given &g_noalloc_scratch would fault.
int scratch_address(double** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return GP_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      return GP_ERR_CUDA;
    }
    g_addr[dev] = static_cast<double*>(p);
  }
  *out = g_addr[dev];
  return GP_OK;
}

}  // namespace

extern "C" int gp_advance_step_noalloc(const gp_grid_desc* grid, const gp_scheme* scheme,
                                       double* Uc, double* Vc, double* Vs0, double* Vs1,
                                       double* Vs2, double dt, void* stream,
                                       gp_step_out* out) {
  if (!grid || !scheme || !Uc || !Vc) return gp::set_last_error(GP_ERR_INVALID, "null argument");
  // the combinations gp_create accepts, then this entry point's own limits
  int rc = gp::validate_scheme(grid, scheme);
  if (rc) return rc;
  if (scheme->rk_stages != 2)
    return gp::set_last_error(GP_ERR_UNSUPPORTED, "the no-allocation step is RK2 only");
  if (scheme->reconstruction != GP_REC_LINEAR && scheme->reconstruction != GP_REC_PARABOLIC)
    return gp::set_last_error(GP_ERR_UNSUPPORTED,
                              "the no-allocation step takes LINEAR or PARABOLIC reconstruction");
  if (!(dt > 0.0)) return gp::set_last_error(GP_ERR_INVALID, "dt must be positive");
  const int ndim = grid->ndim;
  const int nx = grid->nint[0], ny = grid->nint[1], nz = ndim == 3 ? grid->nint[2] : 1;
  const long long n = (long long)nx * ny * nz;
  if (n > kMaxCells)
    return gp::set_last_error(GP_ERR_INVALID,
                              "grid larger than GP_NOALLOC_MAX_CELLS (the static scratch)");
  const bool mhd = scheme->physics != GP_HD;
  if (mhd && (!Vs0 || !Vs1 || (ndim == 3 && !Vs2)))
    return gp::set_last_error(GP_ERR_INVALID, "null face-field pointer");
  for (int d = 0; d < ndim; d++)
    if (grid->lbound[d] != GP_BC_PERIODIC || grid->rbound[d] != GP_BC_PERIODIC)
      return gp::set_last_error(GP_ERR_UNSUPPORTED,
                                "the no-allocation step takes periodic sides only");

  double* base = nullptr;
  rc = scratch_address(&base);
  if (rc) return gp::set_last_error(rc, "cannot find the scratch array on this device");
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  double dx[3];
  gp::cell_widths(grid, dx);
  // carve the scratch
  Scalars* sc = reinterpret_cast<Scalars*>(base);
  double* p = base + kHeader;
  double* U1 = p;               p += 8 * n;
  double* dU = p;               p += 24 * n;
  double* Cdt = p;              p += 3 * n;
  double* B1[3];
  double* B2[3];
  for (int d = 0; d < 3; d++) { B1[d] = p + d * n; }
  p += 3 * n;
  for (int d = 0; d < 3; d++) { B2[d] = p + d * n; }
  p += 3 * n;
  void* ct[3][6];
  const bool mixed = scheme->precision == GP_MIXED;
  for (int d = 0; d < 3; d++)
    for (int r = 0; r < 6; r++) {
      ct[d][r] = mixed ? static_cast<void*>(reinterpret_cast<float*>(p) + (6 * d + r) * n)
                       : static_cast<void*>(p + (6 * d + r) * n);
    }
  p += 18 * n;
  double* Ee[3] = {p, p + n, p + 2 * n};

  // step scalars (the reduction word and the error word start at zero)
  Scalars hs;
  std::memset(&hs, 0, sizeof(hs));
  hs.dt = dt;
  for (int d = 0; d < 3; d++) hs.dtdx[d] = dt / dx[d];
  if (cudaMemcpyAsync(sc, &hs, sizeof(hs), cudaMemcpyHostToDevice, s) != cudaSuccess)
    return gp::set_last_error(GP_ERR_CUDA, "cannot write the step scalars");

  gp::StageDesc d;
  std::memset(&d, 0, sizeof(d));
  d.V = Vc;
  d.Vout = Vc;
  d.dU = dU;
  d.Cdt = Cdt;
  d.dtdx = sc->dtdx;
  d.gamma = scheme->gamma;
  d.small_rho = scheme->small_rho;
  d.small_prs = scheme->small_prs;
  d.invdt_bits = &sc->invdt_bits;
  d.err = &sc->err;
  double* Bn[3] = {Vs0, Vs1, Vs2};
  for (int q = 0; q < 3; q++) {
    d.dx[q] = dx[q];
    d.Ee[q] = Ee[q];
    for (int r = 0; r < 6; r++) d.ct[q][r] = ct[q][r];
  }
  gp::GridDims g{nx, ny, nz, n};
  const bool ppm = scheme->reconstruction == GP_REC_PARABOLIC;
  gp::SchemeKey key{scheme->physics, ndim, scheme->riemann, scheme->ct_emf,
                    ppm ? 4 /* LIM_PPM */ : scheme->limiter};
  int seg = 64;
  {
    const long long cols = (long long)nx * (ndim == 3 ? nz : 1);
    while (seg > 4 && cols * ((ny + seg - 1) / seg) < 148LL * 1024) seg /= 2;
  }
  auto launch = [&](const gp::StageDesc& sd) {
    return mixed ? gp::launch_stage_mixed(sd, g, key, seg, s, nullptr)
                 : gp::launch_stage_fp64(sd, g, key, seg, s, nullptr);
  };
  // stage 1: (U, B) -> (U1, B1)
  d.stage = 1;
  d.U0 = Uc;
  d.Uc = Uc;
  d.Uout = U1;
  for (int q = 0; q < 3; q++) {
    d.Bs[q] = (mhd && q < ndim) ? Bn[q] : nullptr;
    d.Bs0[q] = d.Bs[q];
    d.Bsout[q] = (mhd && q < ndim) ? B1[q] : nullptr;
  }
  if (launch(d) != 0) return gp::set_last_error(GP_ERR_UNSUPPORTED, "scheme not built");
  // stage 2: (U, U1, B, B1) -> (U in place, B2), then B2 -> caller's B
  d.stage = 2;
  d.w0 = d.w1 = d.wr = 0.5;  // RK2 (Src/rk_step.cpp:30-35)
  d.Uc = U1;
  d.Uout = Uc;
  for (int q = 0; q < 3; q++) {
    d.Bs[q] = (mhd && q < ndim) ? B1[q] : nullptr;
    d.Bs0[q] = (mhd && q < ndim) ? Bn[q] : nullptr;
    d.Bsout[q] = (mhd && q < ndim) ? B2[q] : nullptr;
  }
  if (launch(d) != 0) return gp::set_last_error(GP_ERR_UNSUPPORTED, "scheme not built");
  if (mhd)
    for (int q = 0; q < ndim; q++)
      if (cudaMemcpyAsync(Bn[q], B2[q], sizeof(double) * n, cudaMemcpyDeviceToDevice, s) !=
          cudaSuccess)
        return gp::set_last_error(GP_ERR_CUDA, "cannot copy the new face field back");
  // launch failures show here; peeking leaves the thread's error state as it is
  if (cudaPeekAtLastError() != cudaSuccess) return gp::set_last_error(GP_ERR_CUDA, "launch failed");
  if (cudaMemcpyAsync(&hs, sc, sizeof(hs), cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return gp::set_last_error(GP_ERR_CUDA, "cannot read the step scalars");
  if (cudaStreamSynchronize(s) != cudaSuccess)
    return gp::set_last_error(GP_ERR_CUDA, "the step failed on the device");
  // invDt_hyp = max(C_dt)/dim (Src/update_stage.cpp:422-435), NextTimeStep
  double inv;
  std::memcpy(&inv, &hs.invdt_bits, sizeof(inv));
  inv = inv / (double)ndim;
  if (out) {
    out->err_bits = hs.err;
    out->invDt_hyp = inv;
    out->dt_next = gp_next_time_step(inv, scheme->cfl, scheme->cfl_max_var, dt);
  }
  return (hs.err & (1u << 15)) ? GP_ERR_QUIT : GP_OK;
}
