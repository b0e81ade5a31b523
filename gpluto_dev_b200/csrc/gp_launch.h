// gp_launch.h -- host-side launch interface between the C-ABI layer and the
// per-precision kernel translation units (gp_launch.cu compiled twice: FP64
// with -fmad=false, mixed FP32-flux with contraction allowed).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gp {

struct StageDesc {
  const double* V;
  const double* Bs[3];
  const double* Bs0[3];
  double* Bsout[3];
  double* dU;          // float arrays in the mixed form (see gp_launch.cu)
  double* Cdt;
  const double* U0;
  const double* Uc;
  double* Uout;
  double* Vout;
  void* ct[3][6];      // double (FP64 form) or float (mixed form)
  double* Ee[3];       // float arrays in the mixed form
  const double* dtdx;  // device pointer to dt/dx_d
  double dx[3];
  double gamma, small_rho, small_prs;
  int stage;
  double w0, w1, wr;   // combine weights of stages >= 2
  unsigned long long* invdt_bits;
  uint32_t* err;
};

struct GridDims {
  int nx, ny, nz;
  long long n;
  unsigned outflow = 0u;  // bit 2d / 2d+1: low / high side of direction d is outflow
  // domain and ghosted-box cell ranges of a padded grid (see Grid3)
  int ilo[3] = {0, 0, 0}, ihi[3] = {0x3fffffff, 0x3fffffff, 0x3fffffff};
  int glo[3] = {0, 0, 0}, ghi[3] = {0x3fffffff, 0x3fffffff, 0x3fffffff};
};

struct SchemeKey {
  int physics, ndim, riemann, ct, limiter;
};

// Launch the kernels of one RK stage on `s`.  Returns 0 on success, a
// negative value if the scheme combination has no compiled kernels.
// `ev` (may be null) receives an event pair around every kernel launch, in
// launch order (2*stage_launch_count(k) events).
int launch_stage_fp64(const StageDesc& d, const GridDims& g, const SchemeKey& k,
                      int seg, cudaStream_t s, cudaEvent_t* ev);
int launch_stage_mixed(const StageDesc& d, const GridDims& g, const SchemeKey& k,
                       int seg, cudaStream_t s, cudaEvent_t* ev);
int launch_prim2cons(int physics, const double* V, double* U, long long n, double gamma,
                     cudaStream_t s);
// Sets the text returned by gp_last_error on this thread; returns `code`.
int set_last_error(int code, const char* msg);

// Resident blocks per SM the y/z marching sweeps are compiled for
// (SWEEP_THREADS threads each).
int sweep_m_blocks_per_sm(int physics, bool mixed);

// Number of kernel launches one stage issues for this scheme, and their names.
int stage_launch_count(const SchemeKey& k);
const char* stage_kernel_name(const SchemeKey& k, int idx);

}  // namespace gp
