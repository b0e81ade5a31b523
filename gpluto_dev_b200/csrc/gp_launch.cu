// gp_launch.cu -- template dispatch of the stage kernels.
//
// Compiled twice: with GP_MIXED=0 (FP64 everywhere, -fmad=false so that the
// plain form keeps the reference's rounding sequence) and GP_MIXED=1 (FP32
// reconstruction/limiter/Riemann/EMF arithmetic, FP64 accumulation, CT
// update and con2prim).  In the mixed form the per-direction flux
// differences, inverse-dt terms, UCT face data and edge EMFs -- all computed
// from FP32 fluxes -- are stored as float (the StageDesc pointers then point
// at float arrays); the FP64 form stores them as double.
#include "gp_kernels.cuh"
#include "gp_launch.h"

#ifndef GP_MIXED
#define GP_MIXED 0
#endif
// GP_PART selects the schemes this unit instantiates (0 HD, 1 MHD with
// HLLD/HLL, 2 RMHD, 3 MHD with Lax-Friedrichs/HLLC), so that the build
// compiles the four in parallel; the entry points
// launch_stage_{fp64,mixed}_p<part> are joined by gp_launch_dispatch.cu.
#ifndef GP_PART
#error "compile gp_launch.cu with -DGP_PART=0, 1, 2 or 3"
#endif
#define GP_CAT2(a, b) a##b
#define GP_CAT(a, b) GP_CAT2(a, b)

namespace gp {

#if GP_MIXED
using RT = float;
using CTT = float;
#define GP_LAUNCH_STAGE GP_CAT(launch_stage_mixed_p, GP_PART)
#else
using RT = double;
using CTT = double;
#define GP_LAUNCH_STAGE GP_CAT(launch_stage_fp64_p, GP_PART)
#endif

static StageArgs<CTT> make_args(const StageDesc& d) {
  StageArgs<CTT> a;
  a.V = d.V;
  for (int q = 0; q < 3; q++) {
    a.Bs[q] = d.Bs[q];
    a.Bs0[q] = d.Bs0[q];
    a.Bsout[q] = d.Bsout[q];
    a.Ee[q] = reinterpret_cast<CTT*>(d.Ee[q]);
    a.dx[q] = d.dx[q];
    for (int r = 0; r < 6; r++) a.ct[q][r] = static_cast<CTT*>(d.ct[q][r]);
  }
  a.dtdx = d.dtdx;
  a.dU = reinterpret_cast<CTT*>(d.dU);
  a.Cdt = reinterpret_cast<CTT*>(d.Cdt);
  a.U0 = d.U0;
  a.Uc = d.Uc;
  a.Uout = d.Uout;
  a.Vout = d.Vout;
  a.gamma = d.gamma;
  a.small_rho = d.small_rho;
  a.small_prs = d.small_prs;
  a.stage = d.stage;
  a.w0 = d.w0;
  a.w1 = d.w1;
  a.wr = d.wr;
  a.invdt_bits = d.invdt_bits;
  a.err = d.err;
  return a;
}

template <int PHYS, int NV, int NDIM, int RS, int CT, int LIM>
static void run_stage(const StageArgs<CTT>& a, const GridDims& gd, int seg, cudaStream_t s,
                      cudaEvent_t* ev) {
  Grid3 g{gd.nx, gd.ny, gd.nz, gd.n, gd.outflow};
  for (int d = 0; d < 3; d++) {
    g.ilo[d] = gd.ilo[d];
    g.ihi[d] = gd.ihi[d];
    g.glo[d] = gd.glo[d];
    g.ghi[d] = gd.ghi[d];
  }
  int kidx = 0;
  auto pre = [&]() { if (ev) cudaEventRecord(ev[2 * kidx], s); };
  auto post = [&]() { if (ev) cudaEventRecord(ev[2 * kidx + 1], s); kidx++; };
  {
    const int rows = gd.ny * gd.nz;
    const int wpb = SWEEP_THREADS / 32;
    dim3 grid((rows + wpb - 1) / wpb);
    pre();
    sweep_x_kernel<PHYS, NV, NDIM, RS, CT, LIM, RT, CTT><<<grid, SWEEP_THREADS, 0, s>>>(a, g);
    post();
  }
  // y/z sweeps: grid (x-blocks, transverse index x pencil segments); when
  // nx is not a multiple of the block, a 1-D grid over (x, transverse)
  // columns numbered together, so that no block is part-empty (FLAT)
  const bool flat = gd.nx % SWEEP_THREADS != 0;
  auto grid_m = [&](int nt, int nseg) {
    if (flat)
      return dim3((unsigned)(((long long)gd.nx * nt + SWEEP_THREADS - 1) / SWEEP_THREADS * nseg));
    return dim3(gd.nx / SWEEP_THREADS, nt * nseg);
  };
  {
    const dim3 grid = grid_m(gd.nz, (gd.ny + seg - 1) / seg);
    pre();
    if (flat)
      sweep_m_kernel<PHYS, NV, NDIM, RS, CT, LIM, 1, RT, CTT, true><<<grid, SWEEP_THREADS, 0, s>>>(a, g, seg);
    else
      sweep_m_kernel<PHYS, NV, NDIM, RS, CT, LIM, 1, RT, CTT, false><<<grid, SWEEP_THREADS, 0, s>>>(a, g, seg);
    post();
  }
  if constexpr (NDIM == 3) {
    const dim3 grid = grid_m(gd.ny, (gd.nz + seg - 1) / seg);
    pre();
    if (flat)
      sweep_m_kernel<PHYS, NV, NDIM, RS, CT, LIM, 2, RT, CTT, true><<<grid, SWEEP_THREADS, 0, s>>>(a, g, seg);
    else
      sweep_m_kernel<PHYS, NV, NDIM, RS, CT, LIM, 2, RT, CTT, false><<<grid, SWEEP_THREADS, 0, s>>>(a, g, seg);
    post();
  }
  const unsigned nb = (unsigned)((gd.n + 255) / 256);
  if constexpr (PHYS != PHYS_HD) {
    pre();
    if constexpr (CT == CT_ARITH) {
      emf_arith_kernel<NDIM, RT, CTT><<<nb, 256, 0, s>>>(a, g);
    } else if constexpr (CT == CT_CONTACT) {
      emf_contact_kernel<NDIM, RT, CTT><<<nb, 256, 0, s>>>(a, g);
    } else if constexpr (NDIM == 3 && (sizeof(RT) == 8 || five_point<LIM>())) {  // plane-staged EMF
      using T = EmfTile<LIM, CTT>;
      cudaFuncSetAttribute(emf_tile_kernel<LIM, RT, CTT>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, T::SMEM);
      // the longest segment (<= ET_SEGMENT planes) that still gives about
      // four waves of resident blocks over 148 SMs
      const long long cols = (long long)((gd.nx + ETX - 1) / ETX) * ((gd.ny + ETY - 1) / ETY);
      int sz = ET_SEGMENT;
      while (sz > 4 && cols * ((gd.nz + sz - 1) / sz) < 148LL * emf_tile_minb<RT>() * 4) sz /= 2;
      dim3 grid((gd.nx + ETX - 1) / ETX, (gd.ny + ETY - 1) / ETY, (gd.nz + sz - 1) / sz);
      emf_tile_kernel<LIM, RT, CTT><<<grid, dim3(ETX, ETY), T::SMEM, s>>>(a, g, sz);
    } else if constexpr (NDIM == 3) {  // mixed PLM/PPM: z-marching EMF, loads through L1
      // the longest segment (<= EMF_SEGMENT planes) that still gives about
      // four waves of blocks over 148 SMs (3 blocks per SM)
      const long long cols = (long long)((gd.nx + EMF_TX - 1) / EMF_TX) *
                             ((gd.ny + EMF_TY - 1) / EMF_TY);
      int sz = EMF_SEGMENT;
      while (sz > 4 && cols * ((gd.nz + sz - 1) / sz) < 148LL * 3 * 4) sz /= 2;
      dim3 grid((gd.nx + EMF_TX - 1) / EMF_TX, (gd.ny + EMF_TY - 1) / EMF_TY,
                (gd.nz + sz - 1) / sz);
      emf_march_kernel<LIM, RT, CTT><<<grid, dim3(EMF_TX, EMF_TY), 0, s>>>(a, g, sz);
    } else {
      emf_kernel<NDIM, LIM, RT, CTT><<<nb, 256, 0, s>>>(a, g);
    }
    post();
  }
  pre();
  finish_kernel<PHYS, NV, NDIM, CTT><<<nb, 256, 0, s>>>(a, g);
  post();
}

template <int PHYS, int NV, int NDIM, int RS, int CT>
static int by_lim(const StageArgs<CTT>& a, const GridDims& g, int lim, int seg, cudaStream_t s,
                  cudaEvent_t* ev) {
  switch (lim) {
    case LIM_MC: run_stage<PHYS, NV, NDIM, RS, CT, LIM_MC>(a, g, seg, s, ev); return 0;
    case LIM_VL: run_stage<PHYS, NV, NDIM, RS, CT, LIM_VL>(a, g, seg, s, ev); return 0;
    case LIM_MINMOD: run_stage<PHYS, NV, NDIM, RS, CT, LIM_MINMOD>(a, g, seg, s, ev); return 0;
    case LIM_PPM: run_stage<PHYS, NV, NDIM, RS, CT, LIM_PPM>(a, g, seg, s, ev); return 0;
    case LIM_MP5: run_stage<PHYS, NV, NDIM, RS, CT, LIM_MP5>(a, g, seg, s, ev); return 0;
    case LIM_WENOZ: run_stage<PHYS, NV, NDIM, RS, CT, LIM_WENOZ>(a, g, seg, s, ev); return 0;
    case LIM_LIMO3: run_stage<PHYS, NV, NDIM, RS, CT, LIM_LIMO3>(a, g, seg, s, ev); return 0;
    case LIM_WENO3: run_stage<PHYS, NV, NDIM, RS, CT, LIM_WENO3>(a, g, seg, s, ev); return 0;
    case LIM_FLAT: run_stage<PHYS, NV, NDIM, RS, CT, LIM_FLAT>(a, g, seg, s, ev); return 0;
    case LIM_VANALBADA:
      run_stage<PHYS, NV, NDIM, RS, CT, LIM_VANALBADA>(a, g, seg, s, ev);
      return 0;
    case LIM_OSPRE: run_stage<PHYS, NV, NDIM, RS, CT, LIM_OSPRE>(a, g, seg, s, ev); return 0;
    case LIM_UMIST: run_stage<PHYS, NV, NDIM, RS, CT, LIM_UMIST>(a, g, seg, s, ev); return 0;
    default: return -1;
  }
}

template <int NDIM>
static int by_scheme(const StageArgs<CTT>& a, const GridDims& g, const SchemeKey& k, int seg,
                     cudaStream_t s, cudaEvent_t* ev) {
#if GP_PART == 1
  // MHD with the HLLD and HLL solvers
  if (k.physics == PHYS_MHD && k.ct == CT_CONTACT) {
    if (k.riemann == RS_HLLD)
      return by_lim<PHYS_MHD, 8, NDIM, RS_HLLD, CT_CONTACT>(a, g, k.limiter, seg, s, ev);
    if (k.riemann == RS_HLL)
      return by_lim<PHYS_MHD, 8, NDIM, RS_HLL, CT_CONTACT>(a, g, k.limiter, seg, s, ev);
    return -1;
  }
  if (k.physics == PHYS_MHD && k.ct == CT_ARITH) {
    if (k.riemann == RS_HLLD)
      return by_lim<PHYS_MHD, 8, NDIM, RS_HLLD, CT_ARITH>(a, g, k.limiter, seg, s, ev);
    if (k.riemann == RS_HLL)
      return by_lim<PHYS_MHD, 8, NDIM, RS_HLL, CT_ARITH>(a, g, k.limiter, seg, s, ev);
    return -1;
  }
  if (k.physics == PHYS_MHD) {
    if (k.riemann == RS_HLLD && k.ct == CT_UCT_HLLD)
      return by_lim<PHYS_MHD, 8, NDIM, RS_HLLD, CT_UCT_HLLD>(a, g, k.limiter, seg, s, ev);
    if (k.riemann == RS_HLLD && k.ct == CT_UCT_HLL)
      return by_lim<PHYS_MHD, 8, NDIM, RS_HLLD, CT_UCT_HLL>(a, g, k.limiter, seg, s, ev);
    if (k.riemann == RS_HLL && k.ct == CT_UCT_HLL)
      return by_lim<PHYS_MHD, 8, NDIM, RS_HLL, CT_UCT_HLL>(a, g, k.limiter, seg, s, ev);
    return -1;
  }
#endif
#if GP_PART == 3
  // MHD with the Lax-Friedrichs and HLLC solvers (UCT_HLL, ARITHMETIC or CT_CONTACT)
  if (k.physics == PHYS_MHD && k.ct == CT_CONTACT) {
    if (k.riemann == RS_TVDLF)
      return by_lim<PHYS_MHD, 8, NDIM, RS_TVDLF, CT_CONTACT>(a, g, k.limiter, seg, s, ev);
    if (k.riemann == RS_HLLC)
      return by_lim<PHYS_MHD, 8, NDIM, RS_HLLC, CT_CONTACT>(a, g, k.limiter, seg, s, ev);
    return -1;
  }
  if (k.physics == PHYS_MHD && k.ct == CT_ARITH) {
    if (k.riemann == RS_TVDLF)
      return by_lim<PHYS_MHD, 8, NDIM, RS_TVDLF, CT_ARITH>(a, g, k.limiter, seg, s, ev);
    if (k.riemann == RS_HLLC)
      return by_lim<PHYS_MHD, 8, NDIM, RS_HLLC, CT_ARITH>(a, g, k.limiter, seg, s, ev);
    return -1;
  }
  if (k.physics == PHYS_MHD) {
    if (k.riemann == RS_TVDLF && k.ct == CT_UCT_HLL)
      return by_lim<PHYS_MHD, 8, NDIM, RS_TVDLF, CT_UCT_HLL>(a, g, k.limiter, seg, s, ev);
    if (k.riemann == RS_HLLC && k.ct == CT_UCT_HLL)
      return by_lim<PHYS_MHD, 8, NDIM, RS_HLLC, CT_UCT_HLL>(a, g, k.limiter, seg, s, ev);
    return -1;
  }
#endif
#if GP_PART == 2
  if (k.physics == PHYS_RMHD) {
    if (k.riemann == RS_HLLD && k.ct == CT_UCT_HLL)
      return by_lim<PHYS_RMHD, 8, NDIM, RS_HLLD, CT_UCT_HLL>(a, g, k.limiter, seg, s, ev);
    if (k.riemann == RS_HLL && k.ct == CT_UCT_HLL)
      return by_lim<PHYS_RMHD, 8, NDIM, RS_HLL, CT_UCT_HLL>(a, g, k.limiter, seg, s, ev);
    if (k.riemann == RS_TVDLF && k.ct == CT_UCT_HLL)
      return by_lim<PHYS_RMHD, 8, NDIM, RS_TVDLF, CT_UCT_HLL>(a, g, k.limiter, seg, s, ev);
    return -1;
  }
#endif
#if GP_PART == 0
  if (k.physics == PHYS_HD) {
    if (k.riemann == RS_HLLC) return by_lim<PHYS_HD, 5, NDIM, RS_HLLC, 0>(a, g, k.limiter, seg, s, ev);
    if (k.riemann == RS_HLL) return by_lim<PHYS_HD, 5, NDIM, RS_HLL, 0>(a, g, k.limiter, seg, s, ev);
    if (k.riemann == RS_TVDLF)
      return by_lim<PHYS_HD, 5, NDIM, RS_TVDLF, 0>(a, g, k.limiter, seg, s, ev);
    return -1;
  }
#endif
  return -1;
}

int GP_LAUNCH_STAGE(const StageDesc& d, const GridDims& g, const SchemeKey& k, int seg,
                    cudaStream_t s, cudaEvent_t* ev) {
  StageArgs<CTT> a = make_args(d);
  if (k.ndim == 2) return by_scheme<2>(a, g, k, seg, s, ev);
  if (k.ndim == 3) return by_scheme<3>(a, g, k, seg, s, ev);
  return -1;
}

#if !GP_MIXED && GP_PART == 1
int launch_prim2cons(int physics, const double* V, double* U, long long n, double gamma,
                     cudaStream_t s) {
  const unsigned nb = (unsigned)((n + 255) / 256);
  if (physics == PHYS_MHD) prim2cons_kernel<PHYS_MHD, 8><<<nb, 256, 0, s>>>(V, U, n, gamma);
  else if (physics == PHYS_RMHD) prim2cons_kernel<PHYS_RMHD, 8><<<nb, 256, 0, s>>>(V, U, n, gamma);
  else if (physics == PHYS_HD) prim2cons_kernel<PHYS_HD, 5><<<nb, 256, 0, s>>>(V, U, n, gamma);
  else return -1;
  return 0;
}

int stage_launch_count(const SchemeKey& k) {
  int c = 1 + (k.ndim == 3 ? 2 : 1) + 1;  // sweeps + finish
  if (k.physics != PHYS_HD) c += 1;       // emf
  return c;
}

const char* stage_kernel_name(const SchemeKey& k, int idx) {
  static const char* n3m[] = {"sweep_x", "sweep_y", "sweep_z", "emf", "finish"};
  static const char* n2m[] = {"sweep_x", "sweep_y", "emf", "finish"};
  static const char* n3h[] = {"sweep_x", "sweep_y", "sweep_z", "finish"};
  static const char* n2h[] = {"sweep_x", "sweep_y", "finish"};
  if (idx < 0 || idx >= stage_launch_count(k)) return "?";
  if (k.physics != PHYS_HD) return k.ndim == 3 ? n3m[idx] : n2m[idx];
  return k.ndim == 3 ? n3h[idx] : n2h[idx];
}
#endif

}  // namespace gp
