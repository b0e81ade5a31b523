// gp_kernels.cuh -- fused stage kernels of the Godunov step (sm_100a).
//
// Device layout (one grid): interior cells only, structure of arrays,
// x fastest: cell (i,j,k) of variable nv sits at nv*n + i + nx*(j + ny*k).
// Face-normal fields Bs[d] hold the LEFT face of each cell (x_d = i_d - 1/2);
// periodic ghost zones are index wrap-around, never copies (the reference
// fills ghosts by copy, Src/boundary.cpp:502-675; with periodic data the two
// give identical operands, so results agree bit for bit).
//
// One RK stage (Src/update_stage.cpp:57-438 + Src/rk_step.cpp:357-593):
//   sweep_x   : warp per x-row; PLM + Riemann per face, flux difference into
//               dU (=), per-cell inverse dt into Cdt (=), UCT face data.
//   sweep_m<d>: thread per (x, pencil segment) marching along y or z with a
//               register window; dU (+=), Cdt (+=); the last direction fuses
//               the RK combine (writes U_out) and the stage-1 CFL max.
//   emf       : thread per cell, its three edge EMFs (UCT_HLLD / UCT_HLL
//               composition, Src/MHD/CT/ct_emf_average.cpp:535-995).
//   finish    : thread per cell: CT face update of its left faces (and the
//               right faces recomputed for the cell average), RK combine of
//               the faces, cell-centred B average, con2prim -> V, U fixups.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "gp_phys.cuh"
#include "gp_rmhd.cuh"

namespace gp {

constexpr int kNoLimit = 0x3fffffff;

struct Grid3 {
  int nx, ny, nz;
  long long n;  // nx*ny*nz
  // outflow sides handled by index clamping (HD): bit 2d = low side of
  // direction d, bit 2d+1 = high side; every other side wraps
  unsigned outflow = 0u;
  // Grids padded with ghost cells (outflow with constrained transport):
  // the cells [ilo, ihi] are the domain; [glo, ghi] the cells whose faces
  // the reference's sweeps also solve (domain plus its ghost zone).  Only
  // those contribute error bits, and only the domain the CFL maximum.
  int ilo[3] = {0, 0, 0}, ihi[3] = {kNoLimit, kNoLimit, kNoLimit};
  int glo[3] = {0, 0, 0}, ghi[3] = {kNoLimit, kNoLimit, kNoLimit};
};

// whether the face f (along d) of the pencil at transverse cells (ta, tb) is
// one the reference solves: ta, tb inside the ghosted box, f a domain face
__device__ __forceinline__ bool face_counts(const Grid3& g, int d, int f, int a, int ta, int b,
                                            int tb) {
  return f >= g.ilo[d] && f <= g.ihi[d] + 1 && ta >= g.glo[a] && ta <= g.ghi[a] &&
         tb >= g.glo[b] && tb <= g.ghi[b];
}

template <typename CTT>
struct StageArgs {
  const double* V;        // [nvar][n] primitives at stage start
  const double* Bs[3];    // stage-input face fields (left faces)
  const double* Bs0[3];   // face fields at t^n (stage 2)
  double* Bsout[3];       // face fields written by this stage
  CTT* dU;                // [3][nvar][n] flux difference of each direction
  CTT* Cdt;               // [3][n] inverse dt of each direction
  const double* U0;       // U^n
  const double* Uc;       // stage-input U
  double* Uout;           // U written by this stage
  double* Vout;           // primitives written by this stage
  CTT* ct[3][6];          // UCT face data per direction: eb, et, aL, aR, dL, dR
  CTT* Ee[3];             // edge EMFs: Ee[0]=Ex(i,j-1/2,k-1/2), Ee[1]=Ey, Ee[2]=Ez
  const double* dtdx;     // dt/dx_d (3 values in device memory, set per step)
  double dx[3];
  double gamma, small_rho, small_prs;
  int stage;              // 1, 2 (RK2, RK3) or 3 (RK3)
  double w0, w1, wr;      // combine weights of stages >= 2: U = w0 U^n + w1 U_c + wr R
                          // (Src/rk_step.cpp:30-61)
  unsigned long long* invdt_bits;  // max over cells of Cdt (stage 1)
  uint32_t* err;          // OR of error bits
};

__device__ __forceinline__ int wrapi(int i, int n) {
  return i < 0 ? i + n : (i >= n ? i - n : i);
}

// Cell index along direction d for an index up to n past either end: a
// periodic side wraps; an outflow side gives the nearest interior cell, the
// value OutflowBoundary copies into the ghost zone (Src/boundary.cpp:677-780).
__device__ __forceinline__ int gidx(int i, int n, unsigned outflow, int d) {
  if (i < 0) return ((outflow >> (2 * d)) & 1u) ? 0 : i + n;
  if (i >= n) return ((outflow >> (2 * d + 1)) & 1u) ? n - 1 : i - n;
  return i;
}

template <int NV, typename R>
__device__ __forceinline__ void load_cell(const double* __restrict__ V, long long n,
                                          long long c, R* v) {
#pragma unroll
  for (int nv = 0; nv < NV; nv++) v[nv] = (R)__ldg(V + nv * n + c);
}

// Asynchronous global->shared copies (cp.async, per thread, 8 bytes): the
// sweeps stage the next stencil cell while the current face is solved, so the
// prefetch costs no registers.  Each thread reads back only what it staged.
__device__ __forceinline__ void cp_async8(double* smem, const double* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait1() {
  asm volatile("cp.async.wait_group 1;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait0() {
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

#ifndef GP_SWEEP_MINB
#define GP_SWEEP_MINB 3
#endif
constexpr int SWEEP_THREADS = 128;

// Resident 128-thread blocks per SM the sweep kernels are compiled for
// (register budget 65536 / (128 * blocks)), measured at 256^3 on 3-D MHD:
// FP64 x-sweep 3 (168 registers), FP64 y/z sweeps 4 (128), mixed form 5
// (102).  The relativistic solver (FP64 in both forms) runs its x-sweep at
// 2 (5.01 -> 4.83 ms FP64, 4.33 -> 4.06 ms mixed at 192^3: fewer warps
// walking its long code at once) and its y/z sweeps at 3 (at 2 they lost
// 4%).
template <int PHYS, typename R>
constexpr int sweep_x_minb() {
  return PHYS == PHYS_RMHD ? 2 : (sizeof(R) == 4 ? 5 : 3);
}
template <int PHYS, typename R>
constexpr int sweep_m_minb() {
  return PHYS == PHYS_RMHD ? 3 : (sizeof(R) == 4 ? 5 : 4);
}

// whether conserved component nv receives a flux difference that survives
// the stage (the cell-centred field along active directions is overwritten
// by the face average, Src/MHD/CT/ct_field_average.cpp:378-410)
template <int PHYS, int NDIM>
__device__ __forceinline__ constexpr bool rhs_var(int nv) {
  return !(PHYS != PHYS_HD && nv >= BX1 && nv < BX1 + NDIM);
}

// Riemann dispatch for one interface.
template <int PHYS, int RS, int CT, int DIR, typename R>
__device__ __forceinline__ R riemann(const R* vl, const R* vr, R* flux, R gamma, R Bn,
                                     CTFace<R>& ct, uint32_t& err) {
  if constexpr (PHYS == PHYS_MHD) {
    R cm;
    if constexpr (RS == RS_HLLD) cm = mhd_hlld<DIR, CT>(vl, vr, flux, gamma, Bn, ct);
    else if constexpr (RS == RS_TVDLF) cm = mhd_tvdlf<DIR>(vl, vr, flux, gamma, ct);
    else if constexpr (RS == RS_HLLC) cm = mhd_hllc<DIR>(vl, vr, flux, gamma, ct);
    else cm = mhd_hll<DIR>(vl, vr, flux, gamma, ct);
    if constexpr (CT == CT_ARITH || CT == CT_CONTACT) {
      // CT_Store_Arith (Src/MHD/CT/ct_store.hpp:74-93): the face's two
      // induction fluxes, e[b][n] = -F(B_t) and e[t][n] = F(B_b)
      ct.eb = -flux[BX1 + (DIR + 1) % 3];
      ct.et = flux[BX1 + (DIR + 2) % 3];
      if constexpr (CT == CT_CONTACT) {
        // the sign of the mass flux (zero within eps_CT_CONTACT = 1e-6,
        // Src/MHD/CT/ct.hpp:110), kept as the weight the corner
        // integration gives the left cell (Src/MHD/CT/ct_emf_average.cpp:137-143)
        const R fr = flux[RHO];
        ct.aL = fr > R(1.e-6) ? R(1) : (fr < R(-1.e-6) ? R(0) : R(0.5));
      }
    }
    return cm;
  } else if constexpr (PHYS == PHYS_RMHD) {
    if constexpr (sizeof(R) == sizeof(double)) {
      return rmhd_riemann<DIR, RS>(vl, vr, flux, gamma, ct, err);
    } else {
      // the relativistic HLLD (secant iteration, quartic speeds, nested
      // con2prim) is not usable in FP32 at Lorentz factors ~10: the mixed
      // form solves it in FP64 on the FP32 reconstructed states
      double dl[8], dr[8], df[8];
#pragma unroll
      for (int nv = 0; nv < 8; nv++) { dl[nv] = vl[nv]; dr[nv] = vr[nv]; }
      CTFace<double> cd;
      double cm = rmhd_riemann<DIR, RS>(dl, dr, df, (double)gamma, cd, err);
#pragma unroll
      for (int nv = 0; nv < 8; nv++) flux[nv] = (R)df[nv];
      ct.eb = (R)cd.eb; ct.et = (R)cd.et; ct.aL = (R)cd.aL;
      ct.aR = (R)cd.aR; ct.dL = (R)cd.dL; ct.dR = (R)cd.dR;
      return (R)cm;
    }
  } else {
    if constexpr (RS == RS_HLLC) return hd_hllc<DIR>(vl, vr, flux, gamma);
    else if constexpr (RS == RS_TVDLF) return hd_tvdlf<DIR>(vl, vr, flux, gamma);
    else return hd_hll<DIR>(vl, vr, flux, gamma);
  }
}

// Flux difference of one cell along `dir` (Src/MHD/rhs.cpp:383-386, 756,
// 981) and its inverse-dt term (Src/MHD/rhs.cpp:523 and the += at 756, 981),
// written to the direction's own arrays; the finish kernel sums them in the
// order x, y, z as Src/update_stage.cpp:173-184/272-284/369-380 does.
template <int PHYS, int NV, int NDIM, typename R, typename CTT>
__device__ __forceinline__ void cell_update(const StageArgs<CTT>& a, long long n,
                                            long long c, const R* Fl, const R* Fr,
                                            R cml, R cmr, int dir) {
  CTT* du = a.dU + (long long)dir * NV * n;
  if constexpr (sizeof(R) == sizeof(double)) {
    const double dtdx = a.dtdx[dir];
#pragma unroll
    for (int nv = 0; nv < NV; nv++) {
      if (!rhs_var<PHYS, NDIM>(nv)) continue;
      du[nv * n + c] = (CTT)(-dtdx * ((double)Fr[nv] - (double)Fl[nv]));
    }
    // stored in every stage although only stage 1's CFL maximum reads it
    // (Src/update_stage.cpp:422-435): a store conditional on the stage made
    // the FP64 y/z sweeps 40% slower at 256^3
    a.Cdt[(long long)dir * n + c] = (CTT)(0.5 * ((double)cml + (double)cmr) / a.dx[dir]);
  } else {
    // mixed form: the stored difference is FP32, so it is formed in FP32
    // (no widening and narrowing conversions, no FP64 division)
    const R dtdx = (R)a.dtdx[dir];
#pragma unroll
    for (int nv = 0; nv < NV; nv++) {
      if (!rhs_var<PHYS, NDIM>(nv)) continue;
      du[nv * n + c] = (CTT)(-dtdx * (Fr[nv] - Fl[nv]));
    }
    a.Cdt[(long long)dir * n + c] = (CTT)(R(0.5) * (cml + cmr) / (R)a.dx[dir]);
  }
}

// Face data for the edge EMFs: the two face EMFs and, for the upwind
// averages, the four weights; CT_CONTACT keeps one weight (the contact's),
// ARITHMETIC none.
template <int CT, typename R, typename CTT>
__device__ __forceinline__ void store_ct(const StageArgs<CTT>& a, int dir, long long f,
                                         const CTFace<R>& ct) {
  a.ct[dir][0][f] = (CTT)ct.eb;
  a.ct[dir][1][f] = (CTT)ct.et;
  if constexpr (CT == CT_ARITH) return;
  a.ct[dir][2][f] = (CTT)ct.aL;
  if constexpr (CT == CT_CONTACT) return;
  a.ct[dir][3][f] = (CTT)ct.aR;
  a.ct[dir][4][f] = (CTT)ct.dL;
  a.ct[dir][5][f] = (CTT)ct.dR;
}

// ---------------------------------------------------------------------
// x sweep: one warp per x-row, 32 faces per chunk, neighbours by shuffle.
// Face f (between cells f-1 and f) is computed by lane f%32; the lane then
// updates cell f-1.  The first face's flux is kept for cell nx-1.
// ---------------------------------------------------------------------
// Staging area of one 128-thread block: [2 buffers][SL values][128 threads]
// (+ [2 buffers][4 warps][NV] for the second-next cell with PPM).
template <int NV, int LIM = LIM_MC>
constexpr int sweep_x_stage_doubles() {
  return 2 * (2 * NV + 1) * SWEEP_THREADS +
         ((LIM == LIM_PPM || five_point<LIM>()) ? 2 * (SWEEP_THREADS / 32) * NV : 0);
}
template <int NV>
constexpr int sweep_m_stage_doubles() { return 2 * (NV + 1) * SWEEP_THREADS; }

// Piecewise parabolic x-row (one warp per row).  Lane l of a chunk owns
// cell/face f = c0 + l: it forms the constrained value of face f from cells
// f-2..f+1 (neighbours by shuffle, cells c0-1 and c0-2 carried from the
// previous chunk), takes face f+1 from lane l+1 -- or, for lane 31 and the
// last cell of the row, forms it itself from the staged cells f+1 and f+2 --
// and limits the parabola of cell f.  Each face value is computed once,
// which gives the same bits as the reference's per-cell evaluation
// (Src/States/ppm_states.cpp:129-163): both evaluations are one expression
// of the same four cells.
template <int PHYS, int NV, int NDIM, int RS, int CT, typename R, typename CTT>
__device__ __forceinline__ void sweep_x_row_ppm(const StageArgs<CTT>& a, const Grid3& g, int row,
                                                double* stg_, int tid) {
  constexpr unsigned FULL = 0xffffffffu;
  constexpr int SL = 2 * NV + 1;  // staged doubles per lane: V[f], V[f+1], Bs[f]
  constexpr int NW = SWEEP_THREADS / 32;
  double(*stg)[SL][SWEEP_THREADS] = reinterpret_cast<double(*)[SL][SWEEP_THREADS]>(stg_);
  double(*stg2)[NW][NV] = reinterpret_cast<double(*)[NW][NV]>(stg_ + 2 * SL * SWEEP_THREADS);
  const int lane = tid & 31, w = tid >> 5;
  if (row >= g.ny * g.nz) return;  // warp-uniform
  const int nx = g.nx;
  const unsigned ob = g.outflow;
  // faces solved: nx (periodic: face nx is face 0) or nx+1 (outflow high side)
  const int nf = nx + (int)((ob >> 1) & 1u);
  const long long n = g.n;
  const long long rb = (long long)row * nx;
  const R gamma = (R)a.gamma;

  // carried: cells c0-1, c0-2; left state at face c0 (from cell c0-1); flux
  // and signal speed of face c0-1
  R pV1[NV], pV2[NV], pVLn[NV], pF[NV], pCm = R(0);
  {
    R q[5][NV];
#pragma unroll
    for (int m = 0; m < 5; m++) load_cell<NV>(a.V, n, rb + gidx(m - 3, nx, ob, 0), q[m]);
    R vrp[NV];
#pragma unroll
    for (int nv = 0; nv < NV; nv++) {
      const R fa = ppm_face(q[0][nv], q[1][nv], q[2][nv], q[3][nv]);  // face nx-1
      const R fb = ppm_face(q[1][nv], q[2][nv], q[3][nv], q[4][nv]);  // face nx = 0
      R dvp, dvm;
      ppm_cell(q[2][nv], fa, fb, dvp, dvm);
      pVLn[nv] = q[2][nv] + dvp;
      vrp[nv] = q[2][nv] + dvm;
      pV1[nv] = q[2][nv];
      pV2[nv] = q[1][nv];
      pF[nv] = R(0);
    }
    if constexpr (PHYS == PHYS_RMHD) rmhd_vel_limit<NV>(q[2], vrp, pVLn);
  }
  R fF[NV], fCm = R(0);
  R F[NV], cm = R(0);
#pragma unroll
  for (int nv = 0; nv < NV; nv++) { fF[nv] = R(0); F[nv] = R(0); }
  uint32_t err = 0;

  auto stage_chunk = [&](int c0, int b) {
    const int f = c0 + lane;
    const int fc = f < nx ? f : nx - 1;
#pragma unroll
    for (int nv = 0; nv < NV; nv++) cp_async8(&stg[b][nv][tid], a.V + nv * n + rb + fc);
    if (lane == 31 || f + 1 >= nf) {
      const int fp = gidx(fc + 1, nx, ob, 0);
#pragma unroll
      for (int nv = 0; nv < NV; nv++) cp_async8(&stg[b][NV + nv][tid], a.V + nv * n + rb + fp);
    }
    if (f < nf && (lane == 31 || f + 1 >= nf)) {  // one lane per chunk
      const int fp2 = gidx(fc + 2, nx, ob, 0);
#pragma unroll
      for (int nv = 0; nv < NV; nv++) cp_async8(&stg2[b][w][nv], a.V + nv * n + rb + fp2);
    }
    if constexpr (PHYS != PHYS_HD) cp_async8(&stg[b][2 * NV][tid], a.Bs[0] + rb + fc);
    cp_async_commit();
  };
  stage_chunk(0, 0);
  int buf = 0;
  for (int c0 = 0; c0 < nf; c0 += 32, buf ^= 1) {
    const int f = c0 + lane;
    const bool act = f < nf;
    stage_chunk(c0 + 32 < nf ? c0 + 32 : c0, buf ^ 1);   // prefetch the next chunk
    cp_async_wait1();
    const bool selfp1 = (lane == 31) || (f + 1 >= nf);
    R Vc[NV], vL[NV], vR[NV], vLn[NV];
#pragma unroll
    for (int nv = 0; nv < NV; nv++) {
      Vc[nv] = (R)stg[buf][nv][tid];
      const R sp1 = selfp1 ? (R)stg[buf][NV + nv][tid] : R(0);
      const R sp2 = (act && selfp1) ? (R)stg2[buf][w][nv] : R(0);
      const R up1 = __shfl_up_sync(FULL, Vc[nv], 1);
      const R up2 = __shfl_up_sync(FULL, Vc[nv], 2);
      const R dn1 = __shfl_down_sync(FULL, Vc[nv], 1);
      const R vm1 = (lane == 0) ? pV1[nv] : up1;
      const R vm2 = (lane == 0) ? pV2[nv] : ((lane == 1) ? pV1[nv] : up2);
      const R vp1 = selfp1 ? sp1 : dn1;
      const R cf = ppm_face(vm2, vm1, Vc[nv], vp1);            // face f
      const R nxt = __shfl_down_sync(FULL, cf, 1);
      const R cfn = selfp1 ? ppm_face(vm1, Vc[nv], vp1, sp2) : nxt;  // face f+1
      R dvp, dvm;
      ppm_cell(Vc[nv], cf, cfn, dvp, dvm);
      vR[nv] = Vc[nv] + dvm;
      vLn[nv] = Vc[nv] + dvp;
    }
    if constexpr (PHYS == PHYS_RMHD) rmhd_vel_limit<NV>(Vc, vR, vLn);
#pragma unroll
    for (int nv = 0; nv < NV; nv++) {
      R l = __shfl_up_sync(FULL, vLn[nv], 1);
      vL[nv] = (lane == 0) ? pVLn[nv] : l;
    }
    R Bn = R(0);
    if constexpr (PHYS != PHYS_HD) {
      Bn = (R)stg[buf][2 * NV][tid];
      vL[BX1] = Bn;
      vR[BX1] = Bn;
    }
    CTFace<R> ct;
    uint32_t fe = 0;
    cm = riemann<PHYS, RS, CT, 0>(vL, vR, F, gamma, Bn, ct, fe);
#pragma unroll
    for (int nv = 0; nv < NV; nv++)
      if (act && rhs_var<PHYS, NDIM>(nv) && isnan(F[nv])) fe |= ERR_NAN | ERR_QUIT;
    if (fe && face_counts(g, 0, f, 1, row % g.ny, 2, row / g.ny)) err |= fe;
    if constexpr (PHYS != PHYS_HD) {
      if (act) store_ct<CT>(a, 0, rb + f, ct);
    }
    R Fm1[NV];
#pragma unroll
    for (int nv = 0; nv < NV; nv++) {
      R t = __shfl_up_sync(FULL, F[nv], 1);
      Fm1[nv] = (lane == 0) ? pF[nv] : t;
    }
    R cmm1;
    {
      R t = __shfl_up_sync(FULL, cm, 1);
      cmm1 = (lane == 0) ? pCm : t;
    }
    if (act && f >= 1)
      cell_update<PHYS, NV, NDIM>(a, n, rb + (f - 1), Fm1, F, cmm1, cm, 0);
    if (c0 == 0) {
#pragma unroll
      for (int nv = 0; nv < NV; nv++) fF[nv] = F[nv];
      fCm = cm;
    }
#pragma unroll
    for (int nv = 0; nv < NV; nv++) {
      pV2[nv] = __shfl_sync(FULL, Vc[nv], 30);
      pV1[nv] = __shfl_sync(FULL, Vc[nv], 31);
      pVLn[nv] = __shfl_sync(FULL, vLn[nv], 31);
      pF[nv] = __shfl_sync(FULL, F[nv], 31);
    }
    pCm = __shfl_sync(FULL, cm, 31);
  }
  cp_async_wait0();
  if (nf == nx) {  // periodic: the last cell's right face is face 0
    R F0[NV];
#pragma unroll
    for (int nv = 0; nv < NV; nv++) F0[nv] = __shfl_sync(FULL, fF[nv], 0);
    R cm0 = __shfl_sync(FULL, fCm, 0);
    if (lane == ((nx - 1) & 31))
      cell_update<PHYS, NV, NDIM>(a, n, rb + (nx - 1), F, F0, cm, cm0, 0);
  }
  if (err) atomicOr(a.err, err);
}

// MP5 adjustments of one cell's edges (Src/States/mp5_states.cpp:184-213):
// density and pressure edges that came out negative fall back to minmod PLM
// (qm, qp: the neighbours' density and pressure), then, for RMHD, the
// relativistic velocity limiter.
template <int PHYS, int NV, typename R>
__device__ __forceinline__ void mp5_fallback(const R* w0, const R* qm, const R* qp, R* vR,
                                             R* vLn) {
#pragma unroll
  for (int q = 0; q < 2; q++) {
    const int nv = q ? NV - 1 : RHO;
    if (vLn[nv] < R(0) || vR[nv] < R(0)) {
      const R dv = minmod(qp[q] - w0[nv], w0[nv] - qm[q]);
      vLn[nv] = w0[nv] + R(0.5) * dv;
      vR[nv] = w0[nv] - R(0.5) * dv;
    }
  }
  if constexpr (PHYS == PHYS_RMHD) rmhd_vel_limit<NV>(w0, vR, vLn);
}

template <int PHYS, int NV, int NDIM, int RS, int CT, int LIM, typename R, typename CTT>
__device__ __forceinline__ void sweep_x_row_mp5(const StageArgs<CTT>& a, const Grid3& g, int row,
                                                double* stg_, int tid) {
  constexpr unsigned FULL = 0xffffffffu;
  constexpr int SL = 2 * NV + 1;  // staged doubles per lane: V[f], V[f+1], Bs[f]
  constexpr int NW = SWEEP_THREADS / 32;
  double(*stg)[SL][SWEEP_THREADS] = reinterpret_cast<double(*)[SL][SWEEP_THREADS]>(stg_);
  double(*stg2)[NW][NV] = reinterpret_cast<double(*)[NW][NV]>(stg_ + 2 * SL * SWEEP_THREADS);
  const int lane = tid & 31, w = tid >> 5;
  if (row >= g.ny * g.nz) return;  // warp-uniform
  const int nx = g.nx;
  const unsigned ob = g.outflow;
  // faces solved: nx (periodic: face nx is face 0) or nx+1 (outflow high side)
  const int nf = nx + (int)((ob >> 1) & 1u);
  const long long n = g.n;
  const long long rb = (long long)row * nx;
  const R gamma = (R)a.gamma;

  // carried: cells c0-1, c0-2; left state at face c0 (from cell c0-1); flux
  // and signal speed of face c0-1
  R pV1[NV], pV2[NV], pVLn[NV], pF[NV], pCm = R(0);
  {
    R q[5][NV];
#pragma unroll
    for (int m = 0; m < 5; m++) load_cell<NV>(a.V, n, rb + gidx(m - 3, nx, ob, 0), q[m]);
    R vrp[NV];
#pragma unroll
    for (int nv = 0; nv < NV; nv++) {   // cell nx-1 (stencil nx-3 .. nx+1)
      pVLn[nv] = edge5<LIM>(q[0][nv], q[1][nv], q[2][nv], q[3][nv], q[4][nv]);
      vrp[nv] = edge5<LIM>(q[4][nv], q[3][nv], q[2][nv], q[1][nv], q[0][nv]);
      pV1[nv] = q[2][nv];
      pV2[nv] = q[1][nv];
      pF[nv] = R(0);
    }
    {
      const R qm[2] = {q[1][RHO], q[1][NV - 1]}, qp[2] = {q[3][RHO], q[3][NV - 1]};
      mp5_fallback<PHYS, NV>(q[2], qm, qp, vrp, pVLn);
    }
  }
  R fF[NV], fCm = R(0);
  R F[NV], cm = R(0);
#pragma unroll
  for (int nv = 0; nv < NV; nv++) { fF[nv] = R(0); F[nv] = R(0); }
  uint32_t err = 0;

  auto stage_chunk = [&](int c0, int b) {
    const int f = c0 + lane;
    const int fc = f < nx ? f : nx - 1;
#pragma unroll
    for (int nv = 0; nv < NV; nv++) cp_async8(&stg[b][nv][tid], a.V + nv * n + rb + fc);
    if (lane == 31 || f + 1 >= nf) {
      const int fp = gidx(fc + 1, nx, ob, 0);
#pragma unroll
      for (int nv = 0; nv < NV; nv++) cp_async8(&stg[b][NV + nv][tid], a.V + nv * n + rb + fp);
    }
    if (f < nf && (lane == 31 || f + 1 >= nf)) {  // one lane per chunk
      const int fp2 = gidx(fc + 2, nx, ob, 0);
#pragma unroll
      for (int nv = 0; nv < NV; nv++) cp_async8(&stg2[b][w][nv], a.V + nv * n + rb + fp2);
    }
    if constexpr (PHYS != PHYS_HD) cp_async8(&stg[b][2 * NV][tid], a.Bs[0] + rb + fc);
    cp_async_commit();
  };
  stage_chunk(0, 0);
  int buf = 0;
  for (int c0 = 0; c0 < nf; c0 += 32, buf ^= 1) {
    const int f = c0 + lane;
    const bool act = f < nf;
    stage_chunk(c0 + 32 < nf ? c0 + 32 : c0, buf ^ 1);   // prefetch the next chunk
    cp_async_wait1();
    const bool selfp1 = (lane == 31) || (f + 1 >= nf);
    R Vc[NV], vL[NV], vR[NV], vLn[NV], qm[2], qp[2];
    // the lane before the chunk's last active lane takes V(f+2) from that
    // lane's staged V(f+1)
    const bool nextself = __shfl_down_sync(FULL, (int)selfp1, 1) != 0;
#pragma unroll
    for (int nv = 0; nv < NV; nv++) {
      Vc[nv] = (R)stg[buf][nv][tid];
      const R sp1 = selfp1 ? (R)stg[buf][NV + nv][tid] : R(0);
      const R sp2 = (act && selfp1) ? (R)stg2[buf][w][nv] : R(0);
      const R up1 = __shfl_up_sync(FULL, Vc[nv], 1);
      const R up2 = __shfl_up_sync(FULL, Vc[nv], 2);
      const R dn1 = __shfl_down_sync(FULL, Vc[nv], 1);
      const R dn2 = __shfl_down_sync(FULL, Vc[nv], 2);
      const R sp1n = __shfl_down_sync(FULL, sp1, 1);
      const R vm1 = (lane == 0) ? pV1[nv] : up1;
      const R vm2 = (lane == 0) ? pV2[nv] : ((lane == 1) ? pV1[nv] : up2);
      const R vp1 = selfp1 ? sp1 : dn1;
      const R vp2 = selfp1 ? sp2 : (nextself ? sp1n : dn2);
      vLn[nv] = edge5<LIM>(vm2, vm1, Vc[nv], vp1, vp2);   // right edge: face f+1
      vR[nv] = edge5<LIM>(vp2, vp1, Vc[nv], vm1, vm2);    // left edge: face f
      if (nv == RHO) { qm[0] = vm1; qp[0] = vp1; }
      if (nv == NV - 1) { qm[1] = vm1; qp[1] = vp1; }
    }
    mp5_fallback<PHYS, NV>(Vc, qm, qp, vR, vLn);
#pragma unroll
    for (int nv = 0; nv < NV; nv++) {
      R l = __shfl_up_sync(FULL, vLn[nv], 1);
      vL[nv] = (lane == 0) ? pVLn[nv] : l;
    }
    R Bn = R(0);
    if constexpr (PHYS != PHYS_HD) {
      Bn = (R)stg[buf][2 * NV][tid];
      vL[BX1] = Bn;
      vR[BX1] = Bn;
    }
    CTFace<R> ct;
    uint32_t fe = 0;
    cm = riemann<PHYS, RS, CT, 0>(vL, vR, F, gamma, Bn, ct, fe);
#pragma unroll
    for (int nv = 0; nv < NV; nv++)
      if (act && rhs_var<PHYS, NDIM>(nv) && isnan(F[nv])) fe |= ERR_NAN | ERR_QUIT;
    if (fe && face_counts(g, 0, f, 1, row % g.ny, 2, row / g.ny)) err |= fe;
    if constexpr (PHYS != PHYS_HD) {
      if (act) store_ct<CT>(a, 0, rb + f, ct);
    }
    R Fm1[NV];
#pragma unroll
    for (int nv = 0; nv < NV; nv++) {
      R t = __shfl_up_sync(FULL, F[nv], 1);
      Fm1[nv] = (lane == 0) ? pF[nv] : t;
    }
    R cmm1;
    {
      R t = __shfl_up_sync(FULL, cm, 1);
      cmm1 = (lane == 0) ? pCm : t;
    }
    if (act && f >= 1)
      cell_update<PHYS, NV, NDIM>(a, n, rb + (f - 1), Fm1, F, cmm1, cm, 0);
    if (c0 == 0) {
#pragma unroll
      for (int nv = 0; nv < NV; nv++) fF[nv] = F[nv];
      fCm = cm;
    }
#pragma unroll
    for (int nv = 0; nv < NV; nv++) {
      pV2[nv] = __shfl_sync(FULL, Vc[nv], 30);
      pV1[nv] = __shfl_sync(FULL, Vc[nv], 31);
      pVLn[nv] = __shfl_sync(FULL, vLn[nv], 31);
      pF[nv] = __shfl_sync(FULL, F[nv], 31);
    }
    pCm = __shfl_sync(FULL, cm, 31);
  }
  cp_async_wait0();
  if (nf == nx) {  // periodic: the last cell's right face is face 0
    R F0[NV];
#pragma unroll
    for (int nv = 0; nv < NV; nv++) F0[nv] = __shfl_sync(FULL, fF[nv], 0);
    R cm0 = __shfl_sync(FULL, fCm, 0);
    if (lane == ((nx - 1) & 31))
      cell_update<PHYS, NV, NDIM>(a, n, rb + (nx - 1), F, F0, cm, cm0, 0);
  }
  if (err) atomicOr(a.err, err);
}

// One x-row per warp.  `stg_` is the block's staging area
// (sweep_x_stage_doubles<NV>() doubles of shared memory), `tid` the thread's
// index in its 128-thread block.
template <int PHYS, int NV, int NDIM, int RS, int CT, int LIM, typename R, typename CTT>
__device__ __forceinline__ void sweep_x_row(const StageArgs<CTT>& a, const Grid3& g, int row,
                                            double* stg_, int tid) {
  if constexpr (LIM == LIM_PPM) {
    sweep_x_row_ppm<PHYS, NV, NDIM, RS, CT, R, CTT>(a, g, row, stg_, tid);
    return;
  }
  if constexpr (five_point<LIM>()) {
    sweep_x_row_mp5<PHYS, NV, NDIM, RS, CT, LIM, R, CTT>(a, g, row, stg_, tid);
    return;
  }
  constexpr unsigned FULL = 0xffffffffu;
  constexpr int SL = 2 * NV + 1;  // staged doubles per lane: V[f], V[f+1], Bs[f]
  double(*stg)[SL][SWEEP_THREADS] = reinterpret_cast<double(*)[SL][SWEEP_THREADS]>(stg_);
  const int lane = tid & 31;
  if (row >= g.ny * g.nz) return;  // warp-uniform
  const int nx = g.nx;
  const unsigned ob = g.outflow;
  // faces solved: nx (periodic: face nx is face 0) or nx+1 (outflow high side)
  const int nf = nx + (int)((ob >> 1) & 1u);
  const long long n = g.n;
  const long long rb = (long long)row * nx;
  const R gamma = (R)a.gamma;

  // carried state of cell c0-1 (uniform over lanes)
  R pV[NV], pVLn[NV], pF[NV], pCm = R(0);
  {
    R vm[NV], v0[NV], vp[NV];
    load_cell<NV>(a.V, n, rb + gidx(-2, nx, ob, 0), vm);
    load_cell<NV>(a.V, n, rb + gidx(-1, nx, ob, 0), v0);
    load_cell<NV>(a.V, n, rb + 0, vp);
    R pVR[NV];
    if constexpr (three_point<LIM>()) {
      const R dx = (R)a.dx[0];
#pragma unroll
      for (int nv = 0; nv < NV; nv++) {
        pV[nv] = v0[nv];
        pVLn[nv] = edge3<LIM>(vm[nv], v0[nv], vp[nv], dx);
        pVR[nv] = edge3<LIM>(vp[nv], v0[nv], vm[nv], dx);
        pF[nv] = R(0);
      }
      const R qm[2] = {vm[RHO], vm[NV - 1]}, qp[2] = {vp[RHO], vp[NV - 1]};
      mp5_fallback<PHYS, NV>(v0, qm, qp, pVR, pVLn);
    } else {
#pragma unroll
      for (int nv = 0; nv < NV; nv++) {
        R dv = limit<LIM>(vp[nv] - v0[nv], v0[nv] - vm[nv]);
        pV[nv] = v0[nv];
        pVLn[nv] = v0[nv] + R(0.5) * dv;
        pVR[nv] = v0[nv] - R(0.5) * dv;
        pF[nv] = R(0);
      }
      if constexpr (PHYS == PHYS_RMHD) rmhd_vel_limit<NV>(v0, pVR, pVLn);
    }
  }
  R fF[NV], fCm = R(0);  // flux of face 0 (lane 0 of the first chunk)
  R F[NV], cm = R(0);
#pragma unroll
  for (int nv = 0; nv < NV; nv++) { fF[nv] = R(0); F[nv] = R(0); }
  uint32_t err = 0;

  // stage chunk c0 into buffer b: V[f], V[f+1] (lanes that cannot take it
  // from the next lane), Bs[f]
  auto stage_chunk = [&](int c0, int b) {
    const int f = c0 + lane;
    const int fc = f < nx ? f : nx - 1;
#pragma unroll
    for (int nv = 0; nv < NV; nv++) cp_async8(&stg[b][nv][tid], a.V + nv * n + rb + fc);
    if (lane == 31 || f + 1 >= nf) {
      const int fp = gidx(fc + 1, nx, ob, 0);
#pragma unroll
      for (int nv = 0; nv < NV; nv++) cp_async8(&stg[b][NV + nv][tid], a.V + nv * n + rb + fp);
    }
    if constexpr (PHYS != PHYS_HD) cp_async8(&stg[b][2 * NV][tid], a.Bs[0] + rb + fc);
    cp_async_commit();
  };
  stage_chunk(0, 0);
  int buf = 0;
  for (int c0 = 0; c0 < nf; c0 += 32, buf ^= 1) {
    const int f = c0 + lane;
    const bool act = f < nf;
    stage_chunk(c0 + 32 < nf ? c0 + 32 : c0, buf ^ 1);   // prefetch the next chunk
    cp_async_wait1();
    R Vc[NV], Vm1[NV], Vp1[NV], vL[NV], vR[NV], vLn[NV];
    const bool selfp1 = (lane == 31) || (f + 1 >= nf);
#pragma unroll
    for (int nv = 0; nv < NV; nv++) {
      Vc[nv] = (R)stg[buf][nv][tid];
      if (selfp1) Vp1[nv] = (R)stg[buf][NV + nv][tid];
    }
    if constexpr (three_point<LIM>()) {
      const R dx = (R)a.dx[0];
#pragma unroll
      for (int nv = 0; nv < NV; nv++) {
        R up = __shfl_up_sync(FULL, Vc[nv], 1);
        R dn = __shfl_down_sync(FULL, Vc[nv], 1);
        Vm1[nv] = (lane == 0) ? pV[nv] : up;
        if (!selfp1) Vp1[nv] = dn;
        vR[nv] = edge3<LIM>(Vp1[nv], Vc[nv], Vm1[nv], dx);
        vLn[nv] = edge3<LIM>(Vm1[nv], Vc[nv], Vp1[nv], dx);
      }
      const R qm[2] = {Vm1[RHO], Vm1[NV - 1]}, qp[2] = {Vp1[RHO], Vp1[NV - 1]};
      mp5_fallback<PHYS, NV>(Vc, qm, qp, vR, vLn);
    } else {
#pragma unroll
      for (int nv = 0; nv < NV; nv++) {
        R up = __shfl_up_sync(FULL, Vc[nv], 1);
        R dn = __shfl_down_sync(FULL, Vc[nv], 1);
        Vm1[nv] = (lane == 0) ? pV[nv] : up;
        if (!selfp1) Vp1[nv] = dn;
        R dv = limit<LIM>(Vp1[nv] - Vc[nv], Vc[nv] - Vm1[nv]);
        vR[nv] = Vc[nv] - R(0.5) * dv;
        vLn[nv] = Vc[nv] + R(0.5) * dv;
      }
      if constexpr (PHYS == PHYS_RMHD) rmhd_vel_limit<NV>(Vc, vR, vLn);
    }
#pragma unroll
    for (int nv = 0; nv < NV; nv++) {
      R l = __shfl_up_sync(FULL, vLn[nv], 1);
      vL[nv] = (lane == 0) ? pVLn[nv] : l;
    }
    R Bn = R(0);
    if constexpr (PHYS != PHYS_HD) {
      Bn = (R)stg[buf][2 * NV][tid];  // Src/States/plm_states.cpp:184-189
      vL[BX1] = Bn;
      vR[BX1] = Bn;
    }
    CTFace<R> ct;
    uint32_t fe = 0;
    cm = riemann<PHYS, RS, CT, 0>(vL, vR, F, gamma, Bn, ct, fe);
#pragma unroll
    for (int nv = 0; nv < NV; nv++)
      if (act && rhs_var<PHYS, NDIM>(nv) && isnan(F[nv])) fe |= ERR_NAN | ERR_QUIT;
    if (fe && face_counts(g, 0, f, 1, row % g.ny, 2, row / g.ny)) err |= fe;
    if constexpr (PHYS != PHYS_HD) {
      if (act) store_ct<CT>(a, 0, rb + f, ct);
    }
    // flux of face f-1 and cell update of cell f-1
    R Fm1[NV];
#pragma unroll
    for (int nv = 0; nv < NV; nv++) {
      R t = __shfl_up_sync(FULL, F[nv], 1);
      Fm1[nv] = (lane == 0) ? pF[nv] : t;
    }
    R cmm1;
    {
      R t = __shfl_up_sync(FULL, cm, 1);
      cmm1 = (lane == 0) ? pCm : t;
    }
    if (act && f >= 1)
      cell_update<PHYS, NV, NDIM>(a, n, rb + (f - 1), Fm1, F, cmm1, cm, 0);
    if (c0 == 0) {
#pragma unroll
      for (int nv = 0; nv < NV; nv++) fF[nv] = F[nv];
      fCm = cm;
    }
#pragma unroll
    for (int nv = 0; nv < NV; nv++) {
      pV[nv] = __shfl_sync(FULL, Vc[nv], 31);
      pVLn[nv] = __shfl_sync(FULL, vLn[nv], 31);
      pF[nv] = __shfl_sync(FULL, F[nv], 31);
    }
    pCm = __shfl_sync(FULL, cm, 31);
  }
  cp_async_wait0();
  // periodic: cell nx-1 uses F[nx-1] (lane (nx-1)%32 of the last chunk) and
  // F[nx] = F[0]; with an outflow high side face nx was solved in the loop
  if (nf == nx) {
    R F0[NV];
#pragma unroll
    for (int nv = 0; nv < NV; nv++) F0[nv] = __shfl_sync(FULL, fF[nv], 0);
    R cm0 = __shfl_sync(FULL, fCm, 0);
    if (lane == ((nx - 1) & 31))
      cell_update<PHYS, NV, NDIM>(a, n, rb + (nx - 1), F, F0, cm, cm0, 0);
  }
  if (err) atomicOr(a.err, err);
}

template <int PHYS, int NV, int NDIM, int RS, int CT, int LIM, typename R, typename CTT>
__global__ void __launch_bounds__(SWEEP_THREADS, (sweep_x_minb<PHYS, R>()))
    sweep_x_kernel(StageArgs<CTT> a, Grid3 g) {
  __shared__ double stg[sweep_x_stage_doubles<NV, LIM>()];
  const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  sweep_x_row<PHYS, NV, NDIM, RS, CT, LIM, R, CTT>(a, g, row, stg, threadIdx.x);
}

// ---------------------------------------------------------------------
// y / z sweep: thread per (x, pencil segment), marching along DIR with a
// register window of three cells; the cell two steps ahead and the next face
// field are staged into shared memory with cp.async while the current face
// is solved.  Writes the direction's flux differences, inverse-dt terms and
// UCT face data (no loads besides the stencil).
// ---------------------------------------------------------------------
// Piecewise parabolic y/z march: cells m-1, m, m+1 in registers, cell m+2
// staged with cp.async (one iteration ahead: cell m+3 and face m+1 are
// prefetched while face m is solved).  The constrained value of face m+1 is
// formed from cells m-1..m+2 and carried to the next iteration as face m's.
template <int PHYS, int NV, int NDIM, int RS, int CT, int DIR, typename R, typename CTT>
__device__ __forceinline__ void sweep_m_col_ppm(const StageArgs<CTT>& a, const Grid3& g, int i,
                                                int t, int seg, int S, double* stg_, int tid) {
  double(*stg)[NV + 1][SWEEP_THREADS] = reinterpret_cast<double(*)[NV + 1][SWEEP_THREADS]>(stg_);
  const int nd = (DIR == 1) ? g.ny : g.nz;
  const long long n = g.n;
  const R gamma = (R)a.gamma;
  uint32_t err = 0;
  if (i < g.nx) {
    const long long stride = (DIR == 1) ? (long long)g.nx : (long long)g.nx * g.ny;
    const long long base = (DIR == 1) ? i + (long long)g.nx * g.ny * t
                                      : i + (long long)g.nx * t;
    const int m0 = seg * S;
    const int m1 = min(m0 + S, nd);
    auto stage = [&](int mcell, int mface, int b) {
      const long long cc = base + (long long)gidx(mcell, nd, g.outflow, DIR) * stride;
#pragma unroll
      for (int nv = 0; nv < NV; nv++) cp_async8(&stg[b][nv][tid], a.V + nv * n + cc);
      if constexpr (PHYS != PHYS_HD)
        cp_async8(&stg[b][NV][tid], a.Bs[DIR] + base + (long long)gidx(mface, nd, g.outflow, DIR) * stride);
      cp_async_commit();
    };
    stage(m0 + 2, m0, 0);
    R W0[NV], W1[NV], W2[NV], Fm[NV], vLn[NV], Fp[NV], cmp = R(0);
    {
      R q3[NV], q2[NV];
      load_cell<NV>(a.V, n, base + gidx(m0 - 3, nd, g.outflow, DIR) * stride, q3);
      load_cell<NV>(a.V, n, base + gidx(m0 - 2, nd, g.outflow, DIR) * stride, q2);
      load_cell<NV>(a.V, n, base + gidx(m0 - 1, nd, g.outflow, DIR) * stride, W0);
      load_cell<NV>(a.V, n, base + (long long)m0 * stride, W1);
      load_cell<NV>(a.V, n, base + gidx(m0 + 1, nd, g.outflow, DIR) * stride, W2);
      R vrp[NV];
#pragma unroll
      for (int nv = 0; nv < NV; nv++) {
        const R fa = ppm_face(q3[nv], q2[nv], W0[nv], W1[nv]);   // face m0-1
        Fm[nv] = ppm_face(q2[nv], W0[nv], W1[nv], W2[nv]);       // face m0
        R dvp, dvm;
        ppm_cell(W0[nv], fa, Fm[nv], dvp, dvm);                   // cell m0-1
        vLn[nv] = W0[nv] + dvp;
        vrp[nv] = W0[nv] + dvm;
        Fp[nv] = R(0);
      }
      if constexpr (PHYS == PHYS_RMHD) rmhd_vel_limit<NV>(W0, vrp, vLn);
    }
    int buf = 0;
    for (int m = m0; m <= m1; m++, buf ^= 1) {
      stage(m + 3, m + 1, buf ^ 1);   // prefetch for the next iteration
      cp_async_wait1();
      R vL[NV], vR[NV], F[NV], W3[NV];
#pragma unroll
      for (int nv = 0; nv < NV; nv++) {
        W3[nv] = (R)stg[buf][nv][tid];                             // cell m+2
        const R fn = ppm_face(W0[nv], W1[nv], W2[nv], W3[nv]);     // face m+1
        R dvp, dvm;
        ppm_cell(W1[nv], Fm[nv], fn, dvp, dvm);                   // cell m
        vL[nv] = vLn[nv];
        vR[nv] = W1[nv] + dvm;
        vLn[nv] = W1[nv] + dvp;
        Fm[nv] = fn;
      }
      if constexpr (PHYS == PHYS_RMHD) rmhd_vel_limit<NV>(W1, vR, vLn);
      R Bn = R(0);
      if constexpr (PHYS != PHYS_HD) {
        Bn = (R)stg[buf][NV][tid];
        vL[BX1 + DIR] = Bn;
        vR[BX1 + DIR] = Bn;
      }
      CTFace<R> ct;
      uint32_t fe = 0;
      R cm = riemann<PHYS, RS, CT, DIR>(vL, vR, F, gamma, Bn, ct, fe);
#pragma unroll
      for (int nv = 0; nv < NV; nv++)
        if (rhs_var<PHYS, NDIM>(nv) && isnan(F[nv])) fe |= ERR_NAN | ERR_QUIT;
      if (fe && face_counts(g, DIR, m, 0, i, DIR == 1 ? 2 : 1, t)) err |= fe;
      if constexpr (PHYS != PHYS_HD) {
        if (m < m1) store_ct<CT>(a, DIR, base + (long long)gidx(m, nd, g.outflow, DIR) * stride, ct);
      }
      if (m > m0)
        cell_update<PHYS, NV, NDIM>(a, n, base + (long long)(m - 1) * stride, Fp, F, cmp, cm,
                                    DIR);
#pragma unroll
      for (int nv = 0; nv < NV; nv++) {
        W0[nv] = W1[nv];
        W1[nv] = W2[nv];
        W2[nv] = W3[nv];
        Fp[nv] = F[nv];
      }
      cmp = cm;
    }
    cp_async_wait0();
  }
  if (err) atomicOr(a.err, err);
}

template <int PHYS, int NV, int NDIM, int RS, int CT, int LIM, int DIR, typename R,
          typename CTT>
__device__ __forceinline__ void sweep_m_col_mp5(const StageArgs<CTT>& a, const Grid3& g, int i,
                                                int t, int seg, int S, double* stg_, int tid) {
  double(*stg)[NV + 1][SWEEP_THREADS] = reinterpret_cast<double(*)[NV + 1][SWEEP_THREADS]>(stg_);
  const int nd = (DIR == 1) ? g.ny : g.nz;
  const long long n = g.n;
  const R gamma = (R)a.gamma;
  uint32_t err = 0;
  if (i < g.nx) {
    const long long stride = (DIR == 1) ? (long long)g.nx : (long long)g.nx * g.ny;
    const long long base = (DIR == 1) ? i + (long long)g.nx * g.ny * t
                                      : i + (long long)g.nx * t;
    const int m0 = seg * S;
    const int m1 = min(m0 + S, nd);
    auto stage = [&](int mcell, int mface, int b) {
      const long long cc = base + (long long)gidx(mcell, nd, g.outflow, DIR) * stride;
#pragma unroll
      for (int nv = 0; nv < NV; nv++) cp_async8(&stg[b][nv][tid], a.V + nv * n + cc);
      if constexpr (PHYS != PHYS_HD)
        cp_async8(&stg[b][NV][tid], a.Bs[DIR] + base + (long long)gidx(mface, nd, g.outflow, DIR) * stride);
      cp_async_commit();
    };
    stage(m0 + 2, m0, 0);
    // window: Wm = cell m-2, W0 = m-1, W1 = m, W2 = m+1, W3 = m+2
    R Wm[NV], W0[NV], W1[NV], W2[NV], vLn[NV], Fp[NV], cmp = R(0);
    {
      R q3[NV];
      load_cell<NV>(a.V, n, base + gidx(m0 - 3, nd, g.outflow, DIR) * stride, q3);
      load_cell<NV>(a.V, n, base + gidx(m0 - 2, nd, g.outflow, DIR) * stride, Wm);
      load_cell<NV>(a.V, n, base + gidx(m0 - 1, nd, g.outflow, DIR) * stride, W0);
      load_cell<NV>(a.V, n, base + (long long)m0 * stride, W1);
      load_cell<NV>(a.V, n, base + gidx(m0 + 1, nd, g.outflow, DIR) * stride, W2);
      R vrp[NV];
#pragma unroll
      for (int nv = 0; nv < NV; nv++) {   // cell m0-1 (stencil m0-3 .. m0+1)
        vLn[nv] = edge5<LIM>(q3[nv], Wm[nv], W0[nv], W1[nv], W2[nv]);
        vrp[nv] = edge5<LIM>(W2[nv], W1[nv], W0[nv], Wm[nv], q3[nv]);
        Fp[nv] = R(0);
      }
      const R qm[2] = {Wm[RHO], Wm[NV - 1]}, qp[2] = {W1[RHO], W1[NV - 1]};
      mp5_fallback<PHYS, NV>(W0, qm, qp, vrp, vLn);
    }
    int buf = 0;
    for (int m = m0; m <= m1; m++, buf ^= 1) {
      stage(m + 3, m + 1, buf ^ 1);   // prefetch for the next iteration
      cp_async_wait1();
      R vL[NV], vR[NV], F[NV], W3[NV];
#pragma unroll
      for (int nv = 0; nv < NV; nv++) {
        W3[nv] = (R)stg[buf][nv][tid];                             // cell m+2
        vL[nv] = vLn[nv];
        vLn[nv] = edge5<LIM>(Wm[nv], W0[nv], W1[nv], W2[nv], W3[nv]);  // cell m, right
        vR[nv] = edge5<LIM>(W3[nv], W2[nv], W1[nv], W0[nv], Wm[nv]);   // cell m, left
      }
      {
        const R qm[2] = {W0[RHO], W0[NV - 1]}, qp[2] = {W2[RHO], W2[NV - 1]};
        mp5_fallback<PHYS, NV>(W1, qm, qp, vR, vLn);
      }
      R Bn = R(0);
      if constexpr (PHYS != PHYS_HD) {
        Bn = (R)stg[buf][NV][tid];
        vL[BX1 + DIR] = Bn;
        vR[BX1 + DIR] = Bn;
      }
      CTFace<R> ct;
      uint32_t fe = 0;
      R cm = riemann<PHYS, RS, CT, DIR>(vL, vR, F, gamma, Bn, ct, fe);
#pragma unroll
      for (int nv = 0; nv < NV; nv++)
        if (rhs_var<PHYS, NDIM>(nv) && isnan(F[nv])) fe |= ERR_NAN | ERR_QUIT;
      if (fe && face_counts(g, DIR, m, 0, i, DIR == 1 ? 2 : 1, t)) err |= fe;
      if constexpr (PHYS != PHYS_HD) {
        if (m < m1) store_ct<CT>(a, DIR, base + (long long)gidx(m, nd, g.outflow, DIR) * stride, ct);
      }
      if (m > m0)
        cell_update<PHYS, NV, NDIM>(a, n, base + (long long)(m - 1) * stride, Fp, F, cmp, cm,
                                    DIR);
#pragma unroll
      for (int nv = 0; nv < NV; nv++) {
        Wm[nv] = W0[nv];
        W0[nv] = W1[nv];
        W1[nv] = W2[nv];
        W2[nv] = W3[nv];
        Fp[nv] = F[nv];
      }
      cmp = cm;
    }
    cp_async_wait0();
  }
  if (err) atomicOr(a.err, err);
}

// One (x column i, transverse index t, pencil segment seg) per thread: t is
// k for DIR=1 and j for DIR=2; the segment covers cells [seg*S, seg*S+S).
// `stg_` is the block's staging area (sweep_m_stage_doubles<NV>() doubles).
template <int PHYS, int NV, int NDIM, int RS, int CT, int LIM, int DIR, typename R,
          typename CTT>
__device__ __forceinline__ void sweep_m_col(const StageArgs<CTT>& a, const Grid3& g, int i, int t,
                                            int seg, int S, double* stg_, int tid) {
  if constexpr (LIM == LIM_PPM) {
    sweep_m_col_ppm<PHYS, NV, NDIM, RS, CT, DIR, R, CTT>(a, g, i, t, seg, S, stg_, tid);
    return;
  }
  if constexpr (five_point<LIM>()) {
    sweep_m_col_mp5<PHYS, NV, NDIM, RS, CT, LIM, DIR, R, CTT>(a, g, i, t, seg, S, stg_, tid);
    return;
  }
  double(*stg)[NV + 1][SWEEP_THREADS] = reinterpret_cast<double(*)[NV + 1][SWEEP_THREADS]>(stg_);
  const int nd = (DIR == 1) ? g.ny : g.nz;
  const long long n = g.n;
  const R gamma = (R)a.gamma;
  uint32_t err = 0;
  if (i < g.nx) {
    const long long stride = (DIR == 1) ? (long long)g.nx : (long long)g.nx * g.ny;
    const long long base = (DIR == 1) ? i + (long long)g.nx * g.ny * t
                                      : i + (long long)g.nx * t;
    const int m0 = seg * S;
    const int m1 = min(m0 + S, nd);
    auto stage = [&](int mcell, int mface, int b) {
      const long long cc = base + (long long)gidx(mcell, nd, g.outflow, DIR) * stride;
#pragma unroll
      for (int nv = 0; nv < NV; nv++) cp_async8(&stg[b][nv][tid], a.V + nv * n + cc);
      if constexpr (PHYS != PHYS_HD)
        cp_async8(&stg[b][NV][tid], a.Bs[DIR] + base + (long long)gidx(mface, nd, g.outflow, DIR) * stride);
      cp_async_commit();
    };
    stage(m0 + 1, m0, 0);
    R Vp[NV], Vc[NV], vLn[NV], Fp[NV], cmp = R(0);
    {
      R vmm[NV];
      load_cell<NV>(a.V, n, base + gidx(m0 - 2, nd, g.outflow, DIR) * stride, vmm);
      load_cell<NV>(a.V, n, base + gidx(m0 - 1, nd, g.outflow, DIR) * stride, Vp);
      load_cell<NV>(a.V, n, base + (long long)m0 * stride, Vc);
      R vrp[NV];
      if constexpr (three_point<LIM>()) {
        const R dx = (R)a.dx[DIR];
#pragma unroll
        for (int nv = 0; nv < NV; nv++) {
          vLn[nv] = edge3<LIM>(vmm[nv], Vp[nv], Vc[nv], dx);
          vrp[nv] = edge3<LIM>(Vc[nv], Vp[nv], vmm[nv], dx);
          Fp[nv] = R(0);
        }
        const R qm[2] = {vmm[RHO], vmm[NV - 1]}, qp[2] = {Vc[RHO], Vc[NV - 1]};
        mp5_fallback<PHYS, NV>(Vp, qm, qp, vrp, vLn);
      } else {
#pragma unroll
        for (int nv = 0; nv < NV; nv++) {
          R dv = limit<LIM>(Vc[nv] - Vp[nv], Vp[nv] - vmm[nv]);
          vLn[nv] = Vp[nv] + R(0.5) * dv;
          vrp[nv] = Vp[nv] - R(0.5) * dv;
          Fp[nv] = R(0);
        }
        if constexpr (PHYS == PHYS_RMHD) rmhd_vel_limit<NV>(Vp, vrp, vLn);
      }
    }
    int buf = 0;
    for (int m = m0; m <= m1; m++, buf ^= 1) {
      stage(m + 2, m + 1, buf ^ 1);   // prefetch for the next iteration
      cp_async_wait1();
      R Vn[NV], vL[NV], vR[NV], F[NV];
      if constexpr (three_point<LIM>()) {
        const R dx = (R)a.dx[DIR];
#pragma unroll
        for (int nv = 0; nv < NV; nv++) {
          Vn[nv] = (R)stg[buf][nv][tid];
          vL[nv] = vLn[nv];
          vR[nv] = edge3<LIM>(Vn[nv], Vc[nv], Vp[nv], dx);
          vLn[nv] = edge3<LIM>(Vp[nv], Vc[nv], Vn[nv], dx);
        }
        const R qm[2] = {Vp[RHO], Vp[NV - 1]}, qp[2] = {Vn[RHO], Vn[NV - 1]};
        mp5_fallback<PHYS, NV>(Vc, qm, qp, vR, vLn);
      } else {
#pragma unroll
        for (int nv = 0; nv < NV; nv++) {
          Vn[nv] = (R)stg[buf][nv][tid];
          R dv = limit<LIM>(Vn[nv] - Vc[nv], Vc[nv] - Vp[nv]);
          vL[nv] = vLn[nv];
          vR[nv] = Vc[nv] - R(0.5) * dv;
          vLn[nv] = Vc[nv] + R(0.5) * dv;
        }
        if constexpr (PHYS == PHYS_RMHD) rmhd_vel_limit<NV>(Vc, vR, vLn);
      }
      R Bn = R(0);
      if constexpr (PHYS != PHYS_HD) {
        Bn = (R)stg[buf][NV][tid];
        vL[BX1 + DIR] = Bn;
        vR[BX1 + DIR] = Bn;
      }
      CTFace<R> ct;
      uint32_t fe = 0;
      R cm = riemann<PHYS, RS, CT, DIR>(vL, vR, F, gamma, Bn, ct, fe);
#pragma unroll
      for (int nv = 0; nv < NV; nv++)
        if (rhs_var<PHYS, NDIM>(nv) && isnan(F[nv])) fe |= ERR_NAN | ERR_QUIT;
      if (fe && face_counts(g, DIR, m, 0, i, DIR == 1 ? 2 : 1, t)) err |= fe;
      if constexpr (PHYS != PHYS_HD) {
        if (m < m1) store_ct<CT>(a, DIR, base + (long long)gidx(m, nd, g.outflow, DIR) * stride, ct);
      }
      if (m > m0)
        cell_update<PHYS, NV, NDIM>(a, n, base + (long long)(m - 1) * stride, Fp, F, cmp, cm,
                                    DIR);
#pragma unroll
      for (int nv = 0; nv < NV; nv++) {
        Vp[nv] = Vc[nv];
        Vc[nv] = Vn[nv];
        Fp[nv] = F[nv];
      }
      cmp = cm;
    }
    cp_async_wait0();
  }
  if (err) atomicOr(a.err, err);
}

// t is the transverse index (k for DIR=1, j for DIR=2).  FLAT = false:
// grid (x-blocks, t * nseg + seg), the block's columns share one t.  FLAT =
// true (nx not a multiple of the block): a 1-D grid of (column block cb,
// segment) pairs, segments innermost, with the (x, t) columns numbered
// together (col = cb * SWEEP_THREADS + thread, i = col % nx, t = col / nx),
// so that no block is part-empty.
template <int PHYS, int NV, int NDIM, int RS, int CT, int LIM, int DIR, typename R,
          typename CTT, bool FLAT>
__global__ void __launch_bounds__(SWEEP_THREADS, (sweep_m_minb<PHYS, R>()))
    sweep_m_kernel(StageArgs<CTT> a, Grid3 g, int S) {
  __shared__ double stg[sweep_m_stage_doubles<NV>()];
  const int nd = (DIR == 1) ? g.ny : g.nz;
  const int nseg = (nd + S - 1) / S;
  int i, t, seg;
  if constexpr (FLAT) {
    const int nt = (DIR == 1) ? g.nz : g.ny;
    seg = (int)(blockIdx.x % (unsigned)nseg);
    const int col = (int)(blockIdx.x / (unsigned)nseg) * SWEEP_THREADS + (int)threadIdx.x;
    i = col % g.nx;
    t = col / g.nx;
    if (t >= nt) i = g.nx;   // past the last column: the thread stays idle
  } else {
    i = blockIdx.x * SWEEP_THREADS + threadIdx.x;
    t = blockIdx.y / nseg;
    seg = blockIdx.y - t * nseg;
  }
  sweep_m_col<PHYS, NV, NDIM, RS, CT, LIM, DIR, R, CTT>(a, g, i, t, seg, S, stg, threadIdx.x);
}

// ---------------------------------------------------------------------
// UCT edge EMF (Src/MHD/CT/ct_emf_average.cpp:535-995, reconstruction of
// Src/array_reconstruct.cpp:45-206: face field with MC, stored velocities
// with the scheme limiter).
// b[0..W-1], q[0..W-1]: values at the W cells straddling the edge along the
// reconstruction direction, W = emf_width<LIM>() (edge between b[W/2-1] and
// b[W/2]).
// ---------------------------------------------------------------------
template <int LIM>
__device__ __forceinline__ constexpr int emf_width() { return five_point<LIM>() ? 6 : 4; }

template <int LIM, typename R>
__device__ __forceinline__ void uct_terms(const R* b, const R* q, R aL, R aR, R dL, R dR,
                                          R& avg, R& phi, R dx) {
  R bL, bR, vL, vR;
  if constexpr (three_point<LIM>()) {
    // LimO3 / WENO3 edge values of both the face field and the velocity
    // (Src/array_reconstruct.cpp:272-325), dx the cell width along b
    bL = edge3<LIM>(b[0], b[1], b[2], dx);
    bR = edge3<LIM>(b[3], b[2], b[1], dx);
    vL = edge3<LIM>(q[0], q[1], q[2], dx);
    vR = edge3<LIM>(q[3], q[2], q[1], dx);
  } else if constexpr (five_point<LIM>()) {
    // MP5 (WENO-Z) edge values of both the face field and the velocity
    // (Src/array_reconstruct.cpp:327-384): the right edge of cell b[2] and
    // the left edge of cell b[3]
    bL = edge5<LIM>(b[0], b[1], b[2], b[3], b[4]);
    bR = edge5<LIM>(b[5], b[4], b[3], b[2], b[1]);
    vL = edge5<LIM>(q[0], q[1], q[2], q[3], q[4]);
    vR = edge5<LIM>(q[5], q[4], q[3], q[2], q[1]);
  } else if constexpr (LIM == LIM_PPM) {
    // parabolic reconstruction of both the face field and the velocity
    // (Src/MHD/CT/ct_emf_average.cpp:556-559 with RECONSTRUCTION PARABOLIC)
    R p1, m1, p2, m2;
    par3_cell(b[0], b[1], b[2], p1, m1);
    par3_cell(b[1], b[2], b[3], p2, m2);
    bL = b[1] + p1;
    bR = b[2] + m2;
    par3_cell(q[0], q[1], q[2], p1, m1);
    par3_cell(q[1], q[2], q[3], p2, m2);
    vL = q[1] + p1;
    vR = q[2] + m2;
  } else {
    R dbl = limit<LIM_MC>(b[2] - b[1], b[1] - b[0]);
    R dbr = limit<LIM_MC>(b[3] - b[2], b[2] - b[1]);
    R dql = limit<LIM>(q[2] - q[1], q[1] - q[0]);
    R dqr = limit<LIM>(q[3] - q[2], q[2] - q[1]);
    bL = b[1] + R(0.5) * dbl;
    bR = b[2] - R(0.5) * dbr;
    vL = q[1] + R(0.5) * dql;
    vR = q[2] - R(0.5) * dqr;
  }
  phi = dR * bR - dL * bL;
  avg = aL * vL * bL + aR * vR * bR;
}

template <typename R, typename CTT>
__device__ __forceinline__ void face_coef(const StageArgs<CTT>& a, int d, long long f1,
                                          long long f2, R& aL, R& aR, R& dL, R& dR) {
  aL = R(0.5) * ((R)a.ct[d][2][f1] + (R)a.ct[d][2][f2]);
  aR = R(0.5) * ((R)a.ct[d][3][f1] + (R)a.ct[d][3][f2]);
  dL = R(0.5) * ((R)a.ct[d][4][f1] + (R)a.ct[d][4][f2]);
  dR = R(0.5) * ((R)a.ct[d][5][f1] + (R)a.ct[d][5][f2]);
}

// The edge EMFs whose lower corner is cell c (all three in 3-D, Ez in 2-D).
// The wrapped offsets of the stencil rows (index - 2 .. index + 1 along each
// direction; index - 3 .. index + 2 with MP5) are formed once; every operand
// address is then a sum of three.
// Offsets are 32-bit: grids are limited to fewer than 2^31 cells.
template <int NDIM, int LIM, typename R, typename CTT>
__device__ __forceinline__ void emf_cell(const StageArgs<CTT>& a, const Grid3& g, long long c) {
  if (c >= g.n) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int nxy = nx * ny;
  const int ci = (int)c;
  const int i = ci % nx;
  const int j = (ci / nx) % ny;
  const int k = ci / nxy;
  constexpr int W = emf_width<LIM>(), C = W / 2;  // stencil cells i-C .. i+C-1
  int X[W], Y[W], Z[W];
#pragma unroll
  for (int m = 0; m < W; m++) {
    X[m] = wrapi(i - C + m, nx);
    Y[m] = nx * wrapi(j - C + m, ny);
    Z[m] = NDIM == 3 ? nxy * wrapi(k - C + m, nz) : 0;
  }
  R b[W], q[W], aL, aR, dL, dR, avg, phi;
  // Ez at (i-1/2, j-1/2, k)
  {
#pragma unroll
    for (int m = 0; m < W; m++) {
      const int e = X[m] + Y[C] + Z[C];
      b[m] = (R)a.Bs[1][e];
      q[m] = (R)a.ct[1][1][e];
    }
    face_coef<R>(a, 0, X[C] + Y[C - 1] + Z[C], c, aL, aR, dL, dR);
    uct_terms<LIM>(b, q, aL, aR, dL, dR, avg, phi, (R)a.dx[0]);
    R Ez = avg + phi;
#pragma unroll
    for (int m = 0; m < W; m++) {
      const int e = X[C] + Y[m] + Z[C];
      b[m] = (R)a.Bs[0][e];
      q[m] = (R)a.ct[0][0][e];
    }
    face_coef<R>(a, 1, X[C - 1] + Y[C] + Z[C], c, aL, aR, dL, dR);
    uct_terms<LIM>(b, q, aL, aR, dL, dR, avg, phi, (R)a.dx[1]);
    Ez += avg - phi;
    a.Ee[2][c] = (CTT)Ez;
  }
  if constexpr (NDIM == 3) {
    // Ey at (i-1/2, j, k-1/2)
    {
#pragma unroll
      for (int m = 0; m < W; m++) {
        const int e = X[m] + Y[C] + Z[C];
        b[m] = (R)a.Bs[2][e];
        q[m] = (R)a.ct[2][0][e];
      }
      face_coef<R>(a, 0, X[C] + Y[C] + Z[C - 1], c, aL, aR, dL, dR);
      uct_terms<LIM>(b, q, aL, aR, dL, dR, avg, phi, (R)a.dx[0]);
      R Ey = avg - phi;
#pragma unroll
      for (int m = 0; m < W; m++) {
        const int e = X[C] + Y[C] + Z[m];
        b[m] = (R)a.Bs[0][e];
        q[m] = (R)a.ct[0][1][e];
      }
      face_coef<R>(a, 2, X[C - 1] + Y[C] + Z[C], c, aL, aR, dL, dR);
      uct_terms<LIM>(b, q, aL, aR, dL, dR, avg, phi, (R)a.dx[2]);
      Ey += avg + phi;
      a.Ee[1][c] = (CTT)Ey;
    }
    // Ex at (i, j-1/2, k-1/2)
    {
#pragma unroll
      for (int m = 0; m < W; m++) {
        const int e = X[C] + Y[m] + Z[C];
        b[m] = (R)a.Bs[2][e];
        q[m] = (R)a.ct[2][1][e];
      }
      face_coef<R>(a, 1, X[C] + Y[C] + Z[C - 1], c, aL, aR, dL, dR);
      uct_terms<LIM>(b, q, aL, aR, dL, dR, avg, phi, (R)a.dx[1]);
      R Ex = avg + phi;
#pragma unroll
      for (int m = 0; m < W; m++) {
        const int e = X[C] + Y[C] + Z[m];
        b[m] = (R)a.Bs[1][e];
        q[m] = (R)a.ct[1][0][e];
      }
      face_coef<R>(a, 2, X[C] + Y[C - 1] + Z[C], c, aL, aR, dL, dR);
      uct_terms<LIM>(b, q, aL, aR, dL, dR, avg, phi, (R)a.dx[2]);
      Ex += avg - phi;
      a.Ee[0][c] = (CTT)Ex;
    }
  }
}

template <int NDIM, int LIM, typename R, typename CTT>
__global__ void __launch_bounds__(256, 4) emf_kernel(StageArgs<CTT> a, Grid3 g) {
  emf_cell<NDIM, LIM, R, CTT>(a, g, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

// 3-D edge EMFs of the mixed form (FP32 operands), one thread per (i, j)
// column marching k over a segment of `sz` planes; blocks of 32 x 8 columns.
// Same operands and operation order as emf_cell: the z-stencils (Bs_x and
// Bs_y with their velocities along z) roll through a 4-plane register
// window, and the face coefficients of a cell are loaded once and kept for
// the next plane's k-1 neighbour, so the loads that remain (x and y stencils
// of the current plane) fall in the block's 32 x 8 tile and its halo.
constexpr int EMF_TX = 32, EMF_TY = 8, EMF_SEGMENT = 16;

template <typename R, typename CTT>
__device__ __forceinline__ void coef_load(const StageArgs<CTT>& a, int d, int f, R* c) {
#pragma unroll
  for (int q = 0; q < 4; q++) c[q] = (R)a.ct[d][2 + q][f];
}

template <typename R>
__device__ __forceinline__ void coef_pair(const R* f1, const R* f2, R& aL, R& aR, R& dL,
                                          R& dR) {
  aL = R(0.5) * (f1[0] + f2[0]);
  aR = R(0.5) * (f1[1] + f2[1]);
  dL = R(0.5) * (f1[2] + f2[2]);
  dR = R(0.5) * (f1[3] + f2[3]);
}

template <int LIM, typename R, typename CTT>
__global__ void __launch_bounds__(EMF_TX * EMF_TY, 3)
    emf_march_kernel(StageArgs<CTT> a, Grid3 g, int sz) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int i = blockIdx.x * EMF_TX + threadIdx.x;
  const int j = blockIdx.y * EMF_TY + threadIdx.y;
  if (i >= nx || j >= ny) return;
  const int k0 = blockIdx.z * sz, k1 = min(k0 + sz, nz);
  const int nxy = nx * ny;
  int X[4], Y[4];
#pragma unroll
  for (int m = 0; m < 4; m++) {
    X[m] = wrapi(i - 2 + m, nx);
    Y[m] = nx * wrapi(j - 2 + m, ny);
  }
  const int cxy = X[2] + Y[2];
  // z window: plane k-2+m in slot m
  R zb0[4], zq0[4], zb1[4], zq1[4];
#pragma unroll
  for (int m = 0; m < 3; m++) {
    const int e = cxy + nxy * wrapi(k0 - 2 + m, nz);
    zb0[m] = (R)a.Bs[0][e];
    zq0[m] = (R)a.ct[0][1][e];
    zb1[m] = (R)a.Bs[1][e];
    zq1[m] = (R)a.ct[1][0][e];
  }
  R c0m[4], c1m[4];  // face coefficients of directions 0 and 1 at (i, j, k-1)
  {
    const int e = cxy + nxy * wrapi(k0 - 1, nz);
    coef_load<R>(a, 0, e, c0m);
    coef_load<R>(a, 1, e, c1m);
  }
  R b[4], q[4], f1[4], aL, aR, dL, dR, avg, phi;
  for (int k = k0; k < k1; k++) {
    const int Zk = nxy * k;
    const int c = cxy + Zk;
    {
      const int e = cxy + nxy * wrapi(k + 1, nz);
      zb0[3] = (R)a.Bs[0][e];
      zq0[3] = (R)a.ct[0][1][e];
      zb1[3] = (R)a.Bs[1][e];
      zq1[3] = (R)a.ct[1][0][e];
    }
    // The six half-edge terms grouped by the face coefficients they share
    // (each EMF still sums its own two terms in emf_cell's order), so that
    // one set of cell coefficients is live at a time.
    R Ez, Ey, Ex, cc[4];
    coef_load<R>(a, 0, c, cc);
    {  // Ez, first term: Bs_y along x
#pragma unroll
      for (int m = 0; m < 4; m++) {
        const int e = X[m] + Y[2] + Zk;
        b[m] = (R)a.Bs[1][e];
        q[m] = (R)a.ct[1][1][e];
      }
      coef_load<R>(a, 0, X[2] + Y[1] + Zk, f1);
      coef_pair(f1, cc, aL, aR, dL, dR);
      uct_terms<LIM>(b, q, aL, aR, dL, dR, avg, phi, (R)a.dx[0]);
      Ez = avg + phi;
    }
    {  // Ey, first term: Bs_z along x
#pragma unroll
      for (int m = 0; m < 4; m++) {
        const int e = X[m] + Y[2] + Zk;
        b[m] = (R)a.Bs[2][e];
        q[m] = (R)a.ct[2][0][e];
      }
      coef_pair(c0m, cc, aL, aR, dL, dR);
      uct_terms<LIM>(b, q, aL, aR, dL, dR, avg, phi, (R)a.dx[0]);
      Ey = avg - phi;
    }
#pragma unroll
    for (int m = 0; m < 4; m++) c0m[m] = cc[m];
    coef_load<R>(a, 1, c, cc);
    {  // Ez, second term: Bs_x along y
#pragma unroll
      for (int m = 0; m < 4; m++) {
        const int e = X[2] + Y[m] + Zk;
        b[m] = (R)a.Bs[0][e];
        q[m] = (R)a.ct[0][0][e];
      }
      coef_load<R>(a, 1, X[1] + Y[2] + Zk, f1);
      coef_pair(f1, cc, aL, aR, dL, dR);
      uct_terms<LIM>(b, q, aL, aR, dL, dR, avg, phi, (R)a.dx[1]);
      Ez += avg - phi;
    }
    {  // Ex, first term: Bs_z along y
#pragma unroll
      for (int m = 0; m < 4; m++) {
        const int e = X[2] + Y[m] + Zk;
        b[m] = (R)a.Bs[2][e];
        q[m] = (R)a.ct[2][1][e];
      }
      coef_pair(c1m, cc, aL, aR, dL, dR);
      uct_terms<LIM>(b, q, aL, aR, dL, dR, avg, phi, (R)a.dx[1]);
      Ex = avg + phi;
    }
#pragma unroll
    for (int m = 0; m < 4; m++) c1m[m] = cc[m];
    coef_load<R>(a, 2, c, cc);
    {  // Ey, second term: Bs_x along z (window)
      coef_load<R>(a, 2, X[1] + Y[2] + Zk, f1);
      coef_pair(f1, cc, aL, aR, dL, dR);
      uct_terms<LIM>(zb0, zq0, aL, aR, dL, dR, avg, phi, (R)a.dx[2]);
      Ey += avg + phi;
    }
    {  // Ex, second term: Bs_y along z (window)
      coef_load<R>(a, 2, X[2] + Y[1] + Zk, f1);
      coef_pair(f1, cc, aL, aR, dL, dR);
      uct_terms<LIM>(zb1, zq1, aL, aR, dL, dR, avg, phi, (R)a.dx[2]);
      Ex += avg - phi;
    }
    a.Ee[2][c] = (CTT)Ez;
    a.Ee[1][c] = (CTT)Ey;
    a.Ee[0][c] = (CTT)Ex;
#pragma unroll
    for (int m = 0; m < 3; m++) {
      zb0[m] = zb0[m + 1];
      zq0[m] = zq0[m + 1];
      zb1[m] = zb1[m + 1];
      zq1[m] = zq1[m + 1];
    }
  }
}

// Edge EMFs of CT_EMF_AVERAGE ARITHMETIC (Src/MHD/CT/ct_emf_average.cpp:36-96,
// w = 0.25): each edge averages the four face EMFs around it, face d's two
// components stored as ct[d][0] = e[b][d], ct[d][1] = e[t][d].
template <int NDIM, typename R, typename CTT>
__global__ void __launch_bounds__(256) emf_arith_kernel(StageArgs<CTT> a, Grid3 g) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= g.n) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz, nxy = nx * ny;
  const int ci = (int)c, i = ci % nx, j = (ci / nx) % ny, k = ci / nxy;
  const int cxm = ci - i + wrapi(i - 1, nx), cym = ci + nx * (wrapi(j - 1, ny) - j);
  const R w = R(0.25);
  // Ez at (i-1/2, j-1/2, k): e[z][x] = ct[0][0], e[z][y] = ct[1][1]
  a.Ee[2][c] = (CTT)(w * ((R)a.ct[0][0][ci] + (R)a.ct[0][0][cym] + (R)a.ct[1][1][ci] +
                          (R)a.ct[1][1][cxm]));
  if constexpr (NDIM == 3) {
    const int czm = ci + nxy * (wrapi(k - 1, nz) - k);
    // Ex at (i, j-1/2, k-1/2): e[x][z] = ct[2][1], e[x][y] = ct[1][0]
    a.Ee[0][c] = (CTT)(w * ((R)a.ct[2][1][ci] + (R)a.ct[2][1][cym] + (R)a.ct[1][0][ci] +
                            (R)a.ct[1][0][czm]));
    // Ey at (i-1/2, j, k-1/2): e[y][x] = ct[0][1], e[y][z] = ct[2][0]
    a.Ee[1][c] = (CTT)(w * ((R)a.ct[0][1][ci] + (R)a.ct[0][1][czm] + (R)a.ct[2][0][ci] +
                            (R)a.ct[2][0][cxm]));
  }
}

// CT_EMF_AVERAGE CT_CONTACT (Src/MHD/CT/ct_emf.cpp:220-245): per edge the
// four face EMFs summed (CT_EMF_ArithmeticAverage with w = 1), the terms of
// CT_EMF_IntegrateToCorner (Src/MHD/CT/ct_emf_average.cpp:115-290; Gardiner
// & Stone 2005, eqs. 41-50) -- derivatives of E between the faces and the
// cell-centred field -v x B, each taken from the upwind cell of the face's
// contact (weights in ct[d][2]) -- then times 1/4, in the reference's
// operation order.  Thread per cell, its three edges.
template <int NDIM, typename R, typename CTT>
__global__ void __launch_bounds__(256) emf_contact_kernel(StageArgs<CTT> a, Grid3 g) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= g.n) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz, nxy = nx * ny;
  const long long n = g.n;
  const int ci = (int)c, i = ci % nx, j = (ci / nx) % ny, k = ci / nxy;
  const int dx = wrapi(i - 1, nx) - i, dy = nx * (wrapi(j - 1, ny) - j);
  const int dz = NDIM == 3 ? nxy * (wrapi(k - 1, nz) - k) : 0;
  const double* V = a.V;
  // cell-centred inductive field (CT_ComputeCenterEMF, Src/MHD/CT/ct_emf.cpp:333-367)
  auto ecc = [&](int comp, int q) -> R {
    const R vx1 = (R)V[VX1 * n + q], vx2 = (R)V[(VX1 + 1) * n + q], vx3 = (R)V[(VX1 + 2) * n + q];
    const R bx1 = (R)V[BX1 * n + q], bx2 = (R)V[BX2 * n + q], bx3 = (R)V[BX3 * n + q];
    if (comp == 0) return (vx3 * bx2 - vx2 * bx3);
    if (comp == 1) return (vx1 * bx3 - vx3 * bx1);
    return (vx2 * bx1 - vx1 * bx2);
  };
  auto f = [&](int d, int r, int q) -> R { return (R)a.ct[d][r][q]; };
  const R one = R(1);
  {  // Ez at (i-1/2, j-1/2, k): e[z][x] = ct[0][0], e[z][y] = ct[1][1]
    const int c0 = ci, cxm = ci + dx, cym = ci + dy, cxym = ci + dx + dy;
    R E = one * (f(0, 0, c0) + f(0, 0, cym) + f(1, 1, c0) + f(1, 1, cxm));
    const R wS = f(0, 2, cym), wN = f(0, 2, c0);
    E += wS * (f(1, 1, cxm) - ecc(2, cxym)) + (one - wS) * (f(1, 1, c0) - ecc(2, cym)) -
         wN * (ecc(2, cxm) - f(1, 1, cxm)) - (one - wN) * (ecc(2, c0) - f(1, 1, c0));
    const R wW = f(1, 2, cxm), wE = f(1, 2, c0);
    E += wW * (f(0, 0, cym) - ecc(2, cxym)) + (one - wW) * (f(0, 0, c0) - ecc(2, cxm)) -
         wE * (ecc(2, cym) - f(0, 0, cym)) - (one - wE) * (ecc(2, c0) - f(0, 0, c0));
    a.Ee[2][c] = (CTT)(E * R(0.25));
  }
  if constexpr (NDIM == 3) {
    {  // Ex at (i, j-1/2, k-1/2): e[x][z] = ct[2][1], e[x][y] = ct[1][0]
      const int c0 = ci, cym = ci + dy, czm = ci + dz, cyzm = ci + dy + dz;
      R E = one * (f(2, 1, c0) + f(2, 1, cym) + f(1, 0, c0) + f(1, 0, czm));
      const R wS = f(1, 2, czm), wN = f(1, 2, c0);
      E += wS * (f(2, 1, cym) - ecc(0, cyzm)) + (one - wS) * (f(2, 1, c0) - ecc(0, czm)) -
           wN * (ecc(0, cym) - f(2, 1, cym)) - (one - wN) * (ecc(0, c0) - f(2, 1, c0));
      const R wW = f(2, 2, cym), wE = f(2, 2, c0);
      E += wW * (f(1, 0, czm) - ecc(0, cyzm)) + (one - wW) * (f(1, 0, c0) - ecc(0, cym)) -
           wE * (ecc(0, czm) - f(1, 0, czm)) - (one - wE) * (ecc(0, c0) - f(1, 0, c0));
      a.Ee[0][c] = (CTT)(E * R(0.25));
    }
    {  // Ey at (i-1/2, j, k-1/2): e[y][x] = ct[0][1], e[y][z] = ct[2][0]
      const int c0 = ci, cxm = ci + dx, czm = ci + dz, cxzm = ci + dx + dz;
      R E = one * (f(0, 1, c0) + f(0, 1, czm) + f(2, 0, c0) + f(2, 0, cxm));
      const R wS = f(2, 2, cxm), wN = f(2, 2, c0);
      E += wS * (f(0, 1, czm) - ecc(1, cxzm)) + (one - wS) * (f(0, 1, c0) - ecc(1, cxm)) -
           wN * (ecc(1, czm) - f(0, 1, czm)) - (one - wN) * (ecc(1, c0) - f(0, 1, c0));
      const R wW = f(0, 2, czm), wE = f(0, 2, c0);
      E += wW * (f(2, 0, cxm) - ecc(1, cxzm)) + (one - wW) * (f(2, 0, c0) - ecc(1, czm)) -
           wE * (ecc(1, cxm) - f(2, 0, cxm)) - (one - wE) * (ecc(1, c0) - f(2, 0, c0));
      a.Ee[1][c] = (CTT)(E * R(0.25));
    }
  }
}

// 3-D edge EMFs with the in-plane stencils staged in shared memory.  Blocks
// of ETX x ETY (i, j) columns march k over a segment of planes.  While plane
// k is computed, the block's cp.async copies of plane k+1 fill the other half
// of a double buffer: the face fields and velocities along x and along y with
// their stencil halos, and the three directions' face coefficients with their
// i-1 / j-1 neighbours, each tile row a contiguous run of one array.  The
// z-stencils (Bs_x, Bs_y and their velocities along z) roll through a W-plane
// register window and the cell's own face coefficients are kept for the next
// plane's k-1 neighbour.  Operands and operation order are emf_cell's, so the
// FP64 form is bit-identical to it.
constexpr int ETX = 32, ETY = 8, ET_THREADS = ETX * ETY, ET_SEGMENT = 32;

template <int LIM, typename CTT>
struct EmfTile {
  static constexpr int W = emf_width<LIM>(), HL = W / 2;  // stencil i-HL .. i+HL-1
  static constexpr int XW = ETX + W - 1, YH = ETY + W - 1;
  static constexpr int NXG = XW * ETY;              // tiles of the x stencils
  static constexpr int NYG = ETX * YH;              // tiles of the y stencils
  static constexpr int NB2 = XW * YH;               // Bs_z: both stencils
  static constexpr int N0 = ETX * (ETY + 1);        // direction-0 coefficients, j-1 row
  static constexpr int N1 = (ETX + 1) * ETY;        // direction-1 coefficients, i-1 column
  static constexpr int N2 = (ETX + 1) * (ETY + 1);  // direction-2 coefficients, both
  // One plane: Bs_y (x tile), Bs_x (y tile), Bs_z as double; then ct[1][1],
  // ct[2][0] (x tiles), ct[0][0], ct[2][1] (y tiles) and the 4 coefficient
  // arrays of each direction as CTT.
  static constexpr int ND = NXG + NYG + NB2;
  static constexpr int NC = 2 * NXG + 2 * NYG + 4 * (N0 + N1 + N2);
  static constexpr int PLANE = (ND * 8 + NC * (int)sizeof(CTT) + 15) / 16 * 16;
  static constexpr int SMEM = 2 * PLANE + (XW + YH) * 4;  // + wrapped column/row offsets
};

// Resident blocks per SM the tile kernel is compiled for: two FP64 blocks
// (91 KB of shared memory each), three mixed ones (54 KB).
template <typename R>
__host__ __device__ constexpr int emf_tile_minb() { return sizeof(R) == 8 ? 2 : 3; }

__device__ __forceinline__ int wrap_any(int i, int n) {
  const int r = i % n;
  return r < 0 ? r + n : r;
}

__device__ __forceinline__ void cp_async_el(double* s, const double* g) { cp_async8(s, g); }
__device__ __forceinline__ void cp_async_el(float* s, const float* g) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(s);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(g) : "memory");
}

// Copies a TW x TH tile of NA arrays (array q to s + q * TW * TH, row-major)
// whose element (lx, ly) is the cell at wrapped column offset xo[lx + OX] and
// row offset yo[ly + OY] of plane offset zk.
template <int TW, int TH, int OX, int OY, int NA, typename T>
__device__ __forceinline__ void stage_tile(T* s, const T* const (&src)[NA], const int* xo,
                                           const int* yo, int zk, int tid) {
  for (int e = tid; e < TW * TH; e += ET_THREADS) {
    const int ly = e / TW, lx = e - ly * TW;
    const int off = xo[lx + OX] + yo[ly + OY] + zk;
#pragma unroll
    for (int q = 0; q < NA; q++) cp_async_el(s + q * (TW * TH) + e, src[q] + off);
  }
}

template <int LIM, typename R, typename CTT>
__device__ __forceinline__ void emf_stage_plane(const StageArgs<CTT>& a, unsigned char* p,
                                                const int* xo, const int* yo, int zk,
                                                int tid) {
  using T = EmfTile<LIM, CTT>;
  constexpr int HL = T::HL, XW = T::XW, YH = T::YH;
  double* bsy = reinterpret_cast<double*>(p);
  double* bsx = bsy + T::NXG;
  double* bsz = bsx + T::NYG;
  CTT* qx = reinterpret_cast<CTT*>(bsz + T::NB2);  // ct[1][1], ct[2][0]
  CTT* qy = qx + 2 * T::NXG;                       // ct[0][0], ct[2][1]
  CTT* k0 = qy + 2 * T::NYG;
  CTT* k1 = k0 + 4 * T::N0;
  CTT* k2 = k1 + 4 * T::N1;
  {
    const double* s1[1] = {a.Bs[1]};
    stage_tile<XW, ETY, 0, HL, 1>(bsy, s1, xo, yo, zk, tid);
    const double* s0[1] = {a.Bs[0]};
    stage_tile<ETX, YH, HL, 0, 1>(bsx, s0, xo, yo, zk, tid);
    const double* s2[1] = {a.Bs[2]};
    stage_tile<XW, YH, 0, 0, 1>(bsz, s2, xo, yo, zk, tid);
  }
  {
    const CTT* sx[2] = {a.ct[1][1], a.ct[2][0]};
    stage_tile<XW, ETY, 0, HL, 2>(qx, sx, xo, yo, zk, tid);
    const CTT* sy[2] = {a.ct[0][0], a.ct[2][1]};
    stage_tile<ETX, YH, HL, 0, 2>(qy, sy, xo, yo, zk, tid);
  }
  {
    const CTT* c0[4] = {a.ct[0][2], a.ct[0][3], a.ct[0][4], a.ct[0][5]};
    stage_tile<ETX, ETY + 1, HL, HL - 1, 4>(k0, c0, xo, yo, zk, tid);
    const CTT* c1[4] = {a.ct[1][2], a.ct[1][3], a.ct[1][4], a.ct[1][5]};
    stage_tile<ETX + 1, ETY, HL - 1, HL, 4>(k1, c1, xo, yo, zk, tid);
    const CTT* c2[4] = {a.ct[2][2], a.ct[2][3], a.ct[2][4], a.ct[2][5]};
    stage_tile<ETX + 1, ETY + 1, HL - 1, HL - 1, 4>(k2, c2, xo, yo, zk, tid);
  }
}

template <typename R, typename CTT>
__device__ __forceinline__ void coef_tile(const CTT* k, int n, int e, R* c) {
#pragma unroll
  for (int q = 0; q < 4; q++) c[q] = (R)k[q * n + e];
}

template <int LIM, typename R, typename CTT>
__global__ void __launch_bounds__(ET_THREADS, (emf_tile_minb<R>()))
    emf_tile_kernel(StageArgs<CTT> a, Grid3 g, int sz) {
  using T = EmfTile<LIM, CTT>;
  constexpr int W = T::W, HL = T::HL, HR = W - 1 - HL, XW = T::XW, YH = T::YH;
  extern __shared__ __align__(16) unsigned char emf_smem[];
  int* xo = reinterpret_cast<int*>(emf_smem + 2 * T::PLANE);
  int* yo = xo + XW;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int nxy = nx * ny;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * ETX + tx;
  const int i = blockIdx.x * ETX + tx, j = blockIdx.y * ETY + ty;
  const bool valid = i < nx && j < ny;
  const int k0 = blockIdx.z * sz, k1 = min(k0 + sz, nz);
  for (int l = tid; l < XW; l += ET_THREADS) xo[l] = wrap_any(blockIdx.x * ETX - HL + l, nx);
  for (int l = tid; l < YH; l += ET_THREADS) yo[l] = nx * wrap_any(blockIdx.y * ETY - HL + l, ny);
  __syncthreads();
  emf_stage_plane<LIM, R, CTT>(a, emf_smem, xo, yo, nxy * k0, tid);
  cp_async_commit();

  const int cxy = i + nx * j;
  // z window: plane k-HL+m in slot m
  R zb0[W], zq0[W], zb1[W], zq1[W];
  R c0m[4], c1m[4];  // face coefficients of directions 0 and 1 at (i, j, k-1)
  if (valid) {
#pragma unroll
    for (int m = 0; m < W - 1; m++) {
      const int e = cxy + nxy * wrapi(k0 - HL + m, nz);
      zb0[m] = (R)a.Bs[0][e];
      zq0[m] = (R)a.ct[0][1][e];
      zb1[m] = (R)a.Bs[1][e];
      zq1[m] = (R)a.ct[1][0][e];
    }
    const int e = cxy + nxy * wrapi(k0 - 1, nz);
    coef_load<R>(a, 0, e, c0m);
    coef_load<R>(a, 1, e, c1m);
  }
  // this thread's elements of each tile
  const int ex = ty * XW + tx;          // x tiles, stencil start (i-HL, j)
  const int ey = ty * ETX + tx;         // y tiles, stencil start (i, j-HL)
  const int e0 = ty * ETX + tx;         // direction-0 coefficients at (i, j-1); +ETX: (i, j)
  const int e1 = ty * (ETX + 1) + tx;   // direction-1 coefficients at (i-1, j); +1: (i, j)
  const int e2 = ty * (ETX + 1) + tx;   // direction-2: (i, j-1) at e2+1, (i-1, j) at
                                        // e2+ETX+1, (i, j) at e2+ETX+2
  for (int k = k0; k < k1; k++) {
    const int buf = (k - k0) & 1;
    if (valid) {
      const int e = cxy + nxy * wrapi(k + HR, nz);
      zb0[W - 1] = (R)a.Bs[0][e];
      zq0[W - 1] = (R)a.ct[0][1][e];
      zb1[W - 1] = (R)a.Bs[1][e];
      zq1[W - 1] = (R)a.ct[1][0][e];
    }
    cp_async_wait0();
    __syncthreads();  // plane k staged by every thread; plane k-1 read by every thread
    if (k + 1 < k1)
      emf_stage_plane<LIM, R, CTT>(a, emf_smem + (buf ^ 1) * T::PLANE, xo, yo, nxy * (k + 1),
                                   tid);
    cp_async_commit();
    if (valid) {
      unsigned char* p = emf_smem + buf * T::PLANE;
      const double* bsy = reinterpret_cast<const double*>(p);
      const double* bsx = bsy + T::NXG;
      const double* bsz = bsx + T::NYG;
      const CTT* qx = reinterpret_cast<const CTT*>(bsz + T::NB2);
      const CTT* qy = qx + 2 * T::NXG;
      const CTT* kk0 = qy + 2 * T::NYG;
      const CTT* kk1 = kk0 + 4 * T::N0;
      const CTT* kk2 = kk1 + 4 * T::N1;
      R b[W], q[W], f1[4], cc[4], aL, aR, dL, dR, avg, phi, Ez, Ey, Ex;
      coef_tile(kk0, T::N0, e0 + ETX, cc);
      {  // Ez, first term: Bs_y along x
#pragma unroll
        for (int m = 0; m < W; m++) {
          b[m] = (R)bsy[ex + m];
          q[m] = (R)qx[ex + m];
        }
        coef_tile(kk0, T::N0, e0, f1);
        coef_pair(f1, cc, aL, aR, dL, dR);
        uct_terms<LIM>(b, q, aL, aR, dL, dR, avg, phi, (R)a.dx[0]);
        Ez = avg + phi;
      }
      {  // Ey, first term: Bs_z along x
#pragma unroll
        for (int m = 0; m < W; m++) {
          b[m] = (R)bsz[(ty + HL) * XW + tx + m];
          q[m] = (R)qx[T::NXG + ex + m];
        }
        coef_pair(c0m, cc, aL, aR, dL, dR);
        uct_terms<LIM>(b, q, aL, aR, dL, dR, avg, phi, (R)a.dx[0]);
        Ey = avg - phi;
      }
#pragma unroll
      for (int m = 0; m < 4; m++) c0m[m] = cc[m];
      coef_tile(kk1, T::N1, e1 + 1, cc);
      {  // Ez, second term: Bs_x along y
#pragma unroll
        for (int m = 0; m < W; m++) {
          b[m] = (R)bsx[ey + m * ETX];
          q[m] = (R)qy[ey + m * ETX];
        }
        coef_tile(kk1, T::N1, e1, f1);
        coef_pair(f1, cc, aL, aR, dL, dR);
        uct_terms<LIM>(b, q, aL, aR, dL, dR, avg, phi, (R)a.dx[1]);
        Ez += avg - phi;
      }
      {  // Ex, first term: Bs_z along y
#pragma unroll
        for (int m = 0; m < W; m++) {
          b[m] = (R)bsz[(ty + m) * XW + tx + HL];
          q[m] = (R)qy[T::NYG + ey + m * ETX];
        }
        coef_pair(c1m, cc, aL, aR, dL, dR);
        uct_terms<LIM>(b, q, aL, aR, dL, dR, avg, phi, (R)a.dx[1]);
        Ex = avg + phi;
      }
#pragma unroll
      for (int m = 0; m < 4; m++) c1m[m] = cc[m];
      coef_tile(kk2, T::N2, e2 + ETX + 2, cc);
      {  // Ey, second term: Bs_x along z (window)
        coef_tile(kk2, T::N2, e2 + ETX + 1, f1);
        coef_pair(f1, cc, aL, aR, dL, dR);
        uct_terms<LIM>(zb0, zq0, aL, aR, dL, dR, avg, phi, (R)a.dx[2]);
        Ey += avg + phi;
      }
      {  // Ex, second term: Bs_y along z (window)
        coef_tile(kk2, T::N2, e2 + 1, f1);
        coef_pair(f1, cc, aL, aR, dL, dR);
        uct_terms<LIM>(zb1, zq1, aL, aR, dL, dR, avg, phi, (R)a.dx[2]);
        Ex += avg - phi;
      }
      const int c = cxy + nxy * k;
      a.Ee[2][c] = (CTT)Ez;
      a.Ee[1][c] = (CTT)Ey;
      a.Ee[0][c] = (CTT)Ex;
#pragma unroll
      for (int m = 0; m < W - 1; m++) {
        zb0[m] = zb0[m + 1];
        zq0[m] = zq0[m + 1];
        zb1[m] = zb1[m + 1];
        zq1[m] = zq1[m + 1];
      }
    }
  }
  cp_async_wait0();
}

// ---------------------------------------------------------------------
// Stage finish: CT update (Src/MHD/CT/ct_update.cpp:181-423), face RK
// combine (Src/rk_step.cpp:378-385, 536-552), cell-centred average
// (Src/MHD/CT/ct_field_average.cpp:175-200), con2prim
// (Src/mappers3D.cpp:104-194) -- all FP64.
// ---------------------------------------------------------------------
// -(curl E)·dt/dx of face d of the cell at offsets (X[x], Y[y], Z[z]) (the
// wrapped offsets are formed once by the caller)
template <int NDIM, typename CTT>
__device__ __forceinline__ double face_rs_at(const StageArgs<CTT>& a, int d, const int* X,
                                             const int* Y, const int* Z, int x, int y, int z) {
  auto E = [&](int q, int ox, int oy, int oz) -> double {
    return (double)a.Ee[q][X[x + ox] + Y[y + oy] + Z[z + oz]];
  };
  double curlE;
  if (d == 0) {
    curlE = 0.0 + a.dtdx[1] * (E(2, 0, 1, 0) - E(2, 0, 0, 0));
    if (NDIM == 3) curlE = curlE - a.dtdx[2] * (E(1, 0, 0, 1) - E(1, 0, 0, 0));
  } else if (d == 1) {
    curlE = -a.dtdx[0] * (E(2, 1, 0, 0) - E(2, 0, 0, 0));
    if (NDIM == 3) curlE = curlE + a.dtdx[2] * (E(0, 0, 0, 1) - E(0, 0, 0, 0));
  } else {
    curlE = a.dtdx[0] * (E(1, 1, 0, 0) - E(1, 0, 0, 0)) -
            a.dtdx[1] * (E(0, 0, 1, 0) - E(0, 0, 0, 0));
  }
  return -curlE;
}

template <typename CTT>
__device__ __forceinline__ double face_new(const StageArgs<CTT>& a, int d, long long f,
                                           double rs) {
  double bc = a.Bs[d][f];
  if (a.stage == 1) return bc + rs;
  return a.w0 * a.Bs0[d][f] + a.w1 * bc + a.wr * rs;
}

// Stage finish of cell c; returns its inverse-dt sum (0 outside the grid).
template <int PHYS, int NV, int NDIM, typename CTT>
__device__ __forceinline__ double finish_cell(const StageArgs<CTT>& a, const Grid3& g,
                                              long long c) {
  const long long n = g.n;
  double cdt = 0.0;
  if (c < n) {
    double u[8], v[8];
    // RK combine of the cell-centred variables (Src/rk_step.cpp:366-374,
    // 509-517) with Rc = (rhs_x + rhs_y) + rhs_z
#pragma unroll
    for (int nv = 0; nv < NV; nv++) {
      if (!rhs_var<PHYS, NDIM>(nv)) continue;
      double Rc = (double)a.dU[nv * n + c] + (double)a.dU[(NV + nv) * n + c];
      if (NDIM == 3) Rc = Rc + (double)a.dU[(2 * NV + nv) * n + c];
      const double u0 = a.U0[nv * n + c];
      if (a.stage == 1) u[nv] = u0 + Rc;
      else u[nv] = a.w0 * u0 + a.w1 * a.Uc[nv * n + c] + a.wr * Rc;
    }
    if (a.stage == 1) {  // the CFL maximum is a stage-1 quantity
      cdt = (double)a.Cdt[c] + (double)a.Cdt[n + c];
      if (NDIM == 3) cdt = cdt + (double)a.Cdt[2 * n + c];
    }
    if constexpr (PHYS != PHYS_HD) {
      // 32-bit wrapped offsets of the index and its two successors along
      // each direction, formed once (grids hold fewer than 2^31 cells)
      const int nx = g.nx, ny = g.ny, nz = g.nz, nxy = nx * ny;
      const int ci = (int)c;
      const int i = ci % nx, j = (ci / nx) % ny, k = ci / nxy;
      int X[3], Y[3], Z[3];
#pragma unroll
      for (int m = 0; m < 3; m++) {
        X[m] = wrapi(i + m, nx);
        Y[m] = nx * wrapi(j + m, ny);
        Z[m] = NDIM == 3 ? nxy * wrapi(k + m, nz) : 0;
      }
#pragma unroll
      for (int d = 0; d < NDIM; d++) {
        const int di = (d == 0), dj = (d == 1), dk = (d == 2);
        const double bl = face_new(a, d, c, face_rs_at<NDIM>(a, d, X, Y, Z, 0, 0, 0));
        const double br = face_new(a, d, (long long)(X[di] + Y[dj] + Z[dk]),
                                   face_rs_at<NDIM>(a, d, X, Y, Z, di, dj, dk));
        a.Bsout[d][c] = bl;
        u[BX1 + d] = 0.5 * (bl + br);
      }
    }
    uint32_t err = 0;
#pragma unroll
    for (int nv = 0; nv < NV; nv++)
      if (isnan(u[nv])) err |= ERR_NAN | ERR_QUIT;
    bool dom = true;  // a domain cell (not padding)
    if (g.ihi[0] != kNoLimit || g.ihi[1] != kNoLimit || g.ihi[2] != kNoLimit) {
      const int i = (int)(c % g.nx);
      const int j = (int)((c / g.nx) % g.ny);
      const int k = (int)(c / ((long long)g.nx * g.ny));
      dom = i >= g.ilo[0] && i <= g.ihi[0] && j >= g.ilo[1] && j <= g.ihi[1] &&
            k >= g.ilo[2] && k <= g.ihi[2];
    }
    uint32_t le;
    if constexpr (PHYS == PHYS_MHD) le = mhd_cons2prim(u, v, a.gamma, a.small_rho, a.small_prs);
    else if constexpr (PHYS == PHYS_RMHD)
      le = rmhd_cons2prim(u, v, a.gamma, a.small_rho, a.small_prs);
    else le = hd_cons2prim(u, v, a.gamma, a.small_rho, a.small_prs);
    err |= le;
    if (le & ERR_CONS2PRIM_FAIL) err |= ERR_QUIT;
    // An intermediate stage's cell-centred field along the active
    // directions is never read (the next stage takes it from the faces);
    // the final stage (writing in place of U^n) stores every component.
    // FP64 form only: stage-1 finish 1.04 -> 1.00 ms at 256^3, while the
    // mixed form's 40-register finish lost 3% in stage 2 with the condition.
    const bool final_stage = sizeof(CTT) == 4 || a.Uout == a.U0;
#pragma unroll
    for (int nv = 0; nv < NV; nv++) {
      if (final_stage || rhs_var<PHYS, NDIM>(nv)) a.Uout[nv * n + c] = u[nv];
      a.Vout[nv * n + c] = v[nv];
    }
    if (!dom) {
      err = 0;
      cdt = 0.0;
    }
    if (err) atomicOr(a.err, err);
  }
  return cdt;
}

// Stage-1 CFL maximum (Src/update_stage.cpp:422-435, getMax 446-461) on the
// bit patterns of the non-negative inverse time steps, which order like the
// values.  The stored maximum only grows, so an atomic whose value does not exceed a
// (possibly older) read of it cannot change it and is skipped: the result
// is the same, and the contended atomics on the one address drop from one
// per warp to a handful per launch.
__device__ __forceinline__ void max_bits_if_larger(unsigned long long* bits,
                                                   unsigned long long v) {
  if (v > __ldcg(bits)) atomicMax(bits, v);
}

// Warp maximum, then at most one atomic per warp.  All 32 lanes must call it.
__device__ __forceinline__ void warp_invdt_max(unsigned long long* bits, double cdt, int lane) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double other = __shfl_xor_sync(0xffffffffu, cdt, o);
    cdt = GP_MAX(cdt, other);
  }
  if (lane == 0) max_bits_if_larger(bits, (unsigned long long)__double_as_longlong(cdt));
}

// Resident 256-thread blocks per SM: the mixed form's 4-byte loads need
// more requests in flight per byte than the FP64 form's to keep HBM busy.
// Measured at 256^3: mixed 4 blocks 1.01/1.04 ms (stage 1/2), 5 blocks the
// same, 6 blocks (40 registers) 0.92/0.97 ms, 8 blocks 1.12/1.17 ms; the
// FP64 finish gains nothing from 6 (1.02/1.12 against 1.04/1.08 ms).
template <typename CTT>
__host__ __device__ constexpr int finish_minb() { return sizeof(CTT) == 4 ? 6 : 4; }

template <int PHYS, int NV, int NDIM, typename CTT>
__global__ void __launch_bounds__(256, finish_minb<CTT>()) finish_kernel(StageArgs<CTT> a, Grid3 g) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const double cdt = finish_cell<PHYS, NV, NDIM, CTT>(a, g, c);
  // per-warp maximum: a block-wide one (a barrier per block) made the FP64
  // finish 9% slower in stage 1 and 5% in stage 2 at 256^3
  if (a.stage == 1) warp_invdt_max(a.invdt_bits, cdt, threadIdx.x & 31);
}

// Start-up primitive -> conservative map (Src/startup.cpp:542-566).
template <int PHYS, int NV>
__global__ void prim2cons_kernel(const double* __restrict__ V, double* __restrict__ U,
                                 long long n, double gamma) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  double v[8], u[8];
#pragma unroll
  for (int nv = 0; nv < NV; nv++) v[nv] = V[nv * n + c];
  if constexpr (PHYS == PHYS_MHD) mhd_prim2cons(v, u, gamma - 1.0);
  else if constexpr (PHYS == PHYS_RMHD) rmhd_prim2cons(v, u, gamma);
  else hd_prim2cons(v, u, gamma);
#pragma unroll
  for (int nv = 0; nv < NV; nv++) U[nv * n + c] = u[nv];
}

}  // namespace gp
