// gp_phys.cuh -- per-interface physics of the Godunov step for sm_100a.
//
// Device functions for PLM slope limiting, primitive/conservative maps,
// fluxes, signal speeds, the HLLD/HLL (MHD) and HLLC/HLL (HD) Riemann
// solvers and the upwind-CT face data they store.  Every expression keeps the
// operation order of the gPLUTO sources cited beside it so that the FP64
// build (compiled with -fmad=false) reproduces the reference bit for bit.
// The templates are parameterised on the flux arithmetic type R: double for
// the plain form, float for the mixed form (FP32 reconstruction, limiters and
// Riemann fluxes; the callers keep accumulation in FP64).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gp {

// variable indices, Src/MHD/mhd.hpp:21-33 and Src/HD/hd.hpp:21-27
enum : int { RHO = 0, MX1 = 1, MX2 = 2, MX3 = 3, BX1 = 4, BX2 = 5, BX3 = 6 };
constexpr int VX1 = MX1;

// error bits, Src/gpluto.hpp:247-262
constexpr uint32_t ERR_NEGATIVE_RHO = 1u << 0;
constexpr uint32_t ERR_NEGATIVE_ENG = 1u << 1;
constexpr uint32_t ERR_NEGATIVE_PRS = 1u << 2;
constexpr uint32_t ERR_CONS2PRIM_FAIL = 1u << 4;
constexpr uint32_t ERR_ENG_SOLVE_INACCURATE = 1u << 6;
constexpr uint32_t ERR_ENG_SOLVE_NO_SOLUTION = 1u << 7;
constexpr uint32_t ERR_SUPERLUMINAL_SPEED = 1u << 8;
constexpr uint32_t ERR_TOO_MANY_ITERATIONS = 1u << 9;
constexpr uint32_t ERR_NAN = 1u << 11;
constexpr uint32_t ERR_QUIT = 1u << 15;

enum : int { PHYS_HD = 0, PHYS_MHD = 1, PHYS_RMHD = 2 };
// LIM_PPM and LIM_MP5 select piecewise parabolic and monotonicity-preserving
// 5th-order reconstruction (RECONSTRUCTION PARABOLIC / MP5); they are
// carried in the limiter slot of the scheme templates.
enum : int { LIM_FLAT = 0, LIM_MINMOD = 1, LIM_VL = 2, LIM_MC = 3, LIM_PPM = 4, LIM_MP5 = 5,
             LIM_VANALBADA = 6, LIM_OSPRE = 7, LIM_UMIST = 8, LIM_WENOZ = 9, LIM_LIMO3 = 10,
             LIM_WENO3 = 11 };

// MP5 and WENO-Z share the 5-point driver (Src/States/mp5_states.cpp) and
// differ only in the edge value; LimO3 and WENO3 use the same driver with a
// 3-point stencil (the PLM stencil and ghost depth).
template <int LIM>
__host__ __device__ constexpr bool five_point() { return LIM == LIM_MP5 || LIM == LIM_WENOZ; }
template <int LIM>
__host__ __device__ constexpr bool three_point() { return LIM == LIM_LIMO3 || LIM == LIM_WENO3; }
enum : int { RS_HLL = 0, RS_HLLC = 1, RS_HLLD = 2, RS_TVDLF = 3 };
enum : int { CT_UCT_HLL = 0, CT_UCT_HLLD = 1, CT_ARITH = 2, CT_CONTACT = 3 };

template <typename R> __device__ __forceinline__ R rsqrt_(R x);
template <> __device__ __forceinline__ double rsqrt_(double x) { return sqrt(x); }
template <> __device__ __forceinline__ float rsqrt_(float x) { return sqrtf(x); }
template <typename R> __device__ __forceinline__ R rabs(R x) { return fabs(x); }
template <> __device__ __forceinline__ float rabs(float x) { return fabsf(x); }

#define GP_MAX(a, b) ((a) >= (b) ? (a) : (b))      // Src/macros.hpp:191
#define GP_MIN(a, b) ((a) <= (b) ? (a) : (b))      // Src/macros.hpp:194

// ---------------------------------------------------------------------
// PLM slope limiters on a uniform Cartesian grid (SET_*_LIMITER of
// Src/plm_coeffs.hpp:55-110, ABS_MIN of Src/macros.hpp:14) and
// Src/macros.hpp:200; FLAT gives a zero slope.
// ---------------------------------------------------------------------
template <int LIM, typename R>
__device__ __forceinline__ R limit(R dvp, R dvm) {
  if constexpr (LIM == LIM_MC) {
    if (dvp * dvm > R(0)) {
      R qc = R(0.5) * (dvm + dvp);
      R scrh = R(2) * (rabs(dvp) < rabs(dvm) ? dvp : dvm);
      return rabs(qc) < rabs(scrh) ? qc : scrh;
    }
    return R(0);
  } else if constexpr (LIM == LIM_VL) {
    return (dvp * dvm > R(0) ? R(2) * dvp * dvm / (dvp + dvm) : R(0));
  } else if constexpr (LIM == LIM_MINMOD) {
    return (dvp * dvm > R(0) ? (rabs(dvp) < rabs(dvm) ? dvp : dvm) : R(0));
  } else if constexpr (LIM == LIM_VANALBADA) {
    if (dvp * dvm > R(0)) {
      R dpp = dvp * dvp, dmm = dvm * dvm;
      return (dvp * (dmm + R(1.e-18)) + dvm * (dpp + R(1.e-18))) / (dpp + dmm + R(1.e-18));
    }
    return R(0);
  } else if constexpr (LIM == LIM_OSPRE) {
    return (dvp * dvm > R(0)
                ? R(1.5) * dvp * dvm * (dvm + dvp) / (dvp * dvp + dvm * dvm + dvp * dvm)
                : R(0));
  } else if constexpr (LIM == LIM_UMIST) {
    if (dvp * dvm > R(0)) {
      R ddp = R(0.25) * (dvp + R(3) * dvm), ddm = R(0.25) * (dvm + R(3) * dvp);
      R d2 = R(2) * (rabs(dvp) < rabs(dvm) ? dvp : dvm);
      d2 = rabs(d2) < rabs(ddp) ? d2 : ddp;
      return rabs(d2) < rabs(ddm) ? d2 : ddm;
    }
    return R(0);
  } else {
    return R(0);
  }
}

// Src/macros.hpp:200
template <typename R>
__device__ __forceinline__ R minmod(R a, R b) {
  return (a * b > R(0) ? (rabs(a) < rabs(b) ? a : b) : R(0));
}

// MP5 edge value of Suresh & Huynh (1997) (Src/States/states.hpp:32-98,
// MP5_ALPHA 4, reconstruction from cell averages).  The stencil is ordered
// towards the edge: F0 the cell, Fp and Fpp the next cells on the edge's
// side, Fm and Fmm the cells on the other side.
template <typename R>
__device__ __forceinline__ R mp5_edge(R Fmm, R Fm, R F0, R Fp, R Fpp) {
  const R alpha = R(4), epsm = R(1.e-12);
  const R dFp = Fp - F0, dFm = F0 - Fm;
  R f = R(2) * Fmm - R(13) * Fm + R(47) * F0 + R(27) * Fp - R(3) * Fpp;  // Eq. (2.1)
  f /= R(60);
  const R fMP = F0 + minmod(dFp, alpha * dFm);                          // Eq. (2.12)
  if ((f - F0) * (f - fMP) <= epsm) return f;
  const R d2m = Fmm + F0 - R(2) * Fm;
  const R d2 = Fm + Fp - R(2) * F0;
  const R d2p = F0 + Fpp - R(2) * Fp;
  R s1 = minmod(R(4) * d2 - d2p, R(4) * d2p - d2);
  R s2 = minmod(d2, d2p);
  const R dMMp = minmod(s1, s2);                                       // Eq. (2.27)
  s1 = minmod(R(4) * d2m - d2, R(4) * d2 - d2m);
  s2 = minmod(d2, d2m);
  const R dMMm = minmod(s1, s2);
  const R fUL = F0 + alpha * dFm;                                      // Eq. (2.8)
  const R fAV = R(0.5) * (F0 + Fp);                                    // Eq. (2.16)
  const R fMD = fAV - R(0.5) * dMMp;                                   // Eq. (2.28)
  const R fLC = R(0.5) * (R(3) * F0 - Fm) + R(4.0 / 3.0) * dMMm;       // Eq. (2.29)
  s1 = GP_MIN(F0, Fp);
  s1 = GP_MIN(s1, fMD);
  s2 = GP_MIN(F0, fUL);
  s2 = GP_MIN(s2, fLC);
  const R fmin = GP_MAX(s1, s2);                                       // Eq. (2.24a)
  s1 = GP_MAX(F0, Fp);
  s1 = GP_MAX(s1, fMD);
  s2 = GP_MAX(F0, fUL);
  s2 = GP_MAX(s2, fLC);
  const R fmax = GP_MIN(s1, s2);                                       // Eq. (2.24b)
  return f + minmod(fmin - f, fmax - f);                               // Eq. (2.26)
}

// WENO-Z edge value of Borges et al. (2008), the 3rd-order-weights form of
// Src/States/states.hpp:108-166 (no HIGH_ORDER), stencil ordered towards
// the edge as for mp5_edge.  The smoothness floor is 1e-40 in FP64; in the
// mixed form's flushed FP32 it would vanish, so FP32 uses 1e-30.
template <typename R>
__device__ __forceinline__ R wenoz_edge(R Fmm, R Fm, R F0, R Fp, R Fpp) {
  const R c13_12 = R(13.0 / 12.0);
  const R eps = sizeof(R) == 8 ? R(1.e-40) : R(1.e-30);
  R a0 = Fmm - R(2) * Fm + F0;
  R a1 = Fmm - R(4) * Fm + R(3) * F0;
  const R b0 = c13_12 * a0 * a0 + R(0.25) * a1 * a1;
  a0 = Fm - R(2) * F0 + Fp;
  a1 = Fm - Fp;
  const R b1 = c13_12 * a0 * a0 + R(0.25) * a1 * a1;
  a0 = F0 - R(2) * Fp + Fpp;
  a1 = R(3) * F0 - R(4) * Fp + Fpp;
  const R b2 = c13_12 * a0 * a0 + R(0.25) * a1 * a1;
  const R t5 = rabs(b0 - b2);
  a0 = R(1) * (R(1) + t5 / (b0 + eps));
  a1 = R(6) * (R(1) + t5 / (b1 + eps));
  const R a2 = R(3) * (R(1) + t5 / (b2 + eps));
  const R sum_a = R(1) / (a0 + a1 + a2);
  const R w0 = a0 * sum_a, w1 = a1 * sum_a, w2 = a2 * sum_a;
  const R f0 = R(2) * Fmm - R(7) * Fm + R(11) * F0;
  const R f1 = -Fm + R(5) * F0 + R(2) * Fp;
  const R f2 = R(2) * F0 + R(5) * Fp - Fpp;
  return (w0 * f0 + w1 * f1 + w2 * f2) / R(6);
}

// 3-point edge values on a uniform grid of cell width dx, stencil ordered
// towards the edge (Fm the cell away from it, F0 the cell, Fp the cell
// across it).  WENO3: the "improved" weights of Yamaleev & Carpenter (2009),
// Src/States/states.hpp:178-226 without HIGH_ORDER.
template <typename R>
__device__ __forceinline__ R weno3_edge(R Fm, R F0, R Fp, R dx) {
  const R dx2 = dx * dx;
  R b0 = Fp - F0, b1 = Fm - F0;
  b0 = b0 * b0;
  b1 = b1 * b1;
  R tau = Fp - R(2) * F0 + Fm;
  tau = tau * tau;
  const R a0 = R(2) * (R(1) + tau / (dx2 + b0));
  const R a1 = R(1) * (R(1) + tau / (dx2 + b1));
  const R w0 = a0 / (a0 + a1), w1 = a1 / (a0 + a1);
  const R f0 = R(0.5) * (Fp + F0), f1 = R(0.5) * (-Fm + R(3) * F0);
  return w0 * f0 + w1 * f1;
}

// LimO3: the third-order limiter of Cada & Torrilhon (2009), Eq. 3.22, as
// Src/States/states.hpp:239-281 (r = 0.1, blending width 1e-12).
template <typename R>
__device__ __forceinline__ R limo3_edge(R Fm, R F0, R Fp, R dx) {
  const R r = R(0.1), eps = R(1.e-12);
  const R dvp = Fp - F0, dvm = F0 - Fm;
  const R sp = dvp >= R(0) ? R(1) : R(-1);
  const R advp = rabs(dvp), dvm1 = sp * dvm;
  const R q = (R(2) * dvp + dvm) / R(3);
  const R q1 = (R(2) * rabs(dvp) + sp * dvm) / R(3);
  R a = GP_MIN(R(1.5) * advp, R(2) * dvm1);
  a = GP_MIN(q1, a);
  const R b = GP_MAX(R(-0.5) * dvm1, a);
  const R c = GP_MIN(q1, b);
  R psi = sp * GP_MAX(R(0), c);
  R eta = r * dx;
  eta = (dvm * dvm + dvp * dvp) / (eta * eta);
  R lim;
  if (eta <= R(1) - eps) {
    lim = q;
  } else if (eta >= R(1) + eps) {
    lim = psi;
  } else {
    psi = (R(1) - (eta - R(1)) / eps) * q + (R(1) + (eta - R(1)) / eps) * psi;
    lim = R(0.5) * psi;
  }
  return F0 + R(0.5) * lim;
}

template <int LIM, typename R>
__device__ __forceinline__ R edge3(R Fm, R F0, R Fp, R dx) {
  if constexpr (LIM == LIM_LIMO3) return limo3_edge(Fm, F0, Fp, dx);
  else return weno3_edge(Fm, F0, Fp, dx);
}

// The 5-point edge value of the scheme (MP5 or WENO-Z).
template <int LIM, typename R>
__device__ __forceinline__ R edge5(R Fmm, R Fm, R F0, R Fp, R Fpp) {
  if constexpr (LIM == LIM_WENOZ) return wenoz_edge(Fmm, Fm, F0, Fp, Fpp);
  else return mp5_edge(Fmm, Fm, F0, Fp, Fpp);
}

// PPM constrained face value between cells q0 and qp (stencil qm, q0, qp,
// qpp): the uniform-grid 4-point value of
// Src/States/reconstruction_geometry.hpp:97-101, limited to lie between the
// adjacent cell values (Src/States/ppm_states.cpp:139-145).  The reference
// evaluates it once as the right face of cell q0 and once as the left face
// of cell qp; both are this same expression, so it is computed once here.
template <typename R>
__device__ __forceinline__ R ppm_face(R qm, R q0, R qp, R qpp) {
  R f = (-qm + R(7) * (q0 + qp) - qpp) / R(12);
  return q0 + minmod(f - q0, qp - q0);
}

// Parabolic limiter of a cell with constrained face values fm (left) and fp
// (right): Src/States/ppm_states.cpp:147-163.  Returns the increments.
template <typename R>
__device__ __forceinline__ void ppm_cell(R v, R fm, R fp, R& dvp, R& dvm) {
  dvp = fp - v;
  dvm = fm - v;
  if (dvp * dvm >= R(0)) {
    dvp = R(0);
    dvm = R(0);
  } else {
    if (rabs(dvp) >= R(2) * rabs(dvm)) dvp = -R(2) * dvm;
    else if (rabs(dvm) >= R(2) * rabs(dvp)) dvm = -R(2) * dvp;
  }
}

// 3-point parabolic reconstruction of the UCT edge data with PPM
// (Src/array_reconstruct.cpp:208-270, uniform grid): increments of cell q0
// to its right (dqp) and left (dqm) faces.
template <typename R>
__device__ __forceinline__ void par3_cell(R qm, R q0, R qp, R& dqp, R& dqm) {
  R fp = (-qm + R(5) * q0 + R(2) * qp) / R(6);
  R fm = (R(2) * qm + R(5) * q0 - qp) / R(6);
  dqp = fp - q0;
  dqm = fm - q0;
  R dq = qp - q0;
  fp = q0 + minmod(dqp, dq);
  dq = q0 - qm;
  fm = q0 + minmod(dqm, -dq);
  dqp = fp - q0;
  dqm = fm - q0;
  if (dqp * dqm >= R(0)) {
    dqp = R(0);
    dqm = R(0);
  } else {
    if (rabs(dqp) >= R(2) * rabs(dqm)) dqp = -R(2) * dqm;
    else if (rabs(dqm) >= R(2) * rabs(dqp)) dqm = -R(2) * dqp;
  }
}

// ---------------------------------------------------------------------
// Ideal MHD
// ---------------------------------------------------------------------

// Src/MHD/mhd.hpp:906-948
template <typename R>
__device__ __forceinline__ void mhd_prim2cons(const R* v, R* u, R gmm1) {
  u[RHO] = v[RHO];
  u[MX1] = v[RHO] * v[VX1];
  u[MX2] = v[RHO] * v[VX1 + 1];
  u[MX3] = v[RHO] * v[VX1 + 2];
  u[BX1] = v[BX1];
  u[BX2] = v[BX2];
  u[BX3] = v[BX3];
  R kinb2 = v[VX1] * v[VX1] + v[VX1 + 1] * v[VX1 + 1] + v[VX1 + 2] * v[VX1 + 2];
  kinb2 = v[RHO] * kinb2 + v[BX1] * v[BX1] + v[BX2] * v[BX2] + v[BX3] * v[BX3];
  kinb2 *= R(0.5);
  u[7] = kinb2 + v[7] / gmm1;
}

// Src/MHD/mappers.cpp:32-150 (ENERGY_SOLVE); always FP64.
__device__ __forceinline__ uint32_t mhd_cons2prim(double* u, double* v, double gamma,
                                                  double small_rho, double small_prs) {
  uint32_t err = 0;
  double gmm1 = gamma - 1.0;
  if (u[RHO] < 0.0) {
    u[RHO] = small_rho;
    err |= ERR_NEGATIVE_RHO | ERR_CONS2PRIM_FAIL;
  }
  v[RHO] = u[RHO];
  double tau = 1.0 / u[RHO];
  v[VX1] = u[MX1] * tau;
  v[VX1 + 1] = u[MX2] * tau;
  v[VX1 + 2] = u[MX3] * tau;
  v[BX1] = u[BX1];
  v[BX2] = u[BX2];
  v[BX3] = u[BX3];
  double m2 = u[MX1] * u[MX1] + u[MX2] * u[MX2] + u[MX3] * u[MX3];
  double b2 = u[BX1] * u[BX1] + u[BX2] * u[BX2] + u[BX3] * u[BX3];
  double kinb2 = 0.5 * (m2 * tau + b2);
  if (u[7] > 0.0) {
    v[7] = gmm1 * (u[7] - kinb2);
    if (v[7] < 0.0) {
      v[7] = small_prs;
      u[7] = v[7] / gmm1 + kinb2;
      err |= ERR_NEGATIVE_PRS;
    }
  } else {
    u[7] = small_prs / gmm1 + kinb2;
    v[7] = small_prs;
    err |= ERR_NEGATIVE_ENG;
  }
  return err;
}

// Src/MHD/mhd.hpp:163-223 (no background field, no GLM)
template <int DIR, typename R>
__device__ __forceinline__ void mhd_flux(const R* v, const R* u, R* f, R& pt) {
  constexpr int VXn = VX1 + DIR, BXn = BX1 + DIR, MXn = MX1 + DIR;
  R vB = v[VX1] * v[BX1] + v[VX1 + 1] * v[BX2] + v[VX1 + 2] * v[BX3];
  pt = v[7] + R(0.5) * (v[BX1] * v[BX1] + v[BX2] * v[BX2] + v[BX3] * v[BX3]);
  f[RHO] = u[MXn];
  f[MX1] = u[MX1] * v[VXn] - v[BX1] * v[BXn];
  f[MX2] = u[MX2] * v[VXn] - v[BX2] * v[BXn];
  f[MX3] = u[MX3] * v[VXn] - v[BX3] * v[BXn];
  f[BX1] = v[BX1] * v[VXn] - v[BXn] * v[VX1];
  f[BX2] = v[BX2] * v[VXn] - v[BXn] * v[VX1 + 1];
  f[BX3] = v[BX3] * v[VXn] - v[BXn] * v[VX1 + 2];
  f[7] = (u[7] + pt) * v[VXn] - v[BXn] * vB;
  f[MXn] += pt;
}

// Total pressure of mhd_flux (the same expression, so the same value)
template <typename R>
__device__ __forceinline__ R mhd_ptot(const R* v) {
  return v[7] + R(0.5) * (v[BX1] * v[BX1] + v[BX2] * v[BX2] + v[BX3] * v[BX3]);
}

// Src/MHD/mhd.hpp:241-277 with a^2 = gamma p/rho (Src/eos.hpp:96)
template <int DIR, typename R>
__device__ __forceinline__ void mhd_signal_speed(const R* v, R a2, R& cmin, R& cmax) {
  constexpr int VXn = VX1 + DIR;
  R b1 = v[BX1 + DIR], b2 = v[BX1 + (DIR + 1) % 3], b3 = v[BX1 + (DIR + 2) % 3];
  R gpr = a2 * v[RHO];
  R Btmag2 = b2 * b2 + b3 * b3;
  R Bmag2 = b1 * b1 + Btmag2;
  R cf = gpr - Bmag2;
  cf = gpr + Bmag2 + rsqrt_(cf * cf + R(4) * gpr * Btmag2);
  cf = rsqrt_(R(0.5) * cf / v[RHO]);
  cmax = v[VXn] + cf;
  cmin = v[VXn] - cf;
}

// Face data stored for the upwind-CT EMF (Src/MHD/CT/ct_store.hpp):
// eb = emf->e[DIRb][DIR], et = emf->e[DIRt][DIR], and the UCT weights.
template <typename R>
struct CTFace {
  R eb, et, aL, aR, dL, dR;
};

// Src/MHD/CT/ct_store.hpp:154-177
template <int DIR, typename R>
__device__ __forceinline__ void ct_store_ucthll(const R* vl, const R* vr, R Sl, R Sr,
                                                CTFace<R>& c) {
  constexpr int VXt = VX1 + (DIR + 1) % 3, VXb = VX1 + (DIR + 2) % 3;
  R aR_1 = GP_MAX(R(0), Sr);
  R aL_1 = GP_MIN(R(0), Sl);
  R scrh = R(1) / (aR_1 - aL_1);
  c.eb = (aR_1 * vl[VXt] - aL_1 * vr[VXt]) * scrh;
  c.et = -(aR_1 * vl[VXb] - aL_1 * vr[VXb]) * scrh;
  c.aL = aR_1 * scrh;
  c.aR = -aL_1 * scrh;
  c.dR = -aL_1 * aR_1 * scrh;
  c.dL = -aL_1 * aR_1 * scrh;
}

// Src/MHD/CT/ct_store.hpp:252-355 (ideal EOS)
template <int DIR, typename R>
__device__ __forceinline__ void ct_store_ucthlld(const R* ul, const R* ur, const R* vl,
                                                 const R* vr, R Sl, R Sr, R Bn,
                                                 CTFace<R>& c) {
  constexpr int VXn = VX1 + DIR, VXt = VX1 + (DIR + 1) % 3, VXb = VX1 + (DIR + 2) % 3;
  constexpr int MXn = MX1 + DIR;
  int switch_to_hll = 0;
  R aR_1 = GP_MAX(R(0), Sr);
  R aL_1 = GP_MIN(R(0), Sl);
  R dul = Sl - vl[VXn];
  R dur = Sr - vr[VXn];
  R pL = vl[7] + R(0.5) * (vl[BX1] * vl[BX1] + vl[BX2] * vl[BX2] + vl[BX3] * vl[BX3]);
  R pR = vr[7] + R(0.5) * (vr[BX1] * vr[BX1] + vr[BX2] * vr[BX2] + vr[BX3] * vr[BX3]);
  R scrh = R(1) / (dur * ur[RHO] - dul * ul[RHO]);
  R Sc = (dur * ur[MXn] - dul * ul[MXn] - pR + pL) * scrh;
  R usl_RHO = ul[RHO] * dul / (Sl - Sc);
  R usr_RHO = ur[RHO] * dur / (Sr - Sc);
  if (usl_RHO < R(0) || usr_RHO < R(0)) switch_to_hll = 1;
  R sqrL = rsqrt_(usl_RHO);
  R sqrR = rsqrt_(usr_RHO);
  R Sal = Sc - rabs(Bn) / sqrL;
  R Sar = Sc + rabs(Bn) / sqrR;
  R chiL = (vl[VXn] - Sc) * (Sl - Sc) / (Sal + Sl - R(2) * Sc);
  R chiR = (vr[VXn] - Sc) * (Sr - Sc) / (Sar + Sr - R(2) * Sc);
  R nuL = (Sal + Sl) / (rabs(Sal) + rabs(Sl));
  R nuR = (Sar + Sr) / (rabs(Sar) + rabs(Sr));
  R nuLR = (Sal + Sar) / (rabs(Sal) + rabs(Sar));
  if (rabs(Sar - Sal) > R(1.e-9) * rabs(Sr - Sl)) {
    c.dL = R(0.5) * (chiL * nuL - chiL * nuLR) + R(0.5) * (rabs(Sal) - nuLR * Sal);
    c.dR = R(0.5) * (chiR * nuR - chiR * nuLR) + R(0.5) * (rabs(Sar) - nuLR * Sar);
    c.aL = R(0.5) * (R(1) + nuLR);
    c.aR = R(0.5) * (R(1) - nuLR);
  } else {
    c.dL = R(0.5) * chiL * nuL + R(0.5) * rabs(Sal);
    c.dR = R(0.5) * chiR * nuR + R(0.5) * rabs(Sar);
    c.aL = R(0.5);
    c.aR = R(0.5);
  }
  scrh = R(1) / (aR_1 - aL_1);
  if (switch_to_hll) {
    c.aL = aR_1 * scrh;
    c.aR = -aL_1 * scrh;
    c.dR = -aL_1 * aR_1 * scrh;
    c.dL = -aL_1 * aR_1 * scrh;
  }
  c.eb = (aR_1 * vl[VXt] - aL_1 * vr[VXt]) * scrh;
  c.et = -(aR_1 * vl[VXb] - aL_1 * vr[VXb]) * scrh;
}

// HLLD solver, Src/MHD/hlld.cpp:61-514 (ideal EOS).  vl/vr are the
// reconstructed primitive states at the interface (normal field already set
// to the face value).  Returns cmax = max(|Sl|,|Sr|).
template <int DIR, int CT, typename R>
__device__ __forceinline__ R mhd_hlld(const R* vl, const R* vr, R* flux, R gamma, R Bn,
                                      CTFace<R>& ct) {
  constexpr int VXn = VX1 + DIR, VXt = VX1 + (DIR + 1) % 3, VXb = VX1 + (DIR + 2) % 3;
  constexpr int MXn = MX1 + DIR, MXt = MX1 + (DIR + 1) % 3, MXb = MX1 + (DIR + 2) % 3;
  constexpr int BXn = BX1 + DIR, BXt = BX1 + (DIR + 1) % 3, BXb = BX1 + (DIR + 2) % 3;
  R ul[8], ur[8], usl[8], usr[8];
  R Sl, Sr, ptl, ptr;
  const R gmm1 = gamma - R(1);
  mhd_prim2cons(vl, ul, gmm1);
  mhd_prim2cons(vr, ur, gmm1);
  R a2L = gamma * vl[7] / vl[RHO];
  R a2R = gamma * vr[7] / vr[RHO];
  {
    R sl_min, sl_max, sr_min, sr_max;  // Src/MHD/mhd.hpp:295-308
    mhd_signal_speed<DIR>(vl, a2L, sl_min, sl_max);
    mhd_signal_speed<DIR>(vr, a2R, sr_min, sr_max);
    Sl = GP_MIN(sl_min, sr_min);
    Sr = GP_MAX(sl_max, sr_max);
  }
  R cmax = GP_MAX(rabs(Sl), rabs(Sr));
  // The physical fluxes are formed where a region's flux uses them (one
  // side outside the HLL fallback), so they are not live across the star
  // states; every value is the one the reference computes up front.
  ptl = mhd_ptot(vl);
  ptr = mhd_ptot(vr);

  R dul, dur, Bx, Bx1, sBx, pts, SM;
  {
    R scrh = R(1) / (Sr - Sl);
    Bx1 = Bx = (Sr * vr[BXn] - Sl * vl[BXn]) * scrh;
    sBx = (Bx > R(0) ? R(1) : R(-1));
    dul = Sl - vl[VXn];
    dur = Sr - vr[VXn];
    scrh = R(1) / (dur * ur[RHO] - dul * ul[RHO]);
    SM = (dur * ur[MXn] - dul * ul[MXn] - ptr + ptl) * scrh;
    pts = dur * ur[RHO] * ptl - dul * ul[RHO] * ptr +
          vl[RHO] * vr[RHO] * dur * dul * (vr[VXn] - vl[VXn]);
    pts *= scrh;
  }
  usl[RHO] = ul[RHO] * dul / (Sl - SM);
  usr[RHO] = ur[RHO] * dur / (Sr - SM);
  int switch_to_hll = (usl[RHO] < R(0) || usr[RHO] < R(0));
  R sqrL = rsqrt_(usl[RHO]);
  R sqrR = rsqrt_(usr[RHO]);
  R S1L = SM - rabs(Bx) / sqrL;
  R S1R = SM + rabs(Bx) / sqrR;

  R pt_;
  if (Sl >= R(0)) {
    mhd_flux<DIR>(vl, ul, flux, pt_);
  } else if (Sr <= R(0)) {
    mhd_flux<DIR>(vr, ur, flux, pt_);
  } else if (!switch_to_hll) {
    int switch_to_hllc = 0;
    if ((S1L - Sl) < R(1.e-4) * (SM - Sl)) switch_to_hllc = 1;
    if ((S1R - Sr) > -R(1.e-4) * (Sr - SM)) switch_to_hllc = 1;
    R scrhL, scrhR;
    if (!switch_to_hllc) {
      scrhL = (ul[RHO] * dul * dul - Bx * Bx) / (ul[RHO] * dul * (Sl - SM) - Bx * Bx);
      scrhR = (ur[RHO] * dur * dur - Bx * Bx) / (ur[RHO] * dur * (Sr - SM) - Bx * Bx);
      usl[BXn] = Bx1;
      usl[BXt] = ul[BXt] * scrhL;
      usl[BXb] = ul[BXb] * scrhL;
      usr[BXn] = Bx1;
      usr[BXt] = ur[BXt] * scrhR;
      usr[BXb] = ur[BXb] * scrhR;
    } else {
      R scrh = R(1) / (Sr - Sl);
      // mhd_flux's transverse induction components
      const R flt = vl[BXt] * vl[VXn] - vl[BXn] * vl[VXt];
      const R frt = vr[BXt] * vr[VXn] - vr[BXn] * vr[VXt];
      const R flb = vl[BXb] * vl[VXn] - vl[BXn] * vl[VXb];
      const R frb = vr[BXb] * vr[VXn] - vr[BXn] * vr[VXb];
      R Ut = (Sr * ur[BXt] - Sl * ul[BXt] + flt - frt) * scrh;
      R Ub = (Sr * ur[BXb] - Sl * ul[BXb] + flb - frb) * scrh;
      usl[BXn] = usr[BXn] = Bx1;
      usl[BXt] = usr[BXt] = Ut;
      usl[BXb] = usr[BXb] = Ub;
      S1L = S1R = SM;
    }
    scrhL = Bx / (ul[RHO] * dul);
    scrhR = Bx / (ur[RHO] * dur);
    R vsL = vl[VXt] - scrhL * (usl[BXt] - ul[BXt]);
    R vsR = vr[VXt] - scrhR * (usr[BXt] - ur[BXt]);
    R wsL = vl[VXb] - scrhL * (usl[BXb] - ul[BXb]);
    R wsR = vr[VXb] - scrhR * (usr[BXb] - ur[BXb]);
    usl[MXn] = usl[RHO] * SM;
    usr[MXn] = usr[RHO] * SM;
    usl[MXt] = usl[RHO] * vsL;
    usr[MXt] = usr[RHO] * vsR;
    usl[MXb] = usl[RHO] * wsL;
    usr[MXb] = usr[RHO] * wsR;
    scrhL = vl[VXn] * Bx1 + vl[VXt] * ul[BXt] + vl[VXb] * ul[BXb];
    scrhL -= SM * Bx1 + vsL * usl[BXt] + wsL * usl[BXb];
    usl[7] = dul * ul[7] - ptl * vl[VXn] + pts * SM + Bx * scrhL;
    usl[7] /= Sl - SM;
    scrhR = vr[VXn] * Bx1 + vr[VXt] * ur[BXt] + vr[VXb] * ur[BXb];
    scrhR -= SM * Bx1 + vsR * usr[BXt] + wsR * usr[BXb];
    usr[7] = dur * ur[7] - ptr * vr[VXn] + pts * SM + Bx * scrhR;
    usr[7] /= Sr - SM;

    if (S1L >= R(0)) {
      R fl[8];
      mhd_flux<DIR>(vl, ul, fl, pt_);
#pragma unroll
      for (int nv = 0; nv < 8; nv++) flux[nv] = fl[nv] + Sl * (usl[nv] - ul[nv]);
    } else if (S1R <= R(0)) {
      R fr[8];
      mhd_flux<DIR>(vr, ur, fr, pt_);
#pragma unroll
      for (int nv = 0; nv < 8; nv++) flux[nv] = fr[nv] + Sr * (usr[nv] - ur[nv]);
    } else {
      R ussl[8], ussr[8];
      ussl[RHO] = usl[RHO];
      ussr[RHO] = usr[RHO];
      R vss = sqrL * vsL + sqrR * vsR + (usr[BXt] - usl[BXt]) * sBx;
      vss /= sqrL + sqrR;
      R wss = sqrL * wsL + sqrR * wsR + (usr[BXb] - usl[BXb]) * sBx;
      wss /= sqrL + sqrR;
      ussl[MXn] = ussl[RHO] * SM;
      ussr[MXn] = ussr[RHO] * SM;
      ussl[MXt] = ussl[RHO] * vss;
      ussr[MXt] = ussr[RHO] * vss;
      ussl[MXb] = ussl[RHO] * wss;
      ussr[MXb] = ussr[RHO] * wss;
      ussl[BXn] = ussr[BXn] = Bx1;
      ussl[BXt] = sqrL * usr[BXt] + sqrR * usl[BXt] + sqrL * sqrR * (vsR - vsL) * sBx;
      ussl[BXt] /= sqrL + sqrR;
      ussr[BXt] = ussl[BXt];
      ussl[BXb] = sqrL * usr[BXb] + sqrR * usl[BXb] + sqrL * sqrR * (wsR - wsL) * sBx;
      ussl[BXb] /= sqrL + sqrR;
      ussr[BXb] = ussl[BXb];
      scrhL = SM * Bx1 + vsL * usl[BXt] + wsL * usl[BXb];
      scrhL -= SM * Bx1 + vss * ussl[BXt] + wss * ussl[BXb];
      scrhR = SM * Bx1 + vsR * usr[BXt] + wsR * usr[BXb];
      scrhR -= SM * Bx1 + vss * ussr[BXt] + wss * ussr[BXb];
      ussl[7] = usl[7] - sqrL * scrhL * sBx;
      ussr[7] = usr[7] + sqrR * scrhR * sBx;
      if (SM >= R(0)) {
        R fl[8];
        mhd_flux<DIR>(vl, ul, fl, pt_);
#pragma unroll
        for (int nv = 0; nv < 8; nv++)
          flux[nv] = fl[nv] + S1L * (ussl[nv] - usl[nv]) + Sl * (usl[nv] - ul[nv]);
      } else {
        R fr[8];
        mhd_flux<DIR>(vr, ur, fr, pt_);
#pragma unroll
        for (int nv = 0; nv < 8; nv++)
          flux[nv] = fr[nv] + S1R * (ussr[nv] - usr[nv]) + Sr * (usr[nv] - ur[nv]);
      }
    }
  } else {
    R fl[8], fr[8];
    mhd_flux<DIR>(vl, ul, fl, pt_);
    mhd_flux<DIR>(vr, ur, fr, pt_);
    R scrh = R(1) / (Sr - Sl);
#pragma unroll
    for (int nv = 0; nv < 8; nv++) {
      flux[nv] = Sl * Sr * (ur[nv] - ul[nv]) + Sr * fl[nv] - Sl * fr[nv];
      flux[nv] *= scrh;
    }
  }
  if constexpr (CT == CT_UCT_HLLD)
    ct_store_ucthlld<DIR>(ul, ur, vl, vr, Sl, Sr, Bn, ct);
  else
    ct_store_ucthll<DIR>(vl, vr, Sl, Sr, ct);
  return cmax;
}

// HLL solver for MHD, Src/MHD/hll.cpp:50-220 (always UCT_HLL face data)
template <int DIR, typename R>
__device__ __forceinline__ R mhd_hll(const R* vl, const R* vr, R* flux, R gamma,
                                     CTFace<R>& ct) {
  R ul[8], ur[8], fl[8], fr[8], Sl, Sr, pl, pr;
  const R gmm1 = gamma - R(1);
  mhd_prim2cons(vl, ul, gmm1);
  mhd_prim2cons(vr, ur, gmm1);
  R a2L = gamma * vl[7] / vl[RHO];
  R a2R = gamma * vr[7] / vr[RHO];
  {
    R sl_min, sl_max, sr_min, sr_max;
    mhd_signal_speed<DIR>(vl, a2L, sl_min, sl_max);
    mhd_signal_speed<DIR>(vr, a2R, sr_min, sr_max);
    Sl = GP_MIN(sl_min, sr_min);
    Sr = GP_MAX(sl_max, sr_max);
  }
  R bL = GP_MIN(Sl, R(0));
  R bR = GP_MAX(R(0), Sr);
  R cmax = GP_MAX(rabs(Sl), rabs(Sr));
  mhd_flux<DIR>(vl, ul, fl, pl);
  mhd_flux<DIR>(vr, ur, fr, pr);
  R scrh = R(1) / (bR - bL);
#pragma unroll
  for (int nv = 0; nv < 8; nv++) {
    flux[nv] = bL * bR * (ur[nv] - ul[nv]) + bR * fl[nv] - bL * fr[nv];
    flux[nv] *= scrh;
  }
  ct_store_ucthll<DIR>(vl, vr, Sl, Sr, ct);
  return cmax;
}

// HLLC solver for MHD, Src/MHD/hllc.cpp:52-363: one intermediate state on
// each side of the contact, built from the HLL average (no HLL switch
// without multi-D shock flattening); UCT_HLL face data (the caller replaces
// them by the induction fluxes for CT_EMF_AVERAGE ARITHMETIC).
template <int DIR, typename R>
__device__ __forceinline__ R mhd_hllc(const R* vl, const R* vr, R* flux, R gamma,
                                      CTFace<R>& ct) {
  constexpr int VXn = VX1 + DIR;
  constexpr int MXn = MX1 + DIR, MXt = MX1 + (DIR + 1) % 3, MXb = MX1 + (DIR + 2) % 3;
  constexpr int BXn = BX1 + DIR, BXt = BX1 + (DIR + 1) % 3, BXb = BX1 + (DIR + 2) % 3;
  R ul[8], ur[8], fl[8], fr[8], Sl, Sr, pl, pr;
  const R gmm1 = gamma - R(1);
  mhd_prim2cons(vl, ul, gmm1);
  mhd_prim2cons(vr, ur, gmm1);
  R a2L = gamma * vl[7] / vl[RHO];
  R a2R = gamma * vr[7] / vr[RHO];
  {
    R sl_min, sl_max, sr_min, sr_max;
    mhd_signal_speed<DIR>(vl, a2L, sl_min, sl_max);
    mhd_signal_speed<DIR>(vr, a2R, sr_min, sr_max);
    Sl = GP_MIN(sl_min, sr_min);
    Sr = GP_MAX(sl_max, sr_max);
  }
  R cmax = GP_MAX(rabs(Sl), rabs(Sr));
  mhd_flux<DIR>(vl, ul, fl, pl);
  mhd_flux<DIR>(vr, ur, fr, pr);
  if (Sl >= R(0)) {
#pragma unroll
    for (int nv = 0; nv < 8; nv++) flux[nv] = fl[nv];
  } else if (Sr <= R(0)) {
#pragma unroll
    for (int nv = 0; nv < 8; nv++) flux[nv] = fr[nv];
  } else {
    R Uhll[8], Fhll[8], us[8];
    const R scrh = R(1) / (Sr - Sl);
#pragma unroll
    for (int nv = 0; nv < 8; nv++) {
      Uhll[nv] = Sr * ur[nv] - Sl * ul[nv] + fl[nv] - fr[nv];
      Uhll[nv] *= scrh;
      Fhll[nv] = Sl * Sr * (ur[nv] - ul[nv]) + Sr * fl[nv] - Sl * fr[nv];
      Fhll[nv] *= scrh;
    }
    const R Bxs = Uhll[BXn], Bys = Uhll[BXt], Bzs = Uhll[BXb];
    const R vxs = Uhll[MXn] / Uhll[RHO];
    // only the state on the side of the contact the face sees is built
    const bool left = vxs > R(0);
    const R* v = left ? vl : vr;
    const R* u = left ? ul : ur;
    const R* f = left ? fl : fr;
    const R S = left ? Sl : Sr;
    const R p = left ? pl : pr;
    const R vx = v[VXn];
    R vB = v[VX1] * v[BX1] + v[VX1 + 1] * v[BX2] + v[VX1 + 2] * v[BX3];
    R vBs = Uhll[BX1] * Uhll[MX1] + Uhll[BX2] * Uhll[MX2] + Uhll[BX3] * Uhll[MX3];
    vBs /= Uhll[RHO];
    us[RHO] = u[RHO] * (S - vx) / (S - vxs);
    const R ps = Fhll[MXn] + Bxs * Bxs - Fhll[RHO] * vxs;
    us[7] = (u[7] * (S - vx) + ps * vxs - p * vx - Bxs * vBs + v[BXn] * vB) / (S - vxs);
    us[MXn] = us[RHO] * vxs;
    us[MXt] = (u[MXt] * (S - vx) - (Bxs * Bys - v[BXn] * v[BXt])) / (S - vxs);
    us[MXb] = (u[MXb] * (S - vx) - (Bxs * Bzs - v[BXn] * v[BXb])) / (S - vxs);
    us[BXn] = Bxs;
    us[BXt] = Bys;
    us[BXb] = Bzs;
#pragma unroll
    for (int nv = 0; nv < 8; nv++) flux[nv] = f[nv] + S * (us[nv] - u[nv]);
  }
  ct_store_ucthll<DIR>(vl, vr, Sl, Sr, ct);
  return cmax;
}

// Lax-Friedrichs (Rusanov) flux for MHD, Src/MHD/tvdlf.cpp:60-244: the
// signal speed of the arithmetic average state; UCT_HLL face data with
// Sl = -cmax, Sr = cmax.
template <int DIR, typename R>
__device__ __forceinline__ R mhd_tvdlf(const R* vl, const R* vr, R* flux, R gamma,
                                       CTFace<R>& ct) {
  R ul[8], ur[8], fl[8], fr[8], vLR[8], pl, pr, cmax;
  const R gmm1 = gamma - R(1);
  mhd_prim2cons(vl, ul, gmm1);
  mhd_prim2cons(vr, ur, gmm1);
#pragma unroll
  for (int nv = 0; nv < 8; nv++) vLR[nv] = R(0.5) * (vl[nv] + vr[nv]);
  {
    R cminLR, cmaxLR;
    mhd_signal_speed<DIR>(vLR, gamma * vLR[7] / vLR[RHO], cminLR, cmaxLR);
    cmax = GP_MAX(rabs(cminLR), rabs(cmaxLR));
  }
  mhd_flux<DIR>(vl, ul, fl, pl);
  mhd_flux<DIR>(vr, ur, fr, pr);
#pragma unroll
  for (int nv = 0; nv < 8; nv++)
    flux[nv] = R(0.5) * (fl[nv] + fr[nv]) - R(0.5) * cmax * (ur[nv] - ul[nv]);
  ct_store_ucthll<DIR>(vl, vr, -cmax, cmax, ct);
  return cmax;
}

// ---------------------------------------------------------------------
// Hydrodynamics (NVAR = 5: RHO, MX1..3, ENG)
// ---------------------------------------------------------------------

// Src/HD/hd.hpp:392-416
template <typename R>
__device__ __forceinline__ void hd_prim2cons(const R* v, R* u, R gamma) {
  u[RHO] = v[RHO];
  u[MX1] = v[RHO] * v[VX1];
  u[MX2] = v[RHO] * v[VX1 + 1];
  u[MX3] = v[RHO] * v[VX1 + 2];
  R kin = v[VX1] * v[VX1] + v[VX1 + 1] * v[VX1 + 1] + v[VX1 + 2] * v[VX1 + 2];
  kin = v[RHO] * kin * R(0.5);
  u[4] = kin + v[4] / (gamma - R(1));
}

// Src/HD/mappers.cpp:33-140 (ENERGY_SOLVE); FP64.
__device__ __forceinline__ uint32_t hd_cons2prim(double* u, double* v, double gamma,
                                                 double small_rho, double small_prs) {
  uint32_t err = 0;
  double gmm1 = gamma - 1.0;
  if (u[RHO] < 0.0) {
    u[RHO] = small_rho;
    err |= ERR_NEGATIVE_RHO | ERR_CONS2PRIM_FAIL;
  }
  v[RHO] = u[RHO];
  double tau = 1.0 / u[RHO];
  v[VX1] = u[MX1] * tau;
  v[VX1 + 1] = u[MX2] * tau;
  v[VX1 + 2] = u[MX3] * tau;
  double m2 = u[MX1] * u[MX1] + u[MX2] * u[MX2] + u[MX3] * u[MX3];
  double kin = 0.5 * m2 * tau;
  if (u[4] > 0.0) {
    v[4] = gmm1 * (u[4] - kin);
    if (v[4] < 0.0) {
      v[4] = small_prs;
      u[4] = v[4] / gmm1 + kin;
      err |= ERR_NEGATIVE_PRS;
    }
  } else {
    u[4] = small_prs / gmm1 + kin;
    v[4] = small_prs;
    err |= ERR_NEGATIVE_ENG;
  }
  return err;
}

// Src/HD/hd.hpp:105-125
template <int DIR, typename R>
__device__ __forceinline__ void hd_flux(const R* v, const R* u, R* f, R& p) {
  constexpr int VXn = VX1 + DIR, MXn = MX1 + DIR;
  f[RHO] = u[MXn];
  f[MX1] = u[MX1] * v[VXn];
  f[MX2] = u[MX2] * v[VXn];
  f[MX3] = u[MX3] * v[VXn];
  f[4] = (u[4] + v[4]) * v[VXn];
  p = v[4];
  f[MXn] += p;
}

// Src/HD/hllc.cpp:54-260 (ideal EOS)
template <int DIR, typename R>
__device__ __forceinline__ R hd_hllc(const R* vl, const R* vr, R* flux, R gamma) {
  constexpr int VXn = VX1 + DIR, VXt = VX1 + (DIR + 1) % 3, VXb = VX1 + (DIR + 2) % 3;
  constexpr int MXn = MX1 + DIR, MXt = MX1 + (DIR + 1) % 3, MXb = MX1 + (DIR + 2) % 3;
  R ul[5], ur[5], fL[5], fR[5], usl[5], usr[5], Sl, Sr, pl, pr;
  hd_prim2cons(vl, ul, gamma);
  hd_prim2cons(vr, ur, gamma);
  R a2L = gamma * vl[4] / vl[RHO];
  R a2R = gamma * vr[4] / vr[RHO];
  hd_flux<DIR>(vl, ul, fL, pl);
  hd_flux<DIR>(vr, ur, fR, pr);
  {
    R aL = rsqrt_(a2L), aR = rsqrt_(a2R);   // Src/HD/hd.hpp:139-150
    R sl_min = vl[VXn] - aL, sl_max = vl[VXn] + aL;
    R sr_min = vr[VXn] - aR, sr_max = vr[VXn] + aR;
    Sl = GP_MIN(sl_min, sr_min);
    Sr = GP_MAX(sl_max, sr_max);
  }
  R cmax = GP_MAX(rabs(Sl), rabs(Sr));
  if (Sl > R(0)) {
#pragma unroll
    for (int nv = 0; nv < 5; nv++) flux[nv] = fL[nv];
  } else if (Sr < R(0)) {
#pragma unroll
    for (int nv = 0; nv < 5; nv++) flux[nv] = fR[nv];
  } else {
    R vs;
    {
      R qL = vl[4] + ul[MXn] * (vl[VXn] - Sl);
      R qR = vr[4] + ur[MXn] * (vr[VXn] - Sr);
      R wL = vl[RHO] * (vl[VXn] - Sl);
      R wR = vr[RHO] * (vr[VXn] - Sr);
      vs = (qR - qL) / (wR - wL);
    }
    R vxr = vr[VXn], vxl = vl[VXn];
    usl[RHO] = ul[RHO] * (Sl - vxl) / (Sl - vs);
    usr[RHO] = ur[RHO] * (Sr - vxr) / (Sr - vs);
    usl[MXn] = usl[RHO] * vs;
    usr[MXn] = usr[RHO] * vs;
    usl[MXt] = usl[RHO] * vl[VXt];
    usr[MXt] = usr[RHO] * vr[VXt];
    usl[MXb] = usl[RHO] * vl[VXb];
    usr[MXb] = usr[RHO] * vr[VXb];
    usl[4] = ul[4] / vl[RHO] + (vs - vxl) * (vs + vl[4] / (vl[RHO] * (Sl - vxl)));
    usr[4] = ur[4] / vr[RHO] + (vs - vxr) * (vs + vr[4] / (vr[RHO] * (Sr - vxr)));
    usl[4] *= usl[RHO];
    usr[4] *= usr[RHO];
    if (vs >= R(0)) {
#pragma unroll
      for (int nv = 0; nv < 5; nv++) flux[nv] = fL[nv] + Sl * (usl[nv] - ul[nv]);
    } else {
#pragma unroll
      for (int nv = 0; nv < 5; nv++) flux[nv] = fR[nv] + Sr * (usr[nv] - ur[nv]);
    }
  }
  return cmax;
}

// Src/HD/hll.cpp:95-175
// Lax-Friedrichs flux for HD, Src/HD/tvdlf.cpp:100-190: the average state
// takes the mean of |v_n| on the two sides.
template <int DIR, typename R>
__device__ __forceinline__ R hd_tvdlf(const R* vl, const R* vr, R* flux, R gamma) {
  constexpr int VXn = VX1 + DIR;
  R ul[5], ur[5], fL[5], fR[5], vLR[5], pl, pr, cmax;
  hd_prim2cons(vl, ul, gamma);
  hd_prim2cons(vr, ur, gamma);
#pragma unroll
  for (int nv = 0; nv < 5; nv++) vLR[nv] = R(0.5) * (vl[nv] + vr[nv]);
  vLR[VXn] = R(0.5) * (rabs(vl[VXn]) + rabs(vr[VXn]));
  {
    const R a = rsqrt_(gamma * vLR[4] / vLR[RHO]);
    const R cmaxLR = vLR[VXn] + a, cminLR = vLR[VXn] - a;
    cmax = GP_MAX(rabs(cminLR), rabs(cmaxLR));
  }
  hd_flux<DIR>(vl, ul, fL, pl);
  hd_flux<DIR>(vr, ur, fR, pr);
#pragma unroll
  for (int nv = 0; nv < 5; nv++)
    flux[nv] = R(0.5) * (fL[nv] + fR[nv]) - R(0.5) * cmax * (ur[nv] - ul[nv]);
  return cmax;
}

template <int DIR, typename R>
__device__ __forceinline__ R hd_hll(const R* vl, const R* vr, R* flux, R gamma) {
  constexpr int VXn = VX1 + DIR;
  R ul[5], ur[5], fL[5], fR[5], Sl, Sr, pl, pr;
  hd_prim2cons(vl, ul, gamma);
  hd_prim2cons(vr, ur, gamma);
  R a2L = gamma * vl[4] / vl[RHO];
  R a2R = gamma * vr[4] / vr[RHO];
  hd_flux<DIR>(vl, ul, fL, pl);
  hd_flux<DIR>(vr, ur, fR, pr);
  {
    R aL = rsqrt_(a2L), aR = rsqrt_(a2R);
    R sl_min = vl[VXn] - aL, sl_max = vl[VXn] + aL;
    R sr_min = vr[VXn] - aR, sr_max = vr[VXn] + aR;
    Sl = GP_MIN(sl_min, sr_min);
    Sr = GP_MAX(sl_max, sr_max);
  }
  R cmax = GP_MAX(rabs(Sl), rabs(Sr));
  if (Sl > R(0)) {
#pragma unroll
    for (int nv = 0; nv < 5; nv++) flux[nv] = fL[nv];
  } else if (Sr < R(0)) {
#pragma unroll
    for (int nv = 0; nv < 5; nv++) flux[nv] = fR[nv];
  } else {
    R scrh = R(1) / (Sr - Sl);
#pragma unroll
    for (int nv = 0; nv < 5; nv++) {
      flux[nv] = Sl * Sr * (ur[nv] - ul[nv]) + Sr * fL[nv] - Sl * fR[nv];
      flux[nv] *= scrh;
    }
  }
  return cmax;
}

}  // namespace gp
