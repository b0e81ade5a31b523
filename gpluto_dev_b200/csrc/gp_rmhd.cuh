// gp_rmhd.cuh -- special-relativistic MHD interface physics (sm_100a).
//
// Ideal EOS, reduced energy (E - D, Src/RMHD/rmhd.hpp:134-138), quartic fast
// magnetosonic speeds (RMHD_FAST_EIGENVALUES = NO), relativistic HLLD of
// Mignone, Ugliano & Bodo (2009) with the secant iteration on the total
// pressure (Src/RMHD/hlld.cpp:96-554), HLL, UCT_HLL face data, and the
// Newton-Raphson energy inversion (Src/RMHD/rmhd_energy_solve.cpp) with the
// pressure-fix bisection fallback (Src/RMHD/rmhd_pressure_fix.cpp).
// Expressions keep the reference's operation order.  The conservative ->
// primitive inversion always runs in FP64 (also inside the Riemann solver of
// the mixed form).  The quartic's acos/cos/sin are correctly rounded
// (gp_crmath.cuh), so the FP64 form matches the reference wherever glibc's
// results are correctly rounded too.
#pragma once
#include "gp_crmath.cuh"
#include "gp_phys.cuh"

namespace gp {

constexpr uint32_t ERR_PRESSURE_FIX = 1u << 5;

template <typename R>
__device__ __forceinline__ R rmhd_enthalpy(const R* v, R gamma) {  // Src/eos.hpp:38-46
  R gmmr = gamma / (gamma - R(1));
  R theta = v[7] / v[RHO];
  return R(1) + gmmr * theta;
}

// Src/RMHD/rmhd.hpp:535-600
template <typename R>
__device__ __forceinline__ void rmhd_prim2cons(const R* v, R* u, R gamma) {
  R gmmr = gamma / (gamma - R(1));
  R h = rmhd_enthalpy(v, gamma);
  R vx1 = v[VX1], vx2 = v[VX1 + 1], vx3 = v[VX1 + 2];
  R vel2 = vx1 * vx1 + vx2 * vx2 + vx3 * vx3;
  R g2 = R(1) / (R(1) - vel2);
  R g = rsqrt_(g2);
  R ex = vx2 * v[BX3] - vx3 * v[BX2];
  R ey = vx3 * v[BX1] - vx1 * v[BX3];
  R ez = vx1 * v[BX2] - vx2 * v[BX1];
  R e2 = ex * ex + ey * ey + ez * ez;
  R Bmag2 = v[BX1] * v[BX1] + v[BX2] * v[BX2] + v[BX3] * v[BX3];
  R wt = v[RHO] * h * g2;
  u[RHO] = g * v[RHO];
  u[MX1] = wt * vx1 + v[BX2] * ez - v[BX3] * ey;
  u[MX2] = wt * vx2 + v[BX3] * ex - v[BX1] * ez;
  u[MX3] = wt * vx3 + v[BX1] * ey - v[BX2] * ex;
  u[BX1] = v[BX1];
  u[BX2] = v[BX2];
  u[BX3] = v[BX3];
  u[7] = v[7] * (g2 * gmmr - R(1)) + u[RHO] * g2 * vel2 / (g + R(1)) + R(0.5) * (Bmag2 + e2);
}

// Src/RMHD/rmhd.hpp:315-366
template <int DIR, typename R>
__device__ __forceinline__ void rmhd_flux(const R* v, const R* u, R h, R* flux, R& pt) {
  constexpr int VXn = VX1 + DIR, VXt = VX1 + (DIR + 1) % 3, VXb = VX1 + (DIR + 2) % 3;
  constexpr int BXn = BX1 + DIR, BXt = BX1 + (DIR + 1) % 3, BXb = BX1 + (DIR + 2) % 3;
  constexpr int MXn = MX1 + DIR;
  R g = u[RHO] / v[RHO];
  R g2 = g * g;
  R g_2 = R(1) / g2;
  R Bmag2 = v[BX1] * v[BX1] + v[BX2] * v[BX2] + v[BX3] * v[BX3];
  R vB = v[VX1] * v[BX1] + v[VX1 + 1] * v[BX2] + v[VX1 + 2] * v[BX3];
  R b[3];
  b[0] = g * (v[BX1] * g_2 + vB * v[VX1]);
  b[1] = g * (v[BX2] * g_2 + vB * v[VX1 + 1]);
  b[2] = g * (v[BX3] * g_2 + vB * v[VX1 + 2]);
  R b2 = Bmag2 * g_2 + vB * vB;
  pt = v[7] + R(0.5) * b2;
  R wt = v[RHO] * h + b2;
  R wtg2 = wt * g2;
  flux[RHO] = u[RHO] * v[VXn];
  flux[MX1] = wtg2 * v[VX1] * v[VXn] - b[0] * b[DIR];
  flux[MX2] = wtg2 * v[VX1 + 1] * v[VXn] - b[1] * b[DIR];
  flux[MX3] = wtg2 * v[VX1 + 2] * v[VXn] - b[2] * b[DIR];
  flux[BXn] = R(0);
  flux[BXt] = v[VXn] * v[BXt] - v[BXn] * v[VXt];
  flux[BXb] = v[VXn] * v[BXb] - v[BXn] * v[VXb];
  flux[7] = u[MXn];
  flux[7] -= flux[RHO];
  flux[MXn] += pt;
}

// Src/RMHD/rmhd.hpp:390-452 (acos/cos/sin correctly rounded: the roots feed
// discontinuous decisions, so they follow the reference's glibc results bit
// for bit except where glibc itself is not correctly rounded)
__device__ __forceinline__ void cubic_solve(double b, double c, double d, double* z) {
  const double one_3 = 1.0 / 3.0, one_27 = 1.0 / 27.0, sqrt3 = sqrt(3.0);
  double b2 = b * b;
  double Q = b2 * one_3 - c * (1.0 - 1.e-16);
  double R_ = b * (2.0 * b2 - 9.0 * c) * one_27 + d;
  Q = GP_MAX(Q, 0.0);
  double sQ = sqrt(Q) / sqrt3;
  double arg = -1.5 * R_ / (Q * sQ);
  arg = GP_MAX(-1.0, arg);
  arg = GP_MIN(1.0, arg);
  double theta = gpcr::acos_cr(arg) * one_3;   // in [0, pi/3]
  double sn, cs;
  gpcr::sincos_cr(theta, &sn, &cs);
  sn = sqrt3 * sn;
  double p = -b * one_3;
  z[0] = -sQ * (cs + sn) + p;
  z[1] = -sQ * (cs - sn) + p;
  z[2] = 2.0 * sQ * cs + p;
}
__device__ __forceinline__ void cubic_solve(float b, float c, float d, float* z) {
  const float one_3 = 1.0f / 3.0f, one_27 = 1.0f / 27.0f, sqrt3 = sqrtf(3.0f);
  float b2 = b * b;
  float Q = b2 * one_3 - c * (1.0f - 1.e-7f);
  float R_ = b * (2.0f * b2 - 9.0f * c) * one_27 + d;
  Q = GP_MAX(Q, 0.0f);
  float sQ = sqrtf(Q) / sqrt3;
  float arg = -1.5f * R_ / (Q * sQ);
  arg = GP_MAX(-1.0f, arg);
  arg = GP_MIN(1.0f, arg);
  float theta = acosf(arg) * one_3;
  float sn, cs;
  sincosf(theta, &sn, &cs);
  sn = sqrt3 * sn;
  float p = -b * one_3;
  z[0] = -sQ * (cs + sn) + p;
  z[1] = -sQ * (cs - sn) + p;
  z[2] = 2.0f * sQ * cs + p;
}

// Src/RMHD/rmhd.hpp:455-505; returns the smallest and largest roots
template <typename R>
__device__ __forceinline__ void quartic_extremes(R b, R c, R d, R e, R& zmin, R& zmax) {
  R b2 = b * b;
  R p = c - b2 * R(0.375);
  R q = d + b2 * b * R(0.125) - b * c * R(0.5);
  R r = e - R(3) * b2 * b2 / R(256) + b2 * c / R(16) - R(0.25) * b * d;
  R a2 = R(2) * p;
  R a1 = p * p - R(4) * r;
  R a0 = -q * q;
  R u[3];
  cubic_solve(a2, a1, a0, u);
  u[0] = GP_MAX(u[0], R(0));
  u[1] = GP_MAX(u[1], R(0));
  u[2] = GP_MAX(u[2], R(0));
  R sq = R(-0.5) * (q >= R(0) ? R(1) : R(-1));
  R sz1 = sq * rsqrt_(u[0]);
  R sz2 = sq * rsqrt_(u[1]);
  R sz3 = sq * rsqrt_(u[2]);
  R z[4];
  z[0] = R(-0.25) * b + sz1 + sz2 + sz3;
  z[1] = R(-0.25) * b + sz1 - sz2 - sz3;
  z[2] = R(-0.25) * b - sz1 + sz2 - sz3;
  z[3] = R(-0.25) * b - sz1 - sz2 + sz3;
  // insertion sort (Src/RMHD/rmhd.hpp:372-388); only the extremes are used
  zmin = z[0];
  zmax = z[0];
#pragma unroll
  for (int m = 1; m < 4; m++) {
    zmin = (z[m] < zmin) ? z[m] : zmin;
    zmax = (z[m] > zmax) ? z[m] : zmax;
  }
}

// Src/RMHD/rmhd.hpp:631-763
template <int DIR, typename R>
__device__ __forceinline__ void rmhd_signal_speed(const R* v, R cs2, R h, R& cmin, R& cmax) {
  constexpr int VXn = VX1 + DIR, BXn = BX1 + DIR;
  R vB = v[VX1] * v[BX1] + v[VX1 + 1] * v[BX2] + v[VX1 + 2] * v[BX3];
  R u02 = v[VX1] * v[VX1] + v[VX1 + 1] * v[VX1 + 1] + v[VX1 + 2] * v[VX1 + 2];
  R Bm2 = v[BX1] * v[BX1] + v[BX2] * v[BX2] + v[BX3] * v[BX3];
  if (u02 < R(1.e-14)) {
    R w_1 = R(1) / (v[RHO] * h + Bm2);
    R eps2 = cs2 + Bm2 * w_1 * (R(1) - cs2);
    R a0 = cs2 * v[BXn] * v[BXn] * w_1;
    R a1 = -a0 - eps2;
    R del = a1 * a1 - R(4) * a0;
    del = GP_MAX(del, R(0));
    del = rsqrt_(del);
    cmax = rsqrt_(R(0.5) * (-a1 + del));
    cmin = -cmax;
    return;
  }
  R vB2 = vB * vB;
  u02 = R(1) / (R(1) - u02);
  R b2 = Bm2 / u02 + vB2;
  R w_1 = R(1) / (v[RHO] * h + b2);
  R vx = v[VXn];
  R vx2 = vx * vx;
  if (rabs(v[BXn]) < R(1.e-14)) {
    R w = v[RHO] * h;
    R scrh1 = b2 + cs2 * (w - vB2);
    R scrh2 = w * (R(1) - cs2) * u02;
    R del = R(4) * scrh1 * (scrh2 * (R(1) - vx2) + scrh1);
    R a2 = scrh1 + scrh2;
    R a1 = R(-2) * vx * scrh2;
    cmax = R(0.5) * (-a1 + rsqrt_(del)) / a2;
    cmin = R(0.5) * (-a1 - rsqrt_(del)) / a2;
    return;
  }
  R scrh1 = v[BXn] / u02 + vB * vx;
  R scrh2 = scrh1 * scrh1;
  R a2_w = cs2 * w_1;
  R eps2 = (cs2 * v[RHO] * h + b2) * w_1;
  R one_m_eps2 = u02 * v[RHO] * h * (R(1) - cs2) * w_1;
  R scrh = R(2) * (a2_w * vB * scrh1 - eps2 * vx);
  R a4 = one_m_eps2 - a2_w * vB2 + eps2;
  R a3 = R(-4) * vx * one_m_eps2 + scrh;
  R a2 = R(6) * vx2 * one_m_eps2 + a2_w * (vB2 - scrh2) + eps2 * (vx2 - R(1));
  R a1 = R(-4) * vx * vx2 * one_m_eps2 - scrh;
  R a0 = vx2 * vx2 * one_m_eps2 + a2_w * scrh2 - eps2 * vx2;
  scrh = R(1) / a4;
  a3 *= scrh;
  a2 *= scrh;
  a1 *= scrh;
  a0 *= scrh;
  quartic_extremes(a3, a2, a1, a0, cmin, cmax);
}

// ---------------------------------------------------------------------
// conservative -> primitive (FP64 always)
// ---------------------------------------------------------------------

// Src/RMHD/rmhd_energy_solve.cpp:35-209 (ideal EOS, reduced energy)
__device__ __forceinline__ uint32_t rmhd_energy_solve(const double* u, double* v, double gamma) {
  const double acc = 1.e-11;
  const double D = u[RHO];
  const double E = u[7];
  const double S = u[MX1] * u[BX1] + u[MX2] * u[BX2] + u[MX3] * u[BX3];
  const double m2 = u[MX1] * u[MX1] + u[MX2] * u[MX2] + u[MX3] * u[MX3];
  const double B2 = u[BX1] * u[BX1] + u[BX2] * u[BX2] + u[BX3] * u[BX3];
  const double S2 = S * S;
  if (E < 0.0) return ERR_NEGATIVE_ENG;
  double Y1 = -4.0 * (E + D - B2);
  double Y2 = m2 - 2.0 * (E + D) * B2 + B2 * B2;
  double chi = Y1 * Y1 - 12.0 * Y2;
  chi = GP_MAX(0.0, chi);
  double W = (-Y1 + sqrt(chi)) / 6.0;
  W = GP_MAX(D, W);
  double Wp = W - D;
  int done = 0;
  double p = -1.0, lor = 1.0;
  int k;
  for (k = 1; k < 50; k++) {  // bounded Newton iteration (MAX_ITER 50)
    W = Wp + D;
    double W2 = W * W;
    double S2_W2 = S2 / W2;
    Y1 = 1.0 / (W + B2);
    Y2 = Y1 * Y1;
    double vel2 = S2_W2 * Y1 * (Y1 * W + 1.0) + m2 * Y2;
    double one_m_v2 = 1.0 - vel2;
    double lor2 = 1.0 / one_m_v2;
    lor = sqrt(lor2);
    if (vel2 > 1.0) return ERR_ENG_SOLVE_NO_SOLUTION;
    chi = Wp / lor2 - D * vel2 / (lor + 1.0);
    double dv2_dW = -2.0 * Y2 * (3.0 * S2_W2 + Y1 * (S2_W2 * B2 * B2 / W + m2));
    double dchi_dW = one_m_v2 - 0.5 * lor * (D + 2.0 * chi * lor) * dv2_dW;
    double drho_dW = -0.5 * D * lor * dv2_dW;
    double dp_dchi = (gamma - 1.0) / gamma;
    double dp_drho = 0.0;
    p = chi * dp_dchi;
    if (done) break;
    double dp = dp_dchi * dchi_dW + dp_drho * drho_dW;
    double fW = Wp + 0.5 * (B2 + (B2 * m2 - S2) * Y2) - (E + p);
    double dfW = 1.0 - dp - (B2 * m2 - S2) * Y2 * Y1;
    double dW = fW / dfW;
    Wp -= dW;
    if (fabs(dW) < acc * Wp || fabs(fW) < acc) done = 1;
  }
  if (p < 0.0) return ERR_NEGATIVE_PRS;
  if (k == 50) return ERR_TOO_MANY_ITERATIONS;
  if (isnan(p)) return ERR_NAN;
  W = Wp + D;
  v[RHO] = u[RHO] / lor;
  v[7] = p;
  Y1 = 1.0 / (W + B2);
  double scrh = S / W;
  v[VX1] = Y1 * (u[MX1] + scrh * u[BX1]);
  v[VX1 + 1] = Y1 * (u[MX2] + scrh * u[BX2]);
  v[VX1 + 2] = Y1 * (u[MX3] + scrh * u[BX3]);
  return 0;
}

// f(v^2) of the pressure-fix bisection
__device__ __forceinline__ double pfix_W(double D, double plor, double lor, double gamma) {
  return (D + plor * gamma / (gamma - 1.0)) * lor;
}

// Src/RMHD/rmhd_pressure_fix.cpp:22-181 (ideal EOS, reduced energy)
__device__ __forceinline__ uint32_t rmhd_pressure_fix(double* u, double* v, double gamma,
                                                      double small_prs) {
  const double D = u[RHO];
  const double S = u[MX1] * u[BX1] + u[MX2] * u[BX2] + u[MX3] * u[BX3];
  const double m2 = u[MX1] * u[MX1] + u[MX2] * u[MX2] + u[MX3] * u[MX3];
  const double B2 = u[BX1] * u[BX1] + u[BX2] * u[BX2] + u[BX3] * u[BX3];
  const double S2 = S * S;
  const double p = small_prs;
  double v2, v2min, v2max, fmin, f, lor, plor, W, W2;
  v2min = v2 = 0.0;
  lor = 1.0 / sqrt(1.0 - v2);
  plor = p * lor;
  W = pfix_W(D, plor, lor, gamma);
  W2 = W * W;
  f = (S2 * (2.0 * W + B2) + m2 * W2) / ((W + B2) * (W + B2) * W2);
  f -= v2;
  fmin = f;
  v2max = v2 = 1.0 - 1.e-9;
  lor = 1.0 / sqrt(1.0 - v2);
  plor = p * lor;
  W = pfix_W(D, plor, lor, gamma);
  W2 = W * W;
  f = (S2 * (2.0 * W + B2) + m2 * W2) / ((W + B2) * (W + B2) * W2);
  f -= v2;
  int k;
  for (k = 1; k < 50; k++) {  // bounded bisection (MAX_ITER 50)
    v2 = 0.5 * (v2min + v2max);
    lor = 1.0 / sqrt(1.0 - v2);
    plor = p * lor;
    W = pfix_W(D, plor, lor, gamma);
    W2 = W * W;
    f = (S2 * (2.0 * W + B2) + m2 * W2) / ((W + B2) * (W + B2) * W2);
    f -= v2;
    if (f * fmin > 0.0) {
      v2min = v2;
      fmin = f;
    } else {
      v2max = v2;
    }
    if (fabs(f) < 1.e-9) break;
  }
  if (v2 >= 1.0 && k == 50) return ERR_PRESSURE_FIX;
  v[RHO] = D / lor;
  v[7] = p;
  double w_1 = 1.0 / (W + B2);
  double scrh = S / W;
  v[VX1] = w_1 * (u[MX1] + scrh * u[BX1]);
  v[VX1 + 1] = w_1 * (u[MX2] + scrh * u[BX2]);
  v[VX1 + 2] = w_1 * (u[MX3] + scrh * u[BX3]);
  double S2_W2 = S2 / W2;
  u[7] = W - D - p + 0.5 * (1.0 + v2) * B2 - 0.5 * S2_W2;
  return 0;
}

// Src/RMHD/mappers.cpp:33-157 (ENERGY_SOLVE, no PCP)
__device__ __forceinline__ uint32_t rmhd_cons2prim(double* u, double* v, double gamma,
                                                   double small_rho, double small_prs) {
  int fix = 0;
  uint32_t err_mapper = 0;
  v[BX1] = u[BX1];
  v[BX2] = u[BX2];
  v[BX3] = u[BX3];
  if (u[RHO] < 0.0) {
    u[RHO] = small_rho;
    err_mapper |= ERR_NEGATIVE_RHO;
  }
  if (u[7] < 0.0) {
    fix = 1;
    err_mapper |= ERR_NEGATIVE_ENG;
  }
  if (!fix) {
    uint32_t err = rmhd_energy_solve(u, v, gamma);
    if (err) fix = 1;
    err_mapper |= err;
  }
  if (fix) {
    uint32_t err = rmhd_pressure_fix(u, v, gamma, small_prs);
    if (err != 0) err_mapper |= err | ERR_CONS2PRIM_FAIL;
  }
  double scrh = v[VX1] * v[VX1] + v[VX1 + 1] * v[VX1 + 1] + v[VX1 + 2] * v[VX1 + 2];
  if (scrh >= 1.0) err_mapper |= ERR_SUPERLUMINAL_SPEED | ERR_CONS2PRIM_FAIL;
  return err_mapper;
}

// ---------------------------------------------------------------------
// HLLD (Src/RMHD/hlld.cpp)
// ---------------------------------------------------------------------
template <typename R>
struct RState {
  int fail;
  R vx, vy, vz, By, Bz, Kx, Ky, Kz, K2, w, sw;
  R u[8], Rr[8];
  R S, Sa;
};

// Src/RMHD/hlld.cpp:650-735; returns 0 when w < 0
template <int DIR, typename R>
__device__ __forceinline__ int hlld_riemann_state(RState<R>& P, R p, R Bx, int side) {
  constexpr int MXn = MX1 + DIR, MXt = MX1 + (DIR + 1) % 3, MXb = MX1 + (DIR + 2) % 3;
  constexpr int BXn = BX1 + DIR, BXt = BX1 + (DIR + 1) % 3, BXb = BX1 + (DIR + 2) % 3;
  const R S = P.S;
  const R* Rv = P.Rr;
  R A = Rv[MXn] + p * (R(1) - S * S) - S * Rv[7];
  R G = Rv[BXt] * Rv[BXt] + Rv[BXb] * Rv[BXb];
  R C = Rv[BXt] * Rv[MXt] + Rv[BXb] * Rv[MXb];
  R X = Bx * (A * S * Bx + C) - (A + G) * (S * p + Rv[7]);
  R vx = (Bx * (A * Bx + C * S) - (Rv[MXn] + p) * (G + A));
  R vy = (-(A + G - Bx * Bx * (R(1) - S * S)) * Rv[MXt] +
          Rv[BXt] * (C + Bx * (S * Rv[MXn] - Rv[7])));
  R vz = (-(A + G - Bx * Bx * (R(1) - S * S)) * Rv[MXb] +
          Rv[BXb] * (C + Bx * (S * Rv[MXn] - Rv[7])));
  R scrh = vx * Rv[MXn] + vy * Rv[MXt] + vz * Rv[MXb];
  scrh = X * Rv[7] - scrh;
  P.w = p + scrh / (X * S - vx);
  if (P.w < R(0)) return 0;
  P.vx = vx / X;
  P.vy = vy / X;
  P.vz = vz / X;
  P.By = -(Rv[BXt] * (S * p + Rv[7]) - Bx * Rv[MXt]) / A;
  P.Bz = -(Rv[BXb] * (S * p + Rv[7]) - Bx * Rv[MXb]) / A;
  R s = Bx > R(0) ? R(1) : R(-1);
  if (side < 0) s *= R(-1);
  P.sw = s * rsqrt_(P.w);
  scrh = R(1) / (S * p + Rv[7] + Bx * P.sw);
  P.Kx = scrh * (Rv[MXn] + p + Rv[BXn] * P.sw);
  P.Ky = scrh * (Rv[MXt] + Rv[BXt] * P.sw);
  P.Kz = scrh * (Rv[MXb] + Rv[BXb] * P.sw);
  P.K2 = P.Kx * P.Kx + P.Ky * P.Ky + P.Kz * P.Kz;
  return 1;
}

// Src/RMHD/hlld.cpp:561-644
// One deliberate difference: when a Riemann state cannot be built (w < 0) the
// reference discards that status and evaluates the admissibility checks on the
// state's previous (or never set) fields, so with a negative pressure guess
// the result depends on stale stack contents.  Here a failed state always
// fails the star solution (HLL fallback), which is deterministic.
template <int DIR, typename R>
__device__ __forceinline__ R hlld_fstar(RState<R>& PaL, RState<R>& PaR, R p, R Bx, R& Sc) {
  // both sides through one inlined copy of the state builder: inputs (S,
  // R) in, outputs (w, v, B_t, K, sw) back; a failed side keeps its
  // previous outputs, as a direct call would
  int okL = 0, okR = 0;
#pragma unroll 1
  for (int s = 0; s < 2; s++) {
    RState<R> T;
    T.S = s ? PaR.S : PaL.S;
#pragma unroll
    for (int nv = 0; nv < 8; nv++) T.Rr[nv] = s ? PaR.Rr[nv] : PaL.Rr[nv];
    T.w = s ? PaR.w : PaL.w;
    T.vx = s ? PaR.vx : PaL.vx;
    T.vy = s ? PaR.vy : PaL.vy;
    T.vz = s ? PaR.vz : PaL.vz;
    T.By = s ? PaR.By : PaL.By;
    T.Bz = s ? PaR.Bz : PaL.Bz;
    T.sw = s ? PaR.sw : PaL.sw;
    T.Kx = s ? PaR.Kx : PaL.Kx;
    T.Ky = s ? PaR.Ky : PaL.Ky;
    T.Kz = s ? PaR.Kz : PaL.Kz;
    T.K2 = s ? PaR.K2 : PaL.K2;
    const int ok = hlld_riemann_state<DIR>(T, p, Bx, s ? 1 : -1);
    if (s) okR = ok; else okL = ok;
    if (s) {
      PaR.w = T.w; PaR.vx = T.vx; PaR.vy = T.vy; PaR.vz = T.vz; PaR.By = T.By; PaR.Bz = T.Bz;
      PaR.sw = T.sw; PaR.Kx = T.Kx; PaR.Ky = T.Ky; PaR.Kz = T.Kz; PaR.K2 = T.K2;
    } else {
      PaL.w = T.w; PaL.vx = T.vx; PaL.vy = T.vy; PaL.vz = T.vz; PaL.By = T.By; PaL.Bz = T.Bz;
      PaL.sw = T.sw; PaL.Kx = T.Kx; PaL.Ky = T.Ky; PaL.Kz = T.Kz; PaL.K2 = T.K2;
    }
  }
  R dK = PaR.Kx - PaL.Kx + R(1.e-12);
  R Bxc = Bx * dK;
  R Byc = PaR.By * (PaR.Kx - PaR.vx) - PaL.By * (PaL.Kx - PaL.vx) + Bx * (PaR.vy - PaL.vy);
  R Bzc = PaR.Bz * (PaR.Kx - PaR.vx) - PaL.Bz * (PaL.Kx - PaL.vx) + Bx * (PaR.vz - PaL.vz);
  R KLBc = PaL.Kx * Bxc + PaL.Ky * Byc + PaL.Kz * Bzc;
  R KRBc = PaR.Kx * Bxc + PaR.Ky * Byc + PaR.Kz * Bzc;
  R vxcL = PaL.Kx - dK * Bx * (R(1) - PaL.K2) / (PaL.sw * dK - KLBc);
  R vxcR = PaR.Kx - dK * Bx * (R(1) - PaR.K2) / (PaR.sw * dK - KRBc);
  PaL.Sa = PaL.Kx;
  PaR.Sa = PaR.Kx;
  Sc = R(0.5) * (vxcL + vxcR);
  R fun = vxcL - vxcR;
  int success = (vxcL - PaL.Kx) > R(-1.e-6);
  success *= (PaR.Kx - vxcR) > R(-1.e-6);
  success *= (PaL.S - PaL.vx) < R(0);
  success *= (PaR.S - PaR.vx) > R(0);
  success *= (PaR.w - p) > R(0);
  success *= (PaL.w - p) > R(0);
  success *= (PaL.Sa - PaL.S) > R(-1.e-6);
  success *= (PaR.S - PaR.Sa) > R(-1.e-6);
  PaL.fail = !(success && okL && okR);
  return fun;
}

// Src/RMHD/hlld.cpp:741-770
template <int DIR, typename R>
__device__ __forceinline__ void hlld_astate(RState<R>& P, R p, R Bx) {
  constexpr int MXn = MX1 + DIR, MXt = MX1 + (DIR + 1) % 3, MXb = MX1 + (DIR + 2) % 3;
  constexpr int BXn = BX1 + DIR, BXt = BX1 + (DIR + 1) % 3, BXb = BX1 + (DIR + 2) % 3;
  R* ua = P.u;
  const R* Rv = P.Rr;
  R scrh = R(1) / (P.S - P.vx);
  ua[RHO] = Rv[RHO] * scrh;
  ua[BXn] = Bx;
  ua[BXt] = (Rv[BXt] - Bx * P.vy) * scrh;
  ua[BXb] = (Rv[BXb] - Bx * P.vz) * scrh;
  R vB = P.vx * ua[BXn] + P.vy * ua[BXt] + P.vz * ua[BXb];
  ua[7] = (Rv[7] + p * P.vx - vB * Bx) * scrh;
  ua[MXn] = (ua[7] + p) * P.vx - vB * ua[BXn];
  ua[MXt] = (ua[7] + p) * P.vy - vB * ua[BXt];
  ua[MXb] = (ua[7] + p) * P.vz - vB * ua[BXb];
}

// Src/RMHD/hlld.cpp:776-858; PaL.u and PaR.u hold the Alfven states
// (hlld_astate) on entry
template <int DIR, typename R>
__device__ __forceinline__ void hlld_cstate(RState<R>& PaL, RState<R>& PaR, R p, R Bx, R* Uc) {
  constexpr int MXn = MX1 + DIR, MXt = MX1 + (DIR + 1) % 3, MXb = MX1 + (DIR + 2) % 3;
  constexpr int BXn = BX1 + DIR, BXt = BX1 + (DIR + 1) % 3, BXb = BX1 + (DIR + 2) % 3;
  R dK = (PaR.Kx - PaL.Kx) + R(1.e-12);
  R Byc = PaR.By * (PaR.Kx - PaR.vx) - PaL.By * (PaL.Kx - PaL.vx) + Bx * (PaR.vy - PaL.vy);
  R Bzc = PaR.Bz * (PaR.Kx - PaR.vx) - PaL.Bz * (PaL.Kx - PaL.vx) + Bx * (PaR.vz - PaL.vz);
  R Bxc = Bx;
  Byc /= dK;
  Bzc /= dK;
  Uc[BXn] = Bxc;
  Uc[BXt] = Byc;
  Uc[BXb] = Bzc;
  R KLBc = PaL.Kx * Bxc + PaL.Ky * Byc + PaL.Kz * Bzc;
  R KRBc = PaR.Kx * Bxc + PaR.Ky * Byc + PaR.Kz * Bzc;
  R scrhL = (R(1) - PaL.K2) / (PaL.sw - KLBc);
  R scrhR = (R(1) - PaR.K2) / (PaR.sw - KRBc);
  R vxcL = PaL.Kx - Uc[BXn] * scrhL;
  R vxcR = PaR.Kx - Uc[BXn] * scrhR;
  R vycL = PaL.Ky - Uc[BXt] * scrhL;
  R vycR = PaR.Ky - Uc[BXt] * scrhR;
  R vzcL = PaL.Kz - Uc[BXb] * scrhL;
  R vzcR = PaR.Kz - Uc[BXb] * scrhR;
  R vxc = R(0.5) * (vxcL + vxcR);
  R vyc = R(0.5) * (vycL + vycR);
  R vzc = R(0.5) * (vzcL + vzcR);
  const R* ua;
  R Sa, vxa;
  if (vxc > R(0)) {
    ua = PaL.u;
    Sa = PaL.Sa;
    vxa = PaL.vx;
  } else {
    ua = PaR.u;
    Sa = PaR.Sa;
    vxa = PaR.vx;
  }
  R vBc = vxc * Uc[BXn] + vyc * Uc[BXt] + vzc * Uc[BXb];
  Uc[RHO] = ua[RHO] * (Sa - vxa) / (Sa - vxc);
  Uc[7] = (Sa * ua[7] - ua[MXn] + p * vxc - vBc * Bx) / (Sa - vxc);
  Uc[MXn] = (Uc[7] + p) * vxc - vBc * Bx;
  Uc[MXt] = (Uc[7] + p) * vyc - vBc * Uc[BXt];
  Uc[MXb] = (Uc[7] + p) * vzc - vBc * Uc[BXb];
}

// Src/RMHD/hlld.cpp:873-891
__device__ __forceinline__ double hlld_total_pressure(const double* v) {
  double Bmag2 = v[BX1] * v[BX1] + v[BX2] * v[BX2] + v[BX3] * v[BX3];
  double vel2 = v[VX1] * v[VX1] + v[VX1 + 1] * v[VX1 + 1] + v[VX1 + 2] * v[VX1 + 2];
  double vB = v[VX1] * v[BX1] + v[VX1 + 1] * v[BX2] + v[VX1 + 2] * v[BX3];
  return v[7] + 0.5 * (Bmag2 * (1.0 - vel2) + vB * vB);
}

// RMHD Riemann solver (HLLD or HLL) with UCT_HLL face data; returns cmax.
// `err` collects the bits of the nested con2prim (Src/RMHD/hlld.cpp:338-347).
template <int DIR, int RS, typename R>
__device__ __forceinline__ R rmhd_riemann(const R* vl, const R* vr, R* flux, R gamma,
                                          CTFace<R>& ct, uint32_t& err) {
  constexpr int MXn = MX1 + DIR, BXn = BX1 + DIR;
  R ul[8], ur[8], fl[8], fr[8], Sl, Sr, pl, pr;
  rmhd_prim2cons(vl, ul, gamma);
  rmhd_prim2cons(vr, ur, gamma);
  const R hl = rmhd_enthalpy(vl, gamma), hr = rmhd_enthalpy(vr, gamma);
  const R a2L = gamma * (vl[7] / vl[RHO]) / hl;  // Src/eos.hpp:114-119
  const R a2R = gamma * (vr[7] / vr[RHO]) / hr;
  rmhd_flux<DIR>(vl, ul, hl, fl, pl);
  rmhd_flux<DIR>(vr, ur, hr, fr, pr);
  {
    // one inlined copy of the quartic for both states: the left state on
    // the first pass, the right on the second
    R cmn[2], cmx[2];
#pragma unroll 1
    for (int s = 0; s < 2; s++) {
      R q[8];
#pragma unroll
      for (int nv = 0; nv < 8; nv++) q[nv] = s ? vr[nv] : vl[nv];
      R sm, sx;
      rmhd_signal_speed<DIR>(q, s ? a2R : a2L, s ? hr : hl, sm, sx);
      if (s) { cmn[1] = sm; cmx[1] = sx; } else { cmn[0] = sm; cmx[0] = sx; }
    }
    Sl = GP_MIN(cmn[0], cmn[1]);
    Sr = GP_MAX(cmx[0], cmx[1]);
    if constexpr (RS == RS_TVDLF) {
      // Src/RMHD/tvdlf.cpp: the larger of the two states' bounds, Sl = -cmax
      const R cL = GP_MAX(rabs(cmx[0]), rabs(cmn[0])), cR = GP_MAX(rabs(cmx[1]), rabs(cmn[1]));
      Sr = GP_MAX(cL, cR);
      Sl = -Sr;
    }
  }
  const R cmax = RS == RS_TVDLF ? Sr : GP_MAX(rabs(Sl), rabs(Sr));
  if constexpr (RS == RS_TVDLF) {  // Lax-Friedrichs flux
#pragma unroll
    for (int nv = 0; nv < 8; nv++)
      flux[nv] = R(0.5) * (fl[nv] + fr[nv]) - R(0.5) * cmax * (ur[nv] - ul[nv]);
  } else if constexpr (RS != RS_HLLD) {  // Src/RMHD/hll.cpp:180-202
    R bL = GP_MIN(Sl, R(0)), bR = GP_MAX(R(0), Sr);
    R scrh = R(1) / (bR - bL);
#pragma unroll
    for (int nv = 0; nv < 8; nv++) {
      flux[nv] = bL * bR * (ur[nv] - ul[nv]) + bR * fl[nv] - bL * fr[nv];
      flux[nv] *= scrh;
    }
  } else if (Sl >= R(0)) {
#pragma unroll
    for (int nv = 0; nv < 8; nv++) flux[nv] = fl[nv];
  } else if (Sr <= R(0)) {
#pragma unroll
    for (int nv = 0; nv < 8; nv++) flux[nv] = fr[nv];
  } else {
    int switch_to_hll = 0;
    R p0, f0, p, f, Sc;
    const R dS_1 = R(1) / (Sr - Sl);
    R Uhll[8];
    RState<R> PaL = {}, PaR = {};
#pragma unroll
    for (int nv = 0; nv < 8; nv++) {
      Uhll[nv] = Sr * ur[nv] - Sl * ul[nv] + fl[nv] - fr[nv];
      Uhll[nv] *= dS_1;
    }
    PaL.S = Sl;
    PaR.S = Sr;
    PaL.fail = 0;
    const R Bx = Uhll[BXn];
#pragma unroll
    for (int nv = 0; nv < 8; nv++) {
      PaL.Rr[nv] = Sl * ul[nv] - fl[nv];
      PaR.Rr[nv] = Sr * ur[nv] - fr[nv];
    }
    PaL.Rr[7] += PaL.Rr[RHO];
    PaR.Rr[7] += PaR.Rr[RHO];
    R scrh = GP_MAX(pl, pr);
    if (Bx * Bx / scrh < R(0.01)) {
      R a = Sr - Sl;
      R b = PaR.Rr[7] - PaL.Rr[7] + Sr * PaL.Rr[MXn] - Sl * PaR.Rr[MXn];
      R c = PaL.Rr[MXn] * PaR.Rr[7] - PaR.Rr[MXn] * PaL.Rr[7];
      scrh = b * b - R(4) * a * c;
      scrh = GP_MAX(scrh, R(0));
      p0 = R(0.5) * (-b + rsqrt_(scrh)) * dS_1;
    } else {
      double uh[8], vh[8];
#pragma unroll
      for (int nv = 0; nv < 8; nv++) uh[nv] = (double)Uhll[nv];
      uint32_t le = rmhd_cons2prim(uh, vh, (double)gamma, 1.e-12, 1.e-12);
      if (le) {
        err |= le;
        switch_to_hll = 1;
      }
      p0 = (R)hlld_total_pressure(vh);
    }
    // Secant iteration on the total pressure (MAX_ITER 20).  Pass 0 is the
    // initial guess p0 and pass k1 >= 1 the k1-th iterate, so the star-state
    // evaluation has one inlined copy.
    p = p0;
#pragma unroll 1
    for (int k1 = 0; k1 < 20; k1++) {
      f = hlld_fstar<DIR>(PaL, PaR, p, Bx, Sc);
      if (k1 == 0) {
        f0 = f;
        if (isnan((double)f0) || PaL.fail) switch_to_hll = 1;
        if (!(rabs(f0) > R(1.e-12) && !switch_to_hll)) break;  // p stays p0
        p = R(1.025) * p0;
        continue;
      }
      if (f != f || PaL.fail || (k1 > 7) || (rabs(f) > rabs(f0) && k1 > 4)) {
        switch_to_hll = 1;
        break;
      }
      R dp = (p - p0) / (f - f0) * f;
      p0 = p;
      f0 = f;
      p -= dp;
      if (p < R(0)) p = R(1.e-6);
      if (rabs(dp) < R(1.e-5) * p || rabs(f) < R(1.e-6)) break;
    }
    if (PaL.fail) switch_to_hll = 1;
    if (!switch_to_hll) {
      // both Alfven states (each depends only on its own side), one copy each
      hlld_astate<DIR>(PaL, p, Bx);
      hlld_astate<DIR>(PaR, p, Bx);
      if (PaL.Sa >= R(-1.e-6)) {
        PaL.u[7] -= PaL.u[RHO];
#pragma unroll
        for (int nv = 0; nv < 8; nv++) flux[nv] = fl[nv] + Sl * (PaL.u[nv] - ul[nv]);
      } else if (PaR.Sa <= R(1.e-6)) {
        PaR.u[7] -= PaR.u[RHO];
#pragma unroll
        for (int nv = 0; nv < 8; nv++) flux[nv] = fr[nv] + Sr * (PaR.u[nv] - ur[nv]);
      } else {
        R Uc[8];
        hlld_cstate<DIR>(PaL, PaR, p, Bx, Uc);
        if (Sc > R(0)) {
          PaL.u[7] -= PaL.u[RHO];
          Uc[7] -= Uc[RHO];
#pragma unroll
          for (int nv = 0; nv < 8; nv++)
            flux[nv] = fl[nv] + Sl * (PaL.u[nv] - ul[nv]) + PaL.Sa * (Uc[nv] - PaL.u[nv]);
        } else {
          PaR.u[7] -= PaR.u[RHO];
          Uc[7] -= Uc[RHO];
#pragma unroll
          for (int nv = 0; nv < 8; nv++)
            flux[nv] = fr[nv] + Sr * (PaR.u[nv] - ur[nv]) + PaR.Sa * (Uc[nv] - PaR.u[nv]);
        }
      }
    } else {
#pragma unroll
      for (int nv = 0; nv < 8; nv++) {
        flux[nv] = Sr * fl[nv] - Sl * fr[nv] + Sl * Sr * (ur[nv] - ul[nv]);
        flux[nv] *= dS_1;
      }
    }
  }
  ct_store_ucthll<DIR>(vl, vr, Sl, Sr, ct);
  return cmax;
}

// Relativistic velocity limiter, Src/vel_limiter.hpp:13-34: if either
// reconstructed state of a cell is superluminal, both become the cell value.
template <int NV, typename R>
__device__ __forceinline__ void rmhd_vel_limit(const R* vc, R* vr, R* vln) {
  R v2m = vr[VX1] * vr[VX1] + vr[VX1 + 1] * vr[VX1 + 1] + vr[VX1 + 2] * vr[VX1 + 2];
  R v2p = vln[VX1] * vln[VX1] + vln[VX1 + 1] * vln[VX1 + 1] + vln[VX1 + 2] * vln[VX1 + 2];
  if (v2m >= R(1) || v2p >= R(1)) {
#pragma unroll
    for (int nv = 0; nv < NV; nv++) vr[nv] = vln[nv] = vc[nv];
  }
}

}  // namespace gp
