// gp_crmath.cuh -- correctly rounded acos, sin and cos in double precision
// for the trigonometric root formula of the RMHD fast-speed quartic
// (Src/RMHD/rmhd.hpp:390-452: theta = acos(arg)/3, cos(theta), sin(theta)).
//
// Why: the reference calls the C library there.  Its fast-speed roots feed
// discontinuous decisions (the HLLD secant exit, the HLL fallback, the
// pressure fix), so a last-bit difference in these three functions changes a
// few cells by far more than round-off.  A correctly rounded result is the
// one target every accurate library approaches; against glibc 2.39 it
// differs in about 0.04% (acos) to 0.13% (sin) of the calls on these ranges,
// where CUDA's own functions (up to 2 ulp) differ far more often.
//
// Method (double-double arithmetic: Dekker 1971, Knuth TAOCP vol. 2 4.2.2;
// the normalisation and product steps of Hida, Li & Bailey, "Algorithms for
// quad-double precision floating point arithmetic", ARITH-15, 2001):
//
//  * sincos_cr(x), 0 <= x <= 1.125: x = j/16 + r with j = round(16 x), so
//    |r| <= 1/32 and r is exact (Sterbenz); sin r and cos r by their Taylor
//    series (double-double through the r^7 / r^6 terms, double beyond), then
//    the addition formulas with sin(j/16), cos(j/16) held as double-double
//    constants (computed to 300 bits).  Relative error about 2^-100.
//  * acos_cr(x), -1 <= x <= 1: one Newton step on sin(y) = s from the
//    library's asin (a few ulps), with s = x for |x| <= 1/2
//    (acos = pi/2 - asin x) and s = sqrt((1 -+ x)/2) as a double-double
//    otherwise (acos = 2 asin s, or pi - 2 asin s; 1 -+ x is exact there).
//    Newton's error is quadratic in the start error, ~2^-100 relative.
//
// The double-double value is rounded once; the result is the correctly
// rounded one unless the exact value lies within ~2^-47 ulp of a rounding
// midpoint.  That full-accuracy path is the slow path: each function first
// evaluates a fast form (the three leading terms exact, the rest in double,
// error below 2^-68 absolute or 2^-63 relative) and returns its rounding when
// every value within twice that error rounds the same way (Ziv's strategy,
// as in CRlibm); about one call in a thousand defers to the slow path.  The functions compile for the host as well, where the
// CPU tests check them against binary128 on dense argument sweeps.
#pragma once
#include <math.h>

#if defined(__CUDACC__)
#define GP_CR_FN __host__ __device__ __forceinline__
#define GP_CR_SLOW static __host__ __device__ __noinline__
#else
#define GP_CR_FN static inline
#define GP_CR_SLOW static
#endif

namespace gpcr {

struct dd {
  double hi, lo;
};

// |a| >= |b| or a == 0
GP_CR_FN dd fast_two_sum(double a, double b) {
  double s = a + b;
  double e = b - (s - a);
  return {s, e};
}
GP_CR_FN dd two_sum(double a, double b) {
  double s = a + b;
  double bb = s - a;
  double e = (a - (s - bb)) + (b - bb);
  return {s, e};
}
GP_CR_FN dd two_prod(double a, double b) {
  double p = a * b;
  double e = fma(a, b, -p);
  return {p, e};
}
GP_CR_FN dd dd_add(dd a, dd b) {
  dd s = two_sum(a.hi, b.hi);
  dd t = two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = fast_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return fast_two_sum(s.hi, s.lo);
}
GP_CR_FN dd dd_add_d(dd a, double b) {
  dd s = two_sum(a.hi, b);
  s.lo += a.lo;
  return fast_two_sum(s.hi, s.lo);
}
GP_CR_FN dd dd_neg(dd a) { return {-a.hi, -a.lo}; }
GP_CR_FN dd dd_mul(dd a, dd b) {
  dd p = two_prod(a.hi, b.hi);
  double c = fma(a.hi, b.lo, a.lo * b.hi);
  p.lo += c;
  return fast_two_sum(p.hi, p.lo);
}
GP_CR_FN dd dd_mul_d(dd a, double b) {
  dd p = two_prod(a.hi, b);
  p.lo = fma(a.lo, b, p.lo);
  return fast_two_sum(p.hi, p.lo);
}

// sin(j/16), its low part, cos(j/16), its low part; j = 0..18
#define GP_CR_TABLE                                                                       \
  {                                                                                       \
    {0x0.0p+0, 0x0.0p+0, 0x1.0000000000000p+0, 0x0.0p+0},                                 \
    {0x1.ffaaaeeed4edbp-5, -0x1.2d16d32684b69p-59, 0x1.ff0015549f4d3p-1, 0x1.328387b99426fp-55}, \
    {0x1.feaaeee86ee36p-4, -0x1.afcb2bcc6f03bp-59, 0x1.fc015527d5bd3p-1, 0x1.b68f35094efb8p-55}, \
    {0x1.7dc102fbaf2b5p-3, 0x1.5ab50e23c97c3p-59, 0x1.f706bdf9ece1cp-1, -0x1.698c80c36dcb4p-55}, \
    {0x1.faaeed4f31577p-3, -0x1.15d88508e32b8p-57, 0x1.f01549f7deea1p-1, 0x1.d3c1e99e5cafdp-55}, \
    {0x1.3ad129769d3d8p-2, 0x1.03d550487839ap-63, 0x1.e733ea0193d40p-1, -0x1.6428b3546ce13p-55}, \
    {0x1.7710255764214p-2, -0x1.6ead7314bb6cep-57, 0x1.dc6b7eb995912p-1, 0x1.4b364776dcd35p-58}, \
    {0x1.b1d8305321617p-2, -0x1.ae242cb99f519p-56, 0x1.cfc6cfa52ad9fp-1, 0x1.8b5b5508f2a0dp-55}, \
    {0x1.eaee8744b05f0p-2, -0x1.789b43c9b027dp-58, 0x1.c1528065b7d50p-1, -0x1.892111312e828p-55}, \
    {0x1.110d0c4b69c3bp-1, 0x1.d918998809981p-55, 0x1.b11d04162a4c6p-1, 0x1.1dd561efbc0c2p-56}, \
    {0x1.2b91dea88421ep-1, -0x1.fa371db216ab0p-55, 0x1.9f368ed912f85p-1, -0x1.1d200c5791606p-55}, \
    {0x1.44eb381cf386bp-1, -0x1.3ed6c1e6a5505p-55, 0x1.8bb105a5dc900p-1, 0x1.863e03e9474c1p-55}, \
    {0x1.5cffc16bf8f0dp-1, 0x1.96cb370eb578ap-55, 0x1.769fec655211fp-1, -0x1.827d5cf8c68c5p-57}, \
    {0x1.73b7680dea578p-1, -0x1.2248306dc12a2p-56, 0x1.6018526f563dfp-1, 0x1.46ca5e0e432d0p-55}, \
    {0x1.88fb7640b8da2p-1, -0x1.49987c11efaa3p-55, 0x1.4830bd7d4ceb3p-1, 0x1.df77ff20d5448p-55}, \
    {0x1.9cb6a9bbce64bp-1, -0x1.4f3e7a32f8d0cp-56, 0x1.2f011326420e4p-1, 0x1.8e30efe9e96c2p-56}, \
    {0x1.aed548f090ceep-1, 0x1.06374f484e288p-59, 0x1.14a280fb5068cp-1, -0x1.b71edcc9344bcp-55}, \
    {0x1.bf4536c24bb85p-1, 0x1.97632053703f0p-55, 0x1.f25ec6b852fc2p-2, 0x1.445cbca9a80a8p-56}, \
    {0x1.cdf604a1cadcep-1, -0x1.6b50757f2fa40p-56, 0x1.b9865639d0596p-2, -0x1.931bd06786cb9p-56}, \
  }

// Global rather than constant memory: the lanes of a warp index different
// entries, which the constant cache would serialise.
#if defined(__CUDACC__)
static __device__ const double kSinCosTable[19][4] = GP_CR_TABLE;
#endif
static const double kSinCosTableHost[19][4] = GP_CR_TABLE;

GP_CR_FN double sincos_tab(int j, int k) {
#if defined(__CUDA_ARCH__)
  return __ldg(&kSinCosTable[j][k]);
#else
  return kSinCosTableHost[j][k];
#endif
}
#define GP_CR_TAB_J(j, k) sincos_tab(j, k)

// double-double sin and cos of x in [0, 1.125]
GP_CR_FN void sincos_dd(double x, dd& s, dd& c) {
  const int j = (int)(x * 16.0 + 0.5);
  const double r = x - (double)j * 0.0625;
  const dd z = two_prod(r, r);
  // sin r = r + r z (-1/3! + z (1/5! + z (-1/7! + z t))),  t = 1/9! - z/11! + z^2/13!
  const double ts = fma(z.hi, fma(z.hi, 0x1.6124613a86d09p-33, -0x1.ae64567f544e4p-26),
                        0x1.71de3a556c734p-19);
  dd ps = dd_add_d({-0x1.a01a01a01a01ap-13, -0x1.a01a01a01a01ap-73}, z.hi * ts);
  ps = dd_add(dd_mul(z, ps), {0x1.1111111111111p-7, 0x1.1111111111111p-63});
  ps = dd_add(dd_mul(z, ps), {-0x1.5555555555555p-3, -0x1.5555555555555p-57});
  const dd sr = dd_add_d(dd_mul_d(dd_mul(z, ps), r), r);
  // cos r = 1 + z (-1/2 + z (1/4! + z (-1/6! + z t))),  t = 1/8! - z/10! + z^2/12! - z^3/14!
  const double tc = fma(z.hi, fma(z.hi, fma(z.hi, -0x1.93974a8c07c9dp-37, 0x1.1eed8eff8d898p-29),
                                  -0x1.27e4fb7789f5cp-22),
                        0x1.a01a01a01a01ap-16);
  dd pc = dd_add_d({-0x1.6c16c16c16c17p-10, 0x1.f49f49f49f49fp-65}, z.hi * tc);
  pc = dd_add(dd_mul(z, pc), {0x1.5555555555555p-5, 0x1.5555555555555p-59});
  pc = dd_add(dd_mul(z, pc), {-0.5, 0.0});
  const dd cr = dd_add_d(dd_mul(z, pc), 1.0);
  const dd sj = {GP_CR_TAB_J(j, 0), GP_CR_TAB_J(j, 1)};
  const dd cj = {GP_CR_TAB_J(j, 2), GP_CR_TAB_J(j, 3)};
  s = dd_add(dd_mul(sj, cr), dd_mul(cj, sr));
  c = dd_add(dd_mul(cj, cr), dd_neg(dd_mul(sj, sr)));
}

// ---------------------------------------------------------------------
// Full-accuracy paths (relative error ~2^-100), out of line: taken only when
// the fast paths below cannot decide the rounding.
// ---------------------------------------------------------------------
#if defined(GP_CR_COUNT_SLOW) && !defined(__CUDA_ARCH__)
extern long gp_cr_slow_calls;  // host test builds: how often the fast path defers
#define GP_CR_NOTE_SLOW() (++gp_cr_slow_calls)
#else
#define GP_CR_NOTE_SLOW() ((void)0)
#endif

GP_CR_SLOW void sincos_slow(double x, double* sn, double* cs) {
  GP_CR_NOTE_SLOW();
  dd s, c;
  sincos_dd(x, s, c);
  *sn = s.hi + s.lo;
  *cs = c.hi + c.lo;
}

// asin(s) as a double-double for s (double-double) in [-1/2, 1/2]
GP_CR_FN dd asin_dd(dd s) {
  const double y0 = asin(s.hi);
  const double ay = fabs(y0);
  dd sy, cy;
  sincos_dd(ay, sy, cy);
  if (y0 < 0.0) sy = dd_neg(sy);
  const dd e = dd_add(s, dd_neg(sy));            // s - sin(y0), a few ulps of s
  const double delta = (e.hi + e.lo) / cy.hi;    // Newton step
  return two_sum(y0, delta);
}

GP_CR_SLOW double acos_slow(double x) {
  GP_CR_NOTE_SLOW();
  const dd kPi = {0x1.921fb54442d18p+1, 0x1.1a62633145c07p-53};
  const dd kPi2 = {0x1.921fb54442d18p+0, 0x1.1a62633145c07p-54};
  if (fabs(x) <= 0.5) {
    const dd r = dd_add(kPi2, dd_neg(asin_dd({x, 0.0})));
    return r.hi + r.lo;
  }
  const double t = (x > 0.0 ? 1.0 - x : 1.0 + x) * 0.5;   // exact
  const double sh = sqrt(t);
  const double sl = sh > 0.0 ? fma(-sh, sh, t) / (2.0 * sh) : 0.0;
  dd y = asin_dd(fast_two_sum(sh, sl));
  y = {2.0 * y.hi, 2.0 * y.lo};
  if (x < 0.0) y = dd_add(kPi, dd_neg(y));
  return y.hi + y.lo;
}

// ---------------------------------------------------------------------
// Fast paths (Ziv's strategy): evaluate with a proven error bound, and
// return the double nearest to the result only when every value within that
// bound rounds to it; otherwise fall back to the full-accuracy path.
// ---------------------------------------------------------------------

// The double nearest to y when every value within err of y rounds the same
// way (y = hi + lo normalised; rounding is monotonic, so both ends suffice).
GP_CR_FN bool round_certain(dd y, double err, double* out) {
  const double a = y.hi + (y.lo + err);
  const double b = y.hi + (y.lo - err);
  *out = a;
  return a == b;
}

// sin and cos of x in [0, 1.125] as unevaluated sums.  With j = round(16 x),
// r = x - j/16 (exact, |r| <= 1/32), z = r^2 = zh + zl (exact),
// cm = cos r - 1 = -zh/2 + cml and sm = sin r - r:
//   sin x = Sj + Cj r + Sj (-zh/2) + [rest], cos x = Cj - Sj r + Cj (-zh/2) + [rest]
// where the three leading terms are formed exactly (Dekker products, Knuth
// sums) and the rest (below 2^-17) in double.  Error: for j >= 1 below 2^-68
// absolute for both (the double products Cj*sm, Sj*sm and sm's own rounding
// dominate: |sm| <= 2^-17.6, three roundings); for j = 0 (x < 1/32, Sj = 0,
// Cj = 1) sin x = r + sm to 2^-63 relative and cos x = 1 - zh/2 + cml to
// 2^-75.  Measured against binary128 on 4 million arguments: 2^-68.7
// absolute (j >= 1, sin and cos), 2^-64.2 relative (j = 0, sin).  Returned
// with the bounds the rounding test uses: 2^-67 absolute, 2^-62 relative.
GP_CR_FN void sincos_fast(double x, dd& s, dd& c, double& es, double& ec) {
  const int j = (int)(x * 16.0 + 0.5);
  const double r = x - (double)j * 0.0625;
  const dd z = two_prod(r, r);
  const double zh = z.hi;
  // cm = -z/2 + z^2 (1/4! - z/6! + z^2/8! - z^3/10!)
  const double q = fma(zh, fma(zh, fma(zh, -0x1.27e4fb7789f5cp-22, 0x1.a01a01a01a01ap-16),
                               -0x1.6c16c16c16c17p-10),
                       0x1.5555555555555p-5);
  const double cmh = -0.5 * zh;                    // exact
  const double cml = fma(zh * zh, q, -0.5 * z.lo);
  // sm = r z (-1/3! + z (1/5! - z/7! + z^2/9!))
  const double p = fma(zh, fma(zh, fma(zh, 0x1.71de3a556c734p-19, -0x1.a01a01a01a01ap-13),
                               0x1.1111111111111p-7),
                       -0x1.5555555555555p-3);
  const double sm = r * fma(zh, p, z.lo * -0x1.5555555555555p-3);
  const double Sh = GP_CR_TAB_J(j, 0), Sl = GP_CR_TAB_J(j, 1);
  const double Ch = GP_CR_TAB_J(j, 2), Cl = GP_CR_TAB_J(j, 3);
  {  // sin
    const dd a = two_prod(Ch, r);
    const dd b = two_prod(Sh, cmh);
    const dd t1 = two_sum(Sh, a.hi);
    const dd t2 = two_sum(t1.hi, b.hi);
    double rest = a.lo + b.lo;
    rest += Sl;
    rest += Sh * cml;
    rest += Cl * r;
    rest += Sl * cmh;
    rest += Cl * sm;
    rest += t1.lo + t2.lo;
    rest += Ch * sm;
    s = fast_two_sum(t2.hi, rest);
  }
  {  // cos
    const dd a = two_prod(Sh, r);
    const dd b = two_prod(Ch, cmh);
    const dd t1 = two_sum(Ch, -a.hi);
    const dd t2 = two_sum(t1.hi, b.hi);
    double rest = b.lo - a.lo;
    rest += Cl;
    rest += Ch * cml;
    rest -= Sl * r;
    rest += Cl * cmh;
    rest -= Sl * sm;
    rest += t1.lo + t2.lo;
    rest -= Sh * sm;
    c = fast_two_sum(t2.hi, rest);
  }
  es = j == 0 ? 0x1p-62 * fabs(s.hi) : 0x1p-67;
  ec = 0x1p-67;
}

// sin(x) as in sincos_fast (same terms, same bound es) and cos(x) to double
// precision only: the Newton step of acos_cr divides by it, where relative
// accuracy 2^-50 is ample.
GP_CR_FN void sin_fast_cos_d(double x, dd& s, double& es, double& cd) {
  const int j = (int)(x * 16.0 + 0.5);
  const double r = x - (double)j * 0.0625;
  const dd z = two_prod(r, r);
  const double zh = z.hi;
  const double q = fma(zh, fma(zh, fma(zh, -0x1.27e4fb7789f5cp-22, 0x1.a01a01a01a01ap-16),
                               -0x1.6c16c16c16c17p-10),
                       0x1.5555555555555p-5);
  const double cmh = -0.5 * zh;
  const double cml = fma(zh * zh, q, -0.5 * z.lo);
  const double p = fma(zh, fma(zh, fma(zh, 0x1.71de3a556c734p-19, -0x1.a01a01a01a01ap-13),
                               0x1.1111111111111p-7),
                       -0x1.5555555555555p-3);
  const double sm = r * fma(zh, p, z.lo * -0x1.5555555555555p-3);
  const double Sh = GP_CR_TAB_J(j, 0), Sl = GP_CR_TAB_J(j, 1);
  const double Ch = GP_CR_TAB_J(j, 2), Cl = GP_CR_TAB_J(j, 3);
  const dd a = two_prod(Ch, r);
  const dd b = two_prod(Sh, cmh);
  const dd t1 = two_sum(Sh, a.hi);
  const dd t2 = two_sum(t1.hi, b.hi);
  double rest = a.lo + b.lo;
  rest += Sl;
  rest += Sh * cml;
  rest += Cl * r;
  rest += Sl * cmh;
  rest += Cl * sm;
  rest += t1.lo + t2.lo;
  rest += Ch * sm;
  s = fast_two_sum(t2.hi, rest);
  es = j == 0 ? 0x1p-62 * fabs(s.hi) : 0x1p-67;
  cd = Ch + (Ch * (cmh + cml) - Sh * (r + sm));
}

// correctly rounded sin(x) and cos(x), 0 <= x <= 1.125
GP_CR_FN void sincos_cr(double x, double* sn, double* cs) {
  dd s, c;
  double es, ec;
  sincos_fast(x, s, c, es, ec);
  const bool ok = round_certain(s, es, sn) & round_certain(c, ec, cs);
  if (!ok) sincos_slow(x, sn, cs);
}

// correctly rounded acos(x), -1 <= x <= 1: the Newton step of asin_dd on the
// fast sin (its error carried through: |d asin / d sin| = 1/cos <= 1.16 on
// [-1/2, 1/2], doubled where acos = 2 asin), then the rounding test.
GP_CR_FN double acos_cr(double x) {
  const double kPih = 0x1.921fb54442d18p+1, kPil = 0x1.1a62633145c07p-53;
  const double kPi2h = 0x1.921fb54442d18p+0, kPi2l = 0x1.1a62633145c07p-54;
  const bool mid = fabs(x) <= 0.5;
  double sh, sl;
  if (mid) {
    sh = x;
    sl = 0.0;
  } else {
    const double t = (x > 0.0 ? 1.0 - x : 1.0 + x) * 0.5;   // exact
    sh = sqrt(t);
    sl = sh > 0.0 ? fma(-sh, sh, t) / (2.0 * sh) : 0.0;
  }
  const double y0 = asin(sh);
  dd sy;
  double es, cy;
  sin_fast_cos_d(fabs(y0), sy, es, cy);
  if (y0 < 0.0) sy = dd_neg(sy);
  // s - sin(y0): the high parts are within a few ulps (exact difference)
  const double e = (sh - sy.hi) + (sl - sy.lo);
  const double delta = e / cy;
  dd y;
  double err = 1.25 * es;
  if (mid) {
    const dd t = two_sum(kPi2h, -y0);
    y = fast_two_sum(t.hi, (t.lo - delta) + kPi2l);
  } else if (x > 0.0) {
    y = fast_two_sum(2.0 * y0, 2.0 * delta);
    err *= 2.0;
  } else {
    const dd t = two_sum(kPih, -2.0 * y0);
    y = fast_two_sum(t.hi, (t.lo - 2.0 * delta) + kPil);
    err *= 2.0;
  }
  // + the Newton step's own terms (quadratic in a few ulps, relative)
  err += 0x1p-98 * fabs(y.hi);
  double r;
  if (round_certain(y, err, &r)) return r;
  return acos_slow(x);
}

}  // namespace gpcr
