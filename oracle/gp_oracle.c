/*
 * gp_oracle.c -- CPU restatement of the gPLUTO Godunov step (TEST
 * INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
 * bench's cpu_baseline leg as the checker; never linked into the product).
 *
 * Plain C, straight loops over ghost-zone arrays, in the reference's own
 * operation order so that results agree bit for bit with the reference
 * serial build (Config/linux.g++.defs, g++ -O3 on x86-64 without FMA
 * contraction).  Compile with -ffp-contract=off and no fast-math.
 *
 * Scope: Cartesian uniform grid, periodic boundaries, PLM reconstruction
 * (MC / van Leer / minmod), RK2, ideal EOS, physics HD (HLLC, HLL),
 * MHD (HLLD, HLL) with constrained transport (UCT_HLLD, UCT_HLL), RMHD
 * (HLLD, HLL, UCT_HLL) with the Newton energy inversion.
 *
 * Each function cites the reference source it restates (paths relative to
 * the gPLUTO tree).  Parity is pinned against the reference binary through
 * the committed fixtures in tests/golden/.
 */
#include <math.h>
#include <quadmath.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "gp_oracle.h"

#define MAX(a,b)  ( (a) >= (b) ? (a) : (b) )      /* Src/macros.hpp:191 */
#define MIN(a,b)  ( (a) <= (b) ? (a) : (b) )      /* Src/macros.hpp:194 */
#define ABS_MIN(a,b)  (fabs(a) < fabs(b) ? (a):(b))   /* Src/macros.hpp:14 */
#define MINMOD_LIMITER(a,b)  ((a)*(b) > 0.0 ? (fabs(a) < fabs(b) ? (a):(b)):0.0)

/* variable indices: MHD/RMHD (Src/MHD/mhd.hpp:21-33), HD (Src/HD/hd.hpp:21-27) */
enum { RHO = 0, MX1 = 1, MX2 = 2, MX3 = 3, BX1 = 4, BX2 = 5, BX3 = 6 };
#define VX1 MX1

/* error bits, Src/gpluto.hpp:247-262 */
#define ERR_NEGATIVE_RHO   (1u<<0)
#define ERR_NEGATIVE_ENG   (1u<<1)
#define ERR_NEGATIVE_PRS   (1u<<2)
#define ERR_CONS2PRIM_FAIL (1u<<4)
#define ERR_ENG_SOLVE_INACCURATE  (1u<<6)
#define ERR_ENG_SOLVE_NO_SOLUTION (1u<<7)
#define ERR_SUPERLUMINAL_SPEED    (1u<<8)
#define ERR_TOO_MANY_ITERATIONS   (1u<<9)
#define ERR_NAN            (1u<<11)
#define ERR_QUIT           (1u<<15)

typedef struct {
  orc_cfg c;
  int nvar, eng, ng;
  int nt[3], beg[3], end[3];
  long ncell;
  double *Vc, *Uc, *U0, *Rc, *Cdt;
  double *Vs[3], *Bs0[3], *Rs[3];
  int ns[3][3];
  /* CT face data, indexed on a (nt+1)^3 box */
  int ne[3];
  double *e[3][3], *aL[3], *aR[3], *dL[3], *dR[3], *Ee[3];
  double *sv[3];   /* CT_CONTACT: sign of the face's mass flux */
  /* pencil buffers */
  int pmax;
  double *pv, *pvL, *pvR, *pflux, *pcmax, *pBn, *pq, *pqL, *pqR;
  uint32_t err;
} orc_t;

static void orc_rmhd_init(orc_t *o);
static double orc_rmhd_riemann(orc_t *o, int dir, double *vl, double *vr, double *f, long e);
static uint32_t orc_rmhd_cons_to_prim(orc_t *o, double *u, double *v, int i, int j, int k);
static void orc_rmhd_prim_to_cons(const double *v, double *u, double gamma);

/* ------------------------------------------------------------------ */
/* indexing                                                            */
/* ------------------------------------------------------------------ */
static inline long CI(const orc_t *o, int i, int j, int k) {
  return ((long)k*o->nt[1] + j)*o->nt[0] + i;
}
static inline double *VC(orc_t *o, double *A, int nv, int i, int j, int k) {
  return A + (long)nv*o->ncell + CI(o, i, j, k);
}
static inline long SI(const orc_t *o, int d, int i, int j, int k) {
  return ((long)k*o->ns[d][1] + j)*o->ns[d][0] + i;
}
static inline long EI(const orc_t *o, int i, int j, int k) {
  return ((long)k*o->ne[1] + j)*o->ne[0] + i;
}
/* map pencil coordinates (along dir) to (i,j,k): Src/macros.hpp ARRAY_STRIDES,
   RBoxPermuteIndices (dir=IDIR: (i,j,k); JDIR: (j,i,k); KDIR: (j,k,i)) */
static inline void TrueIdx(int dir, int i, int t1, int t2, int *ti, int *tj, int *tk) {
  if (dir == 0) { *ti = i;  *tj = t1; *tk = t2; }
  else if (dir == 1) { *ti = t1; *tj = i;  *tk = t2; }
  else { *ti = t1; *tj = t2; *tk = i; }
}

/* ------------------------------------------------------------------ */
/* physics: MHD                                                        */
/* ------------------------------------------------------------------ */

/* Src/MHD/mhd.hpp:906-948 */
static void MHD_PrimToCons(const double *v, double *u, double gamma) {
  double gmm1 = gamma - 1.0, kinb2;
  u[RHO] = v[RHO];
  u[MX1] = v[RHO]*v[VX1];
  u[MX2] = v[RHO]*v[VX1+1];
  u[MX3] = v[RHO]*v[VX1+2];
  u[BX1] = v[BX1]; u[BX2] = v[BX2]; u[BX3] = v[BX3];
  kinb2  = v[VX1]*v[VX1] + v[VX1+1]*v[VX1+1] + v[VX1+2]*v[VX1+2];
  kinb2  = v[RHO]*kinb2  + v[BX1]*v[BX1] + v[BX2]*v[BX2] + v[BX3]*v[BX3];
  kinb2 *= 0.5;
  u[7] = kinb2 + v[7]/gmm1;
}

/* Src/HD/hd.hpp:392-416 */
static void HD_PrimToCons(const double *v, double *u, double gamma) {
  double kin;
  u[RHO] = v[RHO];
  u[MX1] = v[RHO]*v[VX1];
  u[MX2] = v[RHO]*v[VX1+1];
  u[MX3] = v[RHO]*v[VX1+2];
  kin    = v[VX1]*v[VX1] + v[VX1+1]*v[VX1+1] + v[VX1+2]*v[VX1+2];
  kin    = v[RHO]*kin*0.5;
  u[4]   = kin + v[4]/(gamma - 1.0);
}

/* Src/MHD/mappers.cpp:32-150 (ENERGY_SOLVE branch) */
static uint32_t MHD_ConsToPrim(double *u, double *v, double gamma, double small_rho, double small_prs) {
  uint32_t err = 0;
  double gmm1 = gamma - 1.0, tau, m2, b2, kinb2;
  if (u[RHO] < 0.0) { u[RHO] = small_rho; err |= ERR_NEGATIVE_RHO | ERR_CONS2PRIM_FAIL; }
  v[RHO] = u[RHO];
  tau    = 1.0/u[RHO];
  v[VX1]   = u[MX1]*tau;
  v[VX1+1] = u[MX2]*tau;
  v[VX1+2] = u[MX3]*tau;
  v[BX1] = u[BX1]; v[BX2] = u[BX2]; v[BX3] = u[BX3];
  m2 = u[MX1]*u[MX1] + u[MX2]*u[MX2] + u[MX3]*u[MX3];
  b2 = u[BX1]*u[BX1] + u[BX2]*u[BX2] + u[BX3]*u[BX3];
  kinb2 = 0.5*(m2*tau + b2);
  if (u[7] > 0.0) {
    v[7] = gmm1*(u[7] - kinb2);
    if (v[7] < 0.0) {
      v[7] = small_prs;
      u[7] = v[7]/gmm1 + kinb2;
      err |= ERR_NEGATIVE_PRS;
    }
  } else {
    u[7] = small_prs/gmm1 + kinb2;
    v[7] = small_prs;
    err |= ERR_NEGATIVE_ENG;
  }
  return err;
}

/* Src/HD/mappers.cpp:33-140 (ENERGY_SOLVE branch) */
static uint32_t HD_ConsToPrim(double *u, double *v, double gamma, double small_rho, double small_prs) {
  uint32_t err = 0;
  double gmm1 = gamma - 1.0, tau, m2, kin;
  if (u[RHO] < 0.0) { u[RHO] = small_rho; err |= ERR_NEGATIVE_RHO | ERR_CONS2PRIM_FAIL; }
  v[RHO] = u[RHO];
  tau    = 1.0/u[RHO];
  v[VX1]   = u[MX1]*tau;
  v[VX1+1] = u[MX2]*tau;
  v[VX1+2] = u[MX3]*tau;
  m2  = u[MX1]*u[MX1] + u[MX2]*u[MX2] + u[MX3]*u[MX3];
  kin = 0.5*m2*tau;
  if (u[4] > 0.0) {
    v[4] = gmm1*(u[4] - kin);
    if (v[4] < 0.0) {
      v[4] = small_prs;
      u[4] = v[4]/gmm1 + kin;
      err |= ERR_NEGATIVE_PRS;
    }
  } else {
    u[4] = small_prs/gmm1 + kin;
    v[4] = small_prs;
    err |= ERR_NEGATIVE_ENG;
  }
  return err;
}

/* Src/MHD/mhd.hpp:163-223 (no background field) */
static void MHD_Flux(int dir, const double *v, const double *u, double *flux, double *pt) {
  int VXn = VX1 + dir, BXn = BX1 + dir, MXn = MX1 + dir;
  double vB = v[VX1]*v[BX1] + v[VX1+1]*v[BX2] + v[VX1+2]*v[BX3];
  *pt = v[7] + 0.5*(v[BX1]*v[BX1] + v[BX2]*v[BX2] + v[BX3]*v[BX3]);
  flux[RHO] = u[MXn];
  flux[MX1] = u[MX1]*v[VXn] - v[BX1]*v[BXn];
  flux[MX2] = u[MX2]*v[VXn] - v[BX2]*v[BXn];
  flux[MX3] = u[MX3]*v[VXn] - v[BX3]*v[BXn];
  flux[BX1] = v[BX1]*v[VXn] - v[BXn]*v[VX1];
  flux[BX2] = v[BX2]*v[VXn] - v[BXn]*v[VX1+1];
  flux[BX3] = v[BX3]*v[VXn] - v[BXn]*v[VX1+2];
  flux[7]   = (u[7] + *pt)*v[VXn] - v[BXn]*vB;
  flux[MXn] += *pt;
}

/* Src/HD/hd.hpp:105-125 */
static void HD_Flux(int dir, const double *v, const double *u, double *flux, double *p) {
  int VXn = VX1 + dir, MXn = MX1 + dir;
  flux[RHO] = u[MXn];
  flux[MX1] = u[MX1]*v[VXn];
  flux[MX2] = u[MX2]*v[VXn];
  flux[MX3] = u[MX3]*v[VXn];
  flux[4] = (u[4] + v[4])*v[VXn];
  *p = v[4];
  flux[MXn] += *p;
}

/* Src/MHD/mhd.hpp:241-277 (MaxSignalSpeed) with a2 from Src/eos.hpp:96 */
static void MHD_MaxSignalSpeed(int dir, const double *v, double a2, double *cmin, double *cmax) {
  int VXn = VX1 + dir;
  double b1 = v[BX1 + dir], b2 = v[BX1 + (dir+1)%3], b3 = v[BX1 + (dir+2)%3];
  double gpr = a2*v[RHO];
  double Btmag2 = b2*b2 + b3*b3;
  double Bmag2  = b1*b1 + Btmag2;
  double cf = gpr - Bmag2;
  cf = gpr + Bmag2 + sqrt(cf*cf + 4.0*gpr*Btmag2);
  cf = sqrt(0.5*cf/v[RHO]);
  *cmax = v[VXn] + cf;
  *cmin = v[VXn] - cf;
}

/* Src/HD/hd.hpp:139-150 */
static void HD_MaxSignalSpeed(int dir, const double *v, double a2, double *cmin, double *cmax) {
  double a = sqrt(a2);
  *cmax = v[VX1+dir] + a;
  *cmin = v[VX1+dir] - a;
}

/* ------------------------------------------------------------------ */
/* CT store (Src/MHD/CT/ct_store.hpp)                                  */
/* ------------------------------------------------------------------ */

/* Src/MHD/CT/ct_store.hpp:154-177 */
static void CT_Store_UCTHll(orc_t *o, int dir, const double *vl, const double *vr,
                            double Sl, double Sr, long e) {
  int VXt = VX1 + (dir+1)%3, VXb = VX1 + (dir+2)%3;
  int DIRt = (dir+1)%3, DIRb = (dir+2)%3;
  double aR_1 = MAX(0.0, Sr);
  double aL_1 = MIN(0.0, Sl);
  double scrh = 1.0/(aR_1 - aL_1);
  o->e[DIRb][dir][e] =  (aR_1*vl[VXt] - aL_1*vr[VXt])*scrh;
  o->e[DIRt][dir][e] = -(aR_1*vl[VXb] - aL_1*vr[VXb])*scrh;
  o->aL[dir][e] =  aR_1*scrh;
  o->aR[dir][e] = -aL_1*scrh;
  o->dR[dir][e] = -aL_1*aR_1*scrh;
  o->dL[dir][e] = -aL_1*aR_1*scrh;
}

/* Src/MHD/CT/ct_store.hpp:252-355 (EOS IDEAL) */
static void CT_Store_UCTHlld(orc_t *o, int dir, const double *ul, const double *ur,
                             const double *vl, const double *vr, double Sl, double Sr,
                             double Bn, long e) {
  int VXn = VX1 + dir, VXt = VX1 + (dir+1)%3, VXb = VX1 + (dir+2)%3;
  int MXn = MX1 + dir;
  int DIRt = (dir+1)%3, DIRb = (dir+2)%3;
  int switch_to_hll = 0;
  double scrh;
  double aR_1 = MAX(0.0, Sr);
  double aL_1 = MIN(0.0, Sl);
  double dul = Sl - vl[VXn];
  double dur = Sr - vr[VXn];
  double pL = vl[7] + 0.5*(vl[BX1]*vl[BX1] + vl[BX2]*vl[BX2] + vl[BX3]*vl[BX3]);
  double pR = vr[7] + 0.5*(vr[BX1]*vr[BX1] + vr[BX2]*vr[BX2] + vr[BX3]*vr[BX3]);
  scrh  = 1.0/(dur*ur[RHO] - dul*ul[RHO]);
  double Sc = (dur*ur[MXn] - dul*ul[MXn] - pR + pL)*scrh;
  double usl_RHO = ul[RHO]*dul/(Sl - Sc);
  double usr_RHO = ur[RHO]*dur/(Sr - Sc);
  if (usl_RHO < 0.0 || usr_RHO < 0.0) switch_to_hll = 1;
  double sqrL = sqrt(usl_RHO);
  double sqrR = sqrt(usr_RHO);
  double Sal = Sc - fabs(Bn)/sqrL;
  double Sar = Sc + fabs(Bn)/sqrR;
  double chiL  = (vl[VXn] - Sc)*(Sl - Sc)/(Sal + Sl - 2.0*Sc);
  double chiR  = (vr[VXn] - Sc)*(Sr - Sc)/(Sar + Sr - 2.0*Sc);
  double nuL  = (Sal + Sl)/(fabs(Sal) + fabs(Sl));
  double nuR  = (Sar + Sr)/(fabs(Sar) + fabs(Sr));
  double nuLR = (Sal + Sar)/(fabs(Sal) + fabs(Sar));
  if (fabs(Sar - Sal) > 1.e-9*fabs(Sr-Sl)) {
    o->dL[dir][e] = 0.5*(chiL*nuL - chiL*nuLR) + 0.5*(fabs(Sal) - nuLR*Sal);
    o->dR[dir][e] = 0.5*(chiR*nuR - chiR*nuLR) + 0.5*(fabs(Sar) - nuLR*Sar);
    o->aL[dir][e] = 0.5*(1.0 + nuLR);
    o->aR[dir][e] = 0.5*(1.0 - nuLR);
  } else {
    o->dL[dir][e] = 0.5*chiL*nuL + 0.5*fabs(Sal);
    o->dR[dir][e] = 0.5*chiR*nuR + 0.5*fabs(Sar);
    o->aL[dir][e] = 0.5;
    o->aR[dir][e] = 0.5;
  }
  scrh = 1.0/(aR_1 - aL_1);
  if (switch_to_hll) {
    o->aL[dir][e] =  aR_1*scrh;
    o->aR[dir][e] = -aL_1*scrh;
    o->dR[dir][e] = -aL_1*aR_1*scrh;
    o->dL[dir][e] = -aL_1*aR_1*scrh;
  }
  o->e[DIRb][dir][e] =  (aR_1*vl[VXt] - aL_1*vr[VXt])*scrh;
  o->e[DIRt][dir][e] = -(aR_1*vl[VXb] - aL_1*vr[VXb])*scrh;
}

/* ------------------------------------------------------------------ */
/* Riemann solvers                                                     */
/* ------------------------------------------------------------------ */

/* Src/MHD/hlld.cpp:61-514 (ideal EOS, no background field, no GLM).
   Returns cmax; writes flux[NVAR]. */
static double MHD_HLLD(orc_t *o, int dir, double *vl, double *vr, double *flux, long e,
                       double Bn_face) {
  const double gamma = o->c.gamma;
  int VXn = VX1 + dir, VXt = VX1 + (dir+1)%3, VXb = VX1 + (dir+2)%3;
  int MXn = MX1 + dir, MXt = MX1 + (dir+1)%3, MXb = MX1 + (dir+2)%3;
  int BXn = BX1 + dir, BXt = BX1 + (dir+1)%3, BXb = BX1 + (dir+2)%3;
  int nv, switch_to_hll = 0;
  double ul[8], ur[8], fl[8], fr[8], usl[8], usr[8], Uhll[8];
  double Sl, Sr, ptl, ptr, sqrL, sqrR, cmax;

  MHD_PrimToCons(vl, ul, gamma);
  MHD_PrimToCons(vr, ur, gamma);
  double a2L = gamma*vl[7]/vl[RHO];       /* Src/eos.hpp:96 */
  double a2R = gamma*vr[7]/vr[RHO];
  {
    double sl_min, sl_max, sr_min, sr_max;  /* Src/MHD/mhd.hpp:295-308 */
    MHD_MaxSignalSpeed(dir, vl, a2L, &sl_min, &sl_max);
    MHD_MaxSignalSpeed(dir, vr, a2R, &sr_min, &sr_max);
    Sl = MIN(sl_min, sr_min);
    Sr = MAX(sl_max, sr_max);
  }
  cmax = MAX(fabs(Sl), fabs(Sr));
  MHD_Flux(dir, vl, ul, fl, &ptl);
  MHD_Flux(dir, vr, ur, fr, &ptr);

  double dul, dur, Bx, Bx1, sBx, pts, SM;
  {
    double scrh = 1.0/(Sr - Sl);
    Bx1 = Bx = (Sr*vr[BXn] - Sl*vl[BXn])*scrh;
    sBx = (Bx > 0.0 ? 1.0 : -1.0);
    dul = Sl - vl[VXn];
    dur = Sr - vr[VXn];
    scrh = 1.0/(dur*ur[RHO] - dul*ul[RHO]);
    SM = (dur*ur[MXn] - dul*ul[MXn] - ptr + ptl)*scrh;
    pts = dur*ur[RHO]*ptl - dul*ul[RHO]*ptr + vl[RHO]*vr[RHO]*dur*dul*(vr[VXn] - vl[VXn]);
    pts *= scrh;
  }
  usl[RHO] = ul[RHO]*dul/(Sl - SM);
  usr[RHO] = ur[RHO]*dur/(Sr - SM);
  if (usl[RHO] < 0.0 || usr[RHO] < 0.0) switch_to_hll = 1;
  sqrL = sqrt(usl[RHO]);
  sqrR = sqrt(usr[RHO]);
  double S1L = SM - fabs(Bx)/sqrL;
  double S1R = SM + fabs(Bx)/sqrR;

  if (Sl >= 0.0) {
    for (nv = 0; nv < 8; nv++) flux[nv] = fl[nv];
  } else if (Sr <= 0.0) {
    for (nv = 0; nv < 8; nv++) flux[nv] = fr[nv];
  } else {
    if (!switch_to_hll) {
      int switch_to_hllc = 0;
      if ((S1L - Sl) <  1.e-4*(SM - Sl)) switch_to_hllc = 1;
      if ((S1R - Sr) > -1.e-4*(Sr - SM)) switch_to_hllc = 1;
      double scrhL, scrhR;
      if (!switch_to_hllc) {
        scrhL = (ul[RHO]*dul*dul - Bx*Bx)/(ul[RHO]*dul*(Sl - SM) - Bx*Bx);
        scrhR = (ur[RHO]*dur*dur - Bx*Bx)/(ur[RHO]*dur*(Sr - SM) - Bx*Bx);
        usl[BXn] = Bx1;
        usl[BXt] = ul[BXt]*scrhL;
        usl[BXb] = ul[BXb]*scrhL;
        usr[BXn] = Bx1;
        usr[BXt] = ur[BXt]*scrhR;
        usr[BXb] = ur[BXb]*scrhR;
      } else {
        double scrh = 1.0/(Sr - Sl);
        for (nv = 0; nv < 8; nv++) {
          Uhll[nv]  = Sr*ur[nv] - Sl*ul[nv] + fl[nv] - fr[nv];
          Uhll[nv] *= scrh;
        }
        usl[BXn] = usr[BXn] = Bx1;
        usl[BXt] = usr[BXt] = Uhll[BXt];
        usl[BXb] = usr[BXb] = Uhll[BXb];
        S1L = S1R = SM;
      }
      scrhL = Bx/(ul[RHO]*dul);
      scrhR = Bx/(ur[RHO]*dur);
      double vsL = vl[VXt] - scrhL*(usl[BXt] - ul[BXt]);
      double vsR = vr[VXt] - scrhR*(usr[BXt] - ur[BXt]);
      double wsL = vl[VXb] - scrhL*(usl[BXb] - ul[BXb]);
      double wsR = vr[VXb] - scrhR*(usr[BXb] - ur[BXb]);
      usl[MXn] = usl[RHO]*SM;
      usr[MXn] = usr[RHO]*SM;
      usl[MXt] = usl[RHO]*vsL;
      usr[MXt] = usr[RHO]*vsR;
      usl[MXb] = usl[RHO]*wsL;
      usr[MXb] = usr[RHO]*wsR;
      scrhL  = vl[VXn]*Bx1 + vl[VXt]*ul[BXt] + vl[VXb]*ul[BXb];
      scrhL -= SM*Bx1 + vsL*usl[BXt] + wsL*usl[BXb];
      usl[7]  = dul*ul[7] - ptl*vl[VXn] + pts*SM + Bx*scrhL;
      usl[7] /= Sl - SM;
      scrhR  = vr[VXn]*Bx1 + vr[VXt]*ur[BXt] + vr[VXb]*ur[BXb];
      scrhR -= SM*Bx1 + vsR*usr[BXt] + wsR*usr[BXb];
      usr[7]  = dur*ur[7] - ptr*vr[VXn] + pts*SM + Bx*scrhR;
      usr[7] /= Sr - SM;

      if (S1L >= 0.0) {
        for (nv = 0; nv < 8; nv++) flux[nv] = fl[nv] + Sl*(usl[nv] - ul[nv]);
      } else if (S1R <= 0.0) {
        for (nv = 0; nv < 8; nv++) flux[nv] = fr[nv] + Sr*(usr[nv] - ur[nv]);
      } else {
        double ussl[8], ussr[8];
        ussl[RHO] = usl[RHO];
        ussr[RHO] = usr[RHO];
        double vss = sqrL*vsL + sqrR*vsR + (usr[BXt] - usl[BXt])*sBx;
        vss /= sqrL + sqrR;
        double wss = sqrL*wsL + sqrR*wsR + (usr[BXb] - usl[BXb])*sBx;
        wss /= sqrL + sqrR;
        ussl[MXn] = ussl[RHO]*SM;
        ussr[MXn] = ussr[RHO]*SM;
        ussl[MXt] = ussl[RHO]*vss;
        ussr[MXt] = ussr[RHO]*vss;
        ussl[MXb] = ussl[RHO]*wss;
        ussr[MXb] = ussr[RHO]*wss;
        ussl[BXn] = ussr[BXn] = Bx1;
        ussl[BXt]  = sqrL*usr[BXt] + sqrR*usl[BXt] + sqrL*sqrR*(vsR - vsL)*sBx;
        ussl[BXt] /= sqrL + sqrR;
        ussr[BXt]  = ussl[BXt];
        ussl[BXb]  = sqrL*usr[BXb] + sqrR*usl[BXb] + sqrL*sqrR*(wsR - wsL)*sBx;
        ussl[BXb] /= sqrL + sqrR;
        ussr[BXb]  = ussl[BXb];
        scrhL  = SM*Bx1 + vsL*usl [BXt] + wsL*usl [BXb];
        scrhL -= SM*Bx1 + vss*ussl[BXt] + wss*ussl[BXb];
        scrhR  = SM*Bx1 + vsR*usr [BXt] + wsR*usr [BXb];
        scrhR -= SM*Bx1 + vss*ussr[BXt] + wss*ussr[BXb];
        ussl[7] = usl[7] - sqrL*scrhL*sBx;
        ussr[7] = usr[7] + sqrR*scrhR*sBx;
        if (SM >= 0.0) {
          for (nv = 0; nv < 8; nv++)
            flux[nv] = fl[nv] + S1L*(ussl[nv] - usl[nv]) + Sl*(usl[nv] - ul[nv]);
        } else {
          for (nv = 0; nv < 8; nv++)
            flux[nv] = fr[nv] + S1R*(ussr[nv] - usr[nv]) + Sr*(usr[nv] - ur[nv]);
        }
      }
    } else {
      double scrh = 1.0/(Sr - Sl);
      for (nv = 0; nv < 8; nv++) {
        flux[nv]  = Sl*Sr*(ur[nv] - ul[nv]) + Sr*fl[nv] - Sl*fr[nv];
        flux[nv] *= scrh;
      }
    }
  }
  for (nv = 0; nv < 8; nv++) if (isnan(flux[nv])) o->err |= ERR_NAN | ERR_QUIT;

  if (o->c.ct == ORC_UCT_HLLD) CT_Store_UCTHlld(o, dir, ul, ur, vl, vr, Sl, Sr, Bn_face, e);
  else                         CT_Store_UCTHll(o, dir, vl, vr, Sl, Sr, e);
  return cmax;
}

/* Src/MHD/hll.cpp:50-220 (MHD) */
static double MHD_HLL(orc_t *o, int dir, double *vl, double *vr, double *flux, long e) {
  const double gamma = o->c.gamma;
  int nv;
  double ul[8], ur[8], fl[8], fr[8], Sl, Sr, pl, pr;
  MHD_PrimToCons(vl, ul, gamma);
  MHD_PrimToCons(vr, ur, gamma);
  double a2L = gamma*vl[7]/vl[RHO];
  double a2R = gamma*vr[7]/vr[RHO];
  {
    double sl_min, sl_max, sr_min, sr_max;
    MHD_MaxSignalSpeed(dir, vl, a2L, &sl_min, &sl_max);
    MHD_MaxSignalSpeed(dir, vr, a2R, &sr_min, &sr_max);
    Sl = MIN(sl_min, sr_min);
    Sr = MAX(sl_max, sr_max);
  }
  double bL = MIN(Sl, 0.0);
  double bR = MAX(0.0, Sr);
  double cmax = MAX(fabs(Sl), fabs(Sr));
  MHD_Flux(dir, vl, ul, fl, &pl);
  MHD_Flux(dir, vr, ur, fr, &pr);
  double scrh = 1.0/(bR - bL);
  for (nv = 0; nv < 8; nv++) {
    flux[nv]  = bL*bR*(ur[nv] - ul[nv]) + bR*fl[nv] - bL*fr[nv];
    flux[nv] *= scrh;
  }
  for (nv = 0; nv < 8; nv++) if (isnan(flux[nv])) o->err |= ERR_NAN | ERR_QUIT;
  CT_Store_UCTHll(o, dir, vl, vr, Sl, Sr, e);
  return cmax;
}

/* HLLC for MHD, Src/MHD/hllc.cpp:52-363 (no HLL switch without multi-D
   shock flattening; UCT_HLL face data, or the caller's arithmetic store). */
static double MHD_HLLC(orc_t *o, int dir, double *vl, double *vr, double *flux, long e) {
  const double gamma = o->c.gamma;
  const int VXn = VX1 + dir;
  const int MXn = MX1 + dir, MXt = MX1 + (dir+1)%3, MXb = MX1 + (dir+2)%3;
  const int BXn = BX1 + dir, BXt = BX1 + (dir+1)%3, BXb = BX1 + (dir+2)%3;
  int nv;
  double ul[8], ur[8], fl[8], fr[8], Sl, Sr, pl, pr;
  MHD_PrimToCons(vl, ul, gamma);
  MHD_PrimToCons(vr, ur, gamma);
  double a2L = gamma*vl[7]/vl[RHO];
  double a2R = gamma*vr[7]/vr[RHO];
  {
    double sl_min, sl_max, sr_min, sr_max;
    MHD_MaxSignalSpeed(dir, vl, a2L, &sl_min, &sl_max);
    MHD_MaxSignalSpeed(dir, vr, a2R, &sr_min, &sr_max);
    Sl = MIN(sl_min, sr_min);
    Sr = MAX(sl_max, sr_max);
  }
  double cmax = MAX(fabs(Sl), fabs(Sr));
  MHD_Flux(dir, vl, ul, fl, &pl);
  MHD_Flux(dir, vr, ur, fr, &pr);
  if (Sl >= 0.0) {
    for (nv = 0; nv < 8; nv++) flux[nv] = fl[nv];
  } else if (Sr <= 0.0) {
    for (nv = 0; nv < 8; nv++) flux[nv] = fr[nv];
  } else {
    double Uhll[8], Fhll[8], usl[8], usr[8];
    double scrh = 1.0/(Sr - Sl);
    for (nv = 0; nv < 8; nv++) {
      Uhll[nv]  = Sr*ur[nv] - Sl*ul[nv] + fl[nv] - fr[nv];
      Uhll[nv] *= scrh;
      Fhll[nv]  = Sl*Sr*(ur[nv] - ul[nv]) + Sr*fl[nv] - Sl*fr[nv];
      Fhll[nv] *= scrh;
    }
    double Bxs = Uhll[BXn], Bys = Uhll[BXt], Bzs = Uhll[BXb];
    double vxL = vl[VXn], vxR = vr[VXn];
    double vxs = Uhll[MXn]/Uhll[RHO];
    {
      double vBL = vl[VX1]*vl[BX1] + vl[VX1+1]*vl[BX2] + vl[VX1+2]*vl[BX3];
      double vBR = vr[VX1]*vr[BX1] + vr[VX1+1]*vr[BX2] + vr[VX1+2]*vr[BX3];
      double vBs = Uhll[BX1]*Uhll[MX1] + Uhll[BX2]*Uhll[MX2] + Uhll[BX3]*Uhll[MX3];
      vBs /= Uhll[RHO];
      usl[RHO] = ul[RHO]*(Sl - vxL)/(Sl - vxs);
      usr[RHO] = ur[RHO]*(Sr - vxR)/(Sr - vxs);
      double ps = Fhll[MXn] + Bxs*Bxs - Fhll[RHO]*vxs;
      usl[7] = (ul[7]*(Sl - vxL) + ps*vxs - pl*vxL - Bxs*vBs + vl[BXn]*vBL)/(Sl - vxs);
      usr[7] = (ur[7]*(Sr - vxR) + ps*vxs - pr*vxR - Bxs*vBs + vr[BXn]*vBR)/(Sr - vxs);
    }
    usl[MXn] = usl[RHO]*vxs;
    usr[MXn] = usr[RHO]*vxs;
    usl[MXt] = (ul[MXt]*(Sl - vxL) - (Bxs*Bys - vl[BXn]*vl[BXt]))/(Sl - vxs);
    usr[MXt] = (ur[MXt]*(Sr - vxR) - (Bxs*Bys - vr[BXn]*vr[BXt]))/(Sr - vxs);
    usl[MXb] = (ul[MXb]*(Sl - vxL) - (Bxs*Bzs - vl[BXn]*vl[BXb]))/(Sl - vxs);
    usr[MXb] = (ur[MXb]*(Sr - vxR) - (Bxs*Bzs - vr[BXn]*vr[BXb]))/(Sr - vxs);
    usl[BXn] = usr[BXn] = Bxs;
    usl[BXt] = usr[BXt] = Bys;
    usl[BXb] = usr[BXb] = Bzs;
    if (vxs > 0.0) {
      for (nv = 0; nv < 8; nv++) flux[nv] = fl[nv] + Sl*(usl[nv] - ul[nv]);
    } else {
      for (nv = 0; nv < 8; nv++) flux[nv] = fr[nv] + Sr*(usr[nv] - ur[nv]);
    }
  }
  for (nv = 0; nv < 8; nv++) if (isnan(flux[nv])) o->err |= ERR_NAN | ERR_QUIT;
  CT_Store_UCTHll(o, dir, vl, vr, Sl, Sr, e);
  return cmax;
}

/* Lax-Friedrichs (Rusanov) flux for MHD, Src/MHD/tvdlf.cpp:60-244: the
   signal speed of the arithmetic average state, UCT_HLL face data with
   Sl = -cmax, Sr = cmax. */
static double MHD_TVDLF(orc_t *o, int dir, double *vl, double *vr, double *flux, long e) {
  const double gamma = o->c.gamma;
  int nv;
  double ul[8], ur[8], fl[8], fr[8], vLR[8], pl, pr, cmax;
  MHD_PrimToCons(vl, ul, gamma);
  MHD_PrimToCons(vr, ur, gamma);
  for (nv = 0; nv < 8; nv++) vLR[nv] = 0.5*(vl[nv] + vr[nv]);
  {
    double a2 = gamma*vLR[7]/vLR[RHO], cminLR, cmaxLR;
    MHD_MaxSignalSpeed(dir, vLR, a2, &cminLR, &cmaxLR);
    cmax = MAX(fabs(cminLR), fabs(cmaxLR));
  }
  MHD_Flux(dir, vl, ul, fl, &pl);
  MHD_Flux(dir, vr, ur, fr, &pr);
  for (nv = 0; nv < 8; nv++) flux[nv] = 0.5*(fl[nv] + fr[nv]) - 0.5*cmax*(ur[nv] - ul[nv]);
  for (nv = 0; nv < 8; nv++) if (isnan(flux[nv])) o->err |= ERR_NAN | ERR_QUIT;
  CT_Store_UCTHll(o, dir, vl, vr, -cmax, cmax, e);
  return cmax;
}

/* Lax-Friedrichs flux for HD, Src/HD/tvdlf.cpp:100-190: the average state
   takes the mean of |v_n| on the two sides. */
static double HD_TVDLF(orc_t *o, int dir, double *vl, double *vr, double *flux) {
  const double gamma = o->c.gamma;
  int VXn = VX1 + dir, nv;
  double ul[5], ur[5], fL[5], fR[5], vLR[5], pl, pr, cmax;
  HD_PrimToCons(vl, ul, gamma);
  HD_PrimToCons(vr, ur, gamma);
  for (nv = 0; nv < 5; nv++) vLR[nv] = 0.5*(vl[nv] + vr[nv]);
  vLR[VXn] = 0.5*(fabs(vl[VXn]) + fabs(vr[VXn]));
  {
    double a2 = gamma*vLR[4]/vLR[RHO];
    double a = sqrt(a2);
    double cmaxLR = vLR[VXn] + a;
    double cminLR = vLR[VXn] - a;
    cmax = MAX(fabs(cminLR), fabs(cmaxLR));
  }
  HD_Flux(dir, vl, ul, fL, &pl);
  HD_Flux(dir, vr, ur, fR, &pr);
  for (nv = 0; nv < 5; nv++) flux[nv] = 0.5*(fL[nv] + fR[nv]) - 0.5*cmax*(ur[nv] - ul[nv]);
  for (nv = 0; nv < 5; nv++) if (isnan(flux[nv])) o->err |= ERR_NAN | ERR_QUIT;
  return cmax;
}

/* Src/HD/hllc.cpp:54-260 (ideal EOS) */
static double HD_HLLC(orc_t *o, int dir, double *vl, double *vr, double *flux) {
  const double gamma = o->c.gamma;
  int VXn = VX1 + dir, VXt = VX1 + (dir+1)%3, VXb = VX1 + (dir+2)%3;
  int MXn = MX1 + dir, MXt = MX1 + (dir+1)%3, MXb = MX1 + (dir+2)%3;
  int nv;
  double ul[5], ur[5], fL[5], fR[5], usl[5], usr[5], Sl, Sr, pl, pr;
  HD_PrimToCons(vl, ul, gamma);
  HD_PrimToCons(vr, ur, gamma);
  double a2L = gamma*vl[4]/vl[RHO];
  double a2R = gamma*vr[4]/vr[RHO];
  HD_Flux(dir, vl, ul, fL, &pl);
  HD_Flux(dir, vr, ur, fR, &pr);
  {
    double sl_min, sl_max, sr_min, sr_max;
    HD_MaxSignalSpeed(dir, vl, a2L, &sl_min, &sl_max);
    HD_MaxSignalSpeed(dir, vr, a2R, &sr_min, &sr_max);
    Sl = MIN(sl_min, sr_min);
    Sr = MAX(sl_max, sr_max);
  }
  double cmax = MAX(fabs(Sl), fabs(Sr));
  if (Sl > 0.0) {
    for (nv = 0; nv < 5; nv++) flux[nv] = fL[nv];
  } else if (Sr < 0.0) {
    for (nv = 0; nv < 5; nv++) flux[nv] = fR[nv];
  } else {
    double vs;
    {
      double qL = vl[4] + ul[MXn]*(vl[VXn] - Sl);
      double qR = vr[4] + ur[MXn]*(vr[VXn] - Sr);
      double wL = vl[RHO]*(vl[VXn] - Sl);
      double wR = vr[RHO]*(vr[VXn] - Sr);
      vs = (qR - qL)/(wR - wL);
    }
    {
      double vxr = vr[VXn];
      double vxl = vl[VXn];
      usl[RHO] = ul[RHO]*(Sl - vxl)/(Sl - vs);
      usr[RHO] = ur[RHO]*(Sr - vxr)/(Sr - vs);
      usl[MXn] = usl[RHO]*vs;      usr[MXn] = usr[RHO]*vs;
      usl[MXt] = usl[RHO]*vl[VXt]; usr[MXt] = usr[RHO]*vr[VXt];
      usl[MXb] = usl[RHO]*vl[VXb]; usr[MXb] = usr[RHO]*vr[VXb];
      usl[4] = ul[4]/vl[RHO] + (vs - vxl)*(vs + vl[4]/(vl[RHO]*(Sl - vxl)));
      usr[4] = ur[4]/vr[RHO] + (vs - vxr)*(vs + vr[4]/(vr[RHO]*(Sr - vxr)));
    }
    usl[4] *= usl[RHO];
    usr[4] *= usr[RHO];
    if (vs >= 0.0) {
      for (nv = 0; nv < 5; nv++) flux[nv] = fL[nv] + Sl*(usl[nv] - ul[nv]);
    } else {
      for (nv = 0; nv < 5; nv++) flux[nv] = fR[nv] + Sr*(usr[nv] - ur[nv]);
    }
  }
  for (nv = 0; nv < 5; nv++) if (isnan(flux[nv])) o->err |= ERR_NAN | ERR_QUIT;
  return cmax;
}

/* Src/HD/hll.cpp:95-175 (HD HLL: explicit supersonic branches) */
static double HD_HLL(orc_t *o, int dir, double *vl, double *vr, double *flux) {
  const double gamma = o->c.gamma;
  int nv;
  double ul[5], ur[5], fL[5], fR[5], Sl, Sr, pl, pr;
  HD_PrimToCons(vl, ul, gamma);
  HD_PrimToCons(vr, ur, gamma);
  double a2L = gamma*vl[4]/vl[RHO];
  double a2R = gamma*vr[4]/vr[RHO];
  {
    double sl_min, sl_max, sr_min, sr_max;
    HD_MaxSignalSpeed(dir, vl, a2L, &sl_min, &sl_max);
    HD_MaxSignalSpeed(dir, vr, a2R, &sr_min, &sr_max);
    Sl = MIN(sl_min, sr_min);
    Sr = MAX(sl_max, sr_max);
  }
  double cmax = MAX(fabs(Sl), fabs(Sr));
  HD_Flux(dir, vl, ul, fL, &pl);
  HD_Flux(dir, vr, ur, fR, &pr);
  if (Sl > 0.0) {
    for (nv = 0; nv < 5; nv++) flux[nv] = fL[nv];
  } else if (Sr < 0.0) {
    for (nv = 0; nv < 5; nv++) flux[nv] = fR[nv];
  } else {
    double scrh = 1.0/(Sr - Sl);
    for (nv = 0; nv < 5; nv++) {
      flux[nv]  = Sl*Sr*(ur[nv] - ul[nv]) + Sr*fL[nv] - Sl*fR[nv];
      flux[nv] *= scrh;
    }
  }
  for (nv = 0; nv < 5; nv++) if (isnan(flux[nv])) o->err |= ERR_NAN | ERR_QUIT;
  return cmax;
}

/* ------------------------------------------------------------------ */
/* reconstruction                                                      */
/* ------------------------------------------------------------------ */

/* SET_*_LIMITER of Src/plm_coeffs.hpp:55-110 (uniform Cartesian grid) and
   Src/macros.hpp:200 (minmod); FLAT (and any other label) gives 0 */
static double Limit(int lim, double dvp, double dvm) {
  double dv;
  if (lim == ORC_LIM_MC) {
    if (dvp*dvm > 0.0) {
      double qc = 0.5*(dvm + dvp), scrh = 2.0*ABS_MIN(dvp, dvm);
      dv = ABS_MIN(qc, scrh);
    } else dv = 0.0;
  } else if (lim == ORC_LIM_VL) {
    dv = (dvp*dvm > 0.0 ? 2.0*dvp*dvm/(dvp + dvm) : 0.0);
  } else if (lim == ORC_LIM_MINMOD) {
    dv = (dvp*dvm > 0.0 ? ABS_MIN(dvp, dvm) : 0.0);
  } else if (lim == ORC_LIM_VANALBADA) {
    if (dvp*dvm > 0.0) {
      double dpp = dvp*dvp, dmm = dvm*dvm;
      dv = (dvp*(dmm + 1.e-18) + dvm*(dpp + 1.e-18))/(dpp + dmm + 1.e-18);
    } else dv = 0.0;
  } else if (lim == ORC_LIM_OSPRE) {
    dv = (dvp*dvm > 0.0 ? 1.5*dvp*dvm*(dvm + dvp)/(dvp*dvp + dvm*dvm + dvp*dvm) : 0.0);
  } else if (lim == ORC_LIM_UMIST) {
    if (dvp*dvm > 0.0) {
      double ddp = 0.25*(dvp + 3.0*dvm), ddm = 0.25*(dvm + 3.0*dvp);
      double d2 = 2.0*ABS_MIN(dvp, dvm);
      d2 = ABS_MIN(d2, ddp);
      dv = ABS_MIN(d2, ddm);
    } else dv = 0.0;
  } else {
    dv = 0.0;
  }
  return dv;
}

/* Src/macros.hpp:200 */
static double Minmod(double a, double b) {
  return (a*b > 0.0 ? (fabs(a) < fabs(b) ? a : b) : 0.0);
}

/* Piecewise parabolic states of cell i (primitive limiting):
   Src/States/ppm_states.cpp:129-163 with the uniform-grid face value of
   Src/States/reconstruction_geometry.hpp:97-101.  v points at cell i of a
   pencil with stride `st`; returns the increments to the right (dvp) and
   left (dvm) faces. */
static void PPM_Cell(const double *v, long st, double *dvp_out, double *dvm_out) {
  double vim2 = v[-2*st], vim1 = v[-st], vi = v[0], vip1 = v[st], vip2 = v[2*st];
  double vp = (-vim1 + 7.0*(vi + vip1) - vip2)/12.0;
  double vm = (-vim2 + 7.0*(vim1 + vi) - vip1)/12.0;
  double dv, dvp, dvm;
  dv  = vip1 - vi;
  dvp = vp - vi;
  vp  = vi + Minmod(dvp, dv);
  dv  = vi - vim1;
  dvm = vm - vim1;
  vm  = vim1 + Minmod(dvm, dv);
  dvp = vp - vi;
  dvm = vm - vi;
  if (dvp*dvm >= 0.0) dvp = dvm = 0.0;
  else {
    if      (fabs(dvp) >= 2.0*fabs(dvm)) dvp = -2.0*dvm;
    else if (fabs(dvm) >= 2.0*fabs(dvp)) dvm = -2.0*dvp;
  }
  *dvp_out = dvp;
  *dvm_out = dvm;
}

/* Monotonicity-preserving 5th-order edge value of Suresh & Huynh (1997),
   Src/States/states.hpp:32-98 (MP5_ALPHA 4, cell averages): F points at the
   cell, `st` is the stride between cells, sign +1 gives the right edge and
   -1 the left edge. */
static double MP5_Edge(const double *F, long st, int sign) {
  const double alpha = 4.0, epsm = 1.e-12;
  const double Fpp = F[2*sign*st], Fp = F[sign*st], F0 = F[0], Fm = F[-sign*st],
               Fmm = F[-2*sign*st];
  double dFp = Fp - F0, dFm = F0 - Fm;
  double f = 2.0*Fmm - 13.0*Fm + 47.0*F0 + 27.0*Fp - 3.0*Fpp;   /* Eq. (2.1) */
  f /= 60.0;
  double fMP = F0 + Minmod(dFp, alpha*dFm);                      /* Eq. (2.12) */
  if ((f - F0)*(f - fMP) <= epsm) return f;
  double d2m = Fmm + F0 - 2.0*Fm;
  double d2  = Fm + Fp - 2.0*F0;
  double d2p = F0 + Fpp - 2.0*Fp;
  double scrh1 = Minmod(4.0*d2 - d2p, 4.0*d2p - d2);
  double scrh2 = Minmod(d2, d2p);
  double dMMp = Minmod(scrh1, scrh2);                             /* Eq. (2.27) */
  scrh1 = Minmod(4.0*d2m - d2, 4.0*d2 - d2m);
  scrh2 = Minmod(d2, d2m);
  double dMMm = Minmod(scrh1, scrh2);
  double fUL = F0 + alpha*dFm;                                   /* Eq. (2.8) */
  double fAV = 0.5*(F0 + Fp);                                    /* Eq. (2.16) */
  double fMD = fAV - 0.5*dMMp;                                   /* Eq. (2.28) */
  double fLC = 0.5*(3.0*F0 - Fm) + 4.0/3.0*dMMm;                 /* Eq. (2.29) */
  scrh1 = MIN(F0, Fp); scrh1 = MIN(scrh1, fMD);
  scrh2 = MIN(F0, fUL); scrh2 = MIN(scrh2, fLC);
  double fmin = MAX(scrh1, scrh2);                               /* Eq. (2.24a) */
  scrh1 = MAX(F0, Fp); scrh1 = MAX(scrh1, fMD);
  scrh2 = MAX(F0, fUL); scrh2 = MAX(scrh2, fLC);
  double fmax = MIN(scrh1, scrh2);                               /* Eq. (2.24b) */
  f = f + Minmod(fmin - f, fmax - f);                            /* Eq. (2.26) */
  return f;
}

/* WENO-Z edge value of Borges et al. (2008) with the 3rd-order weights
   (1, 6, 3), Src/States/states.hpp:108-166 without HIGH_ORDER; F points at
   the cell, `st` is the stride, sign +1 the right edge, -1 the left. */
static double WENOZ_Edge(const double *F, long st, int sign) {
  const double Fmm = F[-2*sign*st], Fm = F[-sign*st], F0 = F[0], Fp = F[sign*st],
               Fpp = F[2*sign*st];
  const double c13_12 = 13.0/12.0;
  double a0, a1, a2, b0, b1, b2, t5, sum_a, w0, w1, w2, f0, f1, f2;
  a0 = Fmm - 2.0*Fm + F0;
  a1 = Fmm - 4.0*Fm + 3.0*F0;
  b0 = c13_12*a0*a0 + 0.25*a1*a1;
  a0 = Fm - 2.0*F0 + Fp;
  a1 = Fm - Fp;
  b1 = c13_12*a0*a0 + 0.25*a1*a1;
  a0 = F0 - 2.0*Fp + Fpp;
  a1 = 3.0*F0 - 4.0*Fp + Fpp;
  b2 = c13_12*a0*a0 + 0.25*a1*a1;
  t5 = fabs(b0 - b2);
  a0 = 1.0*(1.0 + t5/(b0 + 1.e-40));
  a1 = 6.0*(1.0 + t5/(b1 + 1.e-40));
  a2 = 3.0*(1.0 + t5/(b2 + 1.e-40));
  sum_a = 1.0/(a0 + a1 + a2);
  w0 = a0*sum_a; w1 = a1*sum_a; w2 = a2*sum_a;
  f0 = 2.0*Fmm - 7.0*Fm + 11.0*F0;
  f1 = -Fm + 5.0*F0 + 2.0*Fp;
  f2 = 2.0*F0 + 5.0*Fp - Fpp;
  return (w0*f0 + w1*f1 + w2*f2)/6.0;
}

/* the 5-point schemes sharing Src/States/mp5_states.cpp */
static int FivePoint(int lim) { return lim == ORC_LIM_MP5 || lim == ORC_LIM_WENOZ; }
static double Edge5(int lim, const double *F, long st, int sign) {
  return lim == ORC_LIM_WENOZ ? WENOZ_Edge(F, st, sign) : MP5_Edge(F, st, sign);
}

/* WENO3 edge value, the "improved" weights of Yamaleev & Carpenter (2009),
   Src/States/states.hpp:178-226 without HIGH_ORDER; dx the cell width. */
static double WENO3_Edge(const double *F, long st, int sign, double dx) {
  const double Fp = F[sign*st], Fm = F[-sign*st], F0 = F[0];
  double a0, a1, b0, b1, w0, w1, f0, f1, tau, dx2;
  dx2 = dx*dx;
  b0 = Fp - F0;
  b1 = Fm - F0;
  b0 = b0*b0;
  b1 = b1*b1;
  tau = (Fp - 2.0*F0 + Fm);
  tau = tau*tau;
  a0 = 2.0*(1.0 + tau/(dx2 + b0));
  a1 = 1.0*(1.0 + tau/(dx2 + b1));
  w0 = a0/(a0 + a1);
  w1 = a1/(a0 + a1);
  f0 = 0.5*(Fp + F0);
  f1 = 0.5*(-Fm + 3.0*F0);
  return (w0*f0 + w1*f1);
}

/* LimO3 edge value (the third-order limiter of Cada & Torrilhon 2009,
   Eq. 3.22), Src/States/states.hpp:239-281. */
static double LimO3_Edge(const double *v, long st, int sign, double dx) {
  const double r = 0.1, eps = 1.e-12;
  double a, b, c, q, q1, lim, eta, psi;
  double dvp = v[sign*st] - v[0];
  double dvm = v[0] - v[-sign*st];
  double sp = (dvp >= 0.0 ? 1.0 : -1.0);
  double advp = fabs(dvp);
  double dvm1 = sp*dvm;
  q  = (2.0*dvp + dvm)/3.0;
  q1 = (2.0*fabs(dvp) + sp*dvm)/3.0;
  a = MIN(1.5*advp, 2.0*dvm1);
  a = MIN(q1, a);
  b = MAX(-0.5*dvm1, a);
  c = MIN(q1, b);
  psi = sp*MAX(0.0, c);
  eta = r*dx;
  eta = (dvm*dvm + dvp*dvp)/(eta*eta);
  if (eta <= 1.0 - eps) {
    lim = q;
  } else if (eta >= 1.0 + eps) {
    lim = psi;
  } else {
    psi = (1.0 - (eta - 1.0)/eps)*q + (1.0 + (eta - 1.0)/eps)*psi;
    lim = 0.5*psi;
  }
  return v[0] + 0.5*lim;
}

/* the 3-point schemes of the same driver */
static int ThreePoint(int lim) { return lim == ORC_LIM_LIMO3 || lim == ORC_LIM_WENO3; }
static double Edge3(int lim, const double *F, long st, int sign, double dx) {
  return lim == ORC_LIM_LIMO3 ? LimO3_Edge(F, st, sign, dx) : WENO3_Edge(F, st, sign, dx);
}

/* ------------------------------------------------------------------ */
/* boundary: Src/boundary.cpp:67-322 + PeriodicBoundary 502-675         */
/* ------------------------------------------------------------------ */
static void AverageStaggered(orc_t *o, int ib, int ie, int jb, int je, int kb, int ke,
                             int write_vc) {
  /* Src/MHD/CT/ct_field_average.cpp:175-200, 378-410 (Cartesian) */
  int i, j, k, d;
  for (k = kb; k <= ke; k++)
  for (j = jb; j <= je; j++)
  for (i = ib; i <= ie; i++) {
    for (d = 0; d < o->c.ndim; d++) {
      int di = (d == 0), dj = (d == 1), dk = (d == 2);
      double bf = 0.5*(o->Vs[d][SI(o,d,i,j,k)] + o->Vs[d][SI(o,d,i+di,j+dj,k+dk)]);
      *VC(o, o->Uc, BX1+d, i, j, k) = bf;
      if (write_vc) *VC(o, o->Vc, BX1+d, i, j, k) = bf;
    }
  }
}

/* Normal staggered field in the ghost zone of an outflow side from
   div B = 0, marching away from the domain: CT_FillStaggeredFields,
   Src/MHD/CT/ct_fill_mag_field.cpp:96-330, with the Cartesian face areas of
   Src/set_geometry.cpp:124,147,165 (uniform grid).  The loops run over the
   whole ghosted extent of the other directions. */
static void CT_FillNormal(orc_t *o, int d, int beg) {
  const int ndim = o->c.ndim;
  const double dx = o->c.dx[0], dy = o->c.dx[1], dz = o->c.dx[2];
  double A[3];
  if (ndim == 2) { A[0] = 1.0*dy; A[1] = dx*1.0; A[2] = 0.0; }
  else           { A[0] = 1.0*dy*dz; A[1] = dx*1.0*dz; A[2] = dx*dy*1.0; }
  int lo[3] = {0, 0, 0}, hi[3] = {o->nt[0]-1, o->nt[1]-1, o->nt[2]-1};
  int i, j, k;
  /* a loop over the two transverse directions; the normal index marches */
  int a = (d == 0) ? 1 : 0, b = (d == 2) ? 1 : 2;
  int t1, t2, m;
  for (t2 = lo[b]; t2 <= hi[b]; t2++)
  for (t1 = lo[a]; t1 <= hi[a]; t1++) {
    int mfirst = beg ? o->beg[d]-1 : o->end[d]+1;
    int mlast  = beg ? 0 : o->nt[d]-1;
    int step = beg ? -1 : 1;
    for (m = mfirst; beg ? (m >= mlast) : (m <= mlast); m += step) {
      int ijk[3];
      ijk[d] = m; ijk[a] = t1; ijk[b] = t2;
      i = ijk[0]; j = ijk[1]; k = ijk[2];
      double dB[3] = {0.0, 0.0, 0.0};
      int c;
      for (c = 0; c < ndim; c++) {
        int di = (c == 0), dj = (c == 1), dk = (c == 2);
        double Bp = o->Vs[c][SI(o,c,i+di,j+dj,k+dk)], Bm = o->Vs[c][SI(o,c,i,j,k)];
        dB[c] = A[c]*Bp - A[c]*Bm;
      }
      int di = (d == 0), dj = (d == 1), dk = (d == 2);
      /* the two transverse contributions in the reference's order */
      double t_a = dB[a], t_b = (b < ndim) ? dB[b] : 0.0;
      if (d == 2) { t_a = dB[0]; t_b = dB[1]; }
      if (beg) {
        double Bp = o->Vs[d][SI(o,d,i+di,j+dj,k+dk)];
        o->Vs[d][SI(o,d,i,j,k)] = (A[d]*Bp + t_a + t_b)/A[d];
      } else {
        double Bm = o->Vs[d][SI(o,d,i,j,k)];
        o->Vs[d][SI(o,d,i+di,j+dj,k+dk)] = (A[d]*Bm - (t_a + t_b))/A[d];
      }
    }
  }
}

static void Boundary(orc_t *o) {
  int side, nv, i, j, k;
  int isMHD = (o->c.physics != ORC_HD);
  for (side = 0; side < 2*o->c.ndim; side++) {
    int d = side/2, beg = (side%2 == 0);
    int lo[3] = {0, 0, 0}, hi[3] = {o->nt[0]-1, o->nt[1]-1, o->nt[2]-1};
    int shift = beg ? o->c.n[d] : -o->c.n[d];
    if (beg) { lo[d] = 0; hi[d] = o->beg[d]-1; }
    else     { lo[d] = o->end[d]+1; hi[d] = o->nt[d]-1; }
    if ((o->c.outflow >> side) & 1) {
      /* OutflowBoundary, Src/boundary.cpp:677-780: every ghost cell copies
         the interior cell next to the boundary; the tangential staggered
         fields are copied the same way (BOXJ/BOXK loops, one face wider) */
      int i0 = beg ? o->beg[d] : o->end[d];
      for (nv = 0; nv < o->nvar; nv++)
        for (k = lo[2]; k <= hi[2]; k++)
        for (j = lo[1]; j <= hi[1]; j++)
        for (i = lo[0]; i <= hi[0]; i++) {
          int s[3] = {i, j, k}; s[d] = i0;
          *VC(o, o->Vc, nv, i, j, k) = *VC(o, o->Vc, nv, s[0], s[1], s[2]);
        }
      if (isMHD) {
        int c;
        for (c = 0; c < o->c.ndim; c++) {
          if (c == d) continue;
          int h[3] = {hi[0], hi[1], hi[2]};
          h[c] += 1;
          for (k = lo[2]; k <= h[2]; k++)
          for (j = lo[1]; j <= h[1]; j++)
          for (i = lo[0]; i <= h[0]; i++) {
            int s[3] = {i, j, k}; s[d] = i0;
            o->Vs[c][SI(o,c,i,j,k)] = o->Vs[c][SI(o,c,s[0],s[1],s[2])];
          }
        }
        CT_FillNormal(o, d, beg);
        /* Src/boundary.cpp:285-307: ghost cell B from faces, copied to Vc */
        AverageStaggered(o, lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], 1);
      }
      continue;
    }
    if ((o->c.userdef >> side) & 1) {
      /* USERDEF (Src/boundary.cpp:238-256): UserDefBoundary fills the ghost
         cells and the tangential staggered fields -- here the inflow rule of
         the parity cases: the domain cell next to the side, then density
         ud_rho and normal velocity ud_vn into the domain; tangential faces
         copied one face wider -- then CT_FillStaggeredFields and the ghost
         cell-centred B, as for an outflow side. */
      int i0 = beg ? o->beg[d] : o->end[d];
      for (k = lo[2]; k <= hi[2]; k++)
      for (j = lo[1]; j <= hi[1]; j++)
      for (i = lo[0]; i <= hi[0]; i++) {
        int s[3] = {i, j, k}; s[d] = i0;
        for (nv = 0; nv < o->nvar; nv++)
          *VC(o, o->Vc, nv, i, j, k) = *VC(o, o->Vc, nv, s[0], s[1], s[2]);
        *VC(o, o->Vc, RHO, i, j, k) = o->c.ud_rho;
        *VC(o, o->Vc, VX1 + d, i, j, k) = beg ? o->c.ud_vn : -o->c.ud_vn;
      }
      if (isMHD) {
        int c;
        for (c = 0; c < o->c.ndim; c++) {
          if (c == d) continue;
          int h[3] = {hi[0], hi[1], hi[2]};
          h[c] += 1;
          for (k = lo[2]; k <= h[2]; k++)
          for (j = lo[1]; j <= h[1]; j++)
          for (i = lo[0]; i <= h[0]; i++) {
            int s[3] = {i, j, k}; s[d] = i0;
            o->Vs[c][SI(o,c,i,j,k)] = o->Vs[c][SI(o,c,s[0],s[1],s[2])];
          }
        }
        CT_FillNormal(o, d, beg);
        AverageStaggered(o, lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], 1);
      }
      continue;
    }
    if (((o->c.reflect | o->c.eqtsym) >> side) & 1) {
      /* ReflectiveBoundary with the signs of FlipSign
         (Src/boundary.cpp:203-216, 838-900, 931-1060): ghost cell m copies
         its mirror image i0 - m; REFLECTIVE (and AXISYMMETRIC, the same in
         Cartesian geometry) flips v_n and B_n, EQTSYMMETRIC flips v_n, B_t
         and B_b.  Normal faces mirror across the boundary face (which keeps
         its value), tangential faces like the cells, one face wider. */
      int eqt = (o->c.eqtsym >> side) & 1;
      double vsign[8];
      int i0 = beg ? 2*o->beg[d] - 1 : 2*o->end[d] + 1;
      for (nv = 0; nv < o->nvar; nv++) vsign[nv] = 1.0;
      vsign[VX1 + d] = -1.0;
      if (isMHD) {
        if (eqt) { vsign[BX1 + (d+1)%3] = -1.0; vsign[BX1 + (d+2)%3] = -1.0; }
        else     vsign[BX1 + d] = -1.0;
      }
      for (nv = 0; nv < o->nvar; nv++)
        for (k = lo[2]; k <= hi[2]; k++)
        for (j = lo[1]; j <= hi[1]; j++)
        for (i = lo[0]; i <= hi[0]; i++) {
          int s[3] = {i, j, k}; s[d] = i0 - s[d];
          *VC(o, o->Vc, nv, i, j, k) = vsign[nv] * *VC(o, o->Vc, nv, s[0], s[1], s[2]);
        }
      if (isMHD) {
        int c;
        for (c = 0; c < o->c.ndim; c++) {
          int h[3] = {hi[0], hi[1], hi[2]};
          if (c != d) h[c] += 1;
          for (k = lo[2]; k <= h[2]; k++)
          for (j = lo[1]; j <= h[1]; j++)
          for (i = lo[0]; i <= h[0]; i++) {
            int t[3] = {i, j, k}, s[3] = {i, j, k};
            if (c == d) {
              if (beg) s[d] = i0 - t[d] + 1;         /* face m from face i0-m+1 */
              else   { t[d] += 1; s[d] = i0 - i*(d==0) - j*(d==1) - k*(d==2); }
            } else {
              s[d] = i0 - t[d];
            }
            o->Vs[c][SI(o,c,t[0],t[1],t[2])] = vsign[BX1 + c] * o->Vs[c][SI(o,c,s[0],s[1],s[2])];
          }
        }
        /* Src/boundary.cpp:260-307: ghost cell B from faces, copied to Vc */
        AverageStaggered(o, lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], 1);
      }
      continue;
    }
    for (nv = 0; nv < o->nvar; nv++)
      for (k = lo[2]; k <= hi[2]; k++)
      for (j = lo[1]; j <= hi[1]; j++)
      for (i = lo[0]; i <= hi[0]; i++) {
        int s[3] = {i, j, k}; s[d] += shift;
        *VC(o, o->Vc, nv, i, j, k) = *VC(o, o->Vc, nv, s[0], s[1], s[2]);
      }
    if (isMHD) {
      int c;
      for (c = 0; c < o->c.ndim; c++) {
        /* BOX_LOOP on the own-direction beg side, BOXI/J/K_LOOP elsewhere */
        int ext = (c == d && beg) ? 0 : 1;
        int h[3] = {hi[0], hi[1], hi[2]};
        h[c] += ext;
        for (k = lo[2]; k <= h[2]; k++)
        for (j = lo[1]; j <= h[1]; j++)
        for (i = lo[0]; i <= h[0]; i++) {
          int s[3] = {i, j, k}; s[d] += shift;
          o->Vs[c][SI(o,c,i,j,k)] = o->Vs[c][SI(o,c,s[0],s[1],s[2])];
        }
      }
      /* Src/boundary.cpp:285-307: ghost cell B from faces, copied to Vc */
      AverageStaggered(o, lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], 1);
    }
  }
}

/* ------------------------------------------------------------------ */
/* sweeps: Src/update_stage.cpp:57-384                                 */
/* ------------------------------------------------------------------ */
static void Sweep(orc_t *o, int dir, double dt) {
  const int nvar = o->nvar, ndim = o->c.ndim;
  const int isMHD = (o->c.physics != ORC_HD);
  int ntr = isMHD ? o->ng : 0;    /* Src/update_stage.cpp:80-90 */
  int t1d = (dir == 0 ? 1 : 0), t2d = (dir == 2 ? 1 : 2);
  int tlo1 = o->beg[t1d], thi1 = o->end[t1d], tlo2 = o->beg[t2d], thi2 = o->end[t2d];
  if (t1d < ndim) { tlo1 -= ntr; thi1 += ntr; }
  if (t2d < ndim) { tlo2 -= ntr; thi2 += ntr; }
  int nd = o->nt[dir], ib = o->beg[dir], ie = o->end[dir];
  double dtdx = dt/o->c.dx[dir];
  int t1, t2, i, nv;
  double *v = o->pv, *vL = o->pvL, *vR = o->pvR, *flux = o->pflux, *cmax = o->pcmax, *Bn = o->pBn;

  for (t2 = tlo2; t2 <= thi2; t2++)
  for (t1 = tlo1; t1 <= thi1; t1++) {
    int ti, tj, tk;
    /* DataToSweep: Src/data2sweep.cpp:48-222 */
    for (i = 0; i < nd; i++) {
      TrueIdx(dir, i, t1, t2, &ti, &tj, &tk);
      for (nv = 0; nv < nvar; nv++) v[i*nvar + nv] = *VC(o, o->Vc, nv, ti, tj, tk);
      if (isMHD) Bn[i] = o->Vs[dir][SI(o, dir, ti, tj, tk)];
    }
    /* Reconstruct: Src/States/plm_states.cpp:99-141, or (PARABOLIC)
       Src/States/ppm_states.cpp:110-164 */
    for (nv = 0; nv < nvar; nv++)
      for (i = ib-1; i <= ie+1; i++) {
        if (FivePoint(o->c.limiter)) {   /* Src/States/mp5_states.cpp:125-182 */
          vL[(i+1)*nvar + nv] = Edge5(o->c.limiter, v + i*nvar + nv, nvar, +1);
          vR[i*nvar + nv]     = Edge5(o->c.limiter, v + i*nvar + nv, nvar, -1);
          continue;
        }
        if (ThreePoint(o->c.limiter)) {  /* Src/States/mp5_states.cpp:164-172 */
          vL[(i+1)*nvar + nv] = Edge3(o->c.limiter, v + i*nvar + nv, nvar, +1, o->c.dx[dir]);
          vR[i*nvar + nv]     = Edge3(o->c.limiter, v + i*nvar + nv, nvar, -1, o->c.dx[dir]);
          continue;
        }
        if (o->c.limiter == ORC_LIM_PPM) {
          double dvp, dvm;
          PPM_Cell(v + i*nvar + nv, nvar, &dvp, &dvm);
          vL[(i+1)*nvar + nv] = v[i*nvar + nv] + dvp;
          vR[i*nvar + nv]     = v[i*nvar + nv] + dvm;
          continue;
        }
        double dvp = v[(i+1)*nvar + nv] - v[i*nvar + nv];
        double dvm = v[i*nvar + nv] - v[(i-1)*nvar + nv];
        double dv = Limit(o->c.limiter, dvp, dvm);
        vL[(i+1)*nvar + nv] = v[i*nvar + nv] + 0.5*dv;
        vR[i*nvar + nv]     = v[i*nvar + nv] - 0.5*dv;
      }
    /* MP5: density and pressure edges that came out negative fall back to
       minmod PLM (Src/States/mp5_states.cpp:184-213, uniform grid) */
    if (FivePoint(o->c.limiter) || ThreePoint(o->c.limiter)) {
      const int qv[2] = {RHO, nvar - 1};
      int q;
      for (i = ib-1; i <= ie+1; i++)
        for (q = 0; q < 2; q++) {
          nv = qv[q];
          if (vL[(i+1)*nvar + nv] < 0.0 || vR[i*nvar + nv] < 0.0) {
            double dvp = (v[(i+1)*nvar + nv] - v[i*nvar + nv])*1.0;
            double dvm = (v[i*nvar + nv] - v[(i-1)*nvar + nv])*1.0;
            double dv = Minmod(dvp, dvm);
            vL[(i+1)*nvar + nv] = v[i*nvar + nv] + 0.5*dv;
            vR[i*nvar + nv]     = v[i*nvar + nv] - 0.5*dv;
          }
        }
    }
    /* relativistic velocity limiter, Src/vel_limiter.hpp:13-34 (applied in
       the adjustment loop before the CT overwrite, plm_states.cpp:166) */
    if (o->c.physics == ORC_RMHD) {
      for (i = ib-1; i <= ie+1; i++) {
        double *r = vR + i*nvar, *l = vL + (i+1)*nvar;
        double v2m = r[VX1]*r[VX1] + r[VX1+1]*r[VX1+1] + r[VX1+2]*r[VX1+2];
        double v2p = l[VX1]*l[VX1] + l[VX1+1]*l[VX1+1] + l[VX1+2]*l[VX1+2];
        if (v2m >= 1.0 || v2p >= 1.0)
          for (nv = 0; nv < nvar; nv++) r[nv] = l[nv] = v[i*nvar + nv];
      }
    }
    /* CT normal-field overwrite: Src/States/plm_states.cpp:184-189 */
    if (isMHD) {
      for (i = ib-1; i <= ie+1; i++) {
        vL[(i+1)*nvar + BX1 + dir] = Bn[i+1];
        vR[i*nvar + BX1 + dir] = Bn[i];
      }
    }
    /* Riemann solver at interfaces i-1/2, i in [ib, ie+1] */
    for (i = ib; i <= ie+1; i++) {
      TrueIdx(dir, i, t1, t2, &ti, &tj, &tk);
      long e = EI(o, ti, tj, tk);
      double *vl = vL + i*nvar, *vr = vR + i*nvar, *f = flux + i*nvar;
      if (o->c.physics == ORC_MHD) {
        if (o->c.solver == ORC_HLLD)       cmax[i] = MHD_HLLD(o, dir, vl, vr, f, e, Bn[i]);
        else if (o->c.solver == ORC_TVDLF) cmax[i] = MHD_TVDLF(o, dir, vl, vr, f, e);
        else if (o->c.solver == ORC_HLLC)  cmax[i] = MHD_HLLC(o, dir, vl, vr, f, e);
        else                               cmax[i] = MHD_HLL(o, dir, vl, vr, f, e);
        if (o->c.ct == ORC_ARITHMETIC || o->c.ct == ORC_CT_CONTACT) {
          /* CT_Store_Arith, Src/MHD/CT/ct_store.hpp:74-93 (replaces the
             UCT data the solver stored); CT_CONTACT adds the sign of the
             mass flux, zero within eps_CT_CONTACT = 1e-6 (ct.hpp:110) */
          int DIRt = (dir+1)%3, DIRb = (dir+2)%3;
          o->e[DIRb][dir][e] = -f[BX1 + DIRt];
          o->e[DIRt][dir][e] =  f[BX1 + DIRb];
          if (o->c.ct == ORC_CT_CONTACT)
            o->sv[dir][e] = f[RHO] > 1.e-6 ? 1.0 : (f[RHO] < -1.e-6 ? -1.0 : 0.0);
        }
      } else if (o->c.physics == ORC_HD) {
        if (o->c.solver == ORC_HLLC)       cmax[i] = HD_HLLC(o, dir, vl, vr, f);
        else if (o->c.solver == ORC_TVDLF) cmax[i] = HD_TVDLF(o, dir, vl, vr, f);
        else                               cmax[i] = HD_HLL(o, dir, vl, vr, f);
      } else {
        cmax[i] = orc_rmhd_riemann(o, dir, vl, vr, f, e);
      }
    }
    /* RightHandSide over the interior box only: Src/MHD/rhs.cpp:383-386, 523 */
    if (t1 < o->beg[t1d] || t1 > o->end[t1d] || t2 < o->beg[t2d] || t2 > o->end[t2d]) continue;
    for (i = ib; i <= ie; i++) {
      TrueIdx(dir, i, t1, t2, &ti, &tj, &tk);
      for (nv = 0; nv < nvar; nv++) {
        double rhs = -dtdx*(flux[(i+1)*nvar + nv] - flux[i*nvar + nv]);
        double *r = VC(o, o->Rc, nv, ti, tj, tk);
        if (dir == 0) *r = rhs; else *r += rhs;    /* Src/update_stage.cpp:173-184 */
      }
      double cdt = 0.5*(cmax[i] + cmax[i+1])/o->c.dx[dir];
      long c = CI(o, ti, tj, tk);
      if (dir == 0) o->Cdt[c] = cdt; else o->Cdt[c] += cdt;
    }
  }
}

/* ------------------------------------------------------------------ */
/* EMF: Src/MHD/CT/ct_emf_average.cpp:535-995 with ArrayReconstruct    */
/* (Src/array_reconstruct.cpp:45-206)                                  */
/* ------------------------------------------------------------------ */

/* Reconstruct Q along `dir` on the pencil at transverse (t1,t2).  Q is either a
   staggered field (stag >= 0, component index) or an EMF face array. */
static void ArrayRec(orc_t *o, int dir, int t1, int t2, int stag, const double *Qe,
                     int lim, double *qL, double *qR) {
  int nd = o->nt[dir], i, ti, tj, tk;
  double *q = o->pq;
  for (i = 0; i < nd; i++) {
    TrueIdx(dir, i, t1, t2, &ti, &tj, &tk);
    q[i] = (stag >= 0) ? o->Vs[stag][SI(o, stag, ti, tj, tk)] : Qe[EI(o, ti, tj, tk)];
  }
  if (ThreePoint(lim)) {
    /* LimO3 / WENO3 branch, Src/array_reconstruct.cpp:272-325 */
    for (i = 1; i < nd-1; i++) {
      qL[i+1] = Edge3(lim, q + i, 1, +1, o->c.dx[dir]);
      qR[i]   = Edge3(lim, q + i, 1, -1, o->c.dx[dir]);
    }
    return;
  }
  if (FivePoint(lim)) {
    /* WENOZ / MP5 branch, Src/array_reconstruct.cpp:327-384 */
    for (i = 2; i < nd-2; i++) {
      qL[i+1] = Edge5(lim, q + i, 1, +1);
      qR[i]   = Edge5(lim, q + i, 1, -1);
    }
    return;
  }
  if (lim == ORC_LIM_PPM) {
    /* PARABOLIC branch, Src/array_reconstruct.cpp:208-270 (uniform grid) */
    for (i = 1; i < nd-1; i++) {
      double qp = (    -q[i-1] + 5.0*q[i] + 2.0*q[i+1])/6.0;
      double qm = ( 2.0*q[i-1] + 5.0*q[i] -     q[i+1])/6.0;
      double dqp = qp - q[i];
      double dqm = qm - q[i];
      double dq  = q[i+1] - q[i];
      qp  = q[i] + Minmod(dqp, dq);
      dq  = q[i] - q[i-1];
      qm  = q[i] + Minmod(dqm, -dq);
      dqp = qp - q[i];
      dqm = qm - q[i];
      if (dqp*dqm >= 0.0) dqp = dqm = 0.0;
      else {
        if      (fabs(dqp) >= 2.0*fabs(dqm)) dqp = -2.0*dqm;
        else if (fabs(dqm) >= 2.0*fabs(dqp)) dqm = -2.0*dqp;
      }
      qL[i+1] = q[i] + dqp;
      qR[i]   = q[i] + dqm;
    }
    return;
  }
  for (i = 1; i < nd-1; i++) {
    double dqp = q[i+1] - q[i];
    double dqm = q[i] - q[i-1];
    double dq = Limit(lim, dqp, dqm);
    qL[i+1] = q[i] + 0.5*dq;
    qR[i]   = q[i] - 0.5*dq;
  }
}

/* CT_CONTACT helpers: the cell-centred inductive field E = -v x B of
   CT_ComputeCenterEMF (Src/MHD/CT/ct_emf.cpp:333-367) and the upwind weight
   of a face's contact sign (Src/MHD/CT/ct_emf_average.cpp:137-143). */
static double Ecc(orc_t *o, int comp, int i, int j, int k) {
  double vx1 = *VC(o, o->Vc, VX1, i, j, k), vx2 = *VC(o, o->Vc, VX1+1, i, j, k);
  double vx3 = *VC(o, o->Vc, VX1+2, i, j, k);
  double Bx1 = *VC(o, o->Vc, BX1, i, j, k), Bx2 = *VC(o, o->Vc, BX2, i, j, k);
  double Bx3 = *VC(o, o->Vc, BX3, i, j, k);
  if (comp == 0) return (vx3*Bx2 - vx2*Bx3);
  if (comp == 1) return (vx1*Bx3 - vx3*Bx1);
  return (vx2*Bx1 - vx1*Bx2);
}
static double ContactW(double s) { return s != 0.0 ? (s > 0.0 ? 1.0 : 0.0) : 0.5; }

/* CT_ComputeEMF with CT_EMF_AVERAGE CT_CONTACT (Src/MHD/CT/ct_emf.cpp:220-245):
   the four face EMFs summed (CT_EMF_ArithmeticAverage with w = 1), the
   upwinded derivative terms of CT_EMF_IntegrateToCorner
   (Src/MHD/CT/ct_emf_average.cpp:115-290, Gardiner & Stone 2005), then
   times 1/4.  Each edge in one pass, in the reference's operation order. */
static void ContactEMF(orc_t *o, int ib, int ie, int jb, int je, int kb, int ke) {
  const int ndim = o->c.ndim;
  int i, j, k;
  double **e0 = o->e[0], **e1 = o->e[1], **e2 = o->e[2];
#define EE(A, ii, jj, kk) (A)[EI(o, ii, jj, kk)]
  for (k = kb; k <= ke; k++)
  for (j = jb; j <= je; j++)
  for (i = ib; i <= ie; i++) {
    double wS, wN, wW, wE, E;
    /* Ez at (i-1/2, j-1/2, k) */
    E = 1.0*(  EE(e2[0], i, j, k) + EE(e2[0], i, j-1, k)
             + EE(e2[1], i, j, k) + EE(e2[1], i-1, j, k));
    wS = ContactW(EE(o->sv[0], i, j-1, k));
    wN = ContactW(EE(o->sv[0], i, j, k));
    E +=   wS*(EE(e2[1], i-1, j, k) - Ecc(o, 2, i-1, j-1, k))
         + (1.0-wS)*(EE(e2[1], i, j, k) - Ecc(o, 2, i, j-1, k))
         - wN*(Ecc(o, 2, i-1, j, k) - EE(e2[1], i-1, j, k))
         - (1.0-wN)*(Ecc(o, 2, i, j, k) - EE(e2[1], i, j, k));
    wW = ContactW(EE(o->sv[1], i-1, j, k));
    wE = ContactW(EE(o->sv[1], i, j, k));
    E +=   wW*(EE(e2[0], i, j-1, k) - Ecc(o, 2, i-1, j-1, k))
         + (1.0-wW)*(EE(e2[0], i, j, k) - Ecc(o, 2, i-1, j, k))
         - wE*(Ecc(o, 2, i, j-1, k) - EE(e2[0], i, j-1, k))
         - (1.0-wE)*(Ecc(o, 2, i, j, k) - EE(e2[0], i, j, k));
    EE(o->Ee[2], i, j, k) = E*0.25;
    if (ndim < 3) continue;
    /* Ex at (i, j-1/2, k-1/2) */
    E = 1.0*(  EE(e0[2], i, j, k) + EE(e0[2], i, j-1, k)
             + EE(e0[1], i, j, k) + EE(e0[1], i, j, k-1));
    wS = ContactW(EE(o->sv[1], i, j, k-1));
    wN = ContactW(EE(o->sv[1], i, j, k));
    E +=   wS*(EE(e0[2], i, j-1, k) - Ecc(o, 0, i, j-1, k-1))
         + (1.0-wS)*(EE(e0[2], i, j, k) - Ecc(o, 0, i, j, k-1))
         - wN*(Ecc(o, 0, i, j-1, k) - EE(e0[2], i, j-1, k))
         - (1.0-wN)*(Ecc(o, 0, i, j, k) - EE(e0[2], i, j, k));
    wW = ContactW(EE(o->sv[2], i, j-1, k));
    wE = ContactW(EE(o->sv[2], i, j, k));
    E +=   wW*(EE(e0[1], i, j, k-1) - Ecc(o, 0, i, j-1, k-1))
         + (1.0-wW)*(EE(e0[1], i, j, k) - Ecc(o, 0, i, j-1, k))
         - wE*(Ecc(o, 0, i, j, k-1) - EE(e0[1], i, j, k-1))
         - (1.0-wE)*(Ecc(o, 0, i, j, k) - EE(e0[1], i, j, k));
    EE(o->Ee[0], i, j, k) = E*0.25;
    /* Ey at (i-1/2, j, k-1/2) */
    E = 1.0*(  EE(e1[0], i, j, k) + EE(e1[0], i, j, k-1)
             + EE(e1[2], i, j, k) + EE(e1[2], i-1, j, k));
    wS = ContactW(EE(o->sv[2], i-1, j, k));
    wN = ContactW(EE(o->sv[2], i, j, k));
    E +=   wS*(EE(e1[0], i, j, k-1) - Ecc(o, 1, i-1, j, k-1))
         + (1.0-wS)*(EE(e1[0], i, j, k) - Ecc(o, 1, i-1, j, k))
         - wN*(Ecc(o, 1, i, j, k-1) - EE(e1[0], i, j, k-1))
         - (1.0-wN)*(Ecc(o, 1, i, j, k) - EE(e1[0], i, j, k));
    wW = ContactW(EE(o->sv[0], i, j, k-1));
    wE = ContactW(EE(o->sv[0], i, j, k));
    E +=   wW*(EE(e1[2], i-1, j, k) - Ecc(o, 1, i-1, j, k-1))
         + (1.0-wW)*(EE(e1[2], i, j, k) - Ecc(o, 1, i, j, k-1))
         - wE*(Ecc(o, 1, i-1, j, k) - EE(e1[2], i-1, j, k))
         - (1.0-wE)*(Ecc(o, 1, i, j, k) - EE(e1[2], i, j, k));
    EE(o->Ee[1], i, j, k) = E*0.25;
  }
#undef EE
}

static void ComputeEMF(orc_t *o) {
  const int ndim = o->c.ndim;
  /* Src/MHD/CT/ct_emf_average.cpp:553-559: MC for B and the scheme limiter
     for velocities with linear reconstruction; parabolic for both with PPM */
  int recV = o->c.limiter,
      recB = (o->c.limiter == ORC_LIM_PPM || FivePoint(o->c.limiter) ||
              ThreePoint(o->c.limiter)) ? o->c.limiter
                                                                         : ORC_LIM_MC;
  int ib = o->beg[0], ie = o->end[0] + 1;
  int jb = o->beg[1], je = o->end[1] + 1;
  int kb = o->beg[2], ke = o->end[2] + (ndim == 3);
  int i, j, k;
  double *bL = o->pqL, *bR = o->pqR, *vL = o->pvL, *vR = o->pvR;   /* scratch */
  double *qL2 = o->pflux, *qR2 = o->pcmax;
  (void)vL; (void)vR;

  if (o->c.ct == ORC_CT_CONTACT) {
    ContactEMF(o, ib, ie, jb, je, kb, ke);
    return;
  }
  if (o->c.ct == ORC_ARITHMETIC) {
    /* CT_EMF_ArithmeticAverage (Src/MHD/CT/ct_emf_average.cpp:36-96),
       w = 0.25, each edge from the four face EMFs around it */
    const double w = 0.25;
    for (k = kb; k <= ke; k++)
    for (j = jb; j <= je; j++)
    for (i = ib; i <= ie; i++) {
      o->Ee[2][EI(o,i,j,k)] = w*(  o->e[2][0][EI(o,i,j,k)] + o->e[2][0][EI(o,i,j-1,k)]
                                 + o->e[2][1][EI(o,i,j,k)] + o->e[2][1][EI(o,i-1,j,k)]);
      if (ndim == 3) {
        o->Ee[0][EI(o,i,j,k)] = w*(  o->e[0][2][EI(o,i,j,k)] + o->e[0][2][EI(o,i,j-1,k)]
                                   + o->e[0][1][EI(o,i,j,k)] + o->e[0][1][EI(o,i,j,k-1)]);
        o->Ee[1][EI(o,i,j,k)] = w*(  o->e[1][0][EI(o,i,j,k)] + o->e[1][0][EI(o,i,j,k-1)]
                                   + o->e[1][2][EI(o,i,j,k)] + o->e[1][2][EI(o,i-1,j,k)]);
      }
    }
    return;
  }

  /* X1a: By and -vx along x -> Ez at (i-1/2, j-1/2, k) */
  for (k = kb; k <= ke; k++)
  for (j = jb; j <= je; j++) {
    ArrayRec(o, 0, j, k, 1, NULL, recB, bL, bR);
    ArrayRec(o, 0, j, k, -1, o->e[2][1], recV, qL2, qR2);
    for (i = ib; i <= ie; i++) {
      double aL = 0.5*(o->aL[0][EI(o,i,j-1,k)] + o->aL[0][EI(o,i,j,k)]);
      double aR = 0.5*(o->aR[0][EI(o,i,j-1,k)] + o->aR[0][EI(o,i,j,k)]);
      double dL = 0.5*(o->dL[0][EI(o,i,j-1,k)] + o->dL[0][EI(o,i,j,k)]);
      double dR = 0.5*(o->dR[0][EI(o,i,j-1,k)] + o->dR[0][EI(o,i,j,k)]);
      double phi = dR*bR[i] - dL*bL[i];
      o->Ee[2][EI(o,i,j,k)] = (aL*qL2[i]*bL[i] + aR*qR2[i]*bR[i]) + phi;
    }
  }
  if (ndim == 3) {
    /* X1b: Bz and vx along x -> Ey at (i-1/2, j, k-1/2) */
    for (k = kb; k <= ke; k++)
    for (j = jb; j <= je; j++) {
      ArrayRec(o, 0, j, k, 2, NULL, recB, bL, bR);
      ArrayRec(o, 0, j, k, -1, o->e[1][2], recV, qL2, qR2);
      for (i = ib; i <= ie; i++) {
        double aL = 0.5*(o->aL[0][EI(o,i,j,k-1)] + o->aL[0][EI(o,i,j,k)]);
        double aR = 0.5*(o->aR[0][EI(o,i,j,k-1)] + o->aR[0][EI(o,i,j,k)]);
        double dL = 0.5*(o->dL[0][EI(o,i,j,k-1)] + o->dL[0][EI(o,i,j,k)]);
        double dR = 0.5*(o->dR[0][EI(o,i,j,k-1)] + o->dR[0][EI(o,i,j,k)]);
        double phi = dR*bR[i] - dL*bL[i];
        o->Ee[1][EI(o,i,j,k)] = (aL*qL2[i]*bL[i] + aR*qR2[i]*bR[i]) - phi;
      }
    }
    /* X2a: Bz and -vy along y -> Ex at (i, j-1/2, k-1/2) */
    for (k = kb; k <= ke; k++)
    for (i = ib; i <= ie; i++) {
      ArrayRec(o, 1, i, k, 2, NULL, recB, bL, bR);
      ArrayRec(o, 1, i, k, -1, o->e[0][2], recV, qL2, qR2);
      for (j = jb; j <= je; j++) {
        double aL = 0.5*(o->aL[1][EI(o,i,j,k-1)] + o->aL[1][EI(o,i,j,k)]);
        double aR = 0.5*(o->aR[1][EI(o,i,j,k-1)] + o->aR[1][EI(o,i,j,k)]);
        double dL = 0.5*(o->dL[1][EI(o,i,j,k-1)] + o->dL[1][EI(o,i,j,k)]);
        double dR = 0.5*(o->dR[1][EI(o,i,j,k-1)] + o->dR[1][EI(o,i,j,k)]);
        double phi = dR*bR[j] - dL*bL[j];
        o->Ee[0][EI(o,i,j,k)] = (aL*qL2[j]*bL[j] + aR*qR2[j]*bR[j]) + phi;
      }
    }
  }
  /* X2b: Bx and vy along y -> complete Ez */
  for (k = kb; k <= ke; k++)
  for (i = ib; i <= ie; i++) {
    ArrayRec(o, 1, i, k, 0, NULL, recB, bL, bR);
    ArrayRec(o, 1, i, k, -1, o->e[2][0], recV, qL2, qR2);
    for (j = jb; j <= je; j++) {
      double aL = 0.5*(o->aL[1][EI(o,i-1,j,k)] + o->aL[1][EI(o,i,j,k)]);
      double aR = 0.5*(o->aR[1][EI(o,i-1,j,k)] + o->aR[1][EI(o,i,j,k)]);
      double dL = 0.5*(o->dL[1][EI(o,i-1,j,k)] + o->dL[1][EI(o,i,j,k)]);
      double dR = 0.5*(o->dR[1][EI(o,i-1,j,k)] + o->dR[1][EI(o,i,j,k)]);
      double phi = dR*bR[j] - dL*bL[j];
      o->Ee[2][EI(o,i,j,k)] += (aL*qL2[j]*bL[j] + aR*qR2[j]*bR[j]) - phi;
    }
  }
  if (ndim == 3) {
    /* X3a: Bx and -vz along z -> complete Ey */
    for (j = jb; j <= je; j++)
    for (i = ib; i <= ie; i++) {
      ArrayRec(o, 2, i, j, 0, NULL, recB, bL, bR);
      ArrayRec(o, 2, i, j, -1, o->e[1][0], recV, qL2, qR2);
      for (k = kb; k <= ke; k++) {
        double aL = 0.5*(o->aL[2][EI(o,i-1,j,k)] + o->aL[2][EI(o,i,j,k)]);
        double aR = 0.5*(o->aR[2][EI(o,i-1,j,k)] + o->aR[2][EI(o,i,j,k)]);
        double dL = 0.5*(o->dL[2][EI(o,i-1,j,k)] + o->dL[2][EI(o,i,j,k)]);
        double dR = 0.5*(o->dR[2][EI(o,i-1,j,k)] + o->dR[2][EI(o,i,j,k)]);
        double phi = dR*bR[k] - dL*bL[k];
        o->Ee[1][EI(o,i,j,k)] += (aL*qL2[k]*bL[k] + aR*qR2[k]*bR[k]) + phi;
      }
    }
    /* X3b: By and vz along z -> complete Ex */
    for (j = jb; j <= je; j++)
    for (i = ib; i <= ie; i++) {
      ArrayRec(o, 2, i, j, 1, NULL, recB, bL, bR);
      ArrayRec(o, 2, i, j, -1, o->e[0][1], recV, qL2, qR2);
      for (k = kb; k <= ke; k++) {
        double aL = 0.5*(o->aL[2][EI(o,i,j-1,k)] + o->aL[2][EI(o,i,j,k)]);
        double aR = 0.5*(o->aR[2][EI(o,i,j-1,k)] + o->aR[2][EI(o,i,j,k)]);
        double dL = 0.5*(o->dL[2][EI(o,i,j-1,k)] + o->dL[2][EI(o,i,j,k)]);
        double dR = 0.5*(o->dR[2][EI(o,i,j-1,k)] + o->dR[2][EI(o,i,j,k)]);
        double phi = dR*bR[k] - dL*bL[k];
        o->Ee[0][EI(o,i,j,k)] += (aL*qL2[k]*bL[k] + aR*qR2[k]*bR[k]) - phi;
      }
    }
  }
}

/* Src/MHD/CT/ct_update.cpp:181-423 (Cartesian) -> Rs = -curl(E) dt */
static void CTUpdate(orc_t *o, double dt) {
  const int ndim = o->c.ndim;
  int i, j, k;
  int ib = o->beg[0], ie = o->end[0], jb = o->beg[1], je = o->end[1], kb = o->beg[2], ke = o->end[2];
  double dtdx1 = dt/o->c.dx[0], dtdx2 = dt/o->c.dx[1], dtdx3 = dt/o->c.dx[2];
  /* Bx1 faces */
  for (k = kb; k <= ke; k++)
  for (j = jb; j <= je; j++)
  for (i = ib; i <= ie+1; i++) {
    double curlE = 0.0 + dtdx2*(o->Ee[2][EI(o,i,j+1,k)] - o->Ee[2][EI(o,i,j,k)]);
    if (ndim == 3) curlE = curlE - dtdx3*(o->Ee[1][EI(o,i,j,k+1)] - o->Ee[1][EI(o,i,j,k)]);
    o->Rs[0][SI(o,0,i,j,k)] = -curlE;
  }
  /* Bx2 faces */
  for (k = kb; k <= ke; k++)
  for (j = jb; j <= je+1; j++)
  for (i = ib; i <= ie; i++) {
    double curlE = -dtdx1*(o->Ee[2][EI(o,i+1,j,k)] - o->Ee[2][EI(o,i,j,k)]);
    if (ndim == 3) curlE = curlE + dtdx3*(o->Ee[0][EI(o,i,j,k+1)] - o->Ee[0][EI(o,i,j,k)]);
    o->Rs[1][SI(o,1,i,j,k)] = -curlE;
  }
  if (ndim == 3) {
    for (k = kb; k <= ke+1; k++)
    for (j = jb; j <= je; j++)
    for (i = ib; i <= ie; i++) {
      double curlE = dtdx1*(o->Ee[1][EI(o,i+1,j,k)] - o->Ee[1][EI(o,i,j,k)])
                   - dtdx2*(o->Ee[0][EI(o,i,j+1,k)] - o->Ee[0][EI(o,i,j,k)]);
      o->Rs[2][SI(o,2,i,j,k)] = -curlE;
    }
  }
}

/* Src/update_stage.cpp:57-438 */
static double UpdateStage(orc_t *o, double dt, int stage) {
  int d;
  for (d = 0; d < o->c.ndim; d++) Sweep(o, d, dt);
  if (o->c.physics != ORC_HD) {
    ComputeEMF(o);
    CTUpdate(o, dt);
  }
  double inv = -1.0;
  if (stage == 1) {
    int i, j, k;
    for (k = o->beg[2]; k <= o->end[2]; k++)
    for (j = o->beg[1]; j <= o->end[1]; j++)
    for (i = o->beg[0]; i <= o->end[0]; i++) inv = MAX(inv, o->Cdt[CI(o,i,j,k)]);
    inv = inv/(double)o->c.ndim;   /* update_stage.cpp:422-435 */
  }
  return inv;
}

/* Src/mappers3D.cpp:76-194 over the interior box */
static void ConsToPrim3D(orc_t *o) {
  int i, j, k, nv;
  double u[8], v[8];
  for (k = o->beg[2]; k <= o->end[2]; k++)
  for (j = o->beg[1]; j <= o->end[1]; j++)
  for (i = o->beg[0]; i <= o->end[0]; i++) {
    uint32_t err = 0;
    for (nv = 0; nv < o->nvar; nv++) {
      u[nv] = *VC(o, o->Uc, nv, i, j, k);
      if (isnan(u[nv])) err |= ERR_NAN | ERR_QUIT;
    }
    uint32_t le;
    if (o->c.physics == ORC_MHD) le = MHD_ConsToPrim(u, v, o->c.gamma, 1.e-12, 1.e-12);
    else if (o->c.physics == ORC_HD) le = HD_ConsToPrim(u, v, o->c.gamma, 1.e-12, 1.e-12);
    else le = orc_rmhd_cons_to_prim(o, u, v, i, j, k);
    err |= le;
    if (le & ERR_CONS2PRIM_FAIL) err |= ERR_QUIT;
    if (le) for (nv = 0; nv < o->nvar; nv++) *VC(o, o->Uc, nv, i, j, k) = u[nv];
    for (nv = 0; nv < o->nvar; nv++) *VC(o, o->Vc, nv, i, j, k) = v[nv];
    o->err |= err;
  }
}

/* U = w0 U0 + w1 U + wr Rc and the same for the faces, then the cell-centred
   B from the faces (Src/rk_step.cpp:509-552) */
static void Combine(orc_t *o, double w0, double w1, double wr) {
  const int ndim = o->c.ndim, nvar = o->nvar;
  int i, j, k, nv, d;
  for (nv = 0; nv < nvar; nv++)
    for (k = o->beg[2]; k <= o->end[2]; k++)
    for (j = o->beg[1]; j <= o->end[1]; j++)
    for (i = o->beg[0]; i <= o->end[0]; i++) {
      double *u = VC(o, o->Uc, nv, i, j, k);
      *u = w0*(*VC(o, o->U0, nv, i, j, k)) + w1*(*u) + wr*(*VC(o, o->Rc, nv, i, j, k));
    }
  if (o->c.physics != ORC_HD) {
    for (k = o->beg[2]; k <= o->end[2] + (ndim == 3); k++)
    for (j = o->beg[1]; j <= o->end[1] + 1; j++)
    for (i = o->beg[0]; i <= o->end[0] + 1; i++)
      for (d = 0; d < ndim; d++) {
        long s = SI(o, d, i, j, k);
        o->Vs[d][s] = w0*o->Bs0[d][s] + w1*o->Vs[d][s] + wr*o->Rs[d][s];
      }
    AverageStaggered(o, o->beg[0], o->end[0], o->beg[1], o->end[1], o->beg[2], o->end[2], 0);
  }
}

/* Src/rk_step.cpp:88-743 (RK2 and RK3 branches) */
double orc_step(void *h, double dt, uint32_t *err_out) {
  orc_t *o = (orc_t *)h;
  const int ndim = o->c.ndim, nvar = o->nvar;
  const int isMHD = (o->c.physics != ORC_HD);
  int i, j, k, nv, d;
  o->err = 0;

  /* stage 1 */
  Boundary(o);
  double invDt = UpdateStage(o, dt, 1);
  for (nv = 0; nv < nvar; nv++)
    for (k = o->beg[2]; k <= o->end[2]; k++)
    for (j = o->beg[1]; j <= o->end[1]; j++)
    for (i = o->beg[0]; i <= o->end[0]; i++) {
      double *u = VC(o, o->Uc, nv, i, j, k), *u0 = VC(o, o->U0, nv, i, j, k);
      *u0 = *u;
      *u = *u0 + 1.0*(*VC(o, o->Rc, nv, i, j, k));
    }
  if (isMHD) {
    for (k = o->beg[2]; k <= o->end[2] + (ndim == 3); k++)
    for (j = o->beg[1]; j <= o->end[1] + 1; j++)
    for (i = o->beg[0]; i <= o->end[0] + 1; i++)
      for (d = 0; d < ndim; d++) {
        long s = SI(o, d, i, j, k);
        o->Bs0[d][s] = o->Vs[d][s];
        o->Vs[d][s] = o->Bs0[d][s] + 1.0*o->Rs[d][s];
      }
    AverageStaggered(o, o->beg[0], o->end[0], o->beg[1], o->end[1], o->beg[2], o->end[2], 0);
  }
  ConsToPrim3D(o);

  /* stage 2 (RK2: 1/2, 1/2, 1/2; RK3: 3/4, 1/4, 1/4) and RK3's stage 3
     (1/3, 2/3, 2/3): Src/rk_step.cpp:30-61, 509-552, 681-727 */
  if (o->c.rk == 3) {
    Boundary(o);
    UpdateStage(o, dt, 2);
    Combine(o, 0.75, 0.25, 0.25);
    ConsToPrim3D(o);
    Boundary(o);
    UpdateStage(o, dt, 3);
    Combine(o, (1.0/3.0), (2.0/3.0), (2.0/3.0));
  } else {
    Boundary(o);
    UpdateStage(o, dt, 2);
    Combine(o, 0.5, 0.5, 0.5);
  }
  ConsToPrim3D(o);
  if (err_out) *err_out = o->err;
  return invDt;
}

/* Src/next_time_step.cpp:20-130 (no MPI, no parabolic terms) */
double orc_next_dt(double invDt_hyp, double cfl, double cfl_max_var, double dt) {
  double dt_new = cfl/invDt_hyp;
  dt_new = MIN(dt_new, cfl_max_var*dt);
  return dt_new;
}

/* ------------------------------------------------------------------ */
/* state I/O (interior, SoA [nv][k][j][i])                             */
/* ------------------------------------------------------------------ */
void orc_set_state(void *h, const double *V, const double *U, const double *Bs) {
  orc_t *o = (orc_t *)h;
  int i, j, k, nv, d;
  long c = 0;
  for (nv = 0; nv < o->nvar; nv++)
    for (k = o->beg[2]; k <= o->end[2]; k++)
    for (j = o->beg[1]; j <= o->end[1]; j++)
    for (i = o->beg[0]; i <= o->end[0]; i++, c++) {
      *VC(o, o->Vc, nv, i, j, k) = V[c];
      *VC(o, o->Uc, nv, i, j, k) = U[c];
    }
  if (o->c.physics != ORC_HD) {
    long n = (long)o->c.n[0]*o->c.n[1]*o->c.n[2];
    for (d = 0; d < o->c.ndim; d++) {
      c = 0;
      for (k = o->beg[2]; k <= o->end[2]; k++)
      for (j = o->beg[1]; j <= o->end[1]; j++)
      for (i = o->beg[0]; i <= o->end[0]; i++, c++)
        o->Vs[d][SI(o, d, i, j, k)] = Bs[d*n + c];
      /* the right boundary face equals the left one (periodic) */
    }
    for (d = 0; d < o->c.ndim; d++) {
      int di = (d == 0), dj = (d == 1), dk = (d == 2);
      for (k = o->beg[2]; k <= o->end[2]; k++)
      for (j = o->beg[1]; j <= o->end[1]; j++)
      for (i = o->beg[0]; i <= o->end[0]; i++) {
        if ((di && i == o->beg[0]) || (dj && j == o->beg[1]) || (dk && k == o->beg[2]))
          o->Vs[d][SI(o, d, i + di*o->c.n[0], j + dj*o->c.n[1], k + dk*o->c.n[2])] =
            o->Vs[d][SI(o, d, i, j, k)];
      }
    }
  }
}

void orc_get_state(void *h, double *V, double *U, double *Bs) {
  orc_t *o = (orc_t *)h;
  int i, j, k, nv, d;
  long c = 0;
  for (nv = 0; nv < o->nvar; nv++)
    for (k = o->beg[2]; k <= o->end[2]; k++)
    for (j = o->beg[1]; j <= o->end[1]; j++)
    for (i = o->beg[0]; i <= o->end[0]; i++, c++) {
      if (V) V[c] = *VC(o, o->Vc, nv, i, j, k);
      if (U) U[c] = *VC(o, o->Uc, nv, i, j, k);
    }
  if (Bs && o->c.physics != ORC_HD) {
    long n = (long)o->c.n[0]*o->c.n[1]*o->c.n[2];
    for (d = 0; d < o->c.ndim; d++) {
      c = 0;
      for (k = o->beg[2]; k <= o->end[2]; k++)
      for (j = o->beg[1]; j <= o->end[1]; j++)
      for (i = o->beg[0]; i <= o->end[0]; i++, c++)
        Bs[d*n + c] = o->Vs[d][SI(o, d, i, j, k)];
    }
  }
}

/* Start-up conversion, Src/startup.cpp:542-566: U = PrimToCons(V) per cell */
void orc_prim_to_cons(int physics, double gamma, long ncell, const double *V, double *U) {
  int nvar = (physics == ORC_HD) ? 5 : 8, nv;
  long c;
  double v[8], u[8];
  for (c = 0; c < ncell; c++) {
    for (nv = 0; nv < nvar; nv++) v[nv] = V[nv*ncell + c];
    if (physics == ORC_MHD) MHD_PrimToCons(v, u, gamma);
    else if (physics == ORC_HD) HD_PrimToCons(v, u, gamma);
    else orc_rmhd_prim_to_cons(v, u, gamma);
    for (nv = 0; nv < nvar; nv++) U[nv*ncell + c] = u[nv];
  }
}

/* ------------------------------------------------------------------ */
/* construction                                                        */
/* ------------------------------------------------------------------ */
void *orc_create(const orc_cfg *cfg) {
  orc_t *o = (orc_t *)calloc(1, sizeof(orc_t));
  int d, e;
  o->c = *cfg;
  o->nvar = (cfg->physics == ORC_HD) ? 5 : 8;
  o->ng = (cfg->limiter == ORC_LIM_PPM || FivePoint(cfg->limiter)) ? 3 : 2;
  /* Src/get_nghost.cpp:33-44 */
  o->ncell = 1;
  for (d = 0; d < 3; d++) {
    if (d < cfg->ndim) { o->nt[d] = cfg->n[d] + 2*o->ng; o->beg[d] = o->ng; }
    else { o->nt[d] = 1; o->beg[d] = 0; o->c.n[d] = 1; }
    o->end[d] = o->beg[d] + o->c.n[d] - 1;
    o->ncell *= o->nt[d];
    o->ne[d] = o->nt[d] + 1;
  }
  o->Vc = calloc((size_t)o->nvar*o->ncell, sizeof(double));
  o->Uc = calloc((size_t)o->nvar*o->ncell, sizeof(double));
  o->U0 = calloc((size_t)o->nvar*o->ncell, sizeof(double));
  o->Rc = calloc((size_t)o->nvar*o->ncell, sizeof(double));
  o->Cdt = calloc((size_t)o->ncell, sizeof(double));
  if (cfg->physics != ORC_HD) {
    long ne = (long)o->ne[0]*o->ne[1]*o->ne[2];
    for (d = 0; d < 3; d++) {
      long ns = 1;
      for (e = 0; e < 3; e++) { o->ns[d][e] = o->nt[e] + (e == d && d < cfg->ndim); ns *= o->ns[d][e]; }
      if (d < cfg->ndim) {
        o->Vs[d] = calloc(ns, sizeof(double));
        o->Bs0[d] = calloc(ns, sizeof(double));
        o->Rs[d] = calloc(ns, sizeof(double));
      }
      o->aL[d] = calloc(ne, sizeof(double));
      o->aR[d] = calloc(ne, sizeof(double));
      o->dL[d] = calloc(ne, sizeof(double));
      o->dR[d] = calloc(ne, sizeof(double));
      o->Ee[d] = calloc(ne, sizeof(double));
      o->sv[d] = calloc(ne, sizeof(double));
      for (e = 0; e < 3; e++) o->e[d][e] = calloc(ne, sizeof(double));
    }
  }
  o->pmax = 0;
  for (d = 0; d < 3; d++) if (o->nt[d] + 2 > o->pmax) o->pmax = o->nt[d] + 2;
  o->pv = calloc((size_t)o->pmax*8, sizeof(double));
  o->pvL = calloc((size_t)o->pmax*8, sizeof(double));
  o->pvR = calloc((size_t)o->pmax*8, sizeof(double));
  o->pflux = calloc((size_t)o->pmax*8, sizeof(double));
  o->pcmax = calloc((size_t)o->pmax*8, sizeof(double));
  o->pBn = calloc((size_t)o->pmax, sizeof(double));
  o->pq = calloc((size_t)o->pmax, sizeof(double));
  o->pqL = calloc((size_t)o->pmax, sizeof(double));
  o->pqR = calloc((size_t)o->pmax, sizeof(double));
  orc_rmhd_init(o);
  return o;
}

void orc_destroy(void *h) {
  orc_t *o = (orc_t *)h;
  int d, e;
  if (!o) return;
  free(o->Vc); free(o->Uc); free(o->U0); free(o->Rc); free(o->Cdt);
  for (d = 0; d < 3; d++) {
    free(o->Vs[d]); free(o->Bs0[d]); free(o->Rs[d]);
    free(o->aL[d]); free(o->aR[d]); free(o->dL[d]); free(o->dR[d]); free(o->Ee[d]);
    free(o->sv[d]);
    for (e = 0; e < 3; e++) free(o->e[d][e]);
  }
  free(o->pv); free(o->pvL); free(o->pvR); free(o->pflux); free(o->pcmax);
  free(o->pBn); free(o->pq); free(o->pqL); free(o->pqR);
  free(o);
}

/* Convenience: run nsteps with the reference dt rule; dt_hist gets the dt
   of every step taken plus the next one (nsteps+1 entries). */
uint32_t orc_run(void *h, int nsteps, double first_dt, double *dt_hist) {
  orc_t *o = (orc_t *)h;
  double dt = first_dt;
  uint32_t err_all = 0, err;
  int n;
  for (n = 0; n < nsteps; n++) {
    if (dt_hist) dt_hist[n] = dt;
    double inv = orc_step(h, dt, &err);
    err_all |= err;
    dt = orc_next_dt(inv, o->c.cfl, o->c.cfl_max_var, dt);
  }
  if (dt_hist) dt_hist[nsteps] = dt;
  return err_all;
}

#include "gp_oracle_rmhd.inc"
