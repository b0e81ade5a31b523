/*
 * gp_oracle.h -- C interface of the CPU restatement of the gPLUTO Godunov
 * step (test infrastructure only; see gp_oracle.c).
 */
#ifndef GP_ORACLE_H
#define GP_ORACLE_H
#include <stdint.h>

enum { ORC_HD = 0, ORC_MHD = 1, ORC_RMHD = 2 };
enum { ORC_LIM_FLAT = 0, ORC_LIM_MINMOD = 1, ORC_LIM_VL = 2, ORC_LIM_MC = 3,
       ORC_LIM_PPM = 4 /* RECONSTRUCTION PARABOLIC (no slope limiter) */,
       ORC_LIM_MP5 = 5 /* RECONSTRUCTION MP5 (no slope limiter) */,
       ORC_LIM_VANALBADA = 6, ORC_LIM_OSPRE = 7, ORC_LIM_UMIST = 8,
       ORC_LIM_WENOZ = 9 /* RECONSTRUCTION WENOZ (no slope limiter) */,
       ORC_LIM_LIMO3 = 10, ORC_LIM_WENO3 = 11 /* RECONSTRUCTION LimO3 / WENO3 */ };
enum { ORC_HLL = 0, ORC_HLLC = 1, ORC_HLLD = 2, ORC_TVDLF = 3 };
enum { ORC_UCT_HLL = 0, ORC_UCT_HLLD = 1, ORC_ARITHMETIC = 2, ORC_CT_CONTACT = 3 };

typedef struct {
  int physics, ndim;
  int n[3];
  int limiter, solver, ct;
  double gamma;
  double dx[3];
  double cfl, cfl_max_var;
  int outflow;   /* bit 2d / 2d+1: low / high side of direction d is OUTFLOW */
  int reflect;   /* same bits: REFLECTIVE (or AXISYMMETRIC, identical in Cartesian) */
  int eqtsym;    /* same bits: EQTSYMMETRIC */
  int rk;        /* TIME_STEPPING: 2 (RK2, also for 0) or 3 (RK3) */
  int userdef;   /* same bits: USERDEF, filled by the inflow rule of the parity cases */
  double ud_rho, ud_vn;  /* the inflow's density and normal speed into the domain */
} orc_cfg;

void    *orc_create(const orc_cfg *cfg);
void     orc_destroy(void *h);
void     orc_set_state(void *h, const double *V, const double *U, const double *Bs);
void     orc_get_state(void *h, double *V, double *U, double *Bs);
double   orc_step(void *h, double dt, uint32_t *err);
double   orc_next_dt(double invDt_hyp, double cfl, double cfl_max_var, double dt);
uint32_t orc_run(void *h, int nsteps, double first_dt, double *dt_hist);
void     orc_set_ulp_nudge(int n);
void     orc_set_cr_trig(int on);
void     orc_set_rmhd_strict(int on);
void     orc_prim_to_cons(int physics, double gamma, long ncell, const double *V, double *U);
#endif
