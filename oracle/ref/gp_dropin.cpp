////////////////////////////////////////////////////////////////////////
// The reference driver with its time step moved onto the B200 library:
// the swap of Src/main.cpp:444-447 that INTEGRATION.md describes, as a
// maintainer would add it to the reference tree.  Test infrastructure:
// oracle/ref/build_dropin.py compiles the reference sources with this file
// and a copy of Src/main.cpp in which
//   - GP_DropIn_Init(&data, &grid, &runtime, &run_config) runs once before
//     the main loop (after Startup has set the initial conditions), and
//   - GP_DropIn_Step(&data, &grid, &Dts) replaces AdvanceStep(&data, &grid,
//     &Dts) (Src/main.cpp:446),
// and links gpluto_dev_b200/_build/libgpluto_b200.so.  Everything else --
// NextTimeStep, CheckForOutput/WriteData, RestartDump, Analysis, the log --
// is the reference's own code, reading Data on the host.
////////////////////////////////////////////////////////////////////////
#include "gpluto.hpp"
#include "gpluto_b200.h"

#include <cstring>

static gp_handle *g_gp = nullptr;

// Src/gpluto.hpp:205-212 side types -> gp_bc
static int GP_Side(int t)
{
  switch (t) {
    case OUTFLOW:      return GP_BC_OUTFLOW;
    case REFLECTIVE:   return GP_BC_REFLECTIVE;
    case AXISYMMETRIC: return GP_BC_AXISYMMETRIC;
    case EQTSYMMETRIC: return GP_BC_EQTSYMMETRIC;
    case USERDEF:      return GP_BC_USERDEF;
    default:           return GP_BC_PERIODIC;
  }
}

static void GP_Arrays(Data *data, double **Uc, double **Vc, double **Vs)
{
  *Uc = &data->Uc(0,0,0,0);
  *Vc = &data->Vc(0,0,0,0);
  for (int d = 0; d < 3; d++) Vs[d] = NULL;
  #ifdef STAGGERED_MHD
  DIM_EXPAND(Vs[0] = &data->Vs[BX1s](0,0,0);  ,
             Vs[1] = &data->Vs[BX1s+1](0,0,0);  ,
             Vs[2] = &data->Vs[BX1s+2](0,0,0);)
  #endif
}

////////////////////////////////////////////////////////////////////////
void GP_DropIn_Init(Data *data, Grid *grid, Runtime *runtime, RunConfig *run_config)
{
  gp_grid_desc g;
  std::memset(&g, 0, sizeof(g));
  g.ndim   = DIMENSIONS;
  g.nghost = grid->nghost[IDIR];
  for (int d = 0; d < 3; d++) {
    g.nint[d] = grid->nint[d];
    g.xbeg[d] = grid->xbeg[d];
    g.xend[d] = grid->xend[d];
    g.dx[d]   = d < DIMENSIONS ? grid->dx[d] : NULL;   // checked: uniform
    g.lbound[d] = GP_Side(grid->lbound[d]);
    g.rbound[d] = GP_Side(grid->rbound[d]);
  }
  gp_scheme s;
  std::memset(&s, 0, sizeof(s));
  #if PHYSICS == MHD
  s.physics = GP_MHD;
  #elif PHYSICS == RMHD
  s.physics = GP_RMHD;
  #else
  s.physics = GP_HD;
  #endif
  #if LIMITER == FLAT_LIM
  s.limiter = GP_LIM_FLAT;
  #elif LIMITER == MINMOD_LIM
  s.limiter = GP_LIM_MINMOD;
  #elif LIMITER == VANLEER_LIM
  s.limiter = GP_LIM_VANLEER;
  #elif LIMITER == VANALBADA_LIM
  s.limiter = GP_LIM_VANALBADA;
  #elif LIMITER == OSPRE_LIM
  s.limiter = GP_LIM_OSPRE;
  #elif LIMITER == UMIST_LIM
  s.limiter = GP_LIM_UMIST;
  #else
  s.limiter = GP_LIM_MC;
  #endif
  const char *rs = runtime->solv_type;
  s.riemann = !strcmp(rs, "hlld") ? GP_RS_HLLD : !strcmp(rs, "hllc") ? GP_RS_HLLC
            : !strcmp(rs, "tvdlf") ? GP_RS_TVDLF : GP_RS_HLL;
  #if defined(STAGGERED_MHD) && CT_EMF_AVERAGE == UCT_HLLD
  s.ct_emf = GP_CT_UCT_HLLD;
  #elif defined(STAGGERED_MHD) && CT_EMF_AVERAGE == ARITHMETIC
  s.ct_emf = GP_CT_ARITHMETIC;
  #else
  s.ct_emf = GP_CT_UCT_HLL;
  #endif
  #if TIME_STEPPING == RK3
  s.rk_stages = 3;
  #else
  s.rk_stages = 2;
  #endif
  #if RECONSTRUCTION == PARABOLIC
  s.reconstruction = GP_REC_PARABOLIC;
  #elif RECONSTRUCTION == MP5
  s.reconstruction = GP_REC_MP5;
  #elif RECONSTRUCTION == WENOZ
  s.reconstruction = GP_REC_WENOZ;
  #elif RECONSTRUCTION == LimO3
  s.reconstruction = GP_REC_LIMO3;
  #elif RECONSTRUCTION == WENO3
  s.reconstruction = GP_REC_WENO3;
  #else
  s.reconstruction = GP_REC_LINEAR;
  #endif
  s.precision   = GP_FP64;
  s.gamma       = run_config->gamma;
  s.cfl         = runtime->cfl;
  s.cfl_max_var = runtime->cfl_max_var;
  s.small_rho   = run_config->small_rho;
  s.small_prs   = run_config->small_prs;
  if (gp_create(&g, &s, NULL, &g_gp) != GP_OK) QuitPLUTO(gp_last_error(), 1);
  double *Uc, *Vc, *Vs[3];
  GP_Arrays(data, &Uc, &Vc, Vs);
  if (gp_upload_state(g_gp, GP_LAYOUT_REFERENCE, Uc, Vc, Vs[0], Vs[1], Vs[2]) != GP_OK)
    QuitPLUTO(gp_last_error(), 1);
  print("> gpluto-b200: the time step runs on the GPU (%s)\n", rs);
}

////////////////////////////////////////////////////////////////////////
void GP_DropIn_Step(Data *data, Grid *grid, timeStep *Dts)
/*
 * In place of AdvanceStep(data, grid, Dts): one step on the device, the
 * inverse time scale for NextTimeStep, and Data refreshed on the host (the
 * ghost zones filled as Boundary() would), so that output, analysis and the
 * log read the new state.
 */
{
  (void)grid;
  gp_step_out out;
  int rc = gp_advance_step(g_gp, Dts->dt, &out);
  if (rc == GP_ERR_QUIT) QuitPLUTO("from gp_advance_step()", out.err_bits);
  if (rc != GP_OK) QuitPLUTO(gp_last_error(), 1);
  Dts->invDt_hyp = out.invDt_hyp;
  double *Uc, *Vc, *Vs[3];
  GP_Arrays(data, &Uc, &Vc, Vs);
  if (gp_download_state(g_gp, GP_LAYOUT_REFERENCE, Uc, Vc, Vs[0], Vs[1], Vs[2]) != GP_OK)
    QuitPLUTO(gp_last_error(), 1);
}
