////////////////////////////////////////////////////////////////////////
// Problem file used to run the reference gPLUTO serial build as a parity
// checker (test infrastructure, never shipped or linked into the product).
//
// It replaces a Test_Problems/*/init.cpp: Init()/InitDomain()/Analysis()/
// UserDefBoundary() have the signatures of
// Test_Problems/MHD/Orszag_Tang/init.cpp:60-190.
//
//  - InitDomain() reads a seeded initial condition written by
//    gpluto_dev_b200/ics.py (file named by $GP_IC_FILE): interior primitive
//    variables and left-face magnetic fields.  Ghost zones are filled by
//    periodic wrap so that the start-up face average
//    (Src/startup.cpp:386-425) sees valid right faces.
//  - Analysis() runs before every step (ini: "analysis -1 1",
//    Src/main.cpp:697-712).  It logs dt and a wall-clock stamp per step and,
//    at step $GP_DUMP_STEP, writes the interior Vc, Uc and Vs to
//    $GP_DUMP_FILE and exits, so the dump holds the state after exactly
//    GP_DUMP_STEP steps.
////////////////////////////////////////////////////////////////////////
#include "gpluto.hpp"
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace {

struct IcFile {
  int loaded = 0;
  int physics, ndim, nx, ny, nz, nvar;
  double gamma, xbeg[3], xend[3];
  std::vector<double> V, Bs;
};

IcFile g_ic;
std::vector<double> g_dt_hist, g_t_hist, g_wall;

void LoadIC() {
  if (g_ic.loaded) return;
  const char *path = std::getenv("GP_IC_FILE");
  if (!path) QuitPLUTO("GP_IC_FILE not set", 1);
  FILE *fp = std::fopen(path, "rb");
  if (!fp) QuitPLUTO("cannot open GP_IC_FILE", 1);
  char magic[4];
  int hdr[7];
  double vals[7];
  if (std::fread(magic, 1, 4, fp) != 4 || std::memcmp(magic, "GPIC", 4))
    QuitPLUTO("bad IC magic", 1);
  if (std::fread(hdr, sizeof(int), 7, fp) != 7) QuitPLUTO("bad IC header", 1);
  if (std::fread(vals, sizeof(double), 7, fp) != 7) QuitPLUTO("bad IC header", 1);
  g_ic.physics = hdr[1]; g_ic.ndim = hdr[2];
  g_ic.nx = hdr[3]; g_ic.ny = hdr[4]; g_ic.nz = hdr[5]; g_ic.nvar = hdr[6];
  g_ic.gamma = vals[0];
  for (int d = 0; d < 3; d++) { g_ic.xbeg[d] = vals[1+d]; g_ic.xend[d] = vals[4+d]; }
  size_t ncell = (size_t)g_ic.nx*g_ic.ny*g_ic.nz;
  g_ic.V.resize(ncell*g_ic.nvar);
  if (std::fread(g_ic.V.data(), sizeof(double), g_ic.V.size(), fp) != g_ic.V.size())
    QuitPLUTO("short IC file (V)", 1);
  if (g_ic.physics != 0) {
    g_ic.Bs.resize(ncell*g_ic.ndim);
    if (std::fread(g_ic.Bs.data(), sizeof(double), g_ic.Bs.size(), fp) != g_ic.Bs.size())
      QuitPLUTO("short IC file (Bs)", 1);
  }
  std::fclose(fp);
  if (g_ic.nvar != NVAR) QuitPLUTO("IC NVAR mismatch", 1);
  g_ic.loaded = 1;
}

inline int Wrap(int i, int n) { i %= n; return i < 0 ? i + n : i; }

}  // namespace

////////////////////////////////////////////////////////////////////////
void Init (double *v, double x1, double x2, double x3, RunConfig &run_config)
{
  LoadIC();
  #if EOS == IDEAL
  run_config.gamma = g_ic.gamma;
  #endif
  int nv;
  NVAR_LOOP(nv) v[nv] = 0.0;
  v[RHO] = 1.0;
  #if HAVE_ENERGY
  v[PRS] = 1.0;
  #endif
}

////////////////////////////////////////////////////////////////////////
void InitDomain (Data *data, Grid *grid)
{
  LoadIC();
  int ibeg = grid->lbeg[IDIR], jbeg = grid->lbeg[JDIR], kbeg = grid->lbeg[KDIR];
  if (grid->nint[IDIR] != g_ic.nx || grid->nint[JDIR] != g_ic.ny ||
      grid->nint[KDIR] != g_ic.nz) QuitPLUTO("IC size mismatch", 1);
  const long nx = g_ic.nx, ny = g_ic.ny, nz = g_ic.nz;

  // cell-centred primitives, ghosts by periodic wrap
  for (int k = 0; k < grid->ntot[KDIR]; k++){
  for (int j = 0; j < grid->ntot[JDIR]; j++){
  for (int i = 0; i < grid->ntot[IDIR]; i++){
    long ii = Wrap(i - ibeg, nx), jj = Wrap(j - jbeg, ny), kk = Wrap(k - kbeg, nz);
    long c = ii + nx*(jj + ny*kk);
    for (int nv = 0; nv < NVAR; nv++)
      data->Vc(i,j,k,nv) = g_ic.V[c + (long)nv*nx*ny*nz];
  }}}

  #ifdef STAGGERED_MHD
  int (*ns)[3] = grid->ntot_stag;
  for (int d = 0; d < DIMENSIONS; d++){
    for (int k = 0; k < ns[d][KDIR]; k++){
    for (int j = 0; j < ns[d][JDIR]; j++){
    for (int i = 0; i < ns[d][IDIR]; i++){
      long ii = Wrap(i - ibeg, nx), jj = Wrap(j - jbeg, ny), kk = Wrap(k - kbeg, nz);
      long c = ii + nx*(jj + ny*kk);
      data->Vs[d](i,j,k) = g_ic.Bs[c + (long)d*nx*ny*nz];
    }}}
  }
  #endif
}

////////////////////////////////////////////////////////////////////////
static void DumpState (Data *data, Grid *grid, const char *path)
{
  FILE *fp = std::fopen(path, "wb");
  if (!fp) QuitPLUTO("cannot open GP_DUMP_FILE", 1);
  int ibeg = grid->lbeg[IDIR], iend = grid->lend[IDIR];
  int jbeg = grid->lbeg[JDIR], jend = grid->lend[JDIR];
  int kbeg = grid->lbeg[KDIR], kend = grid->lend[KDIR];
  int hdr[8] = {1, g_ic.physics, DIMENSIONS, grid->nint[IDIR], grid->nint[JDIR],
                grid->nint[KDIR], NVAR, (int)g_dt_hist.size()};
  std::fwrite("GPDM", 1, 4, fp);
  std::fwrite(hdr, sizeof(int), 8, fp);
  std::fwrite(g_dt_hist.data(), sizeof(double), g_dt_hist.size(), fp);
  std::fwrite(g_t_hist.data(), sizeof(double), g_t_hist.size(), fp);
  std::fwrite(g_wall.data(), sizeof(double), g_wall.size(), fp);
  std::vector<double> buf;
  for (int which = 0; which < 2; which++){
    const Ary4D &A = (which == 0 ? data->Vc : data->Uc);
    for (int nv = 0; nv < NVAR; nv++){
      buf.clear();
      for (int k = kbeg; k <= kend; k++)
      for (int j = jbeg; j <= jend; j++)
      for (int i = ibeg; i <= iend; i++) buf.push_back(A(i,j,k,nv));
      std::fwrite(buf.data(), sizeof(double), buf.size(), fp);
    }
  }
  #ifdef STAGGERED_MHD
  for (int d = 0; d < DIMENSIONS; d++){
    buf.clear();
    for (int k = kbeg; k <= kend; k++)
    for (int j = jbeg; j <= jend; j++)
    for (int i = ibeg; i <= iend; i++) buf.push_back(data->Vs[d](i,j,k));
    std::fwrite(buf.data(), sizeof(double), buf.size(), fp);
  }
  #endif
  std::fclose(fp);
}

////////////////////////////////////////////////////////////////////////
void Analysis (Data *data, Grid *grid)
{
  using clk = std::chrono::steady_clock;
  static const clk::time_point t0 = clk::now();
  g_wall.push_back(std::chrono::duration<double>(clk::now() - t0).count());
  g_dt_hist.push_back(data->Dts->dt);
  g_t_hist.push_back(data->Dts->time);
  const char *s = std::getenv("GP_DUMP_STEP");
  long target = s ? std::atol(s) : -1;
  if (g_stepNumber == target) {
    const char *path = std::getenv("GP_DUMP_FILE");
    if (path) DumpState(data, grid, path);
    std::fflush(stdout);
    std::exit(0);
  }
}

////////////////////////////////////////////////////////////////////////
// USERDEF sides of the parity cases: an inflow.  Every ghost cell of the
// side takes the primitive state of the domain cell next to the side, then
// the fixed density kUdRho and the normal velocity kUdVn pointing into the
// domain; the tangential staggered fields copy the domain face next to the
// side (one face wider along their own direction).  The normal staggered
// field and the ghost cell-centred B are left to the framework
// (CT_FillStaggeredFields and the averages, Src/boundary.cpp:238-307).
static const double kUdRho = 1.25, kUdVn = 0.25;

void UserDefBoundary (const Data *data, RBox *box, int side, Grid *grid)
{
  if (side < X1_BEG || side > X3_END) return;
  const int d = (side - X1_BEG)/2, beg = ((side - X1_BEG)%2 == 0);
  const int m0 = beg ? grid->lbeg[d] : grid->lend[d];
  const int lo[3] = {box->ibeg, box->jbeg, box->kbeg};
  const int hi[3] = {box->iend, box->jend, box->kend};
  for (int k = lo[2]; k <= hi[2]; k++){
  for (int j = lo[1]; j <= hi[1]; j++){
  for (int i = lo[0]; i <= hi[0]; i++){
    int s[3] = {i, j, k};
    s[d] = m0;
    for (int nv = 0; nv < NVAR; nv++) data->Vc(i,j,k,nv) = data->Vc(s[0],s[1],s[2],nv);
    data->Vc(i,j,k,RHO) = kUdRho;
    data->Vc(i,j,k,VX1+d) = beg ? kUdVn : -kUdVn;
  }}}
  #ifdef STAGGERED_MHD
  for (int c = 0; c < DIMENSIONS; c++){
    if (c == d) continue;
    int h[3] = {hi[0], hi[1], hi[2]};
    h[c] += 1;
    for (int k = lo[2]; k <= h[2]; k++){
    for (int j = lo[1]; j <= h[1]; j++){
    for (int i = lo[0]; i <= h[0]; i++){
      int s[3] = {i, j, k};
      s[d] = m0;
      data->Vs[c](i,j,k) = data->Vs[c](s[0],s[1],s[2]);
    }}}
  }
  #endif
}
