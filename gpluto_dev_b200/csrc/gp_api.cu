// gp_api.cu -- C ABI (include/gpluto_b200.h) over the sm_100a stage kernels.
//
// Owns the device state of one grid, orders the RK2 stages exactly like
// AdvanceStep (Src/rk_step.cpp:88-593) and keeps the dt sequence on the
// device so that many steps run without a host round trip
// (NextTimeStep, Src/next_time_step.cpp:20-130, evaluated by a one-thread
// kernel after each step).  There is no CPU fallback: every entry point that
// computes fails with GP_ERR_NO_DEVICE when no CUDA device is present.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/gpluto_b200.h"
#include "gp_checks.h"
#include "gp_launch.h"

namespace {

thread_local char g_err[512] = "";

int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

#define CUDA_TRY(call)                                                              \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess)                                                          \
      return fail(GP_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                  __FILE__, __LINE__);                                              \
  } while (0)

// Per-step scalars living in device memory.
struct StepScalars {
  double dt;                 // dt of the step about to run
  double dtdx[3];            // dt/dx_d for that step
  double invdt;              // stage-1 invDt_hyp of the last step
  double dt_next;            // NextTimeStep of the last step
  unsigned long long invdt_bits;  // running max of C_dt (stage 1)
  uint32_t err;              // OR of error bits since the last reset
  uint32_t pad;
};

// NextTimeStep + bookkeeping; one thread.  Src/update_stage.cpp:422-435
// (invDt_hyp = max(C_dt)/dim) and Src/next_time_step.cpp:80,125.
__global__ void dt_update_kernel(StepScalars* sc, double ndim, double cfl, double cfl_max_var,
                                 double dx0, double dx1, double dx2, double* hist, int slot) {
  double mx = __longlong_as_double((long long)sc->invdt_bits);
  double inv = mx / ndim;
  double dt = sc->dt;
  if (hist) hist[slot] = dt;
  double dtn = cfl / inv;
  dtn = (dtn <= cfl_max_var * dt) ? dtn : cfl_max_var * dt;
  sc->invdt = inv;
  sc->dt_next = dtn;
  sc->dt = dtn;
  sc->dtdx[0] = dtn / dx0;
  sc->dtdx[1] = dtn / dx1;
  sc->dtdx[2] = dtn / dx2;
  sc->invdt_bits = 0ull;
}

constexpr int kBX1 = 4;  // first field component (Src/MHD/mhd.hpp:21-41, Src/RMHD/rmhd.hpp:21-42)

// Device array extents: the domain (n*) sits at offset l* inside the
// allocated extents p* (p = n, l = 0 unless the direction is padded).
struct Pad {
  int nx, ny, nz, px, py, pz, lx, ly, lz;
};

// host layout with extents s* and domain offset o* (reference layout, or
// interior layout with s = n, o = 0) -> domain of the device array
__global__ void gather_kernel(const double* __restrict__ src, double* __restrict__ dst,
                              int nvar, int sx, int sy, int sz, int ox, int oy, int oz, Pad p) {
  long long n = (long long)p.nx * p.ny * p.nz;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * nvar) return;
  int nv = (int)(t / n);
  long long c = t - (long long)nv * n;
  int i = (int)(c % p.nx), j = (int)((c / p.nx) % p.ny), k = (int)(c / ((long long)p.nx * p.ny));
  long long s = (long long)(i + ox) + (long long)sx * ((j + oy) + (long long)sy * (k + oz));
  long long d = (long long)(i + p.lx) + (long long)p.px * ((j + p.ly) + (long long)p.py * (k + p.lz));
  dst[(long long)nv * p.px * p.py * p.pz + d] = src[(long long)nv * sx * sy * sz + s];
}

// device index of host-layout position i (domain-relative) along d: with
// `own` a padded direction reads its own ghost cells; otherwise periodic
// wrap, or the nearest domain cell on an outflow side
__device__ int ghost_src(int i, int n, int l, int own, unsigned clamp, int d) {
  if (own && l > 0) return i + l;
  if (i < 0 && ((clamp >> (2 * d)) & 1u)) return l;
  if (i >= n && ((clamp >> (2 * d + 1)) & 1u)) return l + n - 1;
  return (i % n + n) % n + l;
}

// device array -> host layout with extents s* and domain offset o*; the
// ghost zones come out the way Boundary() fills them.  `clamp` lists the
// outflow sides filled by copying the nearest domain cell.
__global__ void scatter_kernel(const double* __restrict__ src, double* __restrict__ dst,
                               int nvar, int sx, int sy, int sz, int ox, int oy, int oz, Pad p,
                               unsigned clamp, int own) {
  long long ns = (long long)sx * sy * sz;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ns * nvar) return;
  int nv = (int)(t / ns);
  long long s = t - (long long)nv * ns;
  int i = (int)(s % sx), j = (int)((s / sx) % sy), k = (int)(s / ((long long)sx * sy));
  int ii = ghost_src(i - ox, p.nx, p.lx, own, clamp, 0),
      jj = ghost_src(j - oy, p.ny, p.ly, own, clamp, 1),
      kk = ghost_src(k - oz, p.nz, p.lz, own, clamp, 2);
  dst[t] = src[(long long)nv * p.px * p.py * p.pz + ii + (long long)p.px * (jj + (long long)p.py * kk)];
}

// high-side face of a padded direction d (left face of the first ghost cell)
// from the low-side face: the periodic completion of an interior-layout field
__global__ void wrap_face_kernel(double* B, Pad p, int d) {
  const int P[3] = {p.px, p.py, p.pz};
  const int L[3] = {p.lx, p.ly, p.lz};
  const int N[3] = {p.nx, p.ny, p.nz};
  const int a = (d == 0) ? 1 : 0, b = (d == 2) ? 1 : 2;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)P[a] * P[b]) return;
  int q[3];
  q[a] = (int)(t % P[a]);
  q[b] = (int)(t / P[a]);
  q[d] = L[d];
  const long long c0 = (long long)q[0] + (long long)P[0] * (q[1] + (long long)P[1] * q[2]);
  q[d] = L[d] + N[d];
  const long long c1 = (long long)q[0] + (long long)P[0] * (q[1] + (long long)P[1] * q[2]);
  B[c1] = B[c0];
}

// Outflow side of a padded grid with constrained transport (Boundary(),
// Src/boundary.cpp:184-307 for one side): the ghost cells of the side copy
// the domain cell next to it (OutflowBoundary, Src/boundary.cpp:677-780),
// tangential staggered fields likewise; the normal staggered field is
// marched outward from div B = 0 with the Cartesian face areas
// (CT_FillStaggeredFields, Src/MHD/CT/ct_fill_mag_field.cpp:96-330); the
// ghost cells' B is then the average of their faces
// (Src/MHD/CT/ct_field_average.cpp:175-200).  One thread per transverse
// position of the side, over the whole padded extent of the other
// directions; the sides run in the reference's order.  The march reads the
// tangential faces of the neighbouring positions, so every side takes two
// launches: the copies (outflow_copy_kernel), then the march and the
// averages (outflow_march_kernel).
struct SideGeom {
  int P[3], L[3], N[3], d, a, b;
  long long pn;
  __device__ long long idx(int m, int ia, int ib) const {
    int q[3];
    q[d] = m;
    q[a] = ia;
    q[b] = ib;
    return (long long)q[0] + (long long)P[0] * (q[1] + (long long)P[1] * q[2]);
  }
};

__device__ __forceinline__ SideGeom side_geom(const Pad& p, int d) {
  SideGeom s;
  s.P[0] = p.px; s.P[1] = p.py; s.P[2] = p.pz;
  s.L[0] = p.lx; s.L[1] = p.ly; s.L[2] = p.lz;
  s.N[0] = p.nx; s.N[1] = p.ny; s.N[2] = p.nz;
  s.d = d;
  s.a = (d == 0) ? 1 : 0;
  s.b = (d == 2) ? 1 : 2;
  s.pn = (long long)p.px * p.py * p.pz;
  return s;
}

// cell-centred B of the side's ghost cells at transverse position (ta, tb)
// from the faces around each (Src/MHD/CT/ct_field_average.cpp:175-200)
__device__ void ghost_average(const SideGeom& s, double* V, double* const* B, int ndim, int ta,
                              int tb, int beg) {
  const int d = s.d, a = s.a, b = s.b;
  const int L = s.L[d], N = s.N[d], P = s.P[d];
  const int g0 = beg ? 0 : L + N, g1 = beg ? L - 1 : P - 1;
  for (int g = g0; g <= g1; g++) {
    const long long c = s.idx(g, ta, tb);
    for (int e = 0; e < ndim; e++) {
      long long cn;
      if (e == d) {
        if (g + 1 >= P) continue;  // the extra padding cell: not a reference ghost
        cn = s.idx(g + 1, ta, tb);
      } else if (e == a) {
        cn = s.idx(g, (ta + 1) % s.P[a], tb);
      } else {
        cn = s.idx(g, ta, (tb + 1) % s.P[b]);
      }
      V[(kBX1 + e) * s.pn + c] = 0.5 * (B[e][c] + B[e][cn]);
    }
  }
}

__global__ void outflow_copy_kernel(double* __restrict__ V, int nvar, double* B0, double* B1,
                                    double* B2, int nb, Pad p, int d, int beg) {
  const SideGeom s = side_geom(p, d);
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)s.P[s.a] * s.P[s.b]) return;
  const int ta = (int)(t % s.P[s.a]), tb = (int)(t / s.P[s.a]);
  double* B[3] = {B0, B1, B2};
  const int m0 = beg ? s.L[d] : s.L[d] + s.N[d] - 1;      // domain cell next to the side
  const int g0 = beg ? 0 : s.L[d] + s.N[d], g1 = beg ? s.L[d] - 1 : s.P[d] - 1;  // ghosts
  const long long c0 = s.idx(m0, ta, tb);
  for (int g = g0; g <= g1; g++) {
    const long long c = s.idx(g, ta, tb);
    for (int nv = 0; nv < nvar; nv++) V[nv * s.pn + c] = V[nv * s.pn + c0];
    for (int e = 0; e < nb; e++)
      if (e != d) B[e][c] = B[e][c0];
  }
}

__global__ void outflow_march_kernel(double* __restrict__ V, double* B0, double* B1, double* B2,
                                     int ndim, Pad p, int d, int beg, double A0, double A1,
                                     double A2) {
  const SideGeom s = side_geom(p, d);
  const int a = s.a, b = s.b;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)s.P[a] * s.P[b]) return;
  const int ta = (int)(t % s.P[a]), tb = (int)(t / s.P[a]);
  const int L = s.L[d], N = s.N[d], P = s.P[d];
  double* B[3] = {B0, B1, B2};
  const double A[3] = {A0, A1, A2};
  // transverse difference A_e*(B_e(next along e) - B_e(here)) at ghost cell m
  auto dB = [&](int e, int m) -> double {
    if (e >= ndim) return 0.0;
    int ia = ta, ib = tb;
    if (e == a) ia = (ta + 1) % s.P[a];
    else ib = (tb + 1) % s.P[b];
    return A[e] * B[e][s.idx(m, ia, ib)] - A[e] * B[e][s.idx(m, ta, tb)];
  };
  if (beg) {
    for (int m = L - 1; m >= 0; m--)
      B[d][s.idx(m, ta, tb)] = (A[d] * B[d][s.idx(m + 1, ta, tb)] + dB(a, m) + dB(b, m)) / A[d];
  } else {
    for (int m = L + N; m + 1 < P; m++)
      B[d][s.idx(m + 1, ta, tb)] = (A[d] * B[d][s.idx(m, ta, tb)] - (dB(a, m) + dB(b, m))) / A[d];
  }
  ghost_average(s, V, B, ndim, ta, tb, beg);
}

// Mirrored side of a padded grid (ReflectiveBoundary with the signs of
// FlipSign, Src/boundary.cpp:838-1060): ghost cell g copies its mirror image
// across the boundary face times the variable's sign (bit nv of `flip`
// set: -1); the normal staggered field mirrors across the boundary face,
// which keeps its value; tangential faces mirror like the cells.  The extra
// high-side padding cell (not a reference ghost) repeats the last ghost.
__global__ void reflect_copy_kernel(double* __restrict__ V, int nvar, double* B0, double* B1,
                                    double* B2, int nb, Pad p, int d, int beg, unsigned flip) {
  const SideGeom s = side_geom(p, d);
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)s.P[s.a] * s.P[s.b]) return;
  const int ta = (int)(t % s.P[s.a]), tb = (int)(t / s.P[s.a]);
  const int L = s.L[d], N = s.N[d], P = s.P[d];
  double* B[3] = {B0, B1, B2};
  auto sgn = [&](int nv) -> double { return ((flip >> nv) & 1u) ? -1.0 : 1.0; };
  const int g0 = beg ? 0 : L + N, g1 = beg ? L - 1 : L + N + L - 1;   // reference ghosts
  const int i0 = beg ? 2 * L - 1 : 2 * (L + N - 1) + 1;              // mirror of g: i0 - g
  for (int g = g0; g <= g1; g++) {
    const long long c = s.idx(g, ta, tb), cm = s.idx(i0 - g, ta, tb);
    for (int nv = 0; nv < nvar; nv++) V[nv * s.pn + c] = sgn(nv) * V[nv * s.pn + cm];
    for (int e = 0; e < nb; e++) {
      const double se = sgn(kBX1 + e);
      if (e != d) {
        B[e][c] = se * B[e][cm];
      } else if (beg) {
        B[e][c] = se * B[e][s.idx(i0 - g + 1, ta, tb)];        // face g from face i0-g+1
      } else {
        B[e][s.idx(g + 1, ta, tb)] = se * B[e][cm];             // face g+1 from face i0-g
      }
    }
  }
  if (!beg && P - 1 > g1) {  // the extra padding cell: finite copies of the last ghost
    const long long c = s.idx(P - 1, ta, tb), cl = s.idx(g1, ta, tb);
    for (int nv = 0; nv < nvar; nv++) V[nv * s.pn + c] = V[nv * s.pn + cl];
    for (int e = 0; e < nb; e++)
      if (e != d) B[e][c] = B[e][cl];
  }
}

// Ghost cells' B from their faces (Src/boundary.cpp:260-307), after the
// side's faces are all set: its own launch, since it reads the tangential
// faces of the neighbouring positions.
__global__ void ghost_average_kernel(double* __restrict__ V, double* B0, double* B1, double* B2,
                                     int ndim, Pad p, int d, int beg) {
  const SideGeom s = side_geom(p, d);
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)s.P[s.a] * s.P[s.b]) return;
  double* B[3] = {B0, B1, B2};
  ghost_average(s, V, B, ndim, (int)(t % s.P[s.a]), (int)(t / s.P[s.a]), beg);
}

// The extra high-side padding cell of a user-filled side (not a reference
// ghost): finite copies of the last ghost, as for a mirrored side.
__global__ void extra_cell_kernel(double* __restrict__ V, int nvar, double* B0, double* B1,
                                  double* B2, int nb, Pad p, int d) {
  const SideGeom s = side_geom(p, d);
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)s.P[s.a] * s.P[s.b]) return;
  const int ta = (int)(t % s.P[s.a]), tb = (int)(t / s.P[s.a]);
  double* B[3] = {B0, B1, B2};
  const long long c = s.idx(s.P[d] - 1, ta, tb), cl = s.idx(s.P[d] - 2, ta, tb);
  for (int nv = 0; nv < nvar; nv++) V[nv * s.pn + c] = V[nv * s.pn + cl];
  for (int e = 0; e < nb; e++)
    if (e != d) B[e][c] = B[e][cl];
}

bool uniform(const double* dx, int n) {
  if (!dx) return true;
  for (int i = 1; i < n; i++)
    if (dx[i] != dx[0]) return false;
  return true;
}

}  // namespace

struct gp_handle {
  gp_grid_desc grid;
  gp_scheme scheme;
  int nx, ny, nz, ndim, nvar, ng;
  long long n;
  double dx[3];
  cudaStream_t stream;
  bool mixed;
  gp::SchemeKey key;
  int seg;
  // device state
  double* U[2];
  double* V;
  double* dU;
  double* Cdt;
  double* Bs[3][3];   // [rotation buffer][component]
  int bcur;           // buffer holding B^n
  void* ct[3][6];
  double* Ee[3];
  StepScalars* sc;
  StepScalars* sc_host;  // pinned mirror
  double* hist;
  int hist_cap;
  double* stage_buf;     // device staging for reference-layout transfers
  size_t stage_bytes;
  int launches_per_step;
  unsigned outflow;      // outflow sides (bit 2d low, 2d+1 high)
  unsigned reflect;      // reflective (or axisymmetric) sides, same bits
  unsigned eqtsym;       // equatorially symmetric sides, same bits
  unsigned userdef;      // user-filled sides, same bits
  gp_userdef_fn ud_fn;   // the user's fill and its argument
  void* ud_user;
  // Outflow with constrained transport pads the outflow directions with
  // ghost cells filled before every stage (S = ghost cells of the scheme,
  // plus one on the high side so that the outermost ghost's faces exist).
  bool padded;
  int lo[3], hi[3];      // padding cells below / above the domain
  int px, py, pz;        // allocated extents
  long long pn;          // allocated cells
  double A[3];           // Cartesian face areas (Src/set_geometry.cpp:124-165)
};

namespace {

void free_all(gp_handle* h) {
  cudaFree(h->U[0]);
  cudaFree(h->U[1]);
  cudaFree(h->V);
  cudaFree(h->dU);
  cudaFree(h->Cdt);
  for (int b = 0; b < 3; b++)
    for (int d = 0; d < 3; d++) cudaFree(h->Bs[b][d]);
  for (int d = 0; d < 3; d++) {
    for (int r = 0; r < 6; r++) cudaFree(h->ct[d][r]);
    cudaFree(h->Ee[d]);
  }
  cudaFree(h->sc);
  cudaFreeHost(h->sc_host);
  cudaFree(h->hist);
  cudaFree(h->stage_buf);
}

Pad pad_of(const gp_handle* h) {
  return Pad{h->nx, h->ny, h->nz, h->px, h->py, h->pz, h->lo[0], h->lo[1], h->lo[2]};
}

gp::GridDims grid_dims(const gp_handle* h) {
  gp::GridDims g{h->px, h->py, h->pz, h->pn, h->padded ? 0u : h->outflow};
  if (h->padded) {
    const int n[3] = {h->nx, h->ny, h->nz};
    for (int d = 0; d < 3; d++) {
      if (h->lo[d] == 0 && h->hi[d] == 0) continue;  // periodic: every cell counts
      g.ilo[d] = h->lo[d];
      g.ihi[d] = h->lo[d] + n[d] - 1;
      g.glo[d] = 0;                                    // the reference's ghost zone
      g.ghi[d] = h->lo[d] + n[d] - 1 + h->lo[d];
    }
  }
  return g;
}

// ghost zones of the non-periodic sides of a padded grid, sides in the
// reference's order (Src/boundary.cpp:144-310)
int fill_boundaries(gp_handle* h, double* const* Bs, int stage) {
  const Pad p = pad_of(h);
  const int P[3] = {h->px, h->py, h->pz};
  const int nb = h->scheme.physics == GP_HD ? 0 : h->ndim;  // staggered components
  for (int side = 0; side < 2 * h->ndim; side++) {
    const unsigned bit = 1u << side;
    if (!((h->outflow | h->reflect | h->eqtsym | h->userdef) & bit)) continue;
    const int d = side / 2, beg = side % 2 == 0;
    const int a = (d == 0) ? 1 : 0, b = (d == 2) ? 1 : 2;
    const long long nt = (long long)P[a] * P[b];
    const unsigned nblk = (unsigned)((nt + 127) / 128);
    if (h->userdef & bit) {
      // UserDefBoundary, then CT_FillStaggeredFields and the ghost averages
      // (Src/boundary.cpp:238-307)
      if (!h->ud_fn)
        return fail(GP_ERR_INVALID, "USERDEF side %d without a fill (gp_set_userdef_boundary)",
                    side);
      gp_userdef_side u;
      std::memset(&u, 0, sizeof(u));
      const int n[3] = {h->nx, h->ny, h->nz};
      u.side = side;
      u.stage = stage;
      for (int e = 0; e < 3; e++) {
        u.beg[e] = 0;
        u.end[e] = P[e] - 1;
        u.dom_beg[e] = h->lo[e];
        u.nint[e] = n[e];
        u.dims[e] = P[e];
      }
      u.beg[d] = beg ? 0 : h->lo[d] + n[d];
      u.end[d] = beg ? h->lo[d] - 1 : h->lo[d] + n[d] + h->lo[d] - 1;
      u.nvar = h->nvar;
      u.V = h->V;
      for (int e = 0; e < nb; e++) u.Vs[e] = Bs[e];
      const int rc = h->ud_fn(h->ud_user, &u, (void*)h->stream);
      if (rc != 0) return fail(GP_ERR_INVALID, "USERDEF fill of side %d returned %d", side, rc);
      if (!beg)
        extra_cell_kernel<<<nblk, 128, 0, h->stream>>>(h->V, h->nvar, Bs[0], Bs[1], Bs[2], nb, p,
                                                       d);
      if (nb)
        outflow_march_kernel<<<nblk, 128, 0, h->stream>>>(h->V, Bs[0], Bs[1], Bs[2], h->ndim, p,
                                                          d, beg, h->A[0], h->A[1], h->A[2]);
      continue;
    }
    if (h->outflow & bit) {
      outflow_copy_kernel<<<nblk, 128, 0, h->stream>>>(h->V, h->nvar, Bs[0], Bs[1], Bs[2], nb,
                                                       p, d, beg);
      if (nb)
        outflow_march_kernel<<<nblk, 128, 0, h->stream>>>(h->V, Bs[0], Bs[1], Bs[2], h->ndim, p,
                                                          d, beg, h->A[0], h->A[1], h->A[2]);
      continue;
    }
    // FlipSign (Src/boundary.cpp:838-920): v_n always; B_n for REFLECTIVE
    // (and AXISYMMETRIC), B_t and B_b for EQTSYMMETRIC
    unsigned flip = 1u << (1 + d);                                    // VX1 + d
    if (nb) {
      if (h->eqtsym & bit) flip |= (1u << (kBX1 + (d + 1) % 3)) | (1u << (kBX1 + (d + 2) % 3));
      else flip |= 1u << (kBX1 + d);
    }
    reflect_copy_kernel<<<nblk, 128, 0, h->stream>>>(h->V, h->nvar, Bs[0], Bs[1], Bs[2], nb, p,
                                                     d, beg, flip);
    if (nb)
      ghost_average_kernel<<<nblk, 128, 0, h->stream>>>(h->V, Bs[0], Bs[1], Bs[2], h->ndim, p, d,
                                                        beg);
  }
  return GP_OK;
}

int enqueue_step(gp_handle* h, double* hist, int slot, cudaEvent_t* ev = nullptr) {
  const int b0 = h->bcur, b1 = (h->bcur + 1) % 3, b2 = (h->bcur + 2) % 3;
  const bool mhd = h->scheme.physics != GP_HD;
  gp::StageDesc d;
  std::memset(&d, 0, sizeof(d));
  d.dU = h->dU;
  d.Cdt = h->Cdt;
  for (int q = 0; q < 3; q++) {
    d.dx[q] = h->dx[q];
    d.Ee[q] = h->Ee[q];
    for (int r = 0; r < 6; r++) d.ct[q][r] = h->ct[q][r];
  }
  d.dtdx = h->sc->dtdx;
  d.gamma = h->scheme.gamma;
  d.small_rho = h->scheme.small_rho;
  d.small_prs = h->scheme.small_prs;
  d.invdt_bits = &h->sc->invdt_bits;
  d.err = &h->sc->err;
  const int per_stage = gp::stage_launch_count(h->key);
  auto launch = [&](const gp::StageDesc& sd) {
    gp::GridDims g = grid_dims(h);
    cudaEvent_t* e = ev ? ev + (sd.stage - 1) * 2 * per_stage : nullptr;
    return h->mixed ? gp::launch_stage_mixed(sd, g, h->key, h->seg, h->stream, e)
                    : gp::launch_stage_fp64(sd, g, h->key, h->seg, h->stream, e);
  };
  // stage 1: (U^n, B^n) -> (U1, B1)
  if (h->padded) {
    const int r = fill_boundaries(h, h->Bs[b0], 1);
    if (r) return r;
  }
  d.stage = 1;
  d.V = h->V;
  d.Vout = h->V;
  d.U0 = h->U[0];
  d.Uc = h->U[0];
  d.Uout = h->U[1];
  for (int q = 0; q < 3; q++) {
    d.Bs[q] = mhd ? h->Bs[b0][q] : nullptr;
    d.Bs0[q] = d.Bs[q];
    d.Bsout[q] = mhd ? h->Bs[b1][q] : nullptr;
  }
  if (launch(d) != 0) return fail(GP_ERR_UNSUPPORTED, "scheme not compiled");
  if (h->scheme.rk_stages == 3) {
    // RK3 stage 2: (U^n, U1, B^n, B1) -> (U2 in place of U1, B2); stage 3:
    // (U^n, U2, B^n, B2) -> (U^{n+1} in place of U^n, B^{n+1} in B1's buffer).
    // The finish reads only its own cell's U and its neighbours' input faces,
    // so cells update in place and faces rotate (Src/rk_step.cpp:30-61)
    if (h->padded) {
      const int r = fill_boundaries(h, h->Bs[b1], 2);
      if (r) return r;
    }
    d.stage = 2;
    d.w0 = 0.75;
    d.w1 = 0.25;
    d.wr = 0.25;
    d.Uc = h->U[1];
    d.Uout = h->U[1];
    for (int q = 0; q < 3; q++) {
      d.Bs[q] = mhd ? h->Bs[b1][q] : nullptr;
      d.Bs0[q] = mhd ? h->Bs[b0][q] : nullptr;
      d.Bsout[q] = mhd ? h->Bs[b2][q] : nullptr;
    }
    if (launch(d) != 0) return fail(GP_ERR_UNSUPPORTED, "scheme not compiled");
    if (h->padded) {
      const int r = fill_boundaries(h, h->Bs[b2], 3);
      if (r) return r;
    }
    d.stage = 3;
    d.w0 = 1.0 / 3.0;
    d.w1 = 2.0 / 3.0;
    d.wr = 2.0 / 3.0;
    d.Uc = h->U[1];
    d.Uout = h->U[0];
    for (int q = 0; q < 3; q++) {
      d.Bs[q] = mhd ? h->Bs[b2][q] : nullptr;
      d.Bs0[q] = mhd ? h->Bs[b0][q] : nullptr;
      d.Bsout[q] = mhd ? h->Bs[b1][q] : nullptr;
    }
    if (launch(d) != 0) return fail(GP_ERR_UNSUPPORTED, "scheme not compiled");
  } else {
    // stage 2: (U^n, U1, B^n, B1) -> (U^{n+1} in place of U^n, B^{n+1})
    if (h->padded) {
      const int r = fill_boundaries(h, h->Bs[b1], 2);
      if (r) return r;
    }
    d.stage = 2;
    d.w0 = d.w1 = d.wr = 0.5;
    d.Uc = h->U[1];
    d.Uout = h->U[0];
    for (int q = 0; q < 3; q++) {
      d.Bs[q] = mhd ? h->Bs[b1][q] : nullptr;
      d.Bs0[q] = mhd ? h->Bs[b0][q] : nullptr;
      d.Bsout[q] = mhd ? h->Bs[b2][q] : nullptr;
    }
    if (launch(d) != 0) return fail(GP_ERR_UNSUPPORTED, "scheme not compiled");
  }
  dt_update_kernel<<<1, 1, 0, h->stream>>>(h->sc, (double)h->ndim, h->scheme.cfl,
                                          h->scheme.cfl_max_var, h->dx[0], h->dx[1], h->dx[2],
                                          hist, slot);
  CUDA_TRY(cudaGetLastError());
  h->bcur = h->scheme.rk_stages == 3 ? b1 : b2;
  return GP_OK;
}

int set_dt(gp_handle* h, double dt) {
  h->sc_host->dt = dt;
  for (int q = 0; q < 3; q++) h->sc_host->dtdx[q] = dt / h->dx[q];
  h->sc_host->invdt = 0.0;
  h->sc_host->dt_next = 0.0;
  h->sc_host->invdt_bits = 0ull;
  h->sc_host->err = 0u;
  CUDA_TRY(cudaMemcpyAsync(h->sc, h->sc_host, sizeof(StepScalars), cudaMemcpyHostToDevice,
                           h->stream));
  return GP_OK;
}

int check_device() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
    return fail(GP_ERR_NO_DEVICE, "no CUDA device: the Godunov step has no CPU path");
  return GP_OK;
}

}  // namespace

namespace gp {
int set_last_error(int code, const char* msg) { return fail(code, "%s", msg); }

int validate_scheme(const gp_grid_desc* grid, const gp_scheme* scheme) {
  if (!grid || !scheme) return fail(GP_ERR_INVALID, "null argument");
  if (grid->ndim != 2 && grid->ndim != 3) return fail(GP_ERR_UNSUPPORTED, "ndim must be 2 or 3");
  if (scheme->physics != GP_MHD && scheme->physics != GP_HD && scheme->physics != GP_RMHD)
    return fail(GP_ERR_UNSUPPORTED, "physics %d not built", scheme->physics);
  if (scheme->physics == GP_RMHD && (scheme->riemann == GP_RS_HLLC || scheme->ct_emf != GP_CT_UCT_HLL))
    return fail(GP_ERR_UNSUPPORTED, "RMHD is built with HLLD/HLL and UCT_HLL "
                "(the reference RMHD HLLD stores no UCT_HLLD data, Src/RMHD/hlld.cpp:526-537)");
  if (scheme->rk_stages != 2 && scheme->rk_stages != 3)
    return fail(GP_ERR_UNSUPPORTED, "TIME_STEPPING RK2 and RK3 are built");
  if (scheme->precision != GP_FP64 && scheme->precision != GP_MIXED)
    return fail(GP_ERR_INVALID, "bad precision");
  for (int d = 0; d < 3; d++) {
    if (d < grid->ndim) {
      if (grid->nint[d] < 2) return fail(GP_ERR_INVALID, "nint[%d] < 2", d);
      const int lb = grid->lbound[d], rb = grid->rbound[d];
      auto known = [](int t) {
        return (t >= GP_BC_PERIODIC && t <= GP_BC_EQTSYMMETRIC) || t == GP_BC_USERDEF;
      };
      if (!known(lb) || !known(rb))
        return fail(GP_ERR_UNSUPPORTED,
                    "boundary types are periodic, outflow, reflective, axisymmetric, "
                    "eqtsymmetric or userdef");
      if ((lb == GP_BC_PERIODIC) != (rb == GP_BC_PERIODIC))
        return fail(GP_ERR_INVALID, "a periodic direction needs both sides periodic");

      if (!uniform(grid->dx[d], grid->nint[d] + 2 * grid->nghost))
        return fail(GP_ERR_UNSUPPORTED, "non-uniform grid along %d", d);
    }
  }
  if (scheme->physics == GP_MHD && scheme->ct_emf == GP_CT_UCT_HLLD &&
      scheme->riemann != GP_RS_HLLD)
    return fail(GP_ERR_UNSUPPORTED, "UCT_HLLD pairs with hlld only (Src/MHD/hll.cpp:73-77, "
                "Src/MHD/tvdlf.cpp:83-87, Src/MHD/hllc.cpp:79-83)");
  if (scheme->physics != GP_HD && scheme->ct_emf != GP_CT_UCT_HLL &&
      scheme->ct_emf != GP_CT_UCT_HLLD &&
      !((scheme->ct_emf == GP_CT_ARITHMETIC || scheme->ct_emf == GP_CT_CONTACT) &&
        scheme->physics == GP_MHD))
    return fail(GP_ERR_UNSUPPORTED, "CT_EMF_AVERAGE %d not built for this physics",
                scheme->ct_emf);
  if (scheme->riemann < GP_RS_HLL || scheme->riemann > GP_RS_TVDLF)
    return fail(GP_ERR_UNSUPPORTED, "riemann solver %d not built", scheme->riemann);
  if (scheme->physics == GP_HD && scheme->riemann == GP_RS_HLLD)
    return fail(GP_ERR_UNSUPPORTED, "HD has no HLLD solver");
  if (scheme->reconstruction != GP_REC_LINEAR && scheme->reconstruction != GP_REC_PARABOLIC &&
      scheme->reconstruction != GP_REC_MP5 && scheme->reconstruction != GP_REC_WENOZ &&
      scheme->reconstruction != GP_REC_LIMO3 && scheme->reconstruction != GP_REC_WENO3)
    return fail(GP_ERR_UNSUPPORTED, "reconstruction %d not built", scheme->reconstruction);
  if (scheme->reconstruction == GP_REC_LINEAR &&
      !((scheme->limiter >= GP_LIM_FLAT && scheme->limiter <= GP_LIM_MC) ||
        (scheme->limiter >= GP_LIM_VANALBADA && scheme->limiter <= GP_LIM_UMIST)))
    return fail(GP_ERR_UNSUPPORTED, "limiter %d not built", scheme->limiter);
  // ghost depth of the scheme (Src/get_nghost.cpp:33-44): 3 for the
  // PARABOLIC, MP5 and WENOZ stencils, 2 for LINEAR, LimO3 and WENO3
  const bool wide = scheme->reconstruction == GP_REC_PARABOLIC ||
                    scheme->reconstruction == GP_REC_MP5 ||
                    scheme->reconstruction == GP_REC_WENOZ;
  if (wide)
    for (int d = 0; d < grid->ndim; d++)
      if (grid->nint[d] < 4)
        return fail(GP_ERR_INVALID,
                    "PPM, MP5 and WENO-Z need at least 4 cells along each direction");
  return GP_OK;
}

int cell_widths(const gp_grid_desc* grid, double dx[3]) {
  for (int d = 0; d < 3; d++) {
    const int nn = d < grid->ndim ? grid->nint[d] : 1;
    dx[d] = (grid->dx[d] && d < grid->ndim) ? grid->dx[d][0]
                                            : (grid->xend[d] - grid->xbeg[d]) / nn;
    if (!(dx[d] > 0.0)) dx[d] = 1.0;
  }
  return GP_OK;
}
}  // namespace gp

extern "C" {

const char* gp_last_error(void) { return g_err; }

double gp_next_time_step(double invDt_hyp, double cfl, double cfl_max_var, double dt) {
  double dt_new = cfl / invDt_hyp;
  return (dt_new <= cfl_max_var * dt) ? dt_new : cfl_max_var * dt;
}

int gp_create(const gp_grid_desc* grid, const gp_scheme* scheme, void* stream,
              gp_handle** out) {
  if (!grid || !scheme || !out) return fail(GP_ERR_INVALID, "null argument");
  *out = nullptr;
  int rc = gp::validate_scheme(grid, scheme);
  if (rc) return rc;
  const bool wide = scheme->reconstruction == GP_REC_PARABOLIC ||
                    scheme->reconstruction == GP_REC_MP5 ||
                    scheme->reconstruction == GP_REC_WENOZ;
  rc = check_device();
  if (rc) return rc;
  gp_handle* h = new (std::nothrow) gp_handle;
  if (!h) return fail(GP_ERR_NOMEM, "host allocation");
  std::memset(h, 0, sizeof(*h));
  h->grid = *grid;
  h->scheme = *scheme;
  h->ndim = grid->ndim;
  h->nx = grid->nint[0];
  h->ny = grid->nint[1];
  h->nz = grid->ndim == 3 ? grid->nint[2] : 1;
  h->n = (long long)h->nx * h->ny * h->nz;
  for (int d = 0; d < grid->ndim; d++) {
    const int t[2] = {grid->lbound[d], grid->rbound[d]};
    for (int e = 0; e < 2; e++) {
      const unsigned bit = 1u << (2 * d + e);
      if (t[e] == GP_BC_OUTFLOW) h->outflow |= bit;
      // AXISYMMETRIC flips the same components as REFLECTIVE in Cartesian
      // geometry (FlipSign, Src/boundary.cpp:838-920)
      if (t[e] == GP_BC_REFLECTIVE || t[e] == GP_BC_AXISYMMETRIC) h->reflect |= bit;
      if (t[e] == GP_BC_EQTSYMMETRIC) h->eqtsym |= bit;
      if (t[e] == GP_BC_USERDEF) h->userdef |= bit;
    }
  }
  // Non-periodic directions are padded with stored ghost cells filled before
  // every stage: with constrained transport (the staggered field's ghost
  // faces), and for mirrored sides of every physics.  HD outflow alone keeps
  // the clamped ghost index of the sweeps.
  const unsigned nonper = h->outflow | h->reflect | h->eqtsym | h->userdef;
  h->padded = (h->reflect | h->eqtsym | h->userdef) != 0 ||
              (h->outflow != 0 && scheme->physics != GP_HD);
  {
    const int S = wide ? 3 : 2;
    const int nn[3] = {h->nx, h->ny, h->nz};
    int pp[3];
    for (int d = 0; d < 3; d++) {
      const bool pd = h->padded && d < grid->ndim && ((nonper >> (2 * d)) & 3u);
      h->lo[d] = pd ? S : 0;
      h->hi[d] = pd ? S + 1 : 0;
      pp[d] = nn[d] + h->lo[d] + h->hi[d];
    }
    h->px = pp[0];
    h->py = pp[1];
    h->pz = pp[2];
    h->pn = (long long)h->px * h->py * h->pz;
  }
  if (h->pn >= (1LL << 31)) {
    delete h;
    return fail(GP_ERR_UNSUPPORTED, "grids are limited to fewer than 2^31 cells");
  }
  h->nvar = scheme->physics == GP_HD ? 5 : 8;
  h->ng = grid->nghost;
  gp::cell_widths(grid, h->dx);
  // Cartesian face areas in the reference's operation order
  if (h->ndim == 2) {
    h->A[0] = 1.0 * h->dx[1];
    h->A[1] = h->dx[0] * 1.0;
    h->A[2] = 0.0;
  } else {
    h->A[0] = 1.0 * h->dx[1] * h->dx[2];
    h->A[1] = h->dx[0] * 1.0 * h->dx[2];
    h->A[2] = h->dx[0] * h->dx[1] * 1.0;
  }
  h->stream = (cudaStream_t)stream;
  h->mixed = scheme->precision == GP_MIXED;
  h->key = gp::SchemeKey{scheme->physics, grid->ndim, scheme->riemann, scheme->ct_emf,
                         scheme->reconstruction == GP_REC_PARABOLIC ? 4   /* LIM_PPM */
                         : scheme->reconstruction == GP_REC_MP5     ? 5   /* LIM_MP5 */
                         : scheme->reconstruction == GP_REC_WENOZ   ? 9   /* LIM_WENOZ */
                         : scheme->reconstruction == GP_REC_LIMO3   ? 10  /* LIM_LIMO3 */
                         : scheme->reconstruction == GP_REC_WENO3   ? 11  /* LIM_WENO3 */
                                                                    : scheme->limiter};
  // pencil segment for the marching sweeps: enough threads to fill 148 SMs,
  // then, among that length and its halves down to a quarter, the one whose
  // y and z sweeps take the fewest (waves of resident blocks) x (cells a
  // block marches, + 2 for its start-up): a last wave that fills few SMs
  // costs a whole wave.  At 256^3 the FP64 sweeps (4 blocks per SM) take
  // 32 (y/z 1.33 -> 1.29 ms against 64), the mixed ones (5 per SM) keep 64.
  {
    long long cols = (long long)h->px * (h->ndim == 3 ? h->pz : 1);
    int nd = h->py;
    int seg = 64;
    while (seg > 4 && cols * ((nd + seg - 1) / seg) < 148LL * 1024) seg /= 2;
    const long long resident =
        148LL * gp::sweep_m_blocks_per_sm(scheme->physics, h->mixed);
    // blocks of SWEEP_THREADS (128) columns, x and transverse taken together
    const long long cy = ((long long)h->px * (h->ndim == 3 ? h->pz : 1) + 127) / 128;
    const long long cz = ((long long)h->px * h->py + 127) / 128;
    auto cost = [&](int S) {
      long long c = 0;
      const long long by = cy * ((h->py + S - 1) / S);
      c += (by + resident - 1) / resident * (S + 2);
      if (h->ndim == 3) {
        const long long bz = cz * ((h->pz + S - 1) / S);
        c += (bz + resident - 1) / resident * (S + 2);
      }
      return c;
    };
    int best = seg;
    for (int S = seg / 2; S >= 4 && S >= seg / 4; S /= 2)
      if (cost(S) < cost(best)) best = S;
    h->seg = best;
  }
  const size_t cell = sizeof(double) * h->pn;
  const size_t ctb = (h->mixed ? sizeof(float) : sizeof(double)) * h->pn;
  bool ok = true;
  auto alloc = [&](void** p, size_t b) {
    if (ok && cudaMalloc(p, b) != cudaSuccess) ok = false;
  };
  alloc((void**)&h->U[0], cell * h->nvar);
  alloc((void**)&h->U[1], cell * h->nvar);
  alloc((void**)&h->V, cell * h->nvar);
  // flux differences, inverse-dt terms, UCT data and EMFs: float in the mixed form
  const size_t fcell = (h->mixed ? sizeof(float) : sizeof(double)) * h->pn;
  alloc((void**)&h->dU, fcell * h->nvar * 3);
  alloc((void**)&h->Cdt, fcell * 3);
  if (scheme->physics != GP_HD) {
    for (int b = 0; b < 3; b++)
      for (int d = 0; d < h->ndim; d++) alloc((void**)&h->Bs[b][d], cell);
    for (int d = 0; d < h->ndim; d++)
      for (int r = 0; r < 6; r++) alloc(&h->ct[d][r], ctb);
    for (int d = 0; d < 3; d++)
      if (h->ndim == 3 || d == 2) alloc((void**)&h->Ee[d], fcell);
  }
  alloc((void**)&h->sc, sizeof(StepScalars));
  if (ok && cudaMallocHost((void**)&h->sc_host, sizeof(StepScalars)) != cudaSuccess) ok = false;
  if (!ok) {
    cudaGetLastError();
    long long ncell = h->n;
    free_all(h);
    delete h;
    return fail(GP_ERR_NOMEM, "device allocation failed for %lld cells", ncell);
  }
  cudaMemsetAsync(h->sc, 0, sizeof(StepScalars), h->stream);
  cudaMemsetAsync(h->dU, 0, fcell * h->nvar * 3, h->stream);
  cudaMemsetAsync(h->Cdt, 0, fcell * 3, h->stream);
  h->bcur = 0;
  {
    int fills = 0;
    for (int side = 0; side < 2 * h->ndim; side++)
      if (!h->padded || !((nonper >> side) & 1u)) continue;
      else if ((h->userdef >> side) & 1u)  // the extra-cell copy (high side), the march
        fills += (side & 1) + (scheme->physics == GP_HD ? 0 : 1);
      else
        fills += scheme->physics == GP_HD ? 1 : 2;
    h->launches_per_step = scheme->rk_stages * (gp::stage_launch_count(h->key) + fills) + 1;
  }
  if (h->padded) {  // padding cells start finite
    cudaMemsetAsync(h->V, 0, cell * h->nvar, h->stream);
    cudaMemsetAsync(h->U[0], 0, cell * h->nvar, h->stream);
    cudaMemsetAsync(h->U[1], 0, cell * h->nvar, h->stream);
    for (int b = 0; b < 3 && scheme->physics != GP_HD; b++)
      for (int d = 0; d < h->ndim; d++) cudaMemsetAsync(h->Bs[b][d], 0, cell, h->stream);
  }
  *out = h;
  return GP_OK;
}

int gp_destroy(gp_handle* h) {
  if (!h) return GP_OK;
  cudaStreamSynchronize(h->stream);
  free_all(h);
  delete h;
  return GP_OK;
}

static int ensure_stage(gp_handle* h, size_t bytes) {
  if (h->stage_bytes >= bytes) return GP_OK;
  cudaFree(h->stage_buf);
  h->stage_buf = nullptr;
  h->stage_bytes = 0;
  CUDA_TRY(cudaMalloc((void**)&h->stage_buf, bytes));
  h->stage_bytes = bytes;
  return GP_OK;
}

// reference-layout extents of a cell array (s*) and its interior offset (o*)
static void ref_dims(const gp_handle* h, int stag, int* s, int* o) {
  int n[3] = {h->nx, h->ny, h->nz};
  for (int d = 0; d < 3; d++) {
    bool act = d < h->ndim;
    s[d] = n[d] + (act ? 2 * h->ng : 0) + (stag == d ? 1 : 0);
    o[d] = act ? h->ng : 0;
  }
}

// a padded grid's reference layout must have the scheme's ghost depth
static int check_ref_ghosts(gp_handle* h) {
  if (!h->padded) return GP_OK;
  const int S = h->lo[0] > h->lo[1] ? (h->lo[0] > h->lo[2] ? h->lo[0] : h->lo[2])
                                    : (h->lo[1] > h->lo[2] ? h->lo[1] : h->lo[2]);
  if (h->ng != S)
    return fail(GP_ERR_UNSUPPORTED, "reference layout with outflow needs nghost = %d", S);
  return GP_OK;
}

static int upload_one(gp_handle* h, int layout, const double* src, double* dst, int nvar,
                      int stag) {
  const size_t nb = sizeof(double) * h->n * nvar;
  if (layout == GP_LAYOUT_INTERIOR && !h->padded) {
    CUDA_TRY(cudaMemcpyAsync(dst, src, nb, cudaMemcpyHostToDevice, h->stream));
    return GP_OK;
  }
  int s[3], o[3];
  if (layout == GP_LAYOUT_INTERIOR) {
    s[0] = h->nx; s[1] = h->ny; s[2] = h->nz;
    o[0] = o[1] = o[2] = 0;
  } else {
    int rc = check_ref_ghosts(h);
    if (rc) return rc;
    ref_dims(h, stag, s, o);
  }
  size_t tot = sizeof(double) * (size_t)s[0] * s[1] * s[2] * nvar;
  int rc = ensure_stage(h, tot);
  if (rc) return rc;
  CUDA_TRY(cudaMemcpyAsync(h->stage_buf, src, tot, cudaMemcpyHostToDevice, h->stream));
  Pad p = pad_of(h);
  // a face field of a padded direction also has the high-side boundary face
  const bool extra = stag >= 0 && h->padded && h->lo[stag] > 0;
  if (extra && layout == GP_LAYOUT_REFERENCE) {
    if (stag == 0) p.nx += 1;
    if (stag == 1) p.ny += 1;
    if (stag == 2) p.nz += 1;
  }
  long long work = (long long)p.nx * p.ny * p.nz * nvar;
  gather_kernel<<<(unsigned)((work + 255) / 256), 256, 0, h->stream>>>(
      h->stage_buf, dst, nvar, s[0], s[1], s[2], o[0], o[1], o[2], p);
  CUDA_TRY(cudaGetLastError());
  if (extra && layout == GP_LAYOUT_INTERIOR) {
    const int P[3] = {h->px, h->py, h->pz};
    const int a = (stag == 0) ? 1 : 0, b = (stag == 2) ? 1 : 2;
    const long long nt = (long long)P[a] * P[b];
    wrap_face_kernel<<<(unsigned)((nt + 127) / 128), 128, 0, h->stream>>>(dst, pad_of(h), stag);
    CUDA_TRY(cudaGetLastError());
  }
  return GP_OK;
}

// `cons` marks the conserved array: its ghost zones are not part of a padded
// grid's state, so they are given the outflow copy of the domain.
static int download_one(gp_handle* h, int layout, const double* src, double* dst, int nvar,
                        int stag, bool cons = false) {
  const size_t nb = sizeof(double) * h->n * nvar;
  if (layout == GP_LAYOUT_INTERIOR && !h->padded) {
    CUDA_TRY(cudaMemcpyAsync(dst, src, nb, cudaMemcpyDeviceToHost, h->stream));
    return GP_OK;
  }
  int s[3], o[3];
  if (layout == GP_LAYOUT_INTERIOR) {
    s[0] = h->nx; s[1] = h->ny; s[2] = h->nz;
    o[0] = o[1] = o[2] = 0;
  } else {
    int rc = check_ref_ghosts(h);
    if (rc) return rc;
    ref_dims(h, stag, s, o);
  }
  long long tot = (long long)s[0] * s[1] * s[2] * nvar;
  int rc = ensure_stage(h, sizeof(double) * tot);
  if (rc) return rc;
  scatter_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, h->stream>>>(
      src, h->stage_buf, nvar, s[0], s[1], s[2], o[0], o[1], o[2], pad_of(h), h->outflow,
      cons ? 0 : 1);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaMemcpyAsync(dst, h->stage_buf, sizeof(double) * tot, cudaMemcpyDeviceToHost,
                           h->stream));
  return GP_OK;
}

int gp_upload_state(gp_handle* h, int layout, const double* Uc, const double* Vc,
                    const double* Vs0, const double* Vs1, const double* Vs2) {
  if (!h || !Vc) return fail(GP_ERR_INVALID, "null handle or Vc");
  if (layout != GP_LAYOUT_INTERIOR && layout != GP_LAYOUT_REFERENCE)
    return fail(GP_ERR_INVALID, "bad layout");
  int rc = upload_one(h, layout, Vc, h->V, h->nvar, -1);
  if (rc) return rc;
  if (Uc) {
    rc = upload_one(h, layout, Uc, h->U[0], h->nvar, -1);
  } else {
    rc = gp::launch_prim2cons(h->scheme.physics, h->V, h->U[0], h->pn, h->scheme.gamma,
                              h->stream);
    if (rc) return fail(GP_ERR_UNSUPPORTED, "prim2cons not built for this physics");
  }
  if (rc) return rc;
  if (h->scheme.physics != GP_HD) {
    const double* vs[3] = {Vs0, Vs1, Vs2};
    for (int d = 0; d < h->ndim; d++) {
      if (!vs[d]) return fail(GP_ERR_INVALID, "missing Vs%d", d);
      rc = upload_one(h, layout, vs[d], h->Bs[h->bcur][d], 1, d);
      if (rc) return rc;
    }
  }
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return GP_OK;
}

int gp_download_state(gp_handle* h, int layout, double* Uc, double* Vc, double* Vs0,
                      double* Vs1, double* Vs2) {
  if (!h) return fail(GP_ERR_INVALID, "null handle");
  int rc;
  // ghost zones of the current state, as Boundary() would fill them
  if (h->padded && layout == GP_LAYOUT_REFERENCE && (rc = fill_boundaries(h, h->Bs[h->bcur], 0)))
    return rc;
  if (Uc && (rc = download_one(h, layout, h->U[0], Uc, h->nvar, -1, true))) return rc;
  if (Vc && (rc = download_one(h, layout, h->V, Vc, h->nvar, -1))) return rc;
  if (h->scheme.physics != GP_HD) {
    double* vs[3] = {Vs0, Vs1, Vs2};
    for (int d = 0; d < h->ndim; d++)
      if (vs[d] && (rc = download_one(h, layout, h->Bs[h->bcur][d], vs[d], 1, d))) return rc;
  }
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return GP_OK;
}

int gp_advance_step(gp_handle* h, double dt, gp_step_out* out) {
  if (!h) return fail(GP_ERR_INVALID, "null handle");
  if (!(dt > 0.0)) return fail(GP_ERR_INVALID, "dt must be > 0");
  int rc = set_dt(h, dt);
  if (rc) return rc;
  rc = enqueue_step(h, nullptr, 0);
  if (rc) return rc;
  CUDA_TRY(cudaMemcpyAsync(h->sc_host, h->sc, sizeof(StepScalars), cudaMemcpyDeviceToHost,
                           h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (out) {
    out->err_bits = h->sc_host->err;
    out->invDt_hyp = h->sc_host->invdt;
    out->dt_next = h->sc_host->dt_next;
  }
  if (h->sc_host->err & (1u << 15)) return fail(GP_ERR_QUIT, "ERR_QUIT raised (bits 0x%x)", h->sc_host->err);
  return GP_OK;
}

int gp_advance_steps(gp_handle* h, int nsteps, double* dt, double* dt_hist, gp_step_out* out) {
  if (!h || !dt) return fail(GP_ERR_INVALID, "null argument");
  if (nsteps < 0) return fail(GP_ERR_INVALID, "nsteps < 0");
  if (!(*dt > 0.0)) return fail(GP_ERR_INVALID, "dt must be > 0");
  int rc = set_dt(h, *dt);
  if (rc) return rc;
  if (dt_hist && h->hist_cap < nsteps) {
    cudaFree(h->hist);
    h->hist = nullptr;
    h->hist_cap = 0;
    CUDA_TRY(cudaMalloc((void**)&h->hist, sizeof(double) * nsteps));
    h->hist_cap = nsteps;
  }
  for (int s = 0; s < nsteps; s++) {
    rc = enqueue_step(h, dt_hist ? h->hist : nullptr, s);
    if (rc) return rc;
  }
  CUDA_TRY(cudaMemcpyAsync(h->sc_host, h->sc, sizeof(StepScalars), cudaMemcpyDeviceToHost,
                           h->stream));
  if (dt_hist && nsteps > 0)
    CUDA_TRY(cudaMemcpyAsync(dt_hist, h->hist, sizeof(double) * nsteps, cudaMemcpyDeviceToHost,
                             h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  *dt = h->sc_host->dt;
  if (out) {
    out->err_bits = h->sc_host->err;
    out->invDt_hyp = h->sc_host->invdt;
    out->dt_next = h->sc_host->dt_next;
  }
  if (h->sc_host->err & (1u << 15)) return fail(GP_ERR_QUIT, "ERR_QUIT raised (bits 0x%x)", h->sc_host->err);
  return GP_OK;
}

int gp_device_state(gp_handle* h, double** Uc, double** Vc, double** Vs) {
  if (!h) return fail(GP_ERR_INVALID, "null handle");
  if (h->padded)
    return fail(GP_ERR_UNSUPPORTED, "the state of a grid with outflow sides is padded");
  if (Uc) *Uc = h->U[0];
  if (Vc) *Vc = h->V;
  if (Vs)
    for (int d = 0; d < 3; d++) Vs[d] = h->Bs[h->bcur][d];
  return GP_OK;
}

int gp_launches_per_step(const gp_handle* h) { return h ? h->launches_per_step : 0; }

int gp_set_userdef_boundary(gp_handle* h, gp_userdef_fn fn, void* user) {
  if (!h) return fail(GP_ERR_INVALID, "null handle");
  h->ud_fn = fn;
  h->ud_user = user;
  return GP_OK;
}

int gp_profile_steps(gp_handle* h, int nsteps, double* dt, float* kernel_ms, int cap,
                     int* nkernels) {
  if (!h || !dt || !kernel_ms || !nkernels) return fail(GP_ERR_INVALID, "null argument");
  const int nk = h->scheme.rk_stages * gp::stage_launch_count(h->key);
  *nkernels = nk;
  if (cap < nk) return fail(GP_ERR_INVALID, "kernel_ms needs %d entries", nk);
  for (int q = 0; q < nk; q++) kernel_ms[q] = 0.f;
  int rc = set_dt(h, *dt);
  if (rc) return rc;
  cudaEvent_t ev[64];
  for (int q = 0; q < 2 * nk; q++) CUDA_TRY(cudaEventCreate(&ev[q]));
  for (int s = 0; s < nsteps && rc == GP_OK; s++) {
    rc = enqueue_step(h, nullptr, 0, ev);
    if (rc) break;
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) { rc = fail(GP_ERR_CUDA, "%s", cudaGetErrorString(e)); break; }
    for (int q = 0; q < nk; q++) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev[2 * q], ev[2 * q + 1]);
      kernel_ms[q] += ms;
    }
  }
  for (int q = 0; q < 2 * nk; q++) cudaEventDestroy(ev[q]);
  if (rc) return rc;
  for (int q = 0; q < nk; q++) kernel_ms[q] /= (nsteps > 0 ? nsteps : 1);
  CUDA_TRY(cudaMemcpy(h->sc_host, h->sc, sizeof(StepScalars), cudaMemcpyDeviceToHost));
  *dt = h->sc_host->dt;
  return GP_OK;
}

const char* gp_kernel_name(const gp_handle* h, int idx) {
  if (!h) return "?";
  const int per = gp::stage_launch_count(h->key);
  return gp::stage_kernel_name(h->key, idx % per);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Output, restart and the min/max diagnostic in the reference's formats.
// ---------------------------------------------------------------------------
namespace {

constexpr int kDblOutput = 1;          // DBL_OUTPUT, Src/gpluto.hpp:139
constexpr int kMaxOutputTypes = 16;    // Src/gpluto.hpp:184
constexpr int kMaxRestartParams = 12;  // Src/gpluto.hpp:186

// One record of restart.out (Src/structs.hpp:382-390); the reference prints
// sizeof(Restart) = 256 on x86-64.
struct RestartRecord {
  double t;
  double dt;
  double param[kMaxRestartParams];
  int nstep;
  int nfile[kMaxOutputTypes];
  int nfileParticles[kMaxOutputTypes];
  char fill[10];
};
static_assert(sizeof(RestartRecord) == 256, "restart.out record layout");

bool little_endian() {
  const unsigned one = 1u;
  unsigned char b;
  std::memcpy(&b, &one, 1);
  return b == 1;
}

// output variable names in NVAR order (Src/set_var_names.cpp:20-42)
const char* var_name(int physics, int nv) {
  static const char* mhd[8] = {"rho", "vx1", "vx2", "vx3", "Bx1", "Bx2", "Bx3", "prs"};
  static const char* hd[5] = {"rho", "vx1", "vx2", "vx3", "prs"};
  return physics == GP_HD ? hd[nv] : mhd[nv];
}

// interior extents of output variable `stag` (-1: cell centred), with the
// one extra face along a staggered field's own direction
// (Src/bin_io.cpp:309-330)
void out_dims(const gp_handle* h, int stag, int* m) {
  const int n[3] = {h->nx, h->ny, h->nz};
  for (int d = 0; d < 3; d++) m[d] = n[d] + (stag == d ? 1 : 0);
}

void swap4(int* x) {
  unsigned char b[4];
  std::memcpy(b, x, 4);
  const unsigned char r[4] = {b[3], b[2], b[1], b[0]};
  std::memcpy(x, r, 4);
}

void swap8(double* x, size_t n) {
  for (size_t q = 0; q < n; q++) {
    unsigned char b[8];
    std::memcpy(b, x + q, 8);
    for (int e = 0; e < 4; e++) {
      unsigned char t = b[e];
      b[e] = b[7 - e];
      b[7 - e] = t;
    }
    std::memcpy(x + q, b, 8);
  }
}

// DataMinMax (Src/main.cpp:752-900) over the domain cells of V: per variable
// minimum and maximum, and the largest max(|v_x|,|v_y|,|v_z|)/sqrt(p/rho),
// with the reference's MAX/MIN (Src/macros.hpp:191-194).  Grid-stride
// partials per block, then one block over the partials.
constexpr int kMinMaxThreads = 256;
constexpr int kMinMaxBlocks = 592;  // 148 SMs x 4

__device__ __forceinline__ double ref_max(double a, double b) { return a >= b ? a : b; }
__device__ __forceinline__ double ref_min(double a, double b) { return a <= b ? a : b; }

__global__ void __launch_bounds__(kMinMaxThreads) minmax_partial_kernel(
    const double* __restrict__ V, int nvar, int prs, Pad p, double* __restrict__ part) {
  __shared__ double red[kMinMaxThreads];
  double mn[8], mx[8], mach = 0.0;
  for (int nv = 0; nv < 8; nv++) {
    mx[nv] = -1e18;
    mn[nv] = 1e18;
  }
  const long long ncell = (long long)p.nx * p.ny * p.nz;
  const long long pn = (long long)p.px * p.py * p.pz;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < ncell;
       c += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(c % p.nx), j = (int)((c / p.nx) % p.ny);
    const int k = (int)(c / ((long long)p.nx * p.ny));
    const long long q = (i + p.lx) + (long long)p.px * ((j + p.ly) + (long long)p.py * (k + p.lz));
    double v[8];
    for (int nv = 0; nv < nvar; nv++) v[nv] = V[nv * pn + q];
    double cs = v[prs] / v[0];
    cs = sqrt(cs);
    const double mi = fabs(v[1]) / cs, mj = fabs(v[2]) / cs, mk = fabs(v[3]) / cs;
    double lm = ref_max(mi, mj);
    lm = ref_max(lm, mk);
    mach = ref_max(mach, lm);
    for (int nv = 0; nv < nvar; nv++) {
      mx[nv] = ref_max(mx[nv], v[nv]);
      mn[nv] = ref_min(mn[nv], v[nv]);
    }
  }
  const int nq = 2 * nvar + 1;
  for (int qv = 0; qv < nq; qv++) {
    const bool is_min = qv >= nvar && qv < 2 * nvar;
    red[threadIdx.x] = qv < nvar ? mx[qv] : (is_min ? mn[qv - nvar] : mach);
    __syncthreads();
    for (int s = kMinMaxThreads / 2; s > 0; s >>= 1) {
      if ((int)threadIdx.x < s)
        red[threadIdx.x] = is_min ? ref_min(red[threadIdx.x], red[threadIdx.x + s])
                                  : ref_max(red[threadIdx.x], red[threadIdx.x + s]);
      __syncthreads();
    }
    if (threadIdx.x == 0) part[(long long)blockIdx.x * nq + qv] = red[0];
    __syncthreads();
  }
}

__global__ void minmax_final_kernel(const double* __restrict__ part, int nparts, int nvar,
                                    double* __restrict__ out) {
  const int nq = 2 * nvar + 1;
  const int qv = threadIdx.x;
  if (qv >= nq) return;
  const bool is_min = qv >= nvar && qv < 2 * nvar;
  double r = part[qv];
  for (int b = 1; b < nparts; b++)
    r = is_min ? ref_min(r, part[(long long)b * nq + qv]) : ref_max(r, part[(long long)b * nq + qv]);
  out[qv] = r;
}

}  // namespace

extern "C" {

int gp_data_minmax(gp_handle* h, double* vmin, double* vmax, double* mach_max) {
  if (!h || !vmin || !vmax) return fail(GP_ERR_INVALID, "null handle or output");
  const int nq = 2 * h->nvar + 1;
  double* part = nullptr;
  CUDA_TRY(cudaMallocAsync((void**)&part, sizeof(double) * (kMinMaxBlocks + 1) * nq, h->stream));
  const int prs = h->nvar - 1;  // PRS is the last variable (HD 4, MHD/RMHD 7)
  minmax_partial_kernel<<<kMinMaxBlocks, kMinMaxThreads, 0, h->stream>>>(h->V, h->nvar, prs,
                                                                         pad_of(h), part);
  minmax_final_kernel<<<1, 32, 0, h->stream>>>(part, kMinMaxBlocks, h->nvar,
                                               part + (size_t)kMinMaxBlocks * nq);
  double res[17];
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(res, part + (size_t)kMinMaxBlocks * nq, sizeof(double) * nq,
                        cudaMemcpyDeviceToHost, h->stream);
  cudaFreeAsync(part, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return fail(GP_ERR_CUDA, "gp_data_minmax: %s", cudaGetErrorString(e));
  for (int nv = 0; nv < h->nvar; nv++) {
    vmax[nv] = res[nv];
    vmin[nv] = res[h->nvar + nv];
  }
  if (mach_max) *mach_max = res[2 * h->nvar];
  return GP_OK;
}

int gp_write_dbl(gp_handle* h, const char* dir, int nfile, double t, double dt, int nstep) {
  if (!h || !dir || nfile < 0) return fail(GP_ERR_INVALID, "null handle/dir or nfile < 0");
  const bool mhd = h->scheme.physics != GP_HD;
  // current state in the reference layout (ghost zones as Boundary() fills them)
  int s[3], o[3];
  ref_dims(h, -1, s, o);
  std::vector<double> V((size_t)s[0] * s[1] * s[2] * h->nvar);
  std::vector<double> B[3];
  for (int d = 0; mhd && d < h->ndim; d++) {
    int fs[3], fo[3];
    ref_dims(h, d, fs, fo);
    B[d].resize((size_t)fs[0] * fs[1] * fs[2]);
  }
  int rc = gp_download_state(h, GP_LAYOUT_REFERENCE, nullptr, V.data(),
                             B[0].empty() ? nullptr : B[0].data(),
                             B[1].empty() ? nullptr : B[1].data(),
                             B[2].empty() ? nullptr : B[2].data());
  if (rc) return rc;
  // data.NNNN.dbl, single_file mode: the interior of every output variable
  // in turn (Src/write_data.cpp:131-160, FillOutputBuffer 563-601)
  char fname[1024];
  snprintf(fname, sizeof(fname), "%s/data.%04d.dbl", dir, nfile);
  FILE* f = fopen(fname, "wb");
  if (!f) return fail(GP_ERR_IO, "cannot write %s", fname);
  std::vector<double> buf;
  auto dump = [&](const double* src, const int* sext, int stag) -> bool {
    int m[3];
    out_dims(h, stag, m);
    buf.resize((size_t)m[0] * m[1] * m[2]);
    size_t q = 0;
    for (int k = 0; k < m[2]; k++)
      for (int j = 0; j < m[1]; j++)
        for (int i = 0; i < m[0]; i++)
          buf[q++] = src[(i + o[0]) + (size_t)sext[0] * ((j + o[1]) + (size_t)sext[1] * (k + o[2]))];
    return fwrite(buf.data(), sizeof(double), buf.size(), f) == buf.size();
  };
  bool ok = true;
  const size_t ncell = (size_t)s[0] * s[1] * s[2];
  for (int nv = 0; ok && nv < h->nvar; nv++) ok = dump(V.data() + nv * ncell, s, -1);
  for (int d = 0; ok && mhd && d < h->ndim; d++) {
    int fs[3], fo[3];
    ref_dims(h, d, fs, fo);
    ok = dump(B[d].data(), fs, d);
  }
  if (fclose(f) != 0 || !ok) return fail(GP_ERR_IO, "short write to %s", fname);
  // dbl.out: line nfile, written over whatever follows line nfile-1
  // (Src/write_data.cpp:474-503)
  snprintf(fname, sizeof(fname), "%s/dbl.out", dir);
  FILE* fo_ = fopen(fname, nfile == 0 ? "w" : "r+");
  if (!fo_) return fail(GP_ERR_IO, "cannot open %s", fname);
  char sline[512];
  for (int q = 0; q < nfile; q++)
    if (!fgets(sline, sizeof(sline), fo_)) {
      fclose(fo_);
      return fail(GP_ERR_IO, "%s has fewer than %d lines", fname, nfile);
    }
  fseek(fo_, ftell(fo_), SEEK_SET);
  fprintf(fo_, "%d %12.6e %12.6e %d ", nfile, t, dt, nstep);
  fprintf(fo_, "single_file ");
  fprintf(fo_, little_endian() ? "little " : "big ");
  for (int nv = 0; nv < h->nvar; nv++) fprintf(fo_, "%s ", var_name(h->scheme.physics, nv));
  for (int d = 0; mhd && d < h->ndim; d++) fprintf(fo_, "Bx%ds ", d + 1);
  fprintf(fo_, "\n");
  if (fclose(fo_) != 0) return fail(GP_ERR_IO, "cannot write %s", fname);
  // restart.out: record nfile (RestartDump, Src/restart.cpp:423-458)
  RestartRecord r;
  std::memset(&r, 0, sizeof(r));
  r.t = t;
  r.dt = dt;
  r.nstep = nstep;
  for (int q = 0; q < kMaxOutputTypes; q++) r.nfile[q] = r.nfileParticles[q] = -1;
  r.nfile[kDblOutput] = nfile;
  snprintf(fname, sizeof(fname), "%s/restart.out", dir);
  FILE* fr = fopen(fname, nfile == 0 ? "wb" : "r+b");
  if (!fr && nfile > 0) fr = fopen(fname, "wb");
  if (!fr) return fail(GP_ERR_IO, "cannot open %s", fname);
  fseek(fr, (long)nfile * (long)sizeof(RestartRecord), SEEK_SET);
  ok = fwrite(&r, sizeof(r), 1, fr) == 1;
  if (fclose(fr) != 0 || !ok) return fail(GP_ERR_IO, "cannot write %s", fname);
  return GP_OK;
}

int gp_read_dbl(gp_handle* h, const char* dir, int nrestart, double* t, double* dt,
                int* nstep) {
  if (!h || !dir || nrestart < 0) return fail(GP_ERR_INVALID, "null handle/dir or nrestart < 0");
  const bool mhd = h->scheme.physics != GP_HD;
  // 1. dbl.out line nrestart: mode and byte order (Src/restart.cpp:67-104)
  char fname[1024], sline[1024], mode[64] = "", endian[64] = "";
  snprintf(fname, sizeof(fname), "%s/dbl.out", dir);
  FILE* f = fopen(fname, "r");
  if (!f) return fail(GP_ERR_IO, "cannot find %s", fname);
  int line = 0, found = 0;
  while (fgets(sline, sizeof(sline), f)) {
    if (line++ == nrestart) {
      int a, c;
      double x, y;
      found = sscanf(sline, "%d %lf %lf %d %63s %63s", &a, &x, &y, &c, mode, endian) == 6;
      break;
    }
  }
  fclose(f);
  if (!found) return fail(GP_ERR_IO, "output #%d does not exist in %s", nrestart, fname);
  if (std::strcmp(mode, "single_file") != 0)
    return fail(GP_ERR_UNSUPPORTED, "only single_file dbl output is read (found %s)", mode);
  const bool swap = (std::strcmp(endian, "big") == 0) == little_endian();
  // 2. restart.out: the record whose DBL file number is nrestart
  //    (RestartGet, Src/restart.cpp:331-411)
  snprintf(fname, sizeof(fname), "%s/restart.out", dir);
  f = fopen(fname, "rb");
  if (!f) return fail(GP_ERR_IO, "cannot find %s", fname);
  RestartRecord r;
  found = 0;
  while (fread(&r, sizeof(r), 1, f) == 1) {
    int nf = r.nfile[kDblOutput];
    if (swap) swap4(&nf);
    if (nf == nrestart) {
      found = 1;
      break;
    }
  }
  fclose(f);
  if (!found) return fail(GP_ERR_IO, "no record of output #%d in %s", nrestart, fname);
  if (swap) {
    swap8(&r.t, 1);
    swap8(&r.dt, 1);
    swap4(&r.nstep);
  }
  // 3. data.NNNN.dbl into the reference layout; ghost zones take the
  //    nearest interior value (they are refilled before every stage)
  snprintf(fname, sizeof(fname), "%s/data.%04d.dbl", dir, nrestart);
  f = fopen(fname, "rb");
  if (!f) return fail(GP_ERR_IO, "cannot find %s", fname);
  int s[3], o[3];
  ref_dims(h, -1, s, o);
  const size_t ncell = (size_t)s[0] * s[1] * s[2];
  std::vector<double> V(ncell * h->nvar), B[3];
  std::vector<double> buf;
  bool ok = true;
  auto load = [&](double* dst, const int* sext, int stag) -> bool {
    int m[3];
    out_dims(h, stag, m);
    buf.resize((size_t)m[0] * m[1] * m[2]);
    if (fread(buf.data(), sizeof(double), buf.size(), f) != buf.size()) return false;
    if (swap) swap8(buf.data(), buf.size());
    for (int k = 0; k < sext[2]; k++)
      for (int j = 0; j < sext[1]; j++)
        for (int i = 0; i < sext[0]; i++) {
          const int ii = i - o[0] < 0 ? 0 : (i - o[0] >= m[0] ? m[0] - 1 : i - o[0]);
          const int jj = j - o[1] < 0 ? 0 : (j - o[1] >= m[1] ? m[1] - 1 : j - o[1]);
          const int kk = k - o[2] < 0 ? 0 : (k - o[2] >= m[2] ? m[2] - 1 : k - o[2]);
          dst[i + (size_t)sext[0] * (j + (size_t)sext[1] * k)] =
              buf[ii + (size_t)m[0] * (jj + (size_t)m[1] * kk)];
        }
    return true;
  };
  for (int nv = 0; ok && nv < h->nvar; nv++) ok = load(V.data() + nv * ncell, s, -1);
  for (int d = 0; ok && mhd && d < h->ndim; d++) {
    int fs[3], fo[3];
    ref_dims(h, d, fs, fo);
    B[d].resize((size_t)fs[0] * fs[1] * fs[2]);
    ok = load(B[d].data(), fs, d);
  }
  fclose(f);
  if (!ok) return fail(GP_ERR_IO, "%s is shorter than this grid's output", fname);
  // 4. upload; Uc = PrimToCons(Vc) on the device (Src/restart.cpp:276-283)
  int rc = gp_upload_state(h, GP_LAYOUT_REFERENCE, nullptr, V.data(),
                           B[0].empty() ? nullptr : B[0].data(),
                           B[1].empty() ? nullptr : B[1].data(),
                           B[2].empty() ? nullptr : B[2].data());
  if (rc) return rc;
  if (t) *t = r.t;
  if (dt) *dt = r.dt;
  if (nstep) *nstep = r.nstep;
  return GP_OK;
}

}  // extern "C"
