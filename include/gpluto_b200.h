/*
 * gpluto_b200.h -- C ABI of the B200 (sm_100a) Godunov step.
 *
 * Drop-in boundary for gPLUTO's time-step path.  The reference calls
 *     uint32_t AdvanceStep(Data*, Grid*, timeStep*)        (Src/prototypes.hpp:5)
 * from its main loop (Src/main.cpp:444-447), then turns the stage-1 inverse
 * time step into the next dt with
 *     double NextTimeStep(timeStep*, RunConfig*, Runtime*, Grid*)
 *                                                          (Src/prototypes.hpp:155,
 *                                                           Src/next_time_step.cpp:20-130).
 * Below AdvanceStep sit Boundary (Src/boundary.cpp:67), UpdateStage
 * (Src/update_stage.cpp:57), the Riemann-solver plug-in selected by name in
 * SetSolver (Src/MHD/set_solver.cpp:13-54, typedef Src/gpluto.hpp:762),
 * CT_ComputeEMF / CT_Update / CT_AverageStaggeredFields
 * (Src/MHD/CT/ct.hpp:118-142) and ConsToPrim3D (Src/mappers3D.cpp:76).
 * This library replaces all of them with fused CUDA kernels; the host driver,
 * pluto.ini / definitions.hpp configuration and Data/Grid arrays stay on the
 * caller's side and cross this boundary as plain pointers and sizes.
 *
 * Arrays in GP_LAYOUT_REFERENCE follow Data::Vc/Uc (Ary4D, i fastest, variable
 * index slowest, ghost zones included, Src/Array.hpp:471-494) and Data::Vs[d]
 * (Ary3D with one extra point along d, Src/initialize.cpp:424-430).  Arrays in
 * GP_LAYOUT_INTERIOR hold interior cells only ([nv][k][j][i]) and the left
 * face of each cell for Vs.
 *
 * All functions return GP_OK (0) or a negative gp_status.  They are not
 * thread-safe on a single handle; use one handle per host thread.
 */
#ifndef GPLUTO_B200_H
#define GPLUTO_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gp_handle gp_handle;

enum gp_status {
  GP_OK = 0,
  GP_ERR_INVALID = -1,      /* bad argument */
  GP_ERR_UNSUPPORTED = -2,  /* scheme/grid combination not built */
  GP_ERR_CUDA = -3,         /* CUDA runtime error (see gp_last_error) */
  GP_ERR_NOMEM = -4,        /* device allocation failed */
  GP_ERR_QUIT = -5,         /* a kernel raised ERR_QUIT (the reference would QuitPLUTO) */
  GP_ERR_NO_DEVICE = -6,    /* no CUDA device: this library has no CPU path */
  GP_ERR_IO = -7,           /* an output or restart file is missing, short or unwritable */
  GP_ERR_TIMEOUT = -8       /* a batched stage's bounded dependency wait ran out */
};

/* PHYSICS (definitions.hpp) */
enum { GP_HD = 0, GP_MHD = 1, GP_RMHD = 2 };
/* LIMITER (Src/gpluto.hpp:329-335, Src/plm_coeffs.hpp:55-110); 4 and 5 are
   not limiters (they stand for PPM and MP5 inside the library) */
enum { GP_LIM_FLAT = 0, GP_LIM_MINMOD = 1, GP_LIM_VANLEER = 2, GP_LIM_MC = 3,
       GP_LIM_VANALBADA = 6, GP_LIM_OSPRE = 7, GP_LIM_UMIST = 8 };
/* [Solver] in pluto.ini (Src/MHD/set_solver.cpp:35-47); hll, hllc and tvdlf
   for MHD take UCT_HLL, ARITHMETIC or CT_CONTACT (UCT_HLLD needs hlld);
   hllc is HD and MHD only */
enum { GP_RS_HLL = 0, GP_RS_HLLC = 1, GP_RS_HLLD = 2, GP_RS_TVDLF = 3 };
/* CT_EMF_AVERAGE (Src/MHD/CT/ct.hpp:19-27): upwind UCT_HLL / UCT_HLLD, the
   ARITHMETIC average of the face EMFs, or CT_CONTACT (that average with the
   contact-upwinded corner terms, Src/MHD/CT/ct_emf.cpp:220-245); the last
   two for MHD */
enum { GP_CT_UCT_HLL = 0, GP_CT_UCT_HLLD = 1, GP_CT_ARITHMETIC = 2, GP_CT_CONTACT = 3 };
/* [Boundary] types (Src/boundary.cpp:144-310; the reference's values,
   Src/gpluto.hpp:205-212, except periodic): outflow (zero-gradient ghost
   copy, OutflowBoundary Src/boundary.cpp:677-780), reflective,
   axisymmetric and eqtsymmetric (ReflectiveBoundary with the signs of
   FlipSign, 838-1060), userdef (the caller's fill, see
   gp_set_userdef_boundary) */
enum { GP_BC_PERIODIC = 0, GP_BC_OUTFLOW = 1, GP_BC_REFLECTIVE = 2, GP_BC_AXISYMMETRIC = 3,
       GP_BC_EQTSYMMETRIC = 4, GP_BC_USERDEF = 8 };
/* RECONSTRUCTION (definitions.hpp): LINEAR (PLM with LIMITER), PARABOLIC
   (PPM, Src/States/ppm_states.cpp), MP5, WENOZ, LimO3 or WENO3
   (Src/States/mp5_states.cpp) */
enum { GP_REC_LINEAR = 0, GP_REC_PARABOLIC = 1, GP_REC_MP5 = 2, GP_REC_WENOZ = 3,
       GP_REC_LIMO3 = 4, GP_REC_WENO3 = 5 };
/* arithmetic form */
enum { GP_FP64 = 0, GP_MIXED = 1 };
/* host array layouts */
enum { GP_LAYOUT_INTERIOR = 0, GP_LAYOUT_REFERENCE = 1 };

/* Mirrors the parts of Grid (Src/structs.hpp:177-257) the step needs. */
typedef struct gp_grid_desc {
  int ndim;               /* DIMENSIONS: 2 or 3 */
  int nint[3];            /* Grid::nint (1 along inactive directions) */
  int nghost;             /* Grid::nghost, used only by GP_LAYOUT_REFERENCE */
  double xbeg[3], xend[3];
  const double *dx[3];    /* optional Grid::dx, ntot entries; must be uniform */
  int lbound[3], rbound[3];
} gp_grid_desc;

/* Mirrors the compile-time scheme (definitions.hpp) and RunConfig/Runtime
   values (Src/structs.hpp:397-447). */
typedef struct gp_scheme {
  int physics;            /* GP_HD, GP_MHD, GP_RMHD */
  int limiter;            /* GP_LIM_* */
  int riemann;            /* GP_RS_* */
  int ct_emf;             /* GP_CT_* (MHD/RMHD) */
  int rk_stages;          /* TIME_STEPPING: 2 (RK2) */
  int precision;          /* GP_FP64 or GP_MIXED */
  double gamma;           /* RunConfig::gamma */
  double cfl;             /* Runtime::cfl */
  double cfl_max_var;     /* Runtime::cfl_max_var */
  double small_rho;       /* RunConfig::small_rho (1e-12 default) */
  double small_prs;       /* RunConfig::small_prs (1e-12 default) */
  int reconstruction;     /* GP_REC_LINEAR (limiter applies) or another GP_REC_* */
} gp_scheme;

/* Per-step result: what the host needs for NextTimeStep and error handling. */
typedef struct gp_step_out {
  uint32_t err_bits;      /* OR of the ERR_* bits of Src/gpluto.hpp:247-265 */
  double invDt_hyp;       /* timeStep::invDt_hyp of stage 1 */
  double dt_next;         /* NextTimeStep() of this step */
} gp_step_out;

/* Allocate the device state for one grid.  `stream` is a cudaStream_t (NULL:
   the legacy default stream).  Replaces Initialize's allocations
   (Src/initialize.cpp:396-443) and SetSolver (Src/MHD/set_solver.cpp:13). */
int gp_create(const gp_grid_desc *grid, const gp_scheme *scheme, void *stream,
              gp_handle **out);
int gp_destroy(gp_handle *h);

/* Host -> device state.  Uc may be NULL: it is then computed from Vc with the
   start-up PrimToCons map (Src/startup.cpp:542-566).  Vs1/Vs2 are NULL for HD
   and along inactive directions. */
int gp_upload_state(gp_handle *h, int layout, const double *Uc, const double *Vc,
                    const double *Vs0, const double *Vs1, const double *Vs2);
/* Device -> host state (any pointer may be NULL). */
int gp_download_state(gp_handle *h, int layout, double *Uc, double *Vc,
                      double *Vs0, double *Vs1, double *Vs2);

/* One RK step of size dt (AdvanceStep, Src/rk_step.cpp:88-593).  Blocks until
   the step finishes; fills `out` (may be NULL).  Returns GP_ERR_QUIT when a
   kernel raised ERR_QUIT. */
int gp_advance_step(gp_handle *h, double dt, gp_step_out *out);

/* `nsteps` RK steps with the dt sequence kept on the device (each next dt by
   NextTimeStep from the stage-1 reduction), no host round trip between
   steps.  On entry *dt is the first step's dt; on return the dt of the step
   after the last.  dt_hist (nsteps entries, may be NULL) receives the dt of
   every step taken.  out->err_bits is the OR over all steps. */
int gp_advance_steps(gp_handle *h, int nsteps, double *dt, double *dt_hist, gp_step_out *out);

/* NextTimeStep (Src/next_time_step.cpp:80,125) for the host driver. */
double gp_next_time_step(double invDt_hyp, double cfl, double cfl_max_var, double dt);

/* Device pointers of the current state (interior layout), for callers that
   keep data on the GPU.  Valid until the next step. */
int gp_device_state(gp_handle *h, double **Uc, double **Vc, double **Vs);

/* ---- user-defined boundaries -------------------------------------------
   A USERDEF side is filled by the caller, as UserDefBoundary(data, box, side,
   grid) fills it in the reference (Src/boundary.cpp:238-256): before every
   RK stage, in the reference's side order among the other sides, the
   library calls `fn` on the host with the side's ghost box; `fn` enqueues on
   `stream` (a cudaStream_t) the device work that sets, in that box, every
   primitive variable of V and, with a staggered field, the tangential face
   fields Vs[e] (e != the side's direction; their box is one face wider
   along e, which here means the whole array extent).  The library then
   sets the normal face field of the ghost zone from div B = 0
   (CT_FillStaggeredFields, Src/MHD/CT/ct_fill_mag_field.cpp:39) and the
   ghost cells' B from their faces (Src/boundary.cpp:285-307), as for an
   outflow side.  Arrays are the library's padded layout: a direction with
   a non-periodic side stores dom_beg[d] ghost cells below the domain and
   dom_beg[d] + 1 above it (the last one has no counterpart in the
   reference: the library fills it); periodic directions store no ghosts.
   `fn` returns 0, or a nonzero value that makes the step return
   GP_ERR_INVALID.  It is called while the step is being enqueued: work it
   enqueues on `stream` runs in order with the step's kernels. */
typedef struct gp_userdef_side {
  int side;            /* 0..5: X1_BEG, X1_END, X2_BEG, X2_END, X3_BEG, X3_END */
  int stage;           /* the RK stage the boundary is set for: 1, 2 (3 with RK3); 0
                          when gp_download_state fills the reference layout's ghosts */
  int beg[3], end[3];  /* the ghost box (inclusive array indices, i j k) */
  int dom_beg[3];      /* array index of the first domain cell per direction */
  int nint[3];         /* domain cells per direction */
  int dims[3];         /* array extents: cell (i,j,k) is i + dims[0]*(j + dims[1]*k) */
  int nvar;            /* variables of V */
  double *V;           /* device: primitives, [nvar][dims[0]*dims[1]*dims[2]] */
  double *Vs[3];       /* device: left-face fields (NULL for HD and inactive directions) */
} gp_userdef_side;
typedef int (*gp_userdef_fn)(void *user, const gp_userdef_side *side, void *stream);
/* Registers the fill of the handle's USERDEF sides (fn NULL: none; a step
   with USERDEF sides and no fill returns GP_ERR_INVALID). */
int gp_set_userdef_boundary(gp_handle *h, gp_userdef_fn fn, void *user);

/* Kernel launches issued per RK step (for launch accounting). */
int gp_launches_per_step(const gp_handle *h);

/* Instrumented variant of gp_advance_steps for profiling: every kernel of a
   step is bracketed by CUDA events on the handle's stream; kernel_ms[q]
   (cap >= 2*kernels per stage) receives the mean duration of launch q of a
   step, in launch order; *nkernels the number of launches per step (the
   dt update kernel excluded).  Not part of the reference interface. */
int gp_profile_steps(gp_handle *h, int nsteps, double *dt, float *kernel_ms, int cap,
                     int *nkernels);
/* Name of launch q of a step (as ordered by gp_profile_steps). */
const char *gp_kernel_name(const gp_handle *h, int q);

/* ---- output and restart in the reference's .dbl format ------------------
   Replace WriteData for DBL_OUTPUT in single_file mode
   (Src/write_data.cpp:35-160, 474-503), RestartDump
   (Src/restart.cpp:423-458) and RestartFromFile/RestartGet
   (Src/restart.cpp:34-283, 331-411), so that a run on the device and a run
   of the reference can restart from each other's files.

   gp_write_dbl: writes <dir>/data.<nfile %04d>.dbl (the interior of rho,
   vx1..vx3, [Bx1..Bx3,] prs, then the staggered Bx1s..Bx<ndim>s with one
   extra face along their own direction, doubles, x fastest), line nfile of
   <dir>/dbl.out ("nfile t dt nstep single_file little|big names...") and
   record nfile of <dir>/restart.out (256-byte Restart records).  t, dt and
   nstep are the caller's time, the dt of the next step and the step count.

   gp_read_dbl: loads output #nrestart written by either program: Vc and the
   staggered fields from the data file (byte order from dbl.out), Uc =
   PrimToCons(Vc) on the device, and returns the record's t, dt (the next
   step's dt) and nstep.  Errors: GP_ERR_IO for a missing or short file,
   GP_ERR_UNSUPPORTED for multiple_files output. */
int gp_write_dbl(gp_handle *h, const char *dir, int nfile, double t, double dt, int nstep);
int gp_read_dbl(gp_handle *h, const char *dir, int nrestart, double *t, double *dt,
                int *nstep);

/* DataMinMax (Src/main.cpp:752-900) on the device: per variable minimum and
   maximum of the primitive state over the domain cells (vmin, vmax: nvar
   values each, in NVAR order) and the largest Mach number
   max(|vx1|,|vx2|,|vx3|)/sqrt(prs/rho) (mach_max may be NULL). */
int gp_data_minmax(gp_handle *h, double *vmin, double *vmax, double *mach_max);

/* Limits of gp_advance_step_noalloc: the largest grid it accepts (cells) and
   the doubles of device scratch it keeps per cell. */
#define GP_NOALLOC_MAX_CELLS 16384
#define GP_NOALLOC_DOUBLES_PER_CELL 62

/* One RK2 step (the same kernels and results as gp_advance_step) that
   allocates nothing.  No counterpart in the reference: it exists for callers
   that cannot call cudaMalloc -- hosts whose device memory belongs to
   another allocator, loops that must not allocate or grow their device
   footprint.  It synchronizes `stream` before returning (the step scalars
   are read back).  Uc/Vc/Vs0..2 are DEVICE pointers the caller owns,
   interior layout, updated in place (Vs1/Vs2 NULL where unused).  Every
   intermediate lives in one static device array of
   GP_NOALLOC_MAX_CELLS * GP_NOALLOC_DOUBLES_PER_CELL doubles (~8 MB) that
   each GPU loading the library holds until exit; grids of more than
   GP_NOALLOC_MAX_CELLS cells return GP_ERR_INVALID.  The first call on a
   device looks up that array's device address (cudaGetSymbolAddress), so
   make it before any stream capture.  All calls share the array: calls
   that overlap on the GPU race.  It accepts what gp_create accepts (same
   checks, same cell widths: Grid::dx when given) restricted to RK2,
   LINEAR or PARABOLIC reconstruction and periodic sides on every
   direction; anything else returns GP_ERR_UNSUPPORTED.  Returns a
   gp_status with the reason in gp_last_error(); `out` as for
   gp_advance_step. */
int gp_advance_step_noalloc(const gp_grid_desc *grid, const gp_scheme *scheme,
                            double *Uc, double *Vc, double *Vs0, double *Vs1, double *Vs2,
                            double dt, void *stream, gp_step_out *out);

/* ---------------------------------------------------------------------
   Batched step: many independent grids ("slots") in one device pool,
   advanced together: per RK stage one persistent sweep launch and one
   persistent EMF/finish launch over all slots, the launches of a run of
   steps captured once as a CUDA graph.  Each slot keeps
   its own dt sequence (NextTimeStep on the device, exactly as
   gp_advance_steps) and its own step budget; a slot whose budget is spent,
   or that raised ERR_QUIT, stops advancing.  Built schemes: ideal MHD with
   PLM-MC + HLLD + UCT_HLLD, relativistic MHD with PLM-MC + HLLD + UCT_HLL
   (its Riemann solver in FP64 in both forms) and HD with PLM-MC + HLLC,
   2-D and 3-D, FP64 or mixed per slot, RK2, periodic boundaries.  The reference advances one grid per
   process; this has no reference counterpart beyond the step it repeats.
   --------------------------------------------------------------------- */
typedef struct gp_batch gp_batch;

/* Tile shape of one slot (0 = default): `seg` is the pencil segment of the
   y/z sweeps (cells one thread marches), `cells_per_thread` the cells each
   thread of an edge-EMF or finish tile handles. */
typedef struct gp_tile_shape {
  int seg;
  int cells_per_thread;
} gp_tile_shape;

typedef struct gp_slot_status {
  int steps_done;         /* steps completed since admission */
  int steps_left;         /* budget left (0: finished or stopped) */
  uint32_t err_bits;      /* OR of the ERR_* bits since admission */
  double dt;              /* dt of the next step */
  double invDt_hyp;       /* invDt_hyp of the last completed step */
} gp_slot_status;

/* Reserve a device pool of `pool_bytes` holding up to `max_slots` grids.
   `ctas` = blocks of the sweep launch (0: all that fit on the device; the
   EMF/finish launch always uses all that fit).
   `stream` as for gp_create (NULL: the batch creates its own). */
int gp_batch_create(size_t pool_bytes, int max_slots, int ctas, void *stream, gp_batch **out);
int gp_batch_destroy(gp_batch *b);
/* Device bytes a slot of this grid and scheme takes from the pool. */
size_t gp_batch_slot_bytes(const gp_grid_desc *grid, const gp_scheme *scheme);
/* Admit a grid: primitives Vc and face fields Vs0..2 (host, interior layout;
   Vs* NULL for HD) become the slot's state (U from the start-up PrimToCons),
   first step dt0, budget nsteps.  Returns GP_ERR_NOMEM when the pool or the
   slot table is full.  Takes effect at the next gp_batch_advance. */
int gp_batch_add(gp_batch *b, const gp_grid_desc *grid, const gp_scheme *scheme,
                 const gp_tile_shape *shape, const double *Vc, const double *Vs0,
                 const double *Vs1, const double *Vs2, double dt0, int nsteps, int *slot);
/* Change a slot's tile shape, or the blocks of the sweep launch (0: all that
   fit); results do not depend on either.  Take effect at the next
   gp_batch_advance. */
int gp_batch_set_shape(gp_batch *b, int slot, const gp_tile_shape *shape);
int gp_batch_set_ctas(gp_batch *b, int ctas);
/* Release a slot and its pool space (after gp_batch_wait). */
int gp_batch_remove(gp_batch *b, int slot);
/* Enqueue `nsteps` steps of every slot with budget left (asynchronous; the
   graph for this step count is captured on first use). */
int gp_batch_advance(gp_batch *b, int nsteps);
/* Wait for the enqueued steps and refresh every slot's status.  Returns
   GP_ERR_TIMEOUT when a finish tile's bounded wait for its slot's EMF tiles
   ran out (the launch then skips every later tile and ends; the slots being
   advanced hold a partly updated state and should be removed); the report
   clears the condition. */
int gp_batch_wait(gp_batch *b);
/* Host-side fault injection for tests (no reference counterpart): from the
   next gp_batch_advance, slot `slot`'s finish tiles wait for `extra_need`
   more EMF tiles than exist, and a wait gives up after `spin_limit` polls
   (0: the default, about a second).  extra_need 0 removes the fault. */
int gp_batch_inject_wait_fault(gp_batch *b, int slot, int extra_need, long long spin_limit);
int gp_batch_slot_status(const gp_batch *b, int slot, gp_slot_status *st);
/* Copy a slot's state to the host (interior layout; any pointer may be NULL). */
int gp_batch_download(gp_batch *b, int slot, double *Uc, double *Vc, double *Vs0,
                      double *Vs1, double *Vs2);
/* Pool occupancy, slot count and blocks of the persistent launch. */
int gp_batch_info(const gp_batch *b, size_t *pool_used, size_t *pool_bytes, int *slots,
                  int *ctas);

/* Text of the last error on this thread. */
const char *gp_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* GPLUTO_B200_H */
