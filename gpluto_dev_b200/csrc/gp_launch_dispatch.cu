// gp_launch_dispatch.cu -- joins the per-physics launch units of
// gp_launch.cu (compiled once per form and physics, GP_MIXED x GP_PART).
#include "gp_kernels.cuh"
#include "gp_launch.h"

namespace gp {

int sweep_m_blocks_per_sm(int physics, bool mixed) {
  if (physics == PHYS_RMHD)
    return mixed ? sweep_m_minb<PHYS_RMHD, float>() : sweep_m_minb<PHYS_RMHD, double>();
  if (physics == PHYS_MHD)
    return mixed ? sweep_m_minb<PHYS_MHD, float>() : sweep_m_minb<PHYS_MHD, double>();
  return mixed ? sweep_m_minb<PHYS_HD, float>() : sweep_m_minb<PHYS_HD, double>();
}

#define GP_PART_DECL(name)                                                              \
  int name(const StageDesc& d, const GridDims& g, const SchemeKey& k, int seg,         \
           cudaStream_t s, cudaEvent_t* ev);
GP_PART_DECL(launch_stage_fp64_p0)
GP_PART_DECL(launch_stage_fp64_p1)
GP_PART_DECL(launch_stage_fp64_p2)
GP_PART_DECL(launch_stage_fp64_p3)
GP_PART_DECL(launch_stage_mixed_p0)
GP_PART_DECL(launch_stage_mixed_p1)
GP_PART_DECL(launch_stage_mixed_p2)
GP_PART_DECL(launch_stage_mixed_p3)

// the MHD schemes are split over two units by Riemann solver
static bool mhd_part3(const SchemeKey& k) {
  return k.riemann == 1 /* HLLC */ || k.riemann == 3 /* Lax-Friedrichs */;
}

int launch_stage_fp64(const StageDesc& d, const GridDims& g, const SchemeKey& k, int seg,
                      cudaStream_t s, cudaEvent_t* ev) {
  switch (k.physics) {
    case 0: return launch_stage_fp64_p0(d, g, k, seg, s, ev);
    case 1: return mhd_part3(k) ? launch_stage_fp64_p3(d, g, k, seg, s, ev)
                                : launch_stage_fp64_p1(d, g, k, seg, s, ev);
    case 2: return launch_stage_fp64_p2(d, g, k, seg, s, ev);
    default: return -1;
  }
}

int launch_stage_mixed(const StageDesc& d, const GridDims& g, const SchemeKey& k, int seg,
                       cudaStream_t s, cudaEvent_t* ev) {
  switch (k.physics) {
    case 0: return launch_stage_mixed_p0(d, g, k, seg, s, ev);
    case 1: return mhd_part3(k) ? launch_stage_mixed_p3(d, g, k, seg, s, ev)
                                : launch_stage_mixed_p1(d, g, k, seg, s, ev);
    case 2: return launch_stage_mixed_p2(d, g, k, seg, s, ev);
    default: return -1;
  }
}

}  // namespace gp
