// gp_checks.h -- the argument checks shared by the C-ABI entry points
// (gp_api.cu, gp_noalloc.cu).  Not included by the kernel units, which are
// compiled with a GP_MIXED macro that the public header uses as a name.
#pragma once
#include "../../include/gpluto_b200.h"

namespace gp {

// The grid and scheme checks of gp_create (the combinations the kernels are
// built for, with the reference's own refusals); GP_OK or a gp_status with
// the reason written to gp_last_error.
int validate_scheme(const gp_grid_desc* grid, const gp_scheme* scheme);
// Cell widths as gp_create takes them: dx[d][0] when the caller passes the
// grid's widths (which must then be bitwise uniform), else
// (xend - xbeg) / nint; non-positive widths become 1.
int cell_widths(const gp_grid_desc* grid, double dx[3]);

}  // namespace gp
