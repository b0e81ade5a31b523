// Host build of gpluto_dev_b200/csrc/gp_crmath.cuh for the CPU tests, beside
// binary128 evaluations of the same functions (libquadmath) rounded once.
#include <quadmath.h>
#include <stddef.h>
#define GP_CR_COUNT_SLOW 1
#include "../gpluto_dev_b200/csrc/gp_crmath.cuh"

namespace gpcr {
long gp_cr_slow_calls = 0;
}

extern "C" {
long crm_slow_calls(void) { return gpcr::gp_cr_slow_calls; }

// which: 0 acos, 1 sin, 2 cos
void crm_eval(int which, const double* x, double* ours, double* quad, size_t n) {
  for (size_t i = 0; i < n; i++) {
    double s, c;
    switch (which) {
      case 0:
        ours[i] = gpcr::acos_cr(x[i]);
        quad[i] = (double)acosq((__float128)x[i]);
        break;
      case 1:
        gpcr::sincos_cr(x[i], &s, &c);
        ours[i] = s;
        quad[i] = (double)sinq((__float128)x[i]);
        break;
      default:
        gpcr::sincos_cr(x[i], &s, &c);
        ours[i] = c;
        quad[i] = (double)cosq((__float128)x[i]);
        break;
    }
  }
}
}
