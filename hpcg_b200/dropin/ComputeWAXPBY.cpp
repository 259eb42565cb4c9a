// ComputeWAXPBY.cpp (drop-in) -- replaces src/ComputeWAXPBY.cpp
// (interface src/ComputeWAXPBY.hpp:18): w = alpha x + beta y on the GPU with
// the reference's alpha == 1 / beta == 1 rounding branches.
#include "ComputeWAXPBY.hpp"

#include "hpcgx_dropin.hpp"

int ComputeWAXPBY(const local_int_t n, const double alpha, const Vector &x, const double beta,
                  const Vector &y, Vector &w, bool &isOptimized) {
  (void)isOptimized;
  hpcgx_problem *p = hpcgx_dropin::current();
  if (!p) return HPCGX_ESTATE;
  return hpcgx_dropin::report(hpcgx_waxpby_host(p, n, alpha, x.values, beta, y.values, w.values),
                              "ComputeWAXPBY");
}
