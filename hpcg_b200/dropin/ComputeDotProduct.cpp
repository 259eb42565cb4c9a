// ComputeDotProduct.cpp (drop-in) -- replaces src/ComputeDotProduct.cpp
// (interface src/ComputeDotProduct.hpp:18).  One process per problem, so no
// allreduce time is added.
#include "ComputeDotProduct.hpp"

#include "hpcgx_dropin.hpp"

int ComputeDotProduct(const local_int_t n, const Vector &x, const Vector &y, double &result,
                      double &time_allreduce, bool &isOptimized) {
  (void)time_allreduce;
  (void)isOptimized;
  hpcgx_problem *p = hpcgx_dropin::current();
  if (!p) return HPCGX_ESTATE;
  return hpcgx_dropin::report(hpcgx_dot_host(p, n, x.values, y.values, &result),
                              "ComputeDotProduct");
}
