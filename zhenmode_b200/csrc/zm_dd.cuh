// Compensated float64 sums for the budget and ledger reductions: each lane
// keeps a Neumaier sum, lanes, warps and blocks combine as double-double
// values (TwoSum), and partials are folded in a fixed order, so a result does
// not depend on timing.
#pragma once

#include <cuda_runtime.h>

namespace zm {

struct DD {
  double hi, lo;
};

__device__ __forceinline__ DD two_sum(double a, double b) {
  const double s = a + b;
  const double bb = s - a;
  return DD{s, (a - (s - bb)) + (b - bb)};
}

__device__ __forceinline__ DD dd_add(DD x, DD y) {
  DD s = two_sum(x.hi, y.hi);
  const double e = s.lo + (x.lo + y.lo);
  const double hi = s.hi + e;
  return DD{hi, e - (hi - s.hi)};
}

// Neumaier step: running sum x.hi, compensation x.lo
__device__ __forceinline__ void neumaier(DD& x, double v) {
  const double t = x.hi + v;
  if (fabs(x.hi) >= fabs(v)) x.lo += (x.hi - t) + v;
  else x.lo += (v - t) + x.hi;
  x.hi = t;
}

__device__ __forceinline__ DD shfl_dd(DD x, int o) {
  return DD{__shfl_down_sync(0xffffffffu, x.hi, o), __shfl_down_sync(0xffffffffu, x.lo, o)};
}

}  // namespace zm
