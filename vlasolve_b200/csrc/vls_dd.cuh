// vls_dd.cuh -- compensated (double-double) sums for the device scans.
#pragma once

namespace vls {

// Compensated (double-double) arithmetic: TwoSum (Knuth) on hi, lo pairs.
struct dd {
  double hi, lo;
};
__device__ __forceinline__ dd dd_add(dd a, dd b) {
  const double s = a.hi + b.hi;
  const double bb = s - a.hi;
  double e = (a.hi - (s - bb)) + (b.hi - bb);
  e += a.lo + b.lo;
  const double h = s + e;
  return dd{h, e - (h - s)};
}
__device__ __forceinline__ dd dd_shfl_up(dd a, int d) {
  return dd{__shfl_up_sync(0xffffffffu, a.hi, d),
            __shfl_up_sync(0xffffffffu, a.lo, d)};
}
__device__ __forceinline__ dd dd_shfl_down(dd a, int d) {
  return dd{__shfl_down_sync(0xffffffffu, a.hi, d),
            __shfl_down_sync(0xffffffffu, a.lo, d)};
}

}  // namespace vls
