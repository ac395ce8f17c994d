// bvh_exact.h -- exact sign of a quantisation grid corner against a bound,
// shared by the host and device encoders so both round child boxes outward
// identically.
#pragma once

#include <cuda_runtime.h>

#include <cmath>

namespace vt {

// a + b = s + e exactly (Knuth's TwoSum; every operation rounded on its own)
__host__ __device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
#ifdef __CUDA_ARCH__
  s = __dadd_rn(a, b);
  const double bb = __dsub_rn(s, a);
  e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
#else
  s = a + b;
  const double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
#endif
}

// Sign of p + q 2^e - m, exactly (-1, 0, 1): the three terms are summed into a
// nonoverlapping expansion by Shewchuk's (1997) grow-expansion of TwoSums,
// whose largest nonzero component carries the sign of the sum.
__host__ __device__ inline int corner_sign(float p, int q, int e, float m) {
  double comp[3];
  int nc = 0;
  comp[nc++] = (double)p;
  const double terms[2] = {ldexp((double)q, e), -(double)m};
  for (int t = 0; t < 2; ++t) {
    double Q = terms[t];
    double out[3];
    int no = 0;
    for (int i = 0; i < nc; ++i) {
      double s, h;
      two_sum(Q, comp[i], s, h);
      Q = s;
      if (h != 0.0) out[no++] = h;
    }
    out[no++] = Q;
    for (int i = 0; i < no; ++i) comp[i] = out[i];
    nc = no;
  }
  for (int i = nc - 1; i >= 0; --i)
    if (comp[i] != 0.0) return comp[i] > 0.0 ? 1 : -1;
  return 0;
}

}  // namespace vt
