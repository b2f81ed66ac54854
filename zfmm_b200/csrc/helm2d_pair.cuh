// One source-target interaction of zh2devaldirect
// (zfmm2d/src/helmholtz/zhfmm2d.f:773-838), unscaled (the driver applies i/4):
//   pot  += q H0(zk R) + ds (v . (y - x)) zk H1(zk R) / R
//   grad += -q zk H1 (x - y)/R + dipole terms through H1' = (H0 - H2)/2
// with R = sqrt((y1-x1)^2 + (y2-x2)^2) on the principal branch.  The pair is
// skipped unless |zk R| > 1E-16 (a REAL*4 literal in the reference) and
// Im(zk R) > -32, as in the reference.
#pragma once
#include "hank2d.cuh"

namespace zf {

template <bool GRAD>
__device__ __forceinline__ void helm_pair(zdc zk, zdc x1, zdc x2, zdc y1, zdc y2, zdc q, zdc ds,
                                          zdc d1, zdc d2, int ifcharge, int ifdipole, zdc& pot,
                                          zdc& g1, zdc& g2) {
  zdc y1mx1 = y1 - x1, y2mx2 = y2 - x2;
  zdc rz = zsqrt_p(y1mx1 * y1mx1 + y2mx2 * y2mx2);
  zdc z = rz * zk;
  if (!(zabs(z) > (double)1e-16f && z.im > -32.0)) return;  // REAL*4 literal 1E-16
  zdc h0, h1;
  hank01(z, h0, h1);
  zdc irz = zinv(rz);
  zdc zh1 = zk * h1;
  if (ifcharge) {
    pot += q * h0;
    if (GRAD) {
      zdc f = q * (zh1 * irz);
      g1 += f * y1mx1;  // -q zk h1 (x - y)/rz
      g2 += f * y2mx2;
    }
  }
  if (ifdipole) {
    zdc tmp = d1 * y1mx1 + d2 * y2mx2;
    pot += ds * (tmp * (zh1 * irz));
    if (GRAD) {
      zdc h2 = (2.0 * zinv(z)) * h1 - h0;
      zdc dh1 = 0.5 * (h0 - h2);
      zdc irz2 = irz * irz, irz3 = irz2 * irz;
      zdc a = zk * dh1 * irz2 - h1 * irz3;  // multiplies x - y = -(y - x)
      zdc dsz = ds * zk;
      g1 += dsz * ((-a * y1mx1) * tmp) - ds * (zh1 * irz) * d1;
      g2 += dsz * ((-a * y2mx2) * tmp) - ds * (zh1 * irz) * d2;
    }
  }
}

}  // namespace zf
