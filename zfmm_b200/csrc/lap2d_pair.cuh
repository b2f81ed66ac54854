// One source-target interaction of zl2devaldirect (zfmm2d/src/laplace/zlfmm2d.f:600-654):
//   pot  += q log(R) - ds (v . (y - x)) / R^2
//   grad += q (x - y) / R^2 - ds [dipole gradient] / R^4
// with R = sqrt((y1-x1)^2 + (y2-x2)^2) on the principal branch and the pair
// skipped when |R| <= 1e-16, exactly as the reference.
#pragma once
#include "zcomplex.cuh"

namespace zf {

template <bool GRAD>
__device__ __forceinline__ void lap2d_pair(zdc x1, zdc x2, zdc y1, zdc y2, zdc q, zdc ds, zdc d1,
                                           zdc d2, int ifcharge, int ifdipole, zdc& pot, zdc& g1,
                                           zdc& g2) {
  zdc a = y1 - x1, c = y2 - x2;  // y - x
  zdc rsq = a * a + c * c;
  zdc rz = zsqrt_p(rsq);
  if (!(zabs(rz) > (double)1e-16f)) return;  // the reference compares with the REAL*4 literal 1E-16
  zdc irsq = zinv(rsq);
  if (ifcharge) {
    pot += q * zlog_p(rz);
    if (GRAD) {
      zdc f = q * irsq;
      g1 -= f * a;
      g2 -= f * c;
    }
  }
  if (ifdipole) {
    pot -= ds * ((d1 * a + d2 * c) * irsq);
    if (GRAD) {
      // (x - y) enters squared or as a product, so (a, c) may be used directly
      zdc i4 = irsq * irsq;
      zdc t1 = d1 * (a * a - c * c) + 2.0 * (d2 * (a * c));
      zdc t2 = 2.0 * (d1 * (a * c)) + d2 * (c * c - a * a);
      g1 -= ds * (t1 * i4);
      g2 -= ds * (t2 * i4);
    }
  }
}

}  // namespace zf
