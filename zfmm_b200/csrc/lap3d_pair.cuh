// One source-target interaction of zl3devaldirect
// (zfmm3d/src/laplace/zlfmm3d.f:628-683), y = source - target:
//   pot  += q / (4 pi R) - ds (-(y . v)) / (4 pi R^3)
//   grad += q y / (4 pi R^3) - ds [v / (4 pi R^3) + 3 (-(y . v)) y / (4 pi R^5)]
// R = sqrt(y . y) on the principal branch; the pair is skipped when
// |R| <= 1e-16 (REAL*4 literal), as in the reference.
#pragma once
#include "zcomplex.cuh"

namespace zf {

template <bool GRAD>
__device__ __forceinline__ void lap3d_pair(const zdc x[3], const zdc ysrc[3], zdc q, zdc ds,
                                           const zdc v[3], int ifcharge, int ifdipole, zdc& pot,
                                           zdc g[3]) {
  constexpr double PI4I = 0.079577471545947667884;  // 1/(4 pi)
  zdc y0 = ysrc[0] - x[0], y1 = ysrc[1] - x[1], y2 = ysrc[2] - x[2];
  zdc rz = zsqrt_p(y0 * y0 + y1 * y1 + y2 * y2);
  if (!(zabs(rz) > (double)1e-16f)) return;
  zdc ir = zinv(rz);
  zdc r1 = ir * PI4I;
  zdc r3 = r1 * (ir * ir);
  if (ifcharge) {
    pot += q * r1;
    if (GRAD) {
      zdc f = q * r3;
      g[0] += f * y0;
      g[1] += f * y1;
      g[2] += f * y2;
    }
  }
  if (ifdipole) {
    zdc dot = -(y0 * v[0] + y1 * v[1] + y2 * v[2]);
    zdc dr3 = ds * r3;
    pot -= dr3 * dot;
    if (GRAD) {
      zdc dd = ds * (3.0 * (dot * (r3 * (ir * ir))));
      g[0] -= dr3 * v[0] + dd * y0;
      g[1] -= dr3 * v[1] + dd * y1;
      g[2] -= dr3 * v[2] + dd * y2;
    }
  }
}

}  // namespace zf
