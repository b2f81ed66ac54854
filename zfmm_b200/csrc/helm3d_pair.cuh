// One source-target interaction of zh3devaldirect
// (zfmm3d/src/helmholtz/zhfmm3d.f:626-693), x = target - source, R = sqrt(x . x)
// on the principal branch, z = i k R:
//   pot  += q e^z / (4 pi R) - ds (x . v) e^z (1 - z) / (4 pi R^3)
//   grad += -q x e^z (1 - z) / (4 pi R^3)
//           - ds [v e^z (1-z) / (4 pi R^3) + x (x . v) e^z (k^2 - 3 (1-z)/R^2) / (4 pi R^3)]
// skipped when |R| <= 1e-16 (REAL*4 literal), as in the reference.
#pragma once
#include "zcomplex.cuh"

namespace zf {

template <bool GRAD>
__device__ __forceinline__ void helm3d_pair(zdc zk, const zdc x[3], const zdc ysrc[3], zdc q,
                                            zdc ds, const zdc v[3], int ifcharge, int ifdipole,
                                            zdc& pot, zdc g[3]) {
  constexpr double PI4I = 0.079577471545947667884;  // 1/(4 pi)
  zdc x0 = x[0] - ysrc[0], x1 = x[1] - ysrc[1], x2 = x[2] - ysrc[2];
  zdc rz = zsqrt_p(x0 * x0 + x1 * x1 + x2 * x2);
  if (!(zabs(rz) > (double)1e-16f)) return;
  zdc z = zmul_i(zk * rz);
  zdc ez = zexp_p(z);
  zdc ir = zinv(rz);
  zdc r1 = ir * PI4I;
  zdc r3 = r1 * (ir * ir);
  zdc t4 = mkz(1.0) - z;
  if (ifcharge) {
    pot += q * (ez * r1);
    if (GRAD) {
      zdc h = q * (ez * t4 * r3);
      g[0] -= h * x0;
      g[1] -= h * x1;
      g[2] -= h * x2;
    }
  }
  if (ifdipole) {
    zdc dot = x0 * v[0] + x1 * v[1] + x2 * v[2];
    zdc e3 = ez * r3;
    pot -= ds * (e3 * dot * t4);
    if (GRAD) {
      zdc t1 = dot * e3 * (zk * zk - 3.0 * (t4 * (ir * ir)));
      zdc t2 = t4 * e3;
      g[0] -= ds * (v[0] * t2 + x0 * t1);
      g[1] -= ds * (v[1] * t2 + x1 * t1);
      g[2] -= ds * (v[2] * t2 + x2 * t1);
    }
  }
}

}  // namespace zf
