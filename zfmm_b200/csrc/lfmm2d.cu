// 2D Laplace complex-coordinate FMM (zlfmm2d) on the device.
//
// Reference: zfmm2d/src/laplace/zlfmm2d.f (driver :14-234, 8 steps of
// zlfmm2dmain :240-594, kernels :600-915) and zfmm2d/src/laplace/zl2dtrans.f.
//
// The reference writes every expansion in "polar" form about a complex centre
// c: for y - c = (z1, z2) it uses rz = sqrt(z1^2 + z2^2) (principal branch) and
// ez = (z1 + i z2)/rz.  Only the products rz*ez and rz/ez enter the series, and
// with complex coordinates these are the two independent variables
//     zeta = z1 + i z2  (= rz*ez)     xi = z1 - i z2  (= rz/ez = rz^2/zeta)
// so that, term for term,
//     mp(m)  pairs with xi^m,   mp(-m)  with zeta^m,
//     loc(m) pairs with zeta^m, loc(-m) with xi^m,
// and only the m = 0 terms keep log(rz).  The kernels below evaluate exactly
// the reference's series in these variables (no square root or division per
// term); the reference's factors rscale^m are folded into the powers
// ((xi/rscale)^m etc.) so deep levels cannot under- or overflow.
//
// Parallel layout: one warp per box; inside a warp, lane k owns the expansion
// coefficients +-k (k = lane+1, lane+33, ...).  Every target box is written by
// exactly one warp (owner computes, no atomics), as in the reference's OpenMP
// loops over target boxes.
#include <vector>
#include "fmm2d_common.cuh"
#include "lfmm2d.cuh"
#include "lap2d_pair.cuh"

namespace zf {
namespace {

constexpr int WPB = 4;    // warps per block
constexpr int MAXR = 4;   // coefficient slots per lane: p <= 128

__device__ __forceinline__ void split2(zdc a1, zdc a2, zdc& zeta, zdc& xi) {
  // zeta = a1 + i a2, xi = a1 - i a2
  zeta = zdc{a1.re - a2.im, a1.im + a2.re};
  xi = zdc{a1.re + a2.im, a1.im - a2.re};
}

struct LapArgs {
  int p, P;                  // nterms, 2p+1
  const double* carray;      // binomial table (ldc+1)^2, ldc = 2p
  int ldc1;
  const double* rsc;         // rscale per level (= boxsize)
  const int* ilevel;
  const int* iparent;
  const int* nchild;
  const int* ichild;
  const int* isrcse;
  const int* itargse;
  const zdc* zsrc;           // sorted sources (2 per point)
  const zdc* charge;
  const zdc* dipstr;
  const zdc* dipvec;
  const zdc* ztarg;          // sorted targets
  const zdc* zcsrc;          // complex centres
  const zdc* zctarg;
  zdc* mp;                   // [nboxes * P], coefficient m of box b at b*P + p + m
  zdc* loc;
  int ifcharge, ifdipole;
};

#define C_(l, m) __ldg(&A.carray[(l) * A.ldc1 + (m)])

// ---- step 1: P2M, one warp per leaf with sources (zl2dformmp) ----------------
__global__ void __launch_bounds__(32 * WPB) k_p2m(int nb, LapArgs A) {
  int w = blockIdx.x * WPB + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (w >= nb) return;
  int b = w;
  int s0 = A.isrcse[2 * b], s1 = A.isrcse[2 * b + 1];
  if (A.nchild[b] > 0 || s1 < s0) return;
  double rs = A.rsc[A.ilevel[b]];
  zdc c1 = A.zcsrc[2 * b], c2 = A.zcsrc[2 * b + 1];
  int p = A.p;
  zdc accp[MAXR], accm[MAXR], acc0 = mkz(0.0);
#pragma unroll
  for (int r = 0; r < MAXR; r++) { accp[r] = mkz(0.0); accm[r] = mkz(0.0); }
  for (int j = s0; j <= s1; j++) {
    zdc zeta, xi;
    split2(ldz(&A.zsrc[2 * j]) - c1, ldz(&A.zsrc[2 * j + 1]) - c2, zeta, xi);
    zdc xs = xi / rs, zs = zeta / rs;
    zdc q = A.ifcharge ? ldz(&A.charge[j]) : mkz(0.0);
    zdc dx = mkz(0.0), dz = mkz(0.0);
    if (A.ifdipole) {
      zdc ds = ldz(&A.dipstr[j]), d1 = ldz(&A.dipvec[2 * j]), d2 = ldz(&A.dipvec[2 * j + 1]);
      dx = ds * (d1 - zmul_i(d2)) / (2.0 * rs);  // pairs with xi^(m-1)/rs^(m-1)
      dz = ds * (d1 + zmul_i(d2)) / (2.0 * rs);
    }
    if (lane == 0) acc0 += q;
#pragma unroll
    for (int r = 0; r < MAXR; r++) {
      int m = lane + 1 + 32 * r;
      if (m <= p) {
        zdc px1 = zpown(xs, m - 1), pz1 = zpown(zs, m - 1);
        zdc px = px1 * xs, pz = pz1 * zs;
        double h = 0.5 / m;
        accp[r] += dx * px1 - h * (q * px);
        accm[r] += dz * pz1 - h * (q * pz);
      }
    }
  }
  zdc* M = A.mp + (size_t)b * A.P + p;
  if (lane == 0) M[0] = acc0;
#pragma unroll
  for (int r = 0; r < MAXR; r++) {
    int m = lane + 1 + 32 * r;
    if (m <= p) { M[m] = accp[r]; M[-m] = accm[r]; }
  }
}

// ---- step 2: M2M, one warp per parent at level `lev` (zl2dmpmp) ---------------
__global__ void __launch_bounds__(32 * WPB) k_m2m(int lo, int hi, int lev, LapArgs A) {
  extern __shared__ zdc sh[];
  int p = A.p;
  zdc* ax = sh + (threadIdx.x >> 5) * 4 * (p + 1);
  zdc* az = ax + (p + 1);
  zdc* cp = az + (p + 1);
  zdc* cm = cp + (p + 1);
  int b = lo + blockIdx.x * WPB + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (b > hi) return;
  if (A.nchild[b] == 0 || A.isrcse[2 * b + 1] < A.isrcse[2 * b]) return;
  double rs1 = A.rsc[lev], rs2 = A.rsc[lev + 1], rr = rs2 / rs1;
  zdc c1 = A.zcsrc[2 * b], c2 = A.zcsrc[2 * b + 1];
  zdc accp[MAXR], accm[MAXR], acc0 = mkz(0.0);
#pragma unroll
  for (int r = 0; r < MAXR; r++) { accp[r] = mkz(0.0); accm[r] = mkz(0.0); }
  for (int jc = 0; jc < 4; jc++) {
    int jb = A.ichild[4 * b + jc];
    if (A.isrcse[2 * jb + 1] < A.isrcse[2 * jb]) continue;
    zdc zeta0, xi0;
    split2(A.zcsrc[2 * jb] - c1, A.zcsrc[2 * jb + 1] - c2, zeta0, xi0);
    zdc xa = xi0 / rs1, za = zeta0 / rs1;
    const zdc* M2 = A.mp + (size_t)jb * A.P + p;
    for (int j = lane; j <= p; j += 32) {
      ax[j] = zpown(xa, j);
      az[j] = zpown(za, j);
      double f = pow(rr, (double)j);
      cp[j] = f * M2[j];
      cm[j] = f * M2[-j];
    }
    __syncwarp();
    zdc m0 = cp[0];
    if (lane == 0) acc0 += m0;
#pragma unroll
    for (int r = 0; r < MAXR; r++) {
      int k = lane + 1 + 32 * r;
      if (k <= p) {
        zdc sp = (-0.5 / k) * (ax[k] * m0), sm = (-0.5 / k) * (az[k] * m0);
        for (int n = 1; n <= k; n++) {
          double cb = C_(k - 1, k - n);
          sp += cb * (ax[k - n] * cp[n]);
          sm += cb * (az[k - n] * cm[n]);
        }
        accp[r] += sp;
        accm[r] += sm;
      }
    }
    __syncwarp();
  }
  zdc* M = A.mp + (size_t)b * A.P + p;
  if (lane == 0) M[0] = acc0;
#pragma unroll
  for (int r = 0; r < MAXR; r++) {
    int k = lane + 1 + 32 * r;
    if (k <= p) { M[k] = accp[r]; M[-k] = accm[r]; }
  }
}

// ---- steps 4 + 6: M2L over list2 and P2L over list4 (zl2dmploc, zl2dformloc) --
__global__ void __launch_bounds__(32 * WPB) k_m2l_p2l(int nb, LapArgs A, const int* nl2,
                                                     const int* l2, int m2, const int* nl4,
                                                     const int* l4, int m4) {
  extern __shared__ zdc sh[];
  int p = A.p;
  zdc* pu = sh + (threadIdx.x >> 5) * 4 * (p + 1);
  zdc* pub = pu + (p + 1);
  zdc* Aa = pub + (p + 1);
  zdc* Bb = Aa + (p + 1);
  int b = blockIdx.x * WPB + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (b >= nb) return;
  if (A.itargse[2 * b + 1] < A.itargse[2 * b]) return;
  int n2c = nl2[b], n4c = nl4[b];
  if (n2c == 0 && n4c == 0) return;
  double rs = A.rsc[A.ilevel[b]];
  zdc c1 = A.zctarg[2 * b], c2 = A.zctarg[2 * b + 1];
  zdc accp[MAXR], accm[MAXR], acc0 = mkz(0.0);
#pragma unroll
  for (int r = 0; r < MAXR; r++) { accp[r] = mkz(0.0); accm[r] = mkz(0.0); }
  for (int il = 0; il < n2c; il++) {
    int jb = l2[(size_t)b * m2 + il];
    if (A.isrcse[2 * jb + 1] < A.isrcse[2 * jb]) continue;
    zdc z1 = A.zcsrc[2 * jb] - c1, z2 = A.zcsrc[2 * jb + 1] - c2;
    zdc zeta0, xi0;
    split2(z1, z2, zeta0, xi0);
    zdc u = zdc{rs, 0.0} / zeta0, ub = zdc{rs, 0.0} / xi0;
    const zdc* M = A.mp + (size_t)jb * A.P + p;
    zdc part0 = mkz(0.0);
    for (int j = lane; j <= p; j += 32) {
      zdc a = zpown(u, j), bb = zpown(ub, j);
      pu[j] = a;
      pub[j] = bb;
      double sg = (j & 1) ? -1.0 : 1.0;
      Aa[j] = sg * (a * M[-j]);
      Bb[j] = sg * (bb * M[j]);
      if (j > 0) part0 += Aa[j] + Bb[j];
    }
    __syncwarp();
    zdc m0 = M[0];
    for (int o = 16; o; o >>= 1) part0 += shfl_xor_z(part0, o);
    if (lane == 0) {
      zdc r0 = zsqrt_p(z1 * z1 + z2 * z2);
      acc0 += m0 * zlog_p(r0) + part0;
    }
#pragma unroll
    for (int r = 0; r < MAXR; r++) {
      int k = lane + 1 + 32 * r;
      if (k <= p) {
        zdc sp = (-0.5 / k) * m0, sm = sp;
        for (int n = 1; n <= p; n++) {
          double cb = C_(n + k - 1, k);
          sp += cb * Aa[n];
          sm += cb * Bb[n];
        }
        accp[r] += pu[k] * sp;
        accm[r] += pub[k] * sm;
      }
    }
    __syncwarp();
  }
  for (int il = 0; il < n4c; il++) {
    int jb = l4[(size_t)b * m4 + il];
    int s0 = A.isrcse[2 * jb], s1 = A.isrcse[2 * jb + 1];
    for (int j = s0; j <= s1; j++) {
      zdc z1 = ldz(&A.zsrc[2 * j]) - c1, z2 = ldz(&A.zsrc[2 * j + 1]) - c2;
      zdc zeta, xi;
      split2(z1, z2, zeta, xi);
      zdc q = A.ifcharge ? ldz(&A.charge[j]) : mkz(0.0);
      zdc dz = mkz(0.0), dx = mkz(0.0);
      zdc rsq = z1 * z1 + z2 * z2;
      if (lane == 0) {
        zdc t = mkz(0.0);
        if (A.ifcharge) t += q * zlog_p(zsqrt_p(rsq));
        if (A.ifdipole) {
          zdc ds = ldz(&A.dipstr[j]), d1 = ldz(&A.dipvec[2 * j]), d2 = ldz(&A.dipvec[2 * j + 1]);
          t -= ds * ((z1 * d1 + z2 * d2) / rsq);
        }
        acc0 += t;
      }
      if (A.ifdipole) {
        zdc ds = ldz(&A.dipstr[j]), d1 = ldz(&A.dipvec[2 * j]), d2 = ldz(&A.dipvec[2 * j + 1]);
        dz = ds * (d1 + zmul_i(d2)) / (2.0 * zeta);
        dx = ds * (d1 - zmul_i(d2)) / (2.0 * xi);
      }
      zdc wz = zdc{rs, 0.0} / zeta, wx = zdc{rs, 0.0} / xi;
#pragma unroll
      for (int r = 0; r < MAXR; r++) {
        int k = lane + 1 + 32 * r;
        if (k <= p) {
          zdc pz = zpown(wz, k), px = zpown(wx, k);
          double h = 0.5 / k;
          accp[r] -= (h * q + dz) * pz;
          accm[r] -= (h * q + dx) * px;
        }
      }
    }
  }
  zdc* L = A.loc + (size_t)b * A.P + p;
  if (lane == 0) L[0] = acc0;
#pragma unroll
  for (int r = 0; r < MAXR; r++) {
    int k = lane + 1 + 32 * r;
    if (k <= p) { L[k] = accp[r]; L[-k] = accm[r]; }
  }
}

// ---- step 7: L2L into the children at level lev+1 (zl2dlocloc) --------------
__global__ void __launch_bounds__(32 * WPB) k_l2l(int lo, int hi, int lev, LapArgs A,
                                                 const int* nl2, const int* nl4) {
  extern __shared__ zdc sh[];
  int p = A.p;
  zdc* pz = sh + (threadIdx.x >> 5) * 4 * (p + 1);
  zdc* px = pz + (p + 1);
  zdc* lp = px + (p + 1);
  zdc* lm = lp + (p + 1);
  int jb = lo + blockIdx.x * WPB + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (jb > hi) return;
  int b = A.iparent[jb];
  if (A.itargse[2 * b + 1] < A.itargse[2 * b] || (nl2[b] == 0 && nl4[b] == 0)) return;
  if (A.itargse[2 * jb + 1] < A.itargse[2 * jb]) return;
  double rs2 = A.rsc[lev], rs1 = A.rsc[lev + 1], rr = rs1 / rs2;
  zdc zeta0, xi0;
  split2(A.zctarg[2 * b] - A.zctarg[2 * jb], A.zctarg[2 * b + 1] - A.zctarg[2 * jb + 1], zeta0,
         xi0);
  zdc za = zeta0 / rs2, xa = xi0 / rs2;
  const zdc* L2 = A.loc + (size_t)b * A.P + p;
  zdc part0 = mkz(0.0);
  for (int j = lane; j <= p; j += 32) {
    pz[j] = zpown(za, j);
    px[j] = zpown(xa, j);
    lp[j] = L2[j];
    lm[j] = L2[-j];
    if (j > 0) {
      double sg = (j & 1) ? -1.0 : 1.0;
      part0 += sg * (pz[j] * lp[j] + px[j] * lm[j]);
    }
  }
  __syncwarp();
  for (int o = 16; o; o >>= 1) part0 += shfl_xor_z(part0, o);
  zdc* L1 = A.loc + (size_t)jb * A.P + p;
  if (lane == 0) L1[0] += lp[0] + part0;
#pragma unroll
  for (int r = 0; r < MAXR; r++) {
    int k = lane + 1 + 32 * r;
    if (k <= p) {
      zdc sp = mkz(0.0), sm = mkz(0.0);
      for (int n = k; n <= p; n++) {
        double cb = ((n - k) & 1) ? -C_(n, k) : C_(n, k);
        sp += cb * (pz[n - k] * lp[n]);
        sm += cb * (px[n - k] * lm[n]);
      }
      double f = pow(rr, (double)k);
      L1[k] += f * sp;
      L1[-k] += f * sm;
    }
  }
}

// ---- steps 3, 5, 8: P2P (list1), M2T (list3), L2T (own local) per target leaf --
template <bool GRAD>
__global__ void __launch_bounds__(32 * WPB) k_eval(int nb, LapArgs A, const int* nl1,
                                                  const int* l1, int m1, const int* nl3,
                                                  const int* l3, int m3, zdc* potsort,
                                                  zdc* gradsort) {
  int b = blockIdx.x * WPB + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (b >= nb) return;
  int t0 = A.itargse[2 * b], t1 = A.itargse[2 * b + 1];
  if (A.nchild[b] > 0 || t1 < t0) return;
  int ntb = t1 - t0 + 1;
  int pw = 1;
  while (pw < ntb && pw < 32) pw <<= 1;
  int G = 32 / pw;              // lanes per target
  int T = 32 / G;               // targets per round
  int tl = lane / G, r = lane % G;
  int p = A.p;
  double rsb = A.rsc[A.ilevel[b]];
  zdc lc1 = A.zctarg[2 * b], lc2 = A.zctarg[2 * b + 1];
  const zdc* L = A.loc + (size_t)b * A.P + p;
  for (int base = 0; base < ntb; base += T) {
    int ti = t0 + base + tl;
    bool valid = base + tl < ntb;
    zdc pot = mkz(0.0), g1 = mkz(0.0), g2 = mkz(0.0);
    if (valid) {
      zdc x1 = ldz(&A.ztarg[2 * ti]), x2 = ldz(&A.ztarg[2 * ti + 1]);
      // L2T (zl2devalloc).  Boxes on levels 0 and 1 have empty lists 2 and 4,
      // so their local expansion is identically zero and is skipped (this also
      // avoids 0/0 when all points coincide and the root has size 0).
      if (A.ilevel[b] >= 2) {
        zdc zeta, xi;
        split2(x1 - lc1, x2 - lc2, zeta, xi);
        zdc vz = zeta / rsb, vx = xi / rsb;
        if (r == 0) pot += L[0];
        if (r + 1 <= p) {
          zdc stz = zpown(vz, G), stx = zpown(vx, G);
          zdc pz1 = zpown(vz, r), px1 = zpown(vx, r);
          for (int m = r + 1; m <= p; m += G) {
            zdc lpm = ldz(&L[m]), lmm = ldz(&L[-m]);
            zdc a = lpm * pz1, c = lmm * px1;
            pot += a * vz + c * vx;
            if (GRAD) {
              double f = m / rsb;
              g1 += f * (a + c);
              g2 += f * zmul_i(a - c);
            }
            pz1 = pz1 * stz;
            px1 = px1 * stx;
          }
        }
      }
      // M2T (zl2devalmp) over list3
      int n3 = nl3[b];
      for (int il = 0; il < n3; il++) {
        int jb = l3[(size_t)b * m3 + il];
        if (A.isrcse[2 * jb + 1] < A.isrcse[2 * jb]) continue;
        double rs3 = A.rsc[A.ilevel[jb]];
        const zdc* M = A.mp + (size_t)jb * A.P + p;
        zdc z1 = x1 - A.zcsrc[2 * jb], z2 = x2 - A.zcsrc[2 * jb + 1];
        zdc zeta, xi;
        split2(z1, z2, zeta, xi);
        zdc iz = zinv(zeta), ix = zinv(xi);
        if (r == 0) {
          zdc rsq = z1 * z1 + z2 * z2;
          zdc m0 = ldz(&M[0]);
          pot += m0 * zlog_p(zsqrt_p(rsq));
          if (GRAD) {
            zdc f = m0 / rsq;
            g1 += f * z1;
            g2 += f * z2;
          }
        }
        if (r + 1 <= p) {
          zdc wz = rs3 * iz, wx = rs3 * ix;
          zdc stz = zpown(wz, G), stx = zpown(wx, G);
          zdc pz = zpown(wz, r + 1), px = zpown(wx, r + 1);
          for (int m = r + 1; m <= p; m += G) {
            zdc a = ldz(&M[m]) * px, c = ldz(&M[-m]) * pz;
            pot += a + c;
            if (GRAD) {
              zdc ax = a * ix, cz = c * iz;
              g1 -= (double)m * (ax + cz);
              g2 += (double)m * zmul_i(ax - cz);
            }
            pz = pz * stz;
            px = px * stx;
          }
        }
      }
      // P2P (zl2devaldirect) over list1
      int n1 = nl1[b];
      for (int il = 0; il < n1; il++) {
        int jb = l1[(size_t)b * m1 + il];
        int s0 = A.isrcse[2 * jb], s1 = A.isrcse[2 * jb + 1];
        for (int j = s0 + r; j <= s1; j += G) {
          zdc q = A.ifcharge ? ldz(&A.charge[j]) : mkz(0.0);
          zdc ds = mkz(0.0), d1 = mkz(0.0), d2 = mkz(0.0);
          if (A.ifdipole) {
            ds = ldz(&A.dipstr[j]);
            d1 = ldz(&A.dipvec[2 * j]);
            d2 = ldz(&A.dipvec[2 * j + 1]);
          }
          lap2d_pair<GRAD>(x1, x2, ldz(&A.zsrc[2 * j]), ldz(&A.zsrc[2 * j + 1]), q, ds, d1, d2,
                           A.ifcharge, A.ifdipole, pot, g1, g2);
        }
      }
    }
    for (int o = 1; o < G; o <<= 1) {
      pot += shfl_xor_z(pot, o);
      if (GRAD) {
        g1 += shfl_xor_z(g1, o);
        g2 += shfl_xor_z(g2, o);
      }
    }
    if (valid && r == 0) {
      potsort[ti] = pot;
      if (GRAD) {
        gradsort[2 * ti] = g1;
        gradsort[2 * ti + 1] = g2;
      }
    }
  }
}

}  // namespace

int l2dterms(double eps) {
  // l2dterms.f:38-82: first j in 2..100 with (sqrt(2)/2)^j / 1.5^(j+1) < eps
  double z2 = sqrt(2.0) / 2.0;
  for (int j = 2; j <= 100; j++)
    if (pow(z2, j) / pow(1.5, j + 1) < eps) return j;
  return 1;
}

void lndiv2d(double eps, int ns, int nt, int* ndiv, int* idivflag) {
  // lndiv2d.f:17-35 (hndiv2d.f uses the same table)
  *idivflag = 0;
  if (eps >= 0.5e-0) *ndiv = 3;
  else if (eps >= 0.5e-1) *ndiv = 5;
  else if (eps >= 0.5e-2) *ndiv = 8;
  else if (eps >= 0.5e-3) *ndiv = 10;
  else if (eps >= 0.5e-6) *ndiv = 15;
  else if (eps >= 0.5e-9) *ndiv = 20;
  else if (eps >= 0.5e-12) *ndiv = 25;
  else if (eps >= 0.5e-15) *ndiv = 45;
  else *ndiv = ns + nt;
}

// the passes after the set-up for one right-hand side with sorted strengths
// q, ds, dv on a set-up S: writes the sorted, unscaled potentials / gradients
// into potsort / gradsort (zeroed by the caller); ev (optional) gets the step
// boundaries 2..5; *pl (optional) receives the order of every level
int lap2d_core(const Setup2D& S, double eps, const zdc* q, const zdc* ds, const zdc* dv, int ifcharge, int ifdipole, int ifpgh,
         zdc* potsort, zdc* gradsort, cudaStream_t s, cudaEvent_t* ev,
         std::vector<int>* pl) {
  auto cmark = [&](int i) {
    if (ev) ZF_CUDA(cudaEventRecord(ev[i], s));
  };
  const DevTree& t = S.tree;
  int nb = t.nboxes, nlev = t.nlevels;
  int p = l2dterms(eps);
  if (p > 32 * MAXR) throw zf_error(ZF_ERR_ARG, "expansion order too large");
  int P = 2 * p + 1, ldc = 2 * p;
  std::vector<double> carr((size_t)(ldc + 1) * (ldc + 1), 0.0);
  for (int l = 0; l <= ldc; l++) carr[(size_t)l * (ldc + 1)] = 1.0;
  for (int m = 1; m <= ldc; m++) {
    carr[(size_t)m * (ldc + 1) + m] = 1.0;
    for (int l = m + 1; l <= ldc; l++)
      carr[(size_t)l * (ldc + 1) + m] =
          carr[(size_t)(l - 1) * (ldc + 1) + m] + carr[(size_t)(l - 1) * (ldc + 1) + m - 1];
  }
  DevBuf<double> d_carr(carr.size(), s), d_rsc(nlev + 1, s);
  ZF_CUDA(cudaMemcpyAsync(d_carr.get(), carr.data(), carr.size() * sizeof(double),
                          cudaMemcpyHostToDevice, s));
  ZF_CUDA(cudaMemcpyAsync(d_rsc.get(), t.boxsize.data(), (nlev + 1) * sizeof(double),
                          cudaMemcpyHostToDevice, s));
  DevBuf<zdc> mp((size_t)nb * P, s), loc((size_t)nb * P, s);
  mp.zero();
  loc.zero();
  LapArgs A;
  A.p = p; A.P = P; A.carray = d_carr.get(); A.ldc1 = ldc + 1; A.rsc = d_rsc.get();
  A.ilevel = t.ilevel.get(); A.iparent = t.iparent.get(); A.nchild = t.nchild.get();
  A.ichild = t.ichild.get(); A.isrcse = S.isrcse.get(); A.itargse = S.itargse.get();
  A.zsrc = S.zsrcsort.get(); A.charge = q; A.dipstr = ds;
  A.dipvec = dv; A.ztarg = S.ztargsort.get(); A.zcsrc = S.zcsrc.get();
  A.zctarg = S.zctarg.get(); A.mp = mp.get(); A.loc = loc.get();
  A.ifcharge = ifcharge; A.ifdipole = ifdipole;
  size_t smem = (size_t)WPB * 4 * (p + 1) * sizeof(zdc);
  int grid_all = div_up(nb, WPB);
  const DevLists& L = S.lists;
  // step 1
  klaunch(k_p2m, grid_all, 32 * WPB, 0, s, nb, A);
  ZF_LAUNCH_CHECK();
  cmark(2);
  // step 2
  for (int l = nlev - 1; l >= 1; l--) {
    int lo = t.laddr[2 * l], hi = t.laddr[2 * l + 1];
    klaunch(k_m2m, div_up(hi - lo + 1, WPB), 32 * WPB, smem, s, lo, hi, l, A);
  }
  ZF_LAUNCH_CHECK();
  cmark(3);
  // steps 4 + 6
  klaunch(k_m2l_p2l, grid_all, 32 * WPB, smem, s, nb, A, L.n[1].get(), L.list[1].get(), L.mn[1],
                                             L.n[3].get(), L.list[3].get(), L.mn[3]);
  ZF_LAUNCH_CHECK();
  cmark(4);
  // step 7
  for (int l = 1; l <= nlev - 1; l++) {
    int lo = t.laddr[2 * (l + 1)], hi = t.laddr[2 * (l + 1) + 1];
    klaunch(k_l2l, div_up(hi - lo + 1, WPB), 32 * WPB, smem, s, lo, hi, l, A, L.n[1].get(),
                                                           L.n[3].get());
  }
  ZF_LAUNCH_CHECK();
  cmark(5);
  // steps 3, 5, 8
  if (ifpgh > 1)
    klaunch(k_eval<true>, grid_all, 32 * WPB, 0, s, nb, A, L.n[0].get(), L.list[0].get(), L.mn[0],
                                               L.n[2].get(), L.list[2].get(), L.mn[2],
                                               potsort, gradsort);
  else
    klaunch(k_eval<false>, grid_all, 32 * WPB, 0, s, nb, A, L.n[0].get(), L.list[0].get(), L.mn[0],
                                                L.n[2].get(), L.list[2].get(), L.mn[2],
                                                potsort, gradsort);
  ZF_LAUNCH_CHECK();
  if (pl) *pl = std::vector<int>(nlev + 1, p);
  return p;
}

void zlfmm2d_device(double eps, const Inputs2D& in, int isep, zdc* pot, zdc* grad,
                    cudaStream_t s, StepTimes* times) {
  int ns = in.ns, nt = in.nt;
  cudaEvent_t ev[10];
  bool timing = times != nullptr;
  if (timing)
    for (auto& e : ev) ZF_CUDA(cudaEventCreate(&e));
  auto mark = [&](int i) {
    if (timing) ZF_CUDA(cudaEventRecord(ev[i], s));
  };
  long launches0 = launch_counter();
  mark(0);
  TreeParams tp;
  tp.D = 2;
  tp.isep = isep;
  lndiv2d(eps, ns, nt, &tp.ndiv, &tp.idivflag);
  Setup2D S;
  setup2d(in, tp, S, s);
  mark(1);
  std::vector<int> plv;
  DevBuf<zdc> potsort(nt, s), gradsort(in.ifpgh > 1 ? 2 * (size_t)nt : 1, s);
  potsort.zero();
  gradsort.zero();
  const int pord = lap2d_core(S, eps, S.chargesort.get(), S.dipstrsort.get(),
      S.dipvecsort.get(), in.ifcharge, in.ifdipole, in.ifpgh, potsort.get(), gradsort.get(), s,
      timing ? ev : nullptr, &plv);
  mark(6);
  unsort2d(nt, S.itarg.get(), potsort.get(), gradsort.get(), mkz(1.0 / (2.0 * M_PI)), in.ifpgh,
           pot, grad, s);
  mark(7);
  if (timing) {
    ZF_CUDA(cudaEventSynchronize(ev[7]));
    float ms;
    for (int i = 0; i < 7; i++) {
      ZF_CUDA(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]));
      times->ms[i] = ms;
    }
    times->nboxes = S.tree.nboxes;
    times->nlevels = S.tree.nlevels;
    times->nterms = pord;
    for (auto& e : ev) cudaEventDestroy(e);
    times->launches = launch_counter() - launches0;
  }
  if (timing && times->want_counts) {
    count_interactions2d(S, plv.data(), times->counts, s);
  }
}

}  // namespace zf
