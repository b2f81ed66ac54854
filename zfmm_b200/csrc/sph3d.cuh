// Device helpers shared by the 3D FMMs: compact expansion indexing, the
// complex square root and spherical coordinates of the reference
// (zfmm3d/src/common/ztoolbox.f:110-160), translation geometry
// (zrotate.f:32-88) and the point-and-shoot y-rotation (zrotate.f:94-239)
// with one thread per sample angle.
#pragma once
#include "devmem.cuh"
#include "zcomplex.cuh"

namespace zf {

constexpr double kPi = 3.14159265358979323846;
constexpr double kF16 = (double)1e-16f;  // REAL*4 literal 1E-16 of the reference

// Per-order tables in device memory, kept for the life of the process.
struct Tab3 {
  int p, NC, NS, nmax;
  const double* r1;    // [(p+1)^2] ylgndrini rat1, (n, m) at n*(p+1)+m
  const double* r2;    // rat2
  const double* sq;    // sqrt(2n+1), n <= 2p+1
  const double* amat;  // get_amat, (n, m) at n*(2nmax+1)+m+nmax, n <= nmax = 2p
  const double* dinv;  // y-rotation projection weights, (n, |m|) at n*(p+1)+|m|
  const zdc* tw;       // exp(-2 pi i k / (2p+1)), k < 2p+1
};


// tables of order p on the current device (built on first use)
Tab3 get_tab3(int p);

__device__ __forceinline__ int nsrc(const int* se, int b) { return se[2 * b + 1] - se[2 * b] + 1; }

__device__ __forceinline__ int ix3(int n, int m) { return n * n + n + m; }

// degree n of the compact index idx = n*n + n + m
__device__ __forceinline__ int deg3(int idx) {
  int n = (int)sqrtf((float)idx);
  if (n * n > idx) n--;
  if ((n + 1) * (n + 1) <= idx) n++;
  return n;
}

// x^n for n >= 0 by binary powering
__device__ __forceinline__ double ipow(double x, int n) {
  double r = 1.0;
  while (n > 0) {
    if (n & 1) r *= x;
    x *= x;
    n >>= 1;
  }
  return r;
}

// zsqrt (ztoolbox.f:110-124): phase atan2 in (-pi, pi] with -pi taken as pi
__device__ __forceinline__ zdc zsqrt_r(zdc z2) {
  double r = sqrt(zabs(z2));
  double ph = atan2(z2.im, z2.re);
  if (ph == -kPi) ph = kPi;
  ph = ph * 0.5;
  double s, c;
  sincos(ph, &s, &c);
  return mkz(r * c, r * s);
}

struct Sph {
  zdc rz, ct, st, cp, sp, eip;
};

// zcart2sph (ztoolbox.f:132-160)
__device__ __forceinline__ Sph zcart2sph(zdc x0, zdc x1, zdc x2, const zdc* c0) {
  Sph s;
  zdc z1 = x0 - c0[0], z2 = x1 - c0[1], z3 = x2 - c0[2];
  zdc r2 = z1 * z1 + z2 * z2 + z3 * z3;
  s.rz = zsqrt_r(r2);
  s.ct = z3 / s.rz;
  zdc zrxy = zsqrt_r(z1 * z1 + z2 * z2);
  s.st = zrxy / s.rz;
  if (zabs(zrxy) <= kF16) {
    s.cp = mkz(1.0);
    s.sp = mkz(0.0);
    s.eip = mkz(1.0);
  } else {
    s.cp = z1 / zrxy;
    s.sp = z2 / zrxy;
    s.eip = s.cp + zmul_i(s.sp);
  }
  return s;
}

__device__ __forceinline__ void shfl_sum(zdc& v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += shfl_xor_z(v, o);
}

// ---- translations -----------------------------------------------------------
// rotation angles of a translation and the displacement along the rotated z
// axis (zz); the Laplace shifts use zshift = -zz, the Helmholtz shifts +zz
struct Geo {
  bool zr, yr;
  zdc cb, sb, ca, sa, zshift, zz;
};

// geometry of zl3dmpmp / zl3dmploc / zl3dlocloc (zl3dtrans.f:1-321)
__device__ __forceinline__ Geo geo3(const zdc* c0, const zdc* c) {
  Geo g;
  zdc x0 = c[0] - c0[0], x1 = c[1] - c0[1], x2 = c[2] - c0[2];
  g.cb = mkz(1.0);
  g.sb = mkz(0.0);
  g.ca = mkz(1.0);
  g.sa = mkz(0.0);
  double e2 = zabs(x1);
  g.zr = !(e2 <= kF16);
  if (g.zr) {
    zdc rxy = zsqrt_r(x0 * x0 + x1 * x1);
    g.cb = -x0 / rxy;
    g.sb = -x1 / rxy;
    x0 = -rxy;
  }
  double e1 = zabs(x0);
  g.yr = !(e1 <= kF16);
  zdc zz = x2;
  if (g.yr) {
    zdc rxz = zsqrt_r(x0 * x0 + x2 * x2);
    g.ca = x2 / rxz;
    g.sa = x0 / rxz;
    zz = rxz;
  }
  g.zshift = -zz;
  g.zz = zz;
  return g;
}

// z3dyrot sampling (zrotate.f:94-239): thread jj < 2p+1 evaluates the
// expansion `a` on the rotated meridian at angle 2 pi (jj-p)/(2p+1) and
// writes F[n][jj] for every degree n.  Legendre columns stream in registers.
// r1, r2: ylgndrini tables with row stride L >= p+1; sq[n] = sqrt(2n+1).
static __device__ void yrot_sample(int p, int L, const double* __restrict__ r1,
                                   const double* __restrict__ r2, const double* __restrict__ sq,
                                   const zdc* __restrict__ a, zdc* __restrict__ F, zdc ca,
                                   zdc sa) {
  const int NS = 2 * p + 1;
  const int jj = threadIdx.x;
  if (jj >= NS) return;
  const int j = jj - p;
  const double s4i = 1.0 / sqrt(4 * kPi);
  double ph = j * 2 * kPi / (2 * p + 1);
  double sph, cph;
  sincos(ph, &sph, &cph);
  zdc x1 = cph * ca, x2 = mkz(sph);
  zdc zrxy = zsqrt_r(x1 * x1 + x2 * x2);
  zdc ct = (-cph) * sa;
  zdc st = zsqrt_r(mkz(1.0) - (cph * cph) * (mkz(1.0) - ca * ca));
  if (ph == 0) st = (zabs(st + ca) <= zabs(st - ca)) ? -ca : ca;
  zdc cp, sp, eip;
  if (zabs(zrxy) >= kF16) {
    cp = x1 / zrxy;
    sp = x2 / zrxy;
    eip = cp + zmul_i(sp);
  } else {
    cp = mkz(1.0);
    sp = mkz(0.0);
    eip = mkz(1.0);
  }
  zdc z1 = s4i * st, z2 = (st * ca - ct * cp * sa) * s4i, z3 = zmul_i(sp * sa * s4i);
  // myzylgndr2sf (ztoolbox.f:273-327) with z = ct, stheta = st
  const zdc z = ct, zz1 = mkz(1.0) - z * z;
  const zdc u = (zabs(zz1) >= (double)1e-12f) ? -zsqrt_r(zz1) : -st;
  zdc* Fj = F + jj;
  // m = 0
  {
    zdc Ypp = mkz(1.0), Dpp = mkz(0.0), Yp = Ypp, Dp = Dpp;
    {
      zdc a0 = a[0];
      Fj[0] = a0 * (Yp * s4i) - a0 * (Dp * z2 * st);
    }
    if (p >= 1) {
      double c = __ldg(&r1[L]);
      Yp = z * Ypp * c;
      Dp = (z * Dpp + Ypp) * c;
      zdc an = a[ix3(1, 0)];
      zdc y = Yp * sq[1], d = Dp * sq[1];
      Fj[NS] = an * (y * s4i) - an * (d * z2 * st);
    }
    for (int n = 2; n <= p; n++) {
      double c1 = __ldg(&r1[n * L]), c2 = __ldg(&r2[n * L]);
      zdc Y = (c1 * z) * Yp - c2 * Ypp;
      zdc D = c1 * (z * Dp + Yp) - c2 * Dpp;
      Ypp = Yp; Dpp = Dp; Yp = Y; Dp = D;
      zdc an = a[ix3(n, 0)];
      double s = __ldg(&sq[n]);
      zdc y = Y * s, d = D * s;
      Fj[n * NS] = an * (y * s4i) - an * (d * z2 * st);
    }
  }
  zdc Ydiag = mkz(1.0), em = mkz(1.0);
  for (int m = 1; m <= p; m++) {
    double cmm = __ldg(&r1[m * L + m]);
    Ydiag = (m == 1) ? mkz(-cmm) : (Ydiag * u) * cmm;
    em = em * eip;
    zdc emi = zinv(em);
    double sg = (m & 1) ? -1.0 : 1.0;
    double dm = (double)m;
    zdc Yp = Ydiag, Dp = (Ydiag * (double)(-m)) * z;
    zdc Ypp = mkz(0.0), Dpp = mkz(0.0);
    for (int n = m; n <= p; n++) {
      zdc Y, D;
      if (n == m) {
        Y = Yp;
        D = Dp;
      } else if (n == m + 1) {
        double c = __ldg(&r1[n * L + m]);
        Y = (z * Yp) * c;
        D = (z * Dp + zz1 * Yp) * c;
        Ypp = Yp; Dpp = Dp; Yp = Y; Dp = D;
      } else {
        double c1 = __ldg(&r1[n * L + m]), c2 = __ldg(&r2[n * L + m]);
        Y = (c1 * z) * Yp - c2 * Ypp;
        D = c1 * (z * Dp + zz1 * Yp) - c2 * Dpp;
        Ypp = Yp; Dpp = Dp; Yp = Y; Dp = D;
      }
      double s = __ldg(&sq[n]);
      zdc y = Y * s, d = D * s;
      zdc z4 = a[ix3(n, m)] * em, z5 = a[ix3(n, -m)] * emi;
      zdc z6 = z4 + z5;
      zdc add = z6 * (z1 * y - z2 * d) + (dm * y) * (z3 * (z4 - z5));
      Fj[n * NS] += sg * add;
    }
  }
}

// projection of z3dyrot: out(n, m) = dinv(n,|m|) * sum_j F[n][j] e^{-i m j 2 pi/(2p+1)}
// dinv: projection weights of order pT (row stride L); dscale rescales them to
// order p (they carry the factor sqrt(4 pi)/(2p+1)); tw: the 2p+1 twiddles
template <int KMAX, int NT>
__device__ __forceinline__ void yrot_project(int p, int L, const double* __restrict__ dinv,
                                             double dscale, const zdc* __restrict__ F,
                                             zdc* __restrict__ out, const zdc* __restrict__ tw) {
  const int NS = 2 * p + 1, NC = (p + 1) * (p + 1);
#pragma unroll
  for (int k = 0; k < KMAX; k++) {
    int idx = threadIdx.x + k * NT;
    if (idx < NC) {
      int n = deg3(idx), m = idx - n * n - n;
      int step = ((m % NS) + NS) % NS;
      int kk = (int)((((long)m * (-p)) % NS + NS) % NS);
      const zdc* Fn = F + n * NS;
      zdc c0 = mkz(0.0), c1 = mkz(0.0);
      int jj = 0;
      for (; jj + 1 < NS; jj += 2) {
        c0 += Fn[jj] * tw[kk];
        kk += step;
        if (kk >= NS) kk -= NS;
        c1 += Fn[jj + 1] * tw[kk];
        kk += step;
        if (kk >= NS) kk -= NS;
      }
      if (jj < NS) c0 += Fn[jj] * tw[kk];
      out[idx] = (c0 + c1) * (__ldg(&dinv[n * L + (m < 0 ? -m : m)]) * dscale);
    }
  }
}


}  // namespace zf
