// 3D Helmholtz complex-coordinate FMM (zhfmm3d) on the device.
//
// Reference: zfmm3d/src/helmholtz/zhfmm3d.f (driver :1-249, zhfmm3dmain
// :256-600, direct sum :626-693, form/eval :699-1309), the translations of
// zfmm3d/src/helmholtz/zh3dtrans.f:1-780, h3dcommon.f, besseljs3d.f,
// h3dterms.f and hndiv_fast.f.
//
// Layout in HBM: expansions of level l have order p_l (non-increasing with
// l); box b of level l keeps (p_l+1)^2 complex coefficients, compact (n, m)
// order n*n+n+m, at base_l + (b - first box of l) * (p_l+1)^2.
//
// Kernels (one CTA per output box):
//   k_hform3   P2M / P2L: a warp per 32 sources; each lane evaluates its
//              source's scaled spherical Bessel (P2M) or Hankel (P2L) table
//              and streams the Legendre recurrences, the warp reduces every
//              coefficient by shuffles into a per-warp partial expansion.
//   k_htrans3  M2M / M2L / L2L: z-rotation, point-and-shoot y-rotation (one
//              thread per sample angle), the reference's quadrature z-shift,
//              inverse rotations.  The z-shift evaluates the rotated
//              expansion and its normal derivative at nquad = 2.5 p2
//              Gauss-Legendre points of a sphere about the new centre, in
//              chunks of C points: one thread per point computes the radial
//              table, one thread per (point, order m) sums the Legendre
//              column and tabulates the projection column at the real node;
//              one thread per output coefficient then projects with the
//              value/derivative weights g_n / ((g_n^2 + g_n'^2) / 2 pi).
//              Output coefficients accumulate in registers.  Orders whose
//              working arrays exceed shared memory run the same code on a
//              per-CTA workspace in global memory (L2-resident).
//   k_heval3   L2T and M2T: a thread per target.
//   k_hp2p3    list-1 direct interactions with sources staged in shared memory.
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>
#include "helm3d_pair.cuh"
#include "helm3d_special.cuh"
#include "hfmm3d.cuh"
#include "lfmm3d.cuh"
#include "helm3d_prep.cuh"
#include "plan3d.cuh"
#include "sph3d.cuh"

namespace zf {
namespace {

constexpr int HNT = 256;     // threads of the translation kernel
constexpr int HFNT = 128;    // threads of the form kernel (at most)
constexpr int HENT = 128;    // threads of the eval / P2P kernels
constexpr int HPTILE = 128;  // sources per P2P tile
constexpr size_t kSmemMax = 227 * 1024;
constexpr int kGmemCtas = 2 * 148;  // CTAs of the global-workspace variant

// ---- translation kernel ------------------------------------------------------
struct HTransArgs {
  const double *r1, *r2, *sq, *dinv;
  int L, pT;  // tables of order pT, row stride L = pT+1
  const int *ilevel, *iparent, *nchild, *ichild, *isrcse, *itargse;
  const zdc *zcs, *zct;
  HLev lev;
  const ShiftTab* st;  // indexed by the output box's level
  const zdc* in;
  zdc* out;
  const int *nl2, *l2, *nl4;
  int mn2;
  int lo, hi;
  zdc kwave;
  int C, pbuf;
};

struct HSm {
  zdc *sA, *sB, *U, *sEf, *sEb, *sTw1, *sTw2, *sNode;
};

__host__ __device__ inline size_t htrans_layout(int pbuf, int C, zdc* base, HSm* o) {
  size_t NCb = (size_t)(pbuf + 1) * (pbuf + 1), NSb = 2 * pbuf + 1;
  size_t rot = (size_t)(pbuf + 1) * NSb;
  size_t ycd = ((size_t)C * (pbuf + 1) * (pbuf + 2) / 2 + 1) / 2;  // doubles -> zdc
  size_t zsh = 2 * (size_t)C * (pbuf + 2) + 2 * (size_t)C * NSb + ycd;
  size_t U = rot > zsh ? rot : zsh;
  size_t off = 0;
  auto take = [&](size_t n) {
    zdc* p = base ? base + off : nullptr;
    off += n;
    return p;
  };
  HSm s;
  s.sA = take(NCb);
  s.sB = take(NCb);
  s.U = take(U);
  s.sEf = take(NSb);
  s.sEb = take(NSb);
  s.sTw1 = take(NSb);
  s.sTw2 = take(NSb);
  s.sNode = take(6 * (size_t)C);
  if (o) *o = s;
  return off * sizeof(zdc);
}

// KIND 0: M2M into parent box, 1: M2L into target box, 2: L2L into child box.
// GMEM: the working arrays live in a per-CTA slice of `scratch` (global
// memory) instead of shared memory; the grid loops over the boxes.
template <int KIND, int KMAX, bool GMEM>
__global__ void __launch_bounds__(HNT, 1) k_htrans3(HTransArgs A, zdc* scratch, size_t per_cta) {
  extern __shared__ zdc sm[];
  const int tid = threadIdx.x;
  HSm S;
  htrans_layout(A.pbuf, A.C, GMEM ? scratch + blockIdx.x * per_cta : sm, &S);
  const double s4i = 1.0 / sqrt(4 * kPi);
  for (int b = A.lo + blockIdx.x; b <= A.hi; b += gridDim.x) {
    __syncthreads();
    int nin = 0, par = -1;
    if (KIND == 0) {
      if (nsrc(A.isrcse, b) <= 0 || A.nchild[b] == 0) continue;
      nin = A.nchild[b];
    } else if (KIND == 1) {
      if (nsrc(A.itargse, b) <= 0 || A.nl2[b] == 0) continue;
      nin = A.nl2[b];
    } else {
      par = A.iparent[b];
      // zhfmm3d.f:572-576: ((targets and list 2) or list 4) of the parent,
      // and targets in the child
      if (par < 0 || nsrc(A.itargse, b) <= 0) continue;
      if (!((nsrc(A.itargse, par) > 0 && A.nl2[par] > 0) || A.nl4[par] > 0)) continue;
      nin = 1;
    }
    const int lb = A.ilevel[b];
    const int l1 = KIND == 0 ? lb + 1 : (KIND == 1 ? lb : lb - 1), l2 = lb;
    const int p1 = A.lev.p[l1], p2 = A.lev.p[l2];
    const int NC1 = (p1 + 1) * (p1 + 1), NC2 = (p2 + 1) * (p2 + 1);
    const int NS1 = 2 * p1 + 1, NS2 = 2 * p2 + 1, NSb = 2 * A.pbuf + 1;
    const ShiftTab ST = A.st[lb];
    for (int k = tid; k < NS1; k += HNT) {
      double s, c;
      sincospi(2.0 * k / NS1, &s, &c);
      S.sTw1[k] = mkz(c, -s);
    }
    for (int k = tid; k < NS2; k += HNT) {
      double s, c;
      sincospi(2.0 * k / NS2, &s, &c);
      S.sTw2[k] = mkz(c, -s);
    }
    zdc acc[KMAX];
#pragma unroll
    for (int k = 0; k < KMAX; k++) acc[k] = mkz(0.0);
    const zdc* inbase = A.in + A.lev.base[l1];
    for (int it = 0; it < nin; it++) {
      int src;
      const zdc *c0, *c;
      if (KIND == 0) {
        src = A.ichild[8 * b + it];
        if (nsrc(A.isrcse, src) <= 0) continue;
        c0 = A.zcs + 3 * src;
        c = A.zcs + 3 * b;
      } else if (KIND == 1) {
        src = A.l2[(size_t)b * A.mn2 + it];
        if (nsrc(A.isrcse, src) <= 0) continue;
        c0 = A.zcs + 3 * src;
        c = A.zct + 3 * b;
      } else {
        src = par;
        c0 = A.zct + 3 * par;
        c = A.zct + 3 * b;
      }
      Geo g = geo3(c0, c);
      const zdc zsh = g.zz;  // zh3dtrans.f: zshift = xc2(3)
      __syncthreads();
      for (int m = tid; m <= p1; m += HNT) {
        zdc ef = zpown(g.cb + zmul_i(g.sb), m);
        S.sEf[p1 + m] = ef;
        S.sEf[p1 - m] = zinv(ef);
      }
      for (int m = tid; m <= p2; m += HNT) {
        zdc eb = zpown(g.cb - zmul_i(g.sb), m);
        S.sEb[p2 + m] = eb;
        S.sEb[p2 - m] = zinv(eb);
      }
      __syncthreads();
      const zdc* __restrict__ ain = inbase + (size_t)(src - A.lev.lo[l1]) * NC1;
      for (int idx = tid; idx < NC1; idx += HNT) {
        zdc v = ain[idx];
        int n = deg3(idx);
        S.sA[idx] = g.zr ? v * S.sEf[p1 + idx - n * n - n] : v;
      }
      __syncthreads();
      zdc* cur = S.sA;
      zdc* oth = S.sB;
      if (g.yr) {
        yrot_sample(p1, A.L, A.r1, A.r2, A.sq, cur, S.U, g.ca, g.sa);
        __syncthreads();
        yrot_project<KMAX, HNT>(p1, A.L, A.dinv, (2.0 * A.pT + 1.0) / (2.0 * p1 + 1.0), S.U,
                                oth, S.sTw1);
        __syncthreads();
        zdc* t = cur; cur = oth; oth = t;
      }
      // ---- quadrature z-shift: cur (order p1) -> accF/accD (order p2) ----
      zdc accF[KMAX], accD[KMAX];
#pragma unroll
      for (int k = 0; k < KMAX; k++) accF[k] = accD[k] = mkz(0.0);
      const int C = A.C, P2 = A.pbuf + 2;
      zdc* rad = S.U;
      zdc* drad = rad + (size_t)C * P2;
      zdc* Fq = drad + (size_t)C * P2;
      zdc* DFq = Fq + (size_t)C * NSb;
      double* Yc = (double*)(DFq + (size_t)C * NSb);
      const int nY = (p2 + 1) * (p2 + 2) / 2;
      const int ncol = (p1 > p2 ? p1 : p2) + 1;
      for (int q0 = 0; q0 < ST.nq; q0 += C) {
        const int nc = min(C, ST.nq - q0);
        // (a) node geometry and radial tables, one thread per node
        for (int t = tid; t < nc; t += HNT) {
          double x = __ldg(&ST.x[q0 + t]);
          double yi = sqrt(1 - x * x);
          zdc zi = zsh + mkz(ST.r * x);
          zdc ri = zsqrt_r(mkz((ST.r * yi) * (ST.r * yi)) + zi * zi);
          zdc cthi = zi / ri;
          zdc sthi = zsqrt_r(mkz(1.0) - cthi * cthi);
          zdc* nd = S.sNode + 6 * t;
          nd[0] = cthi;
          nd[1] = sthi;
          nd[2] = cthi / ri;
          nd[3] = sthi / ri;
          nd[4] = mkz(yi);
          nd[5] = mkz(x);
          zdc zk = ri * A.kwave;
          zdc* f = rad + (size_t)t * P2;
          zdc* fd = drad + (size_t)t * P2;
          if (KIND == 2) besseljs3d_z(p1, zk, ST.rs1, f, fd);
          else h3dall_z(p1, zk, ST.rs1, f, fd);
          for (int n = 0; n <= p1; n++) fd[n] = A.kwave * fd[n];
        }
        __syncthreads();
        // (b) one thread per (node, order m): the node's value and normal
        // derivative sums of order m, and the projection Legendre column
        for (int item = tid; item < nc * ncol; item += HNT) {
          const int t = item / ncol, m = item - t * ncol;
          const zdc* nd = S.sNode + 6 * t;
          const double x = nd[5].re, yi = nd[4].re;
          zdc* Ft = Fq + (size_t)t * NSb + A.pbuf;
          zdc* Dt = DFq + (size_t)t * NSb + A.pbuf;
          if (m <= p1) {
            const zdc z = nd[0], sthi = nd[1], cr = nd[2], sr = nd[3];
            const zdc zz1 = mkz(1.0) - z * z;
            const zdc u = -zsqrt_r(zz1);
            const zdc* f = rad + (size_t)t * P2;
            const zdc* fd = drad + (size_t)t * P2;
            const double sgm = ((m & 1) ? -1.0 : 1.0) * s4i;
            zdc Ydiag = mkz(1.0);
            for (int k = 1; k <= m; k++) {
              double ckk = __ldg(&A.r1[k * A.L + k]);
              Ydiag = (k == 1) ? mkz(-ckk) : (Ydiag * u) * ckk;
            }
            zdc Yp = Ydiag, Dp = (Ydiag * (double)(-m)) * z, Ypp = mkz(0.0), Dpp = mkz(0.0);
            zdc F0 = mkz(0.0), F1 = mkz(0.0), D0 = mkz(0.0), D1 = mkz(0.0);
            for (int n = m; n <= p1; n++) {
              zdc Y, D;
              if (n == m) {
                Y = Yp;
                D = Dp;
              } else {
                if (n == m + 1) {
                  double cc = __ldg(&A.r1[n * A.L + m]);
                  Y = (z * Yp) * cc;
                  D = (m == 0) ? (z * Dp + Yp) * cc : (z * Dp + zz1 * Yp) * cc;
                } else {
                  double c1 = __ldg(&A.r1[n * A.L + m]), c2 = __ldg(&A.r2[n * A.L + m]);
                  Y = (c1 * z) * Yp - c2 * Ypp;
                  D = (m == 0) ? c1 * (z * Dp + Yp) - c2 * Dpp
                               : c1 * (z * Dp + zz1 * Yp) - c2 * Dpp;
                }
                Ypp = Yp; Dpp = Dp; Yp = Y; Dp = D;
              }
              double sc = __ldg(&A.sq[n]) * sgm;
              zdc yl = Y * sc, dyl = D * sc;
              zdc fn = f[n], fdn = fd[n];
              zdc df_r, df_th, z1;
              if (m == 0) {
                z1 = fn * yl;
                df_r = fdn * yl;
                df_th = -(fn * dyl * sthi);
              } else {
                z1 = fn * yl * sthi;
                df_r = fdn * yl * sthi;
                df_th = -(fn * dyl);
              }
              zdc df_x = df_r * sthi + df_th * cr;
              zdc df_y = df_r * z - df_th * sr;
              zdc df = df_x * yi + df_y * x;
              zdc ap = cur[ix3(n, m)];
              F0 += ap * z1;
              D0 += ap * df;
              if (m > 0) {
                zdc am = cur[ix3(n, -m)];
                F1 += am * z1;
                D1 += am * df;
              }
            }
            Ft[m] = F0;
            Dt[m] = D0;
            if (m > 0) {
              Ft[-m] = F1;
              Dt[-m] = D1;
            }
          } else {
            Ft[m] = Ft[-m] = Dt[m] = Dt[-m] = mkz(0.0);
          }
          if (m <= p2) {
            // zylgndrf at the real node x, times (-1)^m / sqrt(4 pi) and the weight
            const double w = __ldg(&ST.w[q0 + t]) * ((m & 1) ? -1.0 : 1.0) * s4i;
            const double u = -sqrt(1 - x * x);
            double yd = 1.0;
            for (int k = 1; k <= m; k++) yd = (yd * u) * __ldg(&A.r1[k * A.L + k]);
            double yp = yd, ypp = 0.0;
            double* Yt = Yc + (size_t)t * nY;
            for (int n = m; n <= p2; n++) {
              double y;
              if (n == m) {
                y = yp;
              } else if (n == m + 1) {
                y = (x * yp) * __ldg(&A.r1[n * A.L + m]);
                ypp = yp;
                yp = y;
              } else {
                y = (__ldg(&A.r1[n * A.L + m]) * x) * yp - __ldg(&A.r2[n * A.L + m]) * ypp;
                ypp = yp;
                yp = y;
              }
              Yt[jdx(n, m)] = y * __ldg(&A.sq[n]) * w;
            }
          }
        }
        __syncthreads();
        // (c) projection onto the order-p2 coefficients
#pragma unroll
        for (int k = 0; k < KMAX; k++) {
          int idx = tid + k * HNT;
          if (idx < NC2) {
            int n = deg3(idx), m = idx - n * n - n, am = m < 0 ? -m : m;
            int j = jdx(n, am);
            zdc sF = accF[k], sD = accD[k];
            for (int t = 0; t < nc; t++) {
              double y = Yc[(size_t)t * nY + j];
              sF += y * Fq[(size_t)t * NSb + A.pbuf + m];
              sD += y * DFq[(size_t)t * NSb + A.pbuf + m];
            }
            accF[k] = sF;
            accD[k] = sD;
          }
        }
        __syncthreads();
      }
#pragma unroll
      for (int k = 0; k < KMAX; k++) {
        int idx = tid + k * HNT;
        if (idx < NC2) {
          int n = deg3(idx);
          oth[idx] = ST.cF[n] * accF[k] + ST.cD[n] * accD[k];
        }
      }
      __syncthreads();
      {
        zdc* t = cur; cur = oth; oth = t;
      }
      if (g.yr) {
        yrot_sample(p2, A.L, A.r1, A.r2, A.sq, cur, S.U, g.ca, -g.sa);
        __syncthreads();
        yrot_project<KMAX, HNT>(p2, A.L, A.dinv, (2.0 * A.pT + 1.0) / (2.0 * p2 + 1.0), S.U,
                                oth, S.sTw2);
        __syncthreads();
        zdc* t = cur; cur = oth; oth = t;
      }
#pragma unroll
      for (int k = 0; k < KMAX; k++) {
        int idx = tid + k * HNT;
        if (idx < NC2) {
          int n = deg3(idx);
          acc[k] += g.zr ? cur[idx] * S.sEb[p2 + idx - n * n - n] : cur[idx];
        }
      }
    }
    zdc* o = A.out + A.lev.base[l2] + (size_t)(b - A.lev.lo[l2]) * NC2;
#pragma unroll
    for (int k = 0; k < KMAX; k++) {
      int idx = tid + k * HNT;
      if (idx < NC2) {
        if (KIND == 2) o[idx] += acc[k];
        else o[idx] = acc[k];
      }
    }
  }
}

// ---- P2M / P2L ------------------------------------------------------------
struct HFormArgs {
  const double *r1, *r2, *sq;
  int L;
  const int *ilevel, *nchild, *isrcse, *itargse;
  const zdc *zsrc, *charge, *dipstr, *dipvec;
  const zdc *zcs, *zct;
  HLev lev;
  zdc* out;
  const int *nl4, *l4;
  int mn4, nb, ifcharge, ifdipole, pbuf;
  zdc zk;
};

// zh3dformmp (LOCAL = false: j_n) / zh3dformloc (LOCAL = true: h_n)
template <bool LOCAL, bool DIP>
__device__ void hform_range(const HFormArgs& A, int s0, int s1, const zdc* zc, int p,
                            double rscale, zdc* part) {
  const int L = A.L, lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const zdc c4 = zmul_i(A.zk * (1.0 / (4 * kPi)));
  zdc f[PMAXR + 2], fd[DIP ? PMAXR + 2 : 1];
  for (int base = s0 + 32 * w; base <= s1; base += 32 * nw) {
    int i = base + lane;
    bool valid = i <= s1;
    int ii = valid ? i : base;
    zdc q = (valid && A.ifcharge) ? A.charge[ii] : mkz(0.0);
    zdc ds = (valid && DIP) ? A.dipstr[ii] : mkz(0.0);
    Sph s = zcart2sph(A.zsrc[3 * ii], A.zsrc[3 * ii + 1], A.zsrc[3 * ii + 2], zc);
    zdc zrk = s.rz * A.zk;
    if (!LOCAL) besseljs3d_z(p, zrk, rscale, f, DIP ? fd : nullptr);
    else h3dall_z(p, zrk, rscale, f, DIP ? fd : nullptr);
    zdc dzr_ = mkz(0.0), dthz = mkz(0.0), dphz = mkz(0.0);
    if (DIP) {
      zdc v0 = A.dipvec[3 * ii], v1 = A.dipvec[3 * ii + 1], v2 = A.dipvec[3 * ii + 2];
      dzr_ = v0 * (s.st * s.cp) + v1 * (s.st * s.sp) + v2 * s.ct;
      zdc dth_ = v0 * (s.ct * s.cp) + v1 * (s.ct * s.sp) - v2 * s.st;
      zdc dph_ = -(v0 * s.sp) + v1 * s.cp;
      dthz = dth_ / s.rz;
      dphz = dph_ / s.rz;
    }
    const zdc z = s.ct, zz1 = mkz(1.0) - z * z;
    const zdc u = -zsqrt_r(zz1);
    zdc Ydiag = mkz(1.0), em = mkz(1.0);
    for (int m = 0; m <= p; m++) {
      zdc emi = mkz(1.0);
      if (m > 0) {
        double cmm = __ldg(&A.r1[m * L + m]);
        if (DIP) Ydiag = (m == 1) ? mkz(-cmm) : (Ydiag * u) * cmm;
        else Ydiag = (Ydiag * u) * cmm;
        em = em * s.eip;
        emi = zinv(em);
      }
      double sgm = (m & 1) ? -1.0 : 1.0;
      zdc Yp = Ydiag, Dp = DIP ? (Ydiag * (double)(-m)) * z : mkz(0.0);
      zdc Ypp = mkz(0.0), Dpp = mkz(0.0);
      for (int n = m; n <= p; n++) {
        zdc Y, D = mkz(0.0);
        if (n == m) {
          Y = Yp;
          D = Dp;
        } else {
          if (n == m + 1) {
            double c = __ldg(&A.r1[n * L + m]);
            Y = (z * Yp) * c;
            if (DIP) D = (m == 0) ? (z * Dp + Yp) * c : (z * Dp + zz1 * Yp) * c;
          } else {
            double c1 = __ldg(&A.r1[n * L + m]), c2 = __ldg(&A.r2[n * L + m]);
            Y = (c1 * z) * Yp - c2 * Ypp;
            if (DIP) D = (m == 0) ? c1 * (z * Dp + Yp) - c2 * Dpp : c1 * (z * Dp + zz1 * Yp) - c2 * Dpp;
          }
          Ypp = Yp; Dpp = Dp; Yp = Y; Dp = D;
        }
        zdc sc = c4 * (__ldg(&A.sq[n]) * sgm);
        zdc y = Y * sc, dy = D * sc;
        zdc cpos, cneg;
        if (m == 0) {
          zdc c0 = q * f[n] * y;
          if (DIP) c0 += -(ds * A.zk * fd[n] * y * dzr_) + ds * f[n] * dy * s.st * dthz;
          cpos = c0;
          cneg = mkz(0.0);
        } else {
          zdc X = q * f[n] * (DIP ? y * s.st : y), W = mkz(0.0);
          if (DIP) {
            X += -(ds * A.zk * fd[n] * y * s.st * dzr_) + ds * f[n] * dy * dthz;
            W = ds * zmul_i((double)m * f[n] * y * dphz);
          }
          cpos = emi * (X + W);
          cneg = em * (X - W);
        }
        shfl_sum(cpos);
        if (m > 0) shfl_sum(cneg);
        if (lane == 0) {
          part[ix3(n, m)] += cpos;
          if (m > 0) part[ix3(n, -m)] += cneg;
        }
      }
    }
  }
}

template <bool LOCAL, bool DIP>
__global__ void __launch_bounds__(HFNT) k_hform3(HFormArgs A) {
  extern __shared__ zdc sm[];
  const int tid = threadIdx.x, w = tid >> 5, nw = blockDim.x >> 5, nthr = blockDim.x;
  const int b = blockIdx.x;
  if (b >= A.nb) return;
  int l = A.ilevel[b];
  if (!LOCAL) {
    if (A.nchild[b] != 0 || nsrc(A.isrcse, b) <= 0 || l < 2) return;
  } else {
    if (nsrc(A.itargse, b) <= 0 || A.nl4[b] == 0) return;
  }
  const int p = A.lev.p[l], NC = (p + 1) * (p + 1), NCb = (A.pbuf + 1) * (A.pbuf + 1);
  zdc* part = sm + w * NCb;
  for (int k = tid; k < nw * NCb; k += nthr) sm[k] = mkz(0.0);
  __syncthreads();
  if (!LOCAL) {
    hform_range<false, DIP>(A, A.isrcse[2 * b], A.isrcse[2 * b + 1], A.zcs + 3 * b, p,
                            A.lev.rs[l], part);
  } else {
    for (int i = 0; i < A.nl4[b]; i++) {
      int jb = A.l4[(size_t)b * A.mn4 + i];
      if (nsrc(A.isrcse, jb) <= 0) continue;
      hform_range<true, DIP>(A, A.isrcse[2 * jb], A.isrcse[2 * jb + 1], A.zct + 3 * b, p,
                             A.lev.rs[l], part);
    }
  }
  __syncthreads();
  zdc* o = A.out + A.lev.base[l] + (size_t)(b - A.lev.lo[l]) * NC;
  for (int k = tid; k < NC; k += nthr) {
    zdc v = sm[k];
    for (int ww = 1; ww < nw; ww++) v += sm[ww * NCb + k];
    if (LOCAL) o[k] += v;
    else o[k] = v;
  }
}

// ---- L2T / M2T --------------------------------------------------------------
struct HEvalArgs {
  const double *r1, *r2, *sq;
  int L;
  const int *ilevel, *nchild, *isrcse, *itargse;
  const zdc *ztarg, *zcs, *zct;
  HLev lev;
  const zdc *mp, *loc;
  const int *nl3, *l3;
  int mn3, nb, pbuf;
  zdc zk;
  zdc *pot, *grad;
};

// zh3devalmp (LOCAL = false: h_n) / zh3devalloc (LOCAL = true: j_n); the
// gradient is accumulated in spherical components and mapped once
template <bool GRAD, bool LOCAL>
__device__ __forceinline__ void heval_one(const HEvalArgs& A, const zdc* __restrict__ e, int p,
                                          const zdc* x, const zdc* zc, double rscale, zdc& pot,
                                          zdc* grad) {
  const int L = A.L;
  zdc f[PMAXR + 2], fd[GRAD ? PMAXR + 2 : 1];
  Sph s = zcart2sph(x[0], x[1], x[2], zc);
  zdc zrk = s.rz * A.zk;
  if (!LOCAL) h3dall_z(p, zrk, rscale, f, GRAD ? fd : nullptr);
  else besseljs3d_z(p, zrk, rscale, f, GRAD ? fd : nullptr);
  const zdc z = s.ct, zz1 = mkz(1.0) - z * z;
  const zdc u = -zsqrt_r(zz1);
  zdc P = mkz(0.0), Gr = mkz(0.0), Gt = mkz(0.0), Gp = mkz(0.0);
  zdc Ydiag = mkz(1.0), em = mkz(1.0);
  for (int m = 0; m <= p; m++) {
    zdc emi = mkz(1.0);
    if (m > 0) {
      double cmm = __ldg(&A.r1[m * L + m]);
      if (GRAD) Ydiag = (m == 1) ? mkz(-cmm) : (Ydiag * u) * cmm;
      else Ydiag = (Ydiag * u) * cmm;
      em = em * s.eip;
      emi = zinv(em);
    }
    double sgm = (m & 1) ? -1.0 : 1.0;
    zdc Yp = Ydiag, Dp = GRAD ? (Ydiag * (double)(-m)) * z : mkz(0.0);
    zdc Ypp = mkz(0.0), Dpp = mkz(0.0);
    for (int n = m; n <= p; n++) {
      zdc Y, D = mkz(0.0);
      if (n == m) {
        Y = Yp;
        D = Dp;
      } else {
        if (n == m + 1) {
          double c = __ldg(&A.r1[n * L + m]);
          Y = (z * Yp) * c;
          if (GRAD) D = (m == 0) ? (z * Dp + Yp) * c : (z * Dp + zz1 * Yp) * c;
        } else {
          double c1 = __ldg(&A.r1[n * L + m]), c2 = __ldg(&A.r2[n * L + m]);
          Y = (c1 * z) * Yp - c2 * Ypp;
          if (GRAD) D = (m == 0) ? c1 * (z * Dp + Yp) - c2 * Dpp : c1 * (z * Dp + zz1 * Yp) - c2 * Dpp;
        }
        Ypp = Yp; Dpp = Dp; Yp = Y; Dp = D;
      }
      double sc = __ldg(&A.sq[n]) * sgm;
      zdc y = Y * sc;
      if (m == 0) {
        zdc a0 = e[ix3(n, 0)];
        P += a0 * f[n] * y;
        if (GRAD) {
          zdc dy = D * sc;
          Gr += a0 * (A.zk * fd[n] * y);
          Gt -= a0 * (f[n] * dy * s.st);
        }
      } else {
        zdc z1 = e[ix3(n, m)] * em, z2 = e[ix3(n, -m)] * emi;
        zdc Sp = z1 + z2;
        P += (GRAD ? f[n] * y * s.st : f[n] * y) * Sp;
        if (GRAD) {
          zdc dy = D * sc;
          Gr += (A.zk * fd[n] * y * s.st) * Sp;
          Gt -= (f[n] * dy) * Sp;
          Gp += zmul_i((double)m * f[n] * y) * (z1 - z2);
        }
      }
    }
  }
  pot += P;
  if (GRAD) {
    zdc ir = zinv(s.rz);
    zdc ezr0 = s.st * s.cp, ezr1 = s.st * s.sp, ezr2 = s.ct;
    zdc et0 = s.ct * s.cp * ir, et1 = s.ct * s.sp * ir, et2 = -(s.st * ir);
    zdc ep0 = -(s.sp * ir), ep1 = s.cp * ir;
    grad[0] += Gr * ezr0 + Gt * et0 + Gp * ep0;
    grad[1] += Gr * ezr1 + Gt * et1 + Gp * ep1;
    grad[2] += Gr * ezr2 + Gt * et2;
  }
}

template <bool GRAD>
__global__ void __launch_bounds__(HENT) k_heval3(HEvalArgs A) {
  extern __shared__ zdc sm[];
  const int tid = threadIdx.x;
  const int b = blockIdx.x;
  if (b >= A.nb) return;
  const int t0 = A.itargse[2 * b], t1 = A.itargse[2 * b + 1];
  if (A.nchild[b] != 0 || t1 < t0) return;
  const int lb = A.ilevel[b];
  const bool own = lb >= 2;  // levels 0 and 1 receive no local expansion
  int nexp = (own ? 1 : 0) + A.nl3[b];
  if (nexp == 0) return;
  for (int c0 = t0; c0 <= t1; c0 += HENT) {
    int i = c0 + tid;
    bool valid = i <= t1;
    zdc x[3] = {mkz(0.0), mkz(0.0), mkz(0.0)};
    if (valid) {
      x[0] = A.ztarg[3 * i];
      x[1] = A.ztarg[3 * i + 1];
      x[2] = A.ztarg[3 * i + 2];
    }
    zdc pot = mkz(0.0), g[3] = {mkz(0.0), mkz(0.0), mkz(0.0)};
    for (int e = 0; e < nexp; e++) {
      int eb;
      bool loc;
      if (own && e == 0) {
        eb = b;
        loc = true;
      } else {
        eb = A.l3[(size_t)b * A.mn3 + e - (own ? 1 : 0)];
        loc = false;
        if (nsrc(A.isrcse, eb) <= 0) continue;
      }
      const int le = A.ilevel[eb], p = A.lev.p[le], NC = (p + 1) * (p + 1);
      __syncthreads();
      const zdc* src = (loc ? A.loc : A.mp) + A.lev.base[le] + (size_t)(eb - A.lev.lo[le]) * NC;
      for (int k = tid; k < NC; k += HENT) sm[k] = src[k];
      __syncthreads();
      if (valid) {
        if (loc) heval_one<GRAD, true>(A, sm, p, x, A.zct + 3 * eb, A.lev.rs[le], pot, g);
        else heval_one<GRAD, false>(A, sm, p, x, A.zcs + 3 * eb, A.lev.rs[le], pot, g);
      }
    }
    if (valid) {
      A.pot[i] += pot;
      if (GRAD) {
        A.grad[3 * i] += g[0];
        A.grad[3 * i + 1] += g[1];
        A.grad[3 * i + 2] += g[2];
      }
    }
  }
}

// ---- P2P (list 1) and the direct sum -----------------------------------------
struct HSrcTile {
  zdc y[HPTILE][3];
  zdc q[HPTILE], ds[HPTILE];
  zdc v[HPTILE][3];
};

__device__ __forceinline__ void hstage(HSrcTile& S, int j0, int n, const zdc* zsrc,
                                       const zdc* charge, const zdc* dipstr, const zdc* dipvec,
                                       int ifcharge, int ifdipole) {
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    int j = j0 + k;
    S.y[k][0] = ldz(&zsrc[3 * j]);
    S.y[k][1] = ldz(&zsrc[3 * j + 1]);
    S.y[k][2] = ldz(&zsrc[3 * j + 2]);
    S.q[k] = ifcharge ? ldz(&charge[j]) : mkz(0.0);
    if (ifdipole) {
      S.ds[k] = ldz(&dipstr[j]);
      S.v[k][0] = ldz(&dipvec[3 * j]);
      S.v[k][1] = ldz(&dipvec[3 * j + 1]);
      S.v[k][2] = ldz(&dipvec[3 * j + 2]);
    }
  }
}

struct HP2PArgs {
  const int *nchild, *isrcse, *itargse;
  const zdc *zsrc, *charge, *dipstr, *dipvec, *ztarg;
  const int *nl1, *l1;
  int mn1, nb, ifcharge, ifdipole;
  zdc zk;
  zdc *pot, *grad;
};

template <bool GRAD>
__global__ void __launch_bounds__(HENT) k_hp2p3(HP2PArgs A) {
  __shared__ HSrcTile S;
  const int b = blockIdx.x;
  if (b >= A.nb) return;
  const int t0 = A.itargse[2 * b], t1 = A.itargse[2 * b + 1];
  if (A.nchild[b] != 0 || t1 < t0 || A.nl1[b] == 0) return;
  for (int c0 = t0; c0 <= t1; c0 += HENT) {
    int i = c0 + threadIdx.x;
    bool valid = i <= t1;
    zdc x[3] = {mkz(0.0), mkz(0.0), mkz(0.0)};
    if (valid) {
      x[0] = ldz(&A.ztarg[3 * i]);
      x[1] = ldz(&A.ztarg[3 * i + 1]);
      x[2] = ldz(&A.ztarg[3 * i + 2]);
    }
    zdc pot = mkz(0.0), g[3] = {mkz(0.0), mkz(0.0), mkz(0.0)};
    for (int li = 0; li < A.nl1[b]; li++) {
      int jb = A.l1[(size_t)b * A.mn1 + li];
      int s0 = A.isrcse[2 * jb], s1 = A.isrcse[2 * jb + 1];
      for (int j0 = s0; j0 <= s1; j0 += HPTILE) {
        int n = min(HPTILE, s1 - j0 + 1);
        __syncthreads();
        hstage(S, j0, n, A.zsrc, A.charge, A.dipstr, A.dipvec, A.ifcharge, A.ifdipole);
        __syncthreads();
        if (valid)
          for (int k = 0; k < n; k++)
            helm3d_pair<GRAD>(A.zk, x, S.y[k], S.q[k], S.ds[k], S.v[k], A.ifcharge, A.ifdipole,
                              pot, g);
      }
    }
    if (valid) {
      A.pot[i] += pot;
      if (GRAD) {
        A.grad[3 * i] += g[0];
        A.grad[3 * i + 1] += g[1];
        A.grad[3 * i + 2] += g[2];
      }
    }
  }
}

template <bool GRAD>
__global__ void __launch_bounds__(HENT) k_hdirect3d(Inputs3D in, zdc zk, int chunk, zdc* pot,
                                                    zdc* grad, zdc* part) {
  __shared__ HSrcTile S;
  int i = blockIdx.x * HENT + threadIdx.x;
  int j0 = blockIdx.y * chunk, j1 = min(in.ns, j0 + chunk);
  bool valid = i < in.nt;
  zdc x[3] = {mkz(0.0), mkz(0.0), mkz(0.0)};
  if (valid) {
    x[0] = ldz(&in.ztarg[3 * i]);
    x[1] = ldz(&in.ztarg[3 * i + 1]);
    x[2] = ldz(&in.ztarg[3 * i + 2]);
  }
  zdc p = mkz(0.0), g[3] = {mkz(0.0), mkz(0.0), mkz(0.0)};
  for (int t = j0; t < j1; t += HPTILE) {
    int n = min(HPTILE, j1 - t);
    __syncthreads();
    hstage(S, t, n, in.zsrc, in.charge, in.dipstr, in.dipvec, in.ifcharge, in.ifdipole);
    __syncthreads();
    if (valid)
      for (int k = 0; k < n; k++)
        helm3d_pair<GRAD>(zk, x, S.y[k], S.q[k], S.ds[k], S.v[k], in.ifcharge, in.ifdipole, p, g);
  }
  if (!valid) return;
  if (part == nullptr) {
    pot[i] += p;
    if (GRAD)
      for (int d = 0; d < 3; d++) grad[3 * i + d] += g[d];
  } else {
    size_t st = (size_t)in.nt * (GRAD ? 4 : 1);
    zdc* q = part + blockIdx.y * st;
    q[i] = p;
    if (GRAD)
      for (int d = 0; d < 3; d++) q[(size_t)(d + 1) * in.nt + i] = g[d];
  }
}

template <bool GRAD>
__global__ void k_hdirect3d_reduce(int nt, int nsplit, const zdc* part, zdc* pot, zdc* grad) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nt) return;
  size_t st = (size_t)nt * (GRAD ? 4 : 1);
  zdc p = mkz(0.0), g[3] = {mkz(0.0), mkz(0.0), mkz(0.0)};
  for (int k = 0; k < nsplit; k++) {
    const zdc* q = part + k * st;
    p += q[i];
    if (GRAD)
      for (int d = 0; d < 3; d++) g[d] += q[(size_t)(d + 1) * nt + i];
  }
  pot[i] += p;
  if (GRAD)
    for (int d = 0; d < 3; d++) grad[3 * i + d] += g[d];
}

// ---- host helpers -------------------------------------------------------------
// besseljs3d for the host, any order (h3dterms runs it to order 5000); fd is
// filled when non-null
void besseljs3d_host(int n, zdc z, double scale, std::vector<zdc>& f, std::vector<zdc>* fd) {
  const double up2 = 1.0e40, up2inv = 1.0e-40;
  f.assign(n + 1, mkz(0.0));
  if (fd) fd->assign(n + 1, mkz(0.0));
  if (zabs(z) < 1.0e-200) {
    f[0] = mkz(1.0);
    if (fd && n >= 1) (*fd)[1] = mkz(1.0 / (3 * scale));
    return;
  }
  zdc zi = zinv(z), fm1 = mkz(0.0), f0 = mkz(1.0);
  int ntop = n + 100000;
  for (int i = n; i <= n + 100000; i++) {
    zdc f1 = ((2 * i + 1.0) * zi) * f0 - fm1;
    double a = zabs(f1);
    if (a * a > up2) {
      ntop = i + 1;
      break;
    }
    fm1 = f0;
    f0 = f1;
  }
  std::vector<char> isc(ntop + 1, 0);
  std::vector<zdc> t(ntop + 1, mkz(0.0));
  t[ntop - 1] = mkz(1.0);
  for (int i = ntop - 1; i >= 1; i--) {
    t[i - 1] = ((2 * i + 1.0) * zi) * t[i] - t[i + 1];
    double a = zabs(t[i - 1]);
    if (a * a > up2) {
      t[i] = t[i] * up2inv;
      t[i - 1] = t[i - 1] * up2inv;
      isc[i] = 1;
    }
  }
  double sinv = 1.0 / scale, sct = 1.0;
  for (int i = 1; i <= ntop; i++) {
    sct = sct * sinv;
    if (isc[i - 1]) sct = sct * up2inv;
    t[i] = t[i] * sct;
  }
  zdc j0 = zsin_c(z) * zi, j1 = j0 * zi - zcos_c(z) * zi;
  zdc zs = (zabs(j1) > zabs(j0)) ? j1 / (t[1] * scale) : j0 / t[0];
  for (int i = 0; i <= n; i++) f[i] = t[i] * zs;
  if (fd) {
    (*fd)[0] = -(f[1] * scale);
    for (int i = 1; i <= n; i++) {
      double dc1 = i / (2 * i + 1.0), dc2 = 1.0 - dc1;
      dc1 = dc1 * sinv;
      dc2 = dc2 * scale;
      (*fd)[i] = (dc1 * t[i - 1] - dc2 * t[i + 1]) * zs;
    }
  }
}

// Gauss-Legendre nodes (ascending) and weights on [-1, 1] by Newton's method
// on P_n (the reference calls legeexps with itype = 1: the same rule)
void gauss_legendre_host(int n, std::vector<double>& x, std::vector<double>& w) {
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  auto pn = [n](double t, double& p, double& dp) {
    double p0 = 1.0, p1 = t;
    for (int k = 2; k <= n; k++) {
      double p2 = ((2 * k - 1) * t * p1 - (k - 1) * p0) / k;
      p0 = p1;
      p1 = p2;
    }
    p = p1;
    dp = n * (t * p1 - p0) / (t * t - 1.0);
  };
  for (int i = 0; i < n; i++) {
    double t = cos(kPi * (i + 0.75) / (n + 0.5)), p, dp;
    for (int it = 0; it < 100; it++) {
      pn(t, p, dp);
      double dt = p / dp;
      t -= dt;
      if (fabs(dt) < 1e-16) break;
    }
    pn(t, p, dp);
    x[n - 1 - i] = t;
    w[n - 1 - i] = 2.0 / ((1.0 - t * t) * dp * dp);
  }
}

struct H3Key {
  double size, zr, zi, eps;
  int isep;
  bool operator<(const H3Key& o) const {
    return std::tie(size, zr, zi, eps, isep) < std::tie(o.size, o.zr, o.zi, o.eps, o.isep);
  }
};
std::mutex g_h3_mu;
std::map<H3Key, int> g_h3_cache;

size_t htrans_smem(int pbuf, int C) { return htrans_layout(pbuf, C, nullptr, nullptr); }

template <int KIND, int KMAX, bool GMEM>
void launch_htrans_k(const HTransArgs& A, int nblocks, size_t bytes, zdc* scratch,
                     cudaStream_t s) {
  if (GMEM) {
    int grid = std::min(nblocks, kGmemCtas);
    klaunch(k_htrans3<KIND, KMAX, true>, grid, HNT, 0, s, A, scratch, bytes / sizeof(zdc));
  } else {
    ZF_CUDA(cudaFuncSetAttribute(k_htrans3<KIND, KMAX, false>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    klaunch(k_htrans3<KIND, KMAX, false>, nblocks, HNT, bytes, s, A, scratch, (size_t)0);
  }
}

// scratch: kGmemCtas * htrans_smem(pbuf, C) bytes when the working arrays do
// not fit in shared memory, else unused
template <int KIND>
void launch_htrans(const HTransArgs& A, zdc* scratch, cudaStream_t s) {
  int nblocks = A.hi - A.lo + 1;
  if (nblocks <= 0) return;
  size_t bytes = htrans_smem(A.pbuf, A.C);
  int kneed = div_up((long)(A.pbuf + 1) * (A.pbuf + 1), HNT);
  if (bytes <= kSmemMax) {
    if (kneed <= 4) launch_htrans_k<KIND, 4, false>(A, nblocks, bytes, scratch, s);
    else if (kneed <= 8) launch_htrans_k<KIND, 8, false>(A, nblocks, bytes, scratch, s);
    else if (kneed <= 12) launch_htrans_k<KIND, 12, false>(A, nblocks, bytes, scratch, s);
    else launch_htrans_k<KIND, 16, false>(A, nblocks, bytes, scratch, s);
  } else {
    if (!scratch) throw zf_error(ZF_ERR_INTERNAL, "translation workspace missing");
    if (kneed <= 16) launch_htrans_k<KIND, 16, true>(A, nblocks, bytes, scratch, s);
    else if (kneed <= 24) launch_htrans_k<KIND, 24, true>(A, nblocks, bytes, scratch, s);
    else if (kneed <= 32) launch_htrans_k<KIND, 32, true>(A, nblocks, bytes, scratch, s);
    else throw zf_error(ZF_ERR_ARG, "expansion order too large for the 3D translation kernel");
  }
  ZF_LAUNCH_CHECK();
}

int choose_split_h3(int nt, int ns) {
  int tblocks = div_up(nt, HENT);
  int want = 4 * 148;
  int ns_max = std::max(1, div_up(ns, 4 * HPTILE));
  int nsplit = std::max(1, std::min(ns_max, div_up(want, tblocks)));
  return std::min(nsplit, 64);
}

}  // namespace

int h3dterms_host(double size, zdc zk, double eps, int isep) {
  // h3dterms.f:16-75
  H3Key key{size, zk.re, zk.im, eps, isep};
  {
    std::lock_guard<std::mutex> lk(g_h3_mu);
    auto it = g_h3_cache.find(key);
    if (it != g_h3_cache.end()) return it->second;
  }
  const int NT = 5000;
  std::vector<zdc> hf(NT + 2), jf;
  zdc zks = zk * size;
  zdc z1 = zks * (0.5 + isep * 1.0);
  double rscale = 1.0;
  if (zabs(zks) < 1.0) rscale = zabs(zks);
  h3dall_z(NT, z1, rscale, hf.data(), nullptr);
  zdc z2 = zks * sqrt(3.0) / 2.0;
  besseljs3d_host(NT, z2, rscale, jf, nullptr);
  double x0 = zabs(jf[0] * hf[0]) + zabs(jf[1] * hf[1]);
  int nterms = 5000;
  for (int j = 2; j <= NT; j++) {
    double xt = (zabs(jf[j] * hf[j]) + zabs(jf[j - 1] * hf[j - 1])) * zabs(hf[0]) * zabs(zk);
    if (xt < eps * x0) {
      nterms = j + 1;
      break;
    }
  }
  std::lock_guard<std::mutex> lk(g_h3_mu);
  if (g_h3_cache.size() > 4096) g_h3_cache.clear();
  g_h3_cache[key] = nterms;
  return nterms;
}

void zh3ddirect_device(zdc zk, const Inputs3D& in, zdc* pot, zdc* grad, cudaStream_t s) {
  if (in.nt <= 0 || in.ns <= 0) return;
  int nsplit = choose_split_h3(in.nt, in.ns);
  int chunk = div_up(in.ns, nsplit);
  nsplit = div_up(in.ns, chunk);
  bool G = in.ifpgh > 1;
  DevBuf<zdc> part;
  if (nsplit > 1) part.alloc((size_t)nsplit * in.nt * (G ? 4 : 1), s);
  dim3 grid(div_up(in.nt, HENT), nsplit);
  if (G) {
    klaunch(k_hdirect3d<true>, grid, HENT, 0, s, in, zk, chunk, pot, grad, part.get());
    if (nsplit > 1)
      klaunch(k_hdirect3d_reduce<true>, div_up(in.nt, 256), 256, 0, s, in.nt, nsplit, part.get(), pot, grad);
  } else {
    klaunch(k_hdirect3d<false>, grid, HENT, 0, s, in, zk, chunk, pot, grad, part.get());
    if (nsplit > 1)
      klaunch(k_hdirect3d_reduce<false>, div_up(in.nt, 256), 256, 0, s, in.nt, nsplit, part.get(), pot, grad);
  }
  ZF_LAUNCH_CHECK();
}

// orders per level, tables and quadrature z-shift configurations of one
// wavenumber on a set-up (zhfmm3d.f:200-240 and the zh3dtrans.f set-ups)
void helm_prep(const Setup3D& S, double eps, zdc zk, int isep, HelmPrep& H, cudaStream_t s) {
  const DevTree& t = S.tree;
  const int nlev = t.nlevels;
  if (nlev + 1 > ML) throw zf_error(ZF_ERR_ARG, "too many tree levels");
  zdc kw = zk * S.b0;  // zkfmm
  H.kw = kw;
  HLev& lev = H.lev;
  long tot = 0;
  int pmax = 0, pref = 0;
  for (int l = 0; l <= nlev; l++) {
    double r = S.bsz[l] * zabs(kw);
    lev.rs[l] = r > 1.0 ? 1.0 : r;
    int p = h3dterms_host(S.bsz[l], kw, eps, isep) + 0;  // n0 = 0 (zhfmm3d.f:223)
    if (l > 0 && p > pref) p = pref;  // the reference clips to non-increasing orders
    pref = p;
    lev.p[l] = p;
  }
  // Expansions of levels 0 and 1 are never read: lists 2 and 4 are empty there
  // (the level-1 boxes touch), list-3 boxes and local evaluations are at
  // levels >= 2.  They are not formed here (the reference forms the level-1
  // multipoles by M2M and never uses them); p of levels >= 2 bounds the work.
  lev.p[0] = 0;
  if (nlev >= 1) lev.p[1] = 0;
  for (int l = 0; l <= nlev; l++) {
    lev.lo[l] = t.laddr[2 * l];
    lev.base[l] = tot;
    tot += (long)(t.laddr[2 * l + 1] - t.laddr[2 * l] + 1) * (lev.p[l] + 1) * (lev.p[l] + 1);
    if (lev.p[l] > pmax) pmax = lev.p[l];
  }
  if (pmax > PMAXR)
    throw zf_error(ZF_ERR_ARG, "expansion order " + std::to_string(pmax) + " too large");
  H.T = get_tab3(pmax);
  H.pmax = pmax;
  H.tot = tot;
  // quadrature z-shift tables per kind and output level
  std::vector<ShiftTab> sth(3 * ML);
  std::vector<double> xw;  // nodes and weights, all configurations
  std::vector<zdc> cfd;    // cF, cD
  struct Pend {
    int kind, l;
    size_t xo, wo, fo, dpo;
  };
  std::vector<Pend> pend;
  for (int kind = 0; kind < 3; kind++)
    for (int l = 2; l <= nlev; l++) {
      int l1, l2 = l;
      if (kind == 0) {  // parent level l >= 2, children l+1
        if (l >= nlev) continue;
        l1 = l + 1;
      } else if (kind == 1) {
        l1 = l;
      } else {  // child level l, parent l-1 >= 2
        if (l < 3) continue;
        l1 = l - 1;
      }
      int p1 = lev.p[l1], p2 = lev.p[l2];
      int nq = (int)(p2 * 2.5);
      double w1 = S.bsz[l1], w2 = S.bsz[l2];
      double r = kind == 1 ? w1 / 2 * sqrt(3.0) : (kind == 0 ? w1 * sqrt(3.0) : w2 * sqrt(3.0));
      std::vector<double> gx, gw;
      gauss_legendre_host(nq, gx, gw);
      Pend pe{kind, l, xw.size(), 0, cfd.size(), 0};
      xw.insert(xw.end(), gx.begin(), gx.end());
      pe.wo = xw.size();
      xw.insert(xw.end(), gw.begin(), gw.end());
      // projection radial functions at k r: h_n (mpmp) or j_n (mploc, locloc)
      zdc zr = kw * r;
      std::vector<zdc> g(p2 + 2), gd(p2 + 2);
      if (kind == 0) h3dall_z(p2, zr, lev.rs[l2], g.data(), gd.data());
      else besseljs3d_host(p2, zr, lev.rs[l2], g, &gd);
      std::vector<zdc> cF(p2 + 1), cD(p2 + 1);
      for (int n = 0; n <= p2; n++) {
        zdc gdk = kw * gd[n];
        zdc gsum = (g[n] * g[n] + gdk * gdk) * (1.0 / (2 * kPi));
        cF[n] = g[n] / gsum;
        cD[n] = gdk / gsum;
      }
      cfd.insert(cfd.end(), cF.begin(), cF.end());
      pe.dpo = cfd.size();
      cfd.insert(cfd.end(), cD.begin(), cD.end());
      ShiftTab& st = sth[kind * ML + l];
      st.p1 = p1;
      st.p2 = p2;
      st.nq = nq;
      st.r = r;
      st.rs1 = lev.rs[l1];
      pend.push_back(pe);
    }
  DevBuf<double>& dxw = H.dxw;
  DevBuf<zdc>& dcfd = H.dcfd;
  dxw.alloc(std::max<size_t>(xw.size(), 1), s);
  dcfd.alloc(std::max<size_t>(cfd.size(), 1), s);
  if (!xw.empty())
    ZF_CUDA(cudaMemcpyAsync(dxw.get(), xw.data(), xw.size() * sizeof(double),
                            cudaMemcpyHostToDevice, s));
  if (!cfd.empty())
    ZF_CUDA(cudaMemcpyAsync(dcfd.get(), cfd.data(), cfd.size() * sizeof(zdc),
                            cudaMemcpyHostToDevice, s));
  for (auto& pe : pend) {
    ShiftTab& st = sth[pe.kind * ML + pe.l];
    st.x = dxw.get() + pe.xo;
    st.w = dxw.get() + pe.wo;
    st.cF = dcfd.get() + pe.fo;
    st.cD = dcfd.get() + pe.dpo;
  }
  DevBuf<ShiftTab>& dst = H.dst;
  dst.alloc(3 * ML, s);
  H.sth = sth;
  ZF_CUDA(cudaMemcpyAsync(dst.get(), sth.data(), sth.size() * sizeof(ShiftTab),
                          cudaMemcpyHostToDevice, s));
  ZF_CUDA(cudaStreamSynchronize(s));  // the host staging vectors go out of scope below
}

// P2M through L2T/M2T/P2P on a set-up and its wavenumber tables: adds the
// sorted potentials (and gradients, unscaled) of one right-hand side with
// sorted strengths q, ds, dv to potsort / gradsort; ev[2..5] (optional) get
// the step boundaries recorded
namespace {
size_t form_smem(int pmax, int* fw_out) {
  int fw = HFNT / 32;  // warps of the form kernel, one partial expansion each
  while (fw > 1 && (size_t)fw * (pmax + 1) * (pmax + 1) * sizeof(zdc) > kSmemMax) fw /= 2;
  size_t smf = (size_t)fw * (pmax + 1) * (pmax + 1) * sizeof(zdc);
  if (smf > kSmemMax) throw zf_error(ZF_ERR_ARG, "expansion order too large for P2M staging");
  *fw_out = fw;
  return smf;
}
}  // namespace

void helm_form(const Setup3D& S, const HelmPrep& H, const zdc* q, const zdc* ds, const zdc* dv,
               int ifcharge, int ifdipole, bool local, zdc* out, cudaStream_t s) {
  const DevTree& t = S.tree;
  const DevLists& L = S.lists;
  const int nb = t.nboxes, nlev = t.nlevels, pmax = H.pmax;
  if (!local && nlev < 2) return;
  if (local && L.mn[3] <= 0) return;
  HFormArgs F;
  F.r1 = H.T.r1; F.r2 = H.T.r2; F.sq = H.T.sq; F.L = pmax + 1;
  F.ilevel = t.ilevel.get(); F.nchild = t.nchild.get();
  F.isrcse = S.isrcse.get(); F.itargse = S.itargse.get();
  F.zsrc = S.zsrcsort.get(); F.charge = q; F.dipstr = ds;
  F.dipvec = dv; F.zcs = S.zcsrc.get(); F.zct = S.zctarg.get();
  F.lev = H.lev; F.nl4 = L.n[3].get(); F.l4 = L.list[3].get(); F.mn4 = L.mn[3];
  F.nb = nb; F.ifcharge = ifcharge; F.ifdipole = ifdipole; F.pbuf = pmax; F.zk = H.kw;
  F.out = out;
  int fw = 1;
  size_t smf = form_smem(pmax, &fw);
  if (local) {
    if (ifdipole) {
      ZF_CUDA(cudaFuncSetAttribute(k_hform3<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smf));
      klaunch(k_hform3<true, true>, nb, 32 * fw, smf, s, F);
    } else {
      ZF_CUDA(cudaFuncSetAttribute(k_hform3<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smf));
      klaunch(k_hform3<true, false>, nb, 32 * fw, smf, s, F);
    }
  } else {
    if (ifdipole) {
      ZF_CUDA(cudaFuncSetAttribute(k_hform3<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smf));
      klaunch(k_hform3<false, true>, nb, 32 * fw, smf, s, F);
    } else {
      ZF_CUDA(cudaFuncSetAttribute(k_hform3<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smf));
      klaunch(k_hform3<false, false>, nb, 32 * fw, smf, s, F);
    }
  }
  ZF_LAUNCH_CHECK();
}

void helm_eval(const Setup3D& S, const HelmPrep& H, const zdc* q, const zdc* ds, const zdc* dv,
               int ifcharge, int ifdipole, int ifpgh, const zdc* mp, const zdc* loc,
               zdc* potsort, zdc* gradsort, cudaStream_t s) {
  const DevTree& t = S.tree;
  const DevLists& L = S.lists;
  const int nb = t.nboxes, pmax = H.pmax;
  HP2PArgs Pa;
  Pa.nchild = t.nchild.get(); Pa.isrcse = S.isrcse.get(); Pa.itargse = S.itargse.get();
  Pa.zsrc = S.zsrcsort.get(); Pa.charge = q; Pa.dipstr = ds;
  Pa.dipvec = dv; Pa.ztarg = S.ztargsort.get();
  Pa.nl1 = L.n[0].get(); Pa.l1 = L.list[0].get(); Pa.mn1 = L.mn[0]; Pa.nb = nb;
  Pa.ifcharge = ifcharge; Pa.ifdipole = ifdipole; Pa.zk = H.kw;
  Pa.pot = potsort; Pa.grad = gradsort;
  if (ifpgh > 1) klaunch(k_hp2p3<true>, nb, HENT, 0, s, Pa);
  else klaunch(k_hp2p3<false>, nb, HENT, 0, s, Pa);
  ZF_LAUNCH_CHECK();
  HEvalArgs E;
  E.r1 = H.T.r1; E.r2 = H.T.r2; E.sq = H.T.sq; E.L = pmax + 1;
  E.ilevel = t.ilevel.get(); E.nchild = t.nchild.get(); E.isrcse = S.isrcse.get();
  E.itargse = S.itargse.get(); E.ztarg = S.ztargsort.get(); E.zcs = S.zcsrc.get();
  E.zct = S.zctarg.get(); E.lev = H.lev; E.mp = mp; E.loc = loc;
  E.nl3 = L.n[2].get(); E.l3 = L.list[2].get(); E.mn3 = L.mn[2]; E.nb = nb; E.pbuf = pmax;
  E.zk = H.kw; E.pot = potsort; E.grad = gradsort;
  size_t sme = (size_t)(pmax + 1) * (pmax + 1) * sizeof(zdc);
  if (ifpgh > 1) {
    ZF_CUDA(cudaFuncSetAttribute(k_heval3<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sme));
    klaunch(k_heval3<true>, nb, HENT, sme, s, E);
  } else {
    ZF_CUDA(cudaFuncSetAttribute(k_heval3<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sme));
    klaunch(k_heval3<false>, nb, HENT, sme, s, E);
  }
  ZF_LAUNCH_CHECK();
}

void helm_core(const Setup3D& S, const HelmPrep& H, const zdc* q, const zdc* ds, const zdc* dv,
               int ifcharge, int ifdipole, int ifpgh, zdc* potsort, zdc* gradsort,
               cudaStream_t s, cudaEvent_t* ev) {
  auto hmark = [&](int i) {
    if (ev) ZF_CUDA(cudaEventRecord(ev[i], s));
  };
  const DevTree& t = S.tree;
  const DevLists& L = S.lists;
  const int nb = t.nboxes, nlev = t.nlevels;
  const HLev& lev = H.lev;
  const int pmax = H.pmax;
  const long tot = H.tot;
  const Tab3& T = H.T;
  const zdc kw = H.kw;
  const DevBuf<ShiftTab>& dst = H.dst;
  DevBuf<zdc> mp(std::max<long>(tot, 1), s), loc(std::max<long>(tot, 1), s);
  mp.zero();
  loc.zero();
  helm_form(S, H, q, ds, dv, ifcharge, ifdipole, false, mp.get(), s);
  hmark(2);
  HTransArgs A;
  A.r1 = T.r1; A.r2 = T.r2; A.sq = T.sq; A.dinv = T.dinv; A.L = pmax + 1; A.pT = pmax;
  A.ilevel = t.ilevel.get(); A.iparent = t.iparent.get(); A.nchild = t.nchild.get();
  A.ichild = t.ichild.get(); A.isrcse = S.isrcse.get(); A.itargse = S.itargse.get();
  A.zcs = S.zcsrc.get(); A.zct = S.zctarg.get(); A.lev = lev;
  A.nl2 = L.n[1].get(); A.l2 = L.list[1].get(); A.nl4 = L.n[3].get(); A.mn2 = L.mn[1];
  A.kwave = kw;
  A.pbuf = pmax;
  A.C = 16;
  while (A.C > 4 && htrans_smem(pmax, A.C) > kSmemMax) A.C /= 2;
  DevBuf<zdc> hscratch;
  if (htrans_smem(pmax, A.C) > kSmemMax) {
    A.C = 16;
    hscratch.alloc((size_t)kGmemCtas * htrans_smem(pmax, A.C) / sizeof(zdc), s);
  }
  // M2M, finest parents first (parents at levels >= 2)
  A.in = mp.get();
  A.out = mp.get();
  A.st = dst.get() + 0 * ML;
  for (int l = nlev - 1; l >= 2; l--) {
    A.lo = t.laddr[2 * l];
    A.hi = t.laddr[2 * l + 1];
    launch_htrans<0>(A, hscratch.get(), s);
  }
  hmark(3);
  // M2L over levels >= 2, then P2L (list 4)
  A.in = mp.get();
  A.out = loc.get();
  A.st = dst.get() + 1 * ML;
  if (nlev >= 2) {
    A.lo = t.laddr[4];
    A.hi = nb - 1;
    launch_htrans<1>(A, hscratch.get(), s);
  }
  helm_form(S, H, q, ds, dv, ifcharge, ifdipole, true, loc.get(), s);
  hmark(4);
  // L2L, coarsest first: children at level l+1 of parents at level l >= 2
  A.in = loc.get();
  A.out = loc.get();
  A.st = dst.get() + 2 * ML;
  for (int l = 2; l <= nlev - 1; l++) {
    A.lo = t.laddr[2 * (l + 1)];
    A.hi = t.laddr[2 * (l + 1) + 1];
    launch_htrans<2>(A, hscratch.get(), s);
  }
  hmark(5);
  helm_eval(S, H, q, ds, dv, ifcharge, ifdipole, ifpgh, mp.get(), loc.get(), potsort, gradsort, s);
}

void zhfmm3d_device(double eps, zdc zk, const Inputs3D& in, int isep, zdc* pot, zdc* grad,
                    cudaStream_t s, StepTimes* times) {
  int ns = in.ns, nt = in.nt;
  long launches0 = launch_counter();
  cudaEvent_t ev[8];
  bool timing = times != nullptr;
  if (timing)
    for (auto& e : ev) ZF_CUDA(cudaEventCreate(&e));
  auto mark = [&](int i) {
    if (timing) ZF_CUDA(cudaEventRecord(ev[i], s));
  };
  mark(0);
  TreeParams tp;
  tp.D = 3;
  tp.isep = isep;
  tp.idivflag = 0;                 // hndiv resets the driver's idivflag = 2 (zhfmm3d.f:64-67)
  tp.ndiv = lndiv3d(eps, ns, nt);  // hndiv_fast.f: the same table as lndiv
  tp.lr_isep_quirk = 1;
  Setup3D S;
  setup3d(in, tp, S, true, true, s);
  mark(1);
  HelmPrep H;
  helm_prep(S, eps, zk, isep, H, s);
  DevBuf<zdc> potsort(nt, s), gradsort(in.ifpgh > 1 ? 3 * (size_t)nt : 1, s);
  potsort.zero();
  gradsort.zero();
  helm_core(S, H, S.chargesort.get(), S.dipstrsort.get(), S.dipvecsort.get(), in.ifcharge,
            in.ifdipole, in.ifpgh, potsort.get(), gradsort.get(), s, timing ? ev : nullptr);
  mark(6);
  unsort3d(nt, S.itarg.get(), potsort.get(), gradsort.get(), mkz(1.0), mkz(1.0 / S.b0), in.ifpgh,
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
    times->nterms = H.pmax;
    for (auto& e : ev) cudaEventDestroy(e);
    times->launches = launch_counter() - launches0;
    if (times->want_counts) count_interactions3d(S, H.lev.p, 2, 2, 3, times, s);
  }
}

void helm_plan_loop(const Plan3D& P, const HelmPrep& H, int nd, const StrengthsNd& in, int ifpgh,
                    zdc* pot, zdc* grad, cudaStream_t s, StepTimes* times, float prep_ms) {
  const Setup3D& S = P.S;
  const int ns = P.ns, nt = P.nt;
  long launches0 = launch_counter();
  const bool timing = times != nullptr;
  cudaEvent_t ev[8];
  if (timing)
    for (auto& e : ev) ZF_CUDA(cudaEventCreate(&e));
  float acc[8] = {0};
  acc[0] = prep_ms;
  auto mark = [&](int i) {
    if (timing) ZF_CUDA(cudaEventRecord(ev[i], s));
  };
  auto take = [&](int a, int b, int slot) {
    if (!timing) return;
    ZF_CUDA(cudaEventSynchronize(ev[b]));
    float ms;
    ZF_CUDA(cudaEventElapsedTime(&ms, ev[a], ev[b]));
    acc[slot] += ms;
  };
  mark(0);
  DevBuf<zdc> q(ns, s), ds(ns, s), dv(3 * (size_t)ns, s), potsort(nt, s),
      gradsort(ifpgh > 1 ? 3 * (size_t)nt : 1, s);
  mark(1);
  take(0, 1, 0);
  for (int r = 0; r < nd; r++) {
    mark(0);
    gather_strengths_col(S, ns, nd, r, in.ifcharge ? in.charge : nullptr,
                         in.ifdipole ? in.dipstr : nullptr, in.ifdipole ? in.dipvec : nullptr,
                         true, true, q.get(), ds.get(), dv.get(), s);
    potsort.zero();
    gradsort.zero();
    mark(1);
    helm_core(S, H, q.get(), ds.get(), dv.get(), in.ifcharge, in.ifdipole, ifpgh, potsort.get(),
              gradsort.get(), s, timing ? ev : nullptr);
    mark(6);
    unsort3d_col(nt, nd, r, S.itarg.get(), potsort.get(), gradsort.get(), mkz(1.0),
                 mkz(1.0 / S.b0), ifpgh, pot, grad, s);
    mark(7);
    for (int k = 0; k < 7; k++) take(k, k + 1, k);
  }
  if (timing) {
    for (int k = 0; k < 7; k++) times->ms[k] = acc[k];
    times->nboxes = S.tree.nboxes;
    times->nlevels = S.tree.nlevels;
    times->nterms = H.pmax;
    for (auto& e : ev) cudaEventDestroy(e);
    times->launches = launch_counter() - launches0;
    if (times->want_counts) count_interactions3d(S, H.lev.p, 2, 2, 3, times, s);
  }
}

}  // namespace zf
