// 3D Laplace FMM for many right-hand sides on one geometry (a plan).
//
// The same algorithm as zlfmm3d (zfmm3d/src/laplace/zlfmm3d.f:252-622) with
// every expansion, strength and output carrying a right-hand-side index r
// fastest: expansion (box, coefficient n*n+n+m, r) at
// (box * (p+1)^2 + n*n+n+m) * nd + r, strengths q[i*nd + r], potentials
// pot[i*nd + r], gradients grad[(3i+d)*nd + r].  Geometry-dependent work
// (Legendre recurrences, rotation samples, shift tables, pair distances) is
// computed once per box pair, source or target and applied to every
// right-hand side.
//
// Kernels:
//   k_trans3nd  M2M / M2L / L2L.  The point-and-shoot translation of
//               zl3dmpmp / zl3dmploc / zl3dlocloc (zl3dtrans.f:1-540): z-rotation,
//               y-rotation by sampling on the rotated meridian (the
//               recurrences of myzylgndr2sf, ztoolbox.f:273-327) and projection
//               by a DFT (z3dyrot, zrotate.f:94-239), axial shift, inverse
//               rotations.  The y-rotation is streamed one degree n at a time:
//               the sample coefficients of degree n for all angles come from
//               (angle, order) recurrence states held in registers (one state per
//               thread slot), and are applied to 32 right-hand sides (one per
//               lane) as two small complex products, sample then project.  The
//               samples at angles +j and -j share their Legendre values, so the
//               product is formed on sums and differences of the +m / -m
//               coefficients and the projection on the cosine / sine halves of
//               the DFT (a quarter of the direct product's work).  The shifted and
//               rotated expansions of the 32 right-hand sides pass through a
//               per-CTA scratch in global memory (L2-resident).
//   k_form3nd   P2M / P2L: one warp per (box, 32 right-hand sides); lanes
//               stream the source recurrences (lane = source) into a small
//               shared buffer, then sum it against the staged strengths
//               (lane = right-hand side).
//   k_eval3nd   L2T / M2T: a thread per target, the recurrence values applied to
//               RB right-hand sides held in registers.
//   k_p2p3nd    list-1 direct interactions, pair geometry once for RB
//               right-hand sides.
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <vector>
#include "lfmm3d.cuh"
#include "plan3d.cuh"
#include "rot3nd.cuh"
#include "sph3d.cuh"

namespace zf {

namespace {

struct TransNdArgs {
  Tab3 T;
  RotTab R;
  const int *ilevel, *iparent, *nchild, *ichild, *isrcse, *itargse;
  const zdc *zcs, *zct;
  const double* rsc;
  const zdc* in;
  zdc* out;
  zdc* scratch;  // 2 (p+1)^2 RC per CTA
  int* queue;    // work-queue counter, zero at launch
  const int *nl2, *l2, *nl4;
  int mn2, nd, lo, hi;
  int rot_smem;  // 1: the cos / sin tables are staged in shared memory
};

// axial shift X1 -> X2 (scratch, row stride RC)
template <int KIND>
__device__ void shift_nd(const Tab3& T, const XSm& S, const zdc* X1, zdc* X2) {
  const int p = T.p, nmax = T.nmax, ldA = 2 * nmax + 1, lane = threadIdx.x & 31,
            w = threadIdx.x >> 5;
  int t = 0;
  for (int mm = -p; mm <= p; mm++) {
    const int am_ = mm < 0 ? -mm : mm, nbk = (p + 1 - am_ + JB - 1) / JB;
    for (int bk = 0; bk < nbk; bk++, t++) {
      if (t % XW != w) continue;
      const int j0 = am_ + bk * JB;
      zdc acc[JB];
#pragma unroll
      for (int k = 0; k < JB; k++) acc[k] = mkz(0.0);
      if (KIND == 1) {
#pragma unroll 4
        for (int n = am_; n <= p; n++) {
          zdc a = ldcg_z(X1 + ix3(n, mm) * RC + lane);
#pragma unroll
          for (int k = 0; k < JB; k++)
            if (j0 + k <= p) acc[k] += a * S.G[n + j0 + k];
        }
      } else if (KIND == 0) {
        int nhi = min(p, j0 + JB - 1);
#pragma unroll 4
        for (int n = am_; n <= nhi; n++) {
          zdc a = ldcg_z(X1 + ix3(n, mm) * RC + lane);
#pragma unroll
          for (int k = 0; k < JB; k++) {
            int j = j0 + k;
            if (j <= p && n <= j) acc[k] += a * S.G[j - n];
          }
        }
      } else {
#pragma unroll 4
        for (int n = j0; n <= p; n++) {
          zdc a = ldcg_z(X1 + ix3(n, mm) * RC + lane);
#pragma unroll
          for (int k = 0; k < JB; k++) {
            int j = j0 + k;
            if (j <= p && n >= j) acc[k] += a * S.G[n - j];
          }
        }
      }
#pragma unroll
      for (int k = 0; k < JB; k++) {
        int j = j0 + k;
        if (j > p) break;
        double ajk = __ldg(&T.amat[j * ldA + mm + nmax]);
        zdc v = (KIND == 0) ? S.T1[j] * acc[k] / ajk : S.T1[j] * acc[k] * ajk;
        stcg_z(X2 + ix3(j, mm) * RC + lane, v);
      }
    }
  }
}

template <int KIND, int SLOTS>
__global__ void __launch_bounds__(XNT, 1) k_trans3nd(TransNdArgs A) {
  extern __shared__ zdc sm[];
  const Tab3& T = A.T;
  const int p = T.p, NC = T.NC, tid = threadIdx.x;
  XSm S;
  xsm_layout(p, A.rot_smem != 0, sm, &S);
  RotTab Rt = A.R;
  {
    const int L = p + 1, CP = rot_cp(L), KR = rot_kr(L), TP = rot_tp(L);
    if (S.cw) {
      // tables staged once (cw then sw, contiguous in global memory)
      for (int k = tid; k < 2 * CP * TP; k += XNT) S.cw[k] = A.R.cw[k];
    }
    // the padding columns (angles >= p+1) of the sample coefficients stay zero
    for (int k = tid; k < KR * CP; k += XNT) {
      S.Csr[k] = 0.0;
      S.Csi[k] = 0.0;
      S.Cdr[k] = 0.0;
      S.Cdi[k] = 0.0;
    }
  }
  zdc* X1 = A.scratch + (size_t)blockIdx.x * 2 * NC * RC;
  zdc* X2 = X1 + (size_t)NC * RC;
  const double s4 = sqrt(4 * kPi);
  const int nmax = T.nmax, ldA = 2 * nmax + 1;
  const double* __restrict__ am = T.amat;
  const long nd = A.nd;
  // work items (box, pass of 32 right-hand sides) taken from a queue: the
  // boxes' list sizes differ widely, and the passes of one box write disjoint
  // right-hand sides
  __shared__ int s_item;
  const int npass = (A.nd + RC - 1) / RC;
  const int nitems = (A.hi - A.lo + 1) * npass;
  for (;;) {
    __syncthreads();
    if (tid == 0) s_item = atomicAdd(A.queue, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= nitems) break;
    const int b = A.lo + item / npass, r0 = (item % npass) * RC;
    int nin = 0, par = -1;
    if (KIND == 0) {
      if (nsrc(A.isrcse, b) <= 0 || A.nchild[b] == 0) continue;
      nin = A.nchild[b];
    } else if (KIND == 1) {
      if (nsrc(A.itargse, b) <= 0 || A.nl2[b] == 0) continue;
      nin = A.nl2[b];
    } else {
      par = A.iparent[b];
      if (par < 0 || nsrc(A.itargse, b) <= 0 || nsrc(A.itargse, par) <= 0 ||
          (A.nl2[par] == 0 && A.nl4[par] == 0))
        continue;
      nin = 1;
    }
    const int lb = A.ilevel[b];
    {
      const int nval = min(RC, A.nd - r0);
      for (int it = 0; it < nin; it++) {
        int src;
        const zdc *c0, *c;
        double rs0, rs;
        if (KIND == 0) {
          src = A.ichild[8 * b + it];
          if (nsrc(A.isrcse, src) <= 0) continue;
          c0 = A.zcs + 3 * src;
          c = A.zcs + 3 * b;
          rs0 = A.rsc[lb + 1];
          rs = A.rsc[lb];
        } else if (KIND == 1) {
          src = A.l2[(size_t)b * A.mn2 + it];
          if (nsrc(A.isrcse, src) <= 0) continue;
          c0 = A.zcs + 3 * src;
          c = A.zct + 3 * b;
          rs0 = rs = A.rsc[lb];
        } else {
          src = par;
          c0 = A.zct + 3 * par;
          c = A.zct + 3 * b;
          rs0 = A.rsc[lb - 1];
          rs = A.rsc[lb];
        }
        Geo g = geo3(c0, c);
        zdc zsh = g.zshift;
        bool flip = zabs(zsqrt_p(zsh * zsh) - zsh) > kF16;
        zdc rzs = flip ? -zsh : zsh;
        __syncthreads();
        for (int m = tid; m <= p; m += XNT) {
          zdc ef = zpown(g.cb + zmul_i(g.sb), m), eb = zpown(g.cb - zmul_i(g.sb), m);
          S.Ef[p + m] = ef;
          S.Ef[p - m] = zinv(ef);
          S.Eb[p + m] = eb;
          S.Eb[p - m] = zinv(eb);
        }
        if (KIND == 0) {
          zdc rz = rzs / rs0;
          for (int n = tid; n <= p; n += XNT) {
            double yl = __ldg(&T.sq[n]) * ((flip && (n & 1)) ? -1.0 : 1.0);
            S.G[n] = (zpown(rz, n) * (__ldg(&am[n * ldA + nmax]) * yl)) / (2 * n + 1.0);
            S.T1[n] = mkz(s4 * (ipow(rs0, n) / ipow(rs, n)));
          }
        } else if (KIND == 1) {
          zdc rz = rzs / rs0;
          for (int m = tid; m <= 2 * p; m += XNT) {
            double yl = __ldg(&T.sq[m]) * ((flip && (m & 1)) ? -1.0 : 1.0);
            S.G[m] = yl / (zpown(rz, m) * __ldg(&am[m * ldA + nmax]));
          }
          for (int j = tid; j <= p; j += XNT) S.T1[j] = (s4 / (2 * j + 1.0)) / rz;
        } else {
          zdc rz = rzs / rs;
          for (int n = tid; n <= p; n += XNT) {
            double yl = __ldg(&T.sq[n]) * ((flip && (n & 1)) ? -1.0 : 1.0);
            S.G[n] = (zpown(rz, n) * (__ldg(&am[n * ldA + nmax]) * yl)) / (2 * n + 1.0);
            S.T1[n] = mkz(s4 / (2 * n + 1.0) * ((n & 1) ? -1.0 : 1.0));
            S.T2[n] = mkz((2 * n + 1.0) * (ipow(rs, n + 1) / ipow(rs0, n + 1)) *
                          ((n & 1) ? -1.0 : 1.0));
          }
        }
        __syncthreads();
        const zdc* gin = A.in + (size_t)src * NC * nd + r0;
        if (g.yr) rot_nd<SLOTS, 0, KIND>(T, p, p + 1, 1.0, Rt, S, g.ca, g.sa, g.zr, gin, nd, X1, RC, nval);
        else copy_nd<0, KIND>(T, p, S, g.zr, gin, nd, X1, RC, nval);
        __syncthreads();
        shift_nd<KIND>(T, S, X1, X2);
        __syncthreads();
        zdc* gout = A.out + (size_t)b * NC * nd + r0;
        if (g.yr) rot_nd<SLOTS, 1, KIND>(T, p, p + 1, 1.0, Rt, S, g.ca, -g.sa, g.zr, X2, RC, gout, nd, nval);
        else copy_nd<1, KIND>(T, p, S, g.zr, X2, RC, gout, nd, nval);
      }
    }
  }
}

// ---- P2M / P2L ---------------------------------------------------------------
constexpr int FW = 4;  // warps per CTA of the form kernel, one work item each
constexpr int KB = 8;  // (n, m) entries buffered per flush

struct FormNdArgs {
  Tab3 T;
  const int *ilevel, *nchild, *isrcse, *itargse;
  const zdc *zsrc, *q, *ds, *dv;
  const zdc *zcs, *zct;
  const double* rsc;
  zdc* out;
  const int *nl4, *l4;
  int mn4, nb, nd, nchunk, ifcharge, ifdipole;
};

__host__ __device__ inline size_t form_nd_warp_elems(bool dip) { return (dip ? 2 : 1) * (32 * 32 + KB * 2 * 32); }

// zl3dformmp (LOCAL = false) / zl3dformloc (LOCAL = true), zlfmm3d.f:689-1005,
// sources s0..s1 about centre zc, into the 32 right-hand sides r0.. of `o`
template <bool LOCAL, bool DIP>
__device__ void form_range_nd(const FormNdArgs& A, int s0, int s1, const zdc* zc,
                              double rscale, zdc* o, int r0, int nval, zdc* Qt, zdc* Dt,
                              zdc* Gq, zdc* Gd) {
  const Tab3& T = A.T;
  const int p = T.p, L = p + 1, lane = threadIdx.x & 31;
  const long nd = A.nd;
  const double s4 = 1.0 / sqrt(4 * kPi);
  const double* __restrict__ r1 = T.r1;
  const double* __restrict__ r2 = T.r2;
  const double* __restrict__ sq = T.sq;
  for (int base = s0; base <= s1; base += 32) {
    const int cnt = min(32, s1 - base + 1);
    __syncwarp();
    for (int k = 0; k < 32; k++) {
      bool ok = k < cnt && lane < nval;
      Qt[k * 32 + lane] = (ok && A.ifcharge) ? A.q[(long)(base + k) * nd + r0 + lane] : mkz(0.0);
      if (DIP) Dt[k * 32 + lane] = ok ? A.ds[(long)(base + k) * nd + r0 + lane] : mkz(0.0);
    }
    const bool valid = lane < cnt;
    const int ii = valid ? base + lane : base;
    Sph s = zcart2sph(A.zsrc[3 * ii], A.zsrc[3 * ii + 1], A.zsrc[3 * ii + 2], zc);
    zdc rz = s.rz / rscale;
    zdc irz = zinv(rz);
    zdc dzr_ = mkz(0.0), dthz = mkz(0.0), dphz = mkz(0.0);
    if (DIP) {
      zdc v0 = A.dv[3 * ii], v1 = A.dv[3 * ii + 1], v2 = A.dv[3 * ii + 2];
      dzr_ = v0 * (s.st * s.cp) + v1 * (s.st * s.sp) + v2 * s.ct;
      zdc dth_ = v0 * (s.ct * s.cp) + v1 * (s.ct * s.sp) - v2 * s.st;
      zdc dph_ = -(v0 * s.sp) + v1 * s.cp;
      dthz = dth_ / s.rz;
      dphz = dph_ / s.rz;
    }
    const zdc z = s.ct, zz1 = mkz(1.0) - z * z;
    const zdc u = -zsqrt_r(zz1);
    zdc colp = LOCAL ? irz : mkz(1.0);
    zdc Ydiag = mkz(1.0), em = mkz(1.0);
    int e = 0, fm = 0, fn = 0;  // buffered entries and the first (m, n) among them
    auto flush = [&]() {
      __syncwarp();
      int m = fm, n = fn;
      for (int k = 0; k < e; k++) {
        zdc ap = mkz(0.0), an = mkz(0.0);
        const zdc* gq = Gq + k * 64;
        const zdc* gd = Gd + k * 64;
        for (int j = 0; j < 32; j++) {
          zdc qv = Qt[j * 32 + lane];
          ap += gq[j] * qv;
          if (m > 0) an += gq[32 + j] * qv;
          if (DIP) {
            zdc dv = Dt[j * 32 + lane];
            ap += gd[j] * dv;
            if (m > 0) an += gd[32 + j] * dv;
          }
        }
        if (lane < nval) {
          o[(long)ix3(n, m) * nd + lane] += ap;
          if (m > 0) o[(long)ix3(n, -m) * nd + lane] += an;
        }
        if (n < p) n++;
        else {
          m++;
          n = m;
        }
      }
      __syncwarp();
      e = 0;
    };
    for (int m = 0; m <= p; m++) {
      zdc emi = mkz(1.0);
      if (m > 0) {
        double cmm = __ldg(&r1[m * L + m]);
        if (DIP) Ydiag = (m == 1) ? mkz(-cmm) : (Ydiag * u) * cmm;
        else Ydiag = (Ydiag * u) * cmm;
        em = em * s.eip;
        emi = zinv(em);
        colp = colp * (LOCAL ? irz : rz);
      }
      double sgm = (m & 1) ? -1.0 : 1.0;
      zdc Yp = Ydiag, Dp = DIP ? (Ydiag * (double)(-m)) * z : mkz(0.0);
      zdc Ypp = mkz(0.0), Dpp = mkz(0.0);
      zdc rp = colp;
      zdc rpm1 = (m > 0) ? colp * irz : mkz(0.0);
      for (int n = m; n <= p; n++) {
        zdc Y, D = mkz(0.0);
        if (n == m) {
          Y = Yp;
          D = Dp;
        } else {
          if (n == m + 1) {
            double c = __ldg(&r1[n * L + m]);
            Y = (z * Yp) * c;
            if (DIP) D = (m == 0) ? (z * Dp + Yp) * c : (z * Dp + zz1 * Yp) * c;
          } else {
            double c1 = __ldg(&r1[n * L + m]), c2 = __ldg(&r2[n * L + m]);
            Y = (c1 * z) * Yp - c2 * Ypp;
            if (DIP)
              D = (m == 0) ? c1 * (z * Dp + Yp) - c2 * Dpp
                           : c1 * (z * Dp + zz1 * Yp) - c2 * Dpp;
          }
          Ypp = Yp; Dpp = Dp; Yp = Y; Dp = D;
          rpm1 = rp;
          rp = rp * (LOCAL ? irz : rz);
        }
        double f = __ldg(&sq[n]) * (s4 * sgm / (2 * n + 1.0));
        zdc y = Y * f, dy = D * f;
        zdc qp, qn = mkz(0.0), dp = mkz(0.0), dn = mkz(0.0);
        if (m == 0) {
          qp = rp * y;
          if (DIP) {
            zdc dzr, dth;
            if (!LOCAL) {
              dzr = n == 0 ? mkz(0.0) : ((double)n * rpm1 / rscale) * y;
              dth = -(rp * dy * s.st);
            } else {
              dzr = -((double)(n + 1) * y * rp / s.rz);
              dth = -(dy * s.st * rp);
            }
            dp = -(dzr_ * dzr + dthz * dth);
          }
        } else {
          zdc ys = DIP ? s.st * y : y;
          zdc X = rp * ys;
          qp = emi * X;
          qn = em * X;
          if (DIP) {
            zdc DZ, DT, DP;
            if (!LOCAL) {
              DZ = ((double)n * rpm1 / rscale) * y * s.st;
              DT = -(rp * dy);
              DP = rp * y;
            } else {
              DZ = -((double)(n + 1) * y * s.st * rp / s.rz);
              DT = -(dy * rp);
              DP = y * rp;
            }
            zdc V = -(dzr_ * DZ + dthz * DT), W = dphz * zmul_i((double)m * DP);
            dp = emi * (V + W);
            dn = em * (V - W);
          }
        }
        if (!valid) qp = qn = dp = dn = mkz(0.0);
        if (e == 0) {
          fm = m;
          fn = n;
        }
        Gq[e * 64 + lane] = qp;
        Gq[e * 64 + 32 + lane] = qn;
        if (DIP) {
          Gd[e * 64 + lane] = dp;
          Gd[e * 64 + 32 + lane] = dn;
        }
        e++;
        if (e == KB) flush();
      }
    }
    if (e > 0) flush();
  }
}

template <bool LOCAL, bool DIP>
__global__ void __launch_bounds__(FW * 32) k_form3nd(FormNdArgs A) {
  extern __shared__ zdc sm[];
  const int w = threadIdx.x >> 5;
  const long item = (long)blockIdx.x * FW + w;
  if (item >= (long)A.nb * A.nchunk) return;
  const int b = (int)(item / A.nchunk), r0 = (int)(item % A.nchunk) * 32;
  const int nval = min(32, A.nd - r0);
  const int NC = A.T.NC;
  zdc* Qt = sm + (size_t)w * form_nd_warp_elems(DIP);
  zdc* Dt = Qt + 32 * 32;
  zdc* Gq = Dt + (DIP ? 32 * 32 : 0);
  zdc* Gd = Gq + KB * 2 * 32;
  int l = A.ilevel[b];
  zdc* o = A.out + (size_t)b * NC * A.nd + r0;
  if (!LOCAL) {
    if (A.nchild[b] != 0 || nsrc(A.isrcse, b) <= 0 || l < 1) return;
    form_range_nd<false, DIP>(A, A.isrcse[2 * b], A.isrcse[2 * b + 1], A.zcs + 3 * b, A.rsc[l],
                              o, r0, nval, Qt, Dt, Gq, Gd);
  } else {
    if (nsrc(A.itargse, b) <= 0 || A.nl4[b] == 0) return;
    for (int i = 0; i < A.nl4[b]; i++) {
      int jb = A.l4[(size_t)b * A.mn4 + i];
      if (nsrc(A.isrcse, jb) <= 0) continue;
      form_range_nd<true, DIP>(A, A.isrcse[2 * jb], A.isrcse[2 * jb + 1], A.zct + 3 * b,
                               A.rsc[l], o, r0, nval, Qt, Dt, Gq, Gd);
    }
  }
}

// ---- L2T / M2T -------------------------------------------------------------
constexpr int ENT = 128;
constexpr int RB = 8;   // right-hand sides per thread pass of the P2P kernel
constexpr int RBE = 4;  // right-hand sides per thread pass of the L2T / M2T kernel

struct EvalNdArgs {
  Tab3 T;
  const int *ilevel, *nchild, *isrcse, *itargse;
  const zdc *ztarg, *zcs, *zct;
  const double* rsc;
  const zdc *mp, *loc;
  const int *nl3, *l3;
  int mn3, nb, nd;
  zdc *pot, *grad;
};

// zl3devalmp (LOCAL = false) / zl3devalloc (LOCAL = true), zlfmm3d.f:1011-1277,
// for nv <= RBE right-hand sides; e: coefficient rows of stride nd
template <bool GRAD, bool LOCAL>
__device__ __forceinline__ void eval_one_nd(const Tab3& T, const zdc* __restrict__ e, long nd,
                                            int nv, const zdc* x, const zdc* zc, double rscale,
                                            zdc* P, zdc* Gr, zdc* Gt, zdc* Gp) {
  const int p = T.p, L = p + 1;
  const double s4 = 1.0 / sqrt(4 * kPi);
  const double* __restrict__ r1 = T.r1;
  const double* __restrict__ r2 = T.r2;
  const double* __restrict__ sq = T.sq;
  Sph s = zcart2sph(x[0], x[1], x[2], zc);
  zdc rz = s.rz / rscale, irz = zinv(rz);
  const zdc z = s.ct, zz1 = mkz(1.0) - z * z;
  const zdc u = -zsqrt_r(zz1);
  zdc colp = LOCAL ? mkz(1.0) : irz;
  zdc Ydiag = mkz(1.0), em = mkz(1.0);
  for (int m = 0; m <= p; m++) {
    zdc emi = mkz(1.0);
    if (m > 0) {
      double cmm = __ldg(&r1[m * L + m]);
      if (GRAD) Ydiag = (m == 1) ? mkz(-cmm) : (Ydiag * u) * cmm;
      else Ydiag = (Ydiag * u) * cmm;
      em = em * s.eip;
      emi = zinv(em);
      colp = colp * (LOCAL ? rz : irz);
    }
    double sgm = (m & 1) ? -1.0 : 1.0;
    double f0 = s4 * sgm / rscale;
    zdc Yp = Ydiag, Dp = GRAD ? (Ydiag * (double)(-m)) * z : mkz(0.0);
    zdc Ypp = mkz(0.0), Dpp = mkz(0.0);
    zdc rf = colp;
    zdc rfm1 = (LOCAL && m > 0) ? colp * irz : mkz(0.0);
    for (int n = m; n <= p; n++) {
      zdc Y, D = mkz(0.0);
      if (n == m) {
        Y = Yp;
        D = Dp;
      } else {
        if (n == m + 1) {
          double c = __ldg(&r1[n * L + m]);
          Y = (z * Yp) * c;
          if (GRAD) D = (m == 0) ? (z * Dp + Yp) * c : (z * Dp + zz1 * Yp) * c;
        } else {
          double c1 = __ldg(&r1[n * L + m]), c2 = __ldg(&r2[n * L + m]);
          Y = (c1 * z) * Yp - c2 * Ypp;
          if (GRAD)
            D = (m == 0) ? c1 * (z * Dp + Yp) - c2 * Dpp : c1 * (z * Dp + zz1 * Yp) - c2 * Dpp;
        }
        Ypp = Yp; Dpp = Dp; Yp = Y; Dp = D;
        rfm1 = rf;
        rf = rf * (LOCAL ? rz : irz);
      }
      double f = __ldg(&sq[n]) * f0;
      zdc y = Y * f;
      if (m == 0) {
        const zdc* row = e + (long)ix3(n, 0) * nd;
        zdc yr = y * rf, dzr = mkz(0.0), dth = mkz(0.0);
        if (GRAD) {
          zdc dy = D * f;
          if (!LOCAL) {
            dzr = -((double)(n + 1) * y * rf / s.rz);
            dth = -(dy * s.st * rf);
          } else {
            dzr = n == 0 ? mkz(0.0) : ((double)n * rfm1 / rscale) * y;
            dth = -(rf * dy * s.st);
          }
        }
#pragma unroll
        for (int r = 0; r < RBE; r++)
          if (r < nv) {
            zdc c0 = ldz(&row[r]);
            P[r] += c0 * yr;
            if (GRAD) {
              Gr[r] += c0 * dzr;
              Gt[r] += c0 * dth;
            }
          }
      } else {
        const zdc* rowp = e + (long)ix3(n, m) * nd;
        const zdc* rown = e + (long)ix3(n, -m) * nd;
        zdc ys = GRAD ? y * s.st : y;
        zdc ysr = ys * rf, DZ = mkz(0.0), DT = mkz(0.0), DPh = mkz(0.0);
        if (GRAD) {
          zdc dy = D * f;
          if (!LOCAL) {
            DZ = -((double)(n + 1) * ys * rf / s.rz);
            DT = -(dy * rf);
          } else {
            DZ = ((double)n * rfm1 / rscale) * ys;
            DT = -(rf * dy);
          }
          DPh = zmul_i((double)m * y * rf);
        }
#pragma unroll
        for (int r = 0; r < RBE; r++)
          if (r < nv) {
            zdc a = ldz(&rowp[r]) * em, bm = ldz(&rown[r]) * emi;
            zdc Sp = a + bm;
            P[r] += ysr * Sp;
            if (GRAD) {
              Gr[r] += DZ * Sp;
              Gt[r] += DT * Sp;
              Gp[r] += DPh * (a - bm);
            }
          }
      }
    }
  }
}

template <bool GRAD>
__global__ void __launch_bounds__(ENT, 4) k_eval3nd(EvalNdArgs A) {
  const Tab3& T = A.T;
  const int NC = T.NC, tid = threadIdx.x;
  const int b = blockIdx.x;
  if (b >= A.nb) return;
  const int t0 = A.itargse[2 * b], t1 = A.itargse[2 * b + 1];
  if (A.nchild[b] != 0 || t1 < t0) return;
  const int lb = A.ilevel[b];
  const bool own = lb >= 2;
  const int nexp = (own ? 1 : 0) + A.nl3[b];
  if (nexp == 0) return;
  const long nd = A.nd;
  for (int c0 = t0; c0 <= t1; c0 += ENT) {
    const int i = c0 + tid;
    if (i > t1) continue;
    zdc x[3] = {A.ztarg[3 * i], A.ztarg[3 * i + 1], A.ztarg[3 * i + 2]};
    for (int rb = blockIdx.y * RBE; rb < A.nd && rb < (int)(blockIdx.y + 1) * RBE; rb += RBE) {
      const int nv = min(RBE, A.nd - rb);
      zdc P[RBE], Gx[RBE], Gy[RBE], Gz[RBE];
#pragma unroll
      for (int r = 0; r < RBE; r++) P[r] = Gx[r] = Gy[r] = Gz[r] = mkz(0.0);
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
        const zdc* zc = (loc ? A.zct : A.zcs) + 3 * eb;
        const zdc* ex = (loc ? A.loc : A.mp) + (size_t)eb * NC * nd + rb;
        zdc Gr[RBE], Gt[RBE], Gp[RBE], Pe[RBE];
#pragma unroll
        for (int r = 0; r < RBE; r++) Pe[r] = Gr[r] = Gt[r] = Gp[r] = mkz(0.0);
        double rscale = A.rsc[A.ilevel[eb]];
        if (loc) eval_one_nd<GRAD, true>(T, ex, nd, nv, x, zc, rscale, Pe, Gr, Gt, Gp);
        else eval_one_nd<GRAD, false>(T, ex, nd, nv, x, zc, rscale, Pe, Gr, Gt, Gp);
#pragma unroll
        for (int r = 0; r < RBE; r++) P[r] += Pe[r];
        if (GRAD) {
          Sph s = zcart2sph(x[0], x[1], x[2], zc);
          zdc ir = zinv(s.rz);
          zdc ezr0 = s.st * s.cp, ezr1 = s.st * s.sp, ezr2 = s.ct;
          zdc et0 = s.ct * s.cp * ir, et1 = s.ct * s.sp * ir, et2 = -(s.st * ir);
          zdc ep0 = -(s.sp * ir), ep1 = s.cp * ir;
#pragma unroll
          for (int r = 0; r < RBE; r++) {
            Gx[r] += Gr[r] * ezr0 + Gt[r] * et0 + Gp[r] * ep0;
            Gy[r] += Gr[r] * ezr1 + Gt[r] * et1 + Gp[r] * ep1;
            Gz[r] += Gr[r] * ezr2 + Gt[r] * et2;
          }
        }
      }
#pragma unroll
      for (int r = 0; r < RBE; r++)
        if (r < nv) {
          A.pot[(long)i * nd + rb + r] += P[r];
          if (GRAD) {
            A.grad[(3L * i) * nd + rb + r] += Gx[r];
            A.grad[(3L * i + 1) * nd + rb + r] += Gy[r];
            A.grad[(3L * i + 2) * nd + rb + r] += Gz[r];
          }
        }
    }
  }
}

// ---- P2P (list 1) -------------------------------------------------------------
constexpr int PT = 64;  // sources per shared-memory tile

struct P2PNdArgs {
  const int *nchild, *isrcse, *itargse;
  const zdc *zsrc, *q, *ds, *dv, *ztarg;
  const int *nl1, *l1;
  int mn1, nb, nd, ifcharge, ifdipole;
  zdc *pot, *grad;
};

struct SrcTileNd {
  zdc y[PT][3];
  zdc q[PT][RB];
  zdc ds[PT][RB];
  zdc v[PT][3];
};

template <bool GRAD, bool DIP>
__global__ void __launch_bounds__(ENT, 3) k_p2p3nd(P2PNdArgs A) {
  extern __shared__ unsigned char smraw[];
  SrcTileNd& S = *reinterpret_cast<SrcTileNd*>(smraw);
  constexpr double PI4I = 0.079577471545947667884;
  const int b = blockIdx.x;
  if (b >= A.nb) return;
  const int t0 = A.itargse[2 * b], t1 = A.itargse[2 * b + 1];
  if (A.nchild[b] != 0 || t1 < t0 || A.nl1[b] == 0) return;
  const long nd = A.nd;
  for (int c0 = t0; c0 <= t1; c0 += ENT) {
    const int i = c0 + threadIdx.x;
    const bool valid = i <= t1;
    zdc x[3] = {mkz(0.0), mkz(0.0), mkz(0.0)};
    if (valid) {
      x[0] = ldz(&A.ztarg[3 * i]);
      x[1] = ldz(&A.ztarg[3 * i + 1]);
      x[2] = ldz(&A.ztarg[3 * i + 2]);
    }
    for (int rb = blockIdx.y * RB; rb < A.nd && rb < (int)(blockIdx.y + 1) * RB; rb += RB) {
      const int nv = min(RB, A.nd - rb);
      zdc P[RB], G0[RB], G1[RB], G2[RB];
#pragma unroll
      for (int r = 0; r < RB; r++) P[r] = G0[r] = G1[r] = G2[r] = mkz(0.0);
      for (int li = 0; li < A.nl1[b]; li++) {
        const int jb = A.l1[(size_t)b * A.mn1 + li];
        const int s0 = A.isrcse[2 * jb], s1 = A.isrcse[2 * jb + 1];
        for (int j0 = s0; j0 <= s1; j0 += PT) {
          const int n = min(PT, s1 - j0 + 1);
          __syncthreads();
          for (int k = threadIdx.x; k < n; k += ENT) {
            const int j = j0 + k;
            S.y[k][0] = ldz(&A.zsrc[3 * j]);
            S.y[k][1] = ldz(&A.zsrc[3 * j + 1]);
            S.y[k][2] = ldz(&A.zsrc[3 * j + 2]);
            if (DIP) {
              S.v[k][0] = ldz(&A.dv[3 * j]);
              S.v[k][1] = ldz(&A.dv[3 * j + 1]);
              S.v[k][2] = ldz(&A.dv[3 * j + 2]);
            }
          }
          for (int k = threadIdx.x; k < n * RB; k += ENT) {
            const int kk = k / RB, r = k - kk * RB;
            const long off = (long)(j0 + kk) * nd + rb + r;
            S.q[kk][r] = (r < nv && A.ifcharge) ? ldz(&A.q[off]) : mkz(0.0);
            if (DIP) S.ds[kk][r] = r < nv ? ldz(&A.ds[off]) : mkz(0.0);
          }
          __syncthreads();
          if (!valid) continue;
          for (int k = 0; k < n; k++) {
            zdc y0 = S.y[k][0] - x[0], y1 = S.y[k][1] - x[1], y2 = S.y[k][2] - x[2];
            zdc rz = zsqrt_p(y0 * y0 + y1 * y1 + y2 * y2);
            if (!(zabs(rz) > (double)1e-16f)) continue;
            zdc ir = zinv(rz);
            zdc r1 = ir * PI4I;
            zdc r3 = r1 * (ir * ir);
            if (A.ifcharge) {
              // the pair's kernel values once, then one complex MAC per output
              // and right-hand side
              const zdc w0 = r3 * y0, w1 = r3 * y1, w2 = r3 * y2;
#pragma unroll
              for (int r = 0; r < RB; r++) {
                zdc qv = S.q[k][r];
                P[r] += qv * r1;
                if (GRAD) {
                  G0[r] += qv * w0;
                  G1[r] += qv * w1;
                  G2[r] += qv * w2;
                }
              }
            }
            if (DIP) {
              zdc dot = -(y0 * S.v[k][0] + y1 * S.v[k][1] + y2 * S.v[k][2]);
              zdc w3 = r3 * dot;
              zdc dd0 = mkz(0.0), dd1 = mkz(0.0), dd2 = mkz(0.0);
              if (GRAD) {
                zdc t = 3.0 * (dot * (r3 * (ir * ir)));
                dd0 = r3 * S.v[k][0] + t * y0;
                dd1 = r3 * S.v[k][1] + t * y1;
                dd2 = r3 * S.v[k][2] + t * y2;
              }
#pragma unroll
              for (int r = 0; r < RB; r++) {
                zdc dsv = S.ds[k][r];
                P[r] -= dsv * w3;
                if (GRAD) {
                  G0[r] -= dsv * dd0;
                  G1[r] -= dsv * dd1;
                  G2[r] -= dsv * dd2;
                }
              }
            }
          }
        }
      }
      if (valid)
#pragma unroll
        for (int r = 0; r < RB; r++)
          if (r < nv) {
            A.pot[(long)i * nd + rb + r] += P[r];
            if (GRAD) {
              A.grad[(3L * i) * nd + rb + r] += G0[r];
              A.grad[(3L * i + 1) * nd + rb + r] += G1[r];
              A.grad[(3L * i + 2) * nd + rb + r] += G2[r];
            }
          }
    }
  }
}

// ---- host ------------------------------------------------------------------------
template <int KIND, int SLOTS>
void launch_trans_nd_k(const TransNdArgs& A, int grid, size_t sm, cudaStream_t s) {
  ZF_CUDA(cudaFuncSetAttribute(k_trans3nd<KIND, SLOTS>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  klaunch(k_trans3nd<KIND, SLOTS>, grid, XNT, sm, s, A);
}

template <int KIND>
void launch_trans_nd(const TransNdArgs& A, int grid, cudaStream_t s) {
  if (A.hi < A.lo) return;
  grid = std::max(1, std::min(grid, (A.hi - A.lo + 1) * div_up(A.nd, RC)));
  ZF_CUDA(cudaMemsetAsync(A.queue, 0, sizeof(int), s));
  int L = A.T.p + 1;
  TransNdArgs B = A;
  size_t sm = xsm_layout(A.T.p, true, nullptr, nullptr);
  B.rot_smem = sm <= 227 * 1024;
  if (!B.rot_smem) sm = xsm_layout(A.T.p, false, nullptr, nullptr);
  int slots = div_up(L * L, XNT);
  if (slots <= 4) launch_trans_nd_k<KIND, 4>(B, grid, sm, s);
  else if (slots <= 6) launch_trans_nd_k<KIND, 6>(B, grid, sm, s);
  else if (slots <= 8) launch_trans_nd_k<KIND, 8>(B, grid, sm, s);
  else throw zf_error(ZF_ERR_ARG, "expansion order too large for the batched translation");
  ZF_LAUNCH_CHECK();
}

}  // namespace

void plan3d_build(Plan3D& P, double eps, int ns, const zdc* zsrc, int nt, const zdc* ztarg,
                  int isep, cudaStream_t s) {
  if (isep < 1) throw zf_error(ZF_ERR_ARG, "isep must be >= 1");
  P.eps = eps;
  P.isep = isep;
  P.ns = ns;
  P.nt = nt;
  ZF_CUDA(cudaGetDevice(&P.device));
  TreeParams tp;
  tp.D = 3;
  tp.isep = isep;
  tp.idivflag = 0;
  tp.ndiv = lndiv3d(eps, ns, nt);
  tp.lr_isep_quirk = 1;
  setup3d_geom(ns, zsrc, nt, ztarg, tp, P.S, s);
  ZF_CUDA(cudaStreamSynchronize(s));
}

namespace {

// right-hand sides one at a time through the single-solve passes on the plan's
// tree: fewer than kMinBatch right-hand sides (the batched kernels fill 32
// lanes per pass) or orders whose batched working set exceeds shared memory
void lap_plan_loop(const Plan3D& P, int nd, const StrengthsNd& in, int ifpgh, zdc* pot, zdc* grad,
                   cudaStream_t s, StepTimes* times) {
  const Setup3D& S = P.S;
  const int ns = P.ns, nt = P.nt;
  long launches0 = launch_counter();
  const bool timing = times != nullptr;
  cudaEvent_t ev[8];
  if (timing)
    for (auto& e : ev) ZF_CUDA(cudaEventCreate(&e));
  float acc[8] = {0};
  auto mark = [&](int i) {
    if (timing) ZF_CUDA(cudaEventRecord(ev[i], s));
  };
  DevBuf<zdc> q(ns, s), ds(ns, s), dv(3 * (size_t)ns, s), potsort(nt, s),
      gradsort(ifpgh > 1 ? 3 * (size_t)nt : 1, s);
  int p = 0;
  for (int r = 0; r < nd; r++) {
    mark(0);
    gather_strengths_col(S, ns, nd, r, in.ifcharge ? in.charge : nullptr,
                         in.ifdipole ? in.dipstr : nullptr, in.ifdipole ? in.dipvec : nullptr,
                         true, true, q.get(), ds.get(), dv.get(), s);
    potsort.zero();
    gradsort.zero();
    mark(1);
    p = lap_core(S, P.eps, q.get(), ds.get(), dv.get(), in.ifcharge, in.ifdipole, ifpgh,
                 potsort.get(), gradsort.get(), s, timing ? ev : nullptr);
    mark(6);
    unsort3d_col(nt, nd, r, S.itarg.get(), potsort.get(), gradsort.get(), mkz(1.0),
                 mkz(1.0 / S.b0), ifpgh, pot, grad, s);
    mark(7);
    if (timing) {
      ZF_CUDA(cudaEventSynchronize(ev[7]));
      for (int k = 0; k < 7; k++) {
        float ms;
        ZF_CUDA(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
        acc[k] += ms;
      }
    }
  }
  if (timing) {
    for (int k = 0; k < 7; k++) times->ms[k] = acc[k];
    times->nboxes = S.tree.nboxes;
    times->nlevels = S.tree.nlevels;
    times->nterms = p;
    for (auto& e : ev) cudaEventDestroy(e);
    times->launches = launch_counter() - launches0;
    if (times->want_counts) {
      std::vector<int> pl(S.tree.nlevels + 1, p);
      count_interactions3d(S, pl.data(), 1, 1, 2, times, s);
    }
  }
}

constexpr int kMinBatch = 4;

}  // namespace

void zlfmm3d_plan_execute(const Plan3D& P, int nd, const StrengthsNd& in, int ifpgh, zdc* pot,
                          zdc* grad, cudaStream_t s, StepTimes* times) {
  if (nd < kMinBatch ||
      xsm_layout(zl3dterms(P.eps), false, nullptr, nullptr) > 227 * 1024) {
    lap_plan_loop(P, nd, in, ifpgh, pot, grad, s, times);
    return;
  }
  const Setup3D& S = P.S;
  const int ns = P.ns, nt = P.nt;
  long launches0 = launch_counter();
  cudaEvent_t ev[8];
  const bool timing = times != nullptr;
  if (timing)
    for (auto& e : ev) ZF_CUDA(cudaEventCreate(&e));
  auto mark = [&](int i) {
    if (timing) ZF_CUDA(cudaEventRecord(ev[i], s));
  };
  mark(0);
  const DevTree& t = S.tree;
  const DevLists& L = S.lists;
  const int nb = t.nboxes, nlev = t.nlevels;
  const int p = zl3dterms(P.eps);
  Tab3 T = get_tab3(p);
  RotTab R = get_rottab(p);
  const size_t NC = (size_t)T.NC;
  std::vector<double> rsc_h(nlev + 2, 1.0);
  for (int l = 0; l <= nlev; l++) rsc_h[l] = S.bsz[l] > 1.0 ? 1.0 : S.bsz[l];
  DevBuf<double> rsc(rsc_h.size(), s);
  ZF_CUDA(cudaMemcpyAsync(rsc.get(), rsc_h.data(), rsc_h.size() * sizeof(double),
                          cudaMemcpyHostToDevice, s));
  // strengths in tree order, rescaled as the single right-hand-side driver
  DevBuf<zdc> q((size_t)ns * nd, s), ds((size_t)ns * nd, s), dv(3 * (size_t)ns, s);
  gather_strengths_nd(S, ns, nd, in.ifcharge ? in.charge : nullptr,
                      in.ifdipole ? in.dipstr : nullptr, in.ifdipole ? in.dipvec : nullptr,
                      true, true, q.get(), ds.get(), dv.get(), s);
  mark(1);
  DevBuf<zdc> mp(NC * nb * nd, s), loc(NC * nb * nd, s), potsort((size_t)nt * nd, s),
      gradsort(ifpgh > 1 ? 3 * (size_t)nt * nd : 1, s);
  mp.zero();
  loc.zero();
  potsort.zero();
  gradsort.zero();
  int dev = 0, nsm = 148;
  ZF_CUDA(cudaGetDevice(&dev));
  ZF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const int nchunk = div_up(nd, 32);
  // P2M
  FormNdArgs F;
  F.T = T;
  F.ilevel = t.ilevel.get(); F.nchild = t.nchild.get();
  F.isrcse = S.isrcse.get(); F.itargse = S.itargse.get();
  F.zsrc = S.zsrcsort.get(); F.q = q.get(); F.ds = ds.get(); F.dv = dv.get();
  F.zcs = S.zcsrc.get(); F.zct = S.zctarg.get(); F.rsc = rsc.get();
  F.nl4 = L.n[3].get(); F.l4 = L.list[3].get(); F.mn4 = L.mn[3];
  F.nb = nb; F.nd = nd; F.nchunk = nchunk; F.ifcharge = in.ifcharge; F.ifdipole = in.ifdipole;
  const bool dip = in.ifdipole != 0;
  const size_t smf = FW * form_nd_warp_elems(dip) * sizeof(zdc);
  const int fgrid = (int)div_up((long)nb * nchunk, FW);
  auto form = [&](bool local) {
    if (local) {
      if (dip) {
        ZF_CUDA(cudaFuncSetAttribute(k_form3nd<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smf));
        klaunch(k_form3nd<true, true>, fgrid, FW * 32, smf, s, F);
      } else {
        ZF_CUDA(cudaFuncSetAttribute(k_form3nd<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smf));
        klaunch(k_form3nd<true, false>, fgrid, FW * 32, smf, s, F);
      }
    } else {
      if (dip) {
        ZF_CUDA(cudaFuncSetAttribute(k_form3nd<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smf));
        klaunch(k_form3nd<false, true>, fgrid, FW * 32, smf, s, F);
      } else {
        ZF_CUDA(cudaFuncSetAttribute(k_form3nd<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smf));
        klaunch(k_form3nd<false, false>, fgrid, FW * 32, smf, s, F);
      }
    }
    ZF_LAUNCH_CHECK();
  };
  F.out = mp.get();
  if (nlev >= 1) form(false);
  mark(2);
  // translations: a persistent grid of one CTA per SM, scratch per CTA
  const int xgrid = std::max(1, std::min(nsm, nb * nchunk));
  DevBuf<zdc> scratch((size_t)xgrid * 2 * NC * RC, s);
  DevBuf<int> queue(1, s);
  TransNdArgs A;
  A.T = T;
  A.R = R;
  A.ilevel = t.ilevel.get(); A.iparent = t.iparent.get(); A.nchild = t.nchild.get();
  A.ichild = t.ichild.get(); A.isrcse = S.isrcse.get(); A.itargse = S.itargse.get();
  A.zcs = S.zcsrc.get(); A.zct = S.zctarg.get(); A.rsc = rsc.get();
  A.nl2 = L.n[1].get(); A.l2 = L.list[1].get(); A.nl4 = L.n[3].get(); A.mn2 = L.mn[1];
  A.scratch = scratch.get();
  A.queue = queue.get();
  A.nd = nd;
  A.in = mp.get();
  A.out = mp.get();
  for (int l = nlev - 1; l >= 1; l--) {
    A.lo = t.laddr[2 * l];
    A.hi = t.laddr[2 * l + 1];
    launch_trans_nd<0>(A, xgrid, s);
  }
  mark(3);
  A.in = mp.get();
  A.out = loc.get();
  A.lo = 0;
  A.hi = nb - 1;
  launch_trans_nd<1>(A, xgrid, s);
  if (L.mn[3] > 0) {
    F.out = loc.get();
    form(true);
  }
  mark(4);
  A.in = loc.get();
  A.out = loc.get();
  for (int l = 1; l <= nlev - 1; l++) {
    A.lo = t.laddr[2 * (l + 1)];
    A.hi = t.laddr[2 * (l + 1) + 1];
    launch_trans_nd<2>(A, xgrid, s);
  }
  mark(5);
  // P2P, then L2T / M2T
  P2PNdArgs Pa;
  Pa.nchild = t.nchild.get(); Pa.isrcse = S.isrcse.get(); Pa.itargse = S.itargse.get();
  Pa.zsrc = S.zsrcsort.get(); Pa.q = q.get(); Pa.ds = ds.get(); Pa.dv = dv.get();
  Pa.ztarg = S.ztargsort.get();
  Pa.nl1 = L.n[0].get(); Pa.l1 = L.list[0].get(); Pa.mn1 = L.mn[0]; Pa.nb = nb; Pa.nd = nd;
  Pa.ifcharge = in.ifcharge; Pa.ifdipole = in.ifdipole;
  Pa.pot = potsort.get(); Pa.grad = gradsort.get();
  const size_t smp = sizeof(SrcTileNd);
  if (ifpgh > 1) {
    if (dip) {
      ZF_CUDA(cudaFuncSetAttribute(k_p2p3nd<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smp));
      klaunch(k_p2p3nd<true, true>, dim3(nb, div_up(nd, RB)), ENT, smp, s, Pa);
    } else {
      ZF_CUDA(cudaFuncSetAttribute(k_p2p3nd<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smp));
      klaunch(k_p2p3nd<true, false>, dim3(nb, div_up(nd, RB)), ENT, smp, s, Pa);
    }
  } else {
    if (dip) {
      ZF_CUDA(cudaFuncSetAttribute(k_p2p3nd<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smp));
      klaunch(k_p2p3nd<false, true>, dim3(nb, div_up(nd, RB)), ENT, smp, s, Pa);
    } else {
      ZF_CUDA(cudaFuncSetAttribute(k_p2p3nd<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smp));
      klaunch(k_p2p3nd<false, false>, dim3(nb, div_up(nd, RB)), ENT, smp, s, Pa);
    }
  }
  ZF_LAUNCH_CHECK();
  EvalNdArgs E;
  E.T = T;
  E.ilevel = t.ilevel.get(); E.nchild = t.nchild.get(); E.isrcse = S.isrcse.get();
  E.itargse = S.itargse.get(); E.ztarg = S.ztargsort.get(); E.zcs = S.zcsrc.get();
  E.zct = S.zctarg.get(); E.rsc = rsc.get(); E.mp = mp.get(); E.loc = loc.get();
  E.nl3 = L.n[2].get(); E.l3 = L.list[2].get(); E.mn3 = L.mn[2]; E.nb = nb; E.nd = nd;
  E.pot = potsort.get(); E.grad = gradsort.get();
  if (ifpgh > 1) klaunch(k_eval3nd<true>, dim3(nb, div_up(nd, RBE)), ENT, 0, s, E);
  else klaunch(k_eval3nd<false>, dim3(nb, div_up(nd, RBE)), ENT, 0, s, E);
  ZF_LAUNCH_CHECK();
  mark(6);
  unsort3d_nd(nt, nd, S.itarg.get(), potsort.get(), gradsort.get(), mkz(1.0), mkz(1.0 / S.b0),
              ifpgh, pot, grad, s);
  mark(7);
  if (timing) {
    ZF_CUDA(cudaEventSynchronize(ev[7]));
    float ms;
    // steps as the single right-hand-side driver; set-up = the strength gather
    for (int i = 0; i < 7; i++) {
      ZF_CUDA(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]));
      times->ms[i] = ms;
    }
    times->nboxes = nb;
    times->nlevels = nlev;
    times->nterms = p;
    for (auto& e : ev) cudaEventDestroy(e);
    times->launches = launch_counter() - launches0;
    if (times->want_counts) {
      std::vector<int> pl(nlev + 1, p);
      count_interactions3d(S, pl.data(), 1, 1, 2, times, s);
    }
  }
  (void)ns;
}

}  // namespace zf
