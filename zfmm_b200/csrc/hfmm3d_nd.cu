// 3D Helmholtz FMM for many right-hand sides on one geometry (a plan).
//
// The algorithm of zhfmm3d (zfmm3d/src/helmholtz/zhfmm3d.f:256-600) on the
// plan's tree, with the translations batched over the right-hand sides: the
// expansions of every right-hand side live side by side, coefficient (box b of
// level l, n*n+n+m, r) at (base_l + (b - first box of l) (p_l+1)^2 + n*n+n+m) nd
// + r, and one pass of the translation kernel moves 32 right-hand sides
// (one per lane) through the geometry-dependent work of a box pair.
//
//   k_htrans3nd  M2M / M2L / L2L (zh3dmpmp / zh3dmploc / zh3dlocloc,
//                zh3dtrans.f:1-780), one launch per level: z-rotation and
//                point-and-shoot y-rotation of order p1 (the batched rotation
//                shared with the Laplace plans: degree-streamed recurrence
//                states, sample and projection products on FP64 tensor
//                cores), the quadrature z-shift, and the inverse rotations of
//                order p2.  The z-shift evaluates the rotated expansion and its
//                normal derivative at the nq = 2.5 p2 Gauss-Legendre points of a
//                sphere about the new centre and projects them onto the order-p2
//                coefficients.  Its geometry-dependent coefficients (radial
//                functions at every node; per node chunk the value and
//                derivative Legendre columns and the projection columns) are
//                tabulated in shared memory once per box pair; the sums over
//                degrees and nodes then run for the 32 right-hand sides with
//                the lane as the right-hand-side index.
//
//   k_hp2p3nd    list-1 direct interactions: the pair's kernel values (complex
//                distance, e^{ikR}, the gradient factors) once for HRB
//                right-hand sides held in registers.
//   k_heval3nd   L2T / M2T: a thread per target; the radial table and the
//                Legendre recurrences once per (target, expansion) for HRBE
//                right-hand sides.
//
//   k_hform3nd   P2M / P2L: one CTA per (box, 32 right-hand sides), its warps
//                sharing the staged strengths and splitting the orders m; lanes
//                stream the sources' radial tables and recurrences into a small
//                shared buffer, then sum it against the staged strengths
//                (lane = right-hand side).
//
// Fewer than 4 right-hand sides, or orders whose working set exceeds shared
// memory, run every pass per right-hand side.
#include <algorithm>
#include <cmath>
#include <vector>
#include "helm3d_prep.cuh"
#include "helm3d_special.cuh"
#include "hfmm3d.cuh"
#include "lfmm3d.cuh"
#include "plan3d.cuh"
#include "rot3nd.cuh"
#include "sph3d.cuh"

namespace zf {

namespace {

constexpr int QCM = 5;  // nodes per chunk of the z-shift (at most)
constexpr int PB = 8;   // output rows per read-modify-write block of the z-shift
constexpr size_t kHSmemMax = 227 * 1024;

// z-shift tables of one node chunk, aliasing the rotation's work block
struct HSh {
  zdc* node;   // qc x 6: cos, sin of the node's polar angle about the old centre,
               // their ratios to the radius, the node's real sin and cos
  zdc* rad;    // qc x (p1+2): radial functions of the input kind at k r
  zdc* drad;   // qc x (p1+2): their k-scaled derivatives
  zdc* Zc;     // qc x np1: value coefficients of the chunk's nodes, (n, m >= 0) at jdx(n, m)
  zdc* Dc;     // qc x np1: normal-derivative coefficients
  double* Yt;  // qc x np2: projection columns (Legendre at the real node x weight)
};

__host__ __device__ inline size_t hsh_layout(int p1, int p2, int qc, char* base, HSh* o) {
  const size_t P2 = p1 + 2, np1 = (size_t)(p1 + 1) * (p1 + 2) / 2,
               np2 = (size_t)(p2 + 1) * (p2 + 2) / 2;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    void* q = base ? base + off : nullptr;
    off += (bytes + 15) / 16 * 16;
    return q;
  };
  HSh H;
  H.node = (zdc*)take((size_t)qc * 6 * 16);
  H.rad = (zdc*)take((size_t)qc * P2 * 16);
  H.drad = (zdc*)take((size_t)qc * P2 * 16);
  H.Zc = (zdc*)take((size_t)qc * np1 * 16);
  H.Dc = (zdc*)take((size_t)qc * np1 * 16);
  H.Yt = (double*)take((size_t)qc * np2 * 8);
  if (o) *o = H;
  return off;
}

struct HTransNdArgs {
  Tab3 T;  // tables of the largest order, row stride LT
  int LT;
  RotTab R1, R2;  // DFT tables of the two rotation orders
  int p1, p2, pmx, nq, qc, rot_smem;
  double dsc1, dsc2;  // projection-weight rescaling to p1 / p2
  ShiftTab st;
  zdc kwave;
  const int *ilevel, *iparent, *nchild, *ichild, *isrcse, *itargse;
  const zdc *zcs, *zct;
  const zdc* in;
  long base1;  // first coefficient of the input level
  int lo1;     // its first box
  zdc* out;
  long base2;
  int lo2;
  zdc* scratch;
  long scr_per_cta;
  int* queue;  // work-queue counter, zero at launch
  const int *nl2, *l2, *nl4;
  int mn2, nd, lo, hi;
};

// quadrature z-shift of the 32 right-hand sides in X1 (order p1, row stride
// RC) by zsh into X2 (order p2), zh3dmpmp / zh3dmploc / zh3dlocloc after the
// rotations (zh3dtrans.f).  KIND 2 (local input) uses the scaled spherical
// Bessel functions, KIND 0 / 1 (multipole input) the scaled Hankel functions.
template <int KIND>
__device__ void hshift_nd(const HTransNdArgs& A, const HSh& H, zdc zsh, const zdc* X1, zdc* X2) {
  const int p1 = A.p1, p2 = A.p2, nq = A.nq, qc = A.qc, tid = threadIdx.x, lane = tid & 31,
            w = tid >> 5;
  const int P2 = p1 + 2, np1 = (p1 + 1) * (p1 + 2) / 2, np2 = (p2 + 1) * (p2 + 2) / 2;
  const ShiftTab& ST = A.st;
  const int LT = A.LT;
  const double* __restrict__ r1 = A.T.r1;
  const double* __restrict__ r2 = A.T.r2;
  const double* __restrict__ sq = A.T.sq;
  const double s4i = 1.0 / sqrt(4 * kPi);
  if (nq == 0) {  // p2 = 0 configurations have no nodes: the shifted expansion is zero
    for (int idx = tid; idx < (p2 + 1) * (p2 + 1) * RC; idx += XNT) stcg_z(X2 + idx, mkz(0.0));
    __syncthreads();
    return;
  }
  const int ncol = (p1 > p2 ? p1 : p2) + 1;
  const int ntask = 2 * p2 + 1;
  for (int q0 = 0; q0 < nq; q0 += qc) {
    const int nc = min(qc, nq - q0);
    // (a) node geometry and radial tables, one thread per node of the chunk
    for (int t = tid; t < nc; t += XNT) {
      const double x = __ldg(&ST.x[q0 + t]);
      const double yi = sqrt(1 - x * x);
      const zdc zi = zsh + mkz(ST.r * x);
      const zdc ri = zsqrt_r(mkz((ST.r * yi) * (ST.r * yi)) + zi * zi);
      const zdc cthi = zi / ri;
      const zdc sthi = zsqrt_r(mkz(1.0) - cthi * cthi);
      zdc* nd = H.node + 6 * t;
      nd[0] = cthi;
      nd[1] = sthi;
      nd[2] = cthi / ri;
      nd[3] = sthi / ri;
      nd[4] = mkz(yi);
      nd[5] = mkz(x);
      const zdc zk = ri * A.kwave;
      zdc* f = H.rad + (size_t)t * P2;
      zdc* fd = H.drad + (size_t)t * P2;
      if (KIND == 2) besseljs3d_z(p1, zk, ST.rs1, f, fd);
      else h3dall_z(p1, zk, ST.rs1, f, fd);
      for (int n = 0; n <= p1; n++) fd[n] = A.kwave * fd[n];
    }
    __syncthreads();
    // (b) one thread per (node, order m >= 0): the value and normal-derivative
    // coefficients of the expansion's (n, +-m) terms at the node, and the
    // projection column of order m at the real node
    for (int item = tid; item < nc * ncol; item += XNT) {
      const int t = item / ncol, m = item - t * ncol, node = q0 + t;
      const zdc* nd = H.node + 6 * t;
      const double x = nd[5].re, yi = nd[4].re;
      if (m <= p1) {
        const zdc z = nd[0], sthi = nd[1], cr = nd[2], sr = nd[3];
        const zdc zz1 = mkz(1.0) - z * z;
        const zdc u = -zsqrt_r(zz1);
        const zdc* f = H.rad + (size_t)t * P2;
        const zdc* fd = H.drad + (size_t)t * P2;
        zdc* zc = H.Zc + (size_t)t * np1;
        zdc* dc = H.Dc + (size_t)t * np1;
        const double sgm = ((m & 1) ? -1.0 : 1.0) * s4i;
        zdc Ydiag = mkz(1.0);
        for (int k = 1; k <= m; k++) {
          const double ckk = __ldg(&r1[k * LT + k]);
          Ydiag = (k == 1) ? mkz(-ckk) : (Ydiag * u) * ckk;
        }
        zdc Yp = Ydiag, Dp = (Ydiag * (double)(-m)) * z, Ypp = mkz(0.0), Dpp = mkz(0.0);
        for (int n = m; n <= p1; n++) {
          zdc Y, D;
          if (n == m) {
            Y = Yp;
            D = Dp;
          } else {
            if (n == m + 1) {
              const double cc = __ldg(&r1[n * LT + m]);
              Y = (z * Yp) * cc;
              D = (m == 0) ? (z * Dp + Yp) * cc : (z * Dp + zz1 * Yp) * cc;
            } else {
              const double c1 = __ldg(&r1[n * LT + m]), c2 = __ldg(&r2[n * LT + m]);
              Y = (c1 * z) * Yp - c2 * Ypp;
              D = (m == 0) ? c1 * (z * Dp + Yp) - c2 * Dpp : c1 * (z * Dp + zz1 * Yp) - c2 * Dpp;
            }
            Ypp = Yp;
            Dpp = Dp;
            Yp = Y;
            Dp = D;
          }
          const double sc = __ldg(&sq[n]) * sgm;
          const zdc yl = Y * sc, dyl = D * sc;
          const zdc fn = f[n], fdn = fd[n];
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
          const zdc df_x = df_r * sthi + df_th * cr;
          const zdc df_y = df_r * z - df_th * sr;
          zc[jdx(n, m)] = z1;
          dc[jdx(n, m)] = df_x * yi + df_y * x;
        }
      }
      if (m <= p2) {
        // zylgndrf at the real node, times (-1)^m / sqrt(4 pi) and the weight
        const double wq = __ldg(&ST.w[node]) * ((m & 1) ? -1.0 : 1.0) * s4i;
        const double u = -sqrt(1 - x * x);
        double yd = 1.0;
        for (int k = 1; k <= m; k++) yd = (yd * u) * __ldg(&r1[k * LT + k]);
        double yp = yd, ypp = 0.0;
        double* yt = H.Yt + (size_t)t * np2;
        for (int n = m; n <= p2; n++) {
          double y;
          if (n == m) {
            y = yp;
          } else if (n == m + 1) {
            y = (x * yp) * __ldg(&r1[n * LT + m]);
            ypp = yp;
            yp = y;
          } else {
            y = (__ldg(&r1[n * LT + m]) * x) * yp - __ldg(&r2[n * LT + m]) * ypp;
            ypp = yp;
            yp = y;
          }
          yt[jdx(n, m)] = y * __ldg(&sq[n]) * wq;
        }
      }
    }
    __syncthreads();
    // (c) per order m and sign: the node sums of the 32 right-hand sides
    // (lane = right-hand side), then their projection onto the order-p2
    // coefficients (n, +-m), accumulated over the node chunks in X2
    // tasks (m, sign) by decreasing cost, dealt to the warps in snake order
    for (int rnd = 0;; rnd++) {
      const int task = rnd * XW + ((rnd & 1) ? XW - 1 - w : w);
      if (task >= ntask) break;
      const int m = (task + 1) >> 1, mm = (task & 1) ? m : -m;
      zdc F[QCM], D[QCM];
#pragma unroll
      for (int t = 0; t < QCM; t++) F[t] = D[t] = mkz(0.0);
      // the rows of degrees m..p1 in blocks of PB, each block's L2 loads
      // issued together ahead of its products
      for (int n0 = m; n0 <= p1; n0 += PB) {
        zdc a[PB];
#pragma unroll
        for (int k = 0; k < PB; k++)
          a[k] = (n0 + k <= p1) ? ldcg_z(X1 + ix3(n0 + k, mm) * RC + lane) : mkz(0.0);
#pragma unroll
        for (int k = 0; k < PB; k++) {
          if (n0 + k <= p1) {
            const int j = jdx(n0 + k, m);
#pragma unroll
            for (int t = 0; t < QCM; t++) {
              if (t < nc) {
                F[t] += H.Zc[t * np1 + j] * a[k];
                D[t] += H.Dc[t * np1 + j] * a[k];
              }
            }
          }
        }
      }
      // output rows in blocks of PB: the previous chunks' partial sums are
      // fetched together, so their L2 round trips overlap
      for (int nb = m; nb <= p2; nb += PB) {
        zdc old[PB];
#pragma unroll
        for (int k = 0; k < PB; k++)
          old[k] = (q0 > 0 && nb + k <= p2) ? ldcg_z(X2 + ix3(nb + k, mm) * RC + lane) : mkz(0.0);
#pragma unroll
        for (int k = 0; k < PB; k++) {
          const int n = nb + k;
          if (n > p2) break;
          const int j = jdx(n, m);
          zdc sF = mkz(0.0), sD = mkz(0.0);
#pragma unroll
          for (int t = 0; t < QCM; t++) {
            if (t < nc) {
              const double y = H.Yt[t * np2 + j];
              sF += y * F[t];
              sD += y * D[t];
            }
          }
          stcg_z(X2 + ix3(n, mm) * RC + lane, old[k] + ST.cF[n] * sF + ST.cD[n] * sD);
        }
      }
    }
    __syncthreads();
  }
}

template <int KIND, int SLOTS>
__global__ void __launch_bounds__(XNT, 1) k_htrans3nd(HTransNdArgs A) {
  extern __shared__ zdc sm[];
  const int tid = threadIdx.x, p1 = A.p1, p2 = A.p2;
  const int NC1 = (p1 + 1) * (p1 + 1), NC2 = (p2 + 1) * (p2 + 1);
  XSm S;
  xsm_layout(A.pmx, A.rot_smem != 0, sm, &S);
  HSh H;
  hsh_layout(p1, p2, A.qc, (char*)S.Csr, &H);
  if (S.cw) {
    // one rotation order in this launch (p1 = p2): its tables staged once
    const int CP = rot_cp(p1 + 1), TP = rot_tp(p1 + 1);
    for (int k = tid; k < 2 * CP * TP; k += XNT) S.cw[k] = A.R1.cw[k];
  }
  zdc* X1 = A.scratch + (size_t)blockIdx.x * A.scr_per_cta;
  zdc* X2 = X1 + (size_t)NC1 * RC;
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
      // zhfmm3d.f:572-576: ((targets and list 2) or list 4) of the parent,
      // and targets in the child
      if (par < 0 || nsrc(A.itargse, b) <= 0) continue;
      if (!((nsrc(A.itargse, par) > 0 && A.nl2[par] > 0) || A.nl4[par] > 0)) continue;
      nin = 1;
    }
    {
      const int nval = min(RC, A.nd - r0);
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
        const Geo g = geo3(c0, c);
        __syncthreads();
        for (int m = tid; m <= p1; m += XNT) {
          const zdc ef = zpown(g.cb + zmul_i(g.sb), m);
          S.Ef[p1 + m] = ef;
          S.Ef[p1 - m] = zinv(ef);
        }
        for (int m = tid; m <= p2; m += XNT) {
          const zdc eb = zpown(g.cb - zmul_i(g.sb), m);
          S.Eb[p2 + m] = eb;
          S.Eb[p2 - m] = zinv(eb);
        }
        if (g.yr) rot_zero_pad(S, p1);
        __syncthreads();
        const zdc* gin = A.in + (A.base1 + (long)(src - A.lo1) * NC1) * nd + r0;
        if (g.yr)
          rot_nd<SLOTS, 0, 3>(A.T, p1, A.LT, A.dsc1, A.R1, S, g.ca, g.sa, g.zr, gin, nd, X1, RC,
                              nval);
        else
          copy_nd<0, 3>(A.T, p1, S, g.zr, gin, nd, X1, RC, nval);
        __syncthreads();
        hshift_nd<KIND>(A, H, g.zz, X1, X2);
        zdc* gout = A.out + (A.base2 + (long)(b - A.lo2) * NC2) * nd + r0;
        if (g.yr) {
          rot_zero_pad(S, p2);
          __syncthreads();
          rot_nd<SLOTS, 1, 3>(A.T, p2, A.LT, A.dsc2, A.R2, S, g.ca, -g.sa, g.zr, X2, RC, gout, nd,
                              nval);
        } else {
          copy_nd<1, 3>(A.T, p2, S, g.zr, X2, RC, gout, nd, nval);
        }
      }
    }
  }
}

// ---- P2P (list 1), RB right-hand sides per thread pass ---------------------------
constexpr int HNDT = 128;  // threads of the batched P2P and evaluation kernels
constexpr int HRB = 8;     // right-hand sides per thread pass of the P2P kernel
constexpr int HRBE = 4;    // right-hand sides per thread pass of the L2T / M2T kernel
constexpr int HPT = 64;    // sources per shared-memory tile

struct HP2PNdArgs {
  const int *nchild, *isrcse, *itargse;
  const zdc *zsrc, *q, *ds, *dv, *ztarg;
  const int *nl1, *l1;
  int mn1, nb, nd, ifcharge;
  zdc zk;
  zdc *pot, *grad;
};

struct HSrcTileNd {
  zdc y[HPT][3];
  zdc q[HPT][HRB];
  zdc ds[HPT][HRB];
  zdc v[HPT][3];
};

// the pair interaction of zh3devaldirect (zhfmm3d.f:626-693): the pair's kernel
// values once, then one complex MAC per output and right-hand side
template <bool GRAD, bool DIP>
__global__ void __launch_bounds__(HNDT, 3) k_hp2p3nd(HP2PNdArgs A) {
  extern __shared__ unsigned char smraw[];
  HSrcTileNd& S = *reinterpret_cast<HSrcTileNd*>(smraw);
  constexpr double PI4I = 0.079577471545947667884;
  const int b = blockIdx.x;
  if (b >= A.nb) return;
  const int t0 = A.itargse[2 * b], t1 = A.itargse[2 * b + 1];
  if (A.nchild[b] != 0 || t1 < t0 || A.nl1[b] == 0) return;
  const long nd = A.nd;
  const zdc zk = A.zk, zk2 = zk * zk;
  for (int c0 = t0; c0 <= t1; c0 += HNDT) {
    const int i = c0 + threadIdx.x;
    const bool valid = i <= t1;
    zdc x[3] = {mkz(0.0), mkz(0.0), mkz(0.0)};
    if (valid) {
      x[0] = ldz(&A.ztarg[3 * i]);
      x[1] = ldz(&A.ztarg[3 * i + 1]);
      x[2] = ldz(&A.ztarg[3 * i + 2]);
    }
    const int rb = blockIdx.y * HRB;
    const int nv = min(HRB, A.nd - rb);
    zdc P[HRB], G0[HRB], G1[HRB], G2[HRB];
#pragma unroll
    for (int r = 0; r < HRB; r++) P[r] = G0[r] = G1[r] = G2[r] = mkz(0.0);
    for (int li = 0; li < A.nl1[b]; li++) {
      const int jb = A.l1[(size_t)b * A.mn1 + li];
      const int s0 = A.isrcse[2 * jb], s1 = A.isrcse[2 * jb + 1];
      for (int j0 = s0; j0 <= s1; j0 += HPT) {
        const int n = min(HPT, s1 - j0 + 1);
        __syncthreads();
        for (int k = threadIdx.x; k < n; k += HNDT) {
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
        for (int k = threadIdx.x; k < n * HRB; k += HNDT) {
          const int kk = k / HRB, r = k - kk * HRB;
          const long off = (long)(j0 + kk) * nd + rb + r;
          S.q[kk][r] = (r < nv && A.ifcharge) ? ldz(&A.q[off]) : mkz(0.0);
          if (DIP) S.ds[kk][r] = r < nv ? ldz(&A.ds[off]) : mkz(0.0);
        }
        __syncthreads();
        if (!valid) continue;
        for (int k = 0; k < n; k++) {
          const zdc x0 = x[0] - S.y[k][0], x1 = x[1] - S.y[k][1], x2 = x[2] - S.y[k][2];
          const zdc rz = zsqrt_p(x0 * x0 + x1 * x1 + x2 * x2);
          if (!(zabs(rz) > (double)1e-16f)) continue;
          const zdc z = zmul_i(zk * rz);
          const zdc ez = zexp_p(z);
          const zdc ir = zinv(rz);
          const zdc r1 = ir * PI4I;
          const zdc r3 = r1 * (ir * ir);
          const zdc t4 = mkz(1.0) - z;
          if (A.ifcharge) {
            const zdc kq = ez * r1, hq = ez * t4 * r3;
            const zdc w0 = -(hq * x0), w1 = -(hq * x1), w2 = -(hq * x2);
#pragma unroll
            for (int r = 0; r < HRB; r++) {
              const zdc qv = S.q[k][r];
              P[r] += qv * kq;
              if (GRAD) {
                G0[r] += qv * w0;
                G1[r] += qv * w1;
                G2[r] += qv * w2;
              }
            }
          }
          if (DIP) {
            const zdc dot = x0 * S.v[k][0] + x1 * S.v[k][1] + x2 * S.v[k][2];
            const zdc e3 = ez * r3;
            const zdc kd = -(e3 * dot * t4);
            zdc d0 = mkz(0.0), d1 = mkz(0.0), d2 = mkz(0.0);
            if (GRAD) {
              const zdc tt1 = dot * e3 * (zk2 - 3.0 * (t4 * (ir * ir)));
              const zdc tt2 = t4 * e3;
              d0 = -(S.v[k][0] * tt2 + x0 * tt1);
              d1 = -(S.v[k][1] * tt2 + x1 * tt1);
              d2 = -(S.v[k][2] * tt2 + x2 * tt1);
            }
#pragma unroll
            for (int r = 0; r < HRB; r++) {
              const zdc dsv = S.ds[k][r];
              P[r] += dsv * kd;
              if (GRAD) {
                G0[r] += dsv * d0;
                G1[r] += dsv * d1;
                G2[r] += dsv * d2;
              }
            }
          }
        }
      }
    }
    if (valid)
#pragma unroll
      for (int r = 0; r < HRB; r++)
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

// ---- L2T / M2T, HRBE right-hand sides per thread pass ---------------------------
struct HEvalNdArgs {
  const double *r1, *r2, *sq;
  int L;
  const int *ilevel, *nchild, *isrcse, *itargse;
  const zdc *ztarg, *zcs, *zct;
  HLev lev;
  const zdc *mp, *loc;
  const int *nl3, *l3;
  int mn3, nb, nd;
  zdc zk;
  zdc *pot, *grad;
};

// zh3devalmp (LOCAL = false: h_n) / zh3devalloc (LOCAL = true: j_n) of one
// target for nv <= HRBE right-hand sides; e: coefficient rows of stride nd.
// The radial table and the Legendre recurrences are formed once and applied
// to every right-hand side; the gradient accumulates in spherical components.
template <bool GRAD, bool LOCAL>
__device__ __forceinline__ void heval_one_nd(const HEvalNdArgs& A, const zdc* __restrict__ e,
                                             long nd, int nv, int p, const Sph& s, double rscale,
                                             zdc* P, zdc* Gr, zdc* Gt, zdc* Gp) {
  const int L = A.L;
  zdc f[PMAXR + 2], fd[GRAD ? PMAXR + 2 : 1];
  const zdc zrk = s.rz * A.zk;
  if (!LOCAL) h3dall_z(p, zrk, rscale, f, GRAD ? fd : nullptr);
  else besseljs3d_z(p, zrk, rscale, f, GRAD ? fd : nullptr);
  const zdc z = s.ct, zz1 = mkz(1.0) - z * z;
  const zdc u = -zsqrt_r(zz1);
  zdc Ydiag = mkz(1.0), em = mkz(1.0);
  for (int m = 0; m <= p; m++) {
    zdc emi = mkz(1.0);
    if (m > 0) {
      const double cmm = __ldg(&A.r1[m * L + m]);
      if (GRAD) Ydiag = (m == 1) ? mkz(-cmm) : (Ydiag * u) * cmm;
      else Ydiag = (Ydiag * u) * cmm;
      em = em * s.eip;
      emi = zinv(em);
    }
    const double sgm = (m & 1) ? -1.0 : 1.0;
    zdc Yp = Ydiag, Dp = GRAD ? (Ydiag * (double)(-m)) * z : mkz(0.0);
    zdc Ypp = mkz(0.0), Dpp = mkz(0.0);
    for (int n = m; n <= p; n++) {
      zdc Y, D = mkz(0.0);
      if (n == m) {
        Y = Yp;
        D = Dp;
      } else {
        if (n == m + 1) {
          const double c = __ldg(&A.r1[n * L + m]);
          Y = (z * Yp) * c;
          if (GRAD) D = (m == 0) ? (z * Dp + Yp) * c : (z * Dp + zz1 * Yp) * c;
        } else {
          const double c1 = __ldg(&A.r1[n * L + m]), c2 = __ldg(&A.r2[n * L + m]);
          Y = (c1 * z) * Yp - c2 * Ypp;
          if (GRAD)
            D = (m == 0) ? c1 * (z * Dp + Yp) - c2 * Dpp : c1 * (z * Dp + zz1 * Yp) - c2 * Dpp;
        }
        Ypp = Yp;
        Dpp = Dp;
        Yp = Y;
        Dp = D;
      }
      const double sc = __ldg(&A.sq[n]) * sgm;
      const zdc y = Y * sc;
      if (m == 0) {
        const zdc* row = e + (long)ix3(n, 0) * nd;
        const zdc bP = f[n] * y;
        zdc bR = mkz(0.0), bT = mkz(0.0);
        if (GRAD) {
          const zdc dy = D * sc;
          bR = A.zk * fd[n] * y;
          bT = -(f[n] * dy * s.st);
        }
#pragma unroll
        for (int r = 0; r < HRBE; r++)
          if (r < nv) {
            const zdc a0 = ldz(&row[r]);
            P[r] += a0 * bP;
            if (GRAD) {
              Gr[r] += a0 * bR;
              Gt[r] += a0 * bT;
            }
          }
      } else {
        const zdc* rowp = e + (long)ix3(n, m) * nd;
        const zdc* rown = e + (long)ix3(n, -m) * nd;
        const zdc bP = GRAD ? f[n] * y * s.st : f[n] * y;
        zdc bR = mkz(0.0), bT = mkz(0.0), bF = mkz(0.0);
        if (GRAD) {
          const zdc dy = D * sc;
          bR = A.zk * fd[n] * y * s.st;
          bT = -(f[n] * dy);
          bF = zmul_i((double)m * f[n] * y);
        }
#pragma unroll
        for (int r = 0; r < HRBE; r++)
          if (r < nv) {
            const zdc z1 = ldz(&rowp[r]) * em, z2 = ldz(&rown[r]) * emi;
            const zdc Sp = z1 + z2;
            P[r] += bP * Sp;
            if (GRAD) {
              Gr[r] += bR * Sp;
              Gt[r] += bT * Sp;
              Gp[r] += bF * (z1 - z2);
            }
          }
      }
    }
  }
}

template <bool GRAD>
__global__ void __launch_bounds__(HNDT, 4) k_heval3nd(HEvalNdArgs A) {
  const int tid = threadIdx.x;
  const int b = blockIdx.x;
  if (b >= A.nb) return;
  const int t0 = A.itargse[2 * b], t1 = A.itargse[2 * b + 1];
  if (A.nchild[b] != 0 || t1 < t0) return;
  const int lb = A.ilevel[b];
  const bool own = lb >= 2;  // levels 0 and 1 receive no local expansion
  const int nexp = (own ? 1 : 0) + A.nl3[b];
  if (nexp == 0) return;
  const long nd = A.nd;
  const int rb = blockIdx.y * HRBE;
  const int nv = min(HRBE, A.nd - rb);
  for (int c0 = t0; c0 <= t1; c0 += HNDT) {
    const int i = c0 + tid;
    if (i > t1) continue;
    const zdc x[3] = {A.ztarg[3 * i], A.ztarg[3 * i + 1], A.ztarg[3 * i + 2]};
    zdc P[HRBE], Gx[HRBE], Gy[HRBE], Gz[HRBE];
#pragma unroll
    for (int r = 0; r < HRBE; r++) P[r] = Gx[r] = Gy[r] = Gz[r] = mkz(0.0);
    for (int ei = 0; ei < nexp; ei++) {
      int eb;
      bool loc;
      if (own && ei == 0) {
        eb = b;
        loc = true;
      } else {
        eb = A.l3[(size_t)b * A.mn3 + ei - (own ? 1 : 0)];
        loc = false;
        if (nsrc(A.isrcse, eb) <= 0) continue;
      }
      const int le = A.ilevel[eb], p = A.lev.p[le], NC = (p + 1) * (p + 1);
      const zdc* zc = (loc ? A.zct : A.zcs) + 3 * eb;
      const zdc* ex =
          (loc ? A.loc : A.mp) + (A.lev.base[le] + (long)(eb - A.lev.lo[le]) * NC) * nd + rb;
      const Sph s = zcart2sph(x[0], x[1], x[2], zc);
      zdc Gr[HRBE], Gt[HRBE], Gp[HRBE];
#pragma unroll
      for (int r = 0; r < HRBE; r++) Gr[r] = Gt[r] = Gp[r] = mkz(0.0);
      if (loc) heval_one_nd<GRAD, true>(A, ex, nd, nv, p, s, A.lev.rs[le], P, Gr, Gt, Gp);
      else heval_one_nd<GRAD, false>(A, ex, nd, nv, p, s, A.lev.rs[le], P, Gr, Gt, Gp);
      if (GRAD) {
        const zdc ir = zinv(s.rz);
        const zdc ezr0 = s.st * s.cp, ezr1 = s.st * s.sp, ezr2 = s.ct;
        const zdc et0 = s.ct * s.cp * ir, et1 = s.ct * s.sp * ir, et2 = -(s.st * ir);
        const zdc ep0 = -(s.sp * ir), ep1 = s.cp * ir;
#pragma unroll
        for (int r = 0; r < HRBE; r++) {
          Gx[r] += Gr[r] * ezr0 + Gt[r] * et0 + Gp[r] * ep0;
          Gy[r] += Gr[r] * ezr1 + Gt[r] * et1 + Gp[r] * ep1;
          Gz[r] += Gr[r] * ezr2 + Gt[r] * et2;
        }
      }
    }
#pragma unroll
    for (int r = 0; r < HRBE; r++)
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

// ---- P2M / P2L, one warp per (box, 32 right-hand sides) -------------------------
constexpr int HFW = 4;  // warps per CTA of the form kernel, sharing one work item
constexpr int HKB = 2;  // (n, m) entries buffered per flush

struct HFormNdArgs {
  const double *r1, *r2, *sq;
  int L;
  const int *ilevel, *nchild, *isrcse, *itargse;
  const zdc *zsrc, *q, *ds, *dv;
  const zdc *zcs, *zct;
  HLev lev;
  zdc* out;
  const int *nl4, *l4;
  int mn4, nb, nd, nchunk, ifcharge;
  zdc zk;
};

// shared memory of a form CTA: the staged strengths (32 sources x 32
// right-hand sides, charges and dipole strengths) and per warp the buffered
// coefficient weights of HKB (n, +-m) entries
__host__ __device__ inline size_t hform_nd_elems(bool dip) {
  return (dip ? 2 : 1) * (32 * 32 + HFW * HKB * 2 * 32);
}

// zh3dformmp (LOCAL = false: j_n) / zh3dformloc (LOCAL = true: h_n) of sources
// s0..s1 about centre zc at order p into the 32 right-hand sides r0.. of `o`
// (coefficient rows of stride nd).  The CTA's warps share each 32-source
// strength tile; warp w takes the orders m = w, w + HFW, ...: its lanes stream
// one source each through the radial table and the order-m Legendre column,
// buffering the coefficient weights of HKB (n, +-m) entries, and a flush sums
// them against the staged strengths with the lane as the right-hand side.
// The warps write disjoint coefficient rows.
template <bool LOCAL, bool DIP>
__device__ void hform_range_nd(const HFormNdArgs& A, int s0, int s1, const zdc* zc, int p,
                               double rscale, zdc* o, int r0, int nval, zdc* Qt, zdc* Dt,
                               zdc* Gq, zdc* Gd) {
  const int L = A.L, tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const long nd = A.nd;
  const zdc zk = A.zk;
  const zdc c4 = zmul_i(zk * (1.0 / (4 * kPi)));
  zdc f[PMAXR + 2], fd[DIP ? PMAXR + 2 : 1];
  for (int base = s0; base <= s1; base += 32) {
    const int cnt = min(32, s1 - base + 1);
    __syncthreads();
    for (int k = w; k < 32; k += HFW) {
      const bool ok = k < cnt && lane < nval;
      Qt[k * 32 + lane] = (ok && A.ifcharge) ? A.q[(long)(base + k) * nd + r0 + lane] : mkz(0.0);
      if (DIP) Dt[k * 32 + lane] = ok ? A.ds[(long)(base + k) * nd + r0 + lane] : mkz(0.0);
    }
    __syncthreads();
    const bool valid = lane < cnt;
    const int ii = valid ? base + lane : base;
    const Sph s = zcart2sph(A.zsrc[3 * ii], A.zsrc[3 * ii + 1], A.zsrc[3 * ii + 2], zc);
    const zdc zrk = s.rz * zk;
    if (!LOCAL) besseljs3d_z(p, zrk, rscale, f, DIP ? fd : nullptr);
    else h3dall_z(p, zrk, rscale, f, DIP ? fd : nullptr);
    zdc dzr_ = mkz(0.0), dthz = mkz(0.0), dphz = mkz(0.0);
    if (DIP) {
      const zdc v0 = A.dv[3 * ii], v1 = A.dv[3 * ii + 1], v2 = A.dv[3 * ii + 2];
      dzr_ = v0 * (s.st * s.cp) + v1 * (s.st * s.sp) + v2 * s.ct;
      const zdc dth_ = v0 * (s.ct * s.cp) + v1 * (s.ct * s.sp) - v2 * s.st;
      const zdc dph_ = -(v0 * s.sp) + v1 * s.cp;
      dthz = dth_ / s.rz;
      dphz = dph_ / s.rz;
    }
    const zdc z = s.ct, zz1 = mkz(1.0) - z * z;
    const zdc u = -zsqrt_r(zz1);
    int e = 0, fm = 0, fn = 0;  // buffered entries and the first (m, n) among them
    auto flush = [&]() {
      __syncwarp();
      int m = fm, n = fn;
      for (int k = 0; k < e; k++) {
        zdc ap = mkz(0.0), an = mkz(0.0);
        const zdc* gq = Gq + k * 64;
        const zdc* gd = Gd + k * 64;
        for (int j = 0; j < 32; j++) {
          const zdc qv = Qt[j * 32 + lane];
          ap += gq[j] * qv;
          if (m > 0) an += gq[32 + j] * qv;
          if (DIP) {
            const zdc dvv = Dt[j * 32 + lane];
            ap += gd[j] * dvv;
            if (m > 0) an += gd[32 + j] * dvv;
          }
        }
        if (lane < nval) {
          o[(long)ix3(n, m) * nd + lane] += ap;
          if (m > 0) o[(long)ix3(n, -m) * nd + lane] += an;
        }
        if (n < p) n++;
        else {
          m += HFW;
          n = m;
        }
      }
      __syncwarp();
      e = 0;
    };
    // Ydiag(m) and eip^m as the single-solve kernel forms them (running
    // products over m), advanced here to this warp's orders
    zdc Ydiag = mkz(1.0), em = mkz(1.0);
    int mdone = 0;
    for (int m = w; m <= p; m += HFW) {
      for (int k = mdone + 1; k <= m; k++) {
        const double ckk = __ldg(&A.r1[k * L + k]);
        if (DIP) Ydiag = (k == 1) ? mkz(-ckk) : (Ydiag * u) * ckk;
        else Ydiag = (Ydiag * u) * ckk;
        em = em * s.eip;
      }
      mdone = m;
      const zdc emi = m > 0 ? zinv(em) : mkz(1.0);
      const double sgm = (m & 1) ? -1.0 : 1.0;
      zdc Yp = Ydiag, Dp = DIP ? (Ydiag * (double)(-m)) * z : mkz(0.0);
      zdc Ypp = mkz(0.0), Dpp = mkz(0.0);
      for (int n = m; n <= p; n++) {
        zdc Y, D = mkz(0.0);
        if (n == m) {
          Y = Yp;
          D = Dp;
        } else {
          if (n == m + 1) {
            const double c = __ldg(&A.r1[n * L + m]);
            Y = (z * Yp) * c;
            if (DIP) D = (m == 0) ? (z * Dp + Yp) * c : (z * Dp + zz1 * Yp) * c;
          } else {
            const double c1 = __ldg(&A.r1[n * L + m]), c2 = __ldg(&A.r2[n * L + m]);
            Y = (c1 * z) * Yp - c2 * Ypp;
            if (DIP)
              D = (m == 0) ? c1 * (z * Dp + Yp) - c2 * Dpp : c1 * (z * Dp + zz1 * Yp) - c2 * Dpp;
          }
          Ypp = Yp;
          Dpp = Dp;
          Yp = Y;
          Dp = D;
        }
        const zdc sc = c4 * (__ldg(&A.sq[n]) * sgm);
        const zdc y = Y * sc, dy = D * sc;
        zdc qp, qn = mkz(0.0), dp = mkz(0.0), dn = mkz(0.0);
        if (m == 0) {
          qp = f[n] * y;
          if (DIP) dp = -(zk * fd[n] * y * dzr_) + f[n] * dy * s.st * dthz;
        } else {
          const zdc X = f[n] * (DIP ? y * s.st : y);
          qp = emi * X;
          qn = em * X;
          if (DIP) {
            const zdc Xd = -(zk * fd[n] * y * s.st * dzr_) + f[n] * dy * dthz;
            const zdc W = zmul_i((double)m * f[n] * y * dphz);
            dp = emi * (Xd + W);
            dn = em * (Xd - W);
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
        if (e == HKB) flush();
      }
    }
    if (e > 0) flush();
  }
}

template <bool LOCAL, bool DIP>
__global__ void __launch_bounds__(HFW * 32) k_hform3nd(HFormNdArgs A) {
  extern __shared__ zdc sm[];
  const int w = threadIdx.x >> 5;
  const long item = blockIdx.x;
  if (item >= (long)A.nb * A.nchunk) return;
  const int b = (int)(item / A.nchunk), r0 = (int)(item % A.nchunk) * 32;
  const int nval = min(32, A.nd - r0);
  zdc* Qt = sm;
  zdc* Dt = Qt + 32 * 32;
  zdc* Gq = Dt + (DIP ? 32 * 32 : 0) + (size_t)w * HKB * 2 * 32 * (DIP ? 2 : 1);
  zdc* Gd = Gq + HKB * 2 * 32;
  const int l = A.ilevel[b];
  const int p = A.lev.p[l], NC = (p + 1) * (p + 1);
  zdc* o = A.out + (A.lev.base[l] + (long)(b - A.lev.lo[l]) * NC) * A.nd + r0;
  if (!LOCAL) {
    // leaves at levels >= 2 (zhfmm3d.f: the multipoles of levels 0 and 1 are never read)
    if (A.nchild[b] != 0 || nsrc(A.isrcse, b) <= 0 || l < 2) return;
    hform_range_nd<false, DIP>(A, A.isrcse[2 * b], A.isrcse[2 * b + 1], A.zcs + 3 * b, p,
                               A.lev.rs[l], o, r0, nval, Qt, Dt, Gq, Gd);
  } else {
    if (nsrc(A.itargse, b) <= 0 || A.nl4[b] == 0) return;
    for (int i = 0; i < A.nl4[b]; i++) {
      const int jb = A.l4[(size_t)b * A.mn4 + i];
      if (nsrc(A.isrcse, jb) <= 0) continue;
      hform_range_nd<true, DIP>(A, A.isrcse[2 * jb], A.isrcse[2 * jb + 1], A.zct + 3 * b, p,
                                A.lev.rs[l], o, r0, nval, Qt, Dt, Gq, Gd);
    }
  }
}

// one translation launch: its orders, node count and shared-memory plan
struct HLaunch {
  int p1, p2, nq, qc, slots, rot_smem;
  size_t smem;
  bool ok;
};

HLaunch plan_launch(int p1, int p2, int nq) {
  HLaunch h{p1, p2, nq, 0, 0, 0, 0, false};
  const int pmx = std::max(p1, p2);
  h.slots = div_up((long)(pmx + 1) * (pmx + 1), XNT);
  if (h.slots > 8) return h;
  for (int tab = (p1 == p2) ? 1 : 0; tab >= 0; tab--) {
    const size_t off = xsm_work_offset(pmx, tab != 0);
    const size_t rot = xsm_layout(pmx, tab != 0, nullptr, nullptr) - off;
    for (int qc = QCM; qc >= 1; qc--) {
      const size_t tot = off + std::max(rot, hsh_layout(p1, p2, qc, nullptr, nullptr));
      if (tot <= kHSmemMax) {
        h.qc = qc;
        h.rot_smem = tab;
        h.smem = tot;
        h.ok = true;
        return h;
      }
    }
  }
  return h;
}

template <int KIND, int SLOTS>
void launch_htrans_nd_k(const HTransNdArgs& A, int grid, size_t sm, cudaStream_t s) {
  ZF_CUDA(cudaFuncSetAttribute(k_htrans3nd<KIND, SLOTS>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  klaunch(k_htrans3nd<KIND, SLOTS>, grid, XNT, sm, s, A);
}

// boxes lo..hi of output level l2 from input level l1
template <int KIND>
void launch_htrans_nd(HTransNdArgs A, const HelmPrep& H, int l1, int l2, int lo, int hi,
                      int grid, cudaStream_t s) {
  if (hi < lo) return;
  const ShiftTab& st = H.sth[KIND * ML + l2];
  const int p1 = H.lev.p[l1], p2 = H.lev.p[l2];
  const HLaunch h = plan_launch(p1, p2, st.nq);
  if (!h.ok) throw zf_error(ZF_ERR_ARG, "expansion order too large for the batched translation");
  A.p1 = p1;
  A.p2 = p2;
  A.pmx = std::max(p1, p2);
  A.nq = st.nq;
  A.qc = h.qc;
  A.rot_smem = h.rot_smem;
  A.R1 = get_rottab(p1);
  A.R2 = get_rottab(p2);
  A.dsc1 = (2.0 * H.pmax + 1.0) / (2.0 * p1 + 1.0);
  A.dsc2 = (2.0 * H.pmax + 1.0) / (2.0 * p2 + 1.0);
  A.st = st;
  A.base1 = H.lev.base[l1];
  A.lo1 = H.lev.lo[l1];
  A.base2 = H.lev.base[l2];
  A.lo2 = H.lev.lo[l2];
  A.lo = lo;
  A.hi = hi;
  grid = std::max(1, std::min(grid, (hi - lo + 1) * div_up(A.nd, RC)));
  ZF_CUDA(cudaMemsetAsync(A.queue, 0, sizeof(int), s));
  switch (h.slots) {
    case 1: case 2: case 3: case 4: launch_htrans_nd_k<KIND, 4>(A, grid, h.smem, s); break;
    case 5: case 6: launch_htrans_nd_k<KIND, 6>(A, grid, h.smem, s); break;
    default: launch_htrans_nd_k<KIND, 8>(A, grid, h.smem, s); break;
  }
  ZF_LAUNCH_CHECK();
}

constexpr int kMinBatchH = 4;

// every translation launch of the solve fits the batched kernel
bool batched_fits(const Setup3D& S, const HelmPrep& H) {
  const int nlev = S.tree.nlevels;
  for (int l = 2; l <= nlev; l++) {
    for (int kind = 0; kind < 3; kind++) {
      int l1;
      if (kind == 0) {
        if (l >= nlev) continue;
        l1 = l + 1;
      } else if (kind == 1) {
        l1 = l;
      } else {
        if (l < 3) continue;
        l1 = l - 1;
      }
      if (!plan_launch(H.lev.p[l1], H.lev.p[l], H.sth[kind * ML + l].nq).ok) return false;
    }
  }
  return true;
}

}  // namespace

void zhfmm3d_plan_execute(const Plan3D& P, zdc zk, int nd, const StrengthsNd& in, int ifpgh,
                          zdc* pot, zdc* grad, cudaStream_t s, StepTimes* times) {
  const Setup3D& S = P.S;
  const int ns = P.ns, nt = P.nt;
  const bool timing = times != nullptr;
  cudaEvent_t ev[8];
  if (timing)
    for (auto& e : ev) ZF_CUDA(cudaEventCreate(&e));
  auto mark = [&](int i) {
    if (timing) ZF_CUDA(cudaEventRecord(ev[i], s));
  };
  long launches0 = launch_counter();
  mark(0);
  HelmPrep H;
  helm_prep(S, P.eps, zk, P.isep, H, s);
  mark(1);
  if (nd < kMinBatchH || !batched_fits(S, H)) {
    float prep_ms = 0;
    if (timing) {
      ZF_CUDA(cudaEventSynchronize(ev[1]));
      ZF_CUDA(cudaEventElapsedTime(&prep_ms, ev[0], ev[1]));
      for (auto& e : ev) cudaEventDestroy(e);
    }
    helm_plan_loop(P, H, nd, in, ifpgh, pot, grad, s, times, prep_ms);
    return;
  }
  const DevTree& t = S.tree;
  const DevLists& L = S.lists;
  const int nb = t.nboxes, nlev = t.nlevels;
  const long tot = std::max<long>(H.tot, 1);
  DevBuf<zdc> dv(3 * (size_t)ns, s), mpn((size_t)tot * nd, s), locn((size_t)tot * nd, s);
  mpn.zero();
  locn.zero();
  // tree-order strengths with the right-hand side fastest (the gather writes
  // every strength entry, dipole strengths included)
  DevBuf<zdc> qn((size_t)ns * nd, s), dsn((size_t)ns * nd, s);
  gather_strengths_nd(S, ns, nd, in.ifcharge ? in.charge : nullptr,
                      in.ifdipole ? in.dipstr : nullptr, in.ifdipole ? in.dipvec : nullptr, true,
                      true, qn.get(), dsn.get(), dv.get(), s);
  // P2M, and P2L (list 4) before the M2L launches add to it
  const bool dip = in.ifdipole != 0;
  {
    HFormNdArgs F;
    F.r1 = H.T.r1; F.r2 = H.T.r2; F.sq = H.T.sq; F.L = H.pmax + 1;
    F.ilevel = t.ilevel.get(); F.nchild = t.nchild.get();
    F.isrcse = S.isrcse.get(); F.itargse = S.itargse.get();
    F.zsrc = S.zsrcsort.get(); F.q = qn.get(); F.ds = dsn.get(); F.dv = dv.get();
    F.zcs = S.zcsrc.get(); F.zct = S.zctarg.get(); F.lev = H.lev;
    F.nl4 = L.n[3].get(); F.l4 = L.list[3].get(); F.mn4 = L.mn[3];
    F.nb = nb; F.nd = nd; F.nchunk = div_up(nd, 32); F.ifcharge = in.ifcharge; F.zk = H.kw;
    const size_t smf = hform_nd_elems(dip) * sizeof(zdc);
    const int fgrid = nb * F.nchunk;
    auto form = [&](bool local) {
      if (local) {
        if (dip) {
          ZF_CUDA(cudaFuncSetAttribute(k_hform3nd<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smf));
          klaunch(k_hform3nd<true, true>, fgrid, HFW * 32, smf, s, F);
        } else {
          ZF_CUDA(cudaFuncSetAttribute(k_hform3nd<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smf));
          klaunch(k_hform3nd<true, false>, fgrid, HFW * 32, smf, s, F);
        }
      } else {
        if (dip) {
          ZF_CUDA(cudaFuncSetAttribute(k_hform3nd<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smf));
          klaunch(k_hform3nd<false, true>, fgrid, HFW * 32, smf, s, F);
        } else {
          ZF_CUDA(cudaFuncSetAttribute(k_hform3nd<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smf));
          klaunch(k_hform3nd<false, false>, fgrid, HFW * 32, smf, s, F);
        }
      }
      ZF_LAUNCH_CHECK();
    };
    F.out = mpn.get();
    if (nlev >= 2) form(false);
    if (L.mn[3] > 0) {
      F.out = locn.get();
      form(true);
    }
  }
  mark(2);
  int dev = 0, nsm = 148;
  ZF_CUDA(cudaGetDevice(&dev));
  ZF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const int xgrid = std::max(1, std::min(nsm, nb * div_up(nd, RC)));
  const size_t per_cta = 2 * (size_t)(H.pmax + 1) * (H.pmax + 1) * RC;
  DevBuf<zdc> scratch((size_t)xgrid * per_cta, s);
  HTransNdArgs A;
  A.T = H.T;
  A.LT = H.pmax + 1;
  A.kwave = H.kw;
  A.ilevel = t.ilevel.get(); A.iparent = t.iparent.get(); A.nchild = t.nchild.get();
  A.ichild = t.ichild.get(); A.isrcse = S.isrcse.get(); A.itargse = S.itargse.get();
  A.zcs = S.zcsrc.get(); A.zct = S.zctarg.get();
  A.nl2 = L.n[1].get(); A.l2 = L.list[1].get(); A.nl4 = L.n[3].get(); A.mn2 = L.mn[1];
  DevBuf<int> queue(1, s);
  A.scratch = scratch.get();
  A.scr_per_cta = (long)per_cta;
  A.queue = queue.get();
  A.nd = nd;
  // M2M, finest parents first (parents at levels >= 2)
  A.in = mpn.get();
  A.out = mpn.get();
  for (int l = nlev - 1; l >= 2; l--)
    launch_htrans_nd<0>(A, H, l + 1, l, t.laddr[2 * l], t.laddr[2 * l + 1], xgrid, s);
  mark(3);
  // M2L per level >= 2
  A.in = mpn.get();
  A.out = locn.get();
  for (int l = 2; l <= nlev; l++)
    launch_htrans_nd<1>(A, H, l, l, t.laddr[2 * l], t.laddr[2 * l + 1], xgrid, s);
  mark(4);
  // L2L, coarsest first: children at level l+1 of parents at level l >= 2
  A.in = locn.get();
  A.out = locn.get();
  for (int l = 2; l <= nlev - 1; l++)
    launch_htrans_nd<2>(A, H, l, l + 1, t.laddr[2 * (l + 1)], t.laddr[2 * (l + 1) + 1], xgrid, s);
  mark(5);
  // P2P, L2T and M2T batched over the right-hand sides (tree-order strengths
  // and outputs with the right-hand side fastest)
  {
    DevBuf<zdc> potn((size_t)nt * nd, s), gradn(ifpgh > 1 ? 3 * (size_t)nt * nd : 1, s);
    potn.zero();
    gradn.zero();
    HP2PNdArgs Pa;
    Pa.nchild = t.nchild.get(); Pa.isrcse = S.isrcse.get(); Pa.itargse = S.itargse.get();
    Pa.zsrc = S.zsrcsort.get(); Pa.q = qn.get(); Pa.ds = dsn.get(); Pa.dv = dv.get();
    Pa.ztarg = S.ztargsort.get();
    Pa.nl1 = L.n[0].get(); Pa.l1 = L.list[0].get(); Pa.mn1 = L.mn[0]; Pa.nb = nb; Pa.nd = nd;
    Pa.ifcharge = in.ifcharge; Pa.zk = H.kw;
    Pa.pot = potn.get(); Pa.grad = gradn.get();
    const size_t smp = sizeof(HSrcTileNd);
    const dim3 pgrid(nb, div_up(nd, HRB));
    if (ifpgh > 1) {
      if (dip) {
        ZF_CUDA(cudaFuncSetAttribute(k_hp2p3nd<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smp));
        klaunch(k_hp2p3nd<true, true>, pgrid, HNDT, smp, s, Pa);
      } else {
        ZF_CUDA(cudaFuncSetAttribute(k_hp2p3nd<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smp));
        klaunch(k_hp2p3nd<true, false>, pgrid, HNDT, smp, s, Pa);
      }
    } else {
      if (dip) {
        ZF_CUDA(cudaFuncSetAttribute(k_hp2p3nd<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smp));
        klaunch(k_hp2p3nd<false, true>, pgrid, HNDT, smp, s, Pa);
      } else {
        ZF_CUDA(cudaFuncSetAttribute(k_hp2p3nd<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smp));
        klaunch(k_hp2p3nd<false, false>, pgrid, HNDT, smp, s, Pa);
      }
    }
    ZF_LAUNCH_CHECK();
    HEvalNdArgs E;
    E.r1 = H.T.r1; E.r2 = H.T.r2; E.sq = H.T.sq; E.L = H.pmax + 1;
    E.ilevel = t.ilevel.get(); E.nchild = t.nchild.get(); E.isrcse = S.isrcse.get();
    E.itargse = S.itargse.get(); E.ztarg = S.ztargsort.get(); E.zcs = S.zcsrc.get();
    E.zct = S.zctarg.get(); E.lev = H.lev; E.mp = mpn.get(); E.loc = locn.get();
    E.nl3 = L.n[2].get(); E.l3 = L.list[2].get(); E.mn3 = L.mn[2]; E.nb = nb; E.nd = nd;
    E.zk = H.kw; E.pot = potn.get(); E.grad = gradn.get();
    const dim3 egrid(nb, div_up(nd, HRBE));
    if (ifpgh > 1) klaunch(k_heval3nd<true>, egrid, HNDT, 0, s, E);
    else klaunch(k_heval3nd<false>, egrid, HNDT, 0, s, E);
    ZF_LAUNCH_CHECK();
    unsort3d_nd(nt, nd, S.itarg.get(), potn.get(), gradn.get(), mkz(1.0), mkz(1.0 / S.b0),
                ifpgh, pot, grad, s);
  }
  mark(6);
  mark(7);
  if (timing) {
    ZF_CUDA(cudaEventSynchronize(ev[7]));
    float ms;
    // set-up = the wavenumber tables; P2M column = P2M and P2L of every
    // right-hand side; eval = P2P, L2T, M2T and the unsort
    for (int i = 0; i < 7; i++) {
      ZF_CUDA(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]));
      times->ms[i] = ms;
    }
    times->nboxes = nb;
    times->nlevels = nlev;
    times->nterms = H.pmax;
    for (auto& e : ev) cudaEventDestroy(e);
    times->launches = launch_counter() - launches0;
    if (times->want_counts) count_interactions3d(S, H.lev.p, 2, 2, 3, times, s);
  }
}

}  // namespace zf
