// 2D Helmholtz complex-coordinate FMM (zhfmm2d) on the device.
//
// Reference: zfmm2d/src/helmholtz/zhfmm2d.f (driver :14-227, eight steps of
// zhfmm2dmain :233-604, zh2dformmp :610-686, zh2dformloc :692-766,
// zh2devaldirect :773-838, zh2devalmp :844-901, zh2devalloc :907-964) and the
// Graf translations of zfmm2d/src/helmholtz/zh2dtrans.f (zh2dlocloc :6-78,
// zh2dmploc :84-142, zh2dmpmp :225-303).
//
// Expansions are the reference's: mp(m) / loc(m), m = -p..p, p = nterms(level)
// from h2dterms, scaled Bessel/Hankel functions J_m/rscale^m, H_m rscale^m with
// rscale = min(|zk boxsize|/(2 pi), 1), angles through ez = (z1 + i z2)/rz with
// rz = sqrt(z1^2 + z2^2) on the principal branch.
//
// Parallel layout (one warp per box, as in the Laplace path):
//   P2M / P2L:  lane = source (32 at a time) computes its Bessel/Hankel column
//               into shared memory, then lane = coefficient m accumulates;
//   M2M / M2L / L2L: per box pair the Bessel/Hankel table of the pair is built
//               in shared memory (warp-parallel quadrature for H0/H1), then
//               lane = output coefficient runs the dense Toeplitz-structured sum
//               over the (2p+1) input coefficients;
//   L2T / M2T:  lane = target, one streaming recurrence per (target, box)
//               accumulating pot and grad without storing the function table;
//   P2P:        group of lanes per target over the list-1 sources, shuffle
//               reduction.
#include <map>
#include <mutex>
#include <tuple>
#include <vector>
#include "fmm2d_common.cuh"
#include "hank2d.cuh"
#include "helm2d_pair.cuh"
#include "hfmm2d.cuh"
#include "lfmm2d.cuh"

namespace zf {
namespace {

constexpr int WPB = 4;
constexpr int MAXL = 64;  // levels

struct LevelTab {
  long base[MAXL];   // first coefficient (of m = -p) of the first box of the level
  int lo[MAXL];      // first box of the level
  int p[MAXL];       // nterms
  double rs[MAXL];   // rscale
};

struct HelmArgs {
  zdc zk;
  LevelTab T;
  const int* ilevel;
  const int* iparent;
  const int* nchild;
  const int* ichild;
  const int* isrcse;
  const int* itargse;
  const zdc* zsrc;
  const zdc* charge;
  const zdc* dipstr;
  const zdc* dipvec;
  const zdc* ztarg;
  const zdc* zcsrc;
  const zdc* zctarg;
  zdc* mp;
  zdc* loc;
  int ifcharge, ifdipole;
};

// pointer to coefficient 0 of box b's expansion
__device__ __forceinline__ zdc* expo(const HelmArgs& A, zdc* base, int b) {
  int l = A.ilevel[b];
  return base + A.T.base[l] + (long)(b - A.T.lo[l]) * (2 * A.T.p[l] + 1) + A.T.p[l];
}

__device__ __forceinline__ double sgn(int n) { return (n & 1) ? -1.0 : 1.0; }

__device__ __forceinline__ void polar(zdc a1, zdc a2, zdc& rz, zdc& ez) {
  // zcart2polar (toolbox.f:73-82)
  rz = zsqrt_p(a1 * a1 + a2 * a2);
  ez = a1 / rz + zmul_i(a2 / rz);
}

// H0, H1 for a warp-uniform argument: the quadrature nodes of hank01_integral
// are spread over the lanes; the other regions are evaluated by every lane.
__device__ void hank01_warp(zdc z, zdc& h0, zdc& h1) {
  if (z.im == 0.0) z.im = 0.0;
  if (zabs(z) < 2.0 || z.im < 0.0) {
    hank01(z, h0, h1);
    return;
  }
  int lane = threadIdx.x & 31;
  zdc c = zmul_i(zinv(2.0 * z));
  double s = ZF_HQ_STEP * lane, s2 = s * s;
  double w = ZF_HQ_STEP * exp(-s2) * (lane == 0 ? 0.5 : 1.0);
  zdc r = zsqrt_p(mkz(1.0) + s2 * c);
  zdc f0 = w * zinv(r), f1 = (w * s2) * r;
  for (int o = 16; o; o >>= 1) {
    f0 += shfl_xor_z(f0, o);
    f1 += shfl_xor_z(f1, o);
  }
  zdc pre = ZF_SQRT_2_PI * zinv(zsqrt_p(z));
  zdc e = zexp_p(zmul_i(z));
  const double r2 = 0.70710678118654752440;
  h0 = (2.0 * ZF_INV_SQRT_PI) * ((pre * (e * zdc{r2, -r2})) * f0);
  h1 = (4.0 * ZF_INV_SQRT_PI) * ((pre * (e * zdc{-r2, -r2})) * f1);
}

// scaled Hankel table hv[0..n] of a warp-uniform argument into shared memory
__device__ void h2dall_warp(int n, zdc z, double rscale, zdc* hv) {
  int lane = threadIdx.x & 31;
  if (zabs(z) < 1e-200) {
    for (int i = lane; i <= n; i += 32) hv[i] = mkz(0.0);
    __syncwarp();
    return;
  }
  zdc h0, h1;
  hank01_warp(z, h0, h1);
  if (lane == 0) {
    hv[0] = h0;
    if (n >= 1) hv[1] = h1 * rscale;
    double sc2 = rscale * rscale;
    zdc zi = rscale * zinv(z);
    for (int i = 1; i < n; i++) hv[i + 1] = ((2.0 * i) * zi) * hv[i] - sc2 * hv[i - 1];
  }
  __syncwarp();
}

// Scaled Bessel table out[0..nterms+1] = J_n(z)/rscale^n by Miller's backward
// recurrence from the reference's start index, keeping only the entries that
// are returned (the normalisation sum is accumulated during the sweep).
__device__ void jbessel_stream(int nterms, zdc z, double rscale, zdc* out) {
  int top = nterms + 1;
  if (zabs(z) < 1e-200) {
    out[0] = mkz(1.0);
    for (int i = 1; i <= top; i++) out[i] = mkz(0.0);
    return;
  }
  int ntop = jbessel_top(nterms, z);
  zdc zr = rscale * zinv(z);
  double sc2 = rscale * rscale;
  zdc zmul = z.im < 0.0 ? mkz(0.0, 1.0) : mkz(0.0, -1.0);
  // g_{ntop} = 0, g_{ntop-1} = 1
  zdc gp1 = mkz(0.0), g = mkz(1.0), psi = mkz(0.0);
  for (int i = 0; i <= top; i++) out[i] = mkz(0.0);
  // psi accumulates sum_{n>=1} zmul^n rscale^(n-1) g_n in Horner form from the top
  for (int n = ntop - 1; n >= 0; n--) {
    // g holds g_n
    if (n <= top) out[n] = g;
    if (n >= 1) {
      int r = n & 3;
      zdc zn = r == 0 ? mkz(1.0) : (r == 1 ? zmul : (r == 2 ? mkz(-1.0) : -zmul));
      psi = rscale * psi + zn * g;
      zdc gm1 = ((2.0 * n) * zr) * g - sc2 * gp1;
      gp1 = g;
      g = gm1;
      if (zabs(g) > 1e200) {
        g = 1e-200 * g;
        gp1 = 1e-200 * gp1;
        psi = 1e-200 * psi;
        for (int k = n; k <= top; k++) out[k] = 1e-200 * out[k];
      }
    }
  }
  // g_{ntop}=0 contributes nothing; psi misses the factor for the top zero
  psi = 2.0 * rscale * psi + out[0];
  zdc e = z.im < 0.0 ? zexp_p(zmul_i(z)) : zexp_p(-zmul_i(z));
  zdc sc = e / psi;
  for (int i = 0; i <= top; i++) out[i] = out[i] * sc;
}

// ---- step 1 / 6: P2M (zh2dformmp) and P2L (zh2dformloc) ------------------------
constexpr int FCH = 8;  // sources whose function tables are built at once

// Accumulate the expansion about centre (c1, c2) with scale rs and p terms
// from sources [s0, s1].  `tab` is per-warp shared scratch of FCH*(p+2)
// complex; `local` selects Hankel (P2L) or Bessel (P2M) functions.  Lane k
// (< FCH) builds the table of one source, then lane = coefficient m adds the
// contributions of the FCH sources.
__device__ void form_expansion(const HelmArgs& A, int s0, int s1, zdc c1, zdc c2, double rs, int p,
                               bool local, zdc* tab, zdc* accp, zdc* accm, zdc& acc0) {
  int lane = threadIdx.x & 31;
  int P2 = p + 2;
  for (int j0 = s0; j0 <= s1; j0 += FCH) {
    int j = j0 + lane;
    if (lane < FCH && j <= s1) {
      zdc* col = tab + lane * P2;
      zdc rz, ez;
      polar(ldz(&A.zsrc[2 * j]) - c1, ldz(&A.zsrc[2 * j + 1]) - c2, rz, ez);
      zdc z = rz * A.zk;
      if (local) h2dall(p + 1, z, rs, col, 0, nullptr);
      else jbessel_stream(p, z, rs, col);
    }
    __syncwarp();
    int nsrc = min(FCH, s1 - j0 + 1);
    for (int k = 0; k < nsrc; k++) {
      int jj = j0 + k;
      const zdc* f = tab + k * P2;
      zdc a1 = ldz(&A.zsrc[2 * jj]) - c1, a2 = ldz(&A.zsrc[2 * jj + 1]) - c2;
      zdc rzk, ezk;
      polar(a1, a2, rzk, ezk);
      zdc iez = zinv(ezk);
      zdc q = A.ifcharge ? ldz(&A.charge[jj]) : mkz(0.0);
      zdc ds = mkz(0.0), pr = mkz(0.0), pe = mkz(0.0);
      if (A.ifdipole) {
        ds = ldz(&A.dipstr[jj]);
        zdc d1 = ldz(&A.dipvec[2 * jj]), d2 = ldz(&A.dipvec[2 * jj + 1]);
        zdc vr1 = a1 / rzk, vr2 = a2 / rzk;
        pr = vr1 * d1 + vr2 * d2;
        pe = -vr2 * d1 + vr1 * d2;
      }
      zdc pe_rz = pe / rzk, izk = zinv(rzk * A.zk);
      // coefficients m = lane, lane+32, ... (0..p); ezs(-m) = ez^-m, ezs(m) = ez^m
      for (int m = lane, r = 0; m <= p; m += 32, r++) {
        zdc em = zpown(iez, m), ep = zpown(ezk, m);
        zdc fm = f[m];
        zdc fder;  // derivative of the scaled function (h2dall / jbessel2d conventions)
        if (local) fder = (m == 0) ? -f[1] / rs : rs * f[m - 1] - ((double)m * izk) * fm;
        else fder = (m == 0) ? -f[1] * rs : (0.5 / rs) * f[m - 1] - (0.5 * rs) * f[m + 1];
        zdc cm = fm * em * q, cneg = sgn(m) * (fm * ep * q);
        if (A.ifdipole) {
          zdc dr = em * fder * A.zk, dth = fm * zdc{0.0, -(double)m} * em;
          cm -= ds * (dr * pr + dth * pe_rz);
          zdc drn = ep * fder * A.zk, dthn = fm * zdc{0.0, (double)m} * ep;
          cneg -= ds * sgn(m) * (drn * pr + dthn * pe_rz);
        }
        if (m == 0) {
          acc0 += cm;
        } else {
          accp[r] += cm;
          accm[r] += cneg;
        }
      }
    }
    __syncwarp();
  }
}

constexpr int MAXR = 8;  // coefficient slots per lane: p <= 255

__global__ void __launch_bounds__(32 * WPB, 4) k_hp2m(int lo, int hi, HelmArgs A, int pmax) {
  extern __shared__ zdc sh[];
  int b = lo + blockIdx.x * WPB + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (b > hi) return;
  int s0 = A.isrcse[2 * b], s1 = A.isrcse[2 * b + 1];
  if (A.nchild[b] > 0 || s1 < s0 || A.ilevel[b] < 2) return;
  int l = A.ilevel[b], p = A.T.p[l];
  zdc* tab = sh + (threadIdx.x >> 5) * FCH * (pmax + 2);
  zdc accp[MAXR], accm[MAXR], acc0 = mkz(0.0);
#pragma unroll
  for (int r = 0; r < MAXR; r++) accp[r] = accm[r] = mkz(0.0);
  form_expansion(A, s0, s1, A.zcsrc[2 * b], A.zcsrc[2 * b + 1], A.T.rs[l], p, false, tab, accp,
                 accm, acc0);
  zdc* M = expo(A, A.mp, b);
  for (int m = lane, r = 0; m <= p; m += 32, r++) {
    if (m == 0) M[0] = acc0;
    else { M[m] = accp[r]; M[-m] = accm[r]; }
  }
}

// ---- dense translations --------------------------------------------------------
// M2M (zh2dmpmp): children -> parent, level lev
// M2M (zh2dmpmp): the reference's sum over child coefficients n,
//   mp(m) += sum_n (-1)^(m+n) J_(m-n) e^{i(n-m) theta} mp_child(n) w(m, n),
//   w = rs2^|n| rs1^|m-n| / rs1^|m|   (rs1 parent, rs2 child scale, rs2 <= rs1)
// is a Toeplitz product in k = m - n once w is split by the signs of m, n:
// opposite signs (or n = 0): (rs1 rs2)^|n|; same sign, |n| <= |m|:
// (rs2/rs1)^|n|; same sign, |n| > |m|: (rs2/rs1)^|m| (rs1 rs2)^|k|.
__global__ void __launch_bounds__(32 * WPB) k_hm2m(int lo, int hi, int lev, HelmArgs A,
                                                  int stride) {
  extern __shared__ zdc sh[];
  int b = lo + blockIdx.x * WPB + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (b > hi) return;
  if (A.nchild[b] == 0 || A.isrcse[2 * b + 1] < A.isrcse[2 * b]) return;
  int n1 = A.T.p[lev], n2 = A.T.p[lev + 1], nt = n1 + n2;
  double rs1 = A.T.rs[lev], rs2 = A.T.rs[lev + 1];
  zdc* fj = sh + (threadIdx.x >> 5) * stride;   // [nt+2]
  zdc* S1 = fj + (nt + 2) + nt;                  // S1[k], k = -nt..nt
  zdc* S2 = S1 + nt + 1 + nt;                    // S1[k] (rs1 rs2)^|k|
  zdc* uu = S2 + nt + 1 + n2;                    // (rs2/rs1)^|n| mp_child(n), n = -n2..n2
  zdc* ww = uu + n2 + 1 + n2;                    // (rs1 rs2)^|n| mp_child(n)
  double* qa = (double*)(ww + n2 + 1);           // (rs1 rs2)^k, k = 0..nt
  double* qb = qa + nt + 1;                      // (rs2/rs1)^k, k = 0..nt
  zdc accp[MAXR], accm[MAXR], acc0 = mkz(0.0);
#pragma unroll
  for (int r = 0; r < MAXR; r++) accp[r] = accm[r] = mkz(0.0);
  for (int k = lane; k <= nt; k += 32) {
    qa[k] = pow(rs1 * rs2, (double)k);
    qb[k] = pow(rs2 / rs1, (double)k);
  }
  for (int jc = 0; jc < 4; jc++) {
    int jb = A.ichild[4 * b + jc];
    if (A.isrcse[2 * jb + 1] < A.isrcse[2 * jb]) continue;
    zdc rz, e;
    polar(A.zcsrc[2 * b] - A.zcsrc[2 * jb], A.zcsrc[2 * b + 1] - A.zcsrc[2 * jb + 1], rz, e);
    __syncwarp();
    if (lane == 0) jbessel_stream(nt, rz * A.zk, rs1, fj);
    __syncwarp();
    zdc ie = zinv(e);
    // S1[k] = (-1)^k t(k) e^{-ik theta}, t(k) = J_k (k >= 0), (-1)^k J_-k (k < 0)
    for (int k = lane; k <= nt; k += 32) {
      zdc f = fj[k];
      S1[k] = (sgn(k) * f) * zpown(ie, k);
      S1[-k] = f * zpown(e, k);
      S2[k] = S1[k] * qa[k];
      S2[-k] = S1[-k] * qa[k];
    }
    const zdc* M2 = expo(A, A.mp, jb);
    for (int n = lane - n2; n <= n2; n += 32) {
      zdc v = M2[n];
      int an = abs(n);
      uu[n] = qb[an] * v;
      ww[n] = qa[an] * v;
    }
    __syncwarp();
    for (int m = lane, r = 0; m <= n1; m += 32, r++) {
      zdc a1 = mkz(0.0), a2 = mkz(0.0);
      for (int n = -n2; n <= n2; n++) {
        int k = m - n;
        if (n <= 0) a1 += S1[k] * ww[n];
        else if (n <= m) a1 += S1[k] * uu[n];
        else a2 += S2[k] * M2[n];
      }
      zdc sp = a1 + qb[m] * a2;
      if (m == 0) {
        acc0 += sp;
        continue;
      }
      a1 = mkz(0.0);
      a2 = mkz(0.0);
      for (int n = -n2; n <= n2; n++) {
        int k = -m - n;
        if (n >= 0) a1 += S1[k] * ww[n];
        else if (n >= -m) a1 += S1[k] * uu[n];
        else a2 += S2[k] * M2[n];
      }
      accp[r] += sp;
      accm[r] += a1 + qb[m] * a2;
    }
  }
  zdc* M = expo(A, A.mp, b);
  for (int m = lane, r = 0; m <= n1; m += 32, r++) {
    if (m == 0) M[0] = acc0;
    else { M[m] = accp[r]; M[-m] = accm[r]; }
  }
}

// M2L (zh2dmploc) over list 2; R coefficient slots per lane (p < 32 R).  The
// local expansion is written here; P2L (k_hp2l) adds to it afterwards.
template <int R>
__global__ void __launch_bounds__(32 * WPB, 4) k_hm2l(int lo, int hi, HelmArgs A, const int* nl2,
                                                  const int* l2, int m2, int stride) {
  extern __shared__ zdc sh[];
  int b = lo + blockIdx.x * WPB + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (b > hi) return;
  if (A.itargse[2 * b + 1] < A.itargse[2 * b]) return;
  int n2c = nl2[b];
  if (n2c == 0) return;
  int l = A.ilevel[b], p = A.T.p[l], n2 = 2 * p;
  double rs = A.T.rs[l];
  zdc* fh = sh + (threadIdx.x >> 5) * stride;  // [n2+2]
  zdc* T = fh + (n2 + 2);                       // [2*n2+1]
  double* rp = (double*)(T + 2 * n2 + 1);       // rs^k, k = 0..n2
  zdc* bb = T + 2 * n2 + 1 + (n2 + 2) + p;      // b(n), n = -p..p
  zdc* cc = bb + 2 * p + 1;                     // c(n)
  zdc accp[R], accm[R], acc0 = mkz(0.0);
#pragma unroll
  for (int r = 0; r < R; r++) accp[r] = accm[r] = mkz(0.0);
  for (int k = lane; k <= n2; k += 32) rp[k] = pow(rs, (double)k);
  zdc c1 = A.zctarg[2 * b], c2 = A.zctarg[2 * b + 1];
  for (int il = 0; il < n2c; il++) {
    int jb = l2[(size_t)b * m2 + il];
    if (A.isrcse[2 * jb + 1] < A.isrcse[2 * jb]) continue;
    zdc rz, e;
    polar(c1 - A.zcsrc[2 * jb], c2 - A.zcsrc[2 * jb + 1], rz, e);
    __syncwarp();
    h2dall_warp(n2, rz * A.zk, rs, fh);
    zdc ie = zinv(e);
    // Toeplitz symbol T[k] = H_k e^{ik theta} (k = -2p..2p, H_-k = (-1)^k H_k,
    // scaled) and the source coefficients without (b) and with (c) the factor
    // rs^(2|n|): the reference's weight rs^|m| rs^|n| / rs^|n-m| is 1 for n, m
    // of opposite signs and rs^(2 min(|m|,|n|)) otherwise, so
    //   loc(m) = sum_{n<0} T[n-m] b(n) + sum_{0<=n<=m} T[n-m] c(n)
    //          + rs^(2m) sum_{n>m} T[n-m] b(n)        (m >= 0, mirrored for m < 0)
    for (int k = lane; k <= n2; k += 32) {
      zdc f = fh[k];
      T[n2 + k] = f * zpown(e, k);
      T[n2 - k] = (sgn(k) * f) * zpown(ie, k);
    }
    const zdc* M = expo(A, A.mp, jb);
    for (int n = lane - p; n <= p; n += 32) {
      zdc v = M[n];
      bb[n] = v;
      cc[n] = rp[2 * abs(n)] * v;
    }
    __syncwarp();
#pragma unroll
    for (int r = 0; r < R; r++) {
      int m = lane + 32 * r;
      if (m > p) break;
      zdc a1 = mkz(0.0), a2 = mkz(0.0);
      const zdc* Tm = T + n2 - m;  // Tm[n] = T[n - m]
      for (int n = -p; n <= p; n++) {
        zdc t = Tm[n];
        if (n > m) a2 += t * bb[n];
        else a1 += t * (n < 0 ? bb[n] : cc[n]);
      }
      zdc sp = a1 + rp[2 * m] * a2;
      if (m == 0) {
        acc0 += sp;
        continue;
      }
      a1 = mkz(0.0);
      a2 = mkz(0.0);
      const zdc* Tq = T + n2 + m;  // Tq[n] = T[n + m]
      for (int n = -p; n <= p; n++) {
        zdc t = Tq[n];
        if (n < -m) a2 += t * bb[n];
        else a1 += t * (n > 0 ? bb[n] : cc[n]);
      }
      accp[r] += sp;
      accm[r] += a1 + rp[2 * m] * a2;
    }
    __syncwarp();
  }
  zdc* L = expo(A, A.loc, b);
#pragma unroll
  for (int r = 0; r < R; r++) {
    int m = lane + 32 * r;
    if (m > p) break;
    if (m == 0) L[0] = acc0;
    else {
      L[m] = accp[r];
      L[-m] = accm[r];
    }
  }
}

// P2L (zh2dformloc) over list 4, added to the local expansion
__global__ void __launch_bounds__(32 * WPB, 4) k_hp2l(int lo, int hi, HelmArgs A, const int* nl4,
                                                  const int* l4, int m4, int stride) {
  extern __shared__ zdc sh[];
  int b = lo + blockIdx.x * WPB + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (b > hi) return;
  if (A.itargse[2 * b + 1] < A.itargse[2 * b]) return;
  int n4c = nl4[b];
  if (n4c == 0) return;
  int l = A.ilevel[b], p = A.T.p[l];
  double rs = A.T.rs[l];
  zdc* tab = sh + (threadIdx.x >> 5) * stride;  // FCH*(p+2)
  zdc accp[MAXR], accm[MAXR], acc0 = mkz(0.0);
#pragma unroll
  for (int r = 0; r < MAXR; r++) accp[r] = accm[r] = mkz(0.0);
  zdc c1 = A.zctarg[2 * b], c2 = A.zctarg[2 * b + 1];
  for (int il = 0; il < n4c; il++) {
    int jb = l4[(size_t)b * m4 + il];
    int s0 = A.isrcse[2 * jb], s1 = A.isrcse[2 * jb + 1];
    if (s1 < s0) continue;
    __syncwarp();
    form_expansion(A, s0, s1, c1, c2, rs, p, true, tab, accp, accm, acc0);
  }
  zdc* L = expo(A, A.loc, b);
  for (int m = lane, r = 0; m <= p; m += 32, r++) {
    if (m == 0) L[0] += acc0;
    else {
      L[m] += accp[r];
      L[-m] += accm[r];
    }
  }
}

// L2L (zh2dlocloc) into the children at level lev+1
// L2L (zh2dlocloc): loc_child(m) += sum_n t(n-m) e^{i(n-m) theta} loc(n)
//   rs1^|m| rs1^|n-m| / rs2^|n|   (rs1 child, rs2 parent scale, rs1 <= rs2)
// split by signs: same sign with |n| >= |m|: (rs1/rs2)^|n|; same sign with
// |n| < |m| (and n = 0): (rs1/rs2)^|n| rs1^(2|k|); opposite: (rs1/rs2)^|n| rs1^(2|m|).
__global__ void __launch_bounds__(32 * WPB) k_hl2l(int lo, int hi, int lev, HelmArgs A,
                                                  const int* nl2, const int* nl4, int stride) {
  extern __shared__ zdc sh[];
  int jb = lo + blockIdx.x * WPB + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (jb > hi) return;
  int b = A.iparent[jb];
  if (A.itargse[2 * b + 1] < A.itargse[2 * b] || (nl2[b] == 0 && nl4[b] == 0)) return;
  if (A.itargse[2 * jb + 1] < A.itargse[2 * jb]) return;
  int n1 = A.T.p[lev + 1], n2 = A.T.p[lev], nt = n1 + n2;
  double rs1 = A.T.rs[lev + 1], rs2 = A.T.rs[lev];
  zdc* fj = sh + (threadIdx.x >> 5) * stride;   // [nt+2]
  zdc* S1 = fj + (nt + 2) + nt;                  // S1[k] = t(k) e^{ik theta}, k = -nt..nt
  zdc* S3 = S1 + nt + 1 + nt;                    // S1[k] rs1^(2|k|)
  zdc* uu = S3 + nt + 1 + n2;                    // (rs1/rs2)^|n| loc_parent(n)
  double* qa = (double*)(uu + n2 + 1);           // rs1^(2k), k = 0..nt
  double* qb = qa + nt + 1;                      // (rs1/rs2)^k, k = 0..nt
  for (int k = lane; k <= nt; k += 32) {
    qa[k] = pow(rs1, 2.0 * k);
    qb[k] = pow(rs1 / rs2, (double)k);
  }
  zdc rz, e;
  polar(A.zctarg[2 * jb] - A.zctarg[2 * b], A.zctarg[2 * jb + 1] - A.zctarg[2 * b + 1], rz, e);
  if (lane == 0) jbessel_stream(nt, rz * A.zk, rs1, fj);
  __syncwarp();
  zdc ie = zinv(e);
  for (int k = lane; k <= nt; k += 32) {
    zdc f = fj[k];
    S1[k] = f * zpown(e, k);
    S1[-k] = (sgn(k) * f) * zpown(ie, k);
    S3[k] = S1[k] * qa[k];
    S3[-k] = S1[-k] * qa[k];
  }
  const zdc* L2 = expo(A, A.loc, b);
  for (int n = lane - n2; n <= n2; n += 32) uu[n] = qb[abs(n)] * L2[n];
  __syncwarp();
  zdc* L1 = expo(A, A.loc, jb);
  for (int m = lane; m <= n1; m += 32) {
    zdc a1 = mkz(0.0), a2 = mkz(0.0);
    for (int n = -n2; n <= n2; n++) {
      int k = n - m;
      if (n >= m) a1 += S1[k] * uu[n];
      else if (n >= 0) a1 += S3[k] * uu[n];
      else a2 += S1[k] * uu[n];
    }
    L1[m] += a1 + qa[m] * a2;
    if (m == 0) continue;
    a1 = mkz(0.0);
    a2 = mkz(0.0);
    for (int n = -n2; n <= n2; n++) {
      int k = n + m;
      if (n <= -m) a1 += S1[k] * uu[n];
      else if (n <= 0) a1 += S3[k] * uu[n];
      else a2 += S1[k] * uu[n];
    }
    L1[-m] += a1 + qa[m] * a2;
  }
}

// ---- steps 3, 5, 8: P2P (list1), M2T (list3), L2T per target leaf --------------
template <bool GRAD>
__global__ void __launch_bounds__(32 * WPB, 4) k_heval(int nb, HelmArgs A, const int* nl1,
                                                   const int* l1, int m1, const int* nl3,
                                                   const int* l3, int m3, zdc* potsort,
                                                   zdc* gradsort) {
  int b = blockIdx.x * WPB + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (b >= nb) return;
  int t0 = A.itargse[2 * b], t1 = A.itargse[2 * b + 1];
  if (A.nchild[b] > 0 || t1 < t0) return;
  int ntb = t1 - t0 + 1;
  int lb = A.ilevel[b];
  // L2T and M2T: one lane per target
  for (int base = 0; base < ntb; base += 32) {
    int ti = t0 + base + lane;
    if (base + lane < ntb) {
      zdc x1 = ldz(&A.ztarg[2 * ti]), x2 = ldz(&A.ztarg[2 * ti + 1]);
      zdc pot = mkz(0.0), g1 = mkz(0.0), g2 = mkz(0.0);
      // L2T (zh2devalloc): one backward Miller sweep (jbessel2d) accumulating the
      // unnormalised sums; the normalisation e^{-+iz}/psi is applied at the end.
      // Derivative of the scaled Bessel function: fjder(n) = g_{n-1}/rs - (n/z) g_n,
      // fjder(0) = -rs g_1 (equal to the reference's (g_{n-1}/rs - rs g_{n+1})/2).
      if (lb >= 2) {
        int p = A.T.p[lb];
        double rs = A.T.rs[lb];
        const zdc* L = expo(A, A.loc, b);
        zdc a1 = x1 - A.zctarg[2 * b], a2 = x2 - A.zctarg[2 * b + 1];
        zdc zr, ei;
        polar(a1, a2, zr, ei);
        zdc z = zr * A.zk;
        if (zabs(z) >= 1e-200) {
          int ntop = jbessel_top(p, z);
          zdc zrr = rs * zinv(z), izz = zinv(z);
          double sc2 = rs * rs;
          zdc zmul = z.im < 0.0 ? mkz(0.0, 1.0) : mkz(0.0, -1.0);
          zdc iei = zinv(ei);
          zdc gp1 = mkz(0.0), g = mkz(1.0), psi = mkz(0.0);
          zdc sp = mkz(0.0), srad = mkz(0.0), sang = mkz(0.0);
          zdc eip = zpown(ei, p), eim = zpown(iei, p);
          for (int n = ntop - 1; n >= 0; n--) {
            zdc gm1 = n >= 1 ? ((2.0 * n) * zrr) * g - sc2 * gp1 : mkz(0.0);
            if (n <= p) {
              zdc cp = ldz(&L[n]) * eip;
              zdc cm = n == 0 ? mkz(0.0) : sgn(n) * (ldz(&L[-n]) * eim);
              zdc c = cp + cm;
              sp += c * g;
              if (GRAD) {
                zdc fd = n >= 1 ? gm1 / rs - ((double)n * izz) * g : (-rs) * gp1;
                srad += c * fd;
                sang += ((double)n * zmul_i(cp - cm)) * g;
              }
              eip = eip * iei;
              eim = eim * ei;
            }
            if (n >= 1) {
              int rr = n & 3;
              zdc zn = rr == 0 ? mkz(1.0) : (rr == 1 ? zmul : (rr == 2 ? mkz(-1.0) : -zmul));
              psi = rs * psi + zn * g;
              gp1 = g;
              g = gm1;
              if (zabs(g) > 1e200) {
                g = 1e-200 * g; gp1 = 1e-200 * gp1; psi = 1e-200 * psi;
                sp = 1e-200 * sp; srad = 1e-200 * srad; sang = 1e-200 * sang;
              }
            } else {
              psi = 2.0 * rs * psi + g;
            }
          }
          zdc sc = (z.im < 0.0 ? zexp_p(zmul_i(z)) : zexp_p(-zmul_i(z))) / psi;
          pot += sp * sc;
          if (GRAD) {
            zdc rad = (srad * sc) * A.zk, ang = (sang * sc) / zr;
            zdc vr1 = a1 / zr, vr2 = a2 / zr;
            g1 += rad * vr1 - ang * vr2;
            g2 += rad * vr2 + ang * vr1;
          }
        }
      }
      // M2T (zh2devalmp) over list3: streaming forward recurrence of H_n
      int n3 = nl3[b];
      for (int il = 0; il < n3; il++) {
        int jb = l3[(size_t)b * m3 + il];
        if (A.isrcse[2 * jb + 1] < A.isrcse[2 * jb]) continue;
        int lj = A.ilevel[jb], p = A.T.p[lj];
        double rs = A.T.rs[lj];
        const zdc* M = expo(A, A.mp, jb);
        zdc zr, ei;
        zdc a1 = x1 - A.zcsrc[2 * jb], a2 = x2 - A.zcsrc[2 * jb + 1];
        polar(a1, a2, zr, ei);
        zdc z = zr * A.zk;
        if (zabs(z) < 1e-200) continue;
        zdc h0, h1;
        hank01(z, h0, h1);
        zdc iei = zinv(ei), zi = rs * zinv(z), zi1 = zinv(z);
        double sc2 = rs * rs;
        zdc hm1 = mkz(0.0), h = h0, hp = h1 * rs;  // scaled H_{n-1}, H_n, H_{n+1}
        zdc eip = mkz(1.0), eim = mkz(1.0);
        zdc sp = mkz(0.0), srad = mkz(0.0), sang = mkz(0.0);
        for (int n = 0; n <= p; n++) {
          zdc cp = ldz(&M[n]) * eip;
          zdc cm = n == 0 ? mkz(0.0) : sgn(n) * (ldz(&M[-n]) * eim);
          sp += (cp + cm) * h;
          if (GRAD) {
            zdc hd = n == 0 ? -hp / rs : rs * hm1 - ((double)n * zi1) * h;
            srad += (cp + cm) * hd;
            sang += ((double)n * zmul_i(cp - cm)) * h;
          }
          zdc hn = ((2.0 * (n + 1)) * zi) * hp - sc2 * h;
          hm1 = h;
          h = hp;
          hp = hn;
          eip = eip * ei;
          eim = eim * iei;
        }
        pot += sp;
        if (GRAD) {
          zdc vr1 = a1 / zr, vr2 = a2 / zr;
          zdc rad = srad * A.zk, ang = sang / zr;
          g1 += rad * vr1 - ang * vr2;
          g2 += rad * vr2 + ang * vr1;
        }
      }
      potsort[ti] = pot;
      if (GRAD) {
        gradsort[2 * ti] = g1;
        gradsort[2 * ti + 1] = g2;
      }
    }
  }
  __syncwarp();
  // P2P (zh2devaldirect) over list1: group of G lanes per target, added on top
  int pw = 1;
  while (pw < ntb && pw < 32) pw <<= 1;
  int G = 32 / pw, T = 32 / G, tl = lane / G, r = lane % G;
  int n1 = nl1[b];
  for (int base = 0; base < ntb; base += T) {
    int ti = t0 + base + tl;
    bool valid = base + tl < ntb;
    zdc pot = mkz(0.0), g1 = mkz(0.0), g2 = mkz(0.0);
    if (valid) {
      zdc x1 = ldz(&A.ztarg[2 * ti]), x2 = ldz(&A.ztarg[2 * ti + 1]);
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
          helm_pair<GRAD>(A.zk, x1, x2, ldz(&A.zsrc[2 * j]), ldz(&A.zsrc[2 * j + 1]), q, ds, d1, d2,
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
      potsort[ti] += pot;
      if (GRAD) {
        gradsort[2 * ti] += g1;
        gradsort[2 * ti + 1] += g2;
      }
    }
  }
}

}  // namespace

namespace {
// h2dterms for one level.  The reference evaluates H_n(z1) and J_n(z2) up to
// n = 50000 and returns the first n where the product has decayed below eps;
// the answer is found at a few times |z1|.  Here the tables are built to a
// bound that doubles until the criterion fires: J_n from Miller's recurrence
// does not depend on how far above n the recurrence started once it has
// converged, so the values, and the answer, are those of the full tables.
int h2dterms_eval(double bsize, zdc zk, double eps, int isep) {
  const int ntmax = 50000;
  zdc z1 = (zk * bsize) * (0.5 + isep * 1.0);
  double rscale = 1.0;
  const double pi2 = 8 * atan(1.0);
  if (zabs(zk * bsize) < pi2) rscale = zabs(zk * bsize);
  zdc z2 = (zk * bsize) * (sqrt(2.0) / 2.0);
  int nb = 64;
  while (true) {
    int n = nb < ntmax ? nb : ntmax;
    std::vector<zdc> hfun(n + 2), jfun(n + 2);
    h2dall(n, z1, rscale, hfun.data(), 0, nullptr);
    int ntop = jbessel_top(n, z2);
    std::vector<zdc> tmp(ntop + 2);
    jbessel2d(n, z2, rscale, jfun.data(), 0, nullptr, tmp.data(), ntop);
    double x0 = zabs(jfun[0] * hfun[0]) + zabs(jfun[1] * hfun[1]);
    for (int j = 2; j <= n; j++) {
      double x = (zabs(jfun[j] * hfun[j]) + zabs(jfun[j - 1] * hfun[j - 1])) * zabs(hfun[0]);
      if (x < eps * x0) return j + 1;
    }
    if (n >= ntmax) return 10001;  // the reference's "box too big" value
    nb *= 4;
  }
}

struct TermsKey {
  double bsize, zr, zi, eps;
  int isep;
  bool operator<(const TermsKey& o) const {
    return std::tie(bsize, zr, zi, eps, isep) < std::tie(o.bsize, o.zr, o.zi, o.eps, o.isep);
  }
};
std::mutex g_terms_mu;
std::map<TermsKey, int> g_terms_cache;
}  // namespace

int h2dterms_host(double bsize, zdc zk, double eps, int isep) {
  // h2dterms.f:35-97, results cached per (box size, zk, eps, isep)
  TermsKey key{bsize, zk.re, zk.im, eps, isep};
  {
    std::lock_guard<std::mutex> lk(g_terms_mu);
    auto it = g_terms_cache.find(key);
    if (it != g_terms_cache.end()) return it->second;
  }
  int n = h2dterms_eval(bsize, zk, eps, isep);
  std::lock_guard<std::mutex> lk(g_terms_mu);
  if (g_terms_cache.size() > 4096) g_terms_cache.clear();
  g_terms_cache[key] = n;
  return n;
}

// the passes after the set-up for one right-hand side with sorted strengths
// q, ds, dv on a set-up S: writes the sorted, unscaled potentials / gradients
// into potsort / gradsort (zeroed by the caller); ev (optional) gets the step
// boundaries 2..5; *pl (optional) receives the order of every level
int helm2d_core(const Setup2D& S, double eps, zdc zk, int isep, const zdc* q, const zdc* ds, const zdc* dv, int ifcharge, int ifdipole, int ifpgh,
         zdc* potsort, zdc* gradsort, cudaStream_t s, cudaEvent_t* ev,
         std::vector<int>* pl) {
  auto cmark = [&](int i) {
    if (ev) ZF_CUDA(cudaEventRecord(ev[i], s));
  };
  const DevTree& t = S.tree;
  int nb = t.nboxes, nlev = t.nlevels;
  if (nlev + 1 > MAXL) throw zf_error(ZF_ERR_ARG, "too many tree levels");
  HelmArgs A;
  A.zk = zk;
  long tot = 0;
  int pmax = 0;
  // Expansions of levels 0 and 1 are never read: lists 2-4 of those levels are
  // empty (the four level-1 boxes touch), so no box translates or evaluates
  // them.  They are not formed here (the reference forms the level-1
  // multipoles and never uses them); p of levels >= 2 bounds the work.
  for (int l = 0; l <= nlev; l++) {
    double a = zabs(zk * (t.boxsize[l] / (2.0 * ZF_PI)));
    A.T.rs[l] = a < 1.0 ? a : 1.0;
    A.T.p[l] = l >= 2 ? h2dterms_host(t.boxsize[l], zk, eps, isep) : 0;
    if (A.T.p[l] > 32 * MAXR - 1) throw zf_error(ZF_ERR_ARG, "expansion order too large");
    A.T.lo[l] = t.laddr[2 * l];
    A.T.base[l] = tot;
    tot += (long)(t.laddr[2 * l + 1] - t.laddr[2 * l] + 1) * (2 * A.T.p[l] + 1);
    if (A.T.p[l] > pmax) pmax = A.T.p[l];
  }
  DevBuf<zdc> mp(tot, s), loc(tot, s);
  mp.zero();
  loc.zero();
  A.ilevel = t.ilevel.get(); A.iparent = t.iparent.get(); A.nchild = t.nchild.get();
  A.ichild = t.ichild.get(); A.isrcse = S.isrcse.get(); A.itargse = S.itargse.get();
  A.zsrc = S.zsrcsort.get(); A.charge = q; A.dipstr = ds;
  A.dipvec = dv; A.ztarg = S.ztargsort.get(); A.zcsrc = S.zcsrc.get();
  A.zctarg = S.zctarg.get(); A.mp = mp.get(); A.loc = loc.get();
  A.ifcharge = ifcharge; A.ifdipole = ifdipole;
  const DevLists& L = S.lists;
  int grid_all = div_up(nb, WPB);
  // shared-memory strides (complex elements per warp)
  auto dense_stride = [](int ntt) { return (ntt + 2) + (2 * ntt + 1) + (ntt + 1 + 1); };
  // M2M / L2L: J table, two Toeplitz symbols, two weighted input vectors and
  // two real power tables
  auto trans_stride = [](int ntt, int nin) {
    return (ntt + 2) + 2 * (2 * ntt + 1) + 2 * (2 * nin + 1) + (ntt + 1);
  };
  // P2M per level (leaves of levels >= 2), shared memory sized by the level's order
  for (int l = 2; l <= nlev; l++) {
    int pl = A.T.p[l];
    size_t sm_p2m = (size_t)WPB * FCH * (pl + 2) * sizeof(zdc);
    int lo = t.laddr[2 * l], hi = t.laddr[2 * l + 1];
    ZF_CUDA(cudaFuncSetAttribute(k_hp2m, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_p2m));
    klaunch(k_hp2m, div_up(hi - lo + 1, WPB), 32 * WPB, sm_p2m, s, lo, hi, A, pl);
  }
  ZF_LAUNCH_CHECK();
  cmark(2);
  for (int l = nlev - 1; l >= 2; l--) {
    int lo = t.laddr[2 * l], hi = t.laddr[2 * l + 1];
    int stride = trans_stride(A.T.p[l] + A.T.p[l + 1], A.T.p[l + 1]);
    size_t sm = (size_t)WPB * stride * sizeof(zdc);
    ZF_CUDA(cudaFuncSetAttribute(k_hm2m, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    klaunch(k_hm2m, div_up(hi - lo + 1, WPB), 32 * WPB, sm, s, lo, hi, l, A, stride);
  }
  ZF_LAUNCH_CHECK();
  cmark(3);
  // one launch per level (lists 2 and 4 are empty on levels 0 and 1): the
  // shared-memory stride and the register slots follow the level's order, so
  // the many fine-level boxes run at full occupancy
  for (int l = 2; l <= nlev; l++) {
    int pl = A.T.p[l];
    int stride = dense_stride(2 * pl) + 2 * (2 * pl + 1);
    size_t sm = (size_t)WPB * stride * sizeof(zdc);
    int lo = t.laddr[2 * l], hi = t.laddr[2 * l + 1], grid = div_up(hi - lo + 1, WPB);
    auto go = [&](auto kern) {
      ZF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      klaunch(kern, grid, 32 * WPB, sm, s, lo, hi, A, L.n[1].get(), L.list[1].get(), L.mn[1],
              stride);
    };
    int R = (pl + 32) / 32;
    if (R <= 1) go(k_hm2l<1>);
    else if (R <= 2) go(k_hm2l<2>);
    else if (R <= 4) go(k_hm2l<4>);
    else go(k_hm2l<MAXR>);
  }
  ZF_LAUNCH_CHECK();
  if (L.mn[3] > 0)
    for (int l = 2; l <= nlev; l++) {
      int pl = A.T.p[l];
      int stride = FCH * (pl + 2);
      size_t sm = (size_t)WPB * stride * sizeof(zdc);
      int lo = t.laddr[2 * l], hi = t.laddr[2 * l + 1];
      ZF_CUDA(cudaFuncSetAttribute(k_hp2l, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      klaunch(k_hp2l, div_up(hi - lo + 1, WPB), 32 * WPB, sm, s, lo, hi, A, L.n[3].get(),
              L.list[3].get(), L.mn[3], stride);
    }
  ZF_LAUNCH_CHECK();
  cmark(4);
  for (int l = 2; l <= nlev - 1; l++) {
    int lo = t.laddr[2 * (l + 1)], hi = t.laddr[2 * (l + 1) + 1];
    int stride = trans_stride(A.T.p[l] + A.T.p[l + 1], A.T.p[l]);
    size_t sm = (size_t)WPB * stride * sizeof(zdc);
    ZF_CUDA(cudaFuncSetAttribute(k_hl2l, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    klaunch(k_hl2l, div_up(hi - lo + 1, WPB), 32 * WPB, sm, s, lo, hi, l, A, L.n[1].get(),
            L.n[3].get(), stride);
  }
  ZF_LAUNCH_CHECK();
  cmark(5);
  if (ifpgh > 1)
    klaunch(k_heval<true>, grid_all, 32 * WPB, 0, s, nb, A, L.n[0].get(), L.list[0].get(),
            L.mn[0], L.n[2].get(), L.list[2].get(), L.mn[2], potsort, gradsort);
  else
    klaunch(k_heval<false>, grid_all, 32 * WPB, 0, s, nb, A, L.n[0].get(), L.list[0].get(),
            L.mn[0], L.n[2].get(), L.list[2].get(), L.mn[2], potsort, gradsort);
  ZF_LAUNCH_CHECK();
  if (pl) *pl = std::vector<int>(A.T.p, A.T.p + nlev + 1);
  return pmax;
}

void zhfmm2d_device(double eps, zdc zk, const Inputs2D& in, int isep, zdc* pot, zdc* grad,
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
  tp.D = 2;
  tp.isep = isep;
  lndiv2d(eps, ns, nt, &tp.ndiv, &tp.idivflag);  // hndiv2d.f: same table
  Setup2D S;
  setup2d(in, tp, S, s);
  mark(1);
  std::vector<int> plv;
  DevBuf<zdc> potsort(nt, s), gradsort(in.ifpgh > 1 ? 2 * (size_t)nt : 1, s);
  potsort.zero();
  gradsort.zero();
  const int pord = helm2d_core(S, eps, zk, isep, S.chargesort.get(), S.dipstrsort.get(),
      S.dipvecsort.get(), in.ifcharge, in.ifdipole, in.ifpgh, potsort.get(), gradsort.get(), s,
      timing ? ev : nullptr, &plv);
  mark(6);
  unsort2d(nt, S.itarg.get(), potsort.get(), gradsort.get(), mkz(0.0, 0.25), in.ifpgh, pot, grad,
           s);
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
