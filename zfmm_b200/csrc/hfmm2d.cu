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
#include <cmath>
#include <cub/cub.cuh>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>
#include "fmm2d_common.cuh"
#include "hank2d.cuh"
#include "helm2d_pair.cuh"
#include "hfmm2d.cuh"
#include "lfmm2d.cuh"
#include "tc100.cuh"
#include "tune.cuh"

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
  ez = (a1 + zmul_i(a2)) * zinv(rz);
}

constexpr int MAXR = 8;  // M2M / M2L / L2L coefficient slots per lane: p <= 255

// ---- translation tables --------------------------------------------------------
// Every M2L, M2M and L2L translation of the reference (zh2dmploc, zh2dmpmp,
// zh2dlocloc) uses, per box pair, one table of scaled Bessel or Hankel
// functions of z = zk |c1 - c2| and the powers of the pair's angle factor
// e = (d1 + i d2)/|d| (zcart2polar; the reference's ezs(m) = ez^m).  The
// tables depend on the geometry and zk only, so they are built once per
// solve (or per plan and wavenumber) for all pairs, one thread per pair, and
// read by the translation kernels.  Entry k of a table is the pair
//   tab[k] = ( F_k e^k , (-1)^k F_k e^-k ),   k = 0..n,
// with F_k = H_k rs^k (h2dall, M2L) or F_k = J_k / rs^k (jbessel2d, M2M and
// L2L); a Bessel table carries Miller's normalisation factor in tab[n+1].

__device__ __forceinline__ double4 tab_entry(zdc u, zdc v) { return make_double4(u.re, u.im, v.re, v.im); }

// Scaled Hankel functions h2dall(n, z, rs) (h2dcommon.f:71-173: H0/H1, then the
// forward recurrence H_{k+1} = (2k/z) H_k - H_{k-1}; zero table for |z| < 1e-200)
// times the angle powers, running products of e and 1/e.
__device__ void hank_table(zdc z, zdc e, double rs, int n, double4* out) {
  if (zabs(z) < 1e-200) {
    for (int k = 0; k <= n; k++) out[k] = make_double4(0.0, 0.0, 0.0, 0.0);
    return;
  }
  zdc h0, h1;
  hank01(z, h0, h1);
  zdc ie = zinv(e), E = mkz(1.0), IE = mkz(1.0);
  zdc zi = rs * zinv(z);
  double sc2 = rs * rs;
  zdc hm = h0, h = h1 * rs;
  out[0] = tab_entry(h0, h0);
  for (int k = 1; k <= n; k++) {
    E = E * e;
    IE = IE * ie;
    out[k] = tab_entry(h * E, sgn(k) * (h * IE));
    zdc hn = ((2.0 * k) * zi) * h - sc2 * hm;
    hm = h;
    h = hn;
  }
}

// Scaled Bessel functions J_k/rs^k, k = 0..n, by the backward recurrence of
// jbessel2d (cdjseval2d.f:23-221) from the reference's start index, with the
// normalisation sum psi (e^{-+iz} = J0 + 2 sum (-+i)^k J_k) accumulated on the
// way down.  The entries are written unnormalised times the angle powers
// (e^k from e^n downwards); tab[n+1] = (e^{-+iz}/psi, 0) is applied by the
// reader.  On overflow the values written so far are rescaled, as the
// reference does.
__device__ void bessel_table(zdc z, zdc e, double rs, int n, double4* out) {
  if (zabs(z) < 1e-200) {
    out[0] = make_double4(1.0, 0.0, 1.0, 0.0);
    for (int k = 1; k <= n; k++) out[k] = make_double4(0.0, 0.0, 0.0, 0.0);
    out[n + 1] = make_double4(1.0, 0.0, 0.0, 0.0);
    return;
  }
  const int top = n + 1;  // jbessel2d's table runs to nterms + 1
  int ntop = jbessel_top(n, z);
  zdc zr = rs * zinv(z);
  double sc2 = rs * rs;
  zdc zmul = z.im < 0.0 ? mkz(0.0, 1.0) : mkz(0.0, -1.0);
  zdc ie = zinv(e);
  zdc E = zpown(e, n), IE = zpown(ie, n);
  zdc gp1 = mkz(0.0), g = mkz(1.0), psi = mkz(0.0), g0 = mkz(0.0);
  for (int k = ntop - 1; k >= 0; k--) {
    if (k <= n) {
      out[k] = tab_entry(g * E, sgn(k) * (g * IE));
      E = E * ie;
      IE = IE * e;
    }
    if (k == 0) g0 = g;
    if (k >= 1) {
      int r = k & 3;
      zdc zn = r == 0 ? mkz(1.0) : (r == 1 ? zmul : (r == 2 ? mkz(-1.0) : -zmul));
      psi = rs * psi + zn * g;
      zdc gm1 = ((2.0 * k) * zr) * g - sc2 * gp1;
      gp1 = g;
      g = gm1;
      if (zbig(g, 1e200)) {
        g = 1e-200 * g;
        gp1 = 1e-200 * gp1;
        psi = 1e-200 * psi;
        for (int j = k; j <= n; j++) {
          double4 v = out[j];
          out[j] = make_double4(1e-200 * v.x, 1e-200 * v.y, 1e-200 * v.z, 1e-200 * v.w);
        }
      }
    }
  }
  (void)top;
  psi = 2.0 * rs * psi + g0;
  zdc ex = z.im < 0.0 ? zexp_p(zmul_i(z)) : zexp_p(-zmul_i(z));
  zdc sc = ex / psi;
  out[n + 1] = make_double4(sc.re, sc.im, 0.0, 0.0);
}

struct TabArgs {
  double4* tab;
  // per-level real power tables (host-computed): rs^k for the M2L weights,
  // (rs1 rs2)^k and (rs2/rs1)^k for M2M, rs1^(2k) and (rs1/rs2)^k for L2L
  const double* pw;
  long pw_m2l[MAXL], pw_m2m[MAXL], pw_l2l[MAXL];
  long m2l_base[MAXL];   // first entry of the level's M2L tables
  long m2l_pair0[MAXL];  // first translated list-2 pair (pairoff order) of the level
  long ml_base[MAXL];    // first entry of the M2M / L2L tables of the children of level l
};

// The list-2 pairs that are translated: target box with targets, source box
// with sources (the conditions of zh2dmploc's call in the reference's step 3).
// They are numbered box by box in list order (pairoff[b] = first pair of box
// b), and the M2L tables are stored in that order, so the translation kernels
// find the k-th translated pair of box b at pairoff[b] + k.
__device__ __forceinline__ bool m2l_pair_used(const HelmArgs& A, int b, int jb) {
  return A.itargse[2 * b + 1] >= A.itargse[2 * b] && A.isrcse[2 * jb + 1] >= A.isrcse[2 * jb];
}

__global__ void k_m2l_pair_count(int nb, HelmArgs A, const int* nl2, const int* l2, int m2,
                                 int* cnt) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  int c = 0;
  for (int il = 0; il < nl2[b]; il++) c += m2l_pair_used(A, b, l2[(size_t)b * m2 + il]) ? 1 : 0;
  cnt[b] = c;
}

__global__ void k_m2l_pair_fill(int nb, HelmArgs A, const int* nl2, const int* l2, int m2,
                                const int* pairoff, int2* pairs) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  int k = pairoff[b];
  for (int il = 0; il < nl2[b]; il++) {
    int jb = l2[(size_t)b * m2 + il];
    if (m2l_pair_used(A, b, jb)) pairs[k++] = make_int2(b, jb);
  }
}

__global__ void k_m2l_box_flag(int nb, const int* pairoff, int* flag) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < nb) flag[b] = pairoff[b + 1] > pairoff[b] ? 1 : 0;
}
__global__ void k_m2l_box_scatter(int nb, const int* flag, const int* rank, int* boxes) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < nb && flag[b]) boxes[rank[b]] = b;
}

// M2L tables of the translated list-2 pairs q0 .. q1-1 (one thread per pair)
__global__ void __launch_bounds__(128) k_tab_m2l(long q0, long q1, HelmArgs A, TabArgs TA,
                                                 const int2* pairs) {
  long q = q0 + blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (q >= q1) return;
  const int2 pr = pairs[q];
  const int b = pr.x, jb = pr.y;
  int l = A.ilevel[b], p = A.T.p[l];
  zdc rz, e;
  polar(A.zctarg[2 * b] - A.zcsrc[2 * jb], A.zctarg[2 * b + 1] - A.zcsrc[2 * jb + 1], rz, e);
  hank_table(rz * A.zk, e, A.T.rs[l], 2 * p,
             TA.tab + TA.m2l_base[l] + (q - TA.m2l_pair0[l]) * (2 * p + 1));
}

// M2M and L2L tables of every box of levels >= 3 with its parent (one thread
// per child): M2M (zh2dmpmp, child multipole -> parent at the source centres,
// scale of the parent) if both hold sources; L2L (zh2dlocloc, parent local ->
// child at the target centres, scale of the child) if both hold targets and
// the parent has list-2 or list-4 boxes (the reference's step-7 test).
__global__ void __launch_bounds__(128) k_tab_m2m_l2l(int c0, int c1, HelmArgs A, TabArgs TA,
                                                     const int* nl2, const int* nl4) {
  int c = c0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (c > c1) return;
  int lc = A.ilevel[c];
  if (lc < 3) return;
  int b = A.iparent[c], l = lc - 1;
  int nt = A.T.p[l] + A.T.p[lc];
  double4* t = TA.tab + TA.ml_base[l] + (long)(c - A.T.lo[lc]) * 2 * (nt + 2);
  if (A.isrcse[2 * b + 1] >= A.isrcse[2 * b] && A.isrcse[2 * c + 1] >= A.isrcse[2 * c]) {
    zdc rz, e;
    polar(A.zcsrc[2 * b] - A.zcsrc[2 * c], A.zcsrc[2 * b + 1] - A.zcsrc[2 * c + 1], rz, e);
    bessel_table(rz * A.zk, e, A.T.rs[l], nt, t);
  }
  if (A.itargse[2 * b + 1] >= A.itargse[2 * b] && (nl2[b] > 0 || nl4[b] > 0) &&
      A.itargse[2 * c + 1] >= A.itargse[2 * c]) {
    zdc rz, e;
    polar(A.zctarg[2 * c] - A.zctarg[2 * b], A.zctarg[2 * c + 1] - A.zctarg[2 * b + 1], rz, e);
    bessel_table(rz * A.zk, e, A.T.rs[lc], nt, t + (nt + 2));
  }
}

// ---- step 1 / 6: P2M (zh2dformmp) and P2L (zh2dformloc) ------------------------
// One thread per (centre, source) computes the whole coefficient vector of the
// source about the centre (its Bessel or Hankel functions by the same
// recurrences as above, the powers ez^(+-m) as running products) into a
// column of global scratch; then one warp per centre sums its columns, lane i
// holding coefficients m = i - p (i = lane + 32 r).  Every lane of the column
// pass does work, whatever the number of sources per box.

struct SrcTerm {  // per-source factors of the P2M / P2L coefficients
  zdc q, ds, pr, pe_rz, izk;
};

__device__ __forceinline__ SrcTerm src_term(const HelmArgs& A, int j, zdc a1, zdc a2, zdc rzk) {
  SrcTerm t;
  t.q = A.ifcharge ? ldz(&A.charge[j]) : mkz(0.0);
  t.ds = mkz(0.0);
  t.pr = t.pe_rz = mkz(0.0);
  if (A.ifdipole) {
    t.ds = ldz(&A.dipstr[j]);
    zdc d1 = ldz(&A.dipvec[2 * j]), d2 = ldz(&A.dipvec[2 * j + 1]);
    zdc vr1 = a1 / rzk, vr2 = a2 / rzk;
    t.pr = vr1 * d1 + vr2 * d2;
    t.pe_rz = (-vr2 * d1 + vr1 * d2) / rzk;
  }
  t.izk = zinv(rzk * A.zk);
  return t;
}

// coefficients +m and -m of one source from f = F_m, its derivative fder and
// the powers em = ez^-m, ep = ez^m (zh2dformmp / zh2dformloc)
__device__ __forceinline__ void src_coeffs(const HelmArgs& A, const SrcTerm& t, int m, zdc fm,
                                           zdc fder, zdc em, zdc ep, zdc& cpos, zdc& cneg) {
  cpos = fm * em * t.q;
  cneg = sgn(m) * (fm * ep * t.q);
  if (A.ifdipole) {
    zdc dr = em * fder * A.zk, dth = fm * zdc{0.0, -(double)m} * em;
    cpos -= t.ds * (dr * t.pr + dth * t.pe_rz);
    zdc drn = ep * fder * A.zk, dthn = fm * zdc{0.0, (double)m} * ep;
    cneg -= t.ds * sgn(m) * (drn * t.pr + dthn * t.pe_rz);
  }
}

// P2M column of source j about centre (c1, c2): Bessel functions by the
// backward recurrence (coefficients emitted from m = p down to 0); returns
// Miller's normalisation factor of the column, which the column sum applies
// (a rescaling here would read and write the column a second time)
__device__ zdc p2m_column(const HelmArgs& A, int j, zdc c1, zdc c2, double rs, int p, zdc* col,
                          long cs) {
  zdc a1 = ldz(&A.zsrc[2 * j]) - c1, a2 = ldz(&A.zsrc[2 * j + 1]) - c2;
  zdc rzk, ez;
  polar(a1, a2, rzk, ez);
  SrcTerm t = src_term(A, j, a1, a2, rzk);
  zdc z = rzk * A.zk;
  if (zabs(z) < 1e-200) {  // jbessel2d's table for z = 0: J_0 = 1, the rest 0
    for (int m = 0; m <= p; m++) {
      zdc fm = m == 0 ? mkz(1.0) : mkz(0.0);
      zdc fder = m == 1 ? mkz(0.5 / rs) : mkz(0.0);
      zdc cp, cn;
      src_coeffs(A, t, m, fm, fder, mkz(1.0), mkz(1.0), cp, cn);
      col[(p + m) * cs] = cp;
      if (m) col[(p - m) * cs] = cn;
    }
    return mkz(1.0);
  }
  int ntop = jbessel_top(p, z);
  zdc zr = rs * zinv(z);
  double sc2 = rs * rs;
  zdc zmul = z.im < 0.0 ? mkz(0.0, 1.0) : mkz(0.0, -1.0);
  zdc iez = zinv(ez);
  zdc ep = zpown(ez, p), em = zpown(iez, p);
  zdc gp1 = mkz(0.0), g = mkz(1.0), psi = mkz(0.0), g0 = mkz(0.0);
  for (int n = ntop - 1; n >= 0; n--) {
    zdc gm1 = n >= 1 ? ((2.0 * n) * zr) * g - sc2 * gp1 : mkz(0.0);
    if (n <= p) {
      // F_{n-1}, F_n, F_{n+1} = gm1, g, gp1 (unnormalised); jbessel2d's
      // derivative: (F_{n-1}/rs - rs F_{n+1})/2, and -rs F_1 at n = 0
      zdc fder = n == 0 ? (-rs) * gp1 : (0.5 / rs) * gm1 - (0.5 * rs) * gp1;
      zdc cp, cn;
      src_coeffs(A, t, n, g, fder, em, ep, cp, cn);
      col[(p + n) * cs] = cp;
      if (n) col[(p - n) * cs] = cn;
      ep = ep * iez;
      em = em * ez;
    }
    if (n == 0) g0 = g;
    if (n >= 1) {
      int r = n & 3;
      zdc zn = r == 0 ? mkz(1.0) : (r == 1 ? zmul : (r == 2 ? mkz(-1.0) : -zmul));
      psi = rs * psi + zn * g;
      gp1 = g;
      g = gm1;
      if (zbig(g, 1e200)) {
        g = 1e-200 * g;
        gp1 = 1e-200 * gp1;
        psi = 1e-200 * psi;
        for (int m = n; m <= p; m++) {
          col[(p + m) * cs] = 1e-200 * col[(p + m) * cs];
          if (m) col[(p - m) * cs] = 1e-200 * col[(p - m) * cs];
        }
      }
    }
  }
  psi = 2.0 * rs * psi + g0;
  zdc ex = z.im < 0.0 ? zexp_p(zmul_i(z)) : zexp_p(-zmul_i(z));
  return ex / psi;
}

// P2L column of source j about centre (c1, c2): Hankel functions by the
// forward recurrence (h2dall), coefficients emitted from m = 0 up to p
__device__ void p2l_column(const HelmArgs& A, int j, zdc c1, zdc c2, double rs, int p, zdc* col,
                           long cs) {
  zdc a1 = ldz(&A.zsrc[2 * j]) - c1, a2 = ldz(&A.zsrc[2 * j + 1]) - c2;
  zdc rzk, ez;
  polar(a1, a2, rzk, ez);
  SrcTerm t = src_term(A, j, a1, a2, rzk);
  zdc z = rzk * A.zk;
  if (zabs(z) < 1e-200) {  // h2dall's zero table
    for (int i = 0; i <= 2 * p; i++) col[i * cs] = mkz(0.0);
    return;
  }
  zdc h0, h1;
  hank01(z, h0, h1);
  zdc zi = rs * zinv(z);
  double sc2 = rs * rs;
  zdc iez = zinv(ez), ep = mkz(1.0), em = mkz(1.0);
  zdc fm1 = mkz(0.0), f = h0, fp1 = h1 * rs;  // F_{m-1}, F_m, F_{m+1}
  const double irs = 1.0 / rs;
  for (int m = 0; m <= p; m++) {
    zdc fder = m == 0 ? -(fp1 * irs) : rs * fm1 - ((double)m * t.izk) * f;
    zdc cp, cn;
    src_coeffs(A, t, m, f, fder, em, ep, cp, cn);
    col[(p + m) * cs] = cp;
    if (m) col[(p - m) * cs] = cn;
    zdc fn = ((2.0 * (m + 1)) * zi) * fp1 - sc2 * f;
    fm1 = f;
    f = fp1;
    fp1 = fn;
    ep = ep * ez;
    em = em * iez;
  }
}

// The columns of a pass live in global scratch: colbase[b] is the first
// entry of box b's block (P2M: the box's own sources; P2L: the sources of its
// list-4 boxes in list order), stored coefficient-major: coefficient i of the
// box's k-th column at colbase[b] + i n_b + k (n_b columns), so the threads of
// neighbouring sources store to neighbouring addresses.

// leaf box of every source of a leaf of level >= 2 (-1 otherwise): the P2M
// centres, one thread per box
__global__ void k_src_leaf(int nb, HelmArgs A, int* srcleaf) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  int s0 = A.isrcse[2 * b], s1 = A.isrcse[2 * b + 1];
  if (A.nchild[b] > 0 || s1 < s0) return;
  int v = A.ilevel[b] >= 2 ? b : -1;
  for (int j = s0; j <= s1; j++) srcleaf[j] = v;
}

// per-box column counts: P2M sources of leaves of level >= 2 (w1 = sources,
// w2 = sources x (2p+1)); P2L sources of the list-4 boxes of target boxes
// (w3 = sources, w4 = sources x (2p+1))
__global__ void k_form_counts(int nb, HelmArgs A, const int* nl4, const int* l4, int m4,
                              long long* w1, long long* w2, long long* w3, long long* w4) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  int l = A.ilevel[b], P2 = 2 * A.T.p[l] + 1;
  long long c = 0;
  int s0 = A.isrcse[2 * b], s1 = A.isrcse[2 * b + 1];
  if (A.nchild[b] == 0 && s1 >= s0 && l >= 2) c = s1 - s0 + 1;
  w1[b] = c;
  w2[b] = c * P2;
  long long c4 = 0;
  if (A.itargse[2 * b + 1] >= A.itargse[2 * b] && l >= 2)
    for (int il = 0; il < nl4[b]; il++) {
      int jb = l4[(size_t)b * m4 + il];
      int n = A.isrcse[2 * jb + 1] - A.isrcse[2 * jb] + 1;
      if (n > 0) c4 += n;
    }
  w3[b] = c4;
  w4[b] = c4 * P2;
}

// P2M columns, one thread per source
__global__ void __launch_bounds__(128) k_p2m_cols(int ns, HelmArgs A, const int* srcleaf,
                                                  const long long* colcnt,
                                                  const long long* colbase, zdc* cols,
                                                  zdc* colscale) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ns) return;
  int b = srcleaf[j];
  if (b < 0) return;
  int l = A.ilevel[b], p = A.T.p[l];
  zdc* col = cols + colbase[b] + (j - A.isrcse[2 * b]);
  colscale[j] =
      p2m_column(A, j, A.zcsrc[2 * b], A.zcsrc[2 * b + 1], A.T.rs[l], p, col, (long)colcnt[b]);
}

// the (target box, list-4 source) pairs of the P2L columns, box by box in
// list order (pairs[off4[b] + k] = (b, source)), one thread per box
__global__ void k_p2l_pair_fill(int nb, HelmArgs A, const long long* cnt4, const long long* off4,
                                const int* nl4, const int* l4, int m4, int2* pairs) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb || cnt4[b] == 0) return;
  long long k = off4[b];
  for (int il = 0; il < nl4[b]; il++) {
    int jb = l4[(size_t)b * m4 + il];
    for (int j = A.isrcse[2 * jb]; j <= A.isrcse[2 * jb + 1]; j++) pairs[k++] = make_int2(b, j);
  }
}

// P2L columns, one thread per (target box, list-4 source) pair
__global__ void __launch_bounds__(128) k_p2l_cols(long long nq, HelmArgs A, const int2* pairs,
                                                  const long long* off4, const long long* colcnt,
                                                  const long long* colbase, zdc* cols) {
  long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (q >= nq) return;
  const int b = pairs[q].x, j = pairs[q].y;
  int l = A.ilevel[b], p = A.T.p[l];
  zdc* col = cols + colbase[b] + (q - off4[b]);
  p2l_column(A, j, A.zctarg[2 * b], A.zctarg[2 * b + 1], A.T.rs[l], p, col, (long)colcnt[b]);
}

// sums of the columns of every box of one level: warps loop over the boxes, R register
// slots per lane (2p+1 <= 32 R); P2M writes the multipole expansion (its
// columns times their sources' normalisation factors colscale[j]), P2L adds
// to the local expansion
template <int R, bool LOCAL>
__global__ void __launch_bounds__(32 * WPB) k_form_sum(int lo, int hi, HelmArgs A,
                                                       const long long* cnt,
                                                       const long long* colbase,
                                                       const zdc* cols, const zdc* colscale) {
  const int lane = threadIdx.x & 31;
  // every box of the launch is on one level; the warp loops over boxes
  const int p = A.T.p[A.ilevel[lo]], P2 = 2 * p + 1;
  for (int b = lo + blockIdx.x * WPB + (threadIdx.x >> 5); b <= hi; b += gridDim.x * WPB) {
    const long long n = cnt[b];
    if (n == 0) continue;
    const zdc* c = cols + colbase[b];
    zdc acc[R];
#pragma unroll
    for (int r = 0; r < R; r++) acc[r] = mkz(0.0);
    for (long long k = 0; k < n; k++) {
      // P2M: the columns are the box's own sources in order
      const zdc sc = LOCAL ? mkz(1.0) : ldz(&colscale[A.isrcse[2 * b] + k]);
#pragma unroll
      for (int r = 0; r < R; r++) {
        int i = lane + 32 * r;
        if (i < P2) acc[r] += LOCAL ? ldz(&c[i * n + k]) : ldz(&c[i * n + k]) * sc;
      }
    }
    zdc* E = expo(A, LOCAL ? A.loc : A.mp, b) - p;
#pragma unroll
    for (int r = 0; r < R; r++) {
      int i = lane + 32 * r;
      if (i < P2) {
        if (LOCAL) E[i] += acc[r];
        else E[i] = acc[r];
      }
    }
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
// The symbol S1[k] = (-1)^k J_k e^{-ik theta} comes from the pair's table.
// With g(d) = (rs1 rs2)^d for d > 0 and (rs1/rs2)^-d for d <= 0, the weight
// of every term with n of the sign of m (n != 0) is (rs2/rs1)^|m| g(|n|-|m|),
// and (rs1 rs2)^|n| for the others, so with the symbols S3[j] = S1[j] g(-j)
// and S4[k] = S1[k] g(k) the translation is branch-free:
//   mp(m)  = sum_{n<=0} S1[m-n] w(n) + (rs2/rs1)^m sum_{n>0} S3[m-n] mp_c(n)
//   mp(-m) = sum_{n>=0} S1[-m-n] w(n) + (rs2/rs1)^m sum_{n<0} S4[-m-n] mp_c(n)
// (w(n) = (rs1 rs2)^|n| mp_c(n)); rs1/rs2 is at most the box-size ratio, so
// the factors stay within the double range.
template <int R>
__global__ void __launch_bounds__(32 * WPB) k_hm2m(int lo, int hi, int lev, HelmArgs A,
                                                   TabArgs TA, int stride) {
  extern __shared__ zdc sh[];
  const int lane = threadIdx.x & 31;
  if (lo + blockIdx.x * WPB + (threadIdx.x >> 5) > hi) return;
  int n1 = A.T.p[lev], n2 = A.T.p[lev + 1], nt = n1 + n2;
  zdc* S1 = sh + (threadIdx.x >> 5) * stride + nt;  // S1[k], k = -nt..nt
  zdc* S3 = S1 + nt + 1 + nt;                       // S1[j] g(-j)
  zdc* S4 = S3 + nt + 1 + nt;                       // S1[k] g(k)
  zdc* ww = S4 + nt + 1 + n2;                       // (rs1 rs2)^|n| mp_child(n), n = -n2..n2
  zdc* mc = ww + n2 + 1 + n2;                       // mp_child(n)
  const double* qa = TA.pw + TA.pw_m2m[lev];        // (rs1 rs2)^k, k = 0..nt
  const double* qb = qa + nt + 1;                   // (rs2/rs1)^k
  const double* qi = qb + nt + 1;                   // (rs1/rs2)^k
  // the warp loops over the boxes of the level
  for (int b = lo + blockIdx.x * WPB + (threadIdx.x >> 5); b <= hi; b += gridDim.x * WPB) {
    if (A.nchild[b] == 0 || A.isrcse[2 * b + 1] < A.isrcse[2 * b]) continue;
    zdc accp[R], accm[R], acc0 = mkz(0.0);
  #pragma unroll
    for (int r = 0; r < R; r++) accp[r] = accm[r] = mkz(0.0);
    const int lc = lev + 1;
    for (int jc = 0; jc < 4; jc++) {
      int jb = A.ichild[4 * b + jc];
      if (A.isrcse[2 * jb + 1] < A.isrcse[2 * jb]) continue;
      const double4* t = TA.tab + TA.ml_base[lev] + (long)(jb - A.T.lo[lc]) * 2 * (nt + 2);
      double4 nv = t[nt + 1];
      zdc nrm = mkz(nv.x, nv.y);
      __syncwarp();
      for (int k = lane; k <= nt; k += 32) {
        double4 v = t[k];
        zdc u = nrm * mkz(v.x, v.y), vv = nrm * mkz(v.z, v.w);
        S1[k] = vv;   // (-1)^k J_k e^{-ik theta}
        S1[-k] = u;   // J_k e^{ik theta}
        double gp = k > 0 ? qa[k] : 1.0, gm = qi[k];  // g(k), g(-k)
        S3[k] = vv * gm;
        S3[-k] = u * gp;
        S4[k] = vv * gp;
        S4[-k] = u * gm;
      }
      const zdc* M2 = expo(A, A.mp, jb);
      for (int n = lane - n2; n <= n2; n += 32) {
        zdc v = M2[n];
        mc[n] = v;
        ww[n] = qa[abs(n)] * v;
      }
      __syncwarp();
  #pragma unroll
      for (int r = 0; r < R; r++) {
        int m = lane + 32 * r;
        if (m > n1) break;
        zdc a1 = mkz(0.0), a2 = mkz(0.0);
        for (int n = -n2; n <= 0; n++) a1 += S1[m - n] * ww[n];
        for (int n = 1; n <= n2; n++) a2 += S3[m - n] * mc[n];
        zdc sp = a1 + qb[m] * a2;
        if (m == 0) {
          acc0 += sp;
          continue;
        }
        a1 = mkz(0.0);
        a2 = mkz(0.0);
        for (int n = 0; n <= n2; n++) a1 += S1[-m - n] * ww[n];
        for (int n = -n2; n < 0; n++) a2 += S4[-m - n] * mc[n];
        accp[r] += sp;
        accm[r] += a1 + qb[m] * a2;
      }
    }
    zdc* M = expo(A, A.mp, b);
  #pragma unroll
    for (int r = 0; r < R; r++) {
      int m = lane + 32 * r;
      if (m > n1) break;
      if (m == 0) M[0] = acc0;
      else {
        M[m] = accp[r];
        M[-m] = accm[r];
      }
    }
  }
}

// M2L (zh2dmploc) over list 2.  With T[k] = H_k e^{ik theta} (k = -2p..2p,
// H_-k = (-1)^k H_k, scaled) the pair's Toeplitz symbol and b(n) the source
// coefficients, the reference's weight rs^|m| rs^|n| / rs^|n-m| is 1 for n, m
// of opposite signs and rs^(2 min(|m|,|n|)) otherwise, so for m >= 0
//   loc(m)  = sum_{n<0} T[n-m] b(n)  + sum_{n>=0} s(n,m) T[n-m] b(n)
//   loc(-m) = sum_{n<0} T[m-n] b(-n) + sum_{n>=0} s(n,m) T[m-n] b(-n)
// (the second is the first with T and b mirrored), s(n,m) = rs^(2 min(n,m)).
// Lane (h, k) of the warp computes the outputs m0 = 2k + 32r and m0 + 1 of the
// sum with sign sigma = +1 (h = 0: loc(+m)) or -1 (h = 1: loc(-m)), walking n
// upwards with a two-entry window of T: the entry T[sigma(n - m0 - 1)] used
// for m0 + 1 is the entry used for m0 one step earlier, so each step reads one
// entry of T and one of b for two multiply-adds.  T is kept split by parity
// (the lanes of a step read entries of one parity, 2 apart), so that the 16
// lanes of a half read 256 contiguous bytes.  R rounds of 32 outputs
// (p < 32 R).  The local expansion is written here; P2L adds to it afterwards.
__device__ __forceinline__ int tpos(int k, int n2) {  // position of T[k] in the split layout
  return (k & 1) * (n2 + 3) + ((k + n2 + 2) >> 1);
}
// shared-memory entries per warp of k_hm2l at order p: T split by parity with
// its two zero ends, rs^k (as doubles), b(n)
inline int hm2l_stride(int p) { return 2 * (2 * p + 3) + (2 * p + 2) + (2 * p + 1); }

// grid of a warp-per-box kernel whose warps loop over the boxes: as many CTAs
// as the SMs hold at once, and no more than there are groups of WPB boxes
// (a warp whose box has no work then moves on instead of holding its CTA)
template <class K>
int resident_grid(K kern, size_t smem, int nboxes) {
  int dev = 0, nsm = 0, per = 0;
  ZF_CUDA(cudaGetDevice(&dev));
  ZF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  ZF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, 32 * WPB, smem));
  return std::max(1, std::min(div_up(nboxes, WPB), nsm * std::max(per, 1)));
}

template <int R>
__global__ void __launch_bounds__(32 * WPB, R == 1 ? 8 : 4)
    k_hm2l(int nbx, const int* boxes, HelmArgs A, TabArgs TA, const int* pairoff,
           const int* nl2, const int* l2, int m2, int stride) {
  extern __shared__ zdc sh[];
  const int lane = threadIdx.x & 31;
  const int ib = blockIdx.x * WPB + (threadIdx.x >> 5);
  if (ib >= nbx) return;
  // boxes: the level's boxes with translated pairs, one warp each
  const int b = boxes[ib];
  const int l = A.ilevel[b], p = A.T.p[l], n2 = 2 * p;
  zdc* Ts = sh + (threadIdx.x >> 5) * stride;  // T[k], k = -n2-1..n2+1, split by parity
  double* rp = (double*)(Ts + 2 * (n2 + 3));    // rs^k, k = 0..n2
  zdc* bb = Ts + 2 * (n2 + 3) + (n2 + 2) + p;   // b(n), n = -p..p
  const int h = lane >> 4, kq = lane & 15, sg = h ? -1 : 1;
  for (int k = lane; k <= n2; k += 32) rp[k] = TA.pw[TA.pw_m2l[l] + k];
  if (lane == 0) {  // the two ends, read only for outputs m > p (discarded)
    Ts[tpos(-n2 - 1, n2)] = mkz(0.0);
    Ts[tpos(n2 + 1, n2)] = mkz(0.0);
  }
  __syncwarp();
  double rpm0[R], rpm1[R];
#pragma unroll
  for (int r = 0; r < R; r++) {
    const int m0 = 2 * kq + 32 * r;
    rpm0[r] = m0 <= p ? rp[2 * m0] : 0.0;
    rpm1[r] = m0 + 1 <= p ? rp[2 * m0 + 2] : 0.0;
  }
  const int n2c = nl2[b];
  zdc acc0[R], acc1[R];
#pragma unroll
  for (int r = 0; r < R; r++) acc0[r] = acc1[r] = mkz(0.0);
  const double4* tl = TA.tab + TA.m2l_base[l] + (pairoff[b] - TA.m2l_pair0[l]) * (long)(n2 + 1);
  int used = 0;  // translated pairs of the box so far
  for (int il = 0; il < n2c; il++) {
    int jb = l2[(size_t)b * m2 + il];
    if (A.isrcse[2 * jb + 1] < A.isrcse[2 * jb]) continue;
    __syncwarp();
    const double4* t = tl + (long)(used++) * (n2 + 1);
    for (int k = lane; k <= n2; k += 32) {
      double4 v = t[k];
      Ts[tpos(k, n2)] = mkz(v.x, v.y);
      Ts[tpos(-k, n2)] = mkz(v.z, v.w);
    }
    const zdc* M = expo(A, A.mp, jb);
    for (int n = lane - p; n <= p; n += 32) bb[n] = M[n];
    __syncwarp();
#pragma unroll
    for (int r = 0; r < R; r++) {
      const int m0 = 2 * kq + 32 * r;
      if (m0 > p) break;
      zdc prev = Ts[tpos(sg * (-p - 1 - m0), n2)];  // T[sg (n - m0 - 1)] at n = -p
      zdc s0 = mkz(0.0), s1 = mkz(0.0);
      for (int n = -p; n < 0; n++) {
        const zdc bn = bb[sg * n], cur = Ts[tpos(sg * (n - m0), n2)];
        s0 += cur * bn;
        s1 += prev * bn;
        prev = cur;
      }
      const int m1 = m0 + 1;
      for (int n = 0; n <= p; n++) {
        const zdc bn = bb[sg * n], cur = Ts[tpos(sg * (n - m0), n2)];
        const double rn = rp[2 * n];
        s0 += cur * ((n <= m0 ? rn : rpm0[r]) * bn);
        s1 += prev * ((n <= m1 ? rn : rpm1[r]) * bn);
        prev = cur;
      }
      acc0[r] += s0;
      acc1[r] += s1;
    }
  }
  zdc* L = expo(A, A.loc, b);
#pragma unroll
  for (int r = 0; r < R; r++) {
    const int m0 = 2 * kq + 32 * r, m1 = m0 + 1;
    if (m0 > p) break;
    if (m0 > 0 || h == 0) L[sg * m0] = acc0[r];  // loc(0) once, from the + half
    if (m1 <= p) L[sg * m1] = acc1[r];
  }
}

// ---- M2L of many right-hand sides on the tensor cores ------------------------
// For nd right-hand sides sharing one tree, the M2L of a box pair is the same
// complex matrix W (P2 x P2, W[m][n] = w(m, n) T[n - m] with the weights and
// symbol of k_hm2l) applied to nd multipole vectors: a complex product
// loc(P2 x nd) += W mp(P2 x nd), taken as the real product
//   [Re loc; Im loc] += [Re W, -Im W; Im W, Re W] [Re mp; Im mp]
// of a (2 P2) x (2 P2) matrix and (2 P2) x nd panel on the tcgen05 tensor
// cores (TF32 three-term split, FP32 accumulation in tensor memory, tc100.cuh),
// accumulated over all pairs of a target box before it is read back.  Used
// for plan solves at eps >= 1e-7 (the split's ~1e-7 relative accuracy) on
// levels with 2 P2 <= 128.  Right-hand side j of the expansions is
// mp + j * stride; 64 right-hand sides per launch (columns of D).
constexpr int TC_N = 64;

// smem words of the operands: A and B, hi and lo parts
__host__ __device__ inline size_t tc_m2l_smem(int p) {
  int kp = ((2 * (2 * p + 1) + 7) / 8) * 8;
  return (size_t)2 * (128 + TC_N) * kp * 4 + (size_t)(4 * p + 1) * 16 + (size_t)(2 * p + 1) * 8 +
         64;
}

__global__ void __launch_bounds__(128) k_hm2l_tc(int lo, int hi, HelmArgs A, TabArgs TA,
                                                 const int* pairoff, const int* nl2,
                                                 const int* l2, int m2, int nrhs, long stride,
                                                 int* err) {
  extern __shared__ __align__(1024) uint32_t tsm[];
  __shared__ uint64_t mbar;
  __shared__ uint32_t taddr_s;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int l = A.ilevel[lo], p = A.T.p[l], P2 = 2 * p + 1, n2 = 2 * p;
  const int K2 = 2 * P2, Kp = ((K2 + 7) / 8) * 8;
  uint32_t* ah = tsm;
  uint32_t* al = ah + 128 * Kp;
  uint32_t* bh = al + 128 * Kp;
  uint32_t* bl = bh + TC_N * Kp;
  zdc* T = reinterpret_cast<zdc*>(bl + TC_N * Kp);  // T[k], k = -2p..2p at T[n2 + k]
  double* rp = reinterpret_cast<double*>(T + 2 * n2 + 1);
  // padding rows / columns / right-hand sides stay zero
  for (int i = tid; i < 128 * Kp; i += 128) ah[i] = al[i] = 0u;
  for (int i = tid; i < TC_N * Kp; i += 128) bh[i] = bl[i] = 0u;
  for (int k = tid; k <= n2; k += 128) rp[k] = TA.pw[TA.pw_m2l[l] + k];
  if (warp == 0) tc::tmem_alloc(&taddr_s, TC_N);
  if (tid == 0) tc::mbar_init(&mbar, 1);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t taddr = taddr_s;
  const uint32_t idesc = tc::idesc_tf32(128, TC_N);
  const uint32_t achunk = 128 / 8 * 256, bchunk = TC_N / 8 * 256;
  uint32_t phase = 0;
  bool ok = true, pending = false;
  const double big = 3.0e37;  // beyond this an operand does not fit FP32
  for (int b = lo + blockIdx.x; b <= hi && ok; b += gridDim.x) {
    if (A.itargse[2 * b + 1] < A.itargse[2 * b]) continue;
    int n2c = nl2[b];
    if (n2c == 0) continue;
    const double4* tl =
        TA.tab + TA.m2l_base[l] + (pairoff[b] - TA.m2l_pair0[l]) * (long)(n2 + 1);
    int npairs = 0;
    for (int il = 0; il < n2c && ok; il++) {
      int jb = l2[(size_t)b * m2 + il];
      if (A.isrcse[2 * jb + 1] < A.isrcse[2 * jb]) continue;
      // operands of this pair (after the previous pair's MMAs have read theirs)
      if (npairs > 0) {
        ok = tc::mbar_wait(&mbar, phase, tc::kWaitLimit);
        ok = __syncthreads_and(ok);
        if (!ok) break;
        phase ^= 1;
        pending = false;
      }
      const double4* t = tl + (long)npairs * (n2 + 1);
      for (int k = tid; k <= n2; k += 128) {
        double4 v = t[k];
        T[n2 + k] = mkz(v.x, v.y);
        T[n2 - k] = mkz(v.z, v.w);
      }
      __syncthreads();
      bool inrange = true;
      for (int i = tid; i < P2 * P2; i += 128) {
        int mi = i / P2, ni = i - mi * P2, m = mi - p, n = ni - p;
        double w;
        if (m >= 0) w = n < 0 ? 1.0 : rp[2 * min(n, m)];
        else w = n > 0 ? 1.0 : rp[2 * min(-n, -m)];
        zdc W = w * T[n2 + n - m];
        inrange = inrange && fabs(W.re) < big && fabs(W.im) < big;
        uint32_t rh, rl, ih, il_, nh, nl;
        tc::split_tf32((float)W.re, rh, rl);
        tc::split_tf32((float)W.im, ih, il_);
        tc::split_tf32(-(float)W.im, nh, nl);
        uint32_t o1 = tc::kmajor_off(mi, ni, 128) >> 2, o2 = tc::kmajor_off(mi, P2 + ni, 128) >> 2;
        uint32_t o3 = tc::kmajor_off(P2 + mi, ni, 128) >> 2;
        uint32_t o4 = tc::kmajor_off(P2 + mi, P2 + ni, 128) >> 2;
        ah[o1] = rh; al[o1] = rl;    // Re W
        ah[o2] = nh; al[o2] = nl;    // -Im W
        ah[o3] = ih; al[o3] = il_;   // Im W
        ah[o4] = rh; al[o4] = rl;    // Re W
      }
      const zdc* M0 = expo(A, A.mp, jb) - p;
      for (int i = tid; i < nrhs * P2; i += 128) {
        int j = i / P2, ni = i - j * P2;
        zdc v = ldz(M0 + j * stride + ni);
        inrange = inrange && fabs(v.re) < big && fabs(v.im) < big;
        uint32_t h, lw;
        tc::split_tf32((float)v.re, h, lw);
        uint32_t o = tc::kmajor_off(j, ni, TC_N) >> 2;
        bh[o] = h; bl[o] = lw;
        tc::split_tf32((float)v.im, h, lw);
        o = tc::kmajor_off(j, P2 + ni, TC_N) >> 2;
        bh[o] = h; bl[o] = lw;
      }
      if (!inrange) atomicExch(err, 2);
      tc::fence_smem_async();
      tc::fence_before_sync();
      __syncthreads();
      tc::fence_after_sync();
      if (tid == 0) {
        for (int c = 0; c < Kp / 8; c++) {
          uint64_t dah = tc::make_desc(tc::smem_u32(ah) + c * achunk, 128, 256);
          uint64_t dal = tc::make_desc(tc::smem_u32(al) + c * achunk, 128, 256);
          uint64_t dbh = tc::make_desc(tc::smem_u32(bh) + c * bchunk, 128, 256);
          uint64_t dbl = tc::make_desc(tc::smem_u32(bl) + c * bchunk, 128, 256);
          tc::mma_tf32(taddr, dal, dbh, idesc, (npairs > 0 || c > 0) ? 1u : 0u);
          tc::mma_tf32(taddr, dah, dbl, idesc, 1u);
          tc::mma_tf32(taddr, dah, dbh, idesc, 1u);
        }
        tc::mma_commit(&mbar);
      }
      pending = true;
      npairs++;
    }
    if (!ok) break;
    // read the accumulated panel back: row r = 32 warp + lane of D
    zdc* L0 = expo(A, A.loc, b) - p;
    if (npairs > 0) {
      ok = tc::mbar_wait(&mbar, phase, tc::kWaitLimit);
      ok = __syncthreads_and(ok);
      if (!ok) break;
      phase ^= 1;
      pending = false;
      tc::fence_after_sync();
      int r = 32 * warp + lane;
      for (int c0 = 0; c0 < TC_N; c0 += 16) {
        float v[16];
        tc::tmem_ld16(taddr, warp, c0, v);
        if (r < K2) {
          int mi = r < P2 ? r : r - P2;
          double* dst = reinterpret_cast<double*>(L0 + mi) + (r < P2 ? 0 : 1);
#pragma unroll
          for (int i = 0; i < 16; i++)
            if (c0 + i < nrhs) dst[2 * (c0 + i) * stride] = (double)v[i];
        }
      }
      tc::fence_before_sync();
      __syncthreads();  // TMEM read before the next box's first MMA overwrites it
    } else {
      // every list-2 source box was empty: the local expansion is zero
      for (int i = tid; i < nrhs * P2; i += 128) {
        int j = i / P2, ni = i - j * P2;
        L0[j * stride + ni] = mkz(0.0);
      }
    }
  }
  if (!ok && tid == 0) atomicExch(err, 1);
  // an MMA batch that did not report completion: wait once more (bounded)
  // before the tensor memory it writes is released
  if (pending) tc::mbar_wait(&mbar, phase, tc::kWaitLimit);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(taddr, TC_N);
}

// L2L (zh2dlocloc) into the children at level lev+1
// L2L (zh2dlocloc): loc_child(m) += sum_n t(n-m) e^{i(n-m) theta} loc(n)
//   rs1^|m| rs1^|n-m| / rs2^|n|   (rs1 child, rs2 parent scale, rs1 <= rs2)
// split by signs: same sign with |n| >= |m|: (rs1/rs2)^|n|; same sign with
// |n| < |m| (and n = 0): (rs1/rs2)^|n| rs1^(2|k|); opposite: (rs1/rs2)^|n| rs1^(2|m|).
// The symbol S1[k] = J_k e^{ik theta} comes from the pair's table.
template <int R>
__global__ void __launch_bounds__(32 * WPB) k_hl2l(int lo, int hi, int lev, HelmArgs A,
                                                   TabArgs TA, const int* nl2, const int* nl4,
                                                   int stride) {
  extern __shared__ zdc sh[];
  const int lane = threadIdx.x & 31;
  if (lo + blockIdx.x * WPB + (threadIdx.x >> 5) > hi) return;
  int n1 = A.T.p[lev + 1], n2 = A.T.p[lev], nt = n1 + n2;
  zdc* S1 = sh + (threadIdx.x >> 5) * stride + nt;  // S1[k] = t(k) e^{ik theta}, k = -nt..nt
  zdc* S3 = S1 + nt + 1 + nt;                       // S1[k] rs1^(2|k|)
  zdc* uu = S3 + nt + 1 + n2;                       // (rs1/rs2)^|n| loc_parent(n)
  double* qa = (double*)(uu + n2 + 1);              // rs1^(2k), k = 0..nt
  double* qb = qa + nt + 1;                         // (rs1/rs2)^k, k = 0..nt
  for (int k = lane; k <= nt; k += 32) {
    qa[k] = TA.pw[TA.pw_l2l[lev] + k];
    qb[k] = TA.pw[TA.pw_l2l[lev] + nt + 1 + k];
  }
  // the warp loops over the child boxes of the level
  for (int jb = lo + blockIdx.x * WPB + (threadIdx.x >> 5); jb <= hi; jb += gridDim.x * WPB) {
    const int b = A.iparent[jb];
    if (A.itargse[2 * b + 1] < A.itargse[2 * b] || (nl2[b] == 0 && nl4[b] == 0)) continue;
    if (A.itargse[2 * jb + 1] < A.itargse[2 * jb]) continue;
    const double4* t =
        TA.tab + TA.ml_base[lev] + (long)(jb - A.T.lo[lev + 1]) * 2 * (nt + 2) + (nt + 2);
    double4 nv = t[nt + 1];
    zdc nrm = mkz(nv.x, nv.y);
    __syncwarp();
    for (int k = lane; k <= nt; k += 32) {
      double4 v = t[k];
      zdc u = nrm * mkz(v.x, v.y), vv = nrm * mkz(v.z, v.w);
      S1[k] = u;    // J_k e^{ik theta}
      S1[-k] = vv;  // (-1)^k J_k e^{-ik theta}
      S3[k] = u * qa[k];
      S3[-k] = vv * qa[k];
    }
    const zdc* L2 = expo(A, A.loc, b);
    for (int n = lane - n2; n <= n2; n += 32) uu[n] = qb[abs(n)] * L2[n];
    __syncwarp();
    zdc* L1 = expo(A, A.loc, jb);
    // per output the terms with n of the other sign form a plain Toeplitz sum
    // (times rs1^(2|m|)); for the others the symbol S1 or S3 is selected per
    // lane, so the loops have no branches
  #pragma unroll
    for (int r = 0; r < R; r++) {
      int m = lane + 32 * r;
      if (m > n1) break;
      zdc a1 = mkz(0.0), a2 = mkz(0.0);
      for (int n = -n2; n < 0; n++) a2 += S1[n - m] * uu[n];
      for (int n = 0; n <= n2; n++) a1 += (n >= m ? S1[n - m] : S3[n - m]) * uu[n];
      L1[m] += a1 + qa[m] * a2;
      if (m == 0) continue;
      a1 = mkz(0.0);
      a2 = mkz(0.0);
      for (int n = 1; n <= n2; n++) a2 += S1[n + m] * uu[n];
      for (int n = -n2; n <= 0; n++) a1 += (n <= -m ? S1[n + m] : S3[n + m]) * uu[n];
      L1[-m] += a1 + qa[m] * a2;
    }
  }
}

// ---- steps 5, 8: M2T (list 3) and L2T, one thread per target -------------------
// Every target of a leaf box runs its own L2T sweep and its M2T sums, so all
// lanes of a warp work whatever the number of targets per leaf.

// leaf box of every target (-1 for targets of no leaf: none)
__global__ void k_tgt_leaf(int nb, HelmArgs A, int* tgtleaf) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  int t0 = A.itargse[2 * b], t1 = A.itargse[2 * b + 1];
  if (A.nchild[b] > 0 || t1 < t0) return;
  for (int t = t0; t <= t1; t++) tgtleaf[t] = b;
}

template <bool GRAD>
__global__ void __launch_bounds__(128) k_hl2t(int nt, HelmArgs A, const int* tgtleaf,
                                              zdc* potsort, zdc* gradsort) {
  int ti = blockIdx.x * blockDim.x + threadIdx.x;
  if (ti >= nt) return;
  int b = tgtleaf[ti];
  if (b < 0) return;
  int lb = A.ilevel[b];
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
      zdc izz = zinv(z), zrr = rs * izz;
      double sc2 = rs * rs;
      const double irs = 1.0 / rs;
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
            zdc fd = n >= 1 ? gm1 * irs - ((double)n * izz) * g : (-rs) * gp1;
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
          if (zbig(g, 1e200)) {
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
  potsort[ti] = pot;
  if (GRAD) {
    gradsort[2 * ti] = g1;
    gradsort[2 * ti + 1] = g2;
  }
}

// M2T (zh2devalmp) over list 3, added to what L2T wrote.  The (target,
// list-3 box) pairs are numbered target by target in list order (boxes
// without sources left out, as the reference skips them); one thread per pair
// evaluates the box's multipole expansion at the target into scratch, then
// one thread per target adds its pairs in order.  Lanes of a warp thus never
// wait on a neighbour's longer list.
__global__ void k_m2t_count(int nt, HelmArgs A, const int* tgtleaf, const int* nl3,
                            const int* l3, int m3, int* cnt) {
  int ti = blockIdx.x * blockDim.x + threadIdx.x;
  if (ti >= nt) return;
  int b = tgtleaf[ti], c = 0;
  if (b >= 0)
    for (int il = 0; il < nl3[b]; il++) {
      int jb = l3[(size_t)b * m3 + il];
      c += A.isrcse[2 * jb + 1] >= A.isrcse[2 * jb] ? 1 : 0;
    }
  cnt[ti] = c;
}

__global__ void k_m2t_fill(int nt, HelmArgs A, const int* tgtleaf, const int* nl3,
                           const int* l3, int m3, const int* off, int2* pairs) {
  int ti = blockIdx.x * blockDim.x + threadIdx.x;
  if (ti >= nt) return;
  int b = tgtleaf[ti], k = off[ti];
  if (b < 0) return;
  for (int il = 0; il < nl3[b]; il++) {
    int jb = l3[(size_t)b * m3 + il];
    if (A.isrcse[2 * jb + 1] >= A.isrcse[2 * jb]) pairs[k++] = make_int2(ti, jb);
  }
}

// one (target, box) pair: vals[q * W ...] = pot (and the two gradient parts),
// used[q] = 0 when the pair contributes nothing (|zk R| below 1e-200)
template <bool GRAD>
__global__ void __launch_bounds__(128, 5) k_m2t_pairs(long npairs, HelmArgs A, const int2* pairs,
                                                   zdc* vals, int* used) {
  constexpr int W = GRAD ? 3 : 1;
  long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (q >= npairs) return;
  const int ti = pairs[q].x, jb = pairs[q].y;
  const zdc x1 = ldz(&A.ztarg[2 * ti]), x2 = ldz(&A.ztarg[2 * ti + 1]);
  int lj = A.ilevel[jb], p = A.T.p[lj];
  double rs = A.T.rs[lj];
  const zdc* M = expo(A, A.mp, jb);
  zdc zr, ei;
  zdc a1 = x1 - A.zcsrc[2 * jb], a2 = x2 - A.zcsrc[2 * jb + 1];
  polar(a1, a2, zr, ei);
  zdc z = zr * A.zk;
  if (zabs(z) < 1e-200) {
    used[q] = 0;
    return;
  }
  // streaming forward recurrence of H_n
  zdc h0, h1;
  hank01(z, h0, h1);
  zdc iei = zinv(ei), zi1 = zinv(z), zi = rs * zi1;
  double sc2 = rs * rs;
  const double irs = 1.0 / rs;
  zdc hm1 = mkz(0.0), h = h0, hp = h1 * rs;  // scaled H_{n-1}, H_n, H_{n+1}
  zdc eip = mkz(1.0), eim = mkz(1.0);
  zdc sp = mkz(0.0), srad = mkz(0.0), sang = mkz(0.0);
  for (int n = 0; n <= p; n++) {
    zdc cp = ldz(&M[n]) * eip;
    zdc cm = n == 0 ? mkz(0.0) : sgn(n) * (ldz(&M[-n]) * eim);
    sp += (cp + cm) * h;
    if (GRAD) {
      zdc hd = n == 0 ? -(hp * irs) : rs * hm1 - ((double)n * zi1) * h;
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
  used[q] = 1;
  vals[q * W] = sp;
  if (GRAD) {
    zdc vr1 = a1 / zr, vr2 = a2 / zr;
    zdc rad = srad * A.zk, ang = sang / zr;
    vals[q * W + 1] = rad * vr1 - ang * vr2;
    vals[q * W + 2] = rad * vr2 + ang * vr1;
  }
}

// the pairs of every target added to its entry, in list order
template <bool GRAD>
__global__ void k_m2t_sum(int nt, const int* off, const zdc* vals, const int* used,
                          zdc* potsort, zdc* gradsort) {
  constexpr int W = GRAD ? 3 : 1;
  int ti = blockIdx.x * blockDim.x + threadIdx.x;
  if (ti >= nt) return;
  const int q0 = off[ti], q1 = off[ti + 1];
  if (q1 == q0) return;
  zdc pot = potsort[ti], g1 = mkz(0.0), g2 = mkz(0.0);
  if (GRAD) {
    g1 = gradsort[2 * ti];
    g2 = gradsort[2 * ti + 1];
  }
  for (int q = q0; q < q1; q++) {
    if (!used[q]) continue;
    pot += vals[(long)q * W];
    if (GRAD) {
      g1 += vals[(long)q * W + 1];
      g2 += vals[(long)q * W + 2];
    }
  }
  potsort[ti] = pot;
  if (GRAD) {
    gradsort[2 * ti] = g1;
    gradsort[2 * ti + 1] = g2;
  }
}

// ---- step 3: P2P (list 1) one thread per target, added to L2T + M2T ----------
// Consecutive threads take consecutive sorted targets, so a warp covers one to
// a few neighbouring leaves with similar near fields, and no lane idles for
// want of targets in its leaf.  Each thread walks the sources of its list-1
// boxes (in list order, each box's sources in sorted order) as one flat loop,
// so lanes of different leaves in one warp cost the larger of their source
// counts rather than a sum over the boxes of the larger box.
template <bool GRAD>
__global__ void __launch_bounds__(128, 4) k_hp2p(int nt, HelmArgs A, const int* tgtleaf,
                                                 const int* nl1, const int* l1, int m1,
                                                 zdc* potsort, zdc* gradsort) {
  int ti = blockIdx.x * blockDim.x + threadIdx.x;
  if (ti >= nt) return;
  int b = tgtleaf[ti];
  if (b < 0) return;
  const HelmK K = helm_k(A.zk);
  const zdc x1 = ldz(&A.ztarg[2 * ti]), x2 = ldz(&A.ztarg[2 * ti + 1]);
  zdc pot = mkz(0.0), g1 = mkz(0.0), g2 = mkz(0.0);
  const int n1 = nl1[b];
  const int* lb = l1 + (size_t)b * m1;
  int il = 0, j = 0, s1 = -1;  // current source j of box lb[il], last source s1
  while (true) {
    while (j > s1 && il < n1) {  // next list-1 box with sources
      const int jb = lb[il++];
      j = A.isrcse[2 * jb];
      s1 = A.isrcse[2 * jb + 1];
    }
    if (j > s1) break;
    zdc q = A.ifcharge ? ldz(&A.charge[j]) : mkz(0.0);
    zdc ds = mkz(0.0), d1 = mkz(0.0), d2 = mkz(0.0);
    if (A.ifdipole) {
      ds = ldz(&A.dipstr[j]);
      d1 = ldz(&A.dipvec[2 * j]);
      d2 = ldz(&A.dipvec[2 * j + 1]);
    }
    helm_pair<GRAD>(K, x1, x2, ldz(&A.zsrc[2 * j]), ldz(&A.zsrc[2 * j + 1]), q, ds, d1, d2,
                    A.ifcharge, A.ifdipole, pot, g1, g2);
    j++;
  }
  potsort[ti] += pot;
  if (GRAD) {
    gradsort[2 * ti] += g1;
    gradsort[2 * ti + 1] += g2;
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
// Orders, scales and translation tables of the 2D Helmholtz passes for one
// tree and wavenumber (independent of the strengths: built once per solve,
// or once per plan solve for all its right-hand sides).
struct Helm2DPrep {
  HelmArgs A0;  // level table and geometry pointers (strength pointers unset)
  TabArgs TA;
  DevBuf<int> pairoff;
  // boxes with translated list-2 pairs in box order; those of level l are
  // m2l_boxes[m2l_box0[l] .. m2l_box0[l+1])
  DevBuf<int> m2l_boxes;
  std::vector<int> m2l_box0;
  DevBuf<double4> tab;
  DevBuf<double> pw;
  // P2M / P2L column layout: leaf box of every source; per box the number of
  // columns and the first column entry (P2M: own sources; P2L: list-4 sources)
  DevBuf<int> srcleaf, tgtleaf;  // leaf box of every sorted source / target
  // M2T pairs (target, list-3 box with sources): those of target t are
  // m2t_pairs[m2t_off[t] .. m2t_off[t+1])
  DevBuf<int> m2t_off;
  DevBuf<int2> m2t_pairs;
  long m2t_total = 0;
  DevBuf<long long> p2m_cnt, p2m_base, p2l_cnt, p2l_off, p2l_base;
  DevBuf<int2> p2l_pairs;  // (target box, list-4 source) of every P2L column
  long long p2m_total = 0, p2l_nq = 0, p2l_total = 0;
  int ns = 0, nt = 0;
  long tot = 0;
  int pmax = 0;
};

void Helm2DPrepDeleter::operator()(Helm2DPrep* p) const { delete p; }

namespace {
__global__ void k_pairoff_at(const int* pairoff, const int* idx, int n, int* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = pairoff[idx[i]];
}

__global__ void k_last_plus(const int* off, const int* cnt, int nb, int* out) {
  *out = off[nb - 1] + cnt[nb - 1];
}

__global__ void k_totals3(const long long* a, const long long* wa, const long long* b,
                          const long long* wb, const long long* c, const long long* wc, int nb,
                          long long* out) {
  out[0] = a[nb - 1] + wa[nb - 1];
  out[1] = b[nb - 1] + wb[nb - 1];
  out[2] = c[nb - 1] + wc[nb - 1];
}

void excl_scan_ll(const long long* in, long long* out, int n, cudaStream_t s) {
  size_t bytes = 0;
  ZF_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, s));
  DevBuf<char> tmp(bytes, s);
  ZF_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), bytes, in, out, n, s));
}
}  // namespace

Helm2DPrepPtr helm2d_prepare(const Setup2D& S, double eps, zdc zk, int isep, cudaStream_t s) {
  const DevTree& t = S.tree;
  int nb = t.nboxes, nlev = t.nlevels;
  if (nlev + 1 > MAXL) throw zf_error(ZF_ERR_ARG, "too many tree levels");
  Helm2DPrepPtr H(new Helm2DPrep());
  HelmArgs& A = H->A0;
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
  H->tot = tot;
  H->pmax = pmax;
  A.ilevel = t.ilevel.get(); A.iparent = t.iparent.get(); A.nchild = t.nchild.get();
  A.ichild = t.ichild.get(); A.isrcse = S.isrcse.get(); A.itargse = S.itargse.get();
  A.zsrc = S.zsrcsort.get(); A.ztarg = S.ztargsort.get(); A.zcsrc = S.zcsrc.get();
  A.zctarg = S.zctarg.get();
  const DevLists& L = S.lists;
  // translated list-2 pairs: offsets of every box, the pairs themselves, and
  // the first pair of every level
  H->pairoff.alloc(nb + 1, s);
  DevBuf<int2> m2l_pairs;
  {
    DevBuf<int> cnt(nb, s);
    klaunch(k_m2l_pair_count, div_up(nb, 128), 128, 0, s, nb, A, L.n[1].get(), L.list[1].get(),
            L.mn[1], cnt.get());
    size_t bytes = 0;
    ZF_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, cnt.get(), H->pairoff.get(), nb, s));
    DevBuf<char> tmp(bytes, s);
    ZF_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), bytes, cnt.get(), H->pairoff.get(), nb, s));
    klaunch(k_last_plus, 1, 1, 0, s, H->pairoff.get(), cnt.get(), nb, H->pairoff.get() + nb);
  }
  // the boxes with translated pairs (the M2L's work list)
  DevBuf<int> boxrank(nb + 1, s);
  H->m2l_boxes.alloc(nb, s);
  {
    DevBuf<int> fl(nb, s);
    klaunch(k_m2l_box_flag, div_up(nb, 128), 128, 0, s, nb, H->pairoff.get(), fl.get());
    size_t bytes = 0;
    ZF_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, fl.get(), boxrank.get(), nb, s));
    DevBuf<char> tmp(bytes, s);
    ZF_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), bytes, fl.get(), boxrank.get(), nb, s));
    klaunch(k_last_plus, 1, 1, 0, s, boxrank.get(), fl.get(), nb, boxrank.get() + nb);
    klaunch(k_m2l_box_scatter, div_up(nb, 128), 128, 0, s, nb, fl.get(), boxrank.get(),
            H->m2l_boxes.get());
  }
  std::vector<int> idx(nlev + 2);
  for (int l = 0; l <= nlev; l++) idx[l] = t.laddr[2 * l];
  idx[nlev + 1] = nb;
  DevBuf<int> didx(nlev + 2, s), dout(nlev + 2, s);
  ZF_CUDA(cudaMemcpyAsync(didx.get(), idx.data(), idx.size() * sizeof(int),
                          cudaMemcpyHostToDevice, s));
  klaunch(k_pairoff_at, 1, 64, 0, s, H->pairoff.get(), didx.get(), nlev + 2, dout.get());
  DevBuf<int> dbox0(nlev + 2, s);
  klaunch(k_pairoff_at, 1, 64, 0, s, boxrank.get(), didx.get(), nlev + 2, dbox0.get());
  std::vector<int> p0;
  // P2M / P2L column layout
  const int ns = (int)(S.zsrcsort.size() / 2);
  H->ns = ns;
  H->srcleaf.alloc(ns, s);
  H->srcleaf.fill_bytes(0xff);
  klaunch(k_src_leaf, div_up(nb, 128), 128, 0, s, nb, A, H->srcleaf.get());
  const int ntg = (int)(S.ztargsort.size() / 2);
  H->nt = ntg;
  H->tgtleaf.alloc(ntg, s);
  H->tgtleaf.fill_bytes(0xff);
  klaunch(k_tgt_leaf, div_up(nb, 128), 128, 0, s, nb, A, H->tgtleaf.get());
  H->m2t_off.alloc(ntg + 1, s);
  {
    DevBuf<int> cnt(std::max(ntg, 1), s);
    if (ntg > 0) {
      klaunch(k_m2t_count, div_up(ntg, 128), 128, 0, s, ntg, A, H->tgtleaf.get(), L.n[2].get(),
              L.list[2].get(), L.mn[2], cnt.get());
      size_t bytes = 0;
      ZF_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, cnt.get(), H->m2t_off.get(), ntg, s));
      DevBuf<char> tmp(bytes, s);
      ZF_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), bytes, cnt.get(), H->m2t_off.get(), ntg,
                                            s));
      klaunch(k_last_plus, 1, 1, 0, s, H->m2t_off.get(), cnt.get(), ntg, H->m2t_off.get() + ntg);
    } else {
      H->m2t_off.zero();
    }
  }
  H->p2m_cnt.alloc(nb, s);
  H->p2l_cnt.alloc(nb, s);
  H->p2m_base.alloc(nb, s);
  H->p2l_off.alloc(nb, s);
  H->p2l_base.alloc(nb, s);
  {
    DevBuf<long long> w2(nb, s), w4(nb, s), tot(3, s);
    klaunch(k_form_counts, div_up(nb, 128), 128, 0, s, nb, A, L.n[3].get(), L.list[3].get(),
            L.mn[3], H->p2m_cnt.get(), w2.get(), H->p2l_cnt.get(), w4.get());
    excl_scan_ll(w2.get(), H->p2m_base.get(), nb, s);
    excl_scan_ll(H->p2l_cnt.get(), H->p2l_off.get(), nb, s);
    excl_scan_ll(w4.get(), H->p2l_base.get(), nb, s);
    klaunch(k_totals3, 1, 1, 0, s, H->p2m_base.get(), w2.get(), H->p2l_off.get(),
            H->p2l_cnt.get(), H->p2l_base.get(), w4.get(), nb, tot.get());
    long long t3[3];
    ZF_CUDA(cudaMemcpyAsync(t3, tot.get(), sizeof(t3), cudaMemcpyDeviceToHost, s));
    std::vector<int> p0h(nlev + 2);
    ZF_CUDA(cudaMemcpyAsync(p0h.data(), dout.get(), p0h.size() * sizeof(int),
                            cudaMemcpyDeviceToHost, s));
    int m2t_n = 0;
    ZF_CUDA(cudaMemcpyAsync(&m2t_n, H->m2t_off.get() + ntg, sizeof(int), cudaMemcpyDeviceToHost,
                            s));
    H->m2l_box0.assign(nlev + 2, 0);
    ZF_CUDA(cudaMemcpyAsync(H->m2l_box0.data(), dbox0.get(), (nlev + 2) * sizeof(int),
                            cudaMemcpyDeviceToHost, s));
    ZF_CUDA(cudaStreamSynchronize(s));
    H->p2m_total = t3[0];
    H->p2l_nq = t3[1];
    H->p2l_total = t3[2];
    p0.swap(p0h);
    H->p2l_pairs.alloc(std::max(1LL, H->p2l_nq), s);
    if (H->p2l_nq > 0)
      klaunch(k_p2l_pair_fill, div_up(nb, 128), 128, 0, s, nb, A, H->p2l_cnt.get(),
              H->p2l_off.get(), L.n[3].get(), L.list[3].get(), L.mn[3], H->p2l_pairs.get());
    H->m2t_total = m2t_n;
    H->m2t_pairs.alloc(std::max(1, m2t_n), s);
    if (m2t_n > 0)
      klaunch(k_m2t_fill, div_up(ntg, 128), 128, 0, s, ntg, A, H->tgtleaf.get(), L.n[2].get(),
              L.list[2].get(), L.mn[2], H->m2t_off.get(), H->m2t_pairs.get());
  }
  // table layout: M2L tables of levels 2..nlev, then the M2M / L2L tables of
  // the children of levels 2..nlev-1
  TabArgs& TA = H->TA;
  long ntab = 0;
  for (int l = 0; l <= nlev; l++) {
    TA.m2l_pair0[l] = p0[l];
    TA.m2l_base[l] = ntab;
    if (l >= 2) ntab += (long)(p0[l + 1] - p0[l]) * (2 * A.T.p[l] + 1);
  }
  for (int l = 0; l <= nlev; l++) {
    TA.ml_base[l] = ntab;
    if (l >= 2 && l < nlev) {
      int nch = t.laddr[2 * (l + 1) + 1] - t.laddr[2 * (l + 1)] + 1;
      ntab += (long)nch * 2 * (A.T.p[l] + A.T.p[l + 1] + 2);
    }
  }
  H->tab.alloc(ntab > 0 ? ntab : 1, s);
  TA.tab = H->tab.get();
  // real power tables of the translation weights, one block per level
  std::vector<double> pw;
  for (int l = 0; l <= nlev; l++) {
    TA.pw_m2l[l] = (long)pw.size();
    if (l >= 2)
      for (int k = 0; k <= 2 * A.T.p[l]; k++) pw.push_back(std::pow(A.T.rs[l], (double)k));
    TA.pw_m2m[l] = TA.pw_l2l[l] = (long)pw.size();
    if (l >= 2 && l < nlev) {
      int nt = A.T.p[l] + A.T.p[l + 1];
      double rp = A.T.rs[l], rc = A.T.rs[l + 1];  // parent, child scales
      for (int k = 0; k <= nt; k++) pw.push_back(std::pow(rp * rc, (double)k));
      for (int k = 0; k <= nt; k++) pw.push_back(std::pow(rc / rp, (double)k));
      for (int k = 0; k <= nt; k++) pw.push_back(std::pow(rp / rc, (double)k));
      TA.pw_l2l[l] = (long)pw.size();
      for (int k = 0; k <= nt; k++) pw.push_back(std::pow(rc, 2.0 * k));
      for (int k = 0; k <= nt; k++) pw.push_back(std::pow(rc / rp, (double)k));
    }
  }
  H->pw.alloc(pw.size() > 0 ? pw.size() : 1, s);
  if (!pw.empty())
    ZF_CUDA(cudaMemcpyAsync(H->pw.get(), pw.data(), pw.size() * sizeof(double),
                            cudaMemcpyHostToDevice, s));
  TA.pw = H->pw.get();
  if (nlev >= 2) {
    long q0 = p0[2], q1 = p0[nlev + 1];
    m2l_pairs.alloc(std::max(1L, (long)p0[nlev + 1]), s);  // every translated pair
    klaunch(k_m2l_pair_fill, div_up(nb, 128), 128, 0, s, nb, A, L.n[1].get(), L.list[1].get(),
            L.mn[1], H->pairoff.get(), m2l_pairs.get());
    if (q1 > q0)
      tuned_launch("k_tab_m2l", q1 - q0, 128, {32, 64, 128}, [&](int bs) {
        klaunch(k_tab_m2l, div_up(q1 - q0, bs), bs, 0, s, q0, q1, A, TA, m2l_pairs.get());
      }, s);
  }
  if (nlev >= 3) {
    int c0 = t.laddr[6], c1 = nb - 1;
    tuned_launch("k_tab_m2m_l2l", c1 - c0 + 1, 128, {32, 64, 128}, [&](int bs) {
      klaunch(k_tab_m2m_l2l, div_up(c1 - c0 + 1, bs), bs, 0, s, c0, c1, A, TA, L.n[1].get(),
              L.n[3].get());
    }, s);
  }
  ZF_LAUNCH_CHECK();
  return H;
}

// the passes after the set-up for one right-hand side with sorted strengths
// q, ds, dv on a set-up S and its prepared tables H: writes the sorted,
// unscaled potentials / gradients into potsort / gradsort (zeroed by the
// caller); ev (optional) gets the step boundaries 2..5; *pl (optional)
// receives the order of every level
namespace {
enum Stage { ST_UP = 1, ST_M2L = 2, ST_DOWN = 4, ST_ALL = 7 };

// the passes of one right-hand side on expansions mp / loc (zeroed by the
// caller): ST_UP = P2M + M2M, ST_M2L = M2L, ST_DOWN = P2L, L2L, M2T, L2T and P2P
void helm2d_stages(const Setup2D& S, const Helm2DPrep& H, const zdc* q, const zdc* ds,
                   const zdc* dv, int ifcharge, int ifdipole, int ifpgh, zdc* mpp, zdc* locp,
                   int stages, zdc* potsort, zdc* gradsort, cudaStream_t s, cudaEvent_t* ev) {
  auto cmark = [&](int i) {
    if (ev) ZF_CUDA(cudaEventRecord(ev[i], s));
  };
  const DevTree& t = S.tree;
  const int nlev = t.nlevels;
  HelmArgs A = H.A0;
  const TabArgs& TA = H.TA;
  A.charge = q;
  A.dipstr = ds;
  A.dipvec = dv;
  A.mp = mpp;
  A.loc = locp;
  A.ifcharge = ifcharge;
  A.ifdipole = ifdipole;
  const DevLists& L = S.lists;
  // shared memory per warp (complex elements) of the M2M / L2L products: two
  // Toeplitz symbols of 2 nt + 1, two weighted input vectors and two real
  // power tables
  auto trans_stride = [](int ntt, int nin) {
    return 2 * (2 * ntt + 1) + 2 * (2 * nin + 1) + (ntt + 1);
  };
  auto slots = [](int ncoef) { return (ncoef + 31) / 32; };  // register slots per lane
  // a templated launch choosing R from {1, 2, 4, 8, 16} >= need
  auto pickR = [](int need) { return need <= 1 ? 1 : need <= 2 ? 2 : need <= 4 ? 4 : need <= 8 ? 8 : 16; };
  // P2M: columns of every source of a leaf of level >= 2, then per level the
  // sums over each leaf's columns
  if (stages & ST_UP) {
    DevBuf<zdc> cols(H.p2m_total > 0 ? H.p2m_total : 1, s), colscale(H.ns > 0 ? H.ns : 1, s);
    if (H.ns > 0)
      tuned_launch("k_p2m_cols", H.ns, 128, {32, 64, 128}, [&](int bs) {
        klaunch(k_p2m_cols, div_up(H.ns, bs), bs, 0, s, H.ns, A, H.srcleaf.get(),
                H.p2m_cnt.get(), H.p2m_base.get(), cols.get(), colscale.get());
      }, s);
    for (int l = 2; l <= nlev; l++) {
      int P2 = 2 * A.T.p[l] + 1;
      int lo = t.laddr[2 * l], hi = t.laddr[2 * l + 1];
      if (hi < lo) continue;
      auto go = [&](auto kern) {
        klaunch(kern, resident_grid(kern, 0, hi - lo + 1), 32 * WPB, 0, s, lo, hi, A,
                H.p2m_cnt.get(), H.p2m_base.get(), (const zdc*)cols.get(),
                (const zdc*)colscale.get());
      };
      switch (pickR(slots(P2))) {
        case 1: go(k_form_sum<1, false>); break;
        case 2: go(k_form_sum<2, false>); break;
        case 4: go(k_form_sum<4, false>); break;
        case 8: go(k_form_sum<8, false>); break;
        default: go(k_form_sum<16, false>); break;
      }
    }
  }
  ZF_LAUNCH_CHECK();
  cmark(2);
  for (int l = nlev - 1; l >= 2 && (stages & ST_UP); l--) {
    int lo = t.laddr[2 * l], hi = t.laddr[2 * l + 1];
    if (hi < lo) continue;
    int ntt = A.T.p[l] + A.T.p[l + 1], nin = A.T.p[l + 1];
    int stride = 3 * (2 * ntt + 1) + 2 * (2 * nin + 1);
    size_t sm = (size_t)WPB * stride * sizeof(zdc);
    auto go = [&](auto kern) {
      ZF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      klaunch(kern, resident_grid(kern, sm, hi - lo + 1), 32 * WPB, sm, s, lo, hi, l, A, TA,
              stride);
    };
    switch (pickR(slots(A.T.p[l] + 1))) {
      case 1: go(k_hm2m<1>); break;
      case 2: go(k_hm2m<2>); break;
      case 4: go(k_hm2m<4>); break;
      default: go(k_hm2m<MAXR>); break;
    }
  }
  ZF_LAUNCH_CHECK();
  cmark(3);
  // one launch per level (lists 2 and 4 are empty on levels 0 and 1): the
  // shared-memory stride and the register slots follow the level's order
  for (int l = 2; l <= nlev && (stages & ST_M2L); l++) {
    int pl_ = A.T.p[l];
    int stride = hm2l_stride(pl_);
    size_t sm = (size_t)WPB * stride * sizeof(zdc);
    const int nbx = H.m2l_box0[l + 1] - H.m2l_box0[l];
    if (nbx <= 0) continue;
    auto go = [&](auto kern) {
      ZF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      // one warp per box with translated pairs
      klaunch(kern, div_up(nbx, WPB), 32 * WPB, sm, s, nbx, H.m2l_boxes.get() + H.m2l_box0[l],
              A, TA, H.pairoff.get(), L.n[1].get(), L.list[1].get(), L.mn[1], stride);
    };
    switch (pickR(slots(pl_ + 1))) {
      case 1: go(k_hm2l<1>); break;
      case 2: go(k_hm2l<2>); break;
      case 4: go(k_hm2l<4>); break;
      default: go(k_hm2l<MAXR>); break;
    }
  }
  ZF_LAUNCH_CHECK();
  // P2L: columns of every (target box, list-4 source), then per level the sums
  // added to the local expansions
  if (H.p2l_nq > 0 && (stages & ST_DOWN)) {
    DevBuf<zdc> cols(H.p2l_total, s);
    tuned_launch("k_p2l_cols", H.p2l_nq, 128, {32, 64, 128}, [&](int bs) {
      klaunch(k_p2l_cols, div_up(H.p2l_nq, bs), bs, 0, s, H.p2l_nq, A, H.p2l_pairs.get(),
              H.p2l_off.get(), H.p2l_cnt.get(), H.p2l_base.get(), cols.get());
    }, s);
    for (int l = 2; l <= nlev; l++) {
      int P2 = 2 * A.T.p[l] + 1;
      int lo = t.laddr[2 * l], hi = t.laddr[2 * l + 1];
      if (hi < lo) continue;
      auto go = [&](auto kern) {
        klaunch(kern, resident_grid(kern, 0, hi - lo + 1), 32 * WPB, 0, s, lo, hi, A,
                H.p2l_cnt.get(), H.p2l_base.get(), (const zdc*)cols.get(), (const zdc*)nullptr);
      };
      switch (pickR(slots(P2))) {
        case 1: go(k_form_sum<1, true>); break;
        case 2: go(k_form_sum<2, true>); break;
        case 4: go(k_form_sum<4, true>); break;
        case 8: go(k_form_sum<8, true>); break;
        default: go(k_form_sum<16, true>); break;
      }
    }
  }
  ZF_LAUNCH_CHECK();
  cmark(4);
  for (int l = 2; l <= nlev - 1 && (stages & ST_DOWN); l++) {
    int lo = t.laddr[2 * (l + 1)], hi = t.laddr[2 * (l + 1) + 1];
    if (hi < lo) continue;
    int stride = trans_stride(A.T.p[l] + A.T.p[l + 1], A.T.p[l]);
    size_t sm = (size_t)WPB * stride * sizeof(zdc);
    auto go = [&](auto kern) {
      ZF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      klaunch(kern, resident_grid(kern, sm, hi - lo + 1), 32 * WPB, sm, s, lo, hi, l, A, TA,
              L.n[1].get(), L.n[3].get(), stride);
    };
    switch (pickR(slots(A.T.p[l + 1] + 1))) {
      case 1: go(k_hl2l<1>); break;
      case 2: go(k_hl2l<2>); break;
      case 4: go(k_hl2l<4>); break;
      default: go(k_hl2l<MAXR>); break;
    }
  }
  ZF_LAUNCH_CHECK();
  cmark(5);
  // L2T one thread per target (writes), then M2T and P2P one thread per target (add)
  const int ntt = H.nt;
  if (!(stages & ST_DOWN)) {
  } else {
    auto eval = [&](auto l2t, auto m2t, auto msum, auto p2p) {
      tuned_launch(ifpgh > 1 ? "k_hl2t_g" : "k_hl2t", ntt, 128, {64, 128}, [&](int bs) {
        klaunch(l2t, div_up(ntt, bs), bs, 0, s, ntt, A, H.tgtleaf.get(), potsort, gradsort);
      }, s);
      // M2T and P2P add to what L2T wrote (their block sizes are fixed: tuning
      // would have to restore the L2T results before every trial)
      if (H.m2t_total > 0) {
        const int W = ifpgh > 1 ? 3 : 1;
        DevBuf<zdc> vals((size_t)H.m2t_total * W, s);
        DevBuf<int> used(H.m2t_total, s);
        klaunch(m2t, div_up(H.m2t_total, 128L), 128, 0, s, H.m2t_total, A, H.m2t_pairs.get(),
                vals.get(), used.get());
        klaunch(msum, div_up(ntt, 128), 128, 0, s, ntt, H.m2t_off.get(),
                (const zdc*)vals.get(), (const int*)used.get(), potsort, gradsort);
      }
      klaunch(p2p, div_up(ntt, 128), 128, 0, s, ntt, A, H.tgtleaf.get(), L.n[0].get(),
              L.list[0].get(), L.mn[0], potsort, gradsort);
    };
    if (ifpgh > 1) eval(k_hl2t<true>, k_m2t_pairs<true>, k_m2t_sum<true>, k_hp2p<true>);
    else eval(k_hl2t<false>, k_m2t_pairs<false>, k_m2t_sum<false>, k_hp2p<false>);
  }
  ZF_LAUNCH_CHECK();
}
}  // namespace

int helm2d_passes(const Setup2D& S, const Helm2DPrep& H, const zdc* q, const zdc* ds,
                  const zdc* dv, int ifcharge, int ifdipole, int ifpgh, zdc* potsort,
                  zdc* gradsort, cudaStream_t s, cudaEvent_t* ev, std::vector<int>* pl) {
  DevBuf<zdc> mp(H.tot, s), loc(H.tot, s);
  mp.zero();
  loc.zero();
  helm2d_stages(S, H, q, ds, dv, ifcharge, ifdipole, ifpgh, mp.get(), loc.get(), ST_ALL,
                potsort, gradsort, s, ev);
  if (pl) *pl = std::vector<int>(H.A0.T.p, H.A0.T.p + S.tree.nlevels + 1);
  return H.pmax;
}

// nd right-hand sides on one prepared tree (the plan solve): the upward and
// downward passes run per right-hand side; the M2L of levels with
// 2 (2p+1) <= 128 runs for 64 right-hand sides at a time on the tensor cores
// when use_tc (eps >= 1e-7), every other level per right-hand side in FP64.
// Expansions of a group of right-hand sides are kept side by side; charge,
// dipstr (nd, ns), pot (nd, nt), grad (nd, 2, nt) as the plan solve's.
void helm2d_passes_nd(const Setup2D& S, const Helm2DPrep& H, int nd, int ifcharge,
                      const zdc* charge, int ifdipole, const zdc* dipstr, const zdc* dipvec,
                      int ifpgh, bool use_tc, zdc* pot, zdc* grad, cudaStream_t s, float* ms3) {
  const DevTree& t = S.tree;
  const int nlev = t.nlevels, ns = H.ns, nt = H.nt;
  const long tot = H.tot;
  const DevLists& L = S.lists;
  cudaEvent_t ev[4];
  for (auto& e : ev) ZF_CUDA(cudaEventCreate(&e));
  float acc[3] = {0, 0, 0};
  DevBuf<zdc> q(ns, s), ds(ns, s), dv(2 * (size_t)ns, s), potsort(nt, s),
      gradsort(ifpgh > 1 ? 2 * (size_t)nt : 1, s);
  DevBuf<int> err(1, s);
  err.zero();
  // right-hand sides per group: 64 (one tensor-core panel), fewer when the
  // expansions of 64 would exceed 24 GB
  const long budget = 24L << 30;
  const int G = (int)std::max(1L, std::min((long)TC_N, budget / (2 * tot * (long)sizeof(zdc))));
  DevBuf<zdc> mp((size_t)G * tot, s), loc((size_t)G * tot, s);
  for (int r0 = 0; r0 < nd; r0 += G) {
    const int nc = std::min(G, nd - r0);
    mp.zero();
    loc.zero();
    ZF_CUDA(cudaEventRecord(ev[0], s));
    for (int j = 0; j < nc; j++) {
      gather2d_col(S, ns, nd, r0 + j, ifcharge ? charge : nullptr, ifdipole ? dipstr : nullptr,
                   ifdipole ? dipvec : nullptr, q.get(), ds.get(), dv.get(), s);
      helm2d_stages(S, H, q.get(), ds.get(), dv.get(), ifcharge, ifdipole, ifpgh,
                    mp.get() + j * tot, loc.get() + j * tot, ST_UP, nullptr, nullptr, s,
                    nullptr);
    }
    ZF_CUDA(cudaEventRecord(ev[1], s));
    HelmArgs A = H.A0;
    A.mp = mp.get();
    A.loc = loc.get();
    for (int l = 2; l <= nlev; l++) {
      int p = A.T.p[l];
      int lo = t.laddr[2 * l], hi = t.laddr[2 * l + 1];
      if (hi < lo) continue;
      if (use_tc && 2 * (2 * p + 1) <= 128) {
        size_t sm = tc_m2l_smem(p);
        ZF_CUDA(cudaFuncSetAttribute(k_hm2l_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sm));
        // persistent CTAs: as many per SM as the shared memory holds (one CTA
        // builds its next pair's operands while another's MMAs run)
        int per_sm = std::max(1, (int)((227 * 1024) / (sm + 1024)));
        int grid = std::min(hi - lo + 1, 148 * per_sm);
        klaunch(k_hm2l_tc, grid, 128, sm, s, lo, hi, A, H.TA, H.pairoff.get(), L.n[1].get(),
                L.list[1].get(), L.mn[1], nc, tot, err.get());
      } else {
        for (int j = 0; j < nc; j++) {
          HelmArgs Aj = A;
          Aj.mp = mp.get() + j * tot;
          Aj.loc = loc.get() + j * tot;
          int stride = hm2l_stride(p);
          size_t sm = (size_t)WPB * stride * sizeof(zdc);
          auto slots = (p + 1 + 31) / 32;
          auto go = [&](auto kern) {
            ZF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sm));
            const int nbx = H.m2l_box0[l + 1] - H.m2l_box0[l];
            if (nbx > 0)
              klaunch(kern, div_up(nbx, WPB), 32 * WPB, sm, s, nbx,
                      H.m2l_boxes.get() + H.m2l_box0[l], Aj, H.TA, H.pairoff.get(),
                      L.n[1].get(), L.list[1].get(), L.mn[1], stride);
          };
          if (slots <= 1) go(k_hm2l<1>);
          else if (slots <= 2) go(k_hm2l<2>);
          else if (slots <= 4) go(k_hm2l<4>);
          else go(k_hm2l<MAXR>);
        }
      }
    }
    ZF_LAUNCH_CHECK();
    ZF_CUDA(cudaEventRecord(ev[2], s));
    for (int j = 0; j < nc; j++) {
      gather2d_col(S, ns, nd, r0 + j, ifcharge ? charge : nullptr, ifdipole ? dipstr : nullptr,
                   ifdipole ? dipvec : nullptr, q.get(), ds.get(), dv.get(), s);
      potsort.zero();
      gradsort.zero();
      helm2d_stages(S, H, q.get(), ds.get(), dv.get(), ifcharge, ifdipole, ifpgh,
                    mp.get() + j * tot, loc.get() + j * tot, ST_DOWN, potsort.get(),
                    gradsort.get(), s, nullptr);
      unsort2d_col(nt, nd, r0 + j, S.itarg.get(), potsort.get(), gradsort.get(), mkz(0.0, 0.25),
                   ifpgh, pot, grad, s);
    }
    ZF_CUDA(cudaEventRecord(ev[3], s));
    ZF_CUDA(cudaEventSynchronize(ev[3]));
    for (int k = 0; k < 3; k++) {
      float ms;
      ZF_CUDA(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
      acc[k] += ms;
    }
  }
  int h = 0;
  ZF_CUDA(cudaMemcpyAsync(&h, err.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
  ZF_CUDA(cudaStreamSynchronize(s));
  for (auto& e : ev) cudaEventDestroy(e);
  if (h == 1) throw zf_error(ZF_ERR_INTERNAL, "tensor-core M2L: completion wait timed out");
  if (h == 2) {
    // an operand outside the FP32 range: the whole solve again in FP64
    helm2d_passes_nd(S, H, nd, ifcharge, charge, ifdipole, dipstr, dipvec, ifpgh, false, pot,
                     grad, s, ms3);
    return;
  }
  if (ms3)
    for (int k = 0; k < 3; k++) ms3[k] = acc[k];
}

int helm2d_core(const Setup2D& S, double eps, zdc zk, int isep, const zdc* q, const zdc* ds,
                const zdc* dv, int ifcharge, int ifdipole, int ifpgh, zdc* potsort,
                zdc* gradsort, cudaStream_t s, cudaEvent_t* ev, std::vector<int>* pl) {
  Helm2DPrepPtr H = helm2d_prepare(S, eps, zk, isep, s);
  return helm2d_passes(S, *H, q, ds, dv, ifcharge, ifdipole, ifpgh, potsort, gradsort, s, ev, pl);
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
  // the translation tables belong to the set-up: they depend on the tree and
  // zk only
  Helm2DPrepPtr H = helm2d_prepare(S, eps, zk, isep, s);
  mark(1);
  std::vector<int> plv;
  DevBuf<zdc> potsort(nt, s), gradsort(in.ifpgh > 1 ? 2 * (size_t)nt : 1, s);
  potsort.zero();
  gradsort.zero();
  const int pord = helm2d_passes(S, *H, S.chargesort.get(), S.dipstrsort.get(),
                                 S.dipvecsort.get(), in.ifcharge, in.ifdipole, in.ifpgh,
                                 potsort.get(), gradsort.get(), s, timing ? ev : nullptr, &plv);
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
