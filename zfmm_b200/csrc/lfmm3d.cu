// 3D Laplace complex-coordinate FMM (zlfmm3d) on the device.
//
// Reference: zfmm3d/src/laplace/zlfmm3d.f (driver :14-245, zlfmm3dmain
// :252-622, direct sum :628-683, form/eval :689-1277, zl3dterms :1283-1321),
// the point-and-shoot translations of zfmm3d/src/laplace/zl3dtrans.f:1-570,
// the rotations of zfmm3d/src/common/zrotate.f:1-239 and the Legendre
// recurrences of zfmm3d/src/common/yrecursion.f:694-1415 and
// ztoolbox.f:110-327.
//
// Layout in HBM: one expansion per box, compact (n, m) order, coefficient
// (n, m), -n <= m <= n, at n*n + n + m, (p+1)^2 complex doubles per box; the
// expansion order p is the same on every level (the driver rescales the
// geometry to a unit root box).
//
// Kernels (one CTA per output box unless noted):
//   k_form3   P2M (leaves) and P2L (list 4): a warp per 32 sources, each lane
//             streams its source's Legendre recurrences and the warp reduces
//             every coefficient by shuffles into a per-warp partial expansion
//             in shared memory.
//   k_trans3  M2M / M2L / L2L by point and shoot: z-rotation (diagonal),
//             y-rotation by sampling the expansion at 2p+1 points of the
//             rotated meridian (one thread per sample, streaming the Legendre
//             column recurrences) and projecting back with a length-(2p+1)
//             DFT, axial shift (a Toeplitz/Hankel product per order m), and
//             the inverse rotations.  The three working arrays live in shared
//             memory; the output expansion is accumulated in registers.
//   k_eval3   L2T (own local) and M2T (list 3): a thread per target streams the
//             recurrences against the expansion staged in shared memory.
//   k_p2p3    list-1 direct interactions with sources staged through shared
//             memory.
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <vector>
#include "lap3d_pair.cuh"
#include "lfmm3d.cuh"
#include "sph3d.cuh"

namespace zf {

namespace {
Tab3 make_tab3(int p) {
  int L = p + 1, N = p, nmax = 2 * p, NS = 2 * p + 1;
  std::vector<double> r1((size_t)L * L, 0.0), r2((size_t)L * L, 0.0);
  // ylgndrini (yrecursion.f:694)
  auto R1 = [&](int n, int m) -> double& { return r1[(size_t)n * L + m]; };
  auto R2 = [&](int n, int m) -> double& { return r2[(size_t)n * L + m]; };
  R1(0, 0) = 1;
  R2(0, 0) = 1;
  for (int m = 0; m <= N; m++) {
    if (m > 0) {
      R1(m, m) = sqrt((2 * m - 1.0) / (2 * m));
      R2(m, m) = 1;
    }
    if (m < N) {
      R1(m + 1, m) = sqrt(2 * m + 1.0);
      R2(m + 1, m) = 1;
    }
    for (int k = m + 2; k <= N; k++) {
      R1(k, m) = (2 * k - 1) / sqrt((double)(k - m) * (k + m));
      R2(k, m) = sqrt((k + m - 1.0) * (k - m - 1.0)) / sqrt((double)(k - m) * (k + m));
    }
  }
  std::vector<double> sq(2 * p + 2);
  for (int n = 0; n <= 2 * p + 1; n++) sq[n] = sqrt(2 * n + 1.0);
  // get_amat (zl3dtrans.f:546-570)
  std::vector<double> amat((size_t)(nmax + 1) * (2 * nmax + 1), 0.0);
  {
    std::vector<double> facts(2 * nmax + 1);
    facts[0] = 1;
    for (int i = 1; i <= 2 * nmax; i++) facts[i] = sqrt(i + 0.0) * facts[i - 1];
    for (int n = 0; n <= nmax; n++) {
      double cst = ((n & 1) ? -1.0 : 1.0) * sqrt((2 * n + 1) * (1.0 / (4 * kPi)));
      for (int m = -n; m <= n; m++)
        amat[(size_t)n * (2 * nmax + 1) + m + nmax] = cst / facts[n - m] / facts[n + m];
    }
  }
  // zylgndr2sf at z = 0 (u = -1): the divisors yls - dyls of the projection
  // in z3dyrot; dinv = factor * (-1)^m / (yls - dyls), factor = sqrt(4 pi)/(2p+1)
  std::vector<double> Y((size_t)L * L, 0.0), D((size_t)L * L, 0.0), dinv((size_t)L * L, 0.0);
  {
    auto y = [&](int n, int m) -> double& { return Y[(size_t)n * L + m]; };
    auto d = [&](int n, int m) -> double& { return D[(size_t)n * L + m]; };
    double z = 0.0, u = -1.0;
    y(0, 0) = 1;
    d(0, 0) = 0;
    if (N > 0) {
      y(1, 0) = z * y(0, 0) * R1(1, 0);
      d(1, 0) = (z * d(0, 0) + y(0, 0)) * R1(1, 0);
    }
    for (int n = 2; n <= N; n++) {
      y(n, 0) = R1(n, 0) * z * y(n - 1, 0) - R2(n, 0) * y(n - 2, 0);
      d(n, 0) = R1(n, 0) * (z * d(n - 1, 0) + y(n - 1, 0)) - R2(n, 0) * d(n - 2, 0);
    }
    for (int m = 1; m <= N; m++) {
      y(m, m) = (m == 1) ? y(0, 0) * (-1.0) * R1(1, 1) : y(m - 1, m - 1) * u * R1(m, m);
      d(m, m) = y(m, m) * (double)(-m) * z;
      if (m < N) {
        y(m + 1, m) = z * y(m, m) * R1(m + 1, m);
        d(m + 1, m) = (z * d(m, m) + (1 - z * z) * y(m, m)) * R1(m + 1, m);
      }
      for (int n = m + 2; n <= N; n++) {
        y(n, m) = R1(n, m) * z * y(n - 1, m) - R2(n, m) * y(n - 2, m);
        d(n, m) = R1(n, m) * (z * d(n - 1, m) + (1 - z * z) * y(n - 1, m)) - R2(n, m) * d(n - 2, m);
      }
    }
    double factor = sqrt(4 * kPi) / (2 * N + 1);
    for (int n = 0; n <= N; n++)
      for (int m = 0; m <= n; m++) {
        double den = sq[n] * y(n, m) - sq[n] * d(n, m);
        double sg = (m & 1) ? -1.0 : 1.0;
        dinv[(size_t)n * L + m] = factor * sg / den;
      }
  }
  std::vector<zdc> tw(NS);
  for (int k = 0; k < NS; k++) {
    double a = 2 * kPi * k / NS;
    tw[k] = mkz(cos(a), -sin(a));
  }
  // one device block per (device, p), kept for the life of the process
  size_t nd = r1.size() + r2.size() + sq.size() + amat.size() + dinv.size();
  size_t bytes = nd * sizeof(double) + tw.size() * sizeof(zdc) + 64;
  char* base = nullptr;
  ZF_CUDA(cudaMalloc((void**)&base, bytes));
  size_t off = 0;
  auto put = [&](const void* src, size_t nbytes) {
    off = (off + 15) & ~(size_t)15;
    ZF_CUDA(cudaMemcpy(base + off, src, nbytes, cudaMemcpyHostToDevice));
    const void* q = base + off;
    off += nbytes;
    return q;
  };
  Tab3 T;
  T.p = p;
  T.NC = L * L;
  T.NS = NS;
  T.nmax = nmax;
  T.r1 = (const double*)put(r1.data(), r1.size() * sizeof(double));
  T.r2 = (const double*)put(r2.data(), r2.size() * sizeof(double));
  T.sq = (const double*)put(sq.data(), sq.size() * sizeof(double));
  T.amat = (const double*)put(amat.data(), amat.size() * sizeof(double));
  T.dinv = (const double*)put(dinv.data(), dinv.size() * sizeof(double));
  T.tw = (const zdc*)put(tw.data(), tw.size() * sizeof(zdc));
  return T;
}

}  // namespace

std::mutex g_tab_mu;
std::map<std::pair<int, int>, Tab3> g_tabs;

Tab3 get_tab3(int p) {
  int dev = 0;
  ZF_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_tab_mu);
  auto key = std::make_pair(dev, p);
  auto it = g_tabs.find(key);
  if (it != g_tabs.end()) return it->second;
  Tab3 T = make_tab3(p);
  g_tabs[key] = T;
  return T;
}

namespace {

constexpr int TNT = 256;                 // threads of the translation kernel
constexpr int FNT = 128;                 // threads of the form kernel (4 warps)
constexpr int ENT = 128;                 // threads of the eval / P2P kernels
constexpr int PTILE = 128;               // sources per P2P shared-memory tile

struct TransArgs {
  Tab3 T;
  const int *ilevel, *iparent, *nchild, *ichild, *isrcse, *itargse;
  const zdc *zcs, *zct;
  const double* rsc;  // rescaled min(boxsize, 1) per level
  const zdc* in;
  zdc* out;
  const int *nl2, *l2, *nl4;
  int mn2;
  int lo, hi;
};


// KIND 0: M2M into parent box, 1: M2L into target box, 2: L2L into child box
template <int KIND, int KMAX>
__global__ void __launch_bounds__(TNT, 2) k_trans3(TransArgs A) {
  extern __shared__ zdc sm[];
  const Tab3& T = A.T;
  const int p = T.p, NC = T.NC, NS = T.NS, tid = threadIdx.x;
  const int b = A.lo + blockIdx.x;
  if (b > A.hi) return;
  int nin = 0, par = -1;
  if (KIND == 0) {
    if (nsrc(A.isrcse, b) <= 0 || A.nchild[b] == 0) return;
    nin = A.nchild[b];
  } else if (KIND == 1) {
    if (nsrc(A.itargse, b) <= 0 || A.nl2[b] == 0) return;
    nin = A.nl2[b];
  } else {
    par = A.iparent[b];
    if (par < 0 || nsrc(A.itargse, b) <= 0 || nsrc(A.itargse, par) <= 0 ||
        (A.nl2[par] == 0 && A.nl4[par] == 0))
      return;
    nin = 1;
  }
  zdc* sA = sm;
  zdc* sB = sA + NC;
  zdc* sF = sB + NC;
  zdc* sEf = sF + (p + 1) * NS;
  zdc* sEb = sEf + NS;
  zdc* sG = sEb + NS;       // 2p+1
  zdc* sT1 = sG + 2 * p + 1;  // p+1
  zdc* sT2 = sT1 + p + 1;     // p+1
  zdc* sTw = sT2 + p + 1;     // NS
  for (int k = tid; k < NS; k += TNT) sTw[k] = T.tw[k];
  zdc acc[KMAX];
#pragma unroll
  for (int k = 0; k < KMAX; k++) acc[k] = mkz(0.0);
  const int lb = A.ilevel[b];
  const double s4 = sqrt(4 * kPi);
  const int nmax = T.nmax, ldA = 2 * nmax + 1;
  const double* __restrict__ am = T.amat;
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
    // shift_sign (zl3dtrans.f:327-540): the sign of the axial shift
    zdc zsh = g.zshift;
    bool flip = zabs(zsqrt_p(zsh * zsh) - zsh) > kF16;
    zdc rzs = flip ? -zsh : zsh;
    __syncthreads();  // previous translation done with every buffer
    // rotation factors e^{i m b} (forward) and e^{-i m b} (back)
    for (int m = tid; m <= p; m += TNT) {
      zdc ef = zpown(g.cb + zmul_i(g.sb), m), eb = zpown(g.cb - zmul_i(g.sb), m);
      sEf[p + m] = ef;
      sEf[p - m] = zinv(ef);
      sEb[p + m] = eb;
      sEb[p - m] = zinv(eb);
    }
    // shift tables
    if (KIND == 0) {
      zdc rz = rzs / rs0;
      for (int n = tid; n <= p; n += TNT) {
        double yl = __ldg(&T.sq[n]) * ((flip && (n & 1)) ? -1.0 : 1.0);
        sG[n] = (zpown(rz, n) * (__ldg(&am[n * ldA + nmax]) * yl)) / (2 * n + 1.0);
        sT1[n] = mkz(s4 * (ipow(rs0, n) / ipow(rs, n)));
      }
    } else if (KIND == 1) {
      zdc rz = rzs / rs0;
      for (int m = tid; m <= 2 * p; m += TNT) {
        double yl = __ldg(&T.sq[m]) * ((flip && (m & 1)) ? -1.0 : 1.0);
        sG[m] = yl / (zpown(rz, m) * __ldg(&am[m * ldA + nmax]));
      }
      for (int j = tid; j <= p; j += TNT) sT1[j] = (s4 / (2 * j + 1.0)) / rz;
    } else {
      zdc rz = rzs / rs;
      for (int n = tid; n <= p; n += TNT) {
        double yl = __ldg(&T.sq[n]) * ((flip && (n & 1)) ? -1.0 : 1.0);
        sG[n] = (zpown(rz, n) * (__ldg(&am[n * ldA + nmax]) * yl)) / (2 * n + 1.0);
        sT1[n] = mkz(s4 / (2 * n + 1.0) * ((n & 1) ? -1.0 : 1.0));
        sT2[n] = mkz((2 * n + 1.0) * (ipow(rs, n + 1) / ipow(rs0, n + 1)) * ((n & 1) ? -1.0 : 1.0));
      }
    }
    __syncthreads();
    // z-rotated input
    const zdc* __restrict__ ain = A.in + (size_t)src * NC;
#pragma unroll
    for (int k = 0; k < KMAX; k++) {
      int idx = tid + k * TNT;
      if (idx < NC) {
        zdc v = ain[idx];
        int n = deg3(idx);
        sA[idx] = g.zr ? v * sEf[p + idx - n * n - n] : v;
      }
    }
    __syncthreads();
    zdc* cur = sA;
    zdc* oth = sB;
    if (g.yr) {
      yrot_sample(p, p + 1, T.r1, T.r2, T.sq, cur, sF, g.ca, g.sa);
      __syncthreads();
      yrot_project<KMAX, TNT>(p, p + 1, T.dinv, 1.0, sF, oth, sTw);
      __syncthreads();
      zdc* t = cur; cur = oth; oth = t;
    }
    // axial shift: prescale the input in place, then the Toeplitz sums
#pragma unroll
    for (int k = 0; k < KMAX; k++) {
      int idx = tid + k * TNT;
      if (idx < NC) {
        int n = deg3(idx), m = idx - n * n - n;
        double an = __ldg(&am[n * ldA + m + nmax]);
        if (KIND == 0) cur[idx] = cur[idx] * an;
        else if (KIND == 1) cur[idx] = cur[idx] * (((n + m) & 1) ? -an : an);
        else cur[idx] = cur[idx] * sT2[n] / an;
      }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < KMAX; k++) {
      int idx = tid + k * TNT;
      if (idx < NC) {
        int j = deg3(idx), m = idx - j * j - j, am_ = m < 0 ? -m : m;
        zdc s0 = mkz(0.0);
        double ajk = __ldg(&am[j * ldA + m + nmax]);
        if (KIND == 0) {
          for (int n = am_; n <= j; n++) s0 += cur[ix3(n, m)] * sG[j - n];
          oth[idx] = sT1[j] * s0 / ajk;
        } else if (KIND == 1) {
          for (int n = am_; n <= p; n++) s0 += cur[ix3(n, m)] * sG[n + j];
          oth[idx] = sT1[j] * s0 * ajk;
        } else {
          for (int n = j; n <= p; n++) s0 += cur[ix3(n, m)] * sG[n - j];
          oth[idx] = sT1[j] * s0 * ajk;
        }
      }
    }
    __syncthreads();
    {
      zdc* t = cur; cur = oth; oth = t;
    }
    if (g.yr) {
      yrot_sample(p, p + 1, T.r1, T.r2, T.sq, cur, sF, g.ca, -g.sa);
      __syncthreads();
      yrot_project<KMAX, TNT>(p, p + 1, T.dinv, 1.0, sF, oth, sTw);
      __syncthreads();
      zdc* t = cur; cur = oth; oth = t;
    }
#pragma unroll
    for (int k = 0; k < KMAX; k++) {
      int idx = tid + k * TNT;
      if (idx < NC) {
        int n = deg3(idx);
        acc[k] += g.zr ? cur[idx] * sEb[p + idx - n * n - n] : cur[idx];
      }
    }
  }
  zdc* o = A.out + (size_t)b * NC;
#pragma unroll
  for (int k = 0; k < KMAX; k++) {
    int idx = tid + k * TNT;
    if (idx < NC) {
      if (KIND == 2) o[idx] += acc[k];
      else o[idx] = acc[k];
    }
  }
}

// ---- P2M / P2L ------------------------------------------------------------
struct FormArgs {
  Tab3 T;
  const int *ilevel, *nchild, *isrcse, *itargse;
  const zdc *zsrc, *charge, *dipstr, *dipvec;
  const zdc *zcs, *zct;
  const double* rsc;
  zdc* out;
  const int *nl4, *l4;
  int mn4, nb, ifcharge, ifdipole;
};

// zl3dformmp (LOCAL = false) / zl3dformloc (LOCAL = true), zlfmm3d.f:689-1005
template <bool LOCAL, bool DIP>
__device__ void form_range(const FormArgs& A, int s0, int s1, const zdc* zc, double rscale,
                           zdc* part) {
  const Tab3& T = A.T;
  const int p = T.p, L = p + 1, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const double s4 = 1.0 / sqrt(4 * kPi);
  const double* __restrict__ r1 = T.r1;
  const double* __restrict__ r2 = T.r2;
  const double* __restrict__ sq = T.sq;
  for (int base = s0 + 32 * w; base <= s1; base += 32 * (FNT / 32)) {
    int i = base + lane;
    bool valid = i <= s1;
    int ii = valid ? i : base;
    zdc q = (valid && A.ifcharge) ? A.charge[ii] : mkz(0.0);
    zdc ds = (valid && DIP) ? A.dipstr[ii] : mkz(0.0);
    Sph s = zcart2sph(A.zsrc[3 * ii], A.zsrc[3 * ii + 1], A.zsrc[3 * ii + 2], zc);
    zdc rz = s.rz / rscale;
    zdc irz = zinv(rz);
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
    // column start powers: rz^m (multipole) or rz^-(m+1) (local)
    zdc colp = LOCAL ? irz : mkz(1.0);
    zdc Ydiag = mkz(1.0), em = mkz(1.0);
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
      zdc rp = colp;                                 // rz^n or rz^-(n+1)
      zdc rpm1 = (m > 0) ? colp * irz : mkz(0.0);    // rz^(n-1) (multipole dipole)
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
            if (DIP) D = (m == 0) ? c1 * (z * Dp + Yp) - c2 * Dpp : c1 * (z * Dp + zz1 * Yp) - c2 * Dpp;
          }
          Ypp = Yp; Dpp = Dp; Yp = Y; Dp = D;
          rpm1 = rp;
          rp = rp * (LOCAL ? irz : rz);
        }
        double f = __ldg(&sq[n]) * (s4 * sgm / (2 * n + 1.0));
        zdc y = Y * f, dy = D * f;
        zdc cpos, cneg;
        if (m == 0) {
          zdc c0 = q * rp * y;
          if (DIP) {
            zdc dzr, dth;
            if (!LOCAL) {
              dzr = n == 0 ? mkz(0.0) : ((double)n * rpm1 / rscale) * y;
              dth = -(rp * dy * s.st);
            } else {
              dzr = -((double)(n + 1) * y * rp / s.rz);
              dth = -(dy * s.st * rp);
            }
            c0 -= ds * (dzr_ * dzr + dthz * dth);
          }
          cpos = c0;
          cneg = mkz(0.0);
        } else {
          zdc ys = DIP ? s.st * y : y;
          zdc X = q * rp * ys, W = mkz(0.0);
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
            X -= ds * (dzr_ * DZ + dthz * DT);
            W = ds * (dphz * zmul_i((double)m * DP));
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
__global__ void __launch_bounds__(FNT) k_form3(FormArgs A) {
  extern __shared__ zdc sm[];
  const int NC = A.T.NC, tid = threadIdx.x, w = tid >> 5;
  const int b = blockIdx.x;
  if (b >= A.nb) return;
  int l = A.ilevel[b];
  if (!LOCAL) {
    if (A.nchild[b] != 0 || nsrc(A.isrcse, b) <= 0 || l < 1) return;
  } else {
    if (nsrc(A.itargse, b) <= 0 || A.nl4[b] == 0) return;
  }
  zdc* part = sm + w * NC;
  for (int k = tid; k < (FNT / 32) * NC; k += FNT) sm[k] = mkz(0.0);
  __syncthreads();
  if (!LOCAL) {
    form_range<false, DIP>(A, A.isrcse[2 * b], A.isrcse[2 * b + 1], A.zcs + 3 * b, A.rsc[l], part);
  } else {
    for (int i = 0; i < A.nl4[b]; i++) {
      int jb = A.l4[(size_t)b * A.mn4 + i];
      if (nsrc(A.isrcse, jb) <= 0) continue;
      form_range<true, DIP>(A, A.isrcse[2 * jb], A.isrcse[2 * jb + 1], A.zct + 3 * b, A.rsc[l],
                            part);
    }
  }
  __syncthreads();
  zdc* o = A.out + (size_t)b * NC;
  for (int k = tid; k < NC; k += FNT) {
    zdc v = sm[k];
    for (int ww = 1; ww < FNT / 32; ww++) v += sm[ww * NC + k];
    if (LOCAL) o[k] += v;
    else o[k] = v;
  }
}

// ---- L2T / M2T --------------------------------------------------------------
struct EvalArgs {
  Tab3 T;
  const int *ilevel, *nchild, *isrcse, *itargse;
  const zdc *ztarg, *zcs, *zct;
  const double* rsc;
  const zdc *mp, *loc;
  const int *nl3, *l3;
  int mn3, nb;
  zdc *pot, *grad;
};

// zl3devalmp (LOCAL = false) / zl3devalloc (LOCAL = true), zlfmm3d.f:1011-1277;
// the gradient is accumulated in spherical components and mapped once.
template <bool GRAD, bool LOCAL>
__device__ __forceinline__ void eval_one(const Tab3& T, const zdc* __restrict__ e, const zdc* x,
                                         const zdc* zc, double rscale, zdc& pot, zdc* grad) {
  const int p = T.p, L = p + 1;
  const double s4 = 1.0 / sqrt(4 * kPi);
  const double* __restrict__ r1 = T.r1;
  const double* __restrict__ r2 = T.r2;
  const double* __restrict__ sq = T.sq;
  Sph s = zcart2sph(x[0], x[1], x[2], zc);
  zdc rz = s.rz / rscale, irz = zinv(rz);
  const zdc z = s.ct, zz1 = mkz(1.0) - z * z;
  const zdc u = -zsqrt_r(zz1);
  zdc P = mkz(0.0), Gr = mkz(0.0), Gt = mkz(0.0), Gp = mkz(0.0);
  zdc colp = LOCAL ? mkz(1.0) : irz;  // rz^n (local) or rz^-(n+1) (multipole) at n = m
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
    zdc rfm1 = (LOCAL && m > 0) ? colp * irz : mkz(0.0);  // rz^(n-1) (local gradient)
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
          if (GRAD) D = (m == 0) ? c1 * (z * Dp + Yp) - c2 * Dpp : c1 * (z * Dp + zz1 * Yp) - c2 * Dpp;
        }
        Ypp = Yp; Dpp = Dp; Yp = Y; Dp = D;
        rfm1 = rf;
        rf = rf * (LOCAL ? rz : irz);
      }
      double f = __ldg(&sq[n]) * f0;
      zdc y = Y * f;
      if (m == 0) {
        zdc c0 = e[ix3(n, 0)];
        P += c0 * y * rf;
        if (GRAD) {
          zdc dy = D * f;
          zdc dzr, dth;
          if (!LOCAL) {
            dzr = -((double)(n + 1) * y * rf / s.rz);
            dth = -(dy * s.st * rf);
          } else {
            dzr = n == 0 ? mkz(0.0) : ((double)n * rfm1 / rscale) * y;
            dth = -(rf * dy * s.st);
          }
          Gr += c0 * dzr;
          Gt += c0 * dth;
        }
      } else {
        zdc a = e[ix3(n, m)] * em, bm = e[ix3(n, -m)] * emi;
        zdc Sp = a + bm;
        zdc ys = GRAD ? y * s.st : y;
        P += ys * Sp * rf;
        if (GRAD) {
          zdc Sm = a - bm;
          zdc dy = D * f;
          zdc DZ, DT;
          if (!LOCAL) {
            DZ = -((double)(n + 1) * ys * rf / s.rz);
            DT = -(dy * rf);
          } else {
            DZ = ((double)n * rfm1 / rscale) * ys;
            DT = -(rf * dy);
          }
          Gr += DZ * Sp;
          Gt += DT * Sp;
          Gp += zmul_i((double)m * y * rf) * Sm;
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
__global__ void __launch_bounds__(ENT) k_eval3(EvalArgs A) {
  extern __shared__ zdc sm[];
  const Tab3& T = A.T;
  const int NC = T.NC, tid = threadIdx.x;
  const int b = blockIdx.x;
  if (b >= A.nb) return;
  const int t0 = A.itargse[2 * b], t1 = A.itargse[2 * b + 1];
  if (A.nchild[b] != 0 || t1 < t0) return;
  const int lb = A.ilevel[b];
  const bool own = lb >= 2;  // levels 0 and 1 receive no local expansion
  int nexp = (own ? 1 : 0) + A.nl3[b];
  if (nexp == 0) return;
  for (int c0 = t0; c0 <= t1; c0 += ENT) {
    int i = c0 + tid;
    bool valid = i <= t1;
    zdc x[3];
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
      __syncthreads();
      const zdc* src = (loc ? A.loc : A.mp) + (size_t)eb * NC;
      for (int k = tid; k < NC; k += ENT) sm[k] = src[k];
      __syncthreads();
      if (valid) {
        if (loc) eval_one<GRAD, true>(T, sm, x, A.zct + 3 * eb, A.rsc[A.ilevel[eb]], pot, g);
        else eval_one<GRAD, false>(T, sm, x, A.zcs + 3 * eb, A.rsc[A.ilevel[eb]], pot, g);
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
struct P2PArgs {
  const int *nchild, *isrcse, *itargse;
  const zdc *zsrc, *charge, *dipstr, *dipvec, *ztarg;
  const int *nl1, *l1;
  int mn1, nb, ifcharge, ifdipole;
  zdc *pot, *grad;
};

struct SrcTile {
  zdc y[PTILE][3];
  zdc q[PTILE], ds[PTILE];
  zdc v[PTILE][3];
};

__device__ __forceinline__ void stage_sources(SrcTile& S, int j0, int n, const zdc* zsrc,
                                              const zdc* charge, const zdc* dipstr,
                                              const zdc* dipvec, int ifcharge, int ifdipole,
                                              int nthreads) {
  for (int k = threadIdx.x; k < n; k += nthreads) {
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

template <bool GRAD>
__global__ void __launch_bounds__(ENT) k_p2p3(P2PArgs A) {
  __shared__ SrcTile S;
  const int b = blockIdx.x;
  if (b >= A.nb) return;
  const int t0 = A.itargse[2 * b], t1 = A.itargse[2 * b + 1];
  if (A.nchild[b] != 0 || t1 < t0 || A.nl1[b] == 0) return;
  for (int c0 = t0; c0 <= t1; c0 += ENT) {
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
      for (int j0 = s0; j0 <= s1; j0 += PTILE) {
        int n = min(PTILE, s1 - j0 + 1);
        __syncthreads();
        stage_sources(S, j0, n, A.zsrc, A.charge, A.dipstr, A.dipvec, A.ifcharge, A.ifdipole, ENT);
        __syncthreads();
        if (valid)
          for (int k = 0; k < n; k++)
            lap3d_pair<GRAD>(x, S.y[k], S.q[k], S.ds[k], S.v[k], A.ifcharge, A.ifdipole, pot, g);
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
__global__ void __launch_bounds__(ENT) k_direct3d(Inputs3D in, int chunk, zdc* pot, zdc* grad,
                                                  zdc* part) {
  __shared__ SrcTile S;
  int i = blockIdx.x * ENT + threadIdx.x;
  int j0 = blockIdx.y * chunk, j1 = min(in.ns, j0 + chunk);
  bool valid = i < in.nt;
  zdc x[3] = {mkz(0.0), mkz(0.0), mkz(0.0)};
  if (valid) {
    x[0] = ldz(&in.ztarg[3 * i]);
    x[1] = ldz(&in.ztarg[3 * i + 1]);
    x[2] = ldz(&in.ztarg[3 * i + 2]);
  }
  zdc p = mkz(0.0), g[3] = {mkz(0.0), mkz(0.0), mkz(0.0)};
  for (int t = j0; t < j1; t += PTILE) {
    int n = min(PTILE, j1 - t);
    __syncthreads();
    stage_sources(S, t, n, in.zsrc, in.charge, in.dipstr, in.dipvec, in.ifcharge, in.ifdipole, ENT);
    __syncthreads();
    if (valid)
      for (int k = 0; k < n; k++)
        lap3d_pair<GRAD>(x, S.y[k], S.q[k], S.ds[k], S.v[k], in.ifcharge, in.ifdipole, p, g);
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
__global__ void k_direct3d_reduce(int nt, int nsplit, const zdc* part, zdc* pot, zdc* grad) {
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

// ---- interaction counts ---------------------------------------------------------
// per box: the interactions the drivers run, in totals cnt[0..7] and per
// level cnt[16 + k*64 + level] (target level for P2P/M2T/L2T/M2L/P2L, parent
// level for M2M, child level for L2L, leaf level for P2M); lmin: the coarsest
// level at which P2M runs, M2M parents sit, and L2L children sit
__global__ void k_count3(int nb, const int* ilevel, const int* iparent, const int* nchild,
                         const int* ichild, const int* isrcse, const int* itargse, const int* nl1,
                         const int* l1, int m1, const int* nl2, const int* l2, int m2,
                         const int* nl3, const int* l3, int m3, const int* nl4, const int* l4,
                         int m4, int p2m_lmin, int m2m_lmin, int l2l_lmin,
                         unsigned long long* cnt) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  auto ns_ = [&](int x) { return isrcse[2 * x + 1] - isrcse[2 * x] + 1; };
  auto nt_ = [&](int x) { return itargse[2 * x + 1] - itargse[2 * x] + 1; };
  unsigned long long c[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int ntb = nt_(b), nsb = ns_(b), lb = ilevel[b];
  if (nchild[b] == 0 && ntb > 0) {
    for (int i = 0; i < nl1[b]; i++) c[0] += (unsigned long long)ntb * max(0, ns_(l1[(size_t)b * m1 + i]));
    for (int i = 0; i < nl3[b]; i++)
      if (ns_(l3[(size_t)b * m3 + i]) > 0) c[1] += ntb;
    if (lb >= 2) c[2] = ntb;
  }
  if (ntb > 0) {
    for (int i = 0; i < nl2[b]; i++)
      if (ns_(l2[(size_t)b * m2 + i]) > 0) c[3]++;
    for (int i = 0; i < nl4[b]; i++) c[4] += max(0, ns_(l4[(size_t)b * m4 + i]));
  }
  if (nchild[b] > 0 && nsb > 0 && lb >= m2m_lmin)
    for (int k = 0; k < 8; k++)
      if (ns_(ichild[8 * b + k]) > 0) c[5]++;
  if (lb >= l2l_lmin && ntb > 0) {
    int pb = iparent[b];
    if (nt_(pb) > 0 && (nl2[pb] > 0 || nl4[pb] > 0)) c[6] = 1;
  }
  if (nchild[b] == 0 && nsb > 0 && lb >= p2m_lmin) c[7] = nsb;
  for (int k = 0; k < 8; k++)
    if (c[k]) {
      atomicAdd(&cnt[k], c[k]);
      atomicAdd(&cnt[16 + k * 64 + lb], c[k]);
    }
}

// ---- host helpers ---------------------------------------------------------------
size_t trans_smem(int p) {
  size_t NC = (size_t)(p + 1) * (p + 1), NS = 2 * p + 1;
  size_t n = 2 * NC + (p + 1) * NS + 2 * NS + (2 * p + 1) + 2 * (p + 1) + NS;
  return n * sizeof(zdc);
}

template <int KIND, int KMAX>
void launch_trans_k(const TransArgs& A, int nblocks, size_t sm, cudaStream_t s) {
  ZF_CUDA(cudaFuncSetAttribute(k_trans3<KIND, KMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sm));
  klaunch(k_trans3<KIND, KMAX>, nblocks, TNT, sm, s, A);
}

template <int KIND>
void launch_trans(const TransArgs& A, cudaStream_t s) {
  int nblocks = A.hi - A.lo + 1;
  if (nblocks <= 0) return;
  size_t sm = trans_smem(A.T.p);
  int kneed = div_up(A.T.NC, TNT);
  if (kneed <= 4) launch_trans_k<KIND, 4>(A, nblocks, sm, s);
  else if (kneed <= 8) launch_trans_k<KIND, 8>(A, nblocks, sm, s);
  else if (kneed <= 12) launch_trans_k<KIND, 12>(A, nblocks, sm, s);
  else launch_trans_k<KIND, 16>(A, nblocks, sm, s);
  ZF_LAUNCH_CHECK();
}

int choose_split3(int nt, int ns) {
  int tblocks = div_up(nt, ENT);
  int want = 4 * 148;
  int ns_max = std::max(1, div_up(ns, 4 * PTILE));
  int nsplit = std::max(1, std::min(ns_max, div_up(want, tblocks)));
  return std::min(nsplit, 64);
}

}  // namespace

int zl3dterms(double eps) {
  // zlfmm3d.f:1283-1321
  double z1 = 1.5, z2 = sqrt(3.0) / 2.0, jfun = z2, hfun = 1.0 / (z1 * z1);
  for (int j = 2; j <= 1000; j++) {
    hfun = hfun / z1;
    jfun = jfun * z2;
    if (jfun * hfun < eps) return j;
  }
  return 1;
}

int lndiv3d(double eps, int ns, int nt) {
  // lndiv_fast.f:17-35 (idivflag = 0)
  if (eps >= 0.5e-3) return 300;
  if (eps >= 0.5e-15) return 1000;
  return ns + nt;
}

void zl3ddirect_device(const Inputs3D& in, zdc* pot, zdc* grad, cudaStream_t s) {
  if (in.nt <= 0 || in.ns <= 0) return;
  int nsplit = choose_split3(in.nt, in.ns);
  int chunk = div_up(in.ns, nsplit);
  nsplit = div_up(in.ns, chunk);
  bool G = in.ifpgh > 1;
  DevBuf<zdc> part;
  if (nsplit > 1) part.alloc((size_t)nsplit * in.nt * (G ? 4 : 1), s);
  dim3 grid(div_up(in.nt, ENT), nsplit);
  if (G) {
    klaunch(k_direct3d<true>, grid, ENT, 0, s, in, chunk, pot, grad, part.get());
    if (nsplit > 1)
      klaunch(k_direct3d_reduce<true>, div_up(in.nt, 256), 256, 0, s, in.nt, nsplit, part.get(), pot, grad);
  } else {
    klaunch(k_direct3d<false>, grid, ENT, 0, s, in, chunk, pot, grad, part.get());
    if (nsplit > 1)
      klaunch(k_direct3d_reduce<false>, div_up(in.nt, 256), 256, 0, s, in.nt, nsplit, part.get(), pot, grad);
  }
  ZF_LAUNCH_CHECK();
}

// P2M through L2T/M2T/P2P on a set-up: adds the sorted potentials (and
// gradients, unscaled) of one right-hand side with sorted, rescaled strengths
// q, ds, dv to potsort / gradsort; ev[2..5] (optional) get the step boundaries;
// returns the expansion order
int lap_core(const Setup3D& S, double eps, const zdc* q, const zdc* ds, const zdc* dv,
             int ifcharge, int ifdipole, int ifpgh, zdc* potsort, zdc* gradsort, cudaStream_t s,
             cudaEvent_t* ev) {
  auto lmark = [&](int i) {
    if (ev) ZF_CUDA(cudaEventRecord(ev[i], s));
  };
  const DevTree& t = S.tree;
  const DevLists& L = S.lists;
  int nb = t.nboxes, nlev = t.nlevels;
  int p = zl3dterms(eps);
  if (trans_smem(p) > 227 * 1024)
    throw zf_error(ZF_ERR_ARG, "expansion order " + std::to_string(p) +
                                   " too large for the 3D translation kernel (eps too small)");
  Tab3 T = get_tab3(p);
  const size_t NC = (size_t)T.NC;
  std::vector<double> rsc_h(nlev + 2, 1.0);
  for (int l = 0; l <= nlev; l++) rsc_h[l] = S.bsz[l] > 1.0 ? 1.0 : S.bsz[l];
  DevBuf<double> rsc(rsc_h.size(), s);
  ZF_CUDA(cudaMemcpyAsync(rsc.get(), rsc_h.data(), rsc_h.size() * sizeof(double),
                          cudaMemcpyHostToDevice, s));
  DevBuf<zdc> mp(NC * nb, s), loc(NC * nb, s);
  mp.zero();
  loc.zero();
  // P2M
  FormArgs F;
  F.T = T;
  F.ilevel = t.ilevel.get(); F.nchild = t.nchild.get();
  F.isrcse = S.isrcse.get(); F.itargse = S.itargse.get();
  F.zsrc = S.zsrcsort.get(); F.charge = q; F.dipstr = ds;
  F.dipvec = dv; F.zcs = S.zcsrc.get(); F.zct = S.zctarg.get();
  F.rsc = rsc.get(); F.nl4 = L.n[3].get(); F.l4 = L.list[3].get(); F.mn4 = L.mn[3];
  F.nb = nb; F.ifcharge = ifcharge; F.ifdipole = ifdipole;
  size_t smf = (FNT / 32) * NC * sizeof(zdc);
  F.out = mp.get();
  if (nlev >= 1) {
    if (ifdipole) {
      ZF_CUDA(cudaFuncSetAttribute(k_form3<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smf));
      klaunch(k_form3<false, true>, nb, FNT, smf, s, F);
    } else {
      ZF_CUDA(cudaFuncSetAttribute(k_form3<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smf));
      klaunch(k_form3<false, false>, nb, FNT, smf, s, F);
    }
    ZF_LAUNCH_CHECK();
  }
  lmark(2);
  TransArgs A;
  A.T = T;
  A.ilevel = t.ilevel.get(); A.iparent = t.iparent.get(); A.nchild = t.nchild.get();
  A.ichild = t.ichild.get(); A.isrcse = S.isrcse.get(); A.itargse = S.itargse.get();
  A.zcs = S.zcsrc.get(); A.zct = S.zctarg.get(); A.rsc = rsc.get();
  A.nl2 = L.n[1].get(); A.l2 = L.list[1].get(); A.nl4 = L.n[3].get(); A.mn2 = L.mn[1];
  // M2M, finest parents first
  A.in = mp.get();
  A.out = mp.get();
  for (int l = nlev - 1; l >= 1; l--) {
    A.lo = t.laddr[2 * l];
    A.hi = t.laddr[2 * l + 1];
    launch_trans<0>(A, s);
  }
  lmark(3);
  // M2L, then P2L (list 4)
  A.in = mp.get();
  A.out = loc.get();
  A.lo = 0;
  A.hi = nb - 1;
  launch_trans<1>(A, s);
  if (L.mn[3] > 0) {
    F.out = loc.get();
    if (ifdipole) {
      ZF_CUDA(cudaFuncSetAttribute(k_form3<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smf));
      klaunch(k_form3<true, true>, nb, FNT, smf, s, F);
    } else {
      ZF_CUDA(cudaFuncSetAttribute(k_form3<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smf));
      klaunch(k_form3<true, false>, nb, FNT, smf, s, F);
    }
    ZF_LAUNCH_CHECK();
  }
  lmark(4);
  // L2L, coarsest first: children at level l+1 of parents at level l >= 1
  A.in = loc.get();
  A.out = loc.get();
  for (int l = 1; l <= nlev - 1; l++) {
    A.lo = t.laddr[2 * (l + 1)];
    A.hi = t.laddr[2 * (l + 1) + 1];
    launch_trans<2>(A, s);
  }
  lmark(5);
  // P2P (list 1), then L2T and M2T (list 3)
  P2PArgs Pa;
  Pa.nchild = t.nchild.get(); Pa.isrcse = S.isrcse.get(); Pa.itargse = S.itargse.get();
  Pa.zsrc = S.zsrcsort.get(); Pa.charge = q; Pa.dipstr = ds;
  Pa.dipvec = dv; Pa.ztarg = S.ztargsort.get();
  Pa.nl1 = L.n[0].get(); Pa.l1 = L.list[0].get(); Pa.mn1 = L.mn[0]; Pa.nb = nb;
  Pa.ifcharge = ifcharge; Pa.ifdipole = ifdipole; Pa.pot = potsort; Pa.grad = gradsort;
  if (ifpgh > 1) klaunch(k_p2p3<true>, nb, ENT, 0, s, Pa);
  else klaunch(k_p2p3<false>, nb, ENT, 0, s, Pa);
  ZF_LAUNCH_CHECK();
  EvalArgs E;
  E.T = T;
  E.ilevel = t.ilevel.get(); E.nchild = t.nchild.get(); E.isrcse = S.isrcse.get();
  E.itargse = S.itargse.get(); E.ztarg = S.ztargsort.get(); E.zcs = S.zcsrc.get();
  E.zct = S.zctarg.get(); E.rsc = rsc.get(); E.mp = mp.get(); E.loc = loc.get();
  E.nl3 = L.n[2].get(); E.l3 = L.list[2].get(); E.mn3 = L.mn[2]; E.nb = nb;
  E.pot = potsort; E.grad = gradsort;
  size_t sme = NC * sizeof(zdc);
  if (ifpgh > 1) {
    ZF_CUDA(cudaFuncSetAttribute(k_eval3<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sme));
    klaunch(k_eval3<true>, nb, ENT, sme, s, E);
  } else {
    ZF_CUDA(cudaFuncSetAttribute(k_eval3<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sme));
    klaunch(k_eval3<false>, nb, ENT, sme, s, E);
  }
  ZF_LAUNCH_CHECK();
  return p;
}

void zlfmm3d_device(double eps, const Inputs3D& in, int isep, zdc* pot, zdc* grad,
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
  tp.idivflag = 0;
  tp.ndiv = lndiv3d(eps, ns, nt);
  tp.lr_isep_quirk = 1;
  Setup3D S;
  setup3d(in, tp, S, true, true, s);
  mark(1);
  DevBuf<zdc> potsort(nt, s), gradsort(in.ifpgh > 1 ? 3 * (size_t)nt : 1, s);
  potsort.zero();
  gradsort.zero();
  int p = lap_core(S, eps, S.chargesort.get(), S.dipstrsort.get(), S.dipvecsort.get(),
                   in.ifcharge, in.ifdipole, in.ifpgh, potsort.get(), gradsort.get(), s,
                   timing ? ev : nullptr);
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
    times->nterms = p;
    for (auto& e : ev) cudaEventDestroy(e);
    times->launches = launch_counter() - launches0;
    if (times->want_counts) {
      std::vector<int> pl(S.tree.nlevels + 1, p);
      count_interactions3d(S, pl.data(), 1, 1, 2, times, s);
    }
  }
}

void count_interactions3d(const Setup3D& S, const int* p_per_level, int p2m_lmin, int m2m_lmin,
                          int l2l_lmin, StepTimes* times, cudaStream_t s) {
  const DevTree& t = S.tree;
  const DevLists& L = S.lists;
  int nb = t.nboxes;
  DevBuf<unsigned long long> cnt(16 + 8 * 64, s);
  cnt.zero();
  klaunch(k_count3, div_up(nb, 256), 256, 0, s, nb, t.ilevel.get(), t.iparent.get(),
          t.nchild.get(), t.ichild.get(), S.isrcse.get(), S.itargse.get(), L.n[0].get(),
          L.list[0].get(), L.mn[0], L.n[1].get(), L.list[1].get(), L.mn[1], L.n[2].get(),
          L.list[2].get(), L.mn[2], L.n[3].get(), L.list[3].get(), L.mn[3], p2m_lmin, m2m_lmin,
          l2l_lmin, cnt.get());
  std::vector<unsigned long long> h(16 + 8 * 64);
  ZF_CUDA(cudaMemcpyAsync(h.data(), cnt.get(), h.size() * sizeof(unsigned long long),
                          cudaMemcpyDeviceToHost, s));
  ZF_CUDA(cudaStreamSynchronize(s));
  for (int i = 0; i < 16; i++) times->counts[i] = h[i];
  for (int k = 0; k < 8; k++)
    for (int l = 0; l < 64; l++) times->lvl_counts[k][l] = h[16 + k * 64 + l];
  for (int l = 0; l < 64; l++) times->lvl_p[l] = l <= t.nlevels ? p_per_level[l] : 0;
}

}  // namespace zf
