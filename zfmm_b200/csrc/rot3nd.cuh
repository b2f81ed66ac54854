// The batched point-and-shoot y-rotation shared by the batched 3D FMM
// translations (see lfmm3d_nd.cu): degree-streamed (angle, order) recurrence
// states, sample and projection products on FP64 tensor cores, z-rotation on
// load and on store.  Included by the batched Laplace and Helmholtz kernels.
#pragma once
#include <cmath>
#include <map>
#include <mutex>
#include <vector>
#include "sph3d.cuh"

namespace zf {
namespace {

constexpr int XNT = 384;      // threads of the batched translation kernel
constexpr int XW = XNT / 32;  // its warps
constexpr int RC = 32;        // right-hand sides per translation pass (one per lane)
constexpr int JT = 7;         // sample product: angles per warp task
constexpr int MT = 6;         // projection: orders per warp task
constexpr int JB = 8;         // shift: output degrees per warp task
constexpr int LR = 2;         // input rows per warp prefetched into registers

// padded dimensions of the planar shared-memory operands of the rotation
// products (rows of 8 / 4 for the m8n8k4 tiles; strides that spread a
// fragment load over the banks)
__host__ __device__ inline int rot_cp(int L) { return (L + 7) / 8 * 8; }  // angles / orders, padded
__host__ __device__ inline int rot_kr(int L) { return (L + 3) / 4 * 4; }  // product depth, padded
constexpr int RP = RC + 4;                                                // right-hand-side stride
__host__ __device__ inline int rot_tp(int L) { return rot_cp(L) + 4; }    // table row stride

// DFT halves of the projection, [m][jc] with row stride rot_tp(L), rows and
// columns padded with zeros to rot_cp(L): CW(m, jc) = cos(2 pi (jc m mod NS) /
// NS) with CW(m, 0) = 1/2, SW(m, jc) = sin(...) with SW(m, 0) = 0, NS = 2p+1
struct RotTab {
  const double* cw;
  const double* sw;
};

std::mutex g_rot_mu;
std::map<std::pair<int, int>, RotTab> g_rot;

RotTab get_rottab(int p) {
  int dev = 0;
  ZF_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_rot_mu);
  auto key = std::make_pair(dev, p);
  auto it = g_rot.find(key);
  if (it != g_rot.end()) return it->second;
  const int L = p + 1, NS = 2 * p + 1, CP = rot_cp(L), TP = rot_tp(L);
  const size_t one = (size_t)CP * TP;
  std::vector<double> h(2 * one, 0.0);
  for (int m = 0; m <= p; m++)
    for (int jc = 0; jc <= p; jc++) {
      int k = (jc * m) % NS;
      double a = 2 * kPi * k / NS;
      h[(size_t)m * TP + jc] = jc == 0 ? 0.5 : cos(a);
      h[one + (size_t)m * TP + jc] = jc == 0 ? 0.0 : sin(a);
    }
  double* d = nullptr;
  ZF_CUDA(cudaMalloc((void**)&d, h.size() * sizeof(double)));
  ZF_CUDA(cudaMemcpy(d, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
  RotTab R{d, d + one};
  g_rot[key] = R;
  return R;
}

// one m8n8k4 FP64 tensor-core product, c += a b (fragments of the PTX layout:
// a = A[lane/4][lane%4], b = B[lane%4][lane/4], c = C[lane/4][2(lane%4)+{0,1}])
__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

// per-angle constants of one y-rotation (the set-up of myzylgndr2sf in z3dyrot)
struct JCc {
  zdc z, zz1, u, z1, z2, z3, st, eip;
  zdc yd[2], emr[2];  // Ydiag(m) and eip^m of the states starting at degree m, by parity
};

// global-memory streams of the translations (inputs, scratch, outputs) go
// through L2 only, keeping L1 for the recurrence tables
__device__ __forceinline__ zdc ldcg_z(const zdc* p) {
  double2 v = __ldcg(reinterpret_cast<const double2*>(p));
  return mkz(v.x, v.y);
}
__device__ __forceinline__ void stcg_z(zdc* p, zdc v) {
  __stcg(reinterpret_cast<double2*>(p), make_double2(v.re, v.im));
}

struct XSm {
  JCc* jc;
  // planar operands of the rotation products: sample coefficients [m][jc]
  // (stride CP), inputs [m][r] (stride RP), samples [jc][r] (stride RP)
  double *Csr, *Csi, *Cdr, *Cdi, *Asr, *Asi, *Adr, *Adi, *Ssr, *Ssi, *Sdr, *Sdi;
  double *cw, *sw;  // DFT tables staged in shared memory (null: read them from global)
  zdc *Ef, *Eb, *G, *T1, *T2;
  zdc *Ypp, *Dpp;  // recurrence values of degree n-2 per (angle, order) state
  char* work_end;     // end of the rotation's work block (Csr .. Dpp)
  size_t work_bytes;  // its size
};

// layout of the translation kernel's shared memory; returns its size in bytes
// (with_tab: the DFT tables staged too)
__host__ __device__ inline size_t xsm_layout(int p, bool with_tab, void* base, XSm* out) {
  const size_t L = p + 1, NS = 2 * p + 1, CP = rot_cp(p + 1), KR = rot_kr(p + 1),
               TP = rot_tp(p + 1);
  char* b = (char*)base;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    void* q = b ? b + off : nullptr;
    off += (bytes + 15) / 16 * 16;
    return q;
  };
  XSm S;
  S.jc = (JCc*)take(L * sizeof(JCc));
  S.Ef = (zdc*)take(NS * 16);
  S.Eb = (zdc*)take(NS * 16);
  S.G = (zdc*)take(NS * 16);
  S.T1 = (zdc*)take(L * 16);
  S.T2 = (zdc*)take(L * 16);
  S.cw = S.sw = nullptr;
  if (with_tab) {
    S.cw = (double*)take(CP * TP * 8);
    S.sw = (double*)take(CP * TP * 8);
  }
  // the rotation's work arrays, one contiguous block from Csr to the end of Dpp,
  // last in the layout (free between the two rotations of a translation; a
  // caller may alias a larger region from Csr on)
  S.Csr = (double*)take(KR * CP * 8);
  S.Csi = (double*)take(KR * CP * 8);
  S.Cdr = (double*)take(KR * CP * 8);
  S.Cdi = (double*)take(KR * CP * 8);
  S.Asr = (double*)take(KR * RP * 8);
  S.Asi = (double*)take(KR * RP * 8);
  S.Adr = (double*)take(KR * RP * 8);
  S.Adi = (double*)take(KR * RP * 8);
  S.Ssr = (double*)take(CP * RP * 8);
  S.Ssi = (double*)take(CP * RP * 8);
  S.Sdr = (double*)take(CP * RP * 8);
  S.Sdi = (double*)take(CP * RP * 8);
  S.Ypp = (zdc*)take(L * L * 16);
  S.Dpp = (zdc*)take(L * L * 16);
  S.work_end = b ? b + off : nullptr;
  S.work_bytes = off - (size_t)((char*)S.Csr - (char*)b);
  if (out) *out = S;
  return off;
}

// bytes of the layout ahead of the work block (Csr): its offset
__host__ __device__ inline size_t xsm_work_offset(int p, bool with_tab) {
  XSm S;
  xsm_layout(p, with_tab, (void*)(size_t)0x100, &S);
  return (size_t)((char*)S.Csr - (char*)(size_t)0x100);
}

// zero the padding columns (angles p+1 .. rot_cp(p+1)-1) of the sample
// coefficients of an order-p rotation, after the work block was reused
__device__ inline void rot_zero_pad(const XSm& S, int p) {
  const int L = p + 1, CP = rot_cp(L), KR = rot_kr(L), W = CP - L;
  for (int k = threadIdx.x; k < KR * W; k += XNT) {
    const int i = (k / W) * CP + L + k % W;
    S.Csr[i] = 0.0;
    S.Csi[i] = 0.0;
    S.Cdr[i] = 0.0;
    S.Cdi[i] = 0.0;
  }
}

// amat-based factor applied after the first rotation (the prescale of the
// axial shift, zl3dtrans.f)
template <int KIND>
__device__ __forceinline__ zdc prescale(const Tab3& T, const XSm& S, int n, int m, zdc v) {
  if (KIND == 3) return v;  // Helmholtz: the quadrature shift takes the rotated expansion as is
  const int nmax = T.nmax, ldA = 2 * nmax + 1;
  double an = __ldg(&T.amat[n * ldA + m + nmax]);
  if (KIND == 0) return v * an;
  if (KIND == 1) return v * (((n + m) & 1) ? -an : an);
  return v * S.T2[n] / an;
}

// One y-rotation by the angle (ca, sa) of the 32 right-hand sides of an
// expansion of order p.  MODE 0: input from a box expansion in global memory
// (row stride ldin, z-rotated by Ef on load), output written to the scratch
// (row stride RC) with the shift prescale.  MODE 1: input from the scratch,
// output added to a box expansion (row stride ldout) with the inverse
// z-rotation Eb.  nval: right-hand sides of this pass that exist.
template <int SLOTS, int MODE, int KIND>
__device__ void rot_nd(const Tab3& T, int p, int LT, double dsc, const RotTab& R, const XSm& S,
                       zdc ca, zdc sa, bool zr, const zdc* gin, long ldin, zdc* gout, long ldout,
                       int nval) {
  // p: order of the rotated expansion; LT: row stride of the recurrence and
  // projection tables (order >= p); dsc rescales the projection weights to p
  const int L = p + 1, tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int CP = rot_cp(L), TP = rot_tp(L);
  const int g8 = lane >> 2, t4 = lane & 3;  // fragment row / column of the m8n8k4 layout
  const double s4i = 1.0 / sqrt(4 * kPi);
  __syncthreads();
  if (tid < L) {
    const int j = tid;
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
    JCc c;
    c.z1 = s4i * st;
    c.z2 = (st * ca - ct * cp * sa) * s4i;
    c.z3 = zmul_i(sp * sa * s4i);
    c.z = ct;
    c.zz1 = mkz(1.0) - ct * ct;
    c.u = (zabs(c.zz1) >= (double)1e-12f) ? -zsqrt_r(c.zz1) : -st;
    c.st = st;
    c.eip = eip;
    c.yd[0] = mkz(1.0);
    c.emr[0] = mkz(1.0);
    c.yd[1] = mkz(p >= 1 ? -__ldg(&T.r1[LT + 1]) : 0.0);
    c.emr[1] = eip;
    S.jc[j] = c;
  }
  zdc Yp[SLOTS], Dp[SLOTS], em[SLOTS];
#pragma unroll
  for (int s = 0; s < SLOTS; s++) Yp[s] = Dp[s] = em[s] = mkz(0.0);
  __syncthreads();

  // sample coefficients of degree n: Cs = C(j,m) + C(j,-m), Cd = C(j,m) - C(j,-m)
  auto gen = [&](int n) {
#pragma unroll
    for (int s = 0; s < SLOTS; s++) {
      int idx = tid + s * XNT;
      if (idx >= L * L) continue;
      int m = idx / L, jc = idx - m * L;
      if (m > n) continue;
      const JCc& J = S.jc[jc];
      zdc z = J.z;
      zdc Y, D;
      if (n == m) {
        if (m == 0) {
          Y = mkz(1.0);
          D = mkz(0.0);
        } else {
          Y = J.yd[m & 1];
          D = (Y * (double)(-m)) * z;
          em[s] = J.emr[m & 1];
        }
      } else if (n == m + 1) {
        double c = __ldg(&T.r1[n * LT + m]);
        Y = (z * Yp[s]) * c;
        D = (m == 0) ? (z * Dp[s] + Yp[s]) * c : (z * Dp[s] + J.zz1 * Yp[s]) * c;
      } else {
        double c1 = __ldg(&T.r1[n * LT + m]), c2 = __ldg(&T.r2[n * LT + m]);
        zdc ypp = S.Ypp[idx], dpp = S.Dpp[idx];
        Y = (c1 * z) * Yp[s] - c2 * ypp;
        D = (m == 0) ? c1 * (z * Dp[s] + Yp[s]) - c2 * dpp
                     : c1 * (z * Dp[s] + J.zz1 * Yp[s]) - c2 * dpp;
      }
      if (n > m) {
        S.Ypp[idx] = Yp[s];
        S.Dpp[idx] = Dp[s];
      }
      Yp[s] = Y;
      Dp[s] = D;
      double sqn = __ldg(&T.sq[n]);
      zdc y = Y * sqn, d = D * sqn;
      zdc cs, cd;
      if (m == 0) {
        cs = (y * s4i - (d * J.z2) * J.st) * 2.0;
        cd = mkz(0.0);
      } else {
        double sg = (m & 1) ? -1.0 : 1.0;
        zdc P = sg * (J.z1 * y - J.z2 * d);
        zdc Q = (sg * m) * (y * J.z3);
        zdc Cp = (P + Q) * em[s], Cm = (P - Q) * zinv(em[s]);
        cs = Cp + Cm;
        cd = Cp - Cm;
      }
      S.Csr[m * CP + jc] = cs.re;
      S.Csi[m * CP + jc] = cs.im;
      S.Cdr[m * CP + jc] = cd.re;
      S.Cdi[m * CP + jc] = cd.im;
    }
    // Ydiag and eip^m of the states that start at degree n+1 (the sequential
    // products of myzylgndr2sf), one thread per angle
    if (tid < L && n >= 1 && n + 1 <= p) {
      JCc& J = S.jc[tid];
      J.yd[(n + 1) & 1] = (J.yd[n & 1] * J.u) * __ldg(&T.r1[(n + 1) * LT + n + 1]);
      J.emr[(n + 1) & 1] = J.emr[n & 1] * J.eip;
    }
  };
  // inputs of degree n: As = a(n,m) + a(n,-m), Ad = a(n,m) - a(n,-m).  The
  // first LR rows of each warp are fetched into registers before the
  // coefficient generation (hiding the global-memory latency behind it) and
  // committed to shared memory after it; rows beyond (orders p >= LR*XW) load
  // synchronously.
  zdc fa[LR], fb[LR];
  auto fetch_row = [&](int n, int m, zdc& a, zdc& b) {
    a = mkz(0.0);
    b = mkz(0.0);
    if (MODE == 0) {
      if (lane < nval) {
        a = ldcg_z(gin + (long)ix3(n, m) * ldin + lane);
        if (m > 0) b = ldcg_z(gin + (long)ix3(n, -m) * ldin + lane);
      }
    } else {
      a = ldcg_z(gin + ix3(n, m) * RC + lane);
      if (m > 0) b = ldcg_z(gin + ix3(n, -m) * RC + lane);
    }
  };
  auto put_row = [&](int m, zdc a, zdc b) {
    if (MODE == 0 && zr) {
      a = a * S.Ef[p + m];
      b = b * S.Ef[p - m];
    }
    zdc s_ = m == 0 ? a : a + b, d_ = m == 0 ? mkz(0.0) : a - b;
    S.Asr[m * RP + lane] = s_.re;
    S.Asi[m * RP + lane] = s_.im;
    S.Adr[m * RP + lane] = d_.re;
    S.Adi[m * RP + lane] = d_.im;
  };
  auto fetch = [&](int n) {
#pragma unroll
    for (int i = 0; i < LR; i++) {
      int m = w + i * XW;
      if (m <= n) fetch_row(n, m, fa[i], fb[i]);
    }
  };
  auto commit = [&](int n) {
#pragma unroll
    for (int i = 0; i < LR; i++) {
      int m = w + i * XW;
      if (m <= n) put_row(m, fa[i], fb[i]);
    }
    for (int m = w + LR * XW; m <= n; m += XW) {
      zdc a, b;
      fetch_row(n, m, a, b);
      put_row(m, a, b);
    }
  };
  auto store = [&](int n, int m, int r, zdc v) {
    if (MODE == 0) {
      stcg_z(gout + ix3(n, m) * RC + r, prescale<KIND>(T, S, n, m, v));
    } else if (r < nval) {
      zdc* o = gout + (long)ix3(n, m) * ldout + r;
      stcg_z(o, ldcg_z(o) + (zr ? v * S.Eb[p + m] : v));
    }
  };
  const double* cwt = S.cw ? S.cw : R.cw;
  const double* swt = S.sw ? S.sw : R.sw;

  fetch(0);
  gen(0);
  commit(0);
  __syncthreads();
  const int njt = CP / 8;
  for (int n = 0; n <= p; n++) {
    // samples at angles >= 0: S = F(j) + F(-j), D = F(j) - F(-j); complex
    // [jc x m] x [m x r] products on m8n8k4 tiles (4 real MMAs per k-step)
    for (int t = w; t < 4 * njt; t += XW) {
      const int which = t / (2 * njt), rem = t - which * 2 * njt, jt = rem >> 1, rh = rem & 1;
      const double* Cr = which ? S.Cdr : S.Csr;
      const double* Ci = which ? S.Cdi : S.Csi;
      const double* Ar = which ? S.Adr : S.Asr;
      const double* Ai = which ? S.Adi : S.Asi;
      double sr[2][2], si[2][2];
#pragma unroll
      for (int q = 0; q < 2; q++) sr[q][0] = sr[q][1] = si[q][0] = si[q][1] = 0.0;
      const int jc = jt * 8 + g8;
      for (int k0 = 0; k0 <= n; k0 += 4) {
        const int m = k0 + t4;
        const bool ok = m <= n;
        const double are = ok ? Cr[m * CP + jc] : 0.0, aim = ok ? Ci[m * CP + jc] : 0.0;
#pragma unroll
        for (int q = 0; q < 2; q++) {
          const int r = (2 * rh + q) * 8 + g8;
          const double bre = ok ? Ar[m * RP + r] : 0.0, bim = ok ? Ai[m * RP + r] : 0.0;
          dmma(sr[q], are, bre);
          dmma(si[q], are, bim);
          dmma(sr[q], -aim, bim);
          dmma(si[q], aim, bre);
        }
      }
      double* Or = which ? S.Sdr : S.Ssr;
      double* Oi = which ? S.Sdi : S.Ssi;
#pragma unroll
      for (int q = 0; q < 2; q++) {
        const int ro = (jt * 8 + g8) * RP + (2 * rh + q) * 8 + 2 * t4;
        Or[ro] = sr[q][0];
        Or[ro + 1] = sr[q][1];
        Oi[ro] = si[q][0];
        Oi[ro + 1] = si[q][1];
      }
    }
    __syncthreads();
    // projection: X = CW (S + [jc = 0] D), Y = SW D on m8n8k4 tiles, then
    // out(n, +-m) = dinv(n, m) (X -+ i Y)
    const int nmt = (n + 8) / 8;
    for (int t = w; t < nmt * 4; t += XW) {
      const int mt = t >> 2, rt = t & 3;
      double xr[2] = {0.0, 0.0}, xi[2] = {0.0, 0.0}, yr[2] = {0.0, 0.0}, yi[2] = {0.0, 0.0};
      const int mrow = mt * 8 + g8, r = rt * 8 + g8;
      for (int k0 = 0; k0 < CP; k0 += 4) {
        const int jc = k0 + t4;
        const double ac = cwt[mrow * TP + jc], as = swt[mrow * TP + jc];
        double bsr = S.Ssr[jc * RP + r], bsi = S.Ssi[jc * RP + r];
        const double bdr = S.Sdr[jc * RP + r], bdi = S.Sdi[jc * RP + r];
        if (jc == 0) {
          bsr += bdr;
          bsi += bdi;
        }
        dmma(xr, ac, bsr);
        dmma(xi, ac, bsi);
        dmma(yr, as, bdr);
        dmma(yi, as, bdi);
      }
      const int m = mt * 8 + g8;
      if (m <= n) {
        const double dn = __ldg(&T.dinv[n * LT + m]) * dsc;
#pragma unroll
        for (int i = 0; i < 2; i++) {
          const int ro = rt * 8 + 2 * t4 + i;
          const zdc X = mkz(xr[i], xi[i]), iy = zmul_i(mkz(yr[i], yi[i]));
          store(n, m, ro, (X - iy) * dn);
          if (m > 0) store(n, -m, ro, (X + iy) * dn);
        }
      }
    }
    if (n < p) {
      fetch(n + 1);
      gen(n + 1);
      commit(n + 1);
    }
    __syncthreads();
  }
}

// the y-rotation skipped (translation along z): z-rotation and prescale only
template <int MODE, int KIND>
__device__ void copy_nd(const Tab3& T, int p, const XSm& S, bool zr, const zdc* gin, long ldin,
                        zdc* gout, long ldout, int nval) {
  const int NC = (p + 1) * (p + 1), lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  for (int idx = w; idx < NC; idx += XW) {
    int n = deg3(idx), m = idx - n * n - n;
    if (MODE == 0) {
      zdc a = mkz(0.0);
      if (lane < nval) {
        a = ldcg_z(gin + (long)idx * ldin + lane);
        if (zr) a = a * S.Ef[p + m];
      }
      stcg_z(gout + idx * RC + lane, prescale<KIND>(T, S, n, m, a));
    } else if (lane < nval) {
      zdc v = ldcg_z(gin + idx * RC + lane);
      zdc* o = gout + (long)idx * ldout + lane;
      stcg_z(o, ldcg_z(o) + (zr ? v * S.Eb[p + m] : v));
    }
  }
  __syncthreads();
}

}  // namespace
}  // namespace zf
