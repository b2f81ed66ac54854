// 2D driver set-up on the device (see fmm2d_common.cuh).
#include "fmm2d_common.cuh"

namespace zf {
namespace {

constexpr int TB = 256;

__global__ void k_real_parts(const zdc* __restrict__ z, long n2, double* __restrict__ r) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n2) r[i] = z[i].re;
}

// gather sources/strengths (zreorderf, toolbox.f:2-21)
__global__ void k_gather_src(int ns, const int* __restrict__ perm, const zdc* __restrict__ zsrc,
                             const zdc* __restrict__ q, const zdc* __restrict__ ds,
                             const zdc* __restrict__ dv, zdc* zs, zdc* qs, zdc* dss, zdc* dvs) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ns) return;
  int j = perm[i];
  zs[2 * i] = zsrc[2 * j];
  zs[2 * i + 1] = zsrc[2 * j + 1];
  qs[i] = q ? q[j] : mkz(0.0);
  dss[i] = ds ? ds[j] : mkz(0.0);
  dvs[2 * i] = dv ? dv[2 * j] : mkz(0.0);
  dvs[2 * i + 1] = dv ? dv[2 * j + 1] : mkz(0.0);
}

__global__ void k_gather_targ(int nt, const int* __restrict__ perm, const zdc* __restrict__ zt,
                              zdc* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nt) return;
  int j = perm[i];
  out[2 * i] = zt[2 * j];
  out[2 * i + 1] = zt[2 * j + 1];
}

// sums of imaginary parts over each leaf's range: one warp per leaf
__global__ void k_leaf_imag_sum(int nb, const int* __restrict__ nchild,
                                const int* __restrict__ se, const zdc* __restrict__ pts,
                                double* __restrict__ sums) {
  int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= nb || nchild[w] > 0) return;
  int s0 = se[2 * w], s1 = se[2 * w + 1];
  double a = 0, b = 0;
  for (int i = s0 + lane; i <= s1; i += 32) {
    a += pts[2 * i].im;
    b += pts[2 * i + 1].im;
  }
  for (int o = 16; o; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if (lane == 0) { sums[2 * w] = a; sums[2 * w + 1] = b; }
}

__global__ void k_parent_imag_sum(int lo, int hi, const int* nchild, const int* ichild,
                                  double* sums) {
  int b = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (b > hi || nchild[b] == 0) return;
  double a = 0, c = 0;
  for (int k = 0; k < 4; k++) {
    int ch = ichild[4 * b + k];
    a += sums[2 * ch];
    c += sums[2 * ch + 1];
  }
  sums[2 * b] = a;
  sums[2 * b + 1] = c;
}

__global__ void k_centres(int nb, const double* __restrict__ centers, const int* __restrict__ se,
                          const double* __restrict__ sums, zdc* __restrict__ zc) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  int n = se[2 * b + 1] - se[2 * b] + 1;
  if (n > 0) {
    zc[2 * b] = mkz(centers[2 * b], sums[2 * b] / n);
    zc[2 * b + 1] = mkz(centers[2 * b + 1], sums[2 * b + 1] / n);
  } else {
    zc[2 * b] = mkz(0.0);
    zc[2 * b + 1] = mkz(0.0);
  }
}

void complex_centres(const DevTree& t, const DevBuf<int>& se, const DevBuf<zdc>& pts,
                     DevBuf<zdc>& zc, cudaStream_t s) {
  int nb = t.nboxes;
  DevBuf<double> sums(2 * (size_t)nb, s);
  klaunch(k_leaf_imag_sum, div_up((long)nb * 32, TB), TB, 0, s, nb, t.nchild.get(), se.get(),
                                                          pts.get(), sums.get());
  for (int l = t.nlevels - 1; l >= 0; l--) {
    int lo = t.laddr[2 * l], hi = t.laddr[2 * l + 1];
    klaunch(k_parent_imag_sum, div_up(hi - lo + 1, TB), TB, 0, s, lo, hi, t.nchild.get(),
                                                             t.ichild.get(), sums.get());
  }
  zc.alloc(2 * (size_t)nb, s);
  klaunch(k_centres, div_up(nb, TB), TB, 0, s, nb, t.centers.get(), se.get(), sums.get(), zc.get());
  ZF_LAUNCH_CHECK();
}

__global__ void k_unsort(int nt, const int* __restrict__ perm, const zdc* __restrict__ ps,
                         const zdc* __restrict__ gs, zdc scale, int ifpgh, zdc* pot, zdc* grad) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nt) return;
  int j = perm[i];
  pot[j] = ps[i] * scale;
  if (ifpgh > 1) {
    grad[2 * j] = gs[2 * i] * scale;
    grad[2 * j + 1] = gs[2 * i + 1] * scale;
  }
}

// right-hand side r of charge(nd, ns) / dipstr(nd, ns) in tree order; dipvec
// (2, ns) shared by the right-hand sides
__global__ void k_gather_col2(int ns, int nd, int r, const int* __restrict__ perm,
                              const zdc* __restrict__ q, const zdc* __restrict__ ds,
                              const zdc* __restrict__ dv, zdc* qs, zdc* dss, zdc* dvs) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ns) return;
  long j = perm[i];
  qs[i] = q ? q[j * nd + r] : mkz(0.0);
  dss[i] = ds ? ds[j * nd + r] : mkz(0.0);
  dvs[2 * i] = dv ? dv[2 * j] : mkz(0.0);
  dvs[2 * i + 1] = dv ? dv[2 * j + 1] : mkz(0.0);
}

// right-hand side r of pot(nd, nt) / grad(nd, 2, nt)
__global__ void k_unsort_col2(int nt, int nd, int r, const int* __restrict__ perm,
                              const zdc* __restrict__ ps, const zdc* __restrict__ gs, zdc scale,
                              int ifpgh, zdc* pot, zdc* grad) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nt) return;
  long j = perm[i];
  pot[j * nd + r] = ps[i] * scale;
  if (ifpgh > 1) {
    grad[(2 * j) * nd + r] = gs[2 * i] * scale;
    grad[(2 * j + 1) * nd + r] = gs[2 * i + 1] * scale;
  }
}

// one thread per box; the same conditions as the eight steps of the drivers
__global__ void k_count(int nb, const int* ilevel, const int* iparent, const int* nchild,
                        const int* ichild, const int* isrcse, const int* itargse, const int* nl1,
                        const int* l1, int m1, const int* nl2, const int* l2, int m2,
                        const int* nl3, const int* l3, int m3, const int* nl4, const int* l4,
                        int m4, const int* pl, unsigned long long* cnt) {
  // cnt[0..7]: counts; cnt[8..15]: the same interactions weighted by the
  // expansion lengths P = 2p+1 of their levels: [-, M2T sum P, L2T sum P,
  // M2L sum P^2, P2L sum P, M2M sum P_parent P_child, L2L sum P_parent P_child,
  // P2M sum P]
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  auto P_ = [&](int x) { return (unsigned long long)(2 * pl[ilevel[x]] + 1); };
  unsigned long long w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  auto ns_ = [&](int x) { return isrcse[2 * x + 1] - isrcse[2 * x] + 1; };
  auto nt_ = [&](int x) { return itargse[2 * x + 1] - itargse[2 * x] + 1; };
  unsigned long long c[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int ntb = nt_(b), nsb = ns_(b);
  if (nchild[b] == 0 && ntb > 0) {
    for (int i = 0; i < nl1[b]; i++) c[0] += (unsigned long long)ntb * max(0, ns_(l1[(size_t)b * m1 + i]));
    for (int i = 0; i < nl3[b]; i++) {
      int jb = l3[(size_t)b * m3 + i];
      if (ns_(jb) > 0) { c[1] += ntb; w[1] += ntb * P_(jb); }
    }
    if (ilevel[b] >= 2) { c[2] = ntb; w[2] = ntb * P_(b); }
  }
  if (ntb > 0) {
    for (int i = 0; i < nl2[b]; i++)
      if (ns_(l2[(size_t)b * m2 + i]) > 0) { c[3]++; w[3] += P_(b) * P_(b); }
    for (int i = 0; i < nl4[b]; i++) {
      unsigned long long k = max(0, ns_(l4[(size_t)b * m4 + i]));
      c[4] += k;
      w[4] += k * P_(b);
    }
  }
  if (nchild[b] > 0 && nsb > 0 && ilevel[b] >= 1)
    for (int k = 0; k < 4; k++) {
      int ch = ichild[4 * b + k];
      if (ns_(ch) > 0) { c[5]++; w[5] += P_(b) * P_(ch); }
    }
  if (ilevel[b] >= 2 && ntb > 0) {
    int pb = iparent[b];
    if (nt_(pb) > 0 && (nl2[pb] > 0 || nl4[pb] > 0)) { c[6] = 1; w[6] = P_(pb) * P_(b); }
  }
  if (nchild[b] == 0 && nsb > 0 && ilevel[b] >= 1) { c[7] = nsb; w[7] = nsb * P_(b); }
  for (int k = 0; k < 8; k++) {
    if (c[k]) atomicAdd(&cnt[k], c[k]);
    if (w[k]) atomicAdd(&cnt[8 + k], w[k]);
  }
}

}  // namespace

void count_interactions2d(const Setup2D& S, const int* p_per_level, unsigned long long* counts,
                          cudaStream_t s) {
  const DevTree& t = S.tree;
  const DevLists& L = S.lists;
  int nb = t.nboxes;
  DevBuf<unsigned long long> cnt(16, s);
  DevBuf<int> pl(t.nlevels + 1, s);
  ZF_CUDA(cudaMemcpyAsync(pl.get(), p_per_level, (t.nlevels + 1) * sizeof(int),
                          cudaMemcpyHostToDevice, s));
  cnt.zero();
  klaunch(k_count, div_up(nb, 256), 256, 0, s, nb, t.ilevel.get(), t.iparent.get(),
          t.nchild.get(), t.ichild.get(), S.isrcse.get(), S.itargse.get(), L.n[0].get(),
          L.list[0].get(), L.mn[0], L.n[1].get(), L.list[1].get(), L.mn[1], L.n[2].get(),
          L.list[2].get(), L.mn[2], L.n[3].get(), L.list[3].get(), L.mn[3], pl.get(), cnt.get());
  ZF_CUDA(cudaMemcpyAsync(counts, cnt.get(), 16 * sizeof(unsigned long long),
                          cudaMemcpyDeviceToHost, s));
  ZF_CUDA(cudaStreamSynchronize(s));
}

// copy of a device buffer on stream s
template <class T>
void copy_buf(DevBuf<T>& dst, const DevBuf<T>& src, cudaStream_t s) {
  dst.alloc(src.size(), s);
  if (src.size())
    ZF_CUDA(cudaMemcpyAsync(dst.get(), src.get(), src.size() * sizeof(T),
                            cudaMemcpyDeviceToDevice, s));
}

void setup2d(const Inputs2D& in, const TreeParams& tp, Setup2D& S, cudaStream_t s) {
  int ns = in.ns, nt = in.nt;
  // targets that are the sources (the same array) share the sources' tree
  // assignment and order: computed once, copied
  const bool same = in.ztarg == in.zsrc && nt == ns;
  DevBuf<double> srcR(2 * (size_t)ns, s), targR(same ? 0 : 2 * (size_t)nt, s);
  klaunch(k_real_parts, div_up(2L * ns, TB), TB, 0, s, in.zsrc, 2L * ns, srcR.get());
  if (!same) klaunch(k_real_parts, div_up(2L * nt, TB), TB, 0, s, in.ztarg, 2L * nt, targR.get());
  ZF_LAUNCH_CHECK();
  const double* tR = same ? srcR.get() : targR.get();
  build_tree(srcR.get(), ns, tR, nt, tp, S.tree, s);
  sort_points(S.tree, srcR.get(), ns, S.isrc, S.isrcse, s);
  if (same) {
    copy_buf(S.itarg, S.isrc, s);
    copy_buf(S.itargse, S.isrcse, s);
  } else {
    sort_points(S.tree, tR, nt, S.itarg, S.itargse, s);
  }
  if (in.strengths_ready) in.strengths_ready(s);
  S.zsrcsort.alloc(2 * (size_t)ns, s);
  S.chargesort.alloc(ns, s);
  S.dipstrsort.alloc(ns, s);
  S.dipvecsort.alloc(2 * (size_t)ns, s);
  S.ztargsort.alloc(2 * (size_t)nt, s);
  klaunch(k_gather_src, div_up(ns, TB), TB, 0, s, 
      ns, S.isrc.get(), in.zsrc, in.ifcharge ? in.charge : nullptr,
      in.ifdipole ? in.dipstr : nullptr, in.ifdipole ? in.dipvec : nullptr, S.zsrcsort.get(),
      S.chargesort.get(), S.dipstrsort.get(), S.dipvecsort.get());
  klaunch(k_gather_targ, div_up(nt, TB), TB, 0, s, nt, S.itarg.get(), in.ztarg, S.ztargsort.get());
  ZF_LAUNCH_CHECK();
  complex_centres(S.tree, S.isrcse, S.zsrcsort, S.zcsrc, s);
  if (same) copy_buf(S.zctarg, S.zcsrc, s);
  else complex_centres(S.tree, S.itargse, S.ztargsort, S.zctarg, s);
  build_lists(S.tree, S.lists, s);
}

void setup2d_geom(int ns, const zdc* zsrc, int nt, const zdc* ztarg, const TreeParams& tp,
                  Setup2D& S, cudaStream_t s) {
  const bool same = ztarg == zsrc && nt == ns;
  DevBuf<double> srcR(2 * (size_t)ns, s), targR(same ? 0 : 2 * (size_t)nt, s);
  klaunch(k_real_parts, div_up(2L * ns, TB), TB, 0, s, zsrc, 2L * ns, srcR.get());
  if (!same) klaunch(k_real_parts, div_up(2L * nt, TB), TB, 0, s, ztarg, 2L * nt, targR.get());
  ZF_LAUNCH_CHECK();
  const double* tR = same ? srcR.get() : targR.get();
  build_tree(srcR.get(), ns, tR, nt, tp, S.tree, s);
  sort_points(S.tree, srcR.get(), ns, S.isrc, S.isrcse, s);
  if (same) {
    copy_buf(S.itarg, S.isrc, s);
    copy_buf(S.itargse, S.isrcse, s);
  } else {
    sort_points(S.tree, tR, nt, S.itarg, S.itargse, s);
  }
  S.zsrcsort.alloc(2 * (size_t)ns, s);
  S.ztargsort.alloc(2 * (size_t)nt, s);
  klaunch(k_gather_targ, div_up(ns, TB), TB, 0, s, ns, S.isrc.get(), zsrc, S.zsrcsort.get());
  klaunch(k_gather_targ, div_up(nt, TB), TB, 0, s, nt, S.itarg.get(), ztarg, S.ztargsort.get());
  ZF_LAUNCH_CHECK();
  complex_centres(S.tree, S.isrcse, S.zsrcsort, S.zcsrc, s);
  if (same) copy_buf(S.zctarg, S.zcsrc, s);
  else complex_centres(S.tree, S.itargse, S.ztargsort, S.zctarg, s);
  build_lists(S.tree, S.lists, s);
}

void gather2d_col(const Setup2D& S, int ns, int nd, int r, const zdc* charge, const zdc* dipstr,
                  const zdc* dipvec, zdc* q, zdc* ds, zdc* dv, cudaStream_t s) {
  if (ns <= 0) return;
  klaunch(k_gather_col2, div_up(ns, TB), TB, 0, s, ns, nd, r, S.isrc.get(), charge, dipstr,
          dipvec, q, ds, dv);
  ZF_LAUNCH_CHECK();
}

void unsort2d_col(int nt, int nd, int r, const int* itarg, const zdc* potsort,
                  const zdc* gradsort, zdc scale, int ifpgh, zdc* pot, zdc* grad,
                  cudaStream_t s) {
  if (nt <= 0) return;
  klaunch(k_unsort_col2, div_up(nt, TB), TB, 0, s, nt, nd, r, itarg, potsort, gradsort, scale,
          ifpgh, pot, grad);
  ZF_LAUNCH_CHECK();
}

void unsort2d(int nt, const int* itarg, const zdc* potsort, const zdc* gradsort, zdc scale,
              int ifpgh, zdc* pot, zdc* grad, cudaStream_t s) {
  klaunch(k_unsort, div_up(nt, TB), TB, 0, s, nt, itarg, potsort, gradsort, scale, ifpgh, pot, grad);
  ZF_LAUNCH_CHECK();
}

}  // namespace zf
