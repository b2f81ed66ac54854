// 3D driver set-up on the device (see fmm3d_common.cuh).
#include "fmm3d_common.cuh"

namespace zf {
namespace {

constexpr int TB = 256;

__global__ void k_real3(const zdc* __restrict__ z, long n3, double* __restrict__ r) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n3) r[i] = z[i].re;
}

// gather (zreorderf) and rescale by b0inv (zlfmm3d.f:187-200)
__global__ void k_gather3(int ns, const int* __restrict__ perm, const zdc* __restrict__ zsrc,
                          const zdc* __restrict__ q, const zdc* __restrict__ ds,
                          const zdc* __restrict__ dv, const double* __restrict__ b0,
                          double qscale_pow, double dvscale_pow, zdc* zs, zdc* qs, zdc* dss,
                          zdc* dvs) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ns) return;
  double bi = 1.0 / b0[0];
  double qs_f = qscale_pow > 0 ? bi : 1.0;
  double dv_f = dvscale_pow > 0 ? bi * bi : 1.0;
  int j = perm[i];
#pragma unroll
  for (int d = 0; d < 3; d++) zs[3 * i + d] = zsrc[3 * j + d] * bi;
  qs[i] = q ? q[j] * qs_f : mkz(0.0);
  dss[i] = ds ? ds[j] : mkz(0.0);
#pragma unroll
  for (int d = 0; d < 3; d++) dvs[3 * i + d] = dv ? dv[3 * j + d] * dv_f : mkz(0.0);
}

__global__ void k_gather3t(int nt, const int* __restrict__ perm, const zdc* __restrict__ zt,
                           const double* __restrict__ b0, zdc* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nt) return;
  double bi = 1.0 / b0[0];
  int j = perm[i];
#pragma unroll
  for (int d = 0; d < 3; d++) out[3 * i + d] = zt[3 * j + d] * bi;
}

__global__ void k_leaf_imag3(int nb, const int* __restrict__ nchild, const int* __restrict__ se,
                             const zdc* __restrict__ pts, double* __restrict__ sums) {
  int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= nb || nchild[w] > 0) return;
  int s0 = se[2 * w], s1 = se[2 * w + 1];
  double a[3] = {0, 0, 0};
  for (int i = s0 + lane; i <= s1; i += 32)
#pragma unroll
    for (int d = 0; d < 3; d++) a[d] += pts[3 * i + d].im;
#pragma unroll
  for (int d = 0; d < 3; d++)
    for (int o = 16; o; o >>= 1) a[d] += __shfl_xor_sync(0xffffffffu, a[d], o);
  if (lane == 0)
#pragma unroll
    for (int d = 0; d < 3; d++) sums[3 * w + d] = a[d];
}

__global__ void k_parent_imag3(int lo, int hi, const int* nchild, const int* ichild,
                               double* sums) {
  int b = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (b > hi || nchild[b] == 0) return;
  double a[3] = {0, 0, 0};
  for (int k = 0; k < 8; k++) {
    int ch = ichild[8 * b + k];
#pragma unroll
    for (int d = 0; d < 3; d++) a[d] += sums[3 * ch + d];
  }
#pragma unroll
  for (int d = 0; d < 3; d++) sums[3 * b + d] = a[d];
}

// complex centre from the sums of rescaled imaginary parts; real centre rescaled
__global__ void k_centres3(int nb, const double* __restrict__ centers, const int* __restrict__ se,
                           const double* __restrict__ sums, const double* __restrict__ b0,
                           zdc* __restrict__ zc) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  double bi = 1.0 / b0[0];
  int n = se[2 * b + 1] - se[2 * b] + 1;
#pragma unroll
  for (int d = 0; d < 3; d++)
    zc[3 * b + d] = n > 0 ? mkz(centers[3 * b + d] * bi, sums[3 * b + d] / n) : mkz(0.0);
}

void centres3(const DevTree& t, const DevBuf<int>& se, const DevBuf<zdc>& pts, const double* b0,
              DevBuf<zdc>& zc, cudaStream_t s) {
  int nb = t.nboxes;
  DevBuf<double> sums(3 * (size_t)nb, s);
  klaunch(k_leaf_imag3, div_up((long)nb * 32, TB), TB, 0, s, nb, t.nchild.get(), se.get(),
          pts.get(), sums.get());
  for (int l = t.nlevels - 1; l >= 0; l--) {
    int lo = t.laddr[2 * l], hi = t.laddr[2 * l + 1];
    klaunch(k_parent_imag3, div_up(hi - lo + 1, TB), TB, 0, s, lo, hi, t.nchild.get(),
            t.ichild.get(), sums.get());
  }
  zc.alloc(3 * (size_t)nb, s);
  klaunch(k_centres3, div_up(nb, TB), TB, 0, s, nb, t.centers.get(), se.get(), sums.get(), b0,
          zc.get());
  ZF_LAUNCH_CHECK();
}

__global__ void k_unsort3(int nt, const int* __restrict__ perm, const zdc* __restrict__ ps,
                          const zdc* __restrict__ gs, zdc pscale, zdc gscale, int ifpgh, zdc* pot,
                          zdc* grad) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nt) return;
  int j = perm[i];
  pot[j] = ps[i] * pscale;
  if (ifpgh > 1)
#pragma unroll
    for (int d = 0; d < 3; d++) grad[3 * j + d] = gs[3 * i + d] * gscale;
}

__global__ void k_gather_nd(int ns, int nd, const int* __restrict__ perm,
                            const zdc* __restrict__ q, const zdc* __restrict__ ds,
                            const zdc* __restrict__ dv, const double* __restrict__ b0,
                            int rescale_q, int rescale_dv, zdc* qs, zdc* dss, zdc* dvs) {
  long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= (long)ns * nd) return;
  int i = (int)(k / nd), r = (int)(k - (long)i * nd);
  double bi = 1.0 / b0[0];
  long src = (long)perm[i] * nd + r;
  qs[k] = q ? q[src] * (rescale_q ? bi : 1.0) : mkz(0.0);
  dss[k] = ds ? ds[src] : mkz(0.0);
  if (r == 0)
#pragma unroll
    for (int d = 0; d < 3; d++)
      dvs[3 * i + d] = dv ? dv[3 * perm[i] + d] * (rescale_dv ? bi * bi : 1.0) : mkz(0.0);
}

__global__ void k_unsort_nd(int nt, int nd, const int* __restrict__ perm,
                            const zdc* __restrict__ ps, const zdc* __restrict__ gs, zdc pscale,
                            zdc gscale, int ifpgh, zdc* pot, zdc* grad) {
  long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= (long)nt * nd) return;
  int i = (int)(k / nd), r = (int)(k - (long)i * nd);
  long j = perm[i];
  pot[j * nd + r] = ps[k] * pscale;
  if (ifpgh > 1)
#pragma unroll
    for (int d = 0; d < 3; d++)
      grad[(3 * j + d) * nd + r] = gs[(3L * i + d) * nd + r] * gscale;
}

__global__ void k_gather_col(int ns, int nd, int r, const int* __restrict__ perm,
                             const zdc* __restrict__ q, const zdc* __restrict__ ds,
                             const zdc* __restrict__ dv, const double* __restrict__ b0,
                             int rescale_q, int rescale_dv, zdc* qs, zdc* dss, zdc* dvs) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ns) return;
  double bi = 1.0 / b0[0];
  long j = perm[i];
  qs[i] = q ? q[j * nd + r] * (rescale_q ? bi : 1.0) : mkz(0.0);
  dss[i] = ds ? ds[j * nd + r] : mkz(0.0);
#pragma unroll
  for (int d = 0; d < 3; d++)
    dvs[3 * i + d] = dv ? dv[3 * j + d] * (rescale_dv ? bi * bi : 1.0) : mkz(0.0);
}

__global__ void k_unsort_col(int nt, int nd, int r, const int* __restrict__ perm,
                             const zdc* __restrict__ ps, const zdc* __restrict__ gs, zdc pscale,
                             zdc gscale, int ifpgh, zdc* pot, zdc* grad) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nt) return;
  long j = perm[i];
  pot[j * nd + r] = ps[i] * pscale;
  if (ifpgh > 1)
#pragma unroll
    for (int d = 0; d < 3; d++) grad[(3 * j + d) * nd + r] = gs[3 * i + d] * gscale;
}

}  // namespace

void gather_strengths_col(const Setup3D& S, int ns, int nd, int r, const zdc* charge,
                          const zdc* dipstr, const zdc* dipvec, bool rescale_charge,
                          bool rescale_dipvec, zdc* q, zdc* ds, zdc* dv, cudaStream_t s) {
  if (ns <= 0) return;
  klaunch(k_gather_col, div_up(ns, TB), TB, 0, s, ns, nd, r, S.isrc.get(), charge, dipstr,
          dipvec, S.tree.bsz.get(), rescale_charge ? 1 : 0, rescale_dipvec ? 1 : 0, q, ds, dv);
  ZF_LAUNCH_CHECK();
}

void unsort3d_col(int nt, int nd, int r, const int* itarg, const zdc* potsort,
                  const zdc* gradsort, zdc pscale, zdc gscale, int ifpgh, zdc* pot, zdc* grad,
                  cudaStream_t s) {
  if (nt <= 0) return;
  klaunch(k_unsort_col, div_up(nt, TB), TB, 0, s, nt, nd, r, itarg, potsort, gradsort, pscale,
          gscale, ifpgh, pot, grad);
  ZF_LAUNCH_CHECK();
}

// copy of a device buffer on stream s
template <class T>
static void copy_buf3(DevBuf<T>& dst, const DevBuf<T>& src, cudaStream_t s) {
  dst.alloc(src.size(), s);
  if (src.size())
    ZF_CUDA(cudaMemcpyAsync(dst.get(), src.get(), src.size() * sizeof(T),
                            cudaMemcpyDeviceToDevice, s));
}

void setup3d_geom(int ns, const zdc* zsrc, int nt, const zdc* ztarg, const TreeParams& tp,
                  Setup3D& S, cudaStream_t s) {
  // targets that are the sources (the same array) share the sources' tree
  // assignment, order and centres: computed once, copied
  const bool same = ztarg == zsrc && nt == ns;
  DevBuf<double> srcR(3 * (size_t)ns, s), targR(same ? 0 : 3 * (size_t)nt, s);
  klaunch(k_real3, div_up(3L * ns, TB), TB, 0, s, zsrc, 3L * ns, srcR.get());
  if (!same) klaunch(k_real3, div_up(3L * nt, TB), TB, 0, s, ztarg, 3L * nt, targR.get());
  ZF_LAUNCH_CHECK();
  const double* tR = same ? srcR.get() : targR.get();
  build_tree(srcR.get(), ns, tR, nt, tp, S.tree, s);
  sort_points(S.tree, srcR.get(), ns, S.isrc, S.isrcse, s);
  if (same) {
    copy_buf3(S.itarg, S.isrc, s);
    copy_buf3(S.itargse, S.isrcse, s);
  } else {
    sort_points(S.tree, tR, nt, S.itarg, S.itargse, s);
  }
  S.b0 = S.tree.boxsize[0];
  const double* b0 = S.tree.bsz.get();
  S.zsrcsort.alloc(3 * (size_t)ns, s);
  S.ztargsort.alloc(3 * (size_t)nt, s);
  klaunch(k_gather3t, div_up(ns, TB), TB, 0, s, ns, S.isrc.get(), zsrc, b0, S.zsrcsort.get());
  klaunch(k_gather3t, div_up(nt, TB), TB, 0, s, nt, S.itarg.get(), ztarg, b0,
          S.ztargsort.get());
  ZF_LAUNCH_CHECK();
  centres3(S.tree, S.isrcse, S.zsrcsort, b0, S.zcsrc, s);
  if (same) copy_buf3(S.zctarg, S.zcsrc, s);
  else centres3(S.tree, S.itargse, S.ztargsort, b0, S.zctarg, s);
  build_lists(S.tree, S.lists, s);
  S.bsz.resize(S.tree.nlevels + 1);
  for (int l = 0; l <= S.tree.nlevels; l++) S.bsz[l] = S.tree.boxsize[l] / S.b0;
}

void gather_strengths_nd(const Setup3D& S, int ns, int nd, const zdc* charge,
                         const zdc* dipstr, const zdc* dipvec, bool rescale_charge,
                         bool rescale_dipvec, zdc* q, zdc* ds, zdc* dv, cudaStream_t s) {
  if (ns <= 0) return;
  klaunch(k_gather_nd, div_up((long)ns * nd, TB), TB, 0, s, ns, nd, S.isrc.get(), charge,
          dipstr, dipvec, S.tree.bsz.get(), rescale_charge ? 1 : 0, rescale_dipvec ? 1 : 0, q,
          ds, dv);
  ZF_LAUNCH_CHECK();
}

void unsort3d_nd(int nt, int nd, const int* itarg, const zdc* potsort, const zdc* gradsort,
                 zdc pscale, zdc gscale, int ifpgh, zdc* pot, zdc* grad, cudaStream_t s) {
  if (nt <= 0) return;
  klaunch(k_unsort_nd, div_up((long)nt * nd, TB), TB, 0, s, nt, nd, itarg, potsort, gradsort,
          pscale, gscale, ifpgh, pot, grad);
  ZF_LAUNCH_CHECK();
}

void setup3d(const Inputs3D& in, const TreeParams& tp, Setup3D& S, bool rescale_charge,
             bool rescale_dipvec, cudaStream_t s) {
  int ns = in.ns, nt = in.nt;
  // targets that are the sources (the same array) share the sources' tree
  // assignment, order and centres: computed once, copied
  const bool same = in.ztarg == in.zsrc && nt == ns;
  DevBuf<double> srcR(3 * (size_t)ns, s), targR(same ? 0 : 3 * (size_t)nt, s);
  klaunch(k_real3, div_up(3L * ns, TB), TB, 0, s, in.zsrc, 3L * ns, srcR.get());
  if (!same) klaunch(k_real3, div_up(3L * nt, TB), TB, 0, s, in.ztarg, 3L * nt, targR.get());
  ZF_LAUNCH_CHECK();
  const double* tR = same ? srcR.get() : targR.get();
  build_tree(srcR.get(), ns, tR, nt, tp, S.tree, s);
  sort_points(S.tree, srcR.get(), ns, S.isrc, S.isrcse, s);
  if (same) {
    copy_buf3(S.itarg, S.isrc, s);
    copy_buf3(S.itargse, S.isrcse, s);
  } else {
    sort_points(S.tree, tR, nt, S.itarg, S.itargse, s);
  }
  S.b0 = S.tree.boxsize[0];
  const double* b0 = S.tree.bsz.get();  // device copy of boxsize; entry 0 = b0
  if (in.strengths_ready) in.strengths_ready(s);
  S.zsrcsort.alloc(3 * (size_t)ns, s);
  S.chargesort.alloc(ns, s);
  S.dipstrsort.alloc(ns, s);
  S.dipvecsort.alloc(3 * (size_t)ns, s);
  S.ztargsort.alloc(3 * (size_t)nt, s);
  klaunch(k_gather3, div_up(ns, TB), TB, 0, s, ns, S.isrc.get(), in.zsrc,
          in.ifcharge ? in.charge : nullptr, in.ifdipole ? in.dipstr : nullptr,
          in.ifdipole ? in.dipvec : nullptr, b0, rescale_charge ? 1.0 : 0.0,
          rescale_dipvec ? 1.0 : 0.0, S.zsrcsort.get(), S.chargesort.get(), S.dipstrsort.get(),
          S.dipvecsort.get());
  klaunch(k_gather3t, div_up(nt, TB), TB, 0, s, nt, S.itarg.get(), in.ztarg, b0,
          S.ztargsort.get());
  ZF_LAUNCH_CHECK();
  centres3(S.tree, S.isrcse, S.zsrcsort, b0, S.zcsrc, s);
  if (same) copy_buf3(S.zctarg, S.zcsrc, s);
  else centres3(S.tree, S.itargse, S.ztargsort, b0, S.zctarg, s);
  build_lists(S.tree, S.lists, s);
  S.bsz.resize(S.tree.nlevels + 1);
  for (int l = 0; l <= S.tree.nlevels; l++) S.bsz[l] = S.tree.boxsize[l] / S.b0;
}

void unsort3d(int nt, const int* itarg, const zdc* potsort, const zdc* gradsort, zdc pscale,
              zdc gscale, int ifpgh, zdc* pot, zdc* grad, cudaStream_t s) {
  klaunch(k_unsort3, div_up(nt, TB), TB, 0, s, nt, itarg, potsort, gradsort, pscale, gscale, ifpgh,
          pot, grad);
  ZF_LAUNCH_CHECK();
}

}  // namespace zf
