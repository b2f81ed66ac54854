// Device tree builder: refinement, level restriction, renumbering, colleagues,
// point sort and U/V/W/X lists, reproducing the reference's integer results.
//
// Reference algorithm (file:line in the reference tree):
//   bounding box + refinement loop   zfmm2d/src/common/pts_tree2d.f:108-331, 455-611
//   child creation (cumsum order)    zfmm2d/src/common/tree_routs2d.f:9-56
//   stable partition into children   pts_tree2d.f:669-764 (3D: pts_tree3d.f:913-1102)
//   colleagues                       tree_routs2d.f:100-212
//   level restriction                pts_tree2d.f:768-1078, updateflags tree_routs2d.f:218-329
//   renumbering after restriction    pts_tree2d.f:1083-1232
//   final point sort                 pts_tree2d.f:1239-1264
//   lists 1-4                        tree_routs2d.f:463-746 (3D: tree_routs3d.f:414-712)
//
// GPU formulation:
//   * one thread per box of a level (or per point), one launch per level, as the
//     reference's level loops are sequential but its box loops are independent;
//   * new boxes are numbered by an exclusive scan of the refine flags of the
//     level, i.e. children of the r-th refined box get ids nbctr + r*NC + c,
//     which is the reference's cumsum numbering;
//   * the per-level point-to-child assignment runs over a Z-ordered copy of
//     the points (the counts it produces do not depend on the order);
//   * the final point order of pts_tree_sort (a stable recursive partition) is
//     the order of a stable sort of the points by the start offset of their
//     leaf, with leaf offsets from a bottom-up count and a top-down prefix in
//     child order.  cub's radix sort is stable.
// This file is compiled with --fmad=false so that the distance tests see the
// same roundings as the reference (no contracted multiply-adds).
#include <algorithm>
#include <climits>
#include <cmath>
#include <cub/cub.cuh>
#include <vector>
#include "tree.cuh"

namespace zf {

namespace {

constexpr int TB = 256;

template <int D>
__device__ __forceinline__ bool within_tol(const double* a, const double* b, double tol) {
#pragma unroll
  for (int d = 0; d < D; d++)
    if (!(fabs(a[d] - b[d]) <= tol)) return false;
  return true;
}

template <int D>
__device__ __forceinline__ int child_index(const double* p, const double* c) {
  int k = 0;
#pragma unroll
  for (int d = 0; d < D; d++)
    if (!(p[d] - c[d] < 0)) k |= 1 << d;
  return k;
}

// ---- bounding box ------------------------------------------------------------
// min / max that keep a NaN once one is seen (fmin / fmax drop it), so a NaN
// coordinate reaches the root box size, where the host refuses it
__device__ __forceinline__ double nan_min(double a, double b) {
  return (a != a || b != b) ? a + b : fmin(a, b);
}
__device__ __forceinline__ double nan_max(double a, double b) {
  return (a != a || b != b) ? a + b : fmax(a, b);
}

template <int D>
__global__ void k_bbox_partial(const double* __restrict__ a, int na, const double* __restrict__ b,
                               int nb, double* __restrict__ part) {
  double mn[D], mx[D];
#pragma unroll
  for (int d = 0; d < D; d++) { mn[d] = INFINITY; mx[d] = -INFINITY; }
  long tot = (long)na + nb;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < tot; i += (long)gridDim.x * blockDim.x) {
    const double* p = i < na ? a + i * D : b + (i - na) * D;
#pragma unroll
    for (int d = 0; d < D; d++) {
      double v = p[d];
      mn[d] = nan_min(mn[d], v);
      mx[d] = nan_max(mx[d], v);
    }
  }
  __shared__ double smn[D][TB], smx[D][TB];
#pragma unroll
  for (int d = 0; d < D; d++) { smn[d][threadIdx.x] = mn[d]; smx[d][threadIdx.x] = mx[d]; }
  __syncthreads();
  for (int o = TB / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
#pragma unroll
      for (int d = 0; d < D; d++) {
        smn[d][threadIdx.x] = nan_min(smn[d][threadIdx.x], smn[d][threadIdx.x + o]);
        smx[d][threadIdx.x] = nan_max(smx[d][threadIdx.x], smx[d][threadIdx.x + o]);
      }
    __syncthreads();
  }
  if (threadIdx.x == 0)
#pragma unroll
    for (int d = 0; d < D; d++) {
      part[blockIdx.x * 2 * D + d] = smn[d][0];
      part[blockIdx.x * 2 * D + D + d] = smx[d][0];
    }
}

// root box from the partial extrema (single thread)
template <int D>
__global__ void k_root(const double* part, int nparts, double* centers, double* bs0, int* ilevel,
                       int* iparent, int* nchild, int* ichild, int* nsrc, int* ntarg, int ns,
                       int nt) {
  double mn[D], mx[D];
  for (int d = 0; d < D; d++) { mn[d] = INFINITY; mx[d] = -INFINITY; }
  for (int i = 0; i < nparts; i++)
    for (int d = 0; d < D; d++) {
      mn[d] = nan_min(mn[d], part[i * 2 * D + d]);
      mx[d] = nan_max(mx[d], part[i * 2 * D + D + d]);
    }
  double b = mx[0] - mn[0];
  for (int d = 1; d < D; d++)
    if (mx[d] - mn[d] > b || mx[d] - mn[d] != mx[d] - mn[d]) b = mx[d] - mn[d];
  *bs0 = b;
  for (int d = 0; d < D; d++) centers[d] = (mn[d] + mx[d]) / 2;
  ilevel[0] = 0;
  iparent[0] = -1;
  nchild[0] = 0;
  for (int c = 0; c < (1 << D); c++) ichild[c] = -1;
  nsrc[0] = ns;
  ntarg[0] = nt;
}

// ---- refinement --------------------------------------------------------------
// 0/1 flags of the concatenation of in[lo1, lo1+n1) and in[lo2, lo2+n2)
__global__ void k_gt0_2(const int* in, int lo1, int n1, int lo2, int n2, int* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n1 + n2) return;
  out[i] = in[i < n1 ? lo1 + i : lo2 + (i - n1)] > 0 ? 1 : 0;
}

// exclusive prefix of the flags at positions pos[0, np); a position equal to
// the length n gives the total
__global__ void k_pick(const int* flag, const int* rank, int n, const int* pos, int np,
                       int* out) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= np) return;
  int p = pos[k];
  out[k] = p < n ? rank[p] : (n > 0 ? rank[n - 1] + flag[n - 1] : 0);
}

// children of every flagged box of [lo, lo+nb): ids first + rank*NC + c.
// flagmode: children of iflag==1 parents become flag++ (3), of iflag==2 become 0
// (tree_refine_boxes_flag); otherwise plain refinement.
// the NC children of box b, ids base .. base+NC-1, on level lev
template <int D>
__device__ __forceinline__ void make_children_of(int b, int base, double bs, int lev,
                                                 int flagmode, double* centers, int* ilevel,
                                                 int* iparent, int* nchild, int* ichild,
                                                 int* iflag, int* nsrc, int* ntarg) {
  constexpr int NC = 1 << D;
  nchild[b] = NC;
  double cb[D];
#pragma unroll
  for (int d = 0; d < D; d++) cb[d] = centers[b * D + d];
  int pf = iflag[b];
  for (int c = 0; c < NC; c++) {
    int j = base + c;
#pragma unroll
    for (int d = 0; d < D; d++) {
      double sgn = ((c >> d) & 1) ? 1.0 : -1.0;
      centers[j * D + d] = cb[d] + (sgn * bs) / 2;
    }
    iparent[j] = b;
    nchild[j] = 0;
    for (int l = 0; l < NC; l++) ichild[j * NC + l] = -1;
    ichild[b * NC + c] = j;
    ilevel[j] = lev;
    iflag[j] = flagmode ? (pf == 1 ? 3 : 0) : 0;
    if (nsrc) { nsrc[j] = 0; ntarg[j] = 0; }
  }
}

template <int D>
__global__ void k_make_children(int lo, int nb, const int* flag01, const int* rank, int first,
                                double bs, int lev, int flagmode, double* centers, int* ilevel,
                                int* iparent, int* nchild, int* ichild, int* iflag, int* nsrc,
                                int* ntarg) {
  constexpr int NC = 1 << D;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb || !flag01[i]) return;
  make_children_of<D>(lo + i, first + rank[i] * NC, bs, lev, flagmode, centers, ilevel, iparent,
                      nchild, ichild, iflag, nsrc, ntarg);
}


// ---- refinement loop driven from the device -----------------------------------
// lev[2l], lev[2l+1]: first and last box of level l (empty when last < first);
// *nbox: boxes so far; nref[l]: boxes refined on level l.  A level's kernels
// are launched with grids sized by an upper bound ub on its box count and read
// the level's range from lev, so the host does not wait for each level.

// refinement flags of the boxes of level l (iflag, and fl[i] for the i-th box
// of the level, 0 beyond the level's last box)
__global__ void k_level_flags_d(const int* lev, int l, int ub, const int* nsrc, const int* ntarg,
                                int idivflag, int ndiv, int force, int* iflag, int* fl) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ub) return;
  const int lo = lev[2 * l], hi = lev[2 * l + 1];
  int r = 0;
  if (lo + i <= hi) {
    const int b = lo + i;
    r = 1;
    if (!force) {
      int nss = nsrc[b], ntt = ntarg[b];
      int nn = idivflag == 0 ? nss : (idivflag == 1 ? ntt : max(nss, ntt));
      r = nn > ndiv;
    }
    iflag[b] = r;
  }
  fl[i] = r;
}

// the range of level l+1 from the exclusive scan rank of fl (single thread)
__global__ void k_level_advance(int* lev, int l, int ub, const int* fl, const int* rank, int NC,
                                int* nbox, int* nref) {
  const int tot = ub > 0 ? rank[ub - 1] + fl[ub - 1] : 0;
  const int first = *nbox;
  lev[2 * (l + 1)] = first;
  lev[2 * (l + 1) + 1] = first + tot * NC - 1;
  *nbox = first + tot * NC;
  nref[l] = tot;
}

// children of the flagged boxes of level l, numbered from the first box of
// level l+1 in scan order
template <int D>
__global__ void k_make_children_d(const int* lev, int l, int ub, const int* fl, const int* rank,
                                  double bs, double* centers, int* ilevel, int* iparent,
                                  int* nchild, int* ichild, int* iflag, int* nsrc, int* ntarg) {
  constexpr int NC = 1 << D;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ub || !fl[i]) return;
  make_children_of<D>(lev[2 * l] + i, lev[2 * (l + 1)] + rank[i] * NC, bs, l + 1, 0, centers,
                      ilevel, iparent, nchild, ichild, iflag, nsrc, ntarg);
}

// dst = src over the boxes of level l (targets that are the sources)
__global__ void k_copy_level(const int* lev, int l, int ub, const int* src, int* dst) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ub && lev[2 * l] + i <= lev[2 * l + 1]) dst[lev[2 * l] + i] = src[lev[2 * l] + i];
}

template <int D>
__global__ void k_assign(const double* __restrict__ pts, int n, int* __restrict__ pbox,
                         const int* __restrict__ ilevel, const int* __restrict__ nchild,
                         const int* __restrict__ ichild, const double* __restrict__ centers,
                         int lev, int* __restrict__ cnt) {
  constexpr int NC = 1 << D;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int b = pbox[i];
  if (ilevel[b] != lev || nchild[b] == 0) return;
  double p[D];
#pragma unroll
  for (int d = 0; d < D; d++) p[d] = pts[(long)i * D + d];
  int c = child_index<D>(p, centers + b * D);
  int j = ichild[b * NC + c];
  pbox[i] = j;
  // points of one warp mostly fall in the same few boxes (at the coarse levels
  // all of them do): one atomic per distinct box and warp instead of one per
  // point, so the counters of the few coarse boxes are not serialised
  unsigned grp = __match_any_sync(__activemask(), j);
  if ((threadIdx.x & 31) == __ffs(grp) - 1) atomicAdd(&cnt[j], __popc(grp));
}

// ---- Z-order of the points for the assignment passes -------------------------
// Key of a point: its coordinates relative to the root box, quantised to BITS
// bits each and interleaved (Z order), so that the points of one box of any
// level down to BITS are contiguous in key order, up to rounding at the box
// faces.  The level-by-level assignment runs over the points in this order:
// warps then read coalesced coordinates, look up one or two boxes and add to
// one or two counters.  Box counts do not depend on the order, so the tree is
// the same as in input order; the final point order (sort_points) is taken in
// input order.
template <int D>
__global__ void k_zkey(const double* __restrict__ pts, int n, const double* __restrict__ centers,
                       const double* __restrict__ bs0, unsigned long long* __restrict__ key,
                       int* __restrict__ idx) {
  constexpr int BITS = D == 2 ? 31 : 21;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double b = *bs0, top = (double)((1u << BITS) - 1);
  const double sc = b > 0 ? ldexp(1.0, BITS) / b : 0.0;
  unsigned long long k = 0;
#pragma unroll
  for (int d = 0; d < D; d++) {
    double u = (pts[(long)i * D + d] - (centers[d] - 0.5 * b)) * sc;
    u = u < 0 ? 0.0 : (u > top ? top : u);
    unsigned long long q = (unsigned long long)u;
#pragma unroll
    for (int bit = 0; bit < BITS; bit++) k |= ((q >> bit) & 1ull) << (bit * D + d);
  }
  key[i] = k;
  idx[i] = i;
}

template <int D>
__global__ void k_gather_pts(const double* __restrict__ pts, const int* __restrict__ idx, int n,
                             double* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int j = idx[i];
#pragma unroll
  for (int d = 0; d < D; d++) out[(long)i * D + d] = pts[(long)j * D + d];
}

// ---- colleagues --------------------------------------------------------------
template <int D>
__global__ void k_coll(int lo, int hi, double tol, const int* __restrict__ iparent,
                       const int* __restrict__ ichild, const double* __restrict__ centers,
                       int mnbors, int* ncoll, int* coll) {
  constexpr int NC = 1 << D;
  int b = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (b > hi) return;
  int dad = iparent[b];
  int cnt = 0;
  int nd = ncoll[dad];
  for (int i = 0; i < nd; i++) {
    int jb = coll[(long)dad * mnbors + i];
    for (int c = 0; c < NC; c++) {
      int kb = ichild[jb * NC + c];
      if (kb >= 0 && within_tol<D>(centers + kb * D, centers + b * D, tol)) {
        coll[(long)b * mnbors + cnt] = kb;
        cnt++;
      }
    }
  }
  for (int k = cnt; k < mnbors; k++) coll[(long)b * mnbors + k] = -1;
  ncoll[b] = cnt;
}

// The same lists with one lane per colleague of the parent: a group of G
// lanes (G a power of two >= mnbors, within one warp) serves box b; lane i
// tests the children of the parent's i-th colleague in child order, and an
// exclusive prefix of the lanes' counts places them, so the list order is the
// order of k_coll (parent colleague, then child).
template <int D, int G>
__global__ void k_coll_g(int lo, int hi, double tol, const int* __restrict__ iparent,
                         const int* __restrict__ ichild, const double* __restrict__ centers,
                         int mnbors, int* ncoll, int* coll) {
  constexpr int NC = 1 << D;
  const int sub = threadIdx.x & (G - 1);
  const long gi = (blockIdx.x * (long)blockDim.x + threadIdx.x) / G;
  const bool valid = gi <= (long)(hi - lo);
  const int b = valid ? lo + (int)gi : lo;
  const int dad = valid ? iparent[b] : 0;
  const int nd = valid ? ncoll[dad] : 0;
  int found[NC], cnt = 0;
  if (sub < nd) {
    const int jb = coll[(long)dad * mnbors + sub];
#pragma unroll
    for (int c = 0; c < NC; c++) {
      const int kb = ichild[jb * NC + c];
      if (kb >= 0 && within_tol<D>(centers + kb * D, centers + b * D, tol)) found[cnt++] = kb;
    }
  }
  int x = cnt;  // inclusive prefix over the group
#pragma unroll
  for (int o = 1; o < G; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o, G);
    if (sub >= o) x += y;
  }
  const int total = __shfl_sync(0xffffffffu, x, G - 1, G);
  if (!valid) return;
  int* out = coll + (long)b * mnbors;
  for (int k = 0; k < cnt; k++) out[x - cnt + k] = found[k];
  for (int k = total + sub; k < mnbors; k += G) out[k] = -1;
  if (sub == 0) ncoll[b] = total;
}

// colleagues of boxes lo..hi (their parents' lists complete)
template <int D>
void launch_coll(int lo, int hi, double tol, const int* iparent, const int* ichild,
                 const double* centers, int mnbors, int* ncoll, int* coll, cudaStream_t s) {
  if (hi < lo) return;
  const long n = hi - lo + 1;
  if (mnbors <= 16)
    klaunch(k_coll_g<D, 16>, (int)div_up(n * 16, (long)TB), TB, 0, s, lo, hi, tol, iparent,
            ichild, centers, mnbors, ncoll, coll);
  else if (mnbors <= 32)
    klaunch(k_coll_g<D, 32>, (int)div_up(n * 32, (long)TB), TB, 0, s, lo, hi, tol, iparent,
            ichild, centers, mnbors, ncoll, coll);
  else
    klaunch(k_coll<D>, (int)div_up(n, (long)TB), TB, 0, s, lo, hi, tol, iparent, ichild,
            centers, mnbors, ncoll, coll);
}

__global__ void k_coll_root(int* ncoll, int* coll, int mnbors) {
  ncoll[0] = 1;
  coll[0] = 0;
  for (int k = 1; k < mnbors; k++) coll[k] = -1;
}

// ---- level restriction -------------------------------------------------------
template <int D>
__global__ void k_lr_flag1(int lo, int hi, double distest, const int* iparent, const int* nchild,
                           const double* centers, const int* ncoll, const int* coll, int mnbors,
                           int* iflag) {
  int b = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (b > hi) return;
  int idad = iparent[b], igd = iparent[idad];
  for (int i = 0; i < ncoll[igd]; i++) {
    int jb = coll[(long)igd * mnbors + i];
    if (nchild[jb] == 0 && iflag[jb] == 0 &&
        within_tol<D>(centers + jb * D, centers + idad * D, distest))
      iflag[jb] = 1;
  }
}

template <int D>
__global__ void k_lr_flag2(int lo, int hi, double distest, const int* iparent, const int* nchild,
                           const double* centers, const int* ncoll, const int* coll, int mnbors,
                           int* iflag) {
  int b = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (b > hi) return;
  int f = iflag[b];
  if (f != 1 && f != 2) return;
  int idad = iparent[b];
  for (int i = 0; i < ncoll[idad]; i++) {
    int jb = coll[(long)idad * mnbors + i];
    if (nchild[jb] == 0 && iflag[jb] == 0 &&
        within_tol<D>(centers + jb * D, centers + b * D, distest))
      iflag[jb] = 2;
  }
}

template <int D>
__global__ void k_updateflags(int lo, int hi, double distest, const int* nchild, const int* ichild,
                              const double* centers, const int* ncoll, const int* coll,
                              int mnbors, int* iflag) {
  constexpr int NC = 1 << D;
  int b = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (b > hi || iflag[b] != 3) return;
  int f = 0;
  for (int i = 0; i < ncoll[b] && !f; i++) {
    int jb = coll[(long)b * mnbors + i];
    for (int c = 0; c < NC; c++) {
      int kb = ichild[jb * NC + c];
      if (kb >= 0 && nchild[kb] > 0 && within_tol<D>(centers + kb * D, centers + b * D, distest)) {
        f = 1;
        break;
      }
    }
  }
  iflag[b] = f;
}

// boxes per level whose flag is 3 (to be checked by the second pass)
__global__ void k_count_flag3(int n, const int* ilevel, const int* iflag, int* cnt) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  const bool f = b < n && iflag[b] == 3;
  const unsigned m = __ballot_sync(0xffffffffu, f);
  if (!f) return;
  // consecutive boxes share a level: one atomic per level present in the warp
  const int lv = ilevel[b];
  const unsigned grp = __match_any_sync(m, lv);
  if ((threadIdx.x & 31) == __ffs(grp) - 1) atomicAdd(&cnt[lv], __popc(grp));
}

__global__ void k_reset_flags(int n, int* iflag) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < n && iflag[b] != 3) iflag[b] = 0;
}

// renumbering: lev_info[l] = {lo, hi, tlo, thi, base}
__global__ void k_reorg_map(int n, const int* ilevel, const int* lev_info, int* map) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  int l = ilevel[b];
  const int* li = lev_info + 5 * l;
  int m;
  if (l <= 1) m = b;
  else if (b >= li[0] && b <= li[1]) m = li[4] + (b - li[0]);
  else m = li[4] + (li[1] - li[0] + 1) + (b - li[2]);
  map[b] = m;
}

template <int D>
__global__ void k_reorg_scatter(int n, const int* map, const int* ilevel, const int* iparent,
                                const int* nchild, const int* ichild, const int* iflag,
                                const double* centers, int* nilevel, int* niparent, int* nnchild,
                                int* nichild, int* niflag, double* ncenters) {
  constexpr int NC = 1 << D;
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  int m = map[b];
  nilevel[m] = ilevel[b];
  nnchild[m] = nchild[b];
  niflag[m] = iflag[b];
  int p = iparent[b];
  niparent[m] = p < 0 ? -1 : map[p];
  for (int c = 0; c < NC; c++) {
    int ch = ichild[b * NC + c];
    nichild[m * NC + c] = ch < 0 ? -1 : map[ch];
  }
#pragma unroll
  for (int d = 0; d < D; d++) ncenters[m * D + d] = centers[b * D + d];
}

// ---- point sort --------------------------------------------------------------
template <int D>
__global__ void k_descend(const double* __restrict__ pts, int n, const int* __restrict__ nchild,
                          const int* __restrict__ ichild, const double* __restrict__ centers,
                          int* __restrict__ leaf, int* __restrict__ cnt) {
  constexpr int NC = 1 << D;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double p[D];
#pragma unroll
  for (int d = 0; d < D; d++) p[d] = pts[(long)i * D + d];
  int b = 0;
  while (nchild[b] > 0) b = ichild[b * NC + child_index<D>(p, centers + b * D)];
  leaf[i] = b;
  atomicAdd(&cnt[b], 1);
}

template <int D>
__global__ void k_sum_children(int lo, int hi, const int* nchild, const int* ichild, int* cnt) {
  constexpr int NC = 1 << D;
  int b = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (b > hi || nchild[b] == 0) return;
  int s = 0;
  for (int c = 0; c < NC; c++) s += cnt[ichild[b * NC + c]];
  cnt[b] = s;
}

template <int D>
__global__ void k_child_starts(int lo, int hi, const int* nchild, const int* ichild,
                               const int* cnt, int* start) {
  constexpr int NC = 1 << D;
  int b = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (b > hi || nchild[b] == 0) return;
  int s = start[b];
  for (int c = 0; c < NC; c++) {
    int ch = ichild[b * NC + c];
    start[ch] = s;
    s += cnt[ch];
  }
}

__global__ void k_sort_keys(int n, const int* leaf, const int* start, int* key, int* idx) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  key[i] = start[leaf[i]];
  idx[i] = i;
}

__global__ void k_ranges(int nb, const int* start, const int* cnt, int* se) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  se[2 * b] = start[b];
  se[2 * b + 1] = start[b] + cnt[b] - 1;
}

// ---- lists 1..4 ----------------------------------------------------------------
template <int D>
__global__ void k_lists(int nb, int fill, const int* __restrict__ ilevel,
                        const int* __restrict__ iparent, const int* __restrict__ nchild,
                        const int* __restrict__ ichild, const double* __restrict__ C,
                        const int* __restrict__ ncoll, const int* __restrict__ coll, int mnbors,
                        const double* __restrict__ bsz, int isep, int* n1, int* n2, int* n3,
                        int* n4, int* l1, int* l2, int* l3, int* l4, int m1, int m2, int m3,
                        int m4) {
  constexpr int NC = 1 << D;
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  int c1 = 0, c2 = 0, c3 = 0, c4 = 0;
#define PUSH(k, v)                                     \
  do {                                                 \
    if (fill) l##k[(long)b * m##k + c##k] = (v);      \
    c##k++;                                            \
  } while (0)
  if (b == 0) {
    if (nchild[0] == 0) PUSH(1, 0);
  } else {
    int ilev = ilevel[b];
    int dad = iparent[b];
    double sep = 1.05 * isep * bsz[ilev];
    for (int i = 0; i < ncoll[dad]; i++) {
      int jb = coll[(long)dad * mnbors + i];
      for (int c = 0; c < NC; c++) {
        int kb = ichild[jb * NC + c];
        if (kb < 0) continue;
        bool far = false;
#pragma unroll
        for (int d = 0; d < D; d++)
          if (fabs(C[kb * D + d] - C[b * D + d]) >= sep) far = true;
        if (far) PUSH(2, kb);
      }
    }
    double dup = 1.05 * (bsz[ilev] + bsz[ilev + 1]) / 2.0 * isep;
    double ddn = 1.05 * (bsz[ilev] + bsz[ilev - 1]) / 2.0 * isep;
    if (nchild[b] == 0) {
      for (int i = 0; i < ncoll[b]; i++) {
        int jb = coll[(long)b * mnbors + i];
        if (nchild[jb] == 0) {
          PUSH(1, jb);
        } else {
          for (int c = 0; c < NC; c++) {
            int kb = ichild[jb * NC + c];
            if (kb < 0) continue;
            bool near = true;
#pragma unroll
            for (int d = 0; d < D; d++)
              if (!(fabs(C[kb * D + d] - C[b * D + d]) < dup)) near = false;
            if (near) PUSH(1, kb);
            else PUSH(3, kb);
          }
        }
      }
      for (int i = 0; i < ncoll[dad]; i++) {
        int jb = coll[(long)dad * mnbors + i];
        if (nchild[jb] == 0) {
          bool near = true;
#pragma unroll
          for (int d = 0; d < D; d++)
            if (!(fabs(C[jb * D + d] - C[b * D + d]) < ddn)) near = false;
          if (near) PUSH(1, jb);
        }
      }
    }
    for (int i = 0; i < ncoll[dad]; i++) {
      int jb = coll[(long)dad * mnbors + i];
      if (nchild[jb] == 0) {
        bool far = false;
#pragma unroll
        for (int d = 0; d < D; d++)
          if (fabs(C[jb * D + d] - C[b * D + d]) > ddn) far = true;
        if (far) PUSH(4, jb);
      }
    }
  }
#undef PUSH
  n1[b] = c1;
  n2[b] = c2;
  n3[b] = c3;
  n4[b] = c4;
}

// maxima of four count arrays: grid-stride, one atomicMax per block and array
// (out zeroed by the caller)
__global__ void k_max4(int nb, const int* a, const int* b, const int* c, const int* d, int* out) {
  __shared__ int s[4][TB];
  int m0 = 0, m1 = 0, m2 = 0, m3 = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x) {
    m0 = max(m0, a[i]); m1 = max(m1, b[i]); m2 = max(m2, c[i]); m3 = max(m3, d[i]);
  }
  s[0][threadIdx.x] = m0; s[1][threadIdx.x] = m1; s[2][threadIdx.x] = m2; s[3][threadIdx.x] = m3;
  __syncthreads();
  for (int o = TB / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int k = 0; k < 4; k++) s[k][threadIdx.x] = max(s[k][threadIdx.x], s[k][threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x < 4) atomicMax(&out[threadIdx.x], s[threadIdx.x][0]);
}

// ---- host helpers -----------------------------------------------------------
// Page-locked host words that receive the scan results, one block per host
// thread, allocated on the thread's first tree build and freed when the
// thread ends: page-locking and releasing memory on every build would cost
// milliseconds (and the release waits for the device).
constexpr int kPinnedWords = 1024;
struct PinnedWords {
  int* p = nullptr;
  ~PinnedWords() {
    if (p) cudaFreeHost(p);
  }
  int* get() {
    if (!p) ZF_CUDA(cudaMallocHost((void**)&p, kPinnedWords * sizeof(int)));
    return p;
  }
};
int* pinned_words() {
  thread_local PinnedWords w;
  return w.get();
}

struct Scanner {
  DevBuf<char> tmp;
  DevBuf<int> flag01, rank;
  int* h_words = nullptr;  // page-locked result words
  cudaStream_t s;
  explicit Scanner(cudaStream_t st) : s(st) { h_words = pinned_words(); }
  // flags01/rank over the concatenation of src[lo1, lo1+n1) and
  // src[lo2, lo2+n2) in one scan; returns the exclusive prefix at each of
  // `pos` (a position n1+n2 gives the total), with one wait for the host
  std::vector<int> scan_at(const int* src, int lo1, int n1, int lo2, int n2,
                           const std::vector<int>& pos) {
    const int n = n1 + n2, np = (int)pos.size();
    std::vector<int> out(np, 0);
    if (n <= 0 || np == 0) return out;
    if ((int)flag01.size() < n) { flag01.alloc(n, s); rank.alloc(n, s); }
    klaunch(k_gt0_2, div_up(n, TB), TB, 0, s, src, lo1, n1, lo2, n2, flag01.get());
    size_t bytes = 0;
    ZF_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, flag01.get(), rank.get(), n, s));
    if (tmp.size() < bytes) tmp.alloc(bytes, s);
    ZF_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), bytes, flag01.get(), rank.get(), n, s));
    DevBuf<int> dpos(np, s), dout(np, s);
    ZF_CUDA(cudaMemcpyAsync(dpos.get(), pos.data(), np * sizeof(int), cudaMemcpyHostToDevice, s));
    klaunch(k_pick, div_up(np, TB), TB, 0, s, flag01.get(), rank.get(), n, dpos.get(), np,
            dout.get());
    int* h = np <= kPinnedWords ? h_words : out.data();  // above 1024 positions: pageable
    ZF_CUDA(cudaMemcpyAsync(h, dout.get(), np * sizeof(int), cudaMemcpyDeviceToHost, s));
    ZF_CUDA(cudaStreamSynchronize(s));
    if (h != out.data()) std::copy(h, h + np, out.begin());
    return out;
  }
};

struct BoxArrays {
  int D, NC;
  size_t cap = 0;
  cudaStream_t s;
  DevBuf<int> ilevel, iparent, nchild, ichild, iflag, nsrc, ntarg;
  DevBuf<double> centers;
  void reserve(size_t need, size_t n_used) {
    if (need <= cap) return;
    size_t nc = cap ? cap : 1024;
    while (nc < need) nc *= 2;
    ilevel.grow(nc, n_used);
    iparent.grow(nc, n_used);
    nchild.grow(nc, n_used);
    ichild.grow(nc * NC, n_used * NC);
    iflag.grow(nc, n_used);
    nsrc.grow(nc, n_used);
    ntarg.grow(nc, n_used);
    centers.grow(nc * D, n_used * D);
    cap = nc;
  }
};

template <int D>
void colleagues_all(BoxArrays& B, int nlevels, const std::vector<int>& laddr,
                    const std::vector<double>& bsz, int isep, int mnbors, DevBuf<int>& ncoll,
                    DevBuf<int>& coll, cudaStream_t s) {
  klaunch(k_coll_root, 1, 1, 0, s, ncoll.get(), coll.get(), mnbors);
  for (int l = 1; l <= nlevels; l++) {
    int lo = laddr[2 * l], hi = laddr[2 * l + 1];
    if (hi < lo) continue;
    double tol = (double)1.05f * bsz[l] * (double)isep;
    launch_coll<D>(lo, hi, tol, B.iparent.get(), B.ichild.get(), B.centers.get(), mnbors,
                   ncoll.get(), coll.get(), s);
  }
  ZF_LAUNCH_CHECK();
}

// subdivide the flagged boxes (iflag>0) of [lo,hi] and then of [tlo,thi] (the
// children of the second range numbered after those of the first, as two
// successive refinements would number them), with one scan; returns the
// number of new boxes
template <int D>
int refine_flag_ranges(BoxArrays& B, Scanner& S, int& n, int lo, int hi, int tlo, int thi,
                       double bs, int ilev, DevBuf<int>& ncoll, DevBuf<int>& coll, int mnbors,
                       cudaStream_t s) {
  constexpr int NC = 1 << D;
  const int nb1 = hi >= lo ? hi - lo + 1 : 0, nb2 = thi >= tlo ? thi - tlo + 1 : 0;
  if (nb1 + nb2 == 0) return 0;
  const int nref = S.scan_at(B.iflag.get(), lo, nb1, tlo, nb2, {nb1 + nb2})[0];
  if (nref == 0) return 0;
  B.reserve((size_t)n + (size_t)nref * NC, n);
  ncoll.grow(B.cap, n);
  coll.grow(B.cap * mnbors, (size_t)n * mnbors);
  if (nb1 > 0)
    klaunch(k_make_children<D>, div_up(nb1, TB), TB, 0, s, lo, nb1, S.flag01.get(),
            S.rank.get(), n, bs, ilev + 1, 1, B.centers.get(), B.ilevel.get(), B.iparent.get(),
            B.nchild.get(), B.ichild.get(), B.iflag.get(), nullptr, nullptr);
  if (nb2 > 0)
    klaunch(k_make_children<D>, div_up(nb2, TB), TB, 0, s, tlo, nb2, S.flag01.get() + nb1,
            S.rank.get() + nb1, n, bs, ilev + 1, 1, B.centers.get(), B.ilevel.get(),
            B.iparent.get(), B.nchild.get(), B.ichild.get(), B.iflag.get(), nullptr, nullptr);
  ZF_LAUNCH_CHECK();
  n += nref * NC;
  return nref * NC;
}

template <int D>
void reorg(BoxArrays& B, int n, int nlevels, std::vector<int>& laddr, const std::vector<int>& tail,
           cudaStream_t s) {
  constexpr int NC = 1 << D;
  std::vector<int> info(5 * (nlevels + 1), 0);
  int cur = nlevels >= 2 ? laddr[4] : n;
  for (int l = 0; l <= nlevels; l++) {
    info[5 * l + 0] = laddr[2 * l];
    info[5 * l + 1] = laddr[2 * l + 1];
    info[5 * l + 2] = tail[2 * l];
    info[5 * l + 3] = tail[2 * l + 1];
  }
  for (int l = 2; l <= nlevels; l++) {
    int cnt = (laddr[2 * l + 1] - laddr[2 * l] + 1) + (tail[2 * l + 1] - tail[2 * l] + 1);
    info[5 * l + 4] = cur;
    laddr[2 * l] = cur;
    cur += cnt;
    laddr[2 * l + 1] = cur - 1;
  }
  DevBuf<int> d_info(info.size(), s), map(n, s);
  ZF_CUDA(cudaMemcpyAsync(d_info.get(), info.data(), info.size() * sizeof(int),
                          cudaMemcpyHostToDevice, s));
  klaunch(k_reorg_map, div_up(n, TB), TB, 0, s, n, B.ilevel.get(), d_info.get(), map.get());
  DevBuf<int> il(B.cap, s), ip(B.cap, s), nc(B.cap, s), ic(B.cap * NC, s), fl(B.cap, s);
  DevBuf<double> ce(B.cap * D, s);
  klaunch(k_reorg_scatter<D>, div_up(n, TB), TB, 0, s, 
      n, map.get(), B.ilevel.get(), B.iparent.get(), B.nchild.get(), B.ichild.get(),
      B.iflag.get(), B.centers.get(), il.get(), ip.get(), nc.get(), ic.get(), fl.get(), ce.get());
  ZF_LAUNCH_CHECK();
  B.ilevel.swap(il);
  B.iparent.swap(ip);
  B.nchild.swap(nc);
  B.ichild.swap(ic);
  B.iflag.swap(fl);
  B.centers.swap(ce);
  ZF_CUDA(cudaStreamSynchronize(s));  // d_info host vector lifetime
}

// copy of the n points of pts in Z order within the root box (k_zkey)
template <int D>
void zorder_copy(const double* pts, int n, const double* centers, const double* bs0,
                 DevBuf<double>& out, cudaStream_t s) {
  constexpr int BITS = D == 2 ? 31 : 21;
  DevBuf<unsigned long long> key(n, s), key2(n, s);
  DevBuf<int> idx(n, s), idx2(n, s);
  klaunch(k_zkey<D>, div_up(n, TB), TB, 0, s, pts, n, centers, bs0, key.get(), idx.get());
  size_t bytes = 0;
  ZF_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, key.get(), key2.get(), idx.get(),
                                          idx2.get(), n, 0, BITS * D, s));
  DevBuf<char> tmp(bytes, s);
  ZF_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), bytes, key.get(), key2.get(), idx.get(),
                                          idx2.get(), n, 0, BITS * D, s));
  out.alloc((size_t)n * D, s);
  klaunch(k_gather_pts<D>, div_up(n, TB), TB, 0, s, pts, idx2.get(), n, out.get());
  ZF_LAUNCH_CHECK();
}

template <int D>
void build_tree_t(const double* d_src, int ns, const double* d_targ, int nt, const TreeParams& p,
                  DevTree& t, cudaStream_t s) {
  constexpr int NC = 1 << D;
  if (ns < 1 || nt < 1) throw zf_error(ZF_ERR_ARG, "tree needs ns>=1 and nt>=1");
  int mnbors = 1;
  for (int d = 0; d < D; d++) mnbors *= (2 * p.isep + 1);
  BoxArrays B;
  B.D = D;
  B.NC = NC;
  B.s = s;
  B.ilevel.alloc(0, s); B.iparent.alloc(0, s); B.nchild.alloc(0, s); B.ichild.alloc(0, s);
  B.iflag.alloc(0, s); B.nsrc.alloc(0, s); B.ntarg.alloc(0, s); B.centers.alloc(0, s);
  B.reserve(1024, 0);
  Scanner S(s);

  // root
  const int nparts = 296;
  DevBuf<double> part((size_t)nparts * 2 * D, s), d_bs0(1, s);
  klaunch(k_bbox_partial<D>, nparts, TB, 0, s, d_src, ns, d_targ, nt, part.get());
  klaunch(k_root<D>, 1, 1, 0, s, part.get(), nparts, B.centers.get(), d_bs0.get(), B.ilevel.get(),
                            B.iparent.get(), B.nchild.get(), B.ichild.get(), B.nsrc.get(),
                            B.ntarg.get(), ns, nt);
  ZF_LAUNCH_CHECK();
  std::vector<double> bsz(p.nlmax + 2, 0.0);
  ZF_CUDA(cudaMemcpyAsync(bsz.data(), d_bs0.get(), sizeof(double), cudaMemcpyDeviceToHost, s));
  const bool same = d_targ == d_src && nt == ns;
  DevBuf<int> pbs(ns, s), pbt(same ? 0 : nt, s);
  pbs.zero();
  pbt.zero();
  ZF_CUDA(cudaStreamSynchronize(s));
  // a NaN or infinite real part makes the root size non-finite: no tree can be
  // built (the reference would loop or divide by it), so the call is refused
  if (!std::isfinite(bsz[0]))
    throw zf_error(ZF_ERR_ARG, "coordinates must be finite (NaN or Inf in a real part)");
  // the assignment passes run over Z-ordered copies of the points
  DevBuf<double> zs_src, zs_targ;
  zorder_copy<D>(d_src, ns, B.centers.get(), d_bs0.get(), zs_src, s);
  if (!same) zorder_copy<D>(d_targ, nt, B.centers.get(), d_bs0.get(), zs_targ, s);
  const double* a_src = zs_src.get();
  const double* a_targ = same ? a_src : zs_targ.get();

  // Refinement, level by level as in the reference, with the level ranges on
  // the device: a chunk of levels is launched with grids sized by upper
  // bounds on the box counts (a box is refined only with more than ndiv
  // points, so at most (ns + nt) / (ndiv + 1) + 1 boxes of a level are
  // refined, all of them on forced levels), then the host reads the counts
  // back once and stops at the first level that refines nothing.
  const long rmax = ((long)ns + nt) / (p.ndiv + 1) + 1;
  DevBuf<int> dlev(2 * (p.nlmax + 2), s), dnref(p.nlmax + 1, s), dnbox(1, s);
  {
    const int init[3] = {0, 0, 1};  // level 0 = the root; one box
    ZF_CUDA(cudaMemcpyAsync(dlev.get(), init, 2 * sizeof(int), cudaMemcpyHostToDevice, s));
    ZF_CUDA(cudaMemcpyAsync(dnbox.get(), init + 2, sizeof(int), cudaMemcpyHostToDevice, s));
  }
  DevBuf<int> fl, rank;
  DevBuf<char> scan_tmp;
  int* hw = pinned_words();
  int n = 1, nb_cur = 1, l0 = 0, nlevels = -1;
  while (nlevels < 0 && l0 < p.nlmax) {
    // levels l0 .. l1-1 of this chunk, while the boxes they may add stay
    // within max(2^20, 8 n)
    std::vector<long> ub(1, nb_cur);
    long add = 0;
    int l1 = l0;
    while (l1 < p.nlmax) {
      const long u = ub.back(), refined = l1 < p.nlmin ? u : std::min(u, rmax);
      const long next = refined * NC;
      if (l1 > l0 && add + next > std::max(1L << 20, 8L * n)) break;
      if ((long)n + add + next > (long)INT_MAX / 2)
        throw zf_error(ZF_ERR_ARG, "tree too large");
      add += next;
      ub.push_back(next);
      l1++;
    }
    B.reserve((size_t)n + (size_t)add, n);
    long umax = 1;
    for (long u : ub) umax = std::max(umax, u);
    if ((long)fl.size() < umax) {
      fl.alloc(umax, s);
      rank.alloc(umax, s);
    }
    size_t bytes = 0;
    ZF_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, fl.get(), rank.get(), (int)umax, s));
    if (scan_tmp.size() < bytes) scan_tmp.alloc(bytes, s);
    for (int l = l0; l < l1; l++) {
      const int u = (int)ub[l - l0], un = (int)ub[l - l0 + 1];
      bsz[l + 1] = bsz[l] / 2;
      klaunch(k_level_flags_d, div_up(u, TB), TB, 0, s, dlev.get(), l, u, B.nsrc.get(),
              B.ntarg.get(), p.idivflag, p.ndiv, l < p.nlmin ? 1 : 0, B.iflag.get(), fl.get());
      size_t tb = scan_tmp.size();
      ZF_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp.get(), tb, fl.get(), rank.get(), u, s));
      klaunch(k_level_advance, 1, 1, 0, s, dlev.get(), l, u, fl.get(), rank.get(), NC,
              dnbox.get(), dnref.get());
      klaunch(k_make_children_d<D>, div_up(u, TB), TB, 0, s, dlev.get(), l, u, fl.get(),
              rank.get(), bsz[l + 1], B.centers.get(), B.ilevel.get(), B.iparent.get(),
              B.nchild.get(), B.ichild.get(), B.iflag.get(), B.nsrc.get(), B.ntarg.get());
      klaunch(k_assign<D>, div_up(ns, TB), TB, 0, s, a_src, ns, pbs.get(), B.ilevel.get(),
              B.nchild.get(), B.ichild.get(), B.centers.get(), l, B.nsrc.get());
      if (same)  // targets are the sources: the same children, the same counts
        klaunch(k_copy_level, div_up(std::max(un, 1), TB), TB, 0, s, dlev.get(), l + 1, un,
                B.nsrc.get(), B.ntarg.get());
      else
        klaunch(k_assign<D>, div_up(nt, TB), TB, 0, s, a_targ, nt, pbt.get(), B.ilevel.get(),
                B.nchild.get(), B.ichild.get(), B.centers.get(), l, B.ntarg.get());
      ZF_LAUNCH_CHECK();
    }
    // counts of the chunk's levels, the ranges of levels l0+1 .. l1, the box count
    const int nl = l1 - l0;
    ZF_CUDA(cudaMemcpyAsync(hw, dnref.get() + l0, nl * sizeof(int), cudaMemcpyDeviceToHost, s));
    ZF_CUDA(cudaMemcpyAsync(hw + nl, dlev.get() + 2 * (l0 + 1), 2 * nl * sizeof(int),
                            cudaMemcpyDeviceToHost, s));
    ZF_CUDA(cudaMemcpyAsync(hw + 3 * nl, dnbox.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    ZF_CUDA(cudaStreamSynchronize(s));
    for (int k = 0; k < nl && nlevels < 0; k++)
      if (hw[k] == 0) nlevels = l0 + k;
    n = hw[3 * nl];
    nb_cur = hw[nl + 2 * nl - 1] - hw[nl + 2 * nl - 2] + 1;
    l0 = l1;
  }
  if (nlevels < 0) nlevels = p.nlmax;
  std::vector<int> laddr(2 * (nlevels + 1));
  ZF_CUDA(cudaMemcpyAsync(laddr.data(), dlev.get(), laddr.size() * sizeof(int),
                          cudaMemcpyDeviceToHost, s));
  ZF_CUDA(cudaStreamSynchronize(s));
  pbs.release();
  pbt.release();
  zs_src.release();
  zs_targ.release();

  DevBuf<int> ncoll(B.cap, s), coll(B.cap * mnbors, s);
  colleagues_all<D>(B, nlevels, laddr, bsz, p.isep, mnbors, ncoll, coll, s);

  if (nlevels >= 2) {
    // flag and flag+ passes
    B.iflag.zero();
    for (int l = nlevels; l >= 2; l--) {
      int lo = laddr[2 * l], hi = laddr[2 * l + 1];
      double distest = 1.05 * (bsz[l - 1] + bsz[l - 2]) / 2.0;
      distest = distest * p.isep;
      klaunch(k_lr_flag1<D>, div_up(hi - lo + 1, TB), TB, 0, s, lo, hi, distest, B.iparent.get(),
                                                          B.nchild.get(), B.centers.get(),
                                                          ncoll.get(), coll.get(), mnbors,
                                                          B.iflag.get());
    }
    for (int l = nlevels; l >= 1; l--) {
      int lo = laddr[2 * l], hi = laddr[2 * l + 1];
      double distest = 1.05 * (bsz[l] + bsz[l - 1]) / 2.0;
      if (!p.lr_isep_quirk) distest = distest * p.isep;
      klaunch(k_lr_flag2<D>, div_up(hi - lo + 1, TB), TB, 0, s, lo, hi, distest, B.iparent.get(),
                                                          B.nchild.get(), B.centers.get(),
                                                          ncoll.get(), coll.get(), mnbors,
                                                          B.iflag.get());
    }
    ZF_LAUNCH_CHECK();
    std::vector<int> tail(2 * (nlevels + 1));
    for (int l = 0; l <= nlevels; l++) { tail[2 * l] = 0; tail[2 * l + 1] = -1; }
    // the flagged boxes of levels 1 .. nlevels-2 are refined independently of
    // one another (the new boxes are not flagged here): one scan over those
    // levels' boxes, which are contiguous, numbers all of their children
    if (nlevels - 2 >= 1) {
      const int L0 = laddr[2], L1 = laddr[2 * (nlevels - 2) + 1], nall = L1 - L0 + 1;
      std::vector<int> pos;
      for (int l = 1; l <= nlevels - 2; l++) pos.push_back(laddr[2 * l] - L0);
      pos.push_back(nall);
      std::vector<int> r = S.scan_at(B.iflag.get(), L0, nall, 0, 0, pos);
      const int n0 = n, tot = r.back();
      if (tot > 0) {
        B.reserve((size_t)n0 + (size_t)tot * NC, n0);
        ncoll.grow(B.cap, n0);
        coll.grow(B.cap * mnbors, (size_t)n0 * mnbors);
      }
      for (int l = 1; l <= nlevels - 2; l++) {
        const int k = l - 1, lo = laddr[2 * l], nb = laddr[2 * l + 1] - lo + 1;
        if (r[k + 1] > r[k])
          klaunch(k_make_children<D>, div_up(nb, TB), TB, 0, s, lo, nb,
                  S.flag01.get() + (lo - L0), S.rank.get() + (lo - L0), n0, bsz[l + 1], l + 1, 1,
                  B.centers.get(), B.ilevel.get(), B.iparent.get(), B.nchild.get(),
                  B.ichild.get(), B.iflag.get(), nullptr, nullptr);
        tail[2 * (l + 1)] = n0 + NC * r[k];
        tail[2 * (l + 1) + 1] = n0 + NC * r[k + 1] - 1;
      }
      ZF_LAUNCH_CHECK();
      n = n0 + NC * tot;
    }
    reorg<D>(B, n, nlevels, laddr, tail, s);
    ncoll.grow(B.cap, 0);
    coll.grow(B.cap * mnbors, 0);
    colleagues_all<D>(B, nlevels, laddr, bsz, p.isep, mnbors, ncoll, coll, s);

    klaunch(k_reset_flags, div_up(n, TB), TB, 0, s, n, B.iflag.get());
    // a level changes nothing unless some of its boxes have flag 3 or the
    // level above added boxes to it (its tail): the others are skipped
    // without a launch or a wait (flags of existing boxes change only when
    // their own level is processed)
    std::vector<int> nflag3(nlevels + 1, 0);
    {
      DevBuf<int> c3(nlevels + 1, s);
      c3.zero();
      klaunch(k_count_flag3, div_up(n, TB), TB, 0, s, n, B.ilevel.get(), B.iflag.get(), c3.get());
      ZF_CUDA(cudaMemcpyAsync(nflag3.data(), c3.get(), (nlevels + 1) * sizeof(int),
                              cudaMemcpyDeviceToHost, s));
      ZF_CUDA(cudaStreamSynchronize(s));
    }
    for (int l = 0; l <= nlevels; l++) { tail[2 * l] = 0; tail[2 * l + 1] = -1; }
    for (int l = 2; l <= nlevels - 2; l++) {
      if (nflag3[l] == 0 && tail[2 * l + 1] < tail[2 * l]) {
        tail[2 * (l + 1)] = n;
        tail[2 * (l + 1) + 1] = n - 1;
        continue;
      }
      double distest = 1.05 * (bsz[l] + bsz[l + 1]) / 2.0;
      distest = distest * p.isep;
      int lo = laddr[2 * l], hi = laddr[2 * l + 1];
      if (hi >= lo)
        klaunch(k_updateflags<D>, div_up(hi - lo + 1, TB), TB, 0, s, 
            lo, hi, distest, B.nchild.get(), B.ichild.get(), B.centers.get(), ncoll.get(),
            coll.get(), mnbors, B.iflag.get());
      int tlo = tail[2 * l], thi = tail[2 * l + 1];
      if (thi >= tlo)
        klaunch(k_updateflags<D>, div_up(thi - tlo + 1, TB), TB, 0, s, 
            tlo, thi, distest, B.nchild.get(), B.ichild.get(), B.centers.get(), ncoll.get(),
            coll.get(), mnbors, B.iflag.get());
      tail[2 * (l + 1)] = n;
      // the level's boxes and its tail refined with one scan: the children of
      // the tail's boxes are numbered after those of the level's boxes
      refine_flag_ranges<D>(B, S, n, lo, hi, tlo, thi, bsz[l + 1], l, ncoll, coll, mnbors, s);
      tail[2 * (l + 1) + 1] = n - 1;
      int nlo = tail[2 * (l + 1)], nhi = tail[2 * (l + 1) + 1];
      if (nhi >= nlo) {
        double tol = (double)((float)p.isep * 1.05f) * bsz[l + 1];
        launch_coll<D>(nlo, nhi, tol, B.iparent.get(), B.ichild.get(), B.centers.get(), mnbors,
                       ncoll.get(), coll.get(), s);
      }
      ZF_LAUNCH_CHECK();
    }
    reorg<D>(B, n, nlevels, laddr, tail, s);
    ncoll.grow(B.cap, 0);
    coll.grow(B.cap * mnbors, 0);
    colleagues_all<D>(B, nlevels, laddr, bsz, p.isep, mnbors, ncoll, coll, s);
  }

  t.D = D;
  t.NC = NC;
  t.isep = p.isep;
  t.mnbors = mnbors;
  t.nlevels = nlevels;
  t.nboxes = n;
  t.laddr = laddr;
  t.boxsize.assign(bsz.begin(), bsz.begin() + nlevels + 1);
  t.boxsize.push_back(0.0);
  t.ilevel = std::move(B.ilevel);
  t.iparent = std::move(B.iparent);
  t.nchild = std::move(B.nchild);
  t.ichild = std::move(B.ichild);
  t.centers = std::move(B.centers);
  t.ncoll = std::move(ncoll);
  t.coll = std::move(coll);
  t.bsz.alloc(t.boxsize.size(), s);
  ZF_CUDA(cudaMemcpyAsync(t.bsz.get(), t.boxsize.data(), t.boxsize.size() * sizeof(double),
                          cudaMemcpyHostToDevice, s));
  ZF_CUDA(cudaStreamSynchronize(s));
}

template <int D>
void sort_points_t(const DevTree& t, const double* d_pts, int n, DevBuf<int>& perm,
                   DevBuf<int>& se, cudaStream_t s) {
  int nb = t.nboxes;
  DevBuf<int> leaf(n, s), cnt(nb, s), start(nb, s), key(n, s), idx(n, s), key2(n, s);
  cnt.zero();
  perm.alloc(n, s);
  se.alloc(2 * (size_t)nb, s);
  klaunch(k_descend<D>, div_up(n, TB), TB, 0, s, d_pts, n, t.nchild.get(), t.ichild.get(),
                                            t.centers.get(), leaf.get(), cnt.get());
  for (int l = t.nlevels - 1; l >= 0; l--) {
    int lo = t.laddr[2 * l], hi = t.laddr[2 * l + 1];
    klaunch(k_sum_children<D>, div_up(hi - lo + 1, TB), TB, 0, s, lo, hi, t.nchild.get(),
                                                            t.ichild.get(), cnt.get());
  }
  ZF_CUDA(cudaMemsetAsync(start.get(), 0, sizeof(int), s));
  for (int l = 0; l < t.nlevels; l++) {
    int lo = t.laddr[2 * l], hi = t.laddr[2 * l + 1];
    klaunch(k_child_starts<D>, div_up(hi - lo + 1, TB), TB, 0, s, lo, hi, t.nchild.get(),
                                                            t.ichild.get(), cnt.get(), start.get());
  }
  klaunch(k_sort_keys, div_up(n, TB), TB, 0, s, n, leaf.get(), start.get(), key.get(), idx.get());
  ZF_LAUNCH_CHECK();
  int bits = 1;
  while ((1L << bits) <= (long)n) bits++;
  size_t bytes = 0;
  ZF_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, key.get(), key2.get(), idx.get(),
                                          perm.get(), n, 0, bits, s));
  DevBuf<char> tmp(bytes, s);
  ZF_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), bytes, key.get(), key2.get(), idx.get(),
                                          perm.get(), n, 0, bits, s));
  klaunch(k_ranges, div_up(nb, TB), TB, 0, s, nb, start.get(), cnt.get(), se.get());
  ZF_LAUNCH_CHECK();
}

template <int D>
void build_lists_t(const DevTree& t, DevLists& L, cudaStream_t s) {
  int nb = t.nboxes;
  for (int k = 0; k < 4; k++) L.n[k].alloc(nb, s);
  DevBuf<int> mx(4, s);
  int dummy_m = 0;
  klaunch(k_lists<D>, div_up(nb, TB), TB, 0, s, 
      nb, 0, t.ilevel.get(), t.iparent.get(), t.nchild.get(), t.ichild.get(), t.centers.get(),
      t.ncoll.get(), t.coll.get(), t.mnbors, t.bsz.get(), t.isep, L.n[0].get(), L.n[1].get(),
      L.n[2].get(), L.n[3].get(), nullptr, nullptr, nullptr, nullptr, dummy_m, dummy_m, dummy_m,
      dummy_m);
  mx.zero();
  klaunch(k_max4, std::min(div_up(nb, TB), 1184), TB, 0, s, nb, L.n[0].get(), L.n[1].get(),
          L.n[2].get(), L.n[3].get(), mx.get());
  ZF_LAUNCH_CHECK();
  ZF_CUDA(cudaMemcpyAsync(L.mn, mx.get(), 4 * sizeof(int), cudaMemcpyDeviceToHost, s));
  ZF_CUDA(cudaStreamSynchronize(s));
  for (int k = 0; k < 4; k++) {
    L.list[k].alloc((size_t)(L.mn[k] > 0 ? L.mn[k] : 1) * nb, s);
    L.list[k].fill_bytes(0xff);
  }
  klaunch(k_lists<D>, div_up(nb, TB), TB, 0, s, 
      nb, 1, t.ilevel.get(), t.iparent.get(), t.nchild.get(), t.ichild.get(), t.centers.get(),
      t.ncoll.get(), t.coll.get(), t.mnbors, t.bsz.get(), t.isep, L.n[0].get(), L.n[1].get(),
      L.n[2].get(), L.n[3].get(), L.list[0].get(), L.list[1].get(), L.list[2].get(),
      L.list[3].get(), L.mn[0], L.mn[1], L.mn[2], L.mn[3]);
  ZF_LAUNCH_CHECK();
}

}  // namespace

void build_tree(const double* d_src, int ns, const double* d_targ, int nt, const TreeParams& p,
                DevTree& t, cudaStream_t s) {
  if (p.D == 2) build_tree_t<2>(d_src, ns, d_targ, nt, p, t, s);
  else if (p.D == 3) build_tree_t<3>(d_src, ns, d_targ, nt, p, t, s);
  else throw zf_error(ZF_ERR_ARG, "D must be 2 or 3");
}

void sort_points(const DevTree& t, const double* d_pts, int n, DevBuf<int>& perm, DevBuf<int>& se,
                 cudaStream_t s) {
  if (t.D == 2) sort_points_t<2>(t, d_pts, n, perm, se, s);
  else sort_points_t<3>(t, d_pts, n, perm, se, s);
}

void build_lists(const DevTree& t, DevLists& L, cudaStream_t s) {
  if (t.D == 2) build_lists_t<2>(t, L, s);
  else build_lists_t<3>(t, L, s);
}

}  // namespace zf
