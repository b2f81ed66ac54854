// Device-resident adaptive tree, point sort and interaction lists.
//
// Same tree, same box numbering and same lists as the reference's CPU code
// (zfmm2d/src/common/pts_tree2d.f, tree_routs2d.f and their 3D twins), built
// level-synchronously on the GPU: one launch per level and pass, with a prefix
// scan numbering new boxes in parent order exactly as the reference's cumsum.
#pragma once
#include <vector>
#include "devmem.cuh"

namespace zf {

struct TreeParams {
  int D = 2;
  int idivflag = 0;
  int ndiv = 20;
  int nlmin = 0;
  int nlmax = 51;
  int isep = 1;
  int lr_isep_quirk = 0;  // 3D: the flag+ pass omits isep (pts_tree3d.f:1209)
};

struct DevTree {
  int D = 2, NC = 4, isep = 1, mnbors = 9, nlevels = 0, nboxes = 0;
  std::vector<int> laddr;       // host copy, [2*(nlevels+1)] first,last box per level
  std::vector<double> boxsize;  // host copy, [nlevels+2] (last entry 0)
  DevBuf<int> ilevel, iparent, nchild, ichild, ncoll, coll;
  DevBuf<double> centers;       // [nboxes*D]
  DevBuf<double> bsz;           // device copy of boxsize
};

struct DevLists {
  int mn[4] = {0, 0, 0, 0};
  DevBuf<int> n[4];     // counts per box
  DevBuf<int> list[4];  // [mn[k]*nboxes], entry i of box b at b*mn[k]+i
};

// d_src: real coordinates [ns*D], d_targ: [nt*D]
void build_tree(const double* d_src, int ns, const double* d_targ, int nt, const TreeParams& p,
                DevTree& t, cudaStream_t s);
// pts_tree_sort: perm[i] = original index of the i-th sorted point; se[2*b] /
// se[2*b+1] first / last sorted position of box b (last < first when empty)
void sort_points(const DevTree& t, const double* d_pts, int n, DevBuf<int>& perm,
                 DevBuf<int>& se, cudaStream_t s);
void build_lists(const DevTree& t, DevLists& L, cudaStream_t s);

}  // namespace zf
