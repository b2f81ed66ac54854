// Shared set-up of the 3D complex-coordinate FMMs (zlfmm3d / zhfmm3d):
// real parts -> device octree -> sort -> reorder -> complex box centres ->
// rescaling to the unit root box.
//
// Reference: zfmm3d/src/laplace/zlfmm3d.f:60-200 (identical steps in
// zfmm3d/src/helmholtz/zhfmm3d.f:60-200).  After the centres are formed, every
// coordinate, centre and box size is multiplied by b0inv = 1/boxsize(0),
// charges by b0inv and dipole vectors by b0inv^2 (zlfmm3d.f:187-200).
#pragma once
#include <functional>
#include <vector>
#include "tree.cuh"
#include "zcomplex.cuh"

namespace zf {

struct Inputs3D {
  int ns = 0, nt = 0;
  const zdc* zsrc = nullptr;    // zsrc(3,ns)
  const zdc* charge = nullptr;
  const zdc* dipstr = nullptr;
  const zdc* dipvec = nullptr;  // dipvec(3,ns)
  const zdc* ztarg = nullptr;   // ztarg(3,nt)
  int ifcharge = 0, ifdipole = 0, ifpgh = 1;
  // when set, called with the solve's stream before the strengths are first
  // read (the host entry points upload them on a second stream meanwhile)
  std::function<void(cudaStream_t)> strengths_ready;
};

struct Setup3D {
  DevTree tree;
  DevLists lists;
  DevBuf<int> isrc, isrcse, itarg, itargse;
  DevBuf<zdc> zsrcsort, ztargsort, chargesort, dipstrsort, dipvecsort;
  DevBuf<zdc> zcsrc, zctarg;  // [3*nboxes], rescaled
  double b0 = 1.0;            // boxsize(0) before rescaling
  std::vector<double> bsz;    // rescaled box sizes per level
};

// `charge_scale` / `dipvec_scale`: the factors applied to the sorted strengths
// (the Laplace driver uses b0inv and b0inv^2).
void setup3d(const Inputs3D& in, const TreeParams& tp, Setup3D& S, bool rescale_charge,
             bool rescale_dipvec, cudaStream_t s);

// the geometric part of setup3d only (tree, sort, sorted rescaled points,
// complex centres, lists); the strength arrays of S stay empty
void setup3d_geom(int ns, const zdc* zsrc, int nt, const zdc* ztarg, const TreeParams& tp,
                  Setup3D& S, cudaStream_t s);

// strengths of nd right-hand sides in tree order: charge(nd, ns) and
// dipstr(nd, ns) (right-hand side fastest) -> q[i*nd + r], ds[i*nd + r];
// dipvec(3, ns), shared by the right-hand sides -> dv[3*i + d]; the rescaling
// flags as in setup3d.  Null inputs give zeros.
void gather_strengths_nd(const Setup3D& S, int ns, int nd, const zdc* charge, const zdc* dipstr,
                         const zdc* dipvec, bool rescale_charge, bool rescale_dipvec, zdc* q,
                         zdc* ds, zdc* dv, cudaStream_t s);

// pot(nd, nt) = pscale * potsort, grad(nd, 3, nt) = gscale * gradsort, from
// tree order back to the caller's order
void unsort3d_nd(int nt, int nd, const int* itarg, const zdc* potsort, const zdc* gradsort,
                 zdc pscale, zdc gscale, int ifpgh, zdc* pot, zdc* grad, cudaStream_t s);

// right-hand side r of charge(nd, ns), dipstr(nd, ns) into tree order, as
// setup3d's strengths (q[i], ds[i], dv[3i+d]); null inputs give zeros
void gather_strengths_col(const Setup3D& S, int ns, int nd, int r, const zdc* charge,
                          const zdc* dipstr, const zdc* dipvec, bool rescale_charge,
                          bool rescale_dipvec, zdc* q, zdc* ds, zdc* dv, cudaStream_t s);

// right-hand side r of pot(nd, nt) / grad(nd, 3, nt) from one right-hand
// side's sorted potsort / gradsort
void unsort3d_col(int nt, int nd, int r, const int* itarg, const zdc* potsort,
                  const zdc* gradsort, zdc pscale, zdc gscale, int ifpgh, zdc* pot, zdc* grad,
                  cudaStream_t s);

void unsort3d(int nt, const int* itarg, const zdc* potsort, const zdc* gradsort, zdc pscale,
              zdc gscale, int ifpgh, zdc* pot, zdc* grad, cudaStream_t s);

}  // namespace zf
