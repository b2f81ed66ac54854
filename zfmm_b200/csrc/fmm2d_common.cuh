// Shared set-up of the 2D complex-coordinate FMMs (zlfmm2d / zhfmm2d):
// real parts -> device tree -> sort -> reorder -> complex box centres.
//
// Reference: zfmm2d/src/laplace/zlfmm2d.f:70-200 (identical steps in
// zfmm2d/src/helmholtz/zhfmm2d.f:73-195).  The complex centre of a box is its
// real geometric centre plus i times the mean of the imaginary parts of the
// box's sources (resp. targets), computed for every box.
#pragma once
#include <functional>
#include <vector>
#include "tree.cuh"
#include "zcomplex.cuh"

namespace zf {

// Inputs as given by the caller, on the device, Fortran layout:
// zsrc(2,ns), charge(ns), dipstr(ns), dipvec(2,ns), ztarg(2,nt).
struct Inputs2D {
  int ns = 0, nt = 0;
  const zdc* zsrc = nullptr;
  const zdc* charge = nullptr;
  const zdc* dipstr = nullptr;
  const zdc* dipvec = nullptr;
  const zdc* ztarg = nullptr;
  int ifcharge = 0, ifdipole = 0, ifpgh = 1;
  // when set, called with the solve's stream before the strengths are first
  // read (the host entry points upload them on a second stream meanwhile)
  std::function<void(cudaStream_t)> strengths_ready;
};

struct Setup2D {
  DevTree tree;
  DevLists lists;
  DevBuf<int> isrc, isrcse, itarg, itargse;
  DevBuf<zdc> zsrcsort, ztargsort, chargesort, dipstrsort, dipvecsort;
  DevBuf<zdc> zcsrc, zctarg;  // [2*nboxes]
};

// builds everything above for the given tree parameters (ndiv, idivflag, isep)
void setup2d(const Inputs2D& in, const TreeParams& tp, Setup2D& S, cudaStream_t s);

// the geometric part of setup2d only (tree, sort, sorted points, complex
// centres, lists); the strength arrays of S stay empty
void setup2d_geom(int ns, const zdc* zsrc, int nt, const zdc* ztarg, const TreeParams& tp,
                  Setup2D& S, cudaStream_t s);

// right-hand side r of charge(nd, ns), dipstr(nd, ns) (right-hand side fastest)
// and the shared dipvec(2, ns) into tree order; null inputs give zeros
void gather2d_col(const Setup2D& S, int ns, int nd, int r, const zdc* charge, const zdc* dipstr,
                  const zdc* dipvec, zdc* q, zdc* ds, zdc* dv, cudaStream_t s);

// right-hand side r of pot(nd, nt) / grad(nd, 2, nt) from sorted potsort /
// gradsort, times `scale`
void unsort2d_col(int nt, int nd, int r, const int* itarg, const zdc* potsort,
                  const zdc* gradsort, zdc scale, int ifpgh, zdc* pot, zdc* grad,
                  cudaStream_t s);

// interaction counts of the FMM on this tree (host array of 16): [P2P pairs,
// M2T (target, box), L2T targets, M2L box pairs, P2L (box, source), M2M pairs,
// L2L pairs, P2M sources], then the same weighted by the expansion lengths
// P = 2p+1 of their levels (M2L by P^2, M2M/L2L by P_parent P_child)
void count_interactions2d(const Setup2D& S, const int* p_per_level, unsigned long long* counts,
                          cudaStream_t s);

// potsort/gradsort (sorted order) -> pot/grad (user order), times `scale`
void unsort2d(int nt, const int* itarg, const zdc* potsort, const zdc* gradsort, zdc scale,
              int ifpgh, zdc* pot, zdc* grad, cudaStream_t s);

}  // namespace zf
