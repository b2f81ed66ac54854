// 2D Laplace FMM and direct sum entry points (device pointers).
#pragma once
#include "fmm2d_common.cuh"

namespace zf {

struct StepTimes {
  // 0 set-up (tree, sort, lists, centres), 1 P2M, 2 M2M, 3 M2L+P2L,
  // 4 L2L, 5 P2P+M2T+L2T, 6 unsort
  float ms[8] = {0};
  int nboxes = 0, nlevels = 0, nterms = 0;
  // interaction counts of the call: 0 P2P pairs, 1 M2T (target, box), 2 L2T
  // targets, 3 M2L box pairs, 4 P2L (box, source), 5 M2M pairs, 6 L2L pairs,
  // 7 P2M sources
  unsigned long long counts[16] = {0};  // [8..15]: weighted by P (see count_interactions2d)
  long launches = 0;  // kernels of this library launched by the call
  bool want_counts = false;  // also count interactions (extra kernel + sync)
  // 3D drivers: the counts above per level (see count_interactions3d) and the
  // expansion order of each level
  unsigned long long lvl_counts[8][64] = {};
  int lvl_p[64] = {};
};

int l2dterms(double eps);
void lndiv2d(double eps, int ns, int nt, int* ndiv, int* idivflag);

// pot(nt), grad(2,nt) are overwritten (the reference zeroes them first)
void zlfmm2d_device(double eps, const Inputs2D& in, int isep, zdc* pot, zdc* grad,
                    cudaStream_t s, StepTimes* times);

// the passes of zlfmm2d after the set-up for one right-hand side with sorted
// strengths q, ds, dv(2 ns) on set-up S: writes the sorted, unscaled
// potentials / gradients into potsort / gradsort (zeroed by the caller); ev
// (optional, 8 events) gets the step boundaries 2..5; *pl (optional) the
// order of every level; returns the order
int lap2d_core(const Setup2D& S, double eps, const zdc* q, const zdc* ds, const zdc* dv,
               int ifcharge, int ifdipole, int ifpgh, zdc* potsort, zdc* gradsort,
               cudaStream_t s, cudaEvent_t* ev, std::vector<int>* pl);

// zl2devaldirect over all pairs: ADDS the unscaled sums into pot/grad, as the
// reference routine does.  `scratch` may be null (the routine then takes its
// own pool memory) or point to at least direct2d_scratch_elems(nt, ifpgh)
// complex elements.
size_t direct2d_scratch_elems(int nt, int ns, int ifpgh);
void zl2ddirect_device(const Inputs2D& in, zdc* pot, zdc* grad, zdc* scratch, cudaStream_t s);

// Same sum with its scratch in a fixed device array of the library (no device
// allocation); throws when the problem needs more than that array holds.
size_t direct2d_noalloc_capacity();
void zl2ddirect_device_noalloc(const Inputs2D& in, zdc* pot, zdc* grad, cudaStream_t s);

}  // namespace zf
