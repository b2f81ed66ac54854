// 3D Laplace FMM and direct sum entry points (device pointers).
#pragma once
#include "fmm3d_common.cuh"
#include "lfmm2d.cuh"

namespace zf {

// zl3dterms (zfmm3d/src/laplace/zlfmm3d.f:1283-1321)
int zl3dterms(double eps);
// lndiv (zfmm3d/src/common/lndiv_fast.f:17-35)
int lndiv3d(double eps, int ns, int nt);

// pot(nt), grad(3,nt) are overwritten; the 1/(4 pi) is included as in the
// reference.  `times` as in the 2D drivers (counts[] of the 3D passes).
void zlfmm3d_device(double eps, const Inputs3D& in, int isep, zdc* pot, zdc* grad,
                    cudaStream_t s, StepTimes* times);

// the passes of zlfmm3d after the set-up, for one right-hand side with sorted,
// rescaled strengths (q, ds: ns; dv: 3 ns) on a set-up S: ADDS the sorted,
// unscaled potentials / gradients to potsort / gradsort; ev (optional, 8
// events) gets the step boundaries 2..5 recorded; returns the order
int lap_core(const Setup3D& S, double eps, const zdc* q, const zdc* ds, const zdc* dv,
             int ifcharge, int ifdipole, int ifpgh, zdc* potsort, zdc* gradsort, cudaStream_t s,
             cudaEvent_t* ev);

// interaction counts of a 3D FMM on this set-up, totals and per level, into
// times (counts, lvl_counts, lvl_p); p2m_lmin / m2m_lmin / l2l_lmin: the
// coarsest level with P2M leaves / M2M parents / L2L children
void count_interactions3d(const Setup3D& S, const int* p_per_level, int p2m_lmin, int m2m_lmin,
                          int l2l_lmin, StepTimes* times, cudaStream_t s);

// zl3devaldirect over all pairs: ADDS the sums (with 1/(4 pi)) into pot/grad
void zl3ddirect_device(const Inputs3D& in, zdc* pot, zdc* grad, cudaStream_t s);

}  // namespace zf
