// A 3D plan: the geometry of a complex-coordinate FMM (octree on the real
// parts, sorted and rescaled points, complex box centres, interaction lists)
// built once and reused by any number of solves with new strengths, many
// right-hand sides per solve.  The tree depends on eps, ns, nt and the points
// only (lndiv, zfmm3d/src/common/lndiv_fast.f:17-35; the Helmholtz driver uses
// the same table, hndiv_fast.f), so one plan serves both kernels and any
// wavenumber.
#pragma once
#include "fmm3d_common.cuh"
#include "lfmm2d.cuh"

namespace zf {

struct Plan3D {
  double eps = 0;
  int isep = 1, ns = 0, nt = 0, device = 0;
  Setup3D S;
};

// strengths of nd right-hand sides (device pointers): charge(nd, ns),
// dipstr(nd, ns) with the right-hand side fastest, dipvec(3, ns) shared
struct StrengthsNd {
  int ifcharge = 0, ifdipole = 0;
  const zdc* charge = nullptr;
  const zdc* dipstr = nullptr;
  const zdc* dipvec = nullptr;
};

// zsrc(3, ns), ztarg(3, nt) on the device
void plan3d_build(Plan3D& P, double eps, int ns, const zdc* zsrc, int nt, const zdc* ztarg,
                  int isep, cudaStream_t s);

// the plan's geometry to / from a plan file (plan_io.cu); load builds the
// device arrays on the current device
void plan3d_save(const Plan3D& P, const char* path, cudaStream_t s);
void plan3d_load(Plan3D& P, const char* path, cudaStream_t s);

// pot(nd, nt) and grad(nd, 3, nt) (device) are overwritten; scaling as zlfmm3d
void zlfmm3d_plan_execute(const Plan3D& P, int nd, const StrengthsNd& in, int ifpgh, zdc* pot,
                          zdc* grad, cudaStream_t s, StepTimes* times);

// 3D Helmholtz with wavenumber zk on the plan's points: the orders, tables
// and shift configurations of zk are built once per call; 4 or more
// right-hand sides run the batched kernels (hfmm3d_nd.cu), fewer the
// single-solve passes per right-hand side on the plan's tree; same layouts as
// zlfmm3d_plan_execute, scaling as zhfmm3d
void zhfmm3d_plan_execute(const Plan3D& P, zdc zk, int nd, const StrengthsNd& in, int ifpgh,
                          zdc* pot, zdc* grad, cudaStream_t s, StepTimes* times);

}  // namespace zf
