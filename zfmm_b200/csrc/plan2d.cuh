// A 2D plan: the geometry of a complex-coordinate 2D FMM (quadtree on the real
// parts, sorted points, complex box centres, interaction lists) built once and
// reused by any number of solves, right-hand sides and wavenumbers.  The tree
// depends on eps, ns, nt, isep and the points only (lndiv2d / hndiv2d share
// their table), so one plan serves zlfmm2d and zhfmm2d at any zk: the
// two-wavenumber matvecs of a transmission-problem GMRES reuse one tree.
#pragma once
#include "fmm2d_common.cuh"
#include "lfmm2d.cuh"

namespace zf {

struct Plan2D {
  double eps = 0;
  int isep = 1, ns = 0, nt = 0, device = 0;
  Setup2D S;
};

// zsrc(2, ns), ztarg(2, nt) on the device
void plan2d_build(Plan2D& P, double eps, int ns, const zdc* zsrc, int nt, const zdc* ztarg,
                  int isep, cudaStream_t s);

// the plan's geometry to / from a plan file (plan_io.cu); load builds the
// device arrays on the current device
void plan2d_save(const Plan2D& P, const char* path, cudaStream_t s);
void plan2d_load(Plan2D& P, const char* path, cudaStream_t s);

// nd right-hand sides: charge(nd, ns), dipstr(nd, ns) (right-hand side fastest),
// dipvec(2, ns) shared; pot(nd, nt), grad(nd, 2, nt) overwritten, scaled as
// the reference (1/(2 pi) Laplace, i/4 Helmholtz).  zk == nullptr: Laplace.
void fmm2d_plan_execute(const Plan2D& P, const zdc* zk, int nd, int ifcharge, const zdc* charge,
                        int ifdipole, const zdc* dipstr, const zdc* dipvec, int ifpgh,
                        zdc* pot, zdc* grad, cudaStream_t s, StepTimes* times);

}  // namespace zf
