// Per-wavenumber set-up of the 3D Helmholtz FMM shared by the single-solve
// driver (hfmm3d.cu) and the batched plan solves (hfmm3d_nd.cu): orders per
// level (h3dterms, zfmm3d/src/helmholtz/h3dterms.f:16-75), expansion offsets,
// tables of the largest order and the quadrature z-shift configurations of
// zh3dtrans.f (Gauss-Legendre nodes and the projection weights).
#pragma once
#include <vector>
#include "fmm3d_common.cuh"
#include "lfmm2d.cuh"
#include "sph3d.cuh"

namespace zf {

constexpr int ML = 52;      // tree levels (nlmax = 51)
constexpr int PMAXR = 126;  // largest expansion order

struct HLev {
  long base[ML];
  int lo[ML];
  int p[ML];
  double rs[ML];
};

// one quadrature z-shift configuration (per kind and output level)
struct ShiftTab {
  int p1, p2, nq;
  double r, rs1;
  const double* x;  // nq Gauss-Legendre nodes
  const double* w;  // nq weights
  const zdc* cF;    // g_n / ((g_n^2 + g_n'^2) / 2 pi), n <= p2
  const zdc* cD;    // g_n' / (...)
};

__device__ __forceinline__ int jdx(int n, int m) { return n * (n + 1) / 2 + m; }

// per-wavenumber state of a solve: orders per level, expansion offsets,
// tables of the largest order, quadrature z-shift configurations (device
// array dst and its host copy sth, indexed kind * ML + output level)
struct HelmPrep {
  HLev lev;
  int pmax = 0;
  long tot = 0;
  Tab3 T;
  zdc kw;
  DevBuf<double> dxw;
  DevBuf<zdc> dcfd;
  DevBuf<ShiftTab> dst;
  std::vector<ShiftTab> sth;
};

void helm_prep(const Setup3D& S, double eps, zdc zk, int isep, HelmPrep& H, cudaStream_t s);

// P2M through L2T/M2T/P2P of one right-hand side (sorted strengths) on a
// set-up and its wavenumber tables: writes potsort / gradsort (zeroed by the
// caller); ev[2..5] (optional) get the step boundaries
void helm_core(const Setup3D& S, const HelmPrep& H, const zdc* q, const zdc* ds, const zdc* dv,
               int ifcharge, int ifdipole, int ifpgh, zdc* potsort, zdc* gradsort,
               cudaStream_t s, cudaEvent_t* ev);

// the passes separately: P2M into out (local = false; out zeroed by the caller)
// or P2L added into out (local = true), single-right-hand-side layout
void helm_form(const Setup3D& S, const HelmPrep& H, const zdc* q, const zdc* ds, const zdc* dv,
               int ifcharge, int ifdipole, bool local, zdc* out, cudaStream_t s);
// P2P, L2T and M2T of one right-hand side into potsort / gradsort
void helm_eval(const Setup3D& S, const HelmPrep& H, const zdc* q, const zdc* ds, const zdc* dv,
               int ifcharge, int ifdipole, int ifpgh, const zdc* mp, const zdc* loc,
               zdc* potsort, zdc* gradsort, cudaStream_t s);

struct Plan3D;
struct StrengthsNd;
// a plan solve with every right-hand side through the single-solve passes on
// the plan's tree (helm_core), with a prepared wavenumber; prep_ms is added
// to the set-up time reported in times
void helm_plan_loop(const Plan3D& P, const HelmPrep& H, int nd, const StrengthsNd& in, int ifpgh,
                    zdc* pot, zdc* grad, cudaStream_t s, StepTimes* times, float prep_ms);

}  // namespace zf
