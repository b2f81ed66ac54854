// 2D Helmholtz FMM entry points (device pointers).
#pragma once
#include <memory>
#include <vector>
#include "fmm2d_common.cuh"
#include "lfmm2d.cuh"

namespace zf {

// h2dterms (zfmm2d/src/helmholtz/h2dterms.f:35-97) on the host
int h2dterms_host(double bsize, zdc zk, double eps, int isep);

// pot(nt), grad(2,nt) are overwritten; results carry the reference's i/4 factor
void zhfmm2d_device(double eps, zdc zk, const Inputs2D& in, int isep, zdc* pot, zdc* grad,
                    cudaStream_t s, StepTimes* times);

// the passes of zhfmm2d after the set-up, as lap2d_core (orders from
// h2dterms for zk on the set-up's tree)
int helm2d_core(const Setup2D& S, double eps, zdc zk, int isep, const zdc* q, const zdc* ds,
                const zdc* dv, int ifcharge, int ifdipole, int ifpgh, zdc* potsort,
                zdc* gradsort, cudaStream_t s, cudaEvent_t* ev, std::vector<int>* pl);

// Orders, scales and translation tables of the 2D Helmholtz passes for one
// set-up and wavenumber (they do not depend on the strengths): built once and
// used by any number of helm2d_passes calls on that set-up.
struct Helm2DPrep;
struct Helm2DPrepDeleter {
  void operator()(Helm2DPrep* p) const;
};
using Helm2DPrepPtr = std::unique_ptr<Helm2DPrep, Helm2DPrepDeleter>;
Helm2DPrepPtr helm2d_prepare(const Setup2D& S, double eps, zdc zk, int isep, cudaStream_t s);

// the passes of helm2d_core on prepared tables
int helm2d_passes(const Setup2D& S, const Helm2DPrep& H, const zdc* q, const zdc* ds,
                  const zdc* dv, int ifcharge, int ifdipole, int ifpgh, zdc* potsort,
                  zdc* gradsort, cudaStream_t s, cudaEvent_t* ev, std::vector<int>* pl);

// nd right-hand sides on one prepared tree: charge, dipstr (nd, ns) with the
// right-hand side fastest, dipvec (2, ns) shared; pot (nd, nt), grad (nd, 2, nt)
// overwritten with the i/4 scaling.  The M2L of levels with 2(2p+1) <= 128 runs
// on the tcgen05 tensor cores (TF32 three-term split) when use_tc; ms3
// (optional) receives the device times of the upward passes, the M2L and the
// downward passes.
void helm2d_passes_nd(const Setup2D& S, const Helm2DPrep& H, int nd, int ifcharge,
                      const zdc* charge, int ifdipole, const zdc* dipstr, const zdc* dipvec,
                      int ifpgh, bool use_tc, zdc* pot, zdc* grad, cudaStream_t s, float* ms3);

// zh2devaldirect over all pairs: ADDS the unscaled sums (no i/4) into pot/grad
void zh2ddirect_device(zdc zk, const Inputs2D& in, zdc* pot, zdc* grad, cudaStream_t s);

}  // namespace zf
