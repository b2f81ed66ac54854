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

// zh2devaldirect over all pairs: ADDS the unscaled sums (no i/4) into pot/grad
void zh2ddirect_device(zdc zk, const Inputs2D& in, zdc* pot, zdc* grad, cudaStream_t s);

}  // namespace zf
