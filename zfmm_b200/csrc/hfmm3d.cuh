// 3D Helmholtz FMM and direct sum entry points (device pointers).
#pragma once
#include "fmm3d_common.cuh"
#include "lfmm2d.cuh"

namespace zf {

// h3dterms (zfmm3d/src/helmholtz/h3dterms.f:16-75) on the host, cached
int h3dterms_host(double size, zdc zk, double eps, int isep);

// pot(nt), grad(3,nt) are overwritten; the 1/(4 pi) is included as in the
// reference
void zhfmm3d_device(double eps, zdc zk, const Inputs3D& in, int isep, zdc* pot, zdc* grad,
                    cudaStream_t s, StepTimes* times);

// zh3devaldirect over all pairs: ADDS the sums into pot/grad
void zh3ddirect_device(zdc zk, const Inputs3D& in, zdc* pot, zdc* grad, cudaStream_t s);

}  // namespace zf
