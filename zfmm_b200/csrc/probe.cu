// FP64 FMA throughput probe: the denominator of the FP64 roofline of the FMM
// kernels (which are FP64 CUDA-core bound).  Each thread runs 8 independent
// dependent-FMA chains, so the FP64 pipe, not latency, limits the rate.
#include "devmem.cuh"
#include "../../include/zfmm.h"

namespace zf {
namespace {

__global__ void k_fma_probe(int iters, double seed, double* out) {
  double a[8];
#pragma unroll
  for (int k = 0; k < 8; k++) a[k] = seed + threadIdx.x * 1e-9 + k;
  const double m = 0.999999999, c = 1e-12;
  for (int i = 0; i < iters; i++)
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = fma(a[k], m, c);
  double s = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) s += a[k];
  if (s == 12345.678) out[0] = s;  // keeps the chains live
}

}  // namespace
}  // namespace zf

extern "C" double zfmm_probe_fp64_tflops(int iters) {
  using namespace zf;
  try {
    cudaStream_t s = cudaStreamPerThread;
    int dev = 0, nsm = 0;
    ZF_CUDA(cudaGetDevice(&dev));
    ZF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    DevBuf<double> out(1, s);
    dim3 grid(nsm * 8), block(256);
    klaunch(k_fma_probe, grid, block, 0, s, iters, 1.0, out.get());  // warm-up
    cudaEvent_t e0, e1;
    ZF_CUDA(cudaEventCreate(&e0));
    ZF_CUDA(cudaEventCreate(&e1));
    ZF_CUDA(cudaEventRecord(e0, s));
    klaunch(k_fma_probe, grid, block, 0, s, iters, 1.0, out.get());
    ZF_CUDA(cudaEventRecord(e1, s));
    ZF_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    ZF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    double flops = 2.0 * 8.0 * iters * (double)grid.x * block.x;
    return flops / (ms * 1e-3) / 1e12;
  } catch (...) {
    return -1.0;
  }
}
