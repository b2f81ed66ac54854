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

// FP64 tensor-core (DMMA, mma.sync m8n8k4 f64) throughput: 4 independent
// accumulator tiles per warp, 8 x 8 x 4 = 256 FMA per instruction.
__global__ void k_dmma_probe(int iters, double seed, double* out) {
  double a = seed + threadIdx.x * 1e-9, b = 0.999999999;
  double c[4][2];
#pragma unroll
  for (int k = 0; k < 4; k++) c[k][0] = c[k][1] = k * 1e-3;
  for (int i = 0; i < iters; i++)
#pragma unroll
    for (int k = 0; k < 4; k++)
      asm volatile(
          "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
          : "+d"(c[k][0]), "+d"(c[k][1])
          : "d"(a), "d"(b));
  double s = 0;
#pragma unroll
  for (int k = 0; k < 4; k++) s += c[k][0] + c[k][1];
  if (s == 12345.678) out[0] = s;
}

}  // namespace
}  // namespace zf

namespace {
double time_probe(int kind, int iters) {
  using namespace zf;
  try {
    cudaStream_t s = cudaStreamPerThread;
    int dev = 0, nsm = 0;
    ZF_CUDA(cudaGetDevice(&dev));
    ZF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    DevBuf<double> out(1, s);
    dim3 grid(nsm * 8), block(256);
    auto run = [&]() {
      if (kind == 0) klaunch(k_fma_probe, grid, block, 0, s, iters, 1.0, out.get());
      else klaunch(k_dmma_probe, grid, block, 0, s, iters, 1.0, out.get());
    };
    run();  // warm-up
    cudaEvent_t e0, e1;
    ZF_CUDA(cudaEventCreate(&e0));
    ZF_CUDA(cudaEventCreate(&e1));
    ZF_CUDA(cudaEventRecord(e0, s));
    run();
    ZF_CUDA(cudaEventRecord(e1, s));
    ZF_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    ZF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    double flops = kind == 0 ? 2.0 * 8.0 * iters * (double)grid.x * block.x
                             : 2.0 * 256.0 * 4.0 * iters * (double)grid.x * (block.x / 32);
    return flops / (ms * 1e-3) / 1e12;
  } catch (...) {
    return -1.0;
  }
}
}  // namespace

extern "C" double zfmm_probe_fp64_tflops(int iters) { return time_probe(0, iters); }
extern "C" double zfmm_probe_dmma_tflops(int iters) { return time_probe(1, iters); }
