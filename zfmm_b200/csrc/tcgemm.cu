// Self-test of the tcgen05 TF32 three-term product (tc100.cuh): one CTA forms
// D = A B^T for A (128 x K) and B (N x K), FP32 in global memory, through the
// same shared-memory layout, descriptors, MMA sequence, commit / bounded wait
// and tensor-memory read-back that the batched translations use.  It lets a
// test check the building block against an FP64 product on the device the
// library runs on.
#include "../../include/zfmm.h"
#include "devmem.cuh"
#include "tc100.cuh"

namespace zf {
namespace {

__global__ void __launch_bounds__(128) k_tc_selftest(const float* __restrict__ A,
                                                     const float* __restrict__ B, float* D, int N,
                                                     int K, int* err) {
  extern __shared__ __align__(1024) uint32_t tsm[];
  __shared__ uint64_t mbar;
  __shared__ uint32_t taddr_s;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  uint32_t* ah = tsm;
  uint32_t* al = ah + 128 * K;
  uint32_t* bh = al + 128 * K;
  uint32_t* bl = bh + N * K;
  for (int i = tid; i < 128 * K; i += 128) {
    int r = i / K, k = i - r * K;
    uint32_t h, l;
    tc::split_tf32(A[i], h, l);
    uint32_t o = tc::kmajor_off(r, k, 128) >> 2;
    ah[o] = h;
    al[o] = l;
  }
  for (int i = tid; i < N * K; i += 128) {
    int r = i / K, k = i - r * K;
    uint32_t h, l;
    tc::split_tf32(B[i], h, l);
    uint32_t o = tc::kmajor_off(r, k, N) >> 2;
    bh[o] = h;
    bl[o] = l;
  }
  const uint32_t ncols = N <= 32 ? 32 : (N <= 64 ? 64 : (N <= 128 ? 128 : 256));
  if (warp == 0) tc::tmem_alloc(&taddr_s, ncols);
  if (tid == 0) tc::mbar_init(&mbar, 1);
  tc::fence_smem_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t taddr = taddr_s;
  if (tid == 0) {
    const uint32_t idesc = tc::idesc_tf32(128, N);
    const uint32_t achunk = 128 / 8 * 256, bchunk = (uint32_t)N / 8 * 256;
    for (int c = 0; c < K / 8; c++) {
      uint64_t dah = tc::make_desc(tc::smem_u32(ah) + c * achunk, 128, 256);
      uint64_t dal = tc::make_desc(tc::smem_u32(al) + c * achunk, 128, 256);
      uint64_t dbh = tc::make_desc(tc::smem_u32(bh) + c * bchunk, 128, 256);
      uint64_t dbl = tc::make_desc(tc::smem_u32(bl) + c * bchunk, 128, 256);
      tc::mma_tf32(taddr, dal, dbh, idesc, c > 0);
      tc::mma_tf32(taddr, dah, dbl, idesc, 1);
      tc::mma_tf32(taddr, dah, dbh, idesc, 1);
    }
    tc::mma_commit(&mbar);
  }
  bool ok = tc::mbar_wait(&mbar, 0, tc::kWaitLimit);
  ok = __all_sync(0xffffffffu, ok);
  if (!ok && lane == 0) atomicExch(err, 1);
  tc::fence_after_sync();
  if (ok) {
    for (int c0 = 0; c0 < N; c0 += 16) {
      float v[16];
      tc::tmem_ld16(taddr, warp, c0, v);
      float* d = D + (size_t)(32 * warp + lane) * N + c0;
#pragma unroll
      for (int i = 0; i < 16; i++) d[i] = v[i];
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(taddr, ncols);
}

}  // namespace
}  // namespace zf

using namespace zf;

extern "C" int zfmm_tc_selftest(int N, int K, const float* A, const float* B, float* D,
                                void* stream) {
  if (N < 16 || N > 256 || N % 16 || K < 8 || K > 128 || K % 8 || !A || !B || !D) return 1;
  size_t sm = (size_t)2 * (128 + N) * K * sizeof(uint32_t);
  if (sm > 200 * 1024) return 1;
  try {
    cudaStream_t s = (cudaStream_t)stream;
    DevBuf<int> err(1, s);
    err.zero();
    ZF_CUDA(cudaFuncSetAttribute(k_tc_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sm));
    klaunch(k_tc_selftest, 1, 128, sm, s, A, B, D, N, K, err.get());
    ZF_LAUNCH_CHECK();
    int h = 0;
    ZF_CUDA(cudaMemcpyAsync(&h, err.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    ZF_CUDA(cudaStreamSynchronize(s));
    return h ? 4 : 0;
  } catch (const zf_error& e) {
    return e.code;
  }
}
