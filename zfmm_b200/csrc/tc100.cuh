// Fifth-generation tensor cores of sm_100a (tcgen05) for TF32 products with
// FP32 accumulation in tensor memory, as inline PTX.
//
// Operands live in shared memory in the K-major layout without swizzle that
// the tcgen05 shared-memory descriptors describe: 8-row x 16-byte core
// matrices (8 rows x 4 TF32 values), the two K-halves of one 8-deep K step
// LBO bytes apart, successive 8-row groups SBO bytes apart:
//   byte(row, k) = (k / 8) * chunk + (row / 8) * 256 + ((k % 8) / 4) * 128
//                  + (row % 8) * 16 + (k % 4) * 4,    chunk = rows / 8 * 256
// so LBO = 128, SBO = 256 and the descriptor of K step c starts at
// base + c * chunk.  One elected thread issues the MMAs; tcgen05.commit
// arrives on an mbarrier when they are complete; every wait on it is bounded
// and reports a timeout instead of spinning forever.
//
// Accuracy: a value x is split into two TF32 parts hi = tf32(x),
// lo = tf32(x - hi) (relative error of hi + lo about 2^-22); a product A B is
// taken as Ahi Bhi + Ahi Blo + Alo Bhi (the Alo Blo term is below FP32
// rounding), accumulated in FP32.
#pragma once
#include <cstdint>

namespace zf {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of element (row, k) of a K-major operand of `rows` rows
__device__ __forceinline__ uint32_t kmajor_off(int row, int k, int rows) {
  return (uint32_t)((k >> 3) * (rows >> 3) * 256 + (row >> 3) * 256 + ((k & 7) >> 2) * 128 +
                    (row & 7) * 16 + (k & 3) * 4);
}

// shared-memory descriptor (K-major, no swizzle, sm_100 version 1)
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3fff);
  d |= (uint64_t)((lbo >> 4) & 0x3fff) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3fff) << 32;
  d |= (uint64_t)1 << 46;  // version
  return d;               // base offset 0, legacy LBO mode, layout SWIZZLE_NONE
}

// instruction descriptor: D f32, A and B tf32, both K-major, M x N
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// hi / lo TF32 parts of x
__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
  hi = to_tf32(x);
  lo = to_tf32(x - __uint_as_float(hi));
}

// ---- tensor memory ------------------------------------------------------------
// allocate `ncols` columns (a power of two >= 32); the whole warp calls it; the
// address is written to *dst (shared memory)
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(dst)),
               "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}
__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// generic-proxy shared-memory writes visible to the tensor cores
__device__ __forceinline__ void fence_smem_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// D[tmem] (+)= A[adesc] B[bdesc]^T
__device__ __forceinline__ void mma_tf32(uint32_t taddr, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(taddr),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// arrive on the mbarrier once the MMAs issued so far are complete
__device__ __forceinline__ void mma_commit(uint64_t* mbar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(mbar))
      : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count));
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// wait for phase `parity` of the mbarrier; false after `limit` polls
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, long limit) {
  uint32_t a = smem_u32(mbar);
  for (long i = 0; i < limit; i++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 16 consecutive FP32 columns of this thread's TMEM lane (lane = 32 * warp +
// lane id), starting at column `col` of the allocation at `taddr`
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, int warp, int col, float* v) {
  uint32_t a = taddr + ((uint32_t)(32 * warp) << 16) + (uint32_t)col;
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(a));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// bound of every mbarrier wait (polls): far above any MMA batch here, small
// enough that a lost arrival ends the kernel in well under a second
constexpr long kWaitLimit = 1L << 24;

}  // namespace tc
}  // namespace zf
