// Stream-ordered device buffers and error plumbing for the host orchestration.
//
// All scratch is taken from a library-owned stream-ordered memory pool per
// device (cudaMallocFromPoolAsync / cudaFreeAsync on the call's stream).  The
// pool keeps freed memory mapped between calls (release threshold = max), so a
// repeated solve of the same size maps no new pages; zfmm_trim_pool() returns
// the cached memory to the driver.  Errors are thrown as
// zf_error inside the library and turned into status codes at the C ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdexcept>
#include <string>
#include <utility>

namespace zf {

struct zf_error : std::runtime_error {
  int code;
  zf_error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

enum Status {
  ZF_OK = 0,
  ZF_ERR_ARG = 1,
  ZF_ERR_CUDA = 2,
  ZF_ERR_NOMEM = 3,
  ZF_ERR_INTERNAL = 4,
};

// the calling thread's current device's pool (created on first use)
cudaMemPool_t pool();

// Allocation-failure injection (zfmm_fail_alloc_after): true when this
// allocation is the one chosen to fail, which then reports
// cudaErrorMemoryAllocation without calling the allocator.
bool inject_alloc_failure();

inline cudaError_t pool_alloc(void** p, size_t bytes, cudaStream_t s) {
  if (inject_alloc_failure()) return cudaErrorMemoryAllocation;
  return cudaMallocFromPoolAsync(p, bytes, pool(), s);
}

inline void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    int code = (e == cudaErrorMemoryAllocation) ? ZF_ERR_NOMEM : ZF_ERR_CUDA;
    throw zf_error(code, std::string(what) + ": " + cudaGetErrorString(e));
  }
}
#define ZF_CUDA(x) ::zf::cuda_check((x), #x)
#define ZF_LAUNCH_CHECK() ::zf::cuda_check(cudaGetLastError(), "kernel launch")

template <class T>
class DevBuf {
 public:
  DevBuf() = default;
  DevBuf(size_t n, cudaStream_t s) { alloc(n, s); }
  ~DevBuf() { release(); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept { swap(o); }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) { release(); swap(o); }
    return *this;
  }
  void alloc(size_t n, cudaStream_t s) {
    release();
    s_ = s;
    n_ = n;
    if (n) ZF_CUDA(pool_alloc((void**)&p_, n * sizeof(T), s));
  }
  // grow to at least n elements keeping the first `keep` elements
  void grow(size_t n, size_t keep) {
    if (n <= n_) return;
    T* q = nullptr;
    ZF_CUDA(pool_alloc((void**)&q, n * sizeof(T), s_));
    if (keep && p_) ZF_CUDA(cudaMemcpyAsync(q, p_, keep * sizeof(T), cudaMemcpyDeviceToDevice, s_));
    if (p_) cudaFreeAsync(p_, s_);
    p_ = q;
    n_ = n;
  }
  void zero() {
    if (n_) ZF_CUDA(cudaMemsetAsync(p_, 0, n_ * sizeof(T), s_));
  }
  void fill_bytes(int v) {
    if (n_) ZF_CUDA(cudaMemsetAsync(p_, v, n_ * sizeof(T), s_));
  }
  void release() {
    if (p_) cudaFreeAsync(p_, s_);
    p_ = nullptr;
    n_ = 0;
  }
  void swap(DevBuf& o) noexcept {
    std::swap(p_, o.p_);
    std::swap(n_, o.n_);
    std::swap(s_, o.s_);
  }
  T* get() const { return p_; }
  size_t size() const { return n_; }
  cudaStream_t stream() const { return s_; }

 private:
  T* p_ = nullptr;
  size_t n_ = 0;
  cudaStream_t s_ = 0;
};

inline int div_up(long a, long b) { return (int)((a + b - 1) / b); }

// Kernel launches of this library go through klaunch, which counts them per
// host thread (reported as the number of kernels a call launched).
long& launch_counter();
// launches of the library by all host threads of the process
void count_launch_global();

template <typename... KArgs, typename... Args>
inline void klaunch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                    cudaStream_t s, Args&&... args) {
  if (grid.x == 0 || grid.y == 0 || grid.z == 0) return;
  kernel<<<grid, block, smem, s>>>(std::forward<Args>(args)...);
  launch_counter()++;
  count_launch_global();
}

}  // namespace zf
