// extern "C" entry points (include/zfmm.h).
//
// Host-array entry points copy the caller's arrays to the device on the
// per-thread default stream, run the device path and copy pot/grad back, so
// they are synchronous and reentrant across host threads.  Exceptions never
// cross the ABI: they become status codes plus a thread-local message.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <exception>
#include <initializer_list>
#include <thread>
#include <mutex>
#include <string>
#include <vector>
#include "../../include/zfmm.h"
#include "hfmm2d.cuh"
#include "lfmm2d.cuh"
#include "lfmm3d.cuh"
#include "hfmm3d.cuh"
#include "plan2d.cuh"
#include "plan3d.cuh"

using namespace zf;

namespace zf {
long& launch_counter() {
  static thread_local long n = 0;
  return n;
}

namespace {
std::atomic<long> g_launch_total{0};
}
void count_launch_global() { g_launch_total.fetch_add(1, std::memory_order_relaxed); }

namespace {
constexpr int kMaxDev = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pools[kMaxDev] = {};
}  // namespace

std::atomic<long> g_fail_after{-1};  // allocations left before the injected failure

bool inject_alloc_failure() {
  long v = g_fail_after.load(std::memory_order_relaxed);
  while (v >= 0)  // count down; the allocation that finds 0 fails and ends it
    if (g_fail_after.compare_exchange_weak(v, v == 0 ? -1 : v - 1)) return v == 0;
  return false;
}

cudaMemPool_t pool() {
  int dev = 0;
  ZF_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDev) throw zf_error(ZF_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (!g_pools[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p;
    ZF_CUDA(cudaMemPoolCreate(&p, &props));
    unsigned long long keep = ~0ull;
    ZF_CUDA(cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep));
    g_pools[dev] = p;
  }
  return g_pools[dev];
}
}  // namespace zf

namespace {

thread_local std::string g_err;
thread_local int g_timing = 0;
thread_local StepTimes g_times;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

template <class F>
int guarded(F&& f) {
  g_err.clear();
  try {
    f();
    return ZF_OK;
  } catch (const zf_error& e) {
    return fail(e.code, e.what());
  } catch (const std::bad_alloc&) {
    return fail(ZF_ERR_NOMEM, "host allocation failed");
  } catch (const std::exception& e) {
    return fail(ZF_ERR_INTERNAL, e.what());
  }
}

void clamp_flags(int& ifcharge, int& ifdipole, int& ifpgh) {
  // zlfmm2d.f:58-68
  if (ifcharge < 0 || ifcharge > 1) ifcharge = 1;
  if (ifdipole < 0 || ifdipole > 1) ifdipole = 0;
  if (ifpgh < 0 || ifpgh > 2) ifpgh = 1;
}

void check_device() {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) throw zf_error(5, "no CUDA device available");
}

struct HostIn {
  DevBuf<zdc> zsrc, charge, dipstr, dipvec, ztarg;
};

void upload(DevBuf<zdc>& b, const double* h, size_t nz, cudaStream_t s) {
  b.alloc(nz, s);
  if (nz) ZF_CUDA(cudaMemcpyAsync(b.get(), h, nz * sizeof(zdc), cudaMemcpyHostToDevice, s));
}

bool page_locked(const void* p) {
  cudaPointerAttributes a{};
  return p && cudaPointerGetAttributes(&a, p) == cudaSuccess && a.type == cudaMemoryTypeHost;
}

// The strengths (charges, dipole strengths, dipole vectors) of a host-array
// FMM call, uploaded on a second stream while the solve's stream uploads the
// points and builds the tree, which needs only the points.  Page-locked
// arrays are copied asynchronously; pageable ones from a helper thread (a
// pageable copy holds its calling thread until the data is staged).  The
// device buffers are allocated on the solve's stream, which also frees them.
// ready(s) makes the solve's stream wait for the copies (the set-up calls it
// before it gathers the strengths); the destructor waits for them in any case.
class StrengthUpload {
 public:
  StrengthUpload(HostIn& h, int ns, int dim, int ifcharge, const double* charge, int ifdipole,
                 const double* dipstr, const double* dipvec, cudaStream_t s) {
    if (ifcharge == 1) h.charge.alloc(ns, s);  // may throw: nothing created yet
    if (ifdipole == 1) {
      h.dipstr.alloc(ns, s);
      h.dipvec.alloc((size_t)dim * ns, s);
    }
    ZF_CUDA(cudaStreamCreateWithFlags(&aux_, cudaStreamNonBlocking));
    if (cudaEventCreateWithFlags(&ev_, cudaEventDisableTiming) != cudaSuccess) {
      cudaStreamDestroy(aux_);
      throw zf_error(ZF_ERR_CUDA, "cudaEventCreateWithFlags failed");
    }
    ZF_CUDA(cudaEventRecord(ev_, s));  // the buffers exist from here on
    ZF_CUDA(cudaStreamWaitEvent(aux_, ev_, 0));
    struct Copy {
      void* d;
      const void* h;
      size_t bytes;
    };
    std::vector<Copy> copies;
    if (ifcharge == 1) copies.push_back({h.charge.get(), charge, ns * sizeof(zdc)});
    if (ifdipole == 1) {
      copies.push_back({h.dipstr.get(), dipstr, ns * sizeof(zdc)});
      copies.push_back({h.dipvec.get(), dipvec, (size_t)dim * ns * sizeof(zdc)});
    }
    bool pinned = true;
    for (auto& c : copies) pinned = pinned && page_locked(c.h);
    cudaStream_t aux = aux_;
    cudaEvent_t ev = ev_;
    auto run = [copies, aux, ev]() {
      for (auto& c : copies)
        if (c.bytes) ZF_CUDA(cudaMemcpyAsync(c.d, c.h, c.bytes, cudaMemcpyHostToDevice, aux));
      ZF_CUDA(cudaEventRecord(ev, aux));
    };
    if (pinned) {
      run();
    } else {
      int dev = 0;
      ZF_CUDA(cudaGetDevice(&dev));
      th_ = std::thread([this, run, dev]() {
        try {
          ZF_CUDA(cudaSetDevice(dev));
          run();
        } catch (...) {
          err_ = std::current_exception();
        }
      });
    }
  }
  void ready(cudaStream_t s) {
    if (th_.joinable()) th_.join();
    if (err_) std::rethrow_exception(err_);
    ZF_CUDA(cudaStreamWaitEvent(s, ev_, 0));
  }
  ~StrengthUpload() {
    if (th_.joinable()) th_.join();
    cudaStreamSynchronize(aux_);
    cudaEventDestroy(ev_);
    cudaStreamDestroy(aux_);
  }
  StrengthUpload(const StrengthUpload&) = delete;
  StrengthUpload& operator=(const StrengthUpload&) = delete;

 private:
  cudaStream_t aux_ = nullptr;
  cudaEvent_t ev_ = nullptr;
  std::thread th_;
  std::exception_ptr err_;
};

Inputs2D make_inputs(int ns, const double* zsrc, int ifcharge, const double* charge,
                     int ifdipole, const double* dipstr, const double* dipvec, int nt,
                     const double* ztarg, int ifpgh) {
  Inputs2D in;
  in.ns = ns;
  in.nt = nt;
  in.zsrc = reinterpret_cast<const zdc*>(zsrc);
  in.charge = reinterpret_cast<const zdc*>(charge);
  in.dipstr = reinterpret_cast<const zdc*>(dipstr);
  in.dipvec = reinterpret_cast<const zdc*>(dipvec);
  in.ztarg = reinterpret_cast<const zdc*>(ztarg);
  in.ifcharge = ifcharge;
  in.ifdipole = ifdipole;
  in.ifpgh = ifpgh;
  return in;
}

void check_args2d(int ns, int nt, const double* zsrc, const double* ztarg, int ifcharge,
                  const double* charge, int ifdipole, const double* dipstr,
                  const double* dipvec, double* pot, double* grad, int ifpgh) {
  if (ns < 0 || nt < 0) throw zf_error(ZF_ERR_ARG, "ns and nt must be >= 0");
  if ((ns > 0 && !zsrc) || (nt > 0 && (!ztarg || !pot)))
    throw zf_error(ZF_ERR_ARG, "null coordinate or output array");
  if (ns > 0 && ifcharge == 1 && !charge) throw zf_error(ZF_ERR_ARG, "ifcharge=1 needs charge");
  if (ns > 0 && ifdipole == 1 && (!dipstr || !dipvec))
    throw zf_error(ZF_ERR_ARG, "ifdipole=1 needs dipstr and dipvec");
  if (nt > 0 && ifpgh > 1 && !grad) throw zf_error(ZF_ERR_ARG, "ifpgh=2 needs grad");
}

// Device arrays are read and written with 16-byte (double2) accesses: a
// pointer that is not 16-byte aligned is refused here, before any launch,
// instead of faulting the kernel.  Arrays a call does not use (flag off) are
// not checked.
void check_align16(std::initializer_list<const void*> ptrs) {
  for (const void* p : ptrs)
    if (p && (reinterpret_cast<uintptr_t>(p) & 15))
      throw zf_error(ZF_ERR_ARG, "device arrays must be 16-byte aligned");
}

void check_align_dev(const double* zsrc, const double* ztarg, int ifcharge, const double* charge,
                     int ifdipole, const double* dipstr, const double* dipvec, double* pot,
                     double* grad, int ifpgh) {
  check_align16({zsrc, ztarg, pot, ifcharge == 1 ? charge : nullptr,
                 ifdipole == 1 ? dipstr : nullptr, ifdipole == 1 ? dipvec : nullptr,
                 ifpgh > 1 ? grad : nullptr});
}

// device path shared by host and device entry points; zk == nullptr selects
// the Laplace FMM, otherwise Helmholtz with wavenumber *zk
void run_fmm2d(double eps, const zdc* zk, const Inputs2D& in, int isep, zdc* pot, zdc* grad,
               cudaStream_t s) {
  if (in.nt > 0) {
    ZF_CUDA(cudaMemsetAsync(pot, 0, sizeof(zdc) * in.nt, s));
    if (grad) ZF_CUDA(cudaMemsetAsync(grad, 0, sizeof(zdc) * 2 * in.nt, s));
  }
  if (in.ns == 0 || in.nt == 0) return;
  if (isep < 1) throw zf_error(ZF_ERR_ARG, "isep must be >= 1");
  StepTimes t;
  t.want_counts = g_timing >= 2;
  if (zk) zhfmm2d_device(eps, *zk, in, isep, pot, grad, s, g_timing ? &t : nullptr);
  else zlfmm2d_device(eps, in, isep, pot, grad, s, g_timing ? &t : nullptr);
  if (g_timing) g_times = t;
}

int fmm2d_host(double eps, const zdc* zk, int ns, const double* zsrc, int ifcharge,
               const double* charge, int ifdipole, const double* dipstr, const double* dipvec,
               double* pot, double* grad, int nt, const double* ztarg, int ifpgh, int isep) {
  return guarded([&] {
    clamp_flags(ifcharge, ifdipole, ifpgh);
    check_args2d(ns, nt, zsrc, ztarg, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad,
                 ifpgh);
    check_device();
    cudaStream_t s = cudaStreamPerThread;
    HostIn h;
    // targets passed as the source array itself: uploaded once
    const bool same = ztarg == zsrc && nt == ns;
    upload(h.zsrc, zsrc, 2 * (size_t)ns, s);
    if (!same) upload(h.ztarg, ztarg, 2 * (size_t)nt, s);
    StrengthUpload su(h, ns, 2, ifcharge, charge, ifdipole, dipstr, dipvec, s);
    DevBuf<zdc> dpot(nt, s), dgrad(ifpgh > 1 ? 2 * (size_t)nt : 0, s);
    Inputs2D in = make_inputs(ns, (const double*)h.zsrc.get(), ifcharge,
                              (const double*)h.charge.get(), ifdipole,
                              (const double*)h.dipstr.get(), (const double*)h.dipvec.get(), nt,
                              (const double*)(same ? h.zsrc.get() : h.ztarg.get()), ifpgh);
    in.strengths_ready = [&su](cudaStream_t ss) { su.ready(ss); };
    run_fmm2d(eps, zk, in, isep, dpot.get(), ifpgh > 1 ? dgrad.get() : nullptr, s);
    if (nt > 0) {
      ZF_CUDA(cudaMemcpyAsync(pot, dpot.get(), sizeof(zdc) * nt, cudaMemcpyDeviceToHost, s));
      if (grad) {
        if (ifpgh > 1)
          ZF_CUDA(cudaMemcpyAsync(grad, dgrad.get(), sizeof(zdc) * 2 * nt, cudaMemcpyDeviceToHost, s));
        else
          memset(grad, 0, sizeof(zdc) * 2 * nt);
      }
    }
    ZF_CUDA(cudaStreamSynchronize(s));
  });
}

}  // namespace

extern "C" {

const char* zfmm_last_error(void) { return g_err.c_str(); }
void zfmm_fail_alloc_after(long n) { g_fail_after.store(n < 0 ? -1 : n); }
const char* zfmm_version(void) { return "zfmm_b200 0.1 (sm_100a)"; }
void zfmm_set_step_timing(int on) { g_timing = on; }

int zfmm_last_step_times(double* ms7, int* nboxes, int* nlevels, int* nterms) {
  for (int i = 0; i < 7; i++) ms7[i] = g_times.ms[i];
  if (nboxes) *nboxes = g_times.nboxes;
  if (nlevels) *nlevels = g_times.nlevels;
  if (nterms) *nterms = g_times.nterms;
  return 0;
}

int zfmm_last_counts(long long* counts16, long* launches) {
  for (int i = 0; i < 16; i++) counts16[i] = (long long)g_times.counts[i];
  if (launches) *launches = g_times.launches;
  return 0;
}

long zfmm_launch_count(void) { return g_launch_total.load(); }

int zfmm_last_level_counts(long long* counts8x64, int* orders64, int* nlevels) {
  for (int k = 0; k < 8; k++)
    for (int l = 0; l < 64; l++) counts8x64[k * 64 + l] = (long long)g_times.lvl_counts[k][l];
  for (int l = 0; l < 64; l++) orders64[l] = g_times.lvl_p[l];
  if (nlevels) *nlevels = g_times.nlevels;
  return 0;
}

int zfmm_trim_pool(void) {
  return guarded([&] {
    check_device();
    ZF_CUDA(cudaDeviceSynchronize());
    ZF_CUDA(cudaMemPoolTrimTo(pool(), 0));
  });
}

int zfmm_h2dterms(double bsize, const double* zk, double eps, int isep) {
  if (!zk) return -1;
  try {
    return h2dterms_host(bsize, mkz(zk[0], zk[1]), eps, isep);
  } catch (...) {
    return -1;
  }
}

int zfmm_zlfmm2d(double eps, int ns, const double* zsrc, int ifcharge, const double* charge,
                 int ifdipole, const double* dipstr, const double* dipvec, double* pot,
                 double* grad, int nt, const double* ztarg, int ifpgh, int isep, int ifprint) {
  (void)ifprint;
  return fmm2d_host(eps, nullptr, ns, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, pot,
                    grad, nt, ztarg, ifpgh, isep);
}

void zlfmm2d_(const double* eps, const int* ns, const double* zsrc, int* ifcharge,
              const double* charge, int* ifdipole, const double* dipstr, const double* dipvec,
              double* pot, double* grad, const int* nt, const double* ztarg, int* ifpgh,
              const int* isep, const int* ifprint) {
  clamp_flags(*ifcharge, *ifdipole, *ifpgh);  // written back, as the reference does
  int rc = fmm2d_host(*eps, nullptr, *ns, zsrc, *ifcharge, charge, *ifdipole, dipstr, dipvec,
                      pot, grad, *nt, ztarg, *ifpgh, *isep);
  if (rc != 0 && *nt > 0) {
    memset(pot, 0, sizeof(double) * 2 * *nt);
    if (grad) memset(grad, 0, sizeof(double) * 4 * *nt);
  }
  (void)ifprint;
}

int zfmm_zlfmm2d_dev(double eps, int ns, const double* zsrc, int ifcharge, const double* charge,
                     int ifdipole, const double* dipstr, const double* dipvec, double* pot,
                     double* grad, int nt, const double* ztarg, int ifpgh, int isep,
                     void* stream) {
  return guarded([&] {
    clamp_flags(ifcharge, ifdipole, ifpgh);
    check_args2d(ns, nt, zsrc, ztarg, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad,
                 ifpgh);
    check_align_dev(zsrc, ztarg, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad, ifpgh);
    check_device();
    cudaStream_t s = (cudaStream_t)stream;
    Inputs2D in = make_inputs(ns, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, nt, ztarg,
                              ifpgh);
    run_fmm2d(eps, nullptr, in, isep, (zdc*)pot, ifpgh > 1 ? (zdc*)grad : nullptr, s);
    ZF_CUDA(cudaStreamSynchronize(s));
  });
}

namespace {
int direct2d_host(const zdc* zk, int nt, const double* ztarg, int ns, const double* zsrc,
                  const double* charge, const double* dipstr, const double* dipvec, int ifcharge,
                  double* pot, double* grad, int ifdipole, int ifpgh) {
  return guarded([&] {
    check_args2d(ns, nt, zsrc, ztarg, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad,
                 ifpgh);
    if (nt == 0 || ns == 0) return;
    check_device();
    cudaStream_t s = cudaStreamPerThread;
    HostIn h;
    upload(h.zsrc, zsrc, 2 * (size_t)ns, s);
    upload(h.ztarg, ztarg, 2 * (size_t)nt, s);
    if (ifcharge == 1) upload(h.charge, charge, ns, s);
    if (ifdipole == 1) {
      upload(h.dipstr, dipstr, ns, s);
      upload(h.dipvec, dipvec, 2 * (size_t)ns, s);
    }
    DevBuf<zdc> dpot, dgrad;
    upload(dpot, pot, nt, s);
    if (ifpgh > 1) upload(dgrad, grad, 2 * (size_t)nt, s);
    Inputs2D in = make_inputs(ns, (const double*)h.zsrc.get(), ifcharge == 1,
                              (const double*)h.charge.get(), ifdipole == 1,
                              (const double*)h.dipstr.get(), (const double*)h.dipvec.get(), nt,
                              (const double*)h.ztarg.get(), ifpgh);
    if (zk) zh2ddirect_device(*zk, in, dpot.get(), dgrad.get(), s);
    else zl2ddirect_device(in, dpot.get(), dgrad.get(), nullptr, s);
    ZF_CUDA(cudaMemcpyAsync(pot, dpot.get(), sizeof(zdc) * nt, cudaMemcpyDeviceToHost, s));
    if (ifpgh > 1)
      ZF_CUDA(cudaMemcpyAsync(grad, dgrad.get(), sizeof(zdc) * 2 * nt, cudaMemcpyDeviceToHost, s));
    ZF_CUDA(cudaStreamSynchronize(s));
  });
}

}  // namespace

int zfmm_zl2devaldirect(int nt, const double* ztarg, int ns, const double* zsrc,
                        const double* charge, const double* dipstr, const double* dipvec,
                        int ifcharge, double* pot, double* grad, int ifdipole, int ifpgh) {
  return direct2d_host(nullptr, nt, ztarg, ns, zsrc, charge, dipstr, dipvec, ifcharge, pot, grad,
                       ifdipole, ifpgh);
}

void zl2devaldirect_(const int* nt, const double* ztarg, const int* ns, const double* zsrc,
                     const double* charge, const double* dipstr, const double* dipvec,
                     const int* ifcharge, double* pot, double* grad, const int* ifdipole,
                     const int* ifpgh) {
  zfmm_zl2devaldirect(*nt, ztarg, *ns, zsrc, charge, dipstr, dipvec, *ifcharge, pot, grad,
                      *ifdipole, *ifpgh);
}

int zfmm_zl2devaldirect_dev(int nt, const double* ztarg, int ns, const double* zsrc,
                            const double* charge, const double* dipstr, const double* dipvec,
                            int ifcharge, double* pot, double* grad, int ifdipole, int ifpgh,
                            void* stream) {
  return guarded([&] {
    check_args2d(ns, nt, zsrc, ztarg, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad,
                 ifpgh);
    check_align_dev(zsrc, ztarg, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad, ifpgh);
    if (nt == 0 || ns == 0) return;
    check_device();
    cudaStream_t s = (cudaStream_t)stream;
    Inputs2D in = make_inputs(ns, zsrc, ifcharge == 1, charge, ifdipole == 1, dipstr, dipvec, nt,
                              ztarg, ifpgh);
    zl2ddirect_device(in, (zdc*)pot, (zdc*)grad, nullptr, s);
    ZF_CUDA(cudaStreamSynchronize(s));
  });
}

int zfmm_zhfmm2d(double eps, const double* zk, int ns, const double* zsrc, int ifcharge,
                 const double* charge, int ifdipole, const double* dipstr, const double* dipvec,
                 double* pot, double* grad, int nt, const double* ztarg, int ifpgh, int isep,
                 int ifprint) {
  (void)ifprint;
  if (!zk) return fail(ZF_ERR_ARG, "zk is null");
  zdc k = mkz(zk[0], zk[1]);
  return fmm2d_host(eps, &k, ns, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad, nt,
                    ztarg, ifpgh, isep);
}

void zhfmm2d_(const double* eps, const double* zk, const int* ns, const double* zsrc,
              int* ifcharge, const double* charge, int* ifdipole, const double* dipstr,
              const double* dipvec, double* pot, double* grad, const int* nt,
              const double* ztarg, int* ifpgh, const int* isep, const int* ifprint) {
  clamp_flags(*ifcharge, *ifdipole, *ifpgh);  // written back, as the reference does
  zdc k = mkz(zk[0], zk[1]);
  int rc = fmm2d_host(*eps, &k, *ns, zsrc, *ifcharge, charge, *ifdipole, dipstr, dipvec, pot,
                      grad, *nt, ztarg, *ifpgh, *isep);
  if (rc != 0 && *nt > 0) {
    memset(pot, 0, sizeof(double) * 2 * *nt);
    if (grad) memset(grad, 0, sizeof(double) * 4 * *nt);
  }
  (void)ifprint;
}

int zfmm_zhfmm2d_dev(double eps, const double* zk, int ns, const double* zsrc, int ifcharge,
                     const double* charge, int ifdipole, const double* dipstr,
                     const double* dipvec, double* pot, double* grad, int nt, const double* ztarg,
                     int ifpgh, int isep, void* stream) {
  return guarded([&] {
    if (!zk) throw zf_error(ZF_ERR_ARG, "zk is null");
    clamp_flags(ifcharge, ifdipole, ifpgh);
    check_args2d(ns, nt, zsrc, ztarg, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad,
                 ifpgh);
    check_align_dev(zsrc, ztarg, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad, ifpgh);
    check_device();
    cudaStream_t s = (cudaStream_t)stream;
    Inputs2D in = make_inputs(ns, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, nt, ztarg,
                              ifpgh);
    zdc k = mkz(zk[0], zk[1]);
    run_fmm2d(eps, &k, in, isep, (zdc*)pot, ifpgh > 1 ? (zdc*)grad : nullptr, s);
    ZF_CUDA(cudaStreamSynchronize(s));
  });
}

int zfmm_zh2devaldirect(const double* zk, int nt, const double* ztarg, int ns, const double* zsrc,
                        const double* charge, const double* dipstr, const double* dipvec,
                        int ifcharge, double* pot, double* grad, int ifdipole, int ifpgh) {
  if (!zk) return fail(ZF_ERR_ARG, "zk is null");
  zdc k = mkz(zk[0], zk[1]);
  return direct2d_host(&k, nt, ztarg, ns, zsrc, charge, dipstr, dipvec, ifcharge, pot, grad,
                       ifdipole, ifpgh);
}

void zh2devaldirect_(const double* zk, const int* nt, const double* ztarg, const int* ns,
                     const double* zsrc, const double* charge, const double* dipstr,
                     const double* dipvec, const int* ifcharge, double* pot, double* grad,
                     const int* ifdipole, const int* ifpgh) {
  zfmm_zh2devaldirect(zk, *nt, ztarg, *ns, zsrc, charge, dipstr, dipvec, *ifcharge, pot, grad,
                      *ifdipole, *ifpgh);
}

int zfmm_zh2devaldirect_dev(const double* zk, int nt, const double* ztarg, int ns,
                            const double* zsrc, const double* charge, const double* dipstr,
                            const double* dipvec, int ifcharge, double* pot, double* grad,
                            int ifdipole, int ifpgh, void* stream) {
  return guarded([&] {
    if (!zk) throw zf_error(ZF_ERR_ARG, "zk is null");
    check_args2d(ns, nt, zsrc, ztarg, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad,
                 ifpgh);
    check_align_dev(zsrc, ztarg, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad, ifpgh);
    if (nt == 0 || ns == 0) return;
    check_device();
    cudaStream_t s = (cudaStream_t)stream;
    Inputs2D in = make_inputs(ns, zsrc, ifcharge == 1, charge, ifdipole == 1, dipstr, dipvec, nt,
                              ztarg, ifpgh);
    zh2ddirect_device(mkz(zk[0], zk[1]), in, (zdc*)pot, (zdc*)grad, s);
    ZF_CUDA(cudaStreamSynchronize(s));
  });
}

int zfmm_zl2devaldirect_dev_noalloc(int nt, const double* ztarg, int ns, const double* zsrc,
                                    const double* charge, const double* dipstr,
                                    const double* dipvec, int ifcharge, double* pot, double* grad,
                                    int ifdipole, int ifpgh, void* stream) {
  return guarded([&] {
    check_args2d(ns, nt, zsrc, ztarg, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad,
                 ifpgh);
    check_align_dev(zsrc, ztarg, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad, ifpgh);
    if (nt == 0 || ns == 0) return;
    check_device();
    cudaStream_t s = (cudaStream_t)stream;
    Inputs2D in = make_inputs(ns, zsrc, ifcharge == 1, charge, ifdipole == 1, dipstr, dipvec, nt,
                              ztarg, ifpgh);
    zl2ddirect_device_noalloc(in, (zdc*)pot, (zdc*)grad, s);
    ZF_CUDA(cudaStreamSynchronize(s));
  });
}

long zfmm_zl2devaldirect_noalloc_capacity(void) {
  return (long)(direct2d_noalloc_capacity() * sizeof(zdc));
}

int zfmm_tree_dump(int D, int ndiv, int isep, int ns, const double* zsrc, int nt,
                   const double* ztarg, int box_cap, int list_cap, int* nboxes, int* nlevels,
                   int* laddr, int* ilevel, int* iparent, int* nchild, int* ichild,
                   double* centers, int* isrc, int* isrcse, int* itarg, int* itargse, int* nlist,
                   int* lists, int* nlists_total, int* mnlist) {
  return guarded([&] {
    if ((D != 2 && D != 3) || ns < 1 || nt < 1 || !zsrc || !ztarg)
      throw zf_error(ZF_ERR_ARG, "bad tree_dump arguments");
    check_device();
    cudaStream_t s = cudaStreamPerThread;
    std::vector<double> sr((size_t)D * ns), tr((size_t)D * nt);
    for (size_t i = 0; i < sr.size(); i++) sr[i] = zsrc[2 * i];
    for (size_t i = 0; i < tr.size(); i++) tr[i] = ztarg[2 * i];
    DevBuf<double> dsr(sr.size(), s), dtr(tr.size(), s);
    ZF_CUDA(cudaMemcpyAsync(dsr.get(), sr.data(), sr.size() * 8, cudaMemcpyHostToDevice, s));
    ZF_CUDA(cudaMemcpyAsync(dtr.get(), tr.data(), tr.size() * 8, cudaMemcpyHostToDevice, s));
    TreeParams tp;
    tp.D = D;
    tp.ndiv = ndiv;
    tp.isep = isep;
    tp.lr_isep_quirk = D == 3;
    DevTree t;
    build_tree(dsr.get(), ns, dtr.get(), nt, tp, t, s);
    *nboxes = t.nboxes;
    *nlevels = t.nlevels;
    if (box_cap < t.nboxes) return;
    int nb = t.nboxes, NC = 1 << D;
    for (size_t i = 0; i < t.laddr.size(); i++) laddr[i] = t.laddr[i];
    auto d2h = [&](void* dst, const void* src, size_t bytes) {
      ZF_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
    };
    d2h(ilevel, t.ilevel.get(), nb * 4);
    d2h(iparent, t.iparent.get(), nb * 4);
    d2h(nchild, t.nchild.get(), nb * 4);
    d2h(ichild, t.ichild.get(), (size_t)nb * NC * 4);
    d2h(centers, t.centers.get(), (size_t)nb * D * 8);
    DevBuf<int> pi, se;
    sort_points(t, dsr.get(), ns, pi, se, s);
    d2h(isrc, pi.get(), (size_t)ns * 4);
    d2h(isrcse, se.get(), (size_t)nb * 8);
    sort_points(t, dtr.get(), nt, pi, se, s);
    d2h(itarg, pi.get(), (size_t)nt * 4);
    d2h(itargse, se.get(), (size_t)nb * 8);
    DevLists L;
    build_lists(t, L, s);
    std::vector<int> cnt(nb), buf;
    size_t pos = 0;
    for (int k = 0; k < 4; k++) {
      mnlist[k] = L.mn[k];
      d2h(cnt.data(), L.n[k].get(), nb * 4);
      buf.resize((size_t)(L.mn[k] > 0 ? L.mn[k] : 1) * nb);
      d2h(buf.data(), L.list[k].get(), buf.size() * 4);
      ZF_CUDA(cudaStreamSynchronize(s));
      for (int b = 0; b < nb; b++) {
        nlist[k * nb + b] = cnt[b];
        for (int i = 0; i < cnt[b]; i++) {
          if ((long)pos < list_cap) lists[pos] = buf[(size_t)b * L.mn[k] + i];
          pos++;
        }
      }
    }
    *nlists_total = (int)pos;
    ZF_CUDA(cudaStreamSynchronize(s));
  });
}

}  // extern "C"

// ---- 3D Laplace -------------------------------------------------------------
namespace {

Inputs3D make_inputs3(int ns, const double* zsrc, int ifcharge, const double* charge,
                      int ifdipole, const double* dipstr, const double* dipvec, int nt,
                      const double* ztarg, int ifpgh) {
  Inputs3D in;
  in.ns = ns;
  in.nt = nt;
  in.zsrc = reinterpret_cast<const zdc*>(zsrc);
  in.charge = reinterpret_cast<const zdc*>(charge);
  in.dipstr = reinterpret_cast<const zdc*>(dipstr);
  in.dipvec = reinterpret_cast<const zdc*>(dipvec);
  in.ztarg = reinterpret_cast<const zdc*>(ztarg);
  in.ifcharge = ifcharge;
  in.ifdipole = ifdipole;
  in.ifpgh = ifpgh;
  return in;
}

// zk == nullptr selects the Laplace FMM, otherwise Helmholtz with wavenumber *zk
void run_fmm3d(double eps, const zdc* zk, const Inputs3D& in, int isep, zdc* pot, zdc* grad,
               cudaStream_t s) {
  // zlfmm3d.f:36-37: pot and grad are zeroed first
  if (in.nt > 0) {
    ZF_CUDA(cudaMemsetAsync(pot, 0, sizeof(zdc) * in.nt, s));
    if (grad) ZF_CUDA(cudaMemsetAsync(grad, 0, sizeof(zdc) * 3 * in.nt, s));
  }
  if (in.ns == 0 || in.nt == 0) return;
  if (isep < 1) throw zf_error(ZF_ERR_ARG, "isep must be >= 1");
  StepTimes t;
  t.want_counts = g_timing >= 2;
  if (zk) zhfmm3d_device(eps, *zk, in, isep, pot, grad, s, g_timing ? &t : nullptr);
  else zlfmm3d_device(eps, in, isep, pot, grad, s, g_timing ? &t : nullptr);
  if (g_timing) g_times = t;
}

int fmm3d_host(double eps, const zdc* zk, int ns, const double* zsrc, int ifcharge,
               const double* charge, int ifdipole, const double* dipstr, const double* dipvec,
               double* pot, double* grad, int nt, const double* ztarg, int ifpgh, int isep) {
  return guarded([&] {
    clamp_flags(ifcharge, ifdipole, ifpgh);
    check_args2d(ns, nt, zsrc, ztarg, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad,
                 ifpgh);
    check_device();
    cudaStream_t s = cudaStreamPerThread;
    HostIn h;
    // targets passed as the source array itself: uploaded once
    const bool same = ztarg == zsrc && nt == ns;
    upload(h.zsrc, zsrc, 3 * (size_t)ns, s);
    if (!same) upload(h.ztarg, ztarg, 3 * (size_t)nt, s);
    StrengthUpload su(h, ns, 3, ifcharge, charge, ifdipole, dipstr, dipvec, s);
    DevBuf<zdc> dpot(nt, s), dgrad(ifpgh > 1 ? 3 * (size_t)nt : 0, s);
    Inputs3D in = make_inputs3(ns, (const double*)h.zsrc.get(), ifcharge,
                               (const double*)h.charge.get(), ifdipole,
                               (const double*)h.dipstr.get(), (const double*)h.dipvec.get(), nt,
                               (const double*)(same ? h.zsrc.get() : h.ztarg.get()), ifpgh);
    in.strengths_ready = [&su](cudaStream_t ss) { su.ready(ss); };
    run_fmm3d(eps, zk, in, isep, dpot.get(), ifpgh > 1 ? dgrad.get() : nullptr, s);
    if (nt > 0) {
      ZF_CUDA(cudaMemcpyAsync(pot, dpot.get(), sizeof(zdc) * nt, cudaMemcpyDeviceToHost, s));
      if (grad) {
        if (ifpgh > 1)
          ZF_CUDA(cudaMemcpyAsync(grad, dgrad.get(), sizeof(zdc) * 3 * nt, cudaMemcpyDeviceToHost, s));
        else
          memset(grad, 0, sizeof(zdc) * 3 * nt);
      }
    }
    ZF_CUDA(cudaStreamSynchronize(s));
  });
}

int direct3d_host(const zdc* zk, int nt, const double* ztarg, int ns, const double* zsrc,
                  const double* charge, const double* dipstr, const double* dipvec, int ifcharge,
                  double* pot, double* grad, int ifdipole, int ifpgh) {
  return guarded([&] {
    check_args2d(ns, nt, zsrc, ztarg, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad,
                 ifpgh);
    if (nt == 0 || ns == 0) return;
    check_device();
    cudaStream_t s = cudaStreamPerThread;
    HostIn h;
    upload(h.zsrc, zsrc, 3 * (size_t)ns, s);
    upload(h.ztarg, ztarg, 3 * (size_t)nt, s);
    if (ifcharge == 1) upload(h.charge, charge, ns, s);
    if (ifdipole == 1) {
      upload(h.dipstr, dipstr, ns, s);
      upload(h.dipvec, dipvec, 3 * (size_t)ns, s);
    }
    DevBuf<zdc> dpot, dgrad;
    upload(dpot, pot, nt, s);
    if (ifpgh > 1) upload(dgrad, grad, 3 * (size_t)nt, s);
    Inputs3D in = make_inputs3(ns, (const double*)h.zsrc.get(), ifcharge == 1,
                               (const double*)h.charge.get(), ifdipole == 1,
                               (const double*)h.dipstr.get(), (const double*)h.dipvec.get(), nt,
                               (const double*)h.ztarg.get(), ifpgh);
    if (zk) zh3ddirect_device(*zk, in, dpot.get(), dgrad.get(), s);
    else zl3ddirect_device(in, dpot.get(), dgrad.get(), s);
    ZF_CUDA(cudaMemcpyAsync(pot, dpot.get(), sizeof(zdc) * nt, cudaMemcpyDeviceToHost, s));
    if (ifpgh > 1)
      ZF_CUDA(cudaMemcpyAsync(grad, dgrad.get(), sizeof(zdc) * 3 * nt, cudaMemcpyDeviceToHost, s));
    ZF_CUDA(cudaStreamSynchronize(s));
  });
}

}  // namespace

extern "C" {

int zfmm_zlfmm3d(double eps, int ns, const double* zsrc, int ifcharge, const double* charge,
                 int ifdipole, const double* dipstr, const double* dipvec, double* pot,
                 double* grad, int nt, const double* ztarg, int ifpgh, int isep, int ifprint) {
  (void)ifprint;
  return fmm3d_host(eps, nullptr, ns, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, pot,
                    grad, nt, ztarg, ifpgh, isep);
}

void zlfmm3d_(const double* eps, const int* ns, const double* zsrc, int* ifcharge,
              const double* charge, int* ifdipole, const double* dipstr, const double* dipvec,
              double* pot, double* grad, const int* nt, const double* ztarg, int* ifpgh,
              const int* isep, const int* ifprint) {
  clamp_flags(*ifcharge, *ifdipole, *ifpgh);  // written back, as the reference does
  int rc = fmm3d_host(*eps, nullptr, *ns, zsrc, *ifcharge, charge, *ifdipole, dipstr, dipvec,
                      pot, grad, *nt, ztarg, *ifpgh, *isep);
  if (rc != 0 && *nt > 0) {
    memset(pot, 0, sizeof(double) * 2 * *nt);
    if (grad) memset(grad, 0, sizeof(double) * 6 * *nt);
  }
  (void)ifprint;
}

int zfmm_zlfmm3d_dev(double eps, int ns, const double* zsrc, int ifcharge, const double* charge,
                     int ifdipole, const double* dipstr, const double* dipvec, double* pot,
                     double* grad, int nt, const double* ztarg, int ifpgh, int isep,
                     void* stream) {
  return guarded([&] {
    clamp_flags(ifcharge, ifdipole, ifpgh);
    check_args2d(ns, nt, zsrc, ztarg, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad,
                 ifpgh);
    check_align_dev(zsrc, ztarg, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad, ifpgh);
    check_device();
    cudaStream_t s = (cudaStream_t)stream;
    Inputs3D in = make_inputs3(ns, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, nt, ztarg,
                               ifpgh);
    run_fmm3d(eps, nullptr, in, isep, (zdc*)pot, ifpgh > 1 ? (zdc*)grad : nullptr, s);
    ZF_CUDA(cudaStreamSynchronize(s));
  });
}

int zfmm_zl3devaldirect(int nt, const double* ztarg, int ns, const double* zsrc,
                        const double* charge, const double* dipstr, const double* dipvec,
                        int ifcharge, double* pot, double* grad, int ifdipole, int ifpgh) {
  return direct3d_host(nullptr, nt, ztarg, ns, zsrc, charge, dipstr, dipvec, ifcharge, pot, grad,
                       ifdipole, ifpgh);
}

void zl3devaldirect_(const int* nt, const double* ztarg, const int* ns, const double* zsrc,
                     const double* charge, const double* dipstr, const double* dipvec,
                     const int* ifcharge, double* pot, double* grad, const int* ifdipole,
                     const int* ifpgh) {
  zfmm_zl3devaldirect(*nt, ztarg, *ns, zsrc, charge, dipstr, dipvec, *ifcharge, pot, grad,
                      *ifdipole, *ifpgh);
}

int zfmm_zl3devaldirect_dev(int nt, const double* ztarg, int ns, const double* zsrc,
                            const double* charge, const double* dipstr, const double* dipvec,
                            int ifcharge, double* pot, double* grad, int ifdipole, int ifpgh,
                            void* stream) {
  return guarded([&] {
    check_args2d(ns, nt, zsrc, ztarg, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad,
                 ifpgh);
    check_align_dev(zsrc, ztarg, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad, ifpgh);
    if (nt == 0 || ns == 0) return;
    check_device();
    cudaStream_t s = (cudaStream_t)stream;
    Inputs3D in = make_inputs3(ns, zsrc, ifcharge == 1, charge, ifdipole == 1, dipstr, dipvec, nt,
                               ztarg, ifpgh);
    zl3ddirect_device(in, (zdc*)pot, (zdc*)grad, s);
    ZF_CUDA(cudaStreamSynchronize(s));
  });
}

int zfmm_zl3dterms(double eps) { return zl3dterms(eps); }

// ---- 3D Helmholtz ----
int zfmm_zhfmm3d(double eps, const double* zk, int ns, const double* zsrc, int ifcharge,
                 const double* charge, int ifdipole, const double* dipstr, const double* dipvec,
                 double* pot, double* grad, int nt, const double* ztarg, int ifpgh, int isep,
                 int ifprint) {
  (void)ifprint;
  if (!zk) return fail(ZF_ERR_ARG, "zk is null");
  zdc k = mkz(zk[0], zk[1]);
  return fmm3d_host(eps, &k, ns, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad,
                    nt, ztarg, ifpgh, isep);
}

void zhfmm3d_(const double* eps, const double* zk, const int* ns, const double* zsrc,
              int* ifcharge, const double* charge, int* ifdipole, const double* dipstr,
              const double* dipvec, double* pot, double* grad, const int* nt,
              const double* ztarg, int* ifpgh, const int* isep, const int* ifprint) {
  clamp_flags(*ifcharge, *ifdipole, *ifpgh);  // written back, as the reference does
  int rc = zfmm_zhfmm3d(*eps, zk, *ns, zsrc, *ifcharge, charge, *ifdipole, dipstr, dipvec, pot,
                        grad, *nt, ztarg, *ifpgh, *isep, *ifprint);
  if (rc != 0 && *nt > 0) {
    memset(pot, 0, sizeof(double) * 2 * *nt);
    if (grad) memset(grad, 0, sizeof(double) * 6 * *nt);
  }
}

int zfmm_zhfmm3d_dev(double eps, const double* zk, int ns, const double* zsrc, int ifcharge,
                     const double* charge, int ifdipole, const double* dipstr,
                     const double* dipvec, double* pot, double* grad, int nt, const double* ztarg,
                     int ifpgh, int isep, void* stream) {
  return guarded([&] {
    if (!zk) throw zf_error(ZF_ERR_ARG, "zk is null");
    clamp_flags(ifcharge, ifdipole, ifpgh);
    check_args2d(ns, nt, zsrc, ztarg, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad,
                 ifpgh);
    check_align_dev(zsrc, ztarg, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad, ifpgh);
    check_device();
    cudaStream_t s = (cudaStream_t)stream;
    zdc k = mkz(zk[0], zk[1]);
    Inputs3D in = make_inputs3(ns, zsrc, ifcharge, charge, ifdipole, dipstr, dipvec, nt, ztarg,
                               ifpgh);
    run_fmm3d(eps, &k, in, isep, (zdc*)pot, ifpgh > 1 ? (zdc*)grad : nullptr, s);
    ZF_CUDA(cudaStreamSynchronize(s));
  });
}

int zfmm_zh3devaldirect(const double* zk, int nt, const double* ztarg, int ns, const double* zsrc,
                        const double* charge, const double* dipstr, const double* dipvec,
                        int ifcharge, double* pot, double* grad, int ifdipole, int ifpgh) {
  if (!zk) return fail(ZF_ERR_ARG, "zk is null");
  zdc k = mkz(zk[0], zk[1]);
  return direct3d_host(&k, nt, ztarg, ns, zsrc, charge, dipstr, dipvec, ifcharge, pot, grad,
                       ifdipole, ifpgh);
}

void zh3devaldirect_(const double* zk, const int* nt, const double* ztarg, const int* ns,
                     const double* zsrc, const double* charge, const double* dipstr,
                     const double* dipvec, const int* ifcharge, double* pot, double* grad,
                     const int* ifdipole, const int* ifpgh) {
  zfmm_zh3devaldirect(zk, *nt, ztarg, *ns, zsrc, charge, dipstr, dipvec, *ifcharge, pot, grad,
                      *ifdipole, *ifpgh);
}

int zfmm_zh3devaldirect_dev(const double* zk, int nt, const double* ztarg, int ns,
                            const double* zsrc, const double* charge, const double* dipstr,
                            const double* dipvec, int ifcharge, double* pot, double* grad,
                            int ifdipole, int ifpgh, void* stream) {
  return guarded([&] {
    if (!zk) throw zf_error(ZF_ERR_ARG, "zk is null");
    check_args2d(ns, nt, zsrc, ztarg, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad,
                 ifpgh);
    check_align_dev(zsrc, ztarg, ifcharge, charge, ifdipole, dipstr, dipvec, pot, grad, ifpgh);
    if (nt == 0 || ns == 0) return;
    check_device();
    cudaStream_t s = (cudaStream_t)stream;
    Inputs3D in = make_inputs3(ns, zsrc, ifcharge == 1, charge, ifdipole == 1, dipstr, dipvec, nt,
                               ztarg, ifpgh);
    zh3ddirect_device(mkz(zk[0], zk[1]), in, (zdc*)pot, (zdc*)grad, s);
    ZF_CUDA(cudaStreamSynchronize(s));
  });
}

int zfmm_h3dterms(double size, const double* zk, double eps, int isep) {
  if (!zk) return -1;
  try {
    return h3dterms_host(size, mkz(zk[0], zk[1]), eps, isep);
  } catch (...) {
    return -1;
  }
}

}  // extern "C"

// ---- 3D plans: geometry once, many solves of nd right-hand sides ---------------
struct zfmm_plan3d_s {
  zf::Plan3D P;
};

namespace {

void check_plan_args(zfmm_plan3d_s* plan, int nd, int ifcharge, const double* charge,
                     int ifdipole, const double* dipstr, const double* dipvec, int ifpgh,
                     double* pot, double* grad) {
  if (!plan) throw zf_error(ZF_ERR_ARG, "plan is null");
  if (nd < 1) throw zf_error(ZF_ERR_ARG, "nd must be >= 1");
  const Plan3D& P = plan->P;
  if (P.ns > 0 && ifcharge == 1 && !charge) throw zf_error(ZF_ERR_ARG, "ifcharge=1 needs charge");
  if (P.ns > 0 && ifdipole == 1 && (!dipstr || !dipvec))
    throw zf_error(ZF_ERR_ARG, "ifdipole=1 needs dipstr and dipvec");
  if (P.nt > 0 && !pot) throw zf_error(ZF_ERR_ARG, "null pot");
  if (P.nt > 0 && ifpgh > 1 && !grad) throw zf_error(ZF_ERR_ARG, "ifpgh=2 needs grad");
  int dev = 0;
  ZF_CUDA(cudaGetDevice(&dev));
  if (dev != P.device) throw zf_error(ZF_ERR_ARG, "plan was built on another device");
}

// device path of the plan solves: pot / grad zeroed, then the FMM
void run_plan3d(zfmm_plan3d_s* plan, const zdc* zk, int nd, int ifcharge, const zdc* charge,
                int ifdipole, const zdc* dipstr, const zdc* dipvec, int ifpgh, zdc* pot,
                zdc* grad, cudaStream_t s) {
  const Plan3D& P = plan->P;
  if (P.nt > 0) {
    ZF_CUDA(cudaMemsetAsync(pot, 0, sizeof(zdc) * P.nt * (size_t)nd, s));
    if (ifpgh > 1) ZF_CUDA(cudaMemsetAsync(grad, 0, sizeof(zdc) * 3 * P.nt * (size_t)nd, s));
  }
  if (P.ns == 0 || P.nt == 0) return;
  StrengthsNd in;
  in.ifcharge = ifcharge;
  in.ifdipole = ifdipole;
  in.charge = charge;
  in.dipstr = dipstr;
  in.dipvec = dipvec;
  StepTimes t;
  t.want_counts = g_timing >= 2;
  if (zk)
    zhfmm3d_plan_execute(P, *zk, nd, in, ifpgh, pot, ifpgh > 1 ? grad : nullptr, s,
                         g_timing ? &t : nullptr);
  else
    zlfmm3d_plan_execute(P, nd, in, ifpgh, pot, ifpgh > 1 ? grad : nullptr, s,
                         g_timing ? &t : nullptr);
  if (g_timing) g_times = t;
}

int plan3d_create_impl(double eps, int ns, const double* zsrc, int nt, const double* ztarg,
                       int isep, bool host, cudaStream_t s, zfmm_plan3d_s** out) {
  return guarded([&] {
    if (!out) throw zf_error(ZF_ERR_ARG, "null plan output");
    *out = nullptr;
    if (ns < 0 || nt < 0) throw zf_error(ZF_ERR_ARG, "ns and nt must be >= 0");
    if ((ns > 0 && !zsrc) || (nt > 0 && !ztarg))
      throw zf_error(ZF_ERR_ARG, "null coordinate array");
    check_device();
    auto* pl = new zfmm_plan3d_s();
    try {
      HostIn h;
      const zdc* zs = reinterpret_cast<const zdc*>(zsrc);
      const zdc* zt = reinterpret_cast<const zdc*>(ztarg);
      if (!host) check_align16({zsrc, ztarg});
      if (host) {
        // targets passed as the source array itself: uploaded once
        const bool same = ztarg == zsrc && nt == ns;
        upload(h.zsrc, zsrc, 3 * (size_t)ns, s);
        if (!same) upload(h.ztarg, ztarg, 3 * (size_t)nt, s);
        zs = h.zsrc.get();
        zt = same ? zs : h.ztarg.get();
      }
      if (ns > 0 && nt > 0) plan3d_build(pl->P, eps, ns, zs, nt, zt, isep, s);
      else {
        if (isep < 1) throw zf_error(ZF_ERR_ARG, "isep must be >= 1");
        pl->P.eps = eps;
        pl->P.isep = isep;
        pl->P.ns = ns;
        pl->P.nt = nt;
        ZF_CUDA(cudaGetDevice(&pl->P.device));
      }
      ZF_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
      delete pl;
      throw;
    }
    *out = pl;
  });
}

}  // namespace

extern "C" {

int zfmm_plan3d_create(double eps, int ns, const double* zsrc, int nt, const double* ztarg,
                       int isep, zfmm_plan3d* plan) {
  return plan3d_create_impl(eps, ns, zsrc, nt, ztarg, isep, true, cudaStreamPerThread, plan);
}

int zfmm_plan3d_create_dev(double eps, int ns, const double* zsrc, int nt, const double* ztarg,
                           int isep, void* stream, zfmm_plan3d* plan) {
  return plan3d_create_impl(eps, ns, zsrc, nt, ztarg, isep, false, (cudaStream_t)stream, plan);
}

int zfmm_plan3d_destroy(zfmm_plan3d plan) {
  return guarded([&] {
    if (!plan) return;
    // solves may still run on other streams: the plan's memory goes back once
    // the device is idle
    ZF_CUDA(cudaDeviceSynchronize());
    delete plan;
  });
}

int zfmm_plan3d_info(zfmm_plan3d plan, int* nboxes, int* nlevels, int* ns, int* nt) {
  return guarded([&] {
    if (!plan) throw zf_error(ZF_ERR_ARG, "plan is null");
    if (nboxes) *nboxes = plan->P.S.tree.nboxes;
    if (nlevels) *nlevels = plan->P.S.tree.nlevels;
    if (ns) *ns = plan->P.ns;
    if (nt) *nt = plan->P.nt;
  });
}

}  // extern "C"

namespace {

int plan_solve_host(zfmm_plan3d plan, const double* zk, int nd, int ifcharge,
                    const double* charge, int ifdipole, const double* dipstr,
                    const double* dipvec, int ifpgh, double* pot, double* grad) {
  return guarded([&] {
    clamp_flags(ifcharge, ifdipole, ifpgh);
    check_plan_args(plan, nd, ifcharge, charge, ifdipole, dipstr, dipvec, ifpgh, pot, grad);
    const int ns = plan->P.ns, nt = plan->P.nt;
    cudaStream_t s = cudaStreamPerThread;
    HostIn h;
    if (ifcharge == 1) upload(h.charge, charge, (size_t)nd * ns, s);
    if (ifdipole == 1) {
      upload(h.dipstr, dipstr, (size_t)nd * ns, s);
      upload(h.dipvec, dipvec, 3 * (size_t)ns, s);
    }
    DevBuf<zdc> dpot((size_t)nd * nt, s), dgrad(ifpgh > 1 ? 3 * (size_t)nd * nt : 0, s);
    zdc k = zk ? mkz(zk[0], zk[1]) : mkz(0.0);
    run_plan3d(plan, zk ? &k : nullptr, nd, ifcharge, h.charge.get(), ifdipole, h.dipstr.get(),
               h.dipvec.get(), ifpgh, dpot.get(), dgrad.get(), s);
    if (nt > 0) {
      ZF_CUDA(cudaMemcpyAsync(pot, dpot.get(), sizeof(zdc) * nt * (size_t)nd,
                              cudaMemcpyDeviceToHost, s));
      if (grad) {
        if (ifpgh > 1)
          ZF_CUDA(cudaMemcpyAsync(grad, dgrad.get(), sizeof(zdc) * 3 * nt * (size_t)nd,
                                  cudaMemcpyDeviceToHost, s));
        else
          memset(grad, 0, sizeof(zdc) * 3 * nt * (size_t)nd);
      }
    }
    ZF_CUDA(cudaStreamSynchronize(s));
  });
}

int plan_solve_dev(zfmm_plan3d plan, const double* zk, int nd, int ifcharge,
                   const double* charge, int ifdipole, const double* dipstr,
                   const double* dipvec, int ifpgh, double* pot, double* grad, void* stream) {
  return guarded([&] {
    clamp_flags(ifcharge, ifdipole, ifpgh);
    check_plan_args(plan, nd, ifcharge, charge, ifdipole, dipstr, dipvec, ifpgh, pot, grad);
    check_align16({pot, ifcharge == 1 ? charge : nullptr, ifdipole == 1 ? dipstr : nullptr,
                   ifdipole == 1 ? dipvec : nullptr, ifpgh > 1 ? grad : nullptr});
    cudaStream_t s = (cudaStream_t)stream;
    zdc k = zk ? mkz(zk[0], zk[1]) : mkz(0.0);
    run_plan3d(plan, zk ? &k : nullptr, nd, ifcharge, (const zdc*)charge, ifdipole,
               (const zdc*)dipstr, (const zdc*)dipvec, ifpgh, (zdc*)pot, (zdc*)grad, s);
    ZF_CUDA(cudaStreamSynchronize(s));
  });
}

}  // namespace

extern "C" {

int zfmm_zlfmm3d_plan(zfmm_plan3d plan, int nd, int ifcharge, const double* charge,
                      int ifdipole, const double* dipstr, const double* dipvec, int ifpgh,
                      double* pot, double* grad) {
  return plan_solve_host(plan, nullptr, nd, ifcharge, charge, ifdipole, dipstr, dipvec, ifpgh,
                         pot, grad);
}

int zfmm_zlfmm3d_plan_dev(zfmm_plan3d plan, int nd, int ifcharge, const double* charge,
                          int ifdipole, const double* dipstr, const double* dipvec, int ifpgh,
                          double* pot, double* grad, void* stream) {
  return plan_solve_dev(plan, nullptr, nd, ifcharge, charge, ifdipole, dipstr, dipvec, ifpgh,
                        pot, grad, stream);
}

int zfmm_zhfmm3d_plan(zfmm_plan3d plan, const double* zk, int nd, int ifcharge,
                      const double* charge, int ifdipole, const double* dipstr,
                      const double* dipvec, int ifpgh, double* pot, double* grad) {
  if (!zk) return fail(ZF_ERR_ARG, "zk is null");
  return plan_solve_host(plan, zk, nd, ifcharge, charge, ifdipole, dipstr, dipvec, ifpgh, pot,
                         grad);
}

int zfmm_zhfmm3d_plan_dev(zfmm_plan3d plan, const double* zk, int nd, int ifcharge,
                          const double* charge, int ifdipole, const double* dipstr,
                          const double* dipvec, int ifpgh, double* pot, double* grad,
                          void* stream) {
  if (!zk) return fail(ZF_ERR_ARG, "zk is null");
  return plan_solve_dev(plan, zk, nd, ifcharge, charge, ifdipole, dipstr, dipvec, ifpgh, pot,
                        grad, stream);
}

}  // extern "C"

// ---- many independent 3D FMMs in one call -------------------------------------
namespace {

struct ManyArgs {
  int ninst = 0;
  double eps = 0;
  const zdc* zk = nullptr;
  const int *ns = nullptr, *nt = nullptr;
  const double* const* zsrc = nullptr;
  const double* const* charge = nullptr;
  const double* const* dipstr = nullptr;
  const double* const* dipvec = nullptr;
  const double* const* ztarg = nullptr;
  double* const* pot = nullptr;
  double* const* grad = nullptr;
  int ifcharge = 1, ifdipole = 0, ifpgh = 1, isep = 1;
  bool host = true;
};

// Instances are taken largest first from a shared counter by `nworkers` host
// threads, each driving its own CUDA stream, so small instances overlap on the
// GPU.  done_ms[i]: completion time of instance i after the call started.
void run_many(const ManyArgs& M, int nworkers, double* done_ms) {
  int dev = 0;
  ZF_CUDA(cudaGetDevice(&dev));
  std::vector<int> order(M.ninst);
  for (int i = 0; i < M.ninst; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    return (long)M.ns[a] + M.nt[a] > (long)M.ns[b] + M.nt[b];
  });
  std::atomic<int> next{0};
  std::mutex err_mu;
  std::string err;
  int err_code = 0;
  const auto t0 = std::chrono::steady_clock::now();
  auto worker = [&]() {
    cudaStream_t s = nullptr;
    try {
      ZF_CUDA(cudaSetDevice(dev));
      ZF_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
      for (;;) {
        {
          std::lock_guard<std::mutex> lk(err_mu);
          if (err_code) break;
        }
        int k = next.fetch_add(1);
        if (k >= M.ninst) break;
        const int i = order[k];
        const int ns = M.ns[i], nt = M.nt[i];
        if (M.host) {
          HostIn h;
          const bool same = M.ztarg[i] == M.zsrc[i] && nt == ns;  // uploaded once
          upload(h.zsrc, M.zsrc[i], 3 * (size_t)ns, s);
          if (!same) upload(h.ztarg, M.ztarg[i], 3 * (size_t)nt, s);
          if (M.ifcharge == 1) upload(h.charge, M.charge[i], ns, s);
          if (M.ifdipole == 1) {
            upload(h.dipstr, M.dipstr[i], ns, s);
            upload(h.dipvec, M.dipvec[i], 3 * (size_t)ns, s);
          }
          DevBuf<zdc> dpot(nt, s), dgrad(M.ifpgh > 1 ? 3 * (size_t)nt : 0, s);
          Inputs3D in = make_inputs3(ns, (const double*)h.zsrc.get(), M.ifcharge,
                                     (const double*)h.charge.get(), M.ifdipole,
                                     (const double*)h.dipstr.get(), (const double*)h.dipvec.get(),
                                     nt, (const double*)(same ? h.zsrc.get() : h.ztarg.get()),
                                     M.ifpgh);
          run_fmm3d(M.eps, M.zk, in, M.isep, dpot.get(), M.ifpgh > 1 ? dgrad.get() : nullptr, s);
          if (nt > 0) {
            ZF_CUDA(cudaMemcpyAsync(M.pot[i], dpot.get(), sizeof(zdc) * nt,
                                    cudaMemcpyDeviceToHost, s));
            if (M.ifpgh > 1)
              ZF_CUDA(cudaMemcpyAsync(M.grad[i], dgrad.get(), sizeof(zdc) * 3 * nt,
                                      cudaMemcpyDeviceToHost, s));
          }
          ZF_CUDA(cudaStreamSynchronize(s));
        } else {
          Inputs3D in = make_inputs3(ns, M.zsrc[i], M.ifcharge,
                                     M.ifcharge == 1 ? M.charge[i] : nullptr, M.ifdipole,
                                     M.ifdipole == 1 ? M.dipstr[i] : nullptr,
                                     M.ifdipole == 1 ? M.dipvec[i] : nullptr, nt, M.ztarg[i],
                                     M.ifpgh);
          run_fmm3d(M.eps, M.zk, in, M.isep, (zdc*)M.pot[i],
                    M.ifpgh > 1 ? (zdc*)M.grad[i] : nullptr, s);
          ZF_CUDA(cudaStreamSynchronize(s));
        }
        if (done_ms)
          done_ms[i] = std::chrono::duration<double, std::milli>(
                           std::chrono::steady_clock::now() - t0).count();
      }
    } catch (const zf_error& e) {
      std::lock_guard<std::mutex> lk(err_mu);
      if (!err_code) {
        err_code = e.code;
        err = e.what();
      }
    } catch (const std::exception& e) {
      std::lock_guard<std::mutex> lk(err_mu);
      if (!err_code) {
        err_code = ZF_ERR_INTERNAL;
        err = e.what();
      }
    }
    if (s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  };
  std::vector<std::thread> th;
  for (int w = 0; w < nworkers; w++) th.emplace_back(worker);
  for (auto& t : th) t.join();
  if (err_code) throw zf_error(err_code, err);
}

int many_impl(ManyArgs M, int nworkers, double* done_ms) {
  return guarded([&] {
    if (M.ninst < 0) throw zf_error(ZF_ERR_ARG, "ninst must be >= 0");
    if (M.ninst == 0) return;
    if (!M.ns || !M.nt || !M.zsrc || !M.ztarg || !M.pot)
      throw zf_error(ZF_ERR_ARG, "null instance array");
    clamp_flags(M.ifcharge, M.ifdipole, M.ifpgh);
    if (M.isep < 1) throw zf_error(ZF_ERR_ARG, "isep must be >= 1");
    for (int i = 0; i < M.ninst; i++) {
      check_args2d(M.ns[i], M.nt[i], M.zsrc[i], M.ztarg[i], M.ifcharge,
                   M.charge ? M.charge[i] : nullptr, M.ifdipole,
                   M.dipstr ? M.dipstr[i] : nullptr, M.dipvec ? M.dipvec[i] : nullptr,
                   M.pot[i], M.grad ? M.grad[i] : nullptr, M.ifpgh);
      if (!M.host)
        check_align_dev(M.zsrc[i], M.ztarg[i], M.ifcharge, M.charge ? M.charge[i] : nullptr,
                        M.ifdipole, M.dipstr ? M.dipstr[i] : nullptr,
                        M.dipvec ? M.dipvec[i] : nullptr, M.pot[i],
                        M.grad ? M.grad[i] : nullptr, M.ifpgh);
    }
    check_device();
    run_many(M, std::max(1, std::min(nworkers, 64)), done_ms);
  });
}

}  // namespace

extern "C" {

int zfmm_zlfmm3d_many(int ninst, double eps, const int* ns, const double* const* zsrc,
                      int ifcharge, const double* const* charge, int ifdipole,
                      const double* const* dipstr, const double* const* dipvec, const int* nt,
                      const double* const* ztarg, int ifpgh, int isep, double* const* pot,
                      double* const* grad, int nstreams, double* done_ms) {
  ManyArgs M{ninst, eps, nullptr, ns, nt, zsrc, charge, dipstr, dipvec, ztarg, pot, grad,
             ifcharge, ifdipole, ifpgh, isep, true};
  return many_impl(M, nstreams, done_ms);
}

int zfmm_zhfmm3d_many(int ninst, double eps, const double* zk, const int* ns,
                      const double* const* zsrc, int ifcharge, const double* const* charge,
                      int ifdipole, const double* const* dipstr, const double* const* dipvec,
                      const int* nt, const double* const* ztarg, int ifpgh, int isep,
                      double* const* pot, double* const* grad, int nstreams, double* done_ms) {
  if (!zk) return fail(ZF_ERR_ARG, "zk is null");
  zdc k = mkz(zk[0], zk[1]);
  ManyArgs M{ninst, eps, &k, ns, nt, zsrc, charge, dipstr, dipvec, ztarg, pot, grad,
             ifcharge, ifdipole, ifpgh, isep, true};
  return many_impl(M, nstreams, done_ms);
}

int zfmm_zlfmm3d_many_dev(int ninst, double eps, const int* ns, const double* const* zsrc,
                          int ifcharge, const double* const* charge, int ifdipole,
                          const double* const* dipstr, const double* const* dipvec,
                          const int* nt, const double* const* ztarg, int ifpgh, int isep,
                          double* const* pot, double* const* grad, int nstreams,
                          double* done_ms) {
  ManyArgs M{ninst, eps, nullptr, ns, nt, zsrc, charge, dipstr, dipvec, ztarg, pot, grad,
             ifcharge, ifdipole, ifpgh, isep, false};
  return many_impl(M, nstreams, done_ms);
}

int zfmm_zhfmm3d_many_dev(int ninst, double eps, const double* zk, const int* ns,
                          const double* const* zsrc, int ifcharge, const double* const* charge,
                          int ifdipole, const double* const* dipstr,
                          const double* const* dipvec, const int* nt,
                          const double* const* ztarg, int ifpgh, int isep, double* const* pot,
                          double* const* grad, int nstreams, double* done_ms) {
  if (!zk) return fail(ZF_ERR_ARG, "zk is null");
  zdc k = mkz(zk[0], zk[1]);
  ManyArgs M{ninst, eps, &k, ns, nt, zsrc, charge, dipstr, dipvec, ztarg, pot, grad,
             ifcharge, ifdipole, ifpgh, isep, false};
  return many_impl(M, nstreams, done_ms);
}

}  // extern "C"

// ---- 2D plans ----------------------------------------------------------------
struct zfmm_plan2d_s {
  zf::Plan2D P;
};

namespace {

int plan2d_create_impl(double eps, int ns, const double* zsrc, int nt, const double* ztarg,
                       int isep, bool host, cudaStream_t s, zfmm_plan2d_s** out) {
  return guarded([&] {
    if (!out) throw zf_error(ZF_ERR_ARG, "null plan output");
    *out = nullptr;
    if (ns < 0 || nt < 0) throw zf_error(ZF_ERR_ARG, "ns and nt must be >= 0");
    if ((ns > 0 && !zsrc) || (nt > 0 && !ztarg))
      throw zf_error(ZF_ERR_ARG, "null coordinate array");
    if (isep < 1) throw zf_error(ZF_ERR_ARG, "isep must be >= 1");
    check_device();
    auto* pl = new zfmm_plan2d_s();
    try {
      HostIn h;
      const zdc* zs = reinterpret_cast<const zdc*>(zsrc);
      const zdc* zt = reinterpret_cast<const zdc*>(ztarg);
      if (!host) check_align16({zsrc, ztarg});
      if (host) {
        // targets passed as the source array itself: uploaded once
        const bool same = ztarg == zsrc && nt == ns;
        upload(h.zsrc, zsrc, 2 * (size_t)ns, s);
        if (!same) upload(h.ztarg, ztarg, 2 * (size_t)nt, s);
        zs = h.zsrc.get();
        zt = same ? zs : h.ztarg.get();
      }
      if (ns > 0 && nt > 0) plan2d_build(pl->P, eps, ns, zs, nt, zt, isep, s);
      else {
        pl->P.eps = eps;
        pl->P.isep = isep;
        pl->P.ns = ns;
        pl->P.nt = nt;
        ZF_CUDA(cudaGetDevice(&pl->P.device));
      }
      ZF_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
      delete pl;
      throw;
    }
    *out = pl;
  });
}

void check_plan2d_args(zfmm_plan2d_s* plan, int nd, int ifcharge, const double* charge,
                       int ifdipole, const double* dipstr, const double* dipvec, int ifpgh,
                       double* pot, double* grad) {
  if (!plan) throw zf_error(ZF_ERR_ARG, "plan is null");
  if (nd < 1) throw zf_error(ZF_ERR_ARG, "nd must be >= 1");
  const Plan2D& P = plan->P;
  if (P.ns > 0 && ifcharge == 1 && !charge) throw zf_error(ZF_ERR_ARG, "ifcharge=1 needs charge");
  if (P.ns > 0 && ifdipole == 1 && (!dipstr || !dipvec))
    throw zf_error(ZF_ERR_ARG, "ifdipole=1 needs dipstr and dipvec");
  if (P.nt > 0 && !pot) throw zf_error(ZF_ERR_ARG, "null pot");
  if (P.nt > 0 && ifpgh > 1 && !grad) throw zf_error(ZF_ERR_ARG, "ifpgh=2 needs grad");
  int dev = 0;
  ZF_CUDA(cudaGetDevice(&dev));
  if (dev != P.device) throw zf_error(ZF_ERR_ARG, "plan was built on another device");
}

void run_plan2d(zfmm_plan2d_s* plan, const zdc* zk, int nd, int ifcharge, const zdc* charge,
                int ifdipole, const zdc* dipstr, const zdc* dipvec, int ifpgh, zdc* pot,
                zdc* grad, cudaStream_t s) {
  const Plan2D& P = plan->P;
  if (P.nt > 0) {
    ZF_CUDA(cudaMemsetAsync(pot, 0, sizeof(zdc) * P.nt * (size_t)nd, s));
    if (ifpgh > 1) ZF_CUDA(cudaMemsetAsync(grad, 0, sizeof(zdc) * 2 * P.nt * (size_t)nd, s));
  }
  if (P.ns == 0 || P.nt == 0) return;
  StepTimes t;
  t.want_counts = g_timing >= 2;
  fmm2d_plan_execute(P, zk, nd, ifcharge, charge, ifdipole, dipstr, dipvec, ifpgh, pot,
                     ifpgh > 1 ? grad : nullptr, s, g_timing ? &t : nullptr);
  if (g_timing) g_times = t;
}

int plan2d_solve(zfmm_plan2d plan, const double* zk, int nd, int ifcharge, const double* charge,
                 int ifdipole, const double* dipstr, const double* dipvec, int ifpgh, double* pot,
                 double* grad, bool host, void* stream) {
  return guarded([&] {
    clamp_flags(ifcharge, ifdipole, ifpgh);
    check_plan2d_args(plan, nd, ifcharge, charge, ifdipole, dipstr, dipvec, ifpgh, pot, grad);
    zdc k = zk ? mkz(zk[0], zk[1]) : mkz(0.0);
    const zdc* kp = zk ? &k : nullptr;
    if (!host) {
      check_align16({pot, ifcharge == 1 ? charge : nullptr, ifdipole == 1 ? dipstr : nullptr,
                     ifdipole == 1 ? dipvec : nullptr, ifpgh > 1 ? grad : nullptr});
      cudaStream_t s = (cudaStream_t)stream;
      run_plan2d(plan, kp, nd, ifcharge, (const zdc*)charge, ifdipole, (const zdc*)dipstr,
                 (const zdc*)dipvec, ifpgh, (zdc*)pot, (zdc*)grad, s);
      ZF_CUDA(cudaStreamSynchronize(s));
      return;
    }
    const int ns = plan->P.ns, nt = plan->P.nt;
    cudaStream_t s = cudaStreamPerThread;
    HostIn h;
    if (ifcharge == 1) upload(h.charge, charge, (size_t)nd * ns, s);
    if (ifdipole == 1) {
      upload(h.dipstr, dipstr, (size_t)nd * ns, s);
      upload(h.dipvec, dipvec, 2 * (size_t)ns, s);
    }
    DevBuf<zdc> dpot((size_t)nd * nt, s), dgrad(ifpgh > 1 ? 2 * (size_t)nd * nt : 0, s);
    run_plan2d(plan, kp, nd, ifcharge, h.charge.get(), ifdipole, h.dipstr.get(),
               h.dipvec.get(), ifpgh, dpot.get(), dgrad.get(), s);
    if (nt > 0) {
      ZF_CUDA(cudaMemcpyAsync(pot, dpot.get(), sizeof(zdc) * nt * (size_t)nd,
                              cudaMemcpyDeviceToHost, s));
      if (grad) {
        if (ifpgh > 1)
          ZF_CUDA(cudaMemcpyAsync(grad, dgrad.get(), sizeof(zdc) * 2 * nt * (size_t)nd,
                                  cudaMemcpyDeviceToHost, s));
        else
          memset(grad, 0, sizeof(zdc) * 2 * nt * (size_t)nd);
      }
    }
    ZF_CUDA(cudaStreamSynchronize(s));
  });
}

}  // namespace

extern "C" {

int zfmm_plan2d_create(double eps, int ns, const double* zsrc, int nt, const double* ztarg,
                       int isep, zfmm_plan2d* plan) {
  return plan2d_create_impl(eps, ns, zsrc, nt, ztarg, isep, true, cudaStreamPerThread, plan);
}

int zfmm_plan2d_create_dev(double eps, int ns, const double* zsrc, int nt, const double* ztarg,
                           int isep, void* stream, zfmm_plan2d* plan) {
  return plan2d_create_impl(eps, ns, zsrc, nt, ztarg, isep, false, (cudaStream_t)stream, plan);
}

int zfmm_plan2d_destroy(zfmm_plan2d plan) {
  return guarded([&] {
    if (!plan) return;
    ZF_CUDA(cudaDeviceSynchronize());
    delete plan;
  });
}

int zfmm_plan2d_info(zfmm_plan2d plan, int* nboxes, int* nlevels, int* ns, int* nt) {
  return guarded([&] {
    if (!plan) throw zf_error(ZF_ERR_ARG, "plan is null");
    if (nboxes) *nboxes = plan->P.S.tree.nboxes;
    if (nlevels) *nlevels = plan->P.S.tree.nlevels;
    if (ns) *ns = plan->P.ns;
    if (nt) *nt = plan->P.nt;
  });
}

int zfmm_zlfmm2d_plan(zfmm_plan2d plan, int nd, int ifcharge, const double* charge,
                      int ifdipole, const double* dipstr, const double* dipvec, int ifpgh,
                      double* pot, double* grad) {
  return plan2d_solve(plan, nullptr, nd, ifcharge, charge, ifdipole, dipstr, dipvec, ifpgh, pot,
                      grad, true, nullptr);
}

int zfmm_zlfmm2d_plan_dev(zfmm_plan2d plan, int nd, int ifcharge, const double* charge,
                          int ifdipole, const double* dipstr, const double* dipvec, int ifpgh,
                          double* pot, double* grad, void* stream) {
  return plan2d_solve(plan, nullptr, nd, ifcharge, charge, ifdipole, dipstr, dipvec, ifpgh, pot,
                      grad, false, stream);
}

int zfmm_zhfmm2d_plan(zfmm_plan2d plan, const double* zk, int nd, int ifcharge,
                      const double* charge, int ifdipole, const double* dipstr,
                      const double* dipvec, int ifpgh, double* pot, double* grad) {
  if (!zk) return fail(ZF_ERR_ARG, "zk is null");
  return plan2d_solve(plan, zk, nd, ifcharge, charge, ifdipole, dipstr, dipvec, ifpgh, pot, grad,
                      true, nullptr);
}

int zfmm_zhfmm2d_plan_dev(zfmm_plan2d plan, const double* zk, int nd, int ifcharge,
                          const double* charge, int ifdipole, const double* dipstr,
                          const double* dipvec, int ifpgh, double* pot, double* grad,
                          void* stream) {
  if (!zk) return fail(ZF_ERR_ARG, "zk is null");
  return plan2d_solve(plan, zk, nd, ifcharge, charge, ifdipole, dipstr, dipvec, ifpgh, pot, grad,
                      false, stream);
}

}  // extern "C"

// ---- plan files ----------------------------------------------------------------
extern "C" {

int zfmm_plan2d_save(zfmm_plan2d plan, const char* path) {
  return guarded([&] {
    if (!plan || !path) throw zf_error(ZF_ERR_ARG, "plan or path is null");
    if (plan->P.ns == 0 || plan->P.nt == 0) throw zf_error(ZF_ERR_ARG, "empty plan");
    plan2d_save(plan->P, path, cudaStreamPerThread);
  });
}

int zfmm_plan2d_load(const char* path, zfmm_plan2d* out) {
  return guarded([&] {
    if (!path || !out) throw zf_error(ZF_ERR_ARG, "path or plan output is null");
    *out = nullptr;
    check_device();
    auto* pl = new zfmm_plan2d_s();
    try {
      plan2d_load(pl->P, path, cudaStreamPerThread);
    } catch (...) {
      delete pl;
      throw;
    }
    *out = pl;
  });
}

int zfmm_plan3d_save(zfmm_plan3d plan, const char* path) {
  return guarded([&] {
    if (!plan || !path) throw zf_error(ZF_ERR_ARG, "plan or path is null");
    if (plan->P.ns == 0 || plan->P.nt == 0) throw zf_error(ZF_ERR_ARG, "empty plan");
    plan3d_save(plan->P, path, cudaStreamPerThread);
  });
}

int zfmm_plan3d_load(const char* path, zfmm_plan3d* out) {
  return guarded([&] {
    if (!path || !out) throw zf_error(ZF_ERR_ARG, "path or plan output is null");
    *out = nullptr;
    check_device();
    auto* pl = new zfmm_plan3d_s();
    try {
      plan3d_load(pl->P, path, cudaStreamPerThread);
    } catch (...) {
      delete pl;
      throw;
    }
    *out = pl;
  });
}

}  // extern "C"
