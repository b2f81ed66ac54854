// Direct summation zl2devaldirect over all source-target pairs
// (zfmm2d/src/laplace/zlfmm2d.f:600-654) on the device.
//
// One thread per target; sources are staged through shared memory in tiles of
// TILE points (coalesced 16-byte loads of the complex coordinates and
// strengths).  When there are too few targets to fill the 148 SMs, the sources
// are split into `nsplit` slices: each slice writes partial sums to scratch
// memory and a second kernel adds the slices into pot/grad.  Like the
// reference routine, the sums are unscaled and are ADDED to pot/grad.
#include <algorithm>
#include <mutex>
#include "helm2d_pair.cuh"
#include "hfmm2d.cuh"
#include "lap2d_pair.cuh"
#include "lfmm2d.cuh"

namespace zf {
namespace {

constexpr int DTB = 128;   // threads (targets) per block
constexpr int TILE = 128;  // sources per shared-memory tile

template <bool GRAD, bool HELM>
__global__ void __launch_bounds__(DTB) k_direct2d(Inputs2D in, zdc zk, int chunk, zdc* pot,
                                                 zdc* grad, zdc* part) {
  __shared__ zdc sy[TILE][6];  // y1, y2, q, ds, d1, d2
  int i = blockIdx.x * DTB + threadIdx.x;
  int j0 = blockIdx.y * chunk, j1 = min(in.ns, j0 + chunk);
  bool valid = i < in.nt;
  zdc x1 = mkz(0.0), x2 = mkz(0.0);
  if (valid) {
    x1 = ldz(&in.ztarg[2 * i]);
    x2 = ldz(&in.ztarg[2 * i + 1]);
  }
  zdc p = mkz(0.0), g1 = mkz(0.0), g2 = mkz(0.0);
  const HelmK K = helm_k(zk);
  for (int t = j0; t < j1; t += TILE) {
    int n = min(TILE, j1 - t);
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += DTB) {
      int j = t + k;
      sy[k][0] = ldz(&in.zsrc[2 * j]);
      sy[k][1] = ldz(&in.zsrc[2 * j + 1]);
      sy[k][2] = in.ifcharge ? ldz(&in.charge[j]) : mkz(0.0);
      if (in.ifdipole) {
        sy[k][3] = ldz(&in.dipstr[j]);
        sy[k][4] = ldz(&in.dipvec[2 * j]);
        sy[k][5] = ldz(&in.dipvec[2 * j + 1]);
      } else {
        sy[k][3] = sy[k][4] = sy[k][5] = mkz(0.0);
      }
    }
    __syncthreads();
    if (valid)
      for (int k = 0; k < n; k++) {
        if (HELM)
          helm_pair<GRAD>(K, x1, x2, sy[k][0], sy[k][1], sy[k][2], sy[k][3], sy[k][4], sy[k][5],
                          in.ifcharge, in.ifdipole, p, g1, g2);
        else
          lap2d_pair<GRAD>(x1, x2, sy[k][0], sy[k][1], sy[k][2], sy[k][3], sy[k][4], sy[k][5],
                           in.ifcharge, in.ifdipole, p, g1, g2);
      }
  }
  if (!valid) return;
  if (part == nullptr) {
    pot[i] += p;
    if (GRAD) {
      grad[2 * i] += g1;
      grad[2 * i + 1] += g2;
    }
  } else {
    size_t st = (size_t)in.nt * (GRAD ? 3 : 1);
    zdc* q = part + blockIdx.y * st;
    q[i] = p;
    if (GRAD) {
      q[in.nt + i] = g1;
      q[2 * (size_t)in.nt + i] = g2;
    }
  }
}

template <bool GRAD>
__global__ void k_direct2d_reduce(int nt, int nsplit, const zdc* part, zdc* pot, zdc* grad) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nt) return;
  size_t st = (size_t)nt * (GRAD ? 3 : 1);
  zdc p = mkz(0.0), g1 = mkz(0.0), g2 = mkz(0.0);
  for (int k = 0; k < nsplit; k++) {
    const zdc* q = part + k * st;
    p += q[i];
    if (GRAD) {
      g1 += q[nt + i];
      g2 += q[2 * (size_t)nt + i];
    }
  }
  pot[i] += p;
  if (GRAD) {
    grad[2 * i] += g1;
    grad[2 * i + 1] += g2;
  }
}

int choose_split(int nt, int ns) {
  int tblocks = div_up(nt, DTB);
  int want = 4 * 148;  // enough resident blocks for all SMs
  int ns_max = std::max(1, div_up(ns, 4 * TILE));
  int nsplit = std::max(1, std::min(ns_max, div_up(want, tblocks)));
  return std::min(nsplit, 64);
}

}  // namespace

size_t direct2d_scratch_elems(int nt, int ns, int ifpgh) {
  int nsplit = choose_split(nt, ns);
  if (nsplit == 1) return 0;
  return (size_t)nsplit * nt * (ifpgh > 1 ? 3 : 1);
}

namespace {
template <bool HELM>
void direct2d_run(const Inputs2D& in, zdc zk, zdc* pot, zdc* grad, zdc* scratch, cudaStream_t s) {
  if (in.nt <= 0 || in.ns <= 0) return;
  int nsplit = choose_split(in.nt, in.ns);
  int chunk = div_up(in.ns, nsplit);
  nsplit = div_up(in.ns, chunk);
  DevBuf<zdc> own;
  zdc* part = nullptr;
  if (nsplit > 1) {
    size_t need = (size_t)nsplit * in.nt * (in.ifpgh > 1 ? 3 : 1);
    if (scratch) {
      part = scratch;
    } else {
      own.alloc(need, s);
      part = own.get();
    }
  }
  dim3 grid(div_up(in.nt, DTB), nsplit);
  if (in.ifpgh > 1) {
    klaunch(k_direct2d<true, HELM>, grid, DTB, 0, s, in, zk, chunk, pot, grad, part);
    if (part) klaunch(k_direct2d_reduce<true>, div_up(in.nt, 256), 256, 0, s, in.nt, nsplit, part, pot, grad);
  } else {
    klaunch(k_direct2d<false, HELM>, grid, DTB, 0, s, in, zk, chunk, pot, grad, part);
    if (part) klaunch(k_direct2d_reduce<false>, div_up(in.nt, 256), 256, 0, s, in.nt, nsplit, part, pot, grad);
  }
  ZF_LAUNCH_CHECK();
}
}  // namespace

void zl2ddirect_device(const Inputs2D& in, zdc* pot, zdc* grad, zdc* scratch, cudaStream_t s) {
  direct2d_run<false>(in, mkz(0.0), pot, grad, scratch, s);
}

void zh2ddirect_device(zdc zk, const Inputs2D& in, zdc* pot, zdc* grad, cudaStream_t s) {
  direct2d_run<true>(in, zk, pot, grad, nullptr, s);
}

// ---- allocation-free variant ----------------------------------------------
// Scratch of the source-split direct sum lives in this fixed device array
// (8 MiB, held by every GPU that loads the library until the process exits).
// Each call overwrites every partial it reads, so nothing has to be cleared
// between calls; calls that overlap on the GPU (two streams, or two host
// threads) share the array and race.
constexpr size_t kNoAllocScratchElems = (size_t)1 << 19;  // complex elements = 8 MiB
static __device__ __align__(256) zdc g_direct2d_scratch[kNoAllocScratchElems];

namespace {
std::mutex g_scratch_mu;
zdc* g_scratch_ptr[64] = {nullptr};
}  // namespace

size_t direct2d_noalloc_capacity() { return kNoAllocScratchElems; }

// Device address of the scratch array on the current device.  The array's
// name is only a host-side stand-in, so the address is taken once per device
// with cudaGetSymbolAddress (on the first call made on that device).
static zdc* noalloc_scratch() {
  int dev = 0;
  ZF_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) throw zf_error(ZF_ERR_ARG, "device index out of range");
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    ZF_CUDA(cudaGetSymbolAddress(&p, g_direct2d_scratch));
    g_scratch_ptr[dev] = static_cast<zdc*>(p);
  }
  return g_scratch_ptr[dev];
}

void zl2ddirect_device_noalloc(const Inputs2D& in, zdc* pot, zdc* grad, cudaStream_t s) {
  size_t need = direct2d_scratch_elems(in.nt, in.ns, in.ifpgh);
  if (need > kNoAllocScratchElems)
    throw zf_error(ZF_ERR_ARG, "problem needs " + std::to_string(need * sizeof(zdc)) +
                                   " bytes of scratch, more than the fixed " +
                                   std::to_string(kNoAllocScratchElems * sizeof(zdc)) +
                                   " bytes of the allocation-free entry point");
  zl2ddirect_device(in, pot, grad, noalloc_scratch(), s);
}

}  // namespace zf
