// Launch-shape autotuner.
//
// The thread-per-item kernels of the 2D Helmholtz passes (translation tables,
// P2M / P2L columns, L2T + M2T per target) and the warp-per-leaf P2P run with
// a block size chosen per (kernel, work-size bucket, device).  With tuning off
// (the default) every kernel uses its fixed default.  With tuning on
// (zfmm_set_autotune(1) or ZFMM_AUTOTUNE=1 in the environment) the first call
// of a (kernel, bucket, device) times every candidate block size with CUDA
// events on the call's stream (each candidate twice, the second timed) and
// keeps the fastest; later calls reuse it.  Results do not depend on the
// block size (every item is computed by one thread or one warp the same way),
// so tuning changes timings only.  The table can be written to and read from
// a text file (zfmm_autotune_save / zfmm_autotune_load), one line per entry:
// "<kernel> <bucket> <device> <block>".
#pragma once
#include <functional>
#include <string>
#include <vector>
#include <cuda_runtime.h>

namespace zf {

bool autotune_enabled();

// Runs `launch(block)` at least once, with the block size tuned (or cached,
// or the default when tuning is off) for kernel `name` and `work` items.
// When the kernel is not idempotent, `reset` (optional) restores its outputs
// before every timed candidate and before the final run.
int tuned_launch(const char* name, long work, int dflt, const std::vector<int>& cands,
                 const std::function<void(int)>& launch, cudaStream_t s,
                 const std::function<void()>& reset = nullptr);

}  // namespace zf
