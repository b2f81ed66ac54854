/*
 * zfmm_b200 C ABI: B200 (sm_100a) complex-coordinate fast multipole methods.
 *
 * Complex arrays are interleaved (re, im) doubles in Fortran column-major
 * order, exactly the memory of the reference's `complex *16` arrays:
 *   zsrc(d, ns)  -> double[2*d*ns]   (point i, coordinate k at 2*(d*i+k))
 *   charge(ns), dipstr(ns) -> double[2*ns]
 *   dipvec(d, ns) -> double[2*d*ns], pot(nt) -> double[2*nt],
 *   grad(d, nt) -> double[2*d*nt]
 * Integers are 32-bit (the reference's default INTEGER).
 *
 * Two families of entry points:
 *   zlfmm2d_ ...            Fortran-callable (every argument by reference, host
 *                           arrays, trailing underscore); drop-in replacements
 *                           for the reference subroutines.  Like the reference
 *                           they sanitise ifcharge/ifdipole/ifpgh in place and
 *                           report no status (a failure leaves pot/grad zero
 *                           and is readable through zfmm_last_error()).
 *   zfmm_zlfmm2d ...        C entry points returning a status (0 = success),
 *                           host arrays; the *_dev variants take device
 *                           pointers and a cudaStream_t (as void*).
 *
 * Device pointers (every *_dev, *_plan_dev, *_many_dev and *_noalloc entry
 * point) must be 16-byte aligned, as cudaMalloc and torch allocations are:
 * the kernels access complex values as 16-byte pairs.  A misaligned pointer is
 * refused with status 1 before anything is launched.  Host arrays have no
 * alignment requirement.
 *
 * Status codes: 0 ok, 1 bad argument, 2 CUDA error, 3 out of device memory,
 * 4 internal error, 5 the CUDA library is unavailable (no GPU).
 */
#ifndef ZFMM_B200_H
#define ZFMM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces zlfmm2d (zfmm2d/src/laplace/zlfmm2d.f:14-15; MATLAB spec
 * zfmm2d/matlab_linux/zlfmm2d.mw:7).  pot = sum q log(R)/2pi - ..., see the
 * reference header comment (zlfmm2d.f:1-12). */
void zlfmm2d_(const double *eps, const int *ns, const double *zsrc, int *ifcharge,
              const double *charge, int *ifdipole, const double *dipstr, const double *dipvec,
              double *pot, double *grad, const int *nt, const double *ztarg, int *ifpgh,
              const int *isep, const int *ifprint);

/* Replaces zl2devaldirect (zfmm2d/src/laplace/zlfmm2d.f:600-601; MATLAB spec
 * zfmm2d/matlab_linux/zl2devaldirect.mw:6).  Adds the UNSCALED sums
 * (no 1/2pi) into pot/grad, as the reference routine does. */
void zl2devaldirect_(const int *nt, const double *ztarg, const int *ns, const double *zsrc,
                     const double *charge, const double *dipstr, const double *dipvec,
                     const int *ifcharge, double *pot, double *grad, const int *ifdipole,
                     const int *ifpgh);

/* Replaces zhfmm2d (zfmm2d/src/helmholtz/zhfmm2d.f:14-15; MATLAB spec
 * zfmm2d/matlab_linux/zhfmm2d.mw:7).  zk points to one complex (re, im).
 * pot = sum (i/4) q H0(zk R) + dipole terms (zhfmm2d.f:1-12). */
void zhfmm2d_(const double *eps, const double *zk, const int *ns, const double *zsrc,
              int *ifcharge, const double *charge, int *ifdipole, const double *dipstr,
              const double *dipvec, double *pot, double *grad, const int *nt,
              const double *ztarg, int *ifpgh, const int *isep, const int *ifprint);

/* Replaces zh2devaldirect (zfmm2d/src/helmholtz/zhfmm2d.f:773-774; MATLAB spec
 * zfmm2d/matlab_linux/zh2devaldirect.mw:6).  Adds the UNSCALED sums (no i/4). */
void zh2devaldirect_(const double *zk, const int *nt, const double *ztarg, const int *ns,
                     const double *zsrc, const double *charge, const double *dipstr,
                     const double *dipvec, const int *ifcharge, double *pot, double *grad,
                     const int *ifdipole, const int *ifpgh);

/* Replaces zlfmm3d (zfmm3d/src/laplace/zlfmm3d.f:14-15; MATLAB spec
 * zfmm3d/matlab_linux/zlfmm3d.mw:1).  pot = sum q/(4 pi R) + dipole terms;
 * the driver rescales the geometry to a unit root box internally and returns
 * grad in the caller's units (zlfmm3d.f:187-200, :236-240). */
void zlfmm3d_(const double *eps, const int *ns, const double *zsrc, int *ifcharge,
              const double *charge, int *ifdipole, const double *dipstr, const double *dipvec,
              double *pot, double *grad, const int *nt, const double *ztarg, int *ifpgh,
              const int *isep, const int *ifprint);

/* Replaces zl3devaldirect (zfmm3d/src/laplace/zlfmm3d.f:628-629; MATLAB spec
 * zfmm3d/matlab_linux/zl3devaldirect.mw:1).  ADDS the sums (with 1/(4 pi))
 * into pot/grad, as the reference routine does. */
void zl3devaldirect_(const int *nt, const double *ztarg, const int *ns, const double *zsrc,
                     const double *charge, const double *dipstr, const double *dipvec,
                     const int *ifcharge, double *pot, double *grad, const int *ifdipole,
                     const int *ifpgh);

/* Replaces zhfmm3d (zfmm3d/src/helmholtz/zhfmm3d.f:1-2; MATLAB spec
 * zfmm3d/matlab_linux/zhfmm3d.mw:1).  zk points to one complex (re, im).
 * pot = sum q e^{i k R}/(4 pi R) + dipole terms; the driver rescales the
 * geometry to a unit root box (wavenumber zk*boxsize(0)) internally. */
void zhfmm3d_(const double *eps, const double *zk, const int *ns, const double *zsrc,
              int *ifcharge, const double *charge, int *ifdipole, const double *dipstr,
              const double *dipvec, double *pot, double *grad, const int *nt,
              const double *ztarg, int *ifpgh, const int *isep, const int *ifprint);

/* Replaces zh3devaldirect (zfmm3d/src/helmholtz/zhfmm3d.f:626-627; MATLAB spec
 * zfmm3d/matlab_linux/zh3devaldirect.mw:1).  ADDS the sums (with 1/(4 pi)). */
void zh3devaldirect_(const double *zk, const int *nt, const double *ztarg, const int *ns,
                     const double *zsrc, const double *charge, const double *dipstr,
                     const double *dipvec, const int *ifcharge, double *pot, double *grad,
                     const int *ifdipole, const int *ifpgh);

/* C forms of the above (host arrays).  Flags are not modified; out-of-range
 * flags are clamped the same way as the reference (zlfmm2d.f:58-68). */
int zfmm_zlfmm2d(double eps, int ns, const double *zsrc, int ifcharge, const double *charge,
                 int ifdipole, const double *dipstr, const double *dipvec, double *pot,
                 double *grad, int nt, const double *ztarg, int ifpgh, int isep, int ifprint);
int zfmm_zl2devaldirect(int nt, const double *ztarg, int ns, const double *zsrc,
                        const double *charge, const double *dipstr, const double *dipvec,
                        int ifcharge, double *pot, double *grad, int ifdipole, int ifpgh);

int zfmm_zhfmm2d(double eps, const double *zk, int ns, const double *zsrc, int ifcharge,
                 const double *charge, int ifdipole, const double *dipstr, const double *dipvec,
                 double *pot, double *grad, int nt, const double *ztarg, int ifpgh, int isep,
                 int ifprint);
int zfmm_zh2devaldirect(const double *zk, int nt, const double *ztarg, int ns, const double *zsrc,
                        const double *charge, const double *dipstr, const double *dipvec,
                        int ifcharge, double *pot, double *grad, int ifdipole, int ifpgh);

/* Device-pointer forms: every array is device memory, work is queued on
 * `stream` (a cudaStream_t; NULL = legacy default stream).  The FMM returns
 * after its results are complete on that stream. */
int zfmm_zlfmm2d_dev(double eps, int ns, const double *zsrc, int ifcharge, const double *charge,
                     int ifdipole, const double *dipstr, const double *dipvec, double *pot,
                     double *grad, int nt, const double *ztarg, int ifpgh, int isep,
                     void *stream);
int zfmm_zl2devaldirect_dev(int nt, const double *ztarg, int ns, const double *zsrc,
                            const double *charge, const double *dipstr, const double *dipvec,
                            int ifcharge, double *pot, double *grad, int ifdipole, int ifpgh,
                            void *stream);

int zfmm_zhfmm2d_dev(double eps, const double *zk, int ns, const double *zsrc, int ifcharge,
                     const double *charge, int ifdipole, const double *dipstr,
                     const double *dipvec, double *pot, double *grad, int nt, const double *ztarg,
                     int ifpgh, int isep, void *stream);
int zfmm_zh2devaldirect_dev(const double *zk, int nt, const double *ztarg, int ns,
                            const double *zsrc, const double *charge, const double *dipstr,
                            const double *dipvec, int ifcharge, double *pot, double *grad,
                            int ifdipole, int ifpgh, void *stream);

/* 3D Laplace, C forms: host arrays, then device pointers on `stream`. */
int zfmm_zlfmm3d(double eps, int ns, const double *zsrc, int ifcharge, const double *charge,
                 int ifdipole, const double *dipstr, const double *dipvec, double *pot,
                 double *grad, int nt, const double *ztarg, int ifpgh, int isep, int ifprint);
int zfmm_zl3devaldirect(int nt, const double *ztarg, int ns, const double *zsrc,
                        const double *charge, const double *dipstr, const double *dipvec,
                        int ifcharge, double *pot, double *grad, int ifdipole, int ifpgh);
int zfmm_zlfmm3d_dev(double eps, int ns, const double *zsrc, int ifcharge, const double *charge,
                     int ifdipole, const double *dipstr, const double *dipvec, double *pot,
                     double *grad, int nt, const double *ztarg, int ifpgh, int isep,
                     void *stream);
int zfmm_zl3devaldirect_dev(int nt, const double *ztarg, int ns, const double *zsrc,
                            const double *charge, const double *dipstr, const double *dipvec,
                            int ifcharge, double *pot, double *grad, int ifdipole, int ifpgh,
                            void *stream);
/* Expansion order of the 3D Laplace FMM for eps; replaces zl3dterms
 * (zfmm3d/src/laplace/zlfmm3d.f:1283-1321).  Host computation. */
int zfmm_zl3dterms(double eps);

/* 3D Helmholtz, C forms: host arrays, then device pointers on `stream`. */
int zfmm_zhfmm3d(double eps, const double *zk, int ns, const double *zsrc, int ifcharge,
                 const double *charge, int ifdipole, const double *dipstr, const double *dipvec,
                 double *pot, double *grad, int nt, const double *ztarg, int ifpgh, int isep,
                 int ifprint);
int zfmm_zh3devaldirect(const double *zk, int nt, const double *ztarg, int ns, const double *zsrc,
                        const double *charge, const double *dipstr, const double *dipvec,
                        int ifcharge, double *pot, double *grad, int ifdipole, int ifpgh);
int zfmm_zhfmm3d_dev(double eps, const double *zk, int ns, const double *zsrc, int ifcharge,
                     const double *charge, int ifdipole, const double *dipstr,
                     const double *dipvec, double *pot, double *grad, int nt, const double *ztarg,
                     int ifpgh, int isep, void *stream);
int zfmm_zh3devaldirect_dev(const double *zk, int nt, const double *ztarg, int ns,
                            const double *zsrc, const double *charge, const double *dipstr,
                            const double *dipvec, int ifcharge, double *pot, double *grad,
                            int ifdipole, int ifpgh, void *stream);
/* Expansion order of the 3D Helmholtz FMM for a box of (rescaled) size
 * `size` and wavenumber zk = (re, im); replaces h3dterms
 * (zfmm3d/src/helmholtz/h3dterms.f:16-75).  Host computation. */
int zfmm_h3dterms(double size, const double *zk, double eps, int isep);

/* 3D plans (no counterpart in the reference, whose drivers rebuild the tree
 * on every call): the octree, sorted points, complex box centres and
 * interaction lists of one geometry, built once (zlfmm3d.f:60-200 /
 * zhfmm3d.f:60-200 up to the expansions) and reused by any number of solves,
 * each with nd right-hand sides.  The tree depends on eps, the points and isep
 * only, so one plan serves both kernels and every wavenumber.  Arrays of a
 * solve follow the right-hand-side-fastest convention: charge(nd, ns),
 * dipstr(nd, ns), pot(nd, nt), grad(nd, 3, nt); dipvec(3, ns) is shared by all
 * right-hand sides.  A solve with nd = 1 gives the same values as
 * zfmm_zlfmm3d on the same points (to rounding).  create: host arrays, or
 * device pointers on `stream` for _dev; destroy waits for the device. */
typedef struct zfmm_plan3d_s *zfmm_plan3d;
int zfmm_plan3d_create(double eps, int ns, const double *zsrc, int nt, const double *ztarg,
                       int isep, zfmm_plan3d *plan);
int zfmm_plan3d_create_dev(double eps, int ns, const double *zsrc, int nt, const double *ztarg,
                           int isep, void *stream, zfmm_plan3d *plan);
int zfmm_plan3d_destroy(zfmm_plan3d plan);
int zfmm_plan3d_info(zfmm_plan3d plan, int *nboxes, int *nlevels, int *ns, int *nt);
/* 3D Laplace solves on a plan: host arrays, or device pointers on `stream`. */
int zfmm_zlfmm3d_plan(zfmm_plan3d plan, int nd, int ifcharge, const double *charge,
                      int ifdipole, const double *dipstr, const double *dipvec, int ifpgh,
                      double *pot, double *grad);
int zfmm_zlfmm3d_plan_dev(zfmm_plan3d plan, int nd, int ifcharge, const double *charge,
                          int ifdipole, const double *dipstr, const double *dipvec, int ifpgh,
                          double *pot, double *grad, void *stream);
/* 3D Helmholtz solves on a plan, wavenumber zk = (re, im): the plan's tree is
 * reused for every wavenumber and right-hand side. */
int zfmm_zhfmm3d_plan(zfmm_plan3d plan, const double *zk, int nd, int ifcharge,
                      const double *charge, int ifdipole, const double *dipstr,
                      const double *dipvec, int ifpgh, double *pot, double *grad);
int zfmm_zhfmm3d_plan_dev(zfmm_plan3d plan, const double *zk, int nd, int ifcharge,
                          const double *charge, int ifdipole, const double *dipstr,
                          const double *dipvec, int ifpgh, double *pot, double *grad,
                          void *stream);

/* 2D plans, as the 3D ones: the quadtree, sorted points, complex centres and
 * lists of one geometry (zlfmm2d.f:70-200 / zhfmm2d.f:73-195) built once and
 * reused by solves of nd right-hand sides at any wavenumber: charge(nd, ns),
 * dipstr(nd, ns), pot(nd, nt), grad(nd, 2, nt) with the right-hand side
 * fastest, dipvec(2, ns) shared.  Each right-hand side runs the FMM passes on
 * the plan's tree, so a solve equals the single call to rounding. */
typedef struct zfmm_plan2d_s *zfmm_plan2d;
int zfmm_plan2d_create(double eps, int ns, const double *zsrc, int nt, const double *ztarg,
                       int isep, zfmm_plan2d *plan);
int zfmm_plan2d_create_dev(double eps, int ns, const double *zsrc, int nt, const double *ztarg,
                           int isep, void *stream, zfmm_plan2d *plan);
int zfmm_plan2d_destroy(zfmm_plan2d plan);
int zfmm_plan2d_info(zfmm_plan2d plan, int *nboxes, int *nlevels, int *ns, int *nt);
int zfmm_zlfmm2d_plan(zfmm_plan2d plan, int nd, int ifcharge, const double *charge,
                      int ifdipole, const double *dipstr, const double *dipvec, int ifpgh,
                      double *pot, double *grad);
int zfmm_zlfmm2d_plan_dev(zfmm_plan2d plan, int nd, int ifcharge, const double *charge,
                          int ifdipole, const double *dipstr, const double *dipvec, int ifpgh,
                          double *pot, double *grad, void *stream);
int zfmm_zhfmm2d_plan(zfmm_plan2d plan, const double *zk, int nd, int ifcharge,
                      const double *charge, int ifdipole, const double *dipstr,
                      const double *dipvec, int ifpgh, double *pot, double *grad);
int zfmm_zhfmm2d_plan_dev(zfmm_plan2d plan, const double *zk, int nd, int ifcharge,
                          const double *charge, int ifdipole, const double *dipstr,
                          const double *dipvec, int ifpgh, double *pot, double *grad,
                          void *stream);

/* Plan files (no counterpart in the reference): the geometry of a plan
 * (tree, point order and ranges, sorted points, complex centres, lists)
 * written once and read back by a later process, which then solves without
 * rebuilding the tree.  load creates the plan on the current device; a file
 * of the other dimension, another format version, or a truncated file is
 * refused with status 1. */
int zfmm_plan2d_save(zfmm_plan2d plan, const char *path);
int zfmm_plan2d_load(const char *path, zfmm_plan2d *plan);
int zfmm_plan3d_save(zfmm_plan3d plan, const char *path);
int zfmm_plan3d_load(const char *path, zfmm_plan3d *plan);

/* Many independent 3D FMMs in one call (no counterpart in the reference,
 * where each instance is a separate zlfmm3d / zhfmm3d call): instance i has
 * ns[i] sources zsrc[i](3, ns[i]), strengths charge[i], dipstr[i],
 * dipvec[i](3, ns[i]), nt[i] targets ztarg[i](3, nt[i]) and outputs pot[i],
 * grad[i](3, nt[i]), each exactly as the single call with the shared eps, zk,
 * flags and isep.  Instances are taken largest first from a shared queue by
 * `nstreams` host workers, each driving its own CUDA stream, so that small
 * instances overlap on the GPU.  done_ms (optional, ninst entries) receives
 * each instance's completion time in ms after the call started (its latency
 * when all are submitted together).  Host arrays, or device pointers for
 * _dev (the pointer arrays themselves are host memory). */
int zfmm_zlfmm3d_many(int ninst, double eps, const int *ns, const double *const *zsrc,
                      int ifcharge, const double *const *charge, int ifdipole,
                      const double *const *dipstr, const double *const *dipvec, const int *nt,
                      const double *const *ztarg, int ifpgh, int isep, double *const *pot,
                      double *const *grad, int nstreams, double *done_ms);
int zfmm_zhfmm3d_many(int ninst, double eps, const double *zk, const int *ns,
                      const double *const *zsrc, int ifcharge, const double *const *charge,
                      int ifdipole, const double *const *dipstr, const double *const *dipvec,
                      const int *nt, const double *const *ztarg, int ifpgh, int isep,
                      double *const *pot, double *const *grad, int nstreams, double *done_ms);
int zfmm_zlfmm3d_many_dev(int ninst, double eps, const int *ns, const double *const *zsrc,
                          int ifcharge, const double *const *charge, int ifdipole,
                          const double *const *dipstr, const double *const *dipvec,
                          const int *nt, const double *const *ztarg, int ifpgh, int isep,
                          double *const *pot, double *const *grad, int nstreams,
                          double *done_ms);
int zfmm_zhfmm3d_many_dev(int ninst, double eps, const double *zk, const int *ns,
                          const double *const *zsrc, int ifcharge, const double *const *charge,
                          int ifdipole, const double *const *dipstr,
                          const double *const *dipvec, const int *nt,
                          const double *const *ztarg, int ifpgh, int isep, double *const *pot,
                          double *const *grad, int nstreams, double *done_ms);

/* Allocation-free form of zfmm_zl2devaldirect_dev; it has no counterpart in
 * the reference.  For callers that cannot allocate device memory during a
 * solve: code whose device memory is owned by another allocator (a
 * framework's caching pool that has reserved the GPU), or that runs under a
 * fixed memory budget.  Inputs and outputs are the caller's device arrays, as
 * in zfmm_zl2devaldirect_dev; the partial sums of the source-split kernel use
 * a fixed 8 MiB device array inside the library (kept by every GPU that loads
 * the library until the process exits).  No cudaMalloc/cudaFree and no
 * allocating library routine is called.  Problems whose scratch would exceed
 * the array are rejected with status 1 and a message; the capacity in bytes is
 * returned by zfmm_zl2devaldirect_noalloc_capacity().  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress), so make
 * that first call before any stream capture.  All calls share the array:
 * calls that overlap on the GPU (different streams or host threads) race. */
int zfmm_zl2devaldirect_dev_noalloc(int nt, const double *ztarg, int ns, const double *zsrc,
                                    const double *charge, const double *dipstr,
                                    const double *dipvec, int ifcharge, double *pot, double *grad,
                                    int ifdipole, int ifpgh, void *stream);
long zfmm_zl2devaldirect_noalloc_capacity(void);

/* Self-test of the tensor-core building block of the batched translations
 * (no reference counterpart): D = A B^T for A (128 x K), B (N x K), D (128 x N),
 * row-major FP32 device arrays on `stream`, through tcgen05 TF32 MMAs with the
 * three-term split (hi/lo parts, FP32 accumulation in tensor memory).
 * 16 <= N <= 256, N % 16 == 0, 8 <= K <= 128, K % 8 == 0.  Status 4 if the
 * tensor-core completion wait timed out. */
int zfmm_tc_selftest(int N, int K, const float *A, const float *B, float *D, void *stream);

/* Launch-shape autotuner (no reference counterpart).  Off by default (the
 * fixed launch shapes); zfmm_set_autotune(1) or ZFMM_AUTOTUNE=1 in the
 * environment turns it on: the first call of a tunable kernel (2D Helmholtz
 * table, column, evaluation and P2P kernels) for a work-size bucket (log2 of
 * its item count) on a device times each candidate block size and keeps the
 * fastest for later calls.  Results do not change, only timings.  The table
 * can be saved to and loaded from a text file ("<kernel> <bucket> <device>
 * <block>" per line; load refuses a file with a malformed line, status 1). */
void zfmm_set_autotune(int on);
int zfmm_autotune_entries(void);
int zfmm_autotune_save(const char *path);
int zfmm_autotune_load(const char *path);

/* Per-step device times (ms) of the last FMM call on this host thread:
 * [set-up, P2M, M2M, M2L+P2L, L2L, P2P+M2T+L2T, unsort], plus nboxes, nlevels
 * and the expansion order.  Recording adds CUDA events; enable with
 * zfmm_set_step_timing(1); level 2 also counts the interactions (one more
 * kernel and a stream synchronisation after the solve). */
void zfmm_set_step_timing(int on);
int zfmm_last_step_times(double *ms7, int *nboxes, int *nlevels, int *nterms);
/* Interaction counts of the last FMM call made at timing level 2: [P2P pairs,
 * M2T (target, box), L2T targets, M2L box pairs, P2L (box, source), M2M pairs,
 * L2L pairs, P2M sources], then the same interactions weighted by the
 * expansion lengths P = 2p+1 of their levels (M2L by P^2, M2M and L2L by
 * P_parent P_child), and the number of kernels the call launched. */
int zfmm_last_counts(long long *counts16, long *launches);
/* Expansion order of the 2D Helmholtz FMM for boxes of size bsize (host
 * computation, no GPU needed); replaces h2dterms
 * (zfmm2d/src/helmholtz/h2dterms.f:35-97).  zk points to (re, im). */
int zfmm_h2dterms(double bsize, const double *zk, double eps, int isep);
/* 3D FMMs with step timing level 2: the eight interaction counts of
 * zfmm_last_counts per tree level, counts8x64[k*64 + level] (target level for
 * P2P/M2T/L2T/M2L/P2L, parent level for M2M, child level for L2L), and the
 * expansion order of each level, orders64[level]. */
int zfmm_last_level_counts(long long *counts8x64, int *orders64, int *nlevels);
/* Kernels launched by this library so far, by all host threads of the
 * process (the many-instance entry points launch from worker threads). */
long zfmm_launch_count(void);
/* Device scratch comes from a library-owned memory pool per device that keeps
 * freed memory mapped between calls; this returns the cached memory of the
 * current device's pool to the driver (no reference counterpart). */
int zfmm_trim_pool(void);

/* Tree inspection (tests and tools): builds the device tree for real parts of
 * zsrc/ztarg (host arrays, dimension D = 2 or 3) exactly as the D-dimensional
 * driver does for leaf size `ndiv`, and copies it back.  Box numbers are
 * 0-based, -1 = none.  Call once with box_cap = 0 to learn nboxes/nlevels.
 * Arrays: laddr[2*(nlevels+1)], ilevel/iparent/nchild[nboxes],
 * ichild[2^D*nboxes], centers[D*nboxes], isrc[ns], isrcse[2*nboxes],
 * itarg[nt], itargse[2*nboxes], nlist[4*nboxes], lists (the lists of every
 * box concatenated, list k = 0..3 outermost), mnlist[4]. */
int zfmm_tree_dump(int D, int ndiv, int isep, int ns, const double *zsrc, int nt,
                   const double *ztarg, int box_cap, int list_cap, int *nboxes, int *nlevels,
                   int *laddr, int *ilevel, int *iparent, int *nchild, int *ichild,
                   double *centers, int *isrc, int *isrcse, int *itarg, int *itargse, int *nlist,
                   int *lists, int *nlists_total, int *mnlist);

/* Measured FP64 FMA throughput of the current device in TFLOP/s (roofline
 * denominator for the FP64-bound kernels); -1 on error. */
double zfmm_probe_fp64_tflops(int iters);
/* Measured FP64 tensor-core (mma.sync m8n8k4 f64) throughput, TFLOP/s; -1 on
 * error. */
double zfmm_probe_dmma_tflops(int iters);

/* Last error message of this host thread ("" when none). */
const char *zfmm_last_error(void);

/* Failure injection for tests (no reference counterpart): after
 * zfmm_fail_alloc_after(n) the library's (n+1)-th following device
 * allocation fails as an out-of-memory would (status 3, ZF_ERR_NOMEM, from
 * the call that made it; the memory it had taken is returned), and the
 * injection ends.  n < 0 switches it off. */
void zfmm_fail_alloc_after(long n);
/* Library version string. */
const char *zfmm_version(void);

#ifdef __cplusplus
}
#endif
#endif
