// 2D plans (see plan2d.cuh): the set-up of zlfmm2d.f:70-200 / zhfmm2d.f:73-195
// once, then the FMM passes per right-hand side on the stored geometry.
#include <cmath>
#include <vector>
#include "hfmm2d.cuh"
#include "lfmm2d.cuh"
#include "plan2d.cuh"

namespace zf {

void plan2d_build(Plan2D& P, double eps, int ns, const zdc* zsrc, int nt, const zdc* ztarg,
                  int isep, cudaStream_t s) {
  if (isep < 1) throw zf_error(ZF_ERR_ARG, "isep must be >= 1");
  P.eps = eps;
  P.isep = isep;
  P.ns = ns;
  P.nt = nt;
  ZF_CUDA(cudaGetDevice(&P.device));
  TreeParams tp;
  tp.D = 2;
  tp.isep = isep;
  lndiv2d(eps, ns, nt, &tp.ndiv, &tp.idivflag);
  setup2d_geom(ns, zsrc, nt, ztarg, tp, P.S, s);
  ZF_CUDA(cudaStreamSynchronize(s));
}

void fmm2d_plan_execute(const Plan2D& P, const zdc* zk, int nd, int ifcharge, const zdc* charge,
                        int ifdipole, const zdc* dipstr, const zdc* dipvec, int ifpgh,
                        zdc* pot, zdc* grad, cudaStream_t s, StepTimes* times) {
  const Setup2D& S = P.S;
  const int ns = P.ns, nt = P.nt;
  long launches0 = launch_counter();
  const bool timing = times != nullptr;
  cudaEvent_t ev[8];
  if (timing)
    for (auto& e : ev) ZF_CUDA(cudaEventCreate(&e));
  float acc[8] = {0};
  auto mark = [&](int i) {
    if (timing) ZF_CUDA(cudaEventRecord(ev[i], s));
  };
  DevBuf<zdc> q(ns, s), ds(ns, s), dv(2 * (size_t)ns, s), potsort(nt, s),
      gradsort(ifpgh > 1 ? 2 * (size_t)nt : 1, s);
  const zdc scale = zk ? mkz(0.0, 0.25) : mkz(1.0 / (2.0 * M_PI));
  std::vector<int> pl;
  int pord = 0;
  // the Helmholtz orders and translation tables depend on the tree and zk
  // only: built once for all right-hand sides
  Helm2DPrepPtr H;
  if (zk) H = helm2d_prepare(S, P.eps, *zk, P.isep, s);
  if (zk && nd >= 2) {
    // several right-hand sides: M2L of groups of right-hand sides at once, on
    // the tensor cores when eps >= 1e-7 (TF32 three-term split, accurate to
    // about 1e-7 relative), in FP64 otherwise
    mark(0);
    float ms3[3] = {0, 0, 0};
    helm2d_passes_nd(S, *H, nd, ifcharge, charge, ifdipole, dipstr, dipvec, ifpgh,
                     P.eps >= 1e-7, pot, grad, s, timing ? ms3 : nullptr);
    if (timing) {
      for (int k = 0; k < 7; k++) times->ms[k] = 0;
      times->ms[1] = ms3[0];
      times->ms[3] = ms3[1];
      times->ms[5] = ms3[2];
      times->nboxes = S.tree.nboxes;
      times->nlevels = S.tree.nlevels;
      times->nterms = 0;
      for (auto& e : ev) cudaEventDestroy(e);
      times->launches = launch_counter() - launches0;
    }
    return;
  }
  for (int r = 0; r < nd; r++) {
    mark(0);
    gather2d_col(S, ns, nd, r, ifcharge ? charge : nullptr, ifdipole ? dipstr : nullptr,
                 ifdipole ? dipvec : nullptr, q.get(), ds.get(), dv.get(), s);
    potsort.zero();
    gradsort.zero();
    mark(1);
    if (zk)
      pord = helm2d_passes(S, *H, q.get(), ds.get(), dv.get(), ifcharge, ifdipole, ifpgh,
                           potsort.get(), gradsort.get(), s, timing ? ev : nullptr, &pl);
    else
      pord = lap2d_core(S, P.eps, q.get(), ds.get(), dv.get(), ifcharge, ifdipole, ifpgh,
                        potsort.get(), gradsort.get(), s, timing ? ev : nullptr, &pl);
    mark(6);
    unsort2d_col(nt, nd, r, S.itarg.get(), potsort.get(), gradsort.get(), scale, ifpgh, pot, grad,
                 s);
    mark(7);
    if (timing) {
      ZF_CUDA(cudaEventSynchronize(ev[7]));
      for (int k = 0; k < 7; k++) {
        float ms;
        ZF_CUDA(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
        acc[k] += ms;
      }
    }
  }
  if (timing) {
    for (int k = 0; k < 7; k++) times->ms[k] = acc[k];
    times->nboxes = S.tree.nboxes;
    times->nlevels = S.tree.nlevels;
    times->nterms = pord;
    for (auto& e : ev) cudaEventDestroy(e);
    times->launches = launch_counter() - launches0;
    if (times->want_counts && !pl.empty()) count_interactions2d(S, pl.data(), times->counts, s);
  }
}

}  // namespace zf
