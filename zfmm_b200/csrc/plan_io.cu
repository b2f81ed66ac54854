// Plan files: the geometry of a 2D or 3D plan (tree, point permutation and
// ranges, sorted points, complex box centres, interaction lists) written to
// disk once and read back by any later process, so that repeated solves on
// one geometry (GMRES matvecs, adjoint passes, many right-hand sides over
// several runs) skip the integer set-up.  No counterpart in the reference,
// whose drivers rebuild the tree in every call.
//
// Format (little-endian, native sizes): magic "ZFMMPLAN", u32 version, u32 D,
// then the plan scalars, the tree scalars and host vectors, and every device
// array as (u64 element count, u32 element size, raw bytes).  A file of
// another version or dimension, or one that ends early, is refused.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "../../include/zfmm.h"
#include "plan2d.cuh"
#include "plan3d.cuh"

namespace zf {
namespace {

constexpr char kMagic[8] = {'Z', 'F', 'M', 'M', 'P', 'L', 'A', 'N'};
constexpr uint32_t kVersion = 1;

struct File {
  FILE* f = nullptr;
  File(const char* path, const char* mode) : f(fopen(path, mode)) {
    if (!f) throw zf_error(ZF_ERR_ARG, std::string("cannot open plan file ") + path);
  }
  ~File() {
    if (f) fclose(f);
  }
  void put(const void* p, size_t n) {
    if (n && fwrite(p, 1, n, f) != n) throw zf_error(ZF_ERR_INTERNAL, "plan file write failed");
  }
  void get(void* p, size_t n) {
    if (n && fread(p, 1, n, f) != n) throw zf_error(ZF_ERR_ARG, "plan file is truncated");
  }
  template <class T>
  void put_v(const T& v) { put(&v, sizeof v); }
  template <class T>
  T get_v() {
    T v;
    get(&v, sizeof v);
    return v;
  }
  template <class T>
  void put_vec(const std::vector<T>& v) {
    put_v<uint64_t>(v.size());
    put(v.data(), v.size() * sizeof(T));
  }
  template <class T>
  void get_vec(std::vector<T>& v) {
    uint64_t n = get_v<uint64_t>();
    if (n > (1ull << 34)) throw zf_error(ZF_ERR_ARG, "plan file is corrupt");
    v.resize(n);
    get(v.data(), n * sizeof(T));
  }
  template <class T>
  void put_dev(const DevBuf<T>& b, cudaStream_t s) {
    std::vector<T> h(b.size());
    if (!h.empty())
      ZF_CUDA(cudaMemcpyAsync(h.data(), b.get(), h.size() * sizeof(T), cudaMemcpyDeviceToHost, s));
    ZF_CUDA(cudaStreamSynchronize(s));
    put_v<uint64_t>(h.size());
    put_v<uint32_t>(sizeof(T));
    put(h.data(), h.size() * sizeof(T));
  }
  template <class T>
  void get_dev(DevBuf<T>& b, cudaStream_t s) {
    uint64_t n = get_v<uint64_t>();
    uint32_t es = get_v<uint32_t>();
    if (es != sizeof(T) || n > (1ull << 34)) throw zf_error(ZF_ERR_ARG, "plan file is corrupt");
    std::vector<T> h(n);
    get(h.data(), n * sizeof(T));
    b.alloc(n, s);
    if (n) ZF_CUDA(cudaMemcpyAsync(b.get(), h.data(), n * sizeof(T), cudaMemcpyHostToDevice, s));
    ZF_CUDA(cudaStreamSynchronize(s));  // h is freed on return
  }
};

void put_tree(File& F, const DevTree& t, const DevLists& L, cudaStream_t s) {
  for (int v : {t.D, t.NC, t.isep, t.mnbors, t.nlevels, t.nboxes}) F.put_v<int32_t>(v);
  F.put_vec(t.laddr);
  F.put_vec(t.boxsize);
  F.put_dev(t.ilevel, s); F.put_dev(t.iparent, s); F.put_dev(t.nchild, s);
  F.put_dev(t.ichild, s); F.put_dev(t.ncoll, s); F.put_dev(t.coll, s);
  F.put_dev(t.centers, s); F.put_dev(t.bsz, s);
  for (int k = 0; k < 4; k++) F.put_v<int32_t>(L.mn[k]);
  for (int k = 0; k < 4; k++) {
    F.put_dev(L.n[k], s);
    F.put_dev(L.list[k], s);
  }
}

void get_tree(File& F, DevTree& t, DevLists& L, cudaStream_t s) {
  t.D = F.get_v<int32_t>(); t.NC = F.get_v<int32_t>(); t.isep = F.get_v<int32_t>();
  t.mnbors = F.get_v<int32_t>(); t.nlevels = F.get_v<int32_t>(); t.nboxes = F.get_v<int32_t>();
  F.get_vec(t.laddr);
  F.get_vec(t.boxsize);
  // the tree's arrays may be longer than nboxes / nlevels (capacity of the
  // level-by-level build); they are stored and restored as they are
  if (t.nboxes < 1 || t.nlevels < 0 || t.laddr.size() < 2 * (size_t)(t.nlevels + 1))
    throw zf_error(ZF_ERR_ARG, "plan file is corrupt");
  F.get_dev(t.ilevel, s); F.get_dev(t.iparent, s); F.get_dev(t.nchild, s);
  F.get_dev(t.ichild, s); F.get_dev(t.ncoll, s); F.get_dev(t.coll, s);
  F.get_dev(t.centers, s); F.get_dev(t.bsz, s);
  for (int k = 0; k < 4; k++) L.mn[k] = F.get_v<int32_t>();
  for (int k = 0; k < 4; k++) {
    F.get_dev(L.n[k], s);
    F.get_dev(L.list[k], s);
  }
  if (t.ilevel.size() < (size_t)t.nboxes || t.iparent.size() < (size_t)t.nboxes)
    throw zf_error(ZF_ERR_ARG, "plan file is corrupt");
}

void header(File& F, uint32_t D) {
  F.put(kMagic, 8);
  F.put_v<uint32_t>(kVersion);
  F.put_v<uint32_t>(D);
}

void check_header(File& F, uint32_t D) {
  char m[8];
  F.get(m, 8);
  if (memcmp(m, kMagic, 8) != 0) throw zf_error(ZF_ERR_ARG, "not a zfmm_b200 plan file");
  if (F.get_v<uint32_t>() != kVersion) throw zf_error(ZF_ERR_ARG, "plan file version mismatch");
  if (F.get_v<uint32_t>() != D)
    throw zf_error(ZF_ERR_ARG, D == 2 ? "plan file holds a 3D plan" : "plan file holds a 2D plan");
}

}  // namespace

void plan2d_save(const Plan2D& P, const char* path, cudaStream_t s) {
  File F(path, "wb");
  header(F, 2);
  F.put_v<double>(P.eps);
  for (int v : {P.isep, P.ns, P.nt}) F.put_v<int32_t>(v);
  const Setup2D& S = P.S;
  put_tree(F, S.tree, S.lists, s);
  F.put_dev(S.isrc, s); F.put_dev(S.isrcse, s); F.put_dev(S.itarg, s); F.put_dev(S.itargse, s);
  F.put_dev(S.zsrcsort, s); F.put_dev(S.ztargsort, s);
  F.put_dev(S.zcsrc, s); F.put_dev(S.zctarg, s);
}

void plan2d_load(Plan2D& P, const char* path, cudaStream_t s) {
  File F(path, "rb");
  check_header(F, 2);
  P.eps = F.get_v<double>();
  P.isep = F.get_v<int32_t>(); P.ns = F.get_v<int32_t>(); P.nt = F.get_v<int32_t>();
  ZF_CUDA(cudaGetDevice(&P.device));
  Setup2D& S = P.S;
  get_tree(F, S.tree, S.lists, s);
  F.get_dev(S.isrc, s); F.get_dev(S.isrcse, s); F.get_dev(S.itarg, s); F.get_dev(S.itargse, s);
  F.get_dev(S.zsrcsort, s); F.get_dev(S.ztargsort, s);
  F.get_dev(S.zcsrc, s); F.get_dev(S.zctarg, s);
  if (S.isrc.size() < (size_t)P.ns || S.itarg.size() < (size_t)P.nt)
    throw zf_error(ZF_ERR_ARG, "plan file is corrupt");
}

void plan3d_save(const Plan3D& P, const char* path, cudaStream_t s) {
  File F(path, "wb");
  header(F, 3);
  F.put_v<double>(P.eps);
  for (int v : {P.isep, P.ns, P.nt}) F.put_v<int32_t>(v);
  const Setup3D& S = P.S;
  put_tree(F, S.tree, S.lists, s);
  F.put_dev(S.isrc, s); F.put_dev(S.isrcse, s); F.put_dev(S.itarg, s); F.put_dev(S.itargse, s);
  F.put_dev(S.zsrcsort, s); F.put_dev(S.ztargsort, s);
  F.put_dev(S.zcsrc, s); F.put_dev(S.zctarg, s);
  F.put_v<double>(S.b0);
  F.put_vec(S.bsz);
}

void plan3d_load(Plan3D& P, const char* path, cudaStream_t s) {
  File F(path, "rb");
  check_header(F, 3);
  P.eps = F.get_v<double>();
  P.isep = F.get_v<int32_t>(); P.ns = F.get_v<int32_t>(); P.nt = F.get_v<int32_t>();
  ZF_CUDA(cudaGetDevice(&P.device));
  Setup3D& S = P.S;
  get_tree(F, S.tree, S.lists, s);
  F.get_dev(S.isrc, s); F.get_dev(S.isrcse, s); F.get_dev(S.itarg, s); F.get_dev(S.itargse, s);
  F.get_dev(S.zsrcsort, s); F.get_dev(S.ztargsort, s);
  F.get_dev(S.zcsrc, s); F.get_dev(S.zctarg, s);
  S.b0 = F.get_v<double>();
  F.get_vec(S.bsz);
  if (S.isrc.size() < (size_t)P.ns || S.itarg.size() < (size_t)P.nt)
    throw zf_error(ZF_ERR_ARG, "plan file is corrupt");
}

}  // namespace zf
