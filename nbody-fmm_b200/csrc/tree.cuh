// Device workspace and tree state shared by the FMM passes.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "common.cuh"

#define CUDA_TRY(x)                                  \
  do {                                               \
    cudaError_t e__ = (x);                           \
    if (e__ != cudaSuccess) {                        \
      fmm::set_cuda_error(e__, #x, __FILE__, __LINE__); \
      return e__ == cudaErrorMemoryAllocation ? FMM_ERR_OUT_OF_MEMORY : FMM_ERR_CUDA; \
    }                                                \
  } while (0)

namespace fmm {

void set_cuda_error(cudaError_t e, const char *what, const char *file, int line);
const char *last_cuda_error_text();

// Grow-only device buffer.
template <class T>
struct DevBuf {
  T *ptr = nullptr;
  size_t cap = 0;
  bool reserve(size_t n) {
    if (n <= cap) return true;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    size_t want = n + n / 8 + 64;
    if (cudaMalloc((void **)&ptr, want * sizeof(T)) != cudaSuccess) {
      ptr = nullptr;
      return false;
    }
    cap = want;
    return true;
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
  }
};

struct Workspace {
  // per particle
  DevBuf<uint64_t> bkeyA, bkeyB, bkeyC;
  DevBuf<uint32_t> bvalA, bvalB, bvalC, bu32A, bu32B, bu32C;
  DevBuf<int> bleaf_of;
  DevBuf<float4> bpart;      // leaf-relative FP32 offset (hi part) + mass, leaf order
  DevBuf<float4> bpart_lo;   // low part of the offset
  DevBuf<float4> bfar;       // far-field gradient (xyz) and potential (w), leaf order
  // per cell
  DevBuf<uint64_t> bcell_key;
  DevBuf<int> bcell_pbeg, bcell_pend, bcell_parent, bcell_child, bcell_coll;
  DevBuf<uint8_t> baflag;    // adaptive targets, per cell: bit 0 target, bit 1 adaptive leaf
  DevBuf<int> balist;        // adaptive targets: the adaptive leaves, then their count
  // misc
  DevBuf<uint32_t> bscan, bhist;
  DevBuf<unsigned long long> bbox;
  DevBuf<double> bgeom;
  DevBuf<uint32_t> bscalars;
  DevBuf<unsigned int> berr;
  DevBuf<unsigned long long> bcount;  // [0] M2L pairs, [1] near-field pairs, [2] M2L tiles, [3] direct far-field
                                      // pairs, [4] sum over M2L pairs of the target's particle count

  uint64_t *keyA = nullptr, *keyB = nullptr, *keyC = nullptr;
  uint32_t *valA = nullptr, *valB = nullptr, *valC = nullptr, *u32A = nullptr, *u32B = nullptr, *u32C = nullptr;
  int *leaf_of = nullptr;
  float4 *part = nullptr, *part_lo = nullptr, *far = nullptr;
  uint64_t *cell_key = nullptr;
  int *cell_pbeg = nullptr, *cell_pend = nullptr, *cell_parent = nullptr, *cell_child = nullptr, *cell_coll = nullptr;
  uint8_t *aflag = nullptr;
  int *alist = nullptr;
  unsigned long long *box_u64 = nullptr;
  double *geom = nullptr;
  uint32_t *scalars = nullptr;
  unsigned int *dev_err = nullptr;
  unsigned long long *counters = nullptr;
  int64_t launches = 0;
  bool ok = true;

  bool init_small() {
    ok &= bbox.reserve(8) && bgeom.reserve(8) && bscalars.reserve(8) && berr.reserve(4) && bcount.reserve(8);
    counters = bcount.ptr;
    box_u64 = bbox.ptr;
    geom = bgeom.ptr;
    scalars = bscalars.ptr;
    dev_err = berr.ptr;
    return ok;
  }
  bool reserve_particles(int64_t n) {
    size_t m = (size_t)(n > 0 ? n : 1);
    ok &= bkeyA.reserve(m) && bkeyB.reserve(m) && bkeyC.reserve(m) && bvalA.reserve(m) && bvalB.reserve(m) &&
          bvalC.reserve(m) && bu32A.reserve(m) && bu32B.reserve(m) && bu32C.reserve(m) && bleaf_of.reserve(m) &&
          bpart.reserve(m) && bpart_lo.reserve(m) && bfar.reserve(m);
    keyA = bkeyA.ptr; keyB = bkeyB.ptr; keyC = bkeyC.ptr;
    valA = bvalA.ptr; valB = bvalB.ptr; valC = bvalC.ptr;
    u32A = bu32A.ptr; u32B = bu32B.ptr; u32C = bu32C.ptr;
    leaf_of = bleaf_of.ptr;
    part = bpart.ptr;
    part_lo = bpart_lo.ptr;
    far = bfar.ptr;
    return ok;
  }
  bool reserve_cells(int64_t cap, int nc, int ns) {
    size_t m = (size_t)(cap > 0 ? cap : 1);
    ok &= bcell_key.reserve(m) && bcell_pbeg.reserve(m) && bcell_pend.reserve(m) && bcell_parent.reserve(m) &&
          bcell_child.reserve(m * nc) && bcell_coll.reserve(m * ns);
    cell_key = bcell_key.ptr;
    cell_pbeg = bcell_pbeg.ptr;
    cell_pend = bcell_pend.ptr;
    cell_parent = bcell_parent.ptr;
    cell_child = bcell_child.ptr;
    cell_coll = bcell_coll.ptr;
    return ok;
  }
  bool reserve_adaptive(int64_t ncell) {
    ok &= baflag.reserve((size_t)ncell) && balist.reserve((size_t)ncell + 1);
    aflag = baflag.ptr;
    alist = balist.ptr;
    return ok;
  }
  uint32_t *scan_tmp(int nb) {
    ok &= bscan.reserve((size_t)nb);
    return bscan.ptr;
  }
  uint32_t *radix_hist(int nb) {
    ok &= bhist.reserve((size_t)nb * 256);
    return bhist.ptr;
  }
  void release_all() {
    bkeyA.release(); bkeyB.release(); bkeyC.release();
    bvalA.release(); bvalB.release(); bvalC.release();
    bu32A.release(); bu32B.release(); bu32C.release();
    bleaf_of.release(); bpart.release(); bpart_lo.release(); bfar.release();
    bcell_key.release(); bcell_pbeg.release(); bcell_pend.release(); bcell_parent.release();
    bcell_child.release(); bcell_coll.release(); baflag.release(); balist.release();
    bscan.release(); bhist.release(); bbox.release(); bgeom.release(); bscalars.release(); berr.release(); bcount.release();
  }
};

// Result of a tree build.  Cell indices are absolute into the Workspace cell
// arrays; level d holds cells [level_off[d], level_off[d] + level_count[d]),
// levels are contiguous from the root, and every cell covers the contiguous
// particle range [cell_pbeg, cell_pend) of the leaf order.
struct TreeState {
  int dim = 3;
  int64_t n = 0;
  int depth = 0;
  double lo[6] = {0, 0, 0, 0, 0, 0};  // lo[0..2] box min (lo[3..5] scratch)
  double hi[3] = {0, 0, 0};
  std::vector<int> level_count, level_off;
  int cell0 = 0;      // index of the root
  int n_cells = 0;
  int adaptive_leaf = 0;  // adaptive targets: the threshold ws.aflag / ws.alist were computed for (0: none, and
                          // every cell has its colleague row; else only the target cells have one)
  uint64_t *d_leafkey_sorted = nullptr;
  uint32_t *d_perm = nullptr;  // leaf order -> input index
};

void exclusive_scan(Workspace &ws, const uint32_t *in, uint32_t *out, int64_t n, uint32_t *total_dev,
                    cudaStream_t st);
void radix_sort(Workspace &ws, uint64_t *&keys, uint32_t *&vals, uint64_t *&keys_alt, uint32_t *&vals_alt, int64_t n,
                int bits, cudaStream_t st);
int build_tree(Workspace &ws, TreeState &t, const double *d_pos, const double *d_mass, int64_t n, int dim,
               int threshold, cudaStream_t st, int adaptive_leaf = 0);
// Adaptive-target flags of every cell of a built tree into flag[0 .. n_cells)
// and the adaptive leaves into list[0 .. count), count at list[n_cells].
int launch_adaptive_flags(const Workspace &ws, const TreeState &t, int A, uint8_t *flag, int *list, cudaStream_t st);

}  // namespace fmm
