// Expansion passes (P2M, M2M, M2L, L2L, L2P) and the near field.
#pragma once
#include <algorithm>
#include "order.cuh"
#include "tree.cuh"

namespace fmm {

// Operator tables in the layout the contraction kernels read: for each slot a
// K x KP matrix stored input-major (entry [in][out]); KP = 32 * ceil(K/32),
// padded with zeros.  Slots: M2L 343 relative offsets (7^3, index
// (dx+3) + 7(dy+3) + 49(dz+3); |d| <= 1 rows are zero), then 8 M2M and 8 L2L
// child slots.  2D: 49 offsets, 4 + 4 child slots.
struct OpTables {
  int dim = 3, p = 0, K = 0, KP = 0, KS = 0;
  int n_m2l = 0, off_m2m = 0, off_l2l = 0, n_slots = 0;
  DevBuf<float> tab;        // n_slots * K * KP
  DevBuf<double> scratch;   // FP64 staging
  DevBuf<double> tab64;     // FP64 copy of the 3D M2L operators (training-pair probe only)
};

// Page-locked host staging (batch tables uploaded every pass): the copies
// from it are asynchronous, so the buffer is rewritten only after a stream
// synchronisation, which every pass makes before building its tables.
template <class T>
struct HostPinned {
  T *ptr = nullptr;
  size_t cap = 0;
  bool reserve(size_t n, cudaStream_t st) {
    if (n <= cap) return true;
    if (ptr) {
      cudaStreamSynchronize(st);
      cudaFreeHost(ptr);
    }
    ptr = nullptr;
    cap = 0;
    size_t want = std::max(n, (size_t)4096);
    if (cudaHostAlloc((void **)&ptr, want * sizeof(T), cudaHostAllocDefault) != cudaSuccess) {
      ptr = nullptr;
      return false;
    }
    cap = want;
    return true;
  }
  void release() {
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    cap = 0;
  }
};

struct ExpBuffers {
  DevBuf<float> M, L;  // n_cells * KS each (indexed by absolute cell - cell0)
  DevBuf<int> tlist;      // class-grouped cells of levels >= 2 (L2L targets)
  DevBuf<int> tlist_m2l;  // the same restricted to cells with possible M2L pairs
  DevBuf<uint64_t> ckey, ckey_alt, ckey_m2l;  // (level, class) sort keys of those cells
  DevBuf<uint32_t> cval, cval2;
  DevBuf<int4> batches;
  DevBuf<uint32_t> cls_count;
  DevBuf<float4> lvl_off;  // particle offsets from their level-d ancestor's centre, levels 2..D-1
  DevBuf<uint8_t> lact;    // shortcuts, per cell: [0, ncell) M2L contributions, [ncell, 2 ncell) needs L,
                           // [2 ncell, 3 ncell) M2L source, [3 ncell, 4 ncell) how M is formed
  DevBuf<uint64_t> ukey;   // shortcuts: sort keys (two sorts, key and alternate each)
  DevBuf<uint32_t> uval;
  DevBuf<int> p2m_list;    // shortcuts: the cells whose multipole comes straight from their particles, then their count
  DevBuf<int4> batches2;   // shortcuts: batches of the cells that need L2L, then of the M2M rows
  HostPinned<int4> hbatches, hbatches2;  // their host staging
  DevBuf<int> esrc;        // L2L shortcut: per leaf, the cell whose local expansion its particles evaluate
  DevBuf<uint8_t> elev;    //   and that cell's level
  DevBuf<int> m2l_src, m2l_list, m2l_nslots, m2l_tslot;  // per M2L batch: resolved sources and present slots
  DevBuf<uint16_t> tc_img;       // BF16 split operator images for the tensor-core translations
  DevBuf<unsigned int> tc_work;  // zeroed work counters of the tensor-core launches
  DevBuf<uint8_t> order_p16;     // per M2L operator slot: padded width of its pair order
  DevBuf<uint8_t> fdirect;       // per offset (dx+3) + 7(dy+3) + 49(dz+3): not well separated (direct)
  DevBuf<uint8_t> m2l_w;         // per M2L batch and present slot: padded width of its order
  DevBuf<int> m2l_split;         // variable orders: [4][batch][189] (lo slot, lo op, hi slot, hi op) + counts
  DevBuf<uint8_t> m2l_split_w;   // [2][batch][189] widths of the lo / hi lists
  DevBuf<uint16_t> cf;           // learned orders: per-cell features (ORD_CF BF16 values per cell)
  DevBuf<double> frms;           // learned orders: [0] F_rms of the previous pass (G = 1), [1] scratch,
                                 // [2] total mass
  DevBuf<int> ftl;               // adaptive targets: the direct far field's targets per level, then counts
  DevBuf<double> xs;             // adaptive targets: FP64 positions in leaf order (dim per particle)
  DevBuf<uint32_t> ccnt;         // adaptive targets: colleague-sum items per adaptive leaf, then their offsets
  DevBuf<int2> citems;           // adaptive targets: colleague-sum items (adaptive leaf index, source chunk)
};

// Per-pass parameters.
struct PassGeom {
  double lo[3], ext[3], emax;
};

int build_op_tables(OpTables &ops, int dim, int p, int depth, const PassGeom &g, cudaStream_t st, int64_t &launches,
                    bool want64 = false);

// Learned-order settings of a pass, and the training-pair collection hook.
struct OrderOpts {
  int mode = 0;            // FMM_ORDER_*
  int margin = 1;          // FMM_ORDER_GEOMETRIC
  float tol = 2e-6f;       // FMM_ORDER_LEARNED: relative error budget of the truncation
  const float *params = nullptr;  // FMM_ORDER_LEARNED: MLP parameters
  // collection (ntiles = 0: none): sample `ntiles` M2L tiles, write their
  // features and FP64 error labels
  int ntiles = 0;
  unsigned long long seed = 0;
  int *tiles = nullptr;          // [ntiles][2]
  int *pairs = nullptr;          // [ntiles][128][4]
  float *pair_labels = nullptr;  // [ntiles][128][ORD_NQ]
  float *feat = nullptr, *labels = nullptr;
};
void upload_class_tables();

int run_fmm_passes(Workspace &ws, TreeState &t, OpTables &ops, ExpBuffers &eb, const double *d_pos,
                   const double *d_mass, int p, double eps2, double G,
                   const PassGeom &g, double *d_acc, double *d_pot, int m2l_mode, int64_t direct_max,
                   const OrderOpts &order, cudaStream_t st, fmm_stats &stats, cudaEvent_t *ev,
                   int adaptive_leaf = 0, int p2p_chunk = 0, int m2l_run = 0);

}  // namespace fmm
