// Translations (M2L, M2M, L2L) on the 5th-generation tensor cores (tcgen05).
#pragma once
#include "tree.cuh"

namespace fmm {

enum { TC_M2L = 0, TC_M2M = 1, TC_L2L = 2 };

// Largest padded expansion length the tensor-core kernel takes (K <= 176:
// 3D p <= 12, 2D p <= 87).
static constexpr int TC_MAX_P16 = 176;

struct TcArgs {
  int mode;                 // TC_M2L, TC_M2M or TC_L2L
  const int4 *batches;      // {tlist offset, count, level, class}, up to 128 cells each
  const int *tlist;         // class-grouped cells: targets (M2L, L2L) or children (M2M)
  const int *src_tab;       // M2L: [batch][slot][128] source cell per target, -1 if none
  const int *slot_list;     // M2L: [batch][i] present slots
  const int *tslot_list;    // M2L: [batch][i] operator-table slot of each present slot
  const int *nslots;        // M2L: [batch]
  const uint8_t *slot_p16;  // M2L: [batch][i] padded width (16 * ceil(K_i / 16)) of each present slot's
                            // order, null = every slot at full order
  const int *cchild;        // children of each cell (nchild per cell, -1 if absent)
  const int *cparent;       // parent of each cell (M2M destination, L2L source)
  int nchild;               // 8 in 3D, 4 in 2D
  int op_base;              // M2M / L2L: operator-table slot of child class 0
  const float *X;           // source expansions, KS floats per cell
  float *Y;                 // target expansions (accumulated into)
  const uint16_t *bimg;     // BF16 split operator images, 3 * P16^2 per table slot
  int cell0, K, KS, P16;    // P16 = K rounded up to 16
  int img_p16;              // padded width the operator images were built for (0: P16); a narrower
                            // kernel reads the first output tile of wider images (same first-tile width)
  unsigned int *err;
  unsigned long long *tiles;  // M2L: number of (batch, slot) tiles contracted (nullable)
  unsigned long long *widths; // M2L: sum of the tiles' padded widths (nullable)
  int run_slots;            // M2L: slots per work item requested (fmm_config.m2l_run; 0: the launcher's rule)
  int chunk_slots;          // M2L: slots per work item (set by the launcher; a batch of more slots is
                            // split into items whose sums all add into the targets)
};

// Width of the first output tile: one tile up to 128 columns, else two.
__host__ __device__ constexpr int tc_n0(int P16) { return P16 <= 128 ? P16 : ((P16 / 2 + 15) & ~15); }

size_t tc_smem_bytes(int P16);
int tc_build_images(const float *tab, int n_slots, int K, int KP, int P16, uint16_t *img, cudaStream_t st,
                    int64_t &launches);
// Launches one translation pass over nb batches; `work` is a zeroed device
// counter the persistent CTAs take batches from.
int tc_launch(const TcArgs &a, int nb, unsigned int *work, cudaStream_t st, int64_t &launches);

// Splits the present slots of every M2L batch by padded width: slots with
// w <= wsplit into (lo_*), the others into (hi_*), each [batch][189] with counts.
int tc_split_slots(const int *slot_list, const int *tslot_list, const uint8_t *slot_p16, const int *nslots, int nbm,
                   int wsplit, int *lo_slot, int *lo_tslot, uint8_t *lo_w, int *lo_n, int *hi_slot, int *hi_tslot,
                   uint8_t *hi_w, int *hi_n, cudaStream_t st, int64_t &launches);

// Work counters per pass (one per launch).
static constexpr int TC_MAX_LAUNCHES = 80;

}  // namespace fmm
