// Tensor-core (tcgen05) M2L contraction.
#pragma once
#include "tree.cuh"

namespace fmm {

struct TcArgs {
  const int4 *batches;      // {tlist offset, count, level, class}, 128 targets each
  const int *tlist;         // class-grouped M2L target cells
  const int *src_tab;       // [batch][slot][128] source cell per target, -1 if none
  const int *slot_list;     // [batch][i] present slots
  const int *tslot_list;    // [batch][i] operator-table slot of each present slot
  const int *nslots;        // [batch]
  const float *X;           // multipoles, KS floats per cell
  float *Y;                 // local expansions (accumulated into)
  const uint16_t *bimg;     // BF16 operator images, 3 splits per table slot
  int cell0, K, KS, P16;    // P16 = K rounded up to 16
  unsigned int *err;
};

size_t tc_smem_bytes(int P16);
int tc_build_images(const float *tab, int n_m2l, int K, int KP, int P16, uint16_t *img, cudaStream_t st,
                    int64_t &launches);
int tc_launch_m2l(const TcArgs &a, int nb, cudaStream_t st, int64_t &launches);

}  // namespace fmm
