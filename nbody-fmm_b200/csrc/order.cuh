// Learned expansion order of the M2L tiles (FMM_ORDER_LEARNED).
//
// An M2L tile is the unit of tensor-core work: up to 128 target cells of one
// level and child class against their sources at one interaction offset, all
// evaluated at one order.  A small MLP reads the tile's features (level,
// offset geometry, the largest particle counts, the largest source multipole
// norm of every degree relative to the total mass, the target cells' spread)
// and predicts, for every order q in 4..12, the base-10 logarithm of
//   z(q) = max over the tile's pairs of  e(q) / sqrt(n_T) * R^2 / M_tot,
// e(q) the pair's truncation error on its target particles (L2 over them,
// G = 1), R the distance of the cell centres and M_tot the total mass.  The
// tile takes the lowest order with z(q) <= tol F_rms R^2 / (M_tot sqrt(P)),
// which gives every pair the same share of the squared error budget
// tol^2 F_rms^2 n (F_rms the RMS force of the previous pass, P the M2L pairs
// per particle).  Training tiles come from the FMM itself: every pair of a
// sampled tile has its truncation error at every order measured in FP64
// against its direct sum.
#pragma once
#include "tree.cuh"

namespace fmm {

static constexpr int ORD_NF = 32;    // features per pair
static constexpr int ORD_NH = 64;    // hidden width (two hidden layers)
static constexpr int ORD_NQ = 9;     // outputs: orders 4..12
static constexpr int ORD_QMIN = 4;
static constexpr int ORD_QMAX = ORD_QMIN + ORD_NQ - 1;
static constexpr int ORD_CF = 16;    // floats per cell-feature row
// flat FP32 parameter layout: W1 [64][32], b1 [64], W2 [64][64], b2 [64], W3 [16][64] (rows 9..15 zero), b3 [16]
static constexpr int ORD_W1 = 0;
static constexpr int ORD_B1 = ORD_W1 + ORD_NH * ORD_NF;
static constexpr int ORD_W2 = ORD_B1 + ORD_NH;
static constexpr int ORD_B2 = ORD_W2 + ORD_NH * ORD_NH;
static constexpr int ORD_W3 = ORD_B2 + ORD_NH;
static constexpr int ORD_B3 = ORD_W3 + 16 * ORD_NH;
static constexpr int ORD_NPARAM = ORD_B3 + 16;

struct OrderGeom {
  double lo[3], ext[3], emax;
};

// Per-cell features of cells [first, first + count): log2(1 + n),
// log10(|M~_n| / |M~_0|) for n = 1..12 (|M~_n|^2 = sum over m of |M~_n^m|^2)
// and log10 M~_0; with `mode` set only for the cells whose multipole was
// formed (mode != 0), the others are left as they are.  Also the total mass
// of the n particles `part` (mass in w) into *mtot.
int order_cell_features(const float *M, const int *pbeg, const int *pend, int first, int count, int cell0, int p,
                        int KS, const uint8_t *mode, uint16_t *cf, const float4 *part, int64_t n, double *mtot,
                        cudaStream_t st, int64_t &launches);

// The resolved M2L tables and what the tile features read.
struct TileArgs {
  const int4 *batches;
  const int *tlist, *src_tab, *slot_list, *tslot_list, *nslots;
  const int *pbeg, *pend;
  const uint16_t *cf;   // cell features (ORD_CF BF16 values per cell)
  const double *mtot;   // device: total mass
  int cell0;
  float ax, ay, az;     // cell aspect (extent / largest extent)
};

// Samples n tiles {batch, present-slot index} (-1 where the drawn batch has
// no slot), their features ([n][ORD_NF]) and their pairs ([n][128] int4
// {T, S, offset slot, level}, -1 rows where the tile has no pair).
int order_sample_tiles(const TileArgs &a, int nbm, int n, unsigned long long seed, int *tiles, float *feat,
                       int *pairs, cudaStream_t st, int64_t &launches);

// FP64 truncation errors of pairs at orders 4..p: log10(e(q) / sqrt(n_T) R^2)
// per pair ([n][ORD_NQ]; -1e30 for rows without a pair; orders above p: 0).
struct ProbeArgs {
  const int *pairs;
  int n;
  const double *pos, *mass;
  const uint32_t *perm;
  const int *pbeg, *pend;
  const uint64_t *ckey;
  const double *tab64;  // FP64 M2L operators [343][K][KP]
  int p, K, KP;
  OrderGeom g;
  float *labels;
};
int order_probe_errors(const ProbeArgs &a, cudaStream_t st, int64_t &launches);

// Tile labels: the largest pair label of each tile minus log10 M_tot
// ([n][ORD_NQ]); tiles without a pair get zero features and labels.
int order_tile_labels(const float *pair_labels, int n, const double *mtot, float *labels, float *feat,
                      cudaStream_t st, int64_t &launches);

// Hot path: the order of every present slot of every M2L batch from the MLP
// (padded width into slot_p16).  F_rms <= 0 (no previous pass): full order.
struct InferArgs {
  TileArgs t;
  const float *params;   // MLP parameters (FP32; weights rounded to BF16 on load)
  const double *frms;    // device: F_rms of the previous pass, G = 1 units
  const unsigned long long *nt_sum;  // device: sum over M2L pairs of n_T
  int64_t n;
  int p;
  float tol;
  double emax;
  uint8_t *slot_p16;
};
int order_infer(const InferArgs &a, int nbm, cudaStream_t st, int64_t &launches);

// Training on the GPU: Adam on the mean squared error of the predicted log
// errors (labels clamped below at -16), minibatches of `batch` rows taken in
// order from the (pre-shuffled) data.  loss_out: mean loss of each epoch.
int order_train(const float *feat, const float *labels, int n, int epochs, int batch, float lr, float *params,
                float *loss_out, cudaStream_t st, int64_t &launches);

// Forward pass and parameter gradient of the MSE loss on n rows (for the
// gradient check against the CPU oracle).
int order_forward_grad(const float *feat, const float *labels, int n, const float *params, float *pred, float *grad,
                       float *loss, cudaStream_t st, int64_t &launches);

// sum over particles of |acc|^2 / G^2, then F_rms = sqrt(sum / n) into *frms.
int order_force_rms(const double *acc, int64_t n, int dim, double G, double *scratch, double *frms, cudaStream_t st,
                    int64_t &launches);

// Judge: sum over the sampled targets of |acc - ref|^2 and |ref|^2 into out[0..1].
int order_judge_compare(const double *acc, const double *ref, const int64_t *targets, int64_t nt, int dim, double *out,
                        cudaStream_t st, int64_t &launches);

}  // namespace fmm
