// Learned expansion order of each M2L pair (FMM_ORDER_LEARNED).
//
// A small MLP reads the features of an interaction-list pair (level, particle
// counts, the source cell's multipole spectrum by degree, the target cell's
// spread, the offset geometry) and predicts, for every order q in 4..12, the
// base-10 logarithm of the pair's truncation error on the target particles
// relative to the pair's monopole scale M_S sqrt(n_T) / R^2.  A pair takes the
// lowest order whose predicted error fits its share of the error budget.
// Training pairs and their errors come from the FMM itself: sampled M2L pairs
// whose truncation error at every order is measured in FP64 against the
// pair's direct sum.
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

// Per-cell features of cells [first, first + count): log2(1 + n) and
// log10(|M~_n| / |M~_0|) for n = 1..12 (|M~_n|^2 = sum over m of |M~_n^m|^2).
int order_cell_features(const float *M, const int *pbeg, const int *pend, int first, int count, int cell0, int p,
                        int KS, float *cf, cudaStream_t st, int64_t &launches);

// Samples n M2L pairs {T, S, offset slot, level} from the resolved M2L
// tables; -1 entries where the draw found no pair or a cell above the caps.
int order_sample_pairs(const int4 *batches, const int *tlist, const int *src_tab, const int *slot_list,
                       const int *tslot_list, const int *nslots, int nbm, const int *pbeg, const int *pend, int n,
                       unsigned long long seed, int max_nt, int max_ns, int *pairs, cudaStream_t st,
                       int64_t &launches);

// Features of the sampled pairs ([n][ORD_NF]).
int order_pair_features(const int *pairs, int n, const float *cf, int cell0, float ax, float ay, float az,
                        float *feat, cudaStream_t st, int64_t &launches);

// FP64 truncation errors of the sampled pairs at orders 4..p ([n][ORD_NQ],
// log10 of the error over the pair's monopole scale; orders above p = 0).
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

// Hot path: the order of every present slot of every M2L batch (padded
// width into slot_p16) from the MLP, with a row's budget
// log10(tol * F_rms * R^2 / (M_S * sqrt(P))), F_rms the RMS force of the
// previous pass (G = 1 units; <= 0: every slot at full order) and
// P = (sum over M2L pairs of n_T) / n the M2L pairs per particle.
struct InferArgs {
  const int4 *batches;
  const int *tlist, *src_tab, *slot_list, *tslot_list, *nslots;
  const int *pbeg, *pend;
  const float *cf;       // cell features
  const float *M;        // multipoles (M~_0 = source mass)
  const float *params;   // MLP parameters (FP32; weights rounded to BF16 on load)
  const double *frms;    // device: F_rms of the previous pass, G = 1 units
  const unsigned long long *nt_sum;  // device: sum over M2L pairs of n_T
  int64_t n;
  int cell0, KS, p, dim;
  float tol;
  float ax, ay, az;      // cell aspect (extent / largest extent)
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
