/* CPU restatement of the rezucch1/nbody-FMM force pass — TEST INFRASTRUCTURE.
 *
 * This library is the checker for the CUDA path: only tests, the smoke entry
 * and the CPU-baseline leg of bench.py load it.  The product never links it.
 *
 * Conventions shared with the CUDA path:
 *  - positions are row-major n x dim FP64, masses n FP64;
 *  - "grad" is the reference's potential gradient (acceleration = G * grad):
 *      3D: grad_i = -sum_j m_j d_ij / |d_ij|^3,  d_ij = x_i - x_j
 *      2D: grad_i = -sum_j m_j d_ij / |d_ij|^2
 *    (leaf.cpp:118-142 and :81-95); "pot" is phi with grad = nabla phi:
 *      3D: phi_i = sum_j m_j / |d_ij|,  2D: phi_i = -sum_j m_j log |d_ij|.
 */
#ifndef FMM_ORACLE_H
#define FMM_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_tree orc_tree;

/* Tree::init_tree (tree_components/tree.cpp:15-91) + compute_interaction_list
 * (node_i.cpp:23-99), restated with sort-based binning and 64-bit keys. */
orc_tree *orc_tree_build(int dim, int64_t n, const double *pos, unsigned threshold);
void orc_tree_free(orc_tree *t);
int orc_tree_depth(const orc_tree *t);
void orc_tree_box(const orc_tree *t, double *lo, double *hi);
int64_t orc_tree_level_size(const orc_tree *t, int d);
int64_t orc_tree_level_keys(const orc_tree *t, int d, uint64_t *keys);
int64_t orc_tree_leaves(const orc_tree *t, uint64_t *keys, int64_t *start, int64_t *perm);
/* kind 0 = neighbour list (|delta|<=1, self excluded), 1 = interaction list */
int64_t orc_tree_npairs(const orc_tree *t, int d, int kind);
int64_t orc_tree_pairs(const orc_tree *t, int d, int kind, uint64_t *tkey, uint64_t *skey);

/* Morton::encode / decode (morton_code.cpp:9-36): bit b of coordinate i goes
 * to bit i + b*dim. */
uint64_t orc_morton_encode(const uint32_t *c, int dim);
void orc_morton_decode(uint64_t code, int dim, uint32_t *c);

/* FP64 direct sum over all sources for the given targets (all if targets is
 * NULL): grad as above with r^2 -> r^2 + eps2. */
void orc_direct(int dim, int64_t n, const double *pos, const double *mass, double eps2,
                int64_t ntargets, const int64_t *targets, double *grad, double *pot);

/* NaiveUpdate::update (naive_update.cpp:9-35) with its fixed softening:
 * 3D grad -= m d / ((r^2 + 1e-4) r), 2D grad -= m d / (r^2 + 1e-4). */
void orc_naive_ref(int dim, int64_t n, const double *pos, const double *mass, double *grad);

/* Full FMM force pass on the reference's uniform-depth tree, FP64.
 * centre_mode 0: geometric cell centres; 1: the reference's mass centres
 * (leaf.cpp:37-54, node.cpp:70-86).
 * 3D uses correct solid-harmonic operators (the reference's 3D M2M/M2L/L2L
 * are not convergent); 2D follows multipole_set2D.cpp / local_set2D.cpp. */
int orc_fmm(int dim, int64_t n, const double *pos, const double *mass, unsigned p, unsigned threshold,
            int centre_mode, double *grad, double *pot);
/* The same with a near-field softening eps2 (r^2 -> r^2 + eps2 in P2P and
 * in the direct far field) and a direct far field: interaction-list pairs
 * with n_target * n_source <= direct_max are summed particle by particle
 * instead of by M2L (0 = none, as the reference). */
int orc_fmm_ex(int dim, int64_t n, const double *pos, const double *mass, unsigned p, unsigned threshold,
               int centre_mode, double eps2, int64_t direct_max, double *grad, double *pot);
/* Adaptive targets on the uniform tree (3D and 2D, geometric centres): targets stop
 * descending at cells of at most `aleaf` particles, whose particles then sum
 * their colleagues' particles directly (with the W list for large ones). */
int orc_fmm_adaptive(int dim, int64_t n, const double *pos, const double *mass, unsigned p, unsigned threshold,
                     unsigned aleaf, double eps2, int64_t direct_max, int64_t w_direct_max, double *grad,
                     double *pot);
/* orc_fmm_adaptive's flags of every cell, level by level in the order of
 * orc_tree_level_keys: bit 0 active target, bit 1 adaptive leaf.  Returns
 * the number of cells (nothing written if above cap), or -1. */
int64_t orc_adaptive_flags(int dim, int64_t n, const double *pos, unsigned threshold, unsigned aleaf, int64_t cap,
                           uint8_t *flags);

/* Scaled solid harmonics used by the CUDA path, m >= 0 only, packed
 * idx(n,m) = n(n+1)/2 + m, complex as (re, im):
 *   Rs_n^m = R_n^m / sqrt((n-m)!(n+m)!),  Is_n^m = I_n^m * sqrt((n-m)!(n+m)!)
 * where R, I are the reference's Racah-normalised harmonics
 * (power_set3D.cpp:10-48, irregular.cpp:10-57). */
void orc_regular_scaled(unsigned p, const double *r, double *out);
void orc_irregular_scaled(unsigned p, const double *r, double *out);
/* Racah-normalised harmonics in the reference's (L+1)^2 layout. */
void orc_regular_racah(unsigned p, const double *r, double *out);
void orc_irregular_racah(unsigned p, const double *r, double *out);
/* P2M: M_n^m = sum_i m_i conj(Rs_n^m(x_i - c)), packed m >= 0. */
void orc_p2m_3d(unsigned p, int64_t n, const double *pos, const double *mass, const double *c, double *out);

#ifdef __cplusplus
}
#endif
#endif
