/* fmm_gpu.h — C ABI of the B200 FMM force evaluator (libfmmgpu.so).
 *
 * Drop-in boundary for the force pass of rezucch1/nbody-FMM.  The reference's
 * interface is the C++ virtual
 *     SystemUpdateMethod::update(const std::vector<Particle>&)
 *         (src/system_updaters/system_update_method.hpp:24-31)
 * implemented by FMM (src/system_updaters/FMM.cpp:9-12) and NaiveUpdate
 * (src/system_updaters/naive_update.cpp:9-35), and called by
 *     QuadratureMethod::integrate(SystemUpdateMethod*, std::vector<Particle>&, const double&)
 *         (src/quadratures/quadrature_method.hpp:24).
 * A reference-side adapter packs the particles into plain arrays and calls
 * the entry points below (nbody-fmm_b200/cpp/gpu_fmm.hpp: GpuFMM and
 * GpuNaiveUpdate as SystemUpdateMethod implementations).
 *
 * Conventions:
 *  - positions / velocities / accelerations are row-major n x dim FP64
 *    (x0 y0 z0 x1 ...), masses n FP64; all host pointers are caller-owned;
 *  - accelerations follow the reference: a_i = G * grad_i with
 *      3D grad_i = -sum_j m_j (x_i - x_j) / |x_i - x_j|^3     (leaf.cpp:118-142)
 *      2D grad_i = -sum_j m_j (x_i - x_j) / |x_i - x_j|^2     (leaf.cpp:81-95)
 *    and Particle::compute_new_accelaration (particle.cpp:16-21) multiplying by G;
 *  - optional potential output: G * phi, phi_i = sum_j m_j/|d| (3D),
 *    -sum_j m_j log|d| (2D), so that grad = nabla phi;
 *  - every call returns FMM_OK (0) or a negative FMM_ERR_* code; no C++
 *    exception crosses the ABI; fmm_strerror() describes a code;
 *  - one context per host thread; calls on a context are stream-ordered on
 *    the context's stream (or the stream passed to the *_device calls).
 */
#ifndef FMM_GPU_H
#define FMM_GPU_H
#include <stdint.h>

#if defined(__GNUC__)
#define FMM_API __attribute__((visibility("default")))
#else
#define FMM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

enum {
  FMM_OK = 0,
  FMM_ERR_INVALID_ARGUMENT = -1,
  FMM_ERR_CUDA = -2,
  FMM_ERR_OUT_OF_MEMORY = -3,
  FMM_ERR_NONFINITE_INPUT = -4,   /* NaN/Inf position or mass */
  FMM_ERR_NONFINITE_OUTPUT = -5,  /* e.g. coincident particles, as the reference divides by zero */
  FMM_ERR_UNSUPPORTED = -6,
  FMM_ERR_TIMEOUT = -7,
  FMM_ERR_NO_DEVICE = -8,
  FMM_ERR_INTERNAL = -9,
  FMM_ERR_TOO_LARGE = -10,        /* request larger than fmm_direct_noalloc's fixed scratch */
  FMM_ERR_IO = -11                /* a frame file could not be written */
};

/* Order of each M2L pair (FMM_M2L_TC).  FIXED: every pair at p.  GEOMETRIC:
   a pair whose cells are R cell sizes apart is evaluated at the order that
   gives the closest offset's (R = 2) truncation bound at p, plus
   order_margin, clamped to [min(4, p), p].  LEARNED (3D): an MLP set with
   fmm_order_set_model predicts, for each M2L tile (the targets of one tensor-
   core tile at one interaction offset), its pairs' largest truncation error
   at orders 4..12, and the tile takes the lowest order within the pairs'
   share of order_tol (a relative L2 force budget, shared through the RMS
   force of the previous evaluation; the first evaluation of a system runs
   at p).  With
   judge_samples > 0 every learned-order evaluation is checked on that many
   targets against the FP64 direct sum and, if their relative L2 error
   exceeds judge_budget, evaluated again at fixed p (fmm_stats.order_fallbacks);
   judge_every > 1 checks every judge_every-th learned evaluation of a system. */
enum {
  FMM_ORDER_FIXED = 0,
  FMM_ORDER_GEOMETRIC = 1,
  FMM_ORDER_LEARNED = 2
};

/* The order model: a 32 -> 64 -> 64 -> 9 MLP (ReLU), weights used in BF16. */
#define FMM_ORDER_NPARAM 7312
#define FMM_ORDER_NFEAT 32
#define FMM_ORDER_NOUT 9

/* M2L arithmetic. */
enum {
  FMM_M2L_FP32 = 0,  /* SIMT FP32 batched contraction (plain GPU FMM) */
  FMM_M2L_TC = 1     /* M2L, M2M and L2L as tcgen05 tensor-core contractions, 3xBF16 split precision
                        with FP32 accumulation; K <= 176 (3D p <= 12) */
};

/* Direct-sum softening forms. */
enum {
  FMM_SOFT_PLUMMER = 0,   /* r^2 -> r^2 + eps2 in every kernel */
  FMM_SOFT_NAIVE_REF = 1  /* NaiveUpdate's form: 3D m d/((r^2+1e-4) r), 2D m d/(r^2+1e-4) (naive_update.cpp:19-30) */
};

/* Integrators (src/quadratures/). */
enum {
  FMM_INT_SYMPLECTIC_EULER = 0, /* SyplecticEuler::integrate, symplectic_euler.cpp:8-15 */
  FMM_INT_RK4 = 1               /* classical RK4 (RungeKutta4, runge_kutta_4.cpp:10-93, intends this) */
};

typedef struct fmm_config {
  int32_t dim;        /* 2 or 3 (Tensor::dim of the particles) */
  int32_t p;          /* expansion order; the reference hard-codes L = 2 (tree.cpp:94) */
  int32_t leaf_cap;   /* leaf threshold; the reference hard-codes 20 (tree.cpp:32) */
  int32_t m2l_mode;   /* FMM_M2L_* */
  double eps2;        /* softening added to r^2 in the near field (0: the reference FMM) */
  double G;           /* gravitational constant; reference 6.6743e-11 (system_update_method.hpp:17) */
  int32_t device;     /* CUDA device ordinal */
  int32_t direct_max; /* interaction-list pairs (target, source) with n_target * n_source <= direct_max
                         are summed directly (exactly) instead of through M2L; 0 = every pair by M2L
                         as in the reference; -1 = automatic */
  int32_t order_mode; /* FMM_ORDER_*: expansion order of each M2L pair (tensor-core mode only) */
  int32_t order_margin; /* FMM_ORDER_GEOMETRIC: orders added to each reduced pair order */
  float order_tol;      /* FMM_ORDER_LEARNED: relative L2 force budget of the reduced orders (default 2e-6:
                           the tile bound is conservative, the orders it picks add a few 1e-7 to the
                           error of fixed p on the seeded Plummer, mixture and uniform systems) */
  int32_t judge_samples;/* FMM_ORDER_LEARNED: targets checked against the FP64 direct sum (0 = no check) */
  float judge_budget;   /* FMM_ORDER_LEARNED: relative L2 error above which the evaluation is redone at p */
  int32_t judge_every;  /* FMM_ORDER_LEARNED: check every judge_every-th learned evaluation of a system
                           (default 1: every one) */
  int32_t adaptive_leaf;/* adaptive targets (3D trees of depth >= 3; elsewhere ignored): a cell whose parent
                           holds at most this many particles is no target, and each particle sums the
                           particles of the colleagues of its deepest target cell directly.  0 (default):
                           every cell is a target, the reference's uniform tree. */
  int32_t p2p_chunk;    /* adaptive targets: sources per work item of the colleague sums (a multiple of 32 in
                           [32, 4096]; 0: automatic, 256) */
  int32_t m2l_run;      /* FMM_M2L_TC: interaction offsets (slots) per work item of the tensor-core M2L, the
                           batch shape (in [8, 189]; 0: automatic: 24 when there are fewer than four target
                           batches per CTA, else a whole batch) */
} fmm_config;

typedef struct fmm_stats {
  int32_t depth;            /* leaf depth of the last tree */
  int32_t n_levels;
  int64_t n_leaves;
  int64_t n_cells;          /* all levels */
  int64_t m2l_pairs;        /* interaction-list pairs evaluated by M2L */
  int64_t p2p_pairs;        /* particle pairs evaluated directly (near field + direct far field) */
  double ms_tree;           /* device time of the tree build */
  double ms_upward;         /* P2M + M2M */
  double ms_m2l;
  double ms_downward;       /* L2L + L2P */
  double ms_p2p;            /* near field + direct far field + output */
  double ms_total;          /* whole force pass (device time) */
  int64_t m2l_tiles;        /* FMM_M2L_TC: 128-row (target batch, slot) tiles of the M2L contraction */
  double ms_far_direct;     /* the direct far field part of ms_p2p */
  int64_t far_direct_pairs; /* the direct far field part of p2p_pairs */
  int64_t direct_max;       /* the direct-pair threshold the pass used */
  double judge_rel_l2;      /* FMM_ORDER_LEARNED with judge_samples: the checked relative L2 error */
  int64_t order_fallbacks;  /* FMM_ORDER_LEARNED: 1 if the judge sent the evaluation back to fixed p */
  int64_t m2l_width_sum;    /* FMM_M2L_TC: sum over the M2L tiles of their padded width (16 ceil(K_q / 16)) */
  double reserved[7];
} fmm_stats;

typedef struct fmm_ctx fmm_ctx;

FMM_API const char *fmm_strerror(int code);
FMM_API const char *fmm_version(void);

/* Defaults: dim 3, p 8, leaf_cap 64, FP32 M2L, eps2 0, G 1, device 0, direct_max -1. */
FMM_API int fmm_config_default(fmm_config *cfg);

/* Creates a context (allocates device workspace lazily, grown on demand). */
FMM_API int fmm_create(const fmm_config *cfg, fmm_ctx **out);
FMM_API int fmm_destroy(fmm_ctx *ctx);

/* One FMM force pass from host buffers: replaces FMM::update
 * (FMM.cpp:9-12) — builds the tree (Tree::init_tree, tree.cpp:15-91) and runs
 * P2M, M2M, M2L, L2L, L2P and P2P (tree.cpp:93-111).  acc: n x dim, pot
 * nullable.  Synchronous. */
FMM_API int fmm_evaluate(fmm_ctx *ctx, int64_t n, const double *pos, const double *mass, double *acc, double *pot);

/* The same pass on device-resident buffers, ordered on `stream`
 * (a cudaStream_t; NULL = the context's stream).  Returns after enqueueing
 * the work; call fmm_synchronize() before reading the results or the status
 * of the device-side checks. */
FMM_API int fmm_evaluate_device(fmm_ctx *ctx, int64_t n, const double *d_pos, const double *d_mass, double *d_acc,
                        double *d_pot, void *stream);
/* Waits for the context's stream and for the stream of the last
 * fmm_evaluate_device call (which must still exist), not for the whole
 * device, then returns the status of the device-side checks. */
FMM_API int fmm_synchronize(fmm_ctx *ctx);

/* Batched ensemble: nsys independent systems stored one after another in
   the device arrays (system s = elements [offsets[s], offsets[s+1]) of
   n x dim positions, masses, accelerations; offsets: host, nsys + 1 values
   from 0).  Each system gets its own tree and force pass, as fmm_evaluate
   would give it, at fixed p; the passes of different systems run
   concurrently on a pool of `workers` streams (0: min(nsys, 8)), each fed
   by its own host thread.  Synchronous; fmm_last_stats then holds the sums
   of the counts and the wall time in ms_total. */
FMM_API int fmm_evaluate_batched(fmm_ctx *ctx, int32_t nsys, const int64_t *offsets, const double *d_pos,
                                 const double *d_mass, double *d_acc, double *d_pot, int32_t workers);

/* Autotuner: times force evaluations of the given system (device buffers)
   over candidate settings and keeps the fastest in the context: the
   direct-pair threshold (K^2/200 .. K^2/12.5, K the expansion length; five
   candidates) or, with FMM_TUNE_LEAF, a coordinate search: the leaf
   capacity in {32, 64, 128, 256} (which changes the tree: the reference's
   algorithm at that threshold) at the threshold K^2/25, then the thresholds
   K^2/100, K^2/50 and K^2/12.5 at the best capacity (seven candidates).
   Every candidate keeps the configured adaptive_leaf; with FMM_TUNE_ADAPTIVE
   the values 0 (the uniform targets), 16, 32 and 64 are then tried at the
   best candidate's leaf capacity and threshold, then the best threshold
   times 1/sqrt(2) and sqrt(2); with FMM_TUNE_KERNELS the kernel shapes last
   (at most 16 candidates in all).  Adaptive targets change
   only which pairs are summed directly (exactly), not the expansions, so
   the candidates differ in time, not in truncation error.  Learned orders are tuned with them (every candidate is evaluated twice,
   the second timed).  result may be NULL.  Synchronous. */
#define FMM_TUNE_LEAF 1
#define FMM_TUNE_ADAPTIVE 2 /* then adaptive_leaf in {0, 16, 32, 64} at the best of the above, and the
                               threshold times 1/sqrt(2) and sqrt(2) at the best of those */
#define FMM_TUNE_KERNELS 4  /* then the kernel shapes at the best of the above: p2p_chunk in {128, 512}
                               (with adaptive targets) and m2l_run in {24, 189} (tensor-core M2L) */
typedef struct fmm_tune_result {
  int32_t n_candidates;
  int32_t best;            /* index of the chosen candidate */
  int32_t leaf_cap[16];    /* candidates */
  int32_t direct_max[16];
  double ms[16];           /* device time of each candidate's timed evaluation */
  int32_t adaptive_leaf[16];
  int32_t p2p_chunk[16];
  int32_t m2l_run[16];
} fmm_tune_result;
FMM_API int fmm_autotune(fmm_ctx *ctx, int64_t n, const double *d_pos, const double *d_mass, int32_t flags,
                         fmm_tune_result *result, void *stream);

/* FP64 O(N^2) direct sum on the GPU for `ntargets` target indices (all if
 * targets is NULL): replaces NaiveUpdate::update (naive_update.cpp:9-35)
 * when soft_mode is FMM_SOFT_NAIVE_REF; otherwise the Plummer form with
 * cfg.eps2.  Host buffers; acc is ntargets x dim. */
FMM_API int fmm_direct(fmm_ctx *ctx, int64_t n, const double *pos, const double *mass, int64_t ntargets,
               const int64_t *targets, int32_t soft_mode, double *acc, double *pot);
FMM_API int fmm_direct_device(fmm_ctx *ctx, int64_t n, const double *d_pos, const double *d_mass, int64_t ntargets,
                      const int64_t *d_targets, int32_t soft_mode, double *d_acc, double *d_pot, void *stream);

/* Advances pos/vel (host, n x dim, in place) by `steps` steps of `method`
 * with time step dt, the state staying on the device between steps:
 * replaces QuadratureMethod::integrate with an FMM update method
 * (symplectic_euler.cpp:8-15; runge_kutta_4.cpp:10-93).  acc_out (nullable)
 * receives the acceleration of the last force evaluation. */
FMM_API int fmm_integrate(fmm_ctx *ctx, int32_t method, double dt, int32_t steps, int64_t n, double *pos, double *vel,
                  const double *mass, double *acc_out);

/* Tree export, for bit-exact comparison with Tree::init_tree (tree.cpp:15-91).
 * fmm_tree_build builds the tree of `pos` (host) and keeps it; the getters
 * copy it out.  Leaves are in ascending key order, each leaf's particles in
 * input order (tree.cpp:62-66); perm[start[i]..start[i+1]) are the indices
 * of leaf i.  Level d keys are ascending. */
FMM_API int fmm_tree_build(fmm_ctx *ctx, int64_t n, const double *pos);
FMM_API int fmm_tree_depth(fmm_ctx *ctx, int32_t *depth);
FMM_API int fmm_tree_level_size(fmm_ctx *ctx, int32_t level, int64_t *count);
FMM_API int fmm_tree_level_keys(fmm_ctx *ctx, int32_t level, uint64_t *keys);
FMM_API int fmm_tree_leaves(fmm_ctx *ctx, uint64_t *keys, int64_t *start, int64_t *perm);
/* Neighbour (kind 0, |delta| <= 1, self excluded) or interaction (kind 1)
 * list pairs of level d as (target key, source key): the lists of
 * NodeI::compute_interaction_list (node_i.cpp:23-99).  With tkey == NULL
 * only *count is set.  The tree must come from fmm_tree_build (a force pass
 * with adaptive targets keeps colleague rows of its target cells only, and
 * then this returns FMM_ERR_INVALID_ARGUMENT). */
FMM_API int fmm_tree_pairs(fmm_ctx *ctx, int32_t level, int32_t kind, int64_t *count, uint64_t *tkey, uint64_t *skey);

/* Adaptive-target flags (fmm_config.adaptive_leaf = A) of every cell of the
 * tree kept by fmm_tree_build, level by level from the root, each level in
 * ascending key order (the order of fmm_tree_level_keys): bit 0, a target
 * (the root, or a cell whose parent holds more than A particles); bit 1, an
 * adaptive leaf (a target with at most A particles, or a leaf).  flags holds
 * the tree's cell count (the sum of fmm_tree_level_size over its levels).
 * No counterpart in the reference, whose targets are every cell of its
 * uniform-depth tree (tree.cpp:43-69, node_i.cpp:105-120). */
FMM_API int fmm_tree_adaptive_flags(fmm_ctx *ctx, int32_t adaptive_leaf, uint8_t *flags);

/* FP64 direct sum that allocates no device memory and needs no context.
 * It has no counterpart in the reference (whose NaiveUpdate allocates
 * freely on the host).  It is for callers that cannot call cudaMalloc when
 * they need forces: codes whose own pool owns all device memory, callers
 * under a fixed memory budget, and threads that must not block on the
 * device the way cudaMalloc/cudaFree can.  Inputs and outputs are the
 * caller's device buffers (layouts as in fmm_direct_device; targets, if
 * given, must lie in [0, n)); it runs on the current device, ordered on
 * `stream` (NULL = the legacy default stream), and returns after enqueueing.
 * Its only scratch is a fixed array of FMM_NOALLOC_MAX_TARGETS partial sums
 * (8 MiB) that every GPU loading this library holds until the process
 * exits; requests with more than FMM_NOALLOC_MAX_TARGETS targets return
 * FMM_ERR_TOO_LARGE.  The first call on a device looks up that array's
 * device address (cudaGetSymbolAddress), so make it before any stream
 * capture.  All calls on a device share the array: calls that overlap on
 * the GPU (e.g. on two streams at once) race and give wrong results. */
#define FMM_NOALLOC_MAX_TARGETS 262144
FMM_API int fmm_direct_noalloc(int32_t dim, int64_t n, const double *d_pos, const double *d_mass, int64_t ntargets,
                               const int64_t *d_targets, int32_t soft_mode, double eps2, double G, double *d_acc,
                               double *d_pot, void *stream);

/* Frame output: replaces HDF5Exporter (io/hdf5_exporter.cpp:10-128) for a
 * simulation loop that writes a frame per step (main.cpp:85-91).  Each
 * frame holds the reference's datasets, the order and shapes of
 * write_frame (hdf5_exporter.cpp:24-44, 70-73): position, velocity and
 * acceleration as n x 3 FP64 (2D padded with z = 0) and weight as n FP64,
 * stored one after another, little-endian, in `<dir>/<base>_<step:05>.bin`
 * (the reference: `.h5` datasets; libhdf5 is not used).  After every frame
 * `<dir>/<base>.xmf` is rewritten as the reference's temporal collection
 * (hdf5_exporter.cpp:83-128), its data items pointing into the .bin files
 * (Format="Binary", Seek = byte offset of each dataset), so ParaView reads
 * the series as it reads the reference's.  fmm_frames_open creates `dir`
 * (like the constructor, hdf5_exporter.cpp:10-13); a frame of n = 0 is
 * skipped (hdf5_exporter.cpp:22).
 *
 * fmm_frames_write takes host arrays (n x dim positions, velocities and
 * accelerations, n masses; acc may be NULL: zeros) and writes the frame
 * before it returns.  fmm_frames_write_device takes device arrays on the
 * current device: it enqueues a device-to-device snapshot of them on
 * `stream`, after the work already queued there, and returns; work queued
 * on `stream` afterwards may change the arrays at once.  The snapshot is
 * copied to page-locked staging on a stream of the writer's own, and a
 * writer thread writes the file when that copy has completed, so the host
 * copy and the file writing overlap the caller's next steps.  Two frames
 * can be in flight (two snapshots of 80 bytes per particle on the device,
 * two staging buffers on the host); a third call waits for the oldest.
 * Frames are written in call order; all device frames of a writer come
 * from one device.  fmm_frames_flush waits for every frame in flight and
 * returns the first error met (FMM_ERR_IO, FMM_ERR_CUDA); fmm_frames_close
 * flushes and frees. */
typedef struct fmm_frames fmm_frames;
FMM_API int fmm_frames_open(const char *dir, const char *base, int32_t dim, fmm_frames **out);
FMM_API int fmm_frames_write(fmm_frames *f, int64_t n, const double *pos, const double *vel, const double *acc,
                             const double *mass, int32_t step, double time);
FMM_API int fmm_frames_write_device(fmm_frames *f, int64_t n, const double *d_pos, const double *d_vel,
                                    const double *d_acc, const double *d_mass, int32_t step, double time,
                                    void *stream);
FMM_API int fmm_frames_flush(fmm_frames *f);
FMM_API int fmm_frames_close(fmm_frames *f);

/* The reference's simulation loop (main.cpp:85-91: write a frame, then
 * integrate a step) with the state on the device: as fmm_integrate, and
 * before each step s = 0, every, 2 every, ... a frame of the state through
 * fmm_frames_write_device (step number step0 + s, time t0 + s dt; the
 * acceleration of the last force evaluation, zeros before the first step).
 * The frames overlap the following steps; the call flushes them before it
 * returns. */
FMM_API int fmm_integrate_frames(fmm_ctx *ctx, int32_t method, double dt, int32_t steps, int64_t n, double *pos,
                                 double *vel, const double *mass, double *acc_out, fmm_frames *frames, int32_t every,
                                 int32_t step0, double t0);

/* Statistics of the last force pass (per-phase device times, sizes). */
FMM_API int fmm_last_stats(fmm_ctx *ctx, fmm_stats *out);

/* Number of kernel launches the library issued since the context was
 * created (all entry points). */
FMM_API int64_t fmm_launch_count(fmm_ctx *ctx);

/* Learned pair orders.  Parameters are FMM_ORDER_NPARAM floats (host). */
FMM_API int fmm_order_set_model(fmm_ctx *ctx, const float *params, int32_t nparams);
FMM_API int fmm_order_get_model(fmm_ctx *ctx, float *params, int32_t nparams);
/* One force evaluation (fixed p; 3D, FMM_M2L_TC) that samples ntiles of its
   M2L tiles (128 targets at one interaction offset) and writes their
   features (d_feat, ntiles x FMM_ORDER_NFEAT) and labels (d_labels, ntiles x
   FMM_ORDER_NOUT): for every order q in 4..12 the base-10 logarithm of the
   largest over the tile's pairs of e(q) / sqrt(n_T) * R^2 / M_tot, e(q) the
   pair's FP64 truncation error over its target particles (G = 1).  Rows
   where the draw found no tile are all zero.  Device buffers; synchronous. */
FMM_API int fmm_order_collect(fmm_ctx *ctx, int64_t n, const double *d_pos, const double *d_mass, int32_t ntiles,
                              uint64_t seed, float *d_feat, float *d_labels, void *stream);
/* Trains the context's model in place on the GPU (Adam, mean squared error
   of the predicted logarithms; device data, rows used in order);
   loss_out (host, epochs floats) receives the mean loss of each epoch. */
FMM_API int fmm_order_train(fmm_ctx *ctx, const float *d_feat, const float *d_labels, int32_t n, int32_t epochs,
                            int32_t batch, float lr, float *loss_out);
/* Predictions (n x FMM_ORDER_NOUT), the mean squared error and its gradient
   with respect to the parameters, for n rows (device buffers). */
FMM_API int fmm_order_forward_grad(const float *d_feat, const float *d_labels, int32_t n, const float *d_params,
                                   float *d_pred, float *d_grad, float *d_loss, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* FMM_GPU_H */
