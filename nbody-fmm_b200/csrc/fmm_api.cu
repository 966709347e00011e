// C ABI of libfmmgpu.so (declared in include/fmm_gpu.h).
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <thread>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "direct.cuh"
#include "expansions.cuh"
#include "fmm_gpu.h"
#include "m2l_tc.cuh"

namespace fmm {
static thread_local std::string g_cuda_err;
void set_cuda_error(cudaError_t e, const char *what, const char *file, int line) {
  char buf[512];
  snprintf(buf, sizeof(buf), "%s (%s) at %s:%d", cudaGetErrorString(e), what, file, line);
  g_cuda_err = buf;
}
const char *last_cuda_error_text() { return g_cuda_err.c_str(); }
}  // namespace fmm

using namespace fmm;

struct fmm_ctx {
  fmm_config cfg;
  cudaStream_t stream = nullptr;
  cudaStream_t last_stream = nullptr;  // the stream of the last fmm_evaluate_device call (what fmm_synchronize waits on)
  Workspace ws;
  TreeState tree;
  OpTables ops;
  ExpBuffers eb;
  DevBuf<double> d_pos, d_mass, d_acc, d_pot, d_vel, d_x0, d_v0, d_xs, d_vs, d_asum, d_vsum;
  DevBuf<int64_t> d_targets;
  // learned pair orders
  DevBuf<float> order_params;
  bool has_model = false;
  int64_t frms_n = -1;         // system size the cached F_rms belongs to
  int64_t learned_evals = 0;   // learned evaluations of that system so far (judge cadence)
  DevBuf<int64_t> judge_tg;    // judge targets of (judge_n, judge_k)
  DevBuf<double> judge_ref, judge_sum;
  int64_t judge_n = -1, judge_k = -1;
  std::vector<fmm_ctx *> workers;  // batched ensemble: worker contexts (own stream and buffers)
  DevBuf<int> col_pairs, col_tiles;
  DevBuf<float> col_plabels;
  fmm_stats stats;
  cudaEvent_t ev[7] = {};  // pass boundaries; ev[6] ends the direct far field
  bool timing_pending = false;
  bool have_tree = false;
};

static int check_cfg(const fmm_config *c) {
  if (!c) return FMM_ERR_INVALID_ARGUMENT;
  if (c->dim != 2 && c->dim != 3) return FMM_ERR_INVALID_ARGUMENT;
  if (c->p < 0 || c->p > FMM_MAX_P) return FMM_ERR_INVALID_ARGUMENT;
  if (c->dim == 3 && (c->p + 1) * (c->p + 1) > 192) return FMM_ERR_UNSUPPORTED;  // contraction register tile
  if (c->leaf_cap < 1) return FMM_ERR_INVALID_ARGUMENT;
  if (c->m2l_mode != FMM_M2L_FP32 && c->m2l_mode != FMM_M2L_TC) return FMM_ERR_INVALID_ARGUMENT;
  if (!(c->eps2 >= 0.0)) return FMM_ERR_INVALID_ARGUMENT;
  if (c->direct_max < -1) return FMM_ERR_INVALID_ARGUMENT;
  if (c->m2l_mode == FMM_M2L_TC && (c->dim == 3 ? (c->p + 1) * (c->p + 1) : 2 * c->p + 1) > TC_MAX_P16)
    return FMM_ERR_UNSUPPORTED;  // tensor-core tiles hold K <= 176 (p <= 12 in 3D)
  if (c->order_mode != FMM_ORDER_FIXED && c->order_mode != FMM_ORDER_GEOMETRIC && c->order_mode != FMM_ORDER_LEARNED)
    return FMM_ERR_INVALID_ARGUMENT;
  if (c->order_mode == FMM_ORDER_LEARNED && c->dim != 3) return FMM_ERR_UNSUPPORTED;
  if (c->order_mode == FMM_ORDER_LEARNED && !(c->order_tol > 0.f)) return FMM_ERR_INVALID_ARGUMENT;
  if (c->judge_samples < 0 || !(c->judge_budget > 0.f) || c->judge_every < 1) return FMM_ERR_INVALID_ARGUMENT;
  if (c->order_mode != FMM_ORDER_FIXED && c->m2l_mode != FMM_M2L_TC)
    return FMM_ERR_UNSUPPORTED;  // per-pair orders live in the tensor-core kernel; the plain FMM is fixed-p
  if (c->order_margin < 0 || c->order_margin > FMM_MAX_P) return FMM_ERR_INVALID_ARGUMENT;
  if (c->adaptive_leaf < 0) return FMM_ERR_INVALID_ARGUMENT;
  if (c->p2p_chunk != 0 && (c->p2p_chunk < 32 || c->p2p_chunk > 4096 || c->p2p_chunk % 32)) return FMM_ERR_INVALID_ARGUMENT;
  if (c->m2l_run != 0 && (c->m2l_run < 8 || c->m2l_run > 189)) return FMM_ERR_INVALID_ARGUMENT;
  return FMM_OK;
}

extern "C" {

const char *fmm_strerror(int code) {
  switch (code) {
    case FMM_OK: return "ok";
    case FMM_ERR_INVALID_ARGUMENT: return "invalid argument";
    case FMM_ERR_CUDA: return fmm::last_cuda_error_text()[0] ? fmm::last_cuda_error_text() : "CUDA error";
    case FMM_ERR_OUT_OF_MEMORY: return "out of device memory";
    case FMM_ERR_NONFINITE_INPUT: return "non-finite position or mass";
    case FMM_ERR_NONFINITE_OUTPUT: return "non-finite acceleration (coincident particles?)";
    case FMM_ERR_UNSUPPORTED: return "unsupported configuration";
    case FMM_ERR_TIMEOUT: return "device wait timed out";
    case FMM_ERR_NO_DEVICE: return "no CUDA device";
    case FMM_ERR_TOO_LARGE: return "more targets than fmm_direct_noalloc's fixed scratch holds (FMM_NOALLOC_MAX_TARGETS)";
    case FMM_ERR_IO: return "a frame file could not be written";
    default: return "internal error";
  }
}

const char *fmm_version(void) { return "fmmgpu 0.1 (sm_100a)"; }

int fmm_config_default(fmm_config *cfg) {
  if (!cfg) return FMM_ERR_INVALID_ARGUMENT;
  memset(cfg, 0, sizeof(*cfg));
  cfg->dim = 3;
  cfg->p = 8;
  cfg->leaf_cap = 64;
  cfg->m2l_mode = FMM_M2L_FP32;
  cfg->eps2 = 0.0;
  cfg->G = 1.0;
  cfg->device = 0;
  cfg->direct_max = -1;
  cfg->order_mode = FMM_ORDER_FIXED;
  cfg->order_margin = 1;
  cfg->order_tol = 2e-6f;
  cfg->judge_samples = 0;
  cfg->judge_budget = 1e-6f;
  cfg->judge_every = 1;
  return FMM_OK;
}

int fmm_create(const fmm_config *cfg, fmm_ctx **out) {
  if (!out) return FMM_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int rc = check_cfg(cfg);
  if (rc) return rc;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return FMM_ERR_NO_DEVICE;
  if (cfg->device < 0 || cfg->device >= ndev) return FMM_ERR_INVALID_ARGUMENT;
  CUDA_TRY(cudaSetDevice(cfg->device));
  fmm_ctx *c = new (std::nothrow) fmm_ctx();
  if (!c) return FMM_ERR_OUT_OF_MEMORY;
  c->cfg = *cfg;
  memset(&c->stats, 0, sizeof(c->stats));
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return FMM_ERR_CUDA;
  }
  for (auto &e : c->ev) cudaEventCreate(&e);
  if (!c->ws.init_small()) {
    fmm_destroy(c);
    return FMM_ERR_OUT_OF_MEMORY;
  }
  upload_class_tables();
  *out = c;
  return FMM_OK;
}

int fmm_destroy(fmm_ctx *c) {
  if (!c) return FMM_ERR_INVALID_ARGUMENT;
  for (fmm_ctx *w : c->workers) fmm_destroy(w);
  c->workers.clear();
  cudaSetDevice(c->cfg.device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  c->ws.release_all();
  c->ops.tab.release();
  c->ops.scratch.release();
  c->eb.M.release();
  c->eb.L.release();
  c->eb.tlist.release();
  c->eb.batches.release();
  c->eb.cls_count.release();
  c->eb.ckey.release();
  c->eb.ckey_alt.release();
  c->eb.cval.release();
  c->eb.cval2.release();
  c->eb.ckey_m2l.release();
  c->eb.tlist_m2l.release();
  c->eb.lvl_off.release();
  c->eb.m2l_src.release();
  c->eb.m2l_list.release();
  c->eb.m2l_nslots.release();
  c->eb.m2l_tslot.release();
  c->eb.tc_img.release();
  c->eb.tc_work.release();
  c->eb.order_p16.release();
  c->eb.fdirect.release();
  c->eb.m2l_split.release();
  c->eb.lact.release();
  c->eb.batches2.release();
  c->eb.esrc.release();
  c->eb.elev.release();
  c->eb.ukey.release();
  c->eb.p2m_list.release();
  c->eb.ftl.release();
  c->eb.xs.release();
  c->eb.ccnt.release();
  c->eb.citems.release();
  c->eb.hbatches.release();
  c->eb.hbatches2.release();
  c->eb.uval.release();
  c->eb.m2l_split_w.release();
  c->eb.m2l_w.release();
  c->eb.cf.release();
  c->eb.frms.release();
  c->ops.tab64.release();
  c->order_params.release();
  c->judge_tg.release();
  c->judge_ref.release();
  c->judge_sum.release();
  c->col_pairs.release();
  c->col_tiles.release();
  c->col_plabels.release();
  for (auto *b : {&c->d_pos, &c->d_mass, &c->d_acc, &c->d_pot, &c->d_vel, &c->d_x0, &c->d_v0, &c->d_xs, &c->d_vs,
                  &c->d_asum, &c->d_vsum})
    b->release();
  c->d_targets.release();
  for (auto &e : c->ev)
    if (e) cudaEventDestroy(e);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return FMM_OK;
}

// Cut-off of the direct far field: pairs with n_t * n_s <= threshold are
// summed particle by particle.  Automatic: the product at which one pair of
// M2L (2 K^2 flops, K = (p+1)^2 in 3D) costs as much as n_t * n_s direct
// interactions (~20 flops each), scaled by the contraction's lower
// efficiency.
static int64_t direct_threshold(const fmm_config &c) {
  if (c.direct_max >= 0) return c.direct_max;
  int K = c.dim == 3 ? (c.p + 1) * (c.p + 1) : 2 * c.p + 1;
  return std::max<int64_t>(8, (int64_t)(2.0 * K * K / 20.0 / 2.5));
}

// One force pass: tree, operators, expansions, near field.
static int pass(fmm_ctx *c, int64_t n, const double *d_pos, const double *d_mass, double *d_acc, double *d_pot,
                cudaStream_t st, const OrderOpts &oo, bool want64) {
  const int dim = c->cfg.dim;
  CUDA_TRY(cudaEventRecord(c->ev[0], st));
  int rc = build_tree(c->ws, c->tree, d_pos, d_mass, n, dim, c->cfg.leaf_cap, st, c->cfg.adaptive_leaf);
  if (rc) return rc;
  if (!c->ws.ok) return FMM_ERR_OUT_OF_MEMORY;
  c->have_tree = true;
  PassGeom g;
  g.emax = 0;
  for (int d = 0; d < 3; ++d) {
    g.lo[d] = c->tree.lo[d];
    g.ext[d] = d < dim ? c->tree.hi[d] - c->tree.lo[d] : 0.0;
    g.emax = std::max(g.emax, g.ext[d]);
  }
  rc = build_op_tables(c->ops, dim, c->cfg.p, c->tree.depth, g, st, c->ws.launches, want64);
  if (rc) return rc;
  const double jr = c->stats.judge_rel_l2;
  const int64_t fb = c->stats.order_fallbacks;
  memset(&c->stats, 0, sizeof(c->stats));
  c->stats.judge_rel_l2 = jr;
  c->stats.order_fallbacks = fb;
  rc = run_fmm_passes(c->ws, c->tree, c->ops, c->eb, d_pos, d_mass, c->cfg.p, c->cfg.eps2, c->cfg.G, g, d_acc, d_pot,
                      c->cfg.m2l_mode, direct_threshold(c->cfg), oo, st, c->stats, c->ev, c->cfg.adaptive_leaf,
                      c->cfg.p2p_chunk, c->cfg.m2l_run);
  c->stats.direct_max = direct_threshold(c->cfg);
  if (rc) return rc;
  if (!c->ws.ok) return FMM_ERR_OUT_OF_MEMORY;
  c->stats.depth = c->tree.depth;
  c->stats.n_levels = c->tree.depth + 1;
  c->stats.n_leaves = c->tree.level_count[c->tree.depth];
  c->timing_pending = true;
  return FMM_OK;
}

// Relative L2 error of d_acc on judge_samples targets against the FP64
// direct sum (synchronous).
static int judge(fmm_ctx *c, int64_t n, const double *d_pos, const double *d_mass, const double *d_acc,
                 cudaStream_t st, double &rel) {
  const int dim = c->cfg.dim;
  const int64_t k = std::min<int64_t>(c->cfg.judge_samples, n);
  if (c->judge_n != n || c->judge_k != k) {
    std::vector<int64_t> tg(k);
    for (int64_t i = 0; i < k; ++i) tg[i] = (int64_t)(((double)i + 0.5) * (double)n / (double)k);
    if (!c->judge_tg.reserve(k) || !c->judge_ref.reserve((size_t)k * dim) || !c->judge_sum.reserve(2))
      return FMM_ERR_OUT_OF_MEMORY;
    CUDA_TRY(cudaMemcpyAsync(c->judge_tg.ptr, tg.data(), sizeof(int64_t) * k, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    c->judge_n = n;
    c->judge_k = k;
  }
  int rc = direct_sum(d_pos, d_mass, n, c->judge_tg.ptr, k, dim, c->cfg.eps2, FMM_SOFT_PLUMMER, c->cfg.G,
                      c->judge_ref.ptr, nullptr, st, c->ws.launches);
  if (rc) return rc;
  rc = order_judge_compare(d_acc, c->judge_ref.ptr, c->judge_tg.ptr, k, dim, c->judge_sum.ptr, st, c->ws.launches);
  if (rc) return rc;
  double h[2] = {0.0, 0.0};
  CUDA_TRY(cudaMemcpyAsync(h, c->judge_sum.ptr, sizeof(h), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  rel = h[1] > 0.0 ? std::sqrt(h[0] / h[1]) : 0.0;
  return FMM_OK;
}

static int evaluate_device(fmm_ctx *c, int64_t n, const double *d_pos, const double *d_mass, double *d_acc,
                           double *d_pot, cudaStream_t st) {
  if (n < 0 || n > (int64_t)INT32_MAX) return FMM_ERR_INVALID_ARGUMENT;
  if (n == 0) return FMM_OK;
  if (!d_pos || !d_mass || !d_acc) return FMM_ERR_INVALID_ARGUMENT;
  OrderOpts oo;
  oo.mode = c->cfg.order_mode;
  oo.margin = c->cfg.order_margin;
  oo.tol = c->cfg.order_tol;
  const bool learned = c->cfg.order_mode == FMM_ORDER_LEARNED && c->cfg.m2l_mode == FMM_M2L_TC;
  c->stats.judge_rel_l2 = 0.0;
  c->stats.order_fallbacks = 0;
  if (learned) {
    if (!c->has_model) return FMM_ERR_INVALID_ARGUMENT;  // no order model set
    oo.params = c->order_params.ptr;
    if (!c->eb.frms.reserve(3)) return FMM_ERR_OUT_OF_MEMORY;
    if (c->frms_n != n) {  // a new system: its first evaluation runs at fixed p
      CUDA_TRY(cudaMemsetAsync(c->eb.frms.ptr, 0, 3 * sizeof(double), st));
      c->frms_n = n;
      c->learned_evals = 0;
    }
  }
  int rc = pass(c, n, d_pos, d_mass, d_acc, d_pot, st, oo, false);
  if (rc) return rc;
  if (!learned) return FMM_OK;
  if (c->cfg.judge_samples > 0 && c->learned_evals++ % c->cfg.judge_every == 0) {
    double rel = 0.0;
    rc = judge(c, n, d_pos, d_mass, d_acc, st, rel);
    if (rc) return rc;
    c->stats.judge_rel_l2 = rel;
    if (rel > c->cfg.judge_budget) {  // the judge rejects the reduced orders: fixed p
      OrderOpts fx;
      rc = pass(c, n, d_pos, d_mass, d_acc, d_pot, st, fx, false);
      if (rc) return rc;
      c->stats.order_fallbacks = 1;
    }
  }
  // the RMS force the next evaluation budgets with
  return order_force_rms(d_acc, n, c->cfg.dim, c->cfg.G, c->eb.frms.ptr + 1, c->eb.frms.ptr, st, c->ws.launches);
}

static int finish(fmm_ctx *c, cudaStream_t st) {
  CUDA_TRY(cudaStreamSynchronize(st));
  unsigned int herr = 0;
  CUDA_TRY(cudaMemcpy(&herr, c->ws.dev_err, sizeof(herr), cudaMemcpyDeviceToHost));
  if (c->timing_pending) {
    unsigned long long cnt[6] = {0, 0, 0, 0, 0, 0};
    CUDA_TRY(cudaMemcpy(cnt, c->ws.counters, sizeof(cnt), cudaMemcpyDeviceToHost));
    c->stats.m2l_pairs = (int64_t)cnt[0];
    c->stats.p2p_pairs = (int64_t)(cnt[1] + cnt[3]);
    c->stats.far_direct_pairs = (int64_t)cnt[3];
    c->stats.m2l_tiles = (int64_t)cnt[2];
    c->stats.m2l_width_sum = (int64_t)cnt[5];
    float ms[5] = {0, 0, 0, 0, 0};
    for (int i = 0; i < 5; ++i) cudaEventElapsedTime(&ms[i], c->ev[i], c->ev[i + 1]);
    c->stats.ms_tree = ms[0];
    c->stats.ms_upward = ms[1];
    c->stats.ms_m2l = ms[2];
    c->stats.ms_downward = ms[3];
    c->stats.ms_p2p = ms[4];
    float fd = 0.f;
    if (cudaEventElapsedTime(&fd, c->ev[4], c->ev[6]) != cudaSuccess) fd = 0.f;
    c->stats.ms_far_direct = fd;
    float tot = 0;
    cudaEventElapsedTime(&tot, c->ev[0], c->ev[5]);
    c->stats.ms_total = tot;
    c->timing_pending = false;
  }
  if (herr & FMM_DEV_ERR_NONFINITE_INPUT) return FMM_ERR_NONFINITE_INPUT;
  if (herr & FMM_DEV_ERR_NONFINITE_OUTPUT) return FMM_ERR_NONFINITE_OUTPUT;
  if (herr & FMM_DEV_ERR_TIMEOUT) return FMM_ERR_TIMEOUT;
  return FMM_OK;
}

int fmm_evaluate_device(fmm_ctx *c, int64_t n, const double *d_pos, const double *d_mass, double *d_acc,
                        double *d_pot, void *stream) {
  if (!c) return FMM_ERR_INVALID_ARGUMENT;
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  c->last_stream = st;
  return evaluate_device(c, n, d_pos, d_mass, d_acc, d_pot, st);
}

int fmm_evaluate_batched(fmm_ctx *c, int32_t nsys, const int64_t *offsets, const double *d_pos, const double *d_mass,
                         double *d_acc, double *d_pot, int32_t workers) {
  if (!c || nsys < 0 || !offsets || workers < 0) return FMM_ERR_INVALID_ARGUMENT;
  if (nsys == 0) return FMM_OK;
  if (offsets[0] != 0) return FMM_ERR_INVALID_ARGUMENT;
  for (int s = 0; s < nsys; ++s)
    if (offsets[s + 1] < offsets[s] || offsets[s + 1] - offsets[s] > (int64_t)INT32_MAX) return FMM_ERR_INVALID_ARGUMENT;
  if (offsets[nsys] > 0 && (!d_pos || !d_mass || !d_acc)) return FMM_ERR_INVALID_ARGUMENT;
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  const int W = std::max(1, std::min<int>(workers > 0 ? std::min(workers, 32) : 8, nsys));
  while ((int)c->workers.size() < W) {
    fmm_config wc = c->cfg;
    wc.order_mode = FMM_ORDER_FIXED;  // a worker's next system is a new one: fixed p
    wc.judge_samples = 0;
    fmm_ctx *w = nullptr;
    int rc = fmm_create(&wc, &w);
    if (rc) return rc;
    c->workers.push_back(w);
  }
  const int dim = c->cfg.dim;
  std::atomic<int> next{0}, err{0};
  std::vector<fmm_stats> st(W);
  auto work = [&](int wi) {
    fmm_ctx *w = c->workers[wi];
    w->cfg.leaf_cap = c->cfg.leaf_cap;  // the parent's settings, as tuned
    w->cfg.direct_max = c->cfg.direct_max;
    memset(&st[wi], 0, sizeof(fmm_stats));
    if (cudaSetDevice(w->cfg.device) != cudaSuccess) {
      err = FMM_ERR_CUDA;
      return;
    }
    while (!err) {
      const int s = next++;
      if (s >= nsys) break;
      const int64_t off = offsets[s], n = offsets[s + 1] - off;
      if (n == 0) continue;
      int rc = evaluate_device(w, n, d_pos + off * dim, d_mass + off, d_acc + off * dim, d_pot ? d_pot + off : nullptr,
                               w->stream);
      if (!rc) rc = finish(w, w->stream);
      if (rc) {
        err = rc;
        break;
      }
      st[wi].n_cells += w->stats.n_cells;
      st[wi].m2l_pairs += w->stats.m2l_pairs;
      st[wi].p2p_pairs += w->stats.p2p_pairs;
      st[wi].far_direct_pairs += w->stats.far_direct_pairs;
      st[wi].n_leaves += w->stats.n_leaves;
    }
  };
  const auto t0 = std::chrono::steady_clock::now();
  std::vector<std::thread> th;
  for (int i = 1; i < W; ++i) th.emplace_back(work, i);
  work(0);
  for (auto &t : th) t.join();
  const double wall = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  memset(&c->stats, 0, sizeof(c->stats));
  for (const auto &x : st) {
    c->stats.n_cells += x.n_cells;
    c->stats.m2l_pairs += x.m2l_pairs;
    c->stats.p2p_pairs += x.p2p_pairs;
    c->stats.far_direct_pairs += x.far_direct_pairs;
    c->stats.n_leaves += x.n_leaves;
  }
  c->stats.ms_total = wall;
  c->timing_pending = false;
  return err.load();
}

int fmm_autotune(fmm_ctx *c, int64_t n, const double *d_pos, const double *d_mass, int32_t flags,
                 fmm_tune_result *result, void *stream) {
  if (!c || n <= 0 || n > (int64_t)INT32_MAX || !d_pos || !d_mass) return FMM_ERR_INVALID_ARGUMENT;
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  const int dim = c->cfg.dim;
  if (!c->d_acc.reserve((size_t)n * dim)) return FMM_ERR_OUT_OF_MEMORY;
  const int K = dim == 3 ? (c->cfg.p + 1) * (c->cfg.p + 1) : 2 * c->cfg.p + 1;
  const double base = (double)K * K / 25.0;
  fmm_tune_result res;
  memset(&res, 0, sizeof(res));
  const fmm_config saved = c->cfg;
  cudaEvent_t e0, e1;
  CUDA_TRY(cudaEventCreate(&e0));
  CUDA_TRY(cudaEventCreate(&e1));
  int rc = FMM_OK;
  double best = 1e300;
  auto threshold = [&](double f) { return (int32_t)std::max(8.0, base * f); };
  auto trial = [&](int lc, int32_t dm, int32_t al, int32_t pc, int32_t mr) {
    if (rc || res.n_candidates >= 16) return;
    const int k = res.n_candidates++;
    c->cfg.leaf_cap = lc;
    c->cfg.direct_max = dm;
    c->cfg.adaptive_leaf = al;
    c->cfg.p2p_chunk = pc;
    c->cfg.m2l_run = mr;
    res.leaf_cap[k] = lc;
    res.direct_max[k] = dm;
    res.adaptive_leaf[k] = al;
    res.p2p_chunk[k] = pc;
    res.m2l_run[k] = mr;
    const bool twice = c->cfg.order_mode == FMM_ORDER_LEARNED;
    c->frms_n = -1;  // learned orders: start the system afresh
    for (int r = 0; r < (twice ? 2 : 1) && !rc; ++r) rc = evaluate_device(c, n, d_pos, d_mass, c->d_acc.ptr, nullptr, st);
    if (!rc) rc = finish(c, st);
    if (!rc && cudaEventRecord(e0, st) != cudaSuccess) rc = FMM_ERR_CUDA;
    if (!rc) rc = evaluate_device(c, n, d_pos, d_mass, c->d_acc.ptr, nullptr, st);
    if (!rc && cudaEventRecord(e1, st) != cudaSuccess) rc = FMM_ERR_CUDA;
    if (!rc) rc = finish(c, st);
    float ms = 0.f;
    if (!rc && cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) rc = FMM_ERR_CUDA;
    if (rc) return;
    res.ms[k] = ms;
    if (ms < best) {
      best = ms;
      res.best = k;
    }
  };
  // coordinate search: the leaf capacity at the default threshold, then the
  // threshold at the best capacity
  const int32_t al0 = saved.adaptive_leaf, pc0 = saved.p2p_chunk, mr0 = saved.m2l_run;
  if (flags & FMM_TUNE_LEAF) {
    for (int lc : {32, 64, 128, 256}) trial(lc, threshold(1.0), al0, pc0, mr0);
    const int lc = res.leaf_cap[res.best];
    for (double f : {0.25, 0.5, 2.0}) trial(lc, threshold(f), al0, pc0, mr0);
  } else {
    for (double f : {0.125, 0.25, 0.5, 1.0, 2.0}) trial(saved.leaf_cap, threshold(f), al0, pc0, mr0);
  }
  // then the adaptive-target threshold at the best leaf capacity and
  // direct-pair threshold, and the direct-pair threshold once more, a factor
  // sqrt(2) either side of the best: the adaptive targets move the balance
  // between direct pairs and M2L
  if ((flags & FMM_TUNE_ADAPTIVE) && !rc) {
    int b = res.best;
    for (int32_t al : {0, 16, 32, 64})
      if (al != al0) trial(res.leaf_cap[b], res.direct_max[b], al, pc0, mr0);
    b = res.best;
    const double dm = (double)res.direct_max[b];
    for (double f : {0.70710678118654752, 1.41421356237309505})
      trial(res.leaf_cap[b], (int32_t)std::max(8.0, dm * f), res.adaptive_leaf[b], pc0, mr0);
  }
  // then the kernel shapes: the colleague-sum chunk (adaptive targets) and
  // the tensor-core M2L work-item length (the batch shape)
  if ((flags & FMM_TUNE_KERNELS) && !rc) {
    int b = res.best;
    if (res.adaptive_leaf[b] > 0 && c->cfg.dim == 3)
      for (int32_t pc : {128, 512}) trial(res.leaf_cap[b], res.direct_max[b], res.adaptive_leaf[b], pc, mr0);
    b = res.best;
    if (c->cfg.m2l_mode == FMM_M2L_TC)
      for (int32_t mr : {24, 189})
        trial(res.leaf_cap[b], res.direct_max[b], res.adaptive_leaf[b], res.p2p_chunk[b], mr);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->cfg = saved;
  if (rc) return rc;
  c->cfg.leaf_cap = res.leaf_cap[res.best];
  c->cfg.direct_max = res.direct_max[res.best];
  c->cfg.adaptive_leaf = res.adaptive_leaf[res.best];
  c->cfg.p2p_chunk = res.p2p_chunk[res.best];
  c->cfg.m2l_run = res.m2l_run[res.best];
  c->frms_n = -1;
  if (result) *result = res;
  return FMM_OK;
}

// Waits for the context's own stream and the stream of the last
// fmm_evaluate_device call, not for the whole device: other work of the host
// process (other libraries' streams) is not waited for.
int fmm_synchronize(fmm_ctx *c) {
  if (!c) return FMM_ERR_INVALID_ARGUMENT;
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  if (c->last_stream && c->last_stream != c->stream) CUDA_TRY(cudaStreamSynchronize(c->last_stream));
  return finish(c, c->stream);
}

static int upload(fmm_ctx *c, int64_t n, const double *pos, const double *mass) {
  const int dim = c->cfg.dim;
  if (!c->d_pos.reserve((size_t)n * dim) || !c->d_mass.reserve((size_t)n) || !c->d_acc.reserve((size_t)n * dim) ||
      !c->d_pot.reserve((size_t)n))
    return FMM_ERR_OUT_OF_MEMORY;
  CUDA_TRY(cudaMemcpyAsync(c->d_pos.ptr, pos, sizeof(double) * n * dim, cudaMemcpyHostToDevice, c->stream));
  if (mass) CUDA_TRY(cudaMemcpyAsync(c->d_mass.ptr, mass, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
  return FMM_OK;
}

int fmm_evaluate(fmm_ctx *c, int64_t n, const double *pos, const double *mass, double *acc, double *pot) {
  if (!c || n < 0 || (n > 0 && (!pos || !mass || !acc))) return FMM_ERR_INVALID_ARGUMENT;
  if (n == 0) return FMM_OK;
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  int rc = upload(c, n, pos, mass);
  if (rc) return rc;
  rc = evaluate_device(c, n, c->d_pos.ptr, c->d_mass.ptr, c->d_acc.ptr, pot ? c->d_pot.ptr : nullptr, c->stream);
  if (rc) return rc;
  const int dim = c->cfg.dim;
  CUDA_TRY(cudaMemcpyAsync(acc, c->d_acc.ptr, sizeof(double) * n * dim, cudaMemcpyDeviceToHost, c->stream));
  if (pot) CUDA_TRY(cudaMemcpyAsync(pot, c->d_pot.ptr, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
  return finish(c, c->stream);
}

int fmm_direct_device(fmm_ctx *c, int64_t n, const double *d_pos, const double *d_mass, int64_t ntargets,
                      const int64_t *d_targets, int32_t soft_mode, double *d_acc, double *d_pot, void *stream) {
  if (!c || n < 0 || ntargets < 0) return FMM_ERR_INVALID_ARGUMENT;
  if (soft_mode != FMM_SOFT_PLUMMER && soft_mode != FMM_SOFT_NAIVE_REF) return FMM_ERR_INVALID_ARGUMENT;
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  return direct_sum(d_pos, d_mass, n, d_targets, ntargets, c->cfg.dim, c->cfg.eps2, soft_mode, c->cfg.G, d_acc, d_pot,
                    st, c->ws.launches);
}

int fmm_direct(fmm_ctx *c, int64_t n, const double *pos, const double *mass, int64_t ntargets,
               const int64_t *targets, int32_t soft_mode, double *acc, double *pot) {
  if (!c || n < 0 || (n > 0 && (!pos || !mass || !acc))) return FMM_ERR_INVALID_ARGUMENT;
  if (n == 0) return FMM_OK;
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  const int dim = c->cfg.dim;
  int64_t nt = targets ? ntargets : n;
  for (int64_t i = 0; targets && i < nt; ++i)
    if (targets[i] < 0 || targets[i] >= n) return FMM_ERR_INVALID_ARGUMENT;
  int rc = upload(c, n, pos, mass);
  if (rc) return rc;
  if (!c->d_acc.reserve((size_t)nt * dim) || !c->d_pot.reserve((size_t)nt)) return FMM_ERR_OUT_OF_MEMORY;
  const int64_t *dt = nullptr;
  if (targets) {
    if (!c->d_targets.reserve((size_t)nt)) return FMM_ERR_OUT_OF_MEMORY;
    CUDA_TRY(cudaMemcpyAsync(c->d_targets.ptr, targets, sizeof(int64_t) * nt, cudaMemcpyHostToDevice, c->stream));
    dt = c->d_targets.ptr;
  }
  rc = direct_sum(c->d_pos.ptr, c->d_mass.ptr, n, dt, nt, dim, c->cfg.eps2, soft_mode, c->cfg.G, c->d_acc.ptr,
                  pot ? c->d_pot.ptr : nullptr, c->stream, c->ws.launches);
  if (rc) return rc;
  CUDA_TRY(cudaMemcpyAsync(acc, c->d_acc.ptr, sizeof(double) * nt * dim, cudaMemcpyDeviceToHost, c->stream));
  if (pot) CUDA_TRY(cudaMemcpyAsync(pot, c->d_pot.ptr, sizeof(double) * nt, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return FMM_OK;
}

// The integrator loop, optionally with a device frame of the state before
// every `every`-th step (the reference's driver: main.cpp:85-91).
static int integrate(fmm_ctx *c, int32_t method, double dt, int32_t steps, int64_t n, double *pos, double *vel,
                     const double *mass, double *acc_out, fmm_frames *frames, int32_t every, int32_t step0,
                     double t0) {
  if (!c || n < 0 || steps < 0 || (n > 0 && (!pos || !vel || !mass))) return FMM_ERR_INVALID_ARGUMENT;
  if (method != FMM_INT_SYMPLECTIC_EULER && method != FMM_INT_RK4) return FMM_ERR_INVALID_ARGUMENT;
  if (frames && (every < 1 || step0 < 0)) return FMM_ERR_INVALID_ARGUMENT;
  if (n == 0 || steps == 0) return FMM_OK;
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  const int dim = c->cfg.dim;
  const int64_t nd = n * dim;
  int rc = upload(c, n, pos, mass);
  if (rc) return rc;
  if (!c->d_vel.reserve(nd)) return FMM_ERR_OUT_OF_MEMORY;
  CUDA_TRY(cudaMemcpyAsync(c->d_vel.ptr, vel, sizeof(double) * nd, cudaMemcpyHostToDevice, c->stream));
  double *x = c->d_pos.ptr, *v = c->d_vel.ptr, *a = c->d_acc.ptr;
  cudaStream_t st = c->stream;
  for (int s = 0; s < steps; ++s) {
    if (frames && s % every == 0) {  // no acceleration before the first step: zeros
      rc = fmm_frames_write_device(frames, n, x, v, s ? a : nullptr, c->d_mass.ptr, step0 + s, t0 + s * dt, st);
      if (rc) return rc;
    }
    if (method == FMM_INT_SYMPLECTIC_EULER) {
      rc = evaluate_device(c, n, x, c->d_mass.ptr, a, nullptr, st);
      if (rc) return rc;
      se_update(x, v, a, nd, dt, st, c->ws.launches);
    } else {
      if (!c->d_xs.reserve(nd) || !c->d_vs.reserve(nd) || !c->d_asum.reserve(nd) || !c->d_vsum.reserve(nd))
        return FMM_ERR_OUT_OF_MEMORY;
      double *xs = c->d_xs.ptr, *vs = c->d_vs.ptr;
      rc = evaluate_device(c, n, x, c->d_mass.ptr, a, nullptr, st);
      if (rc) return rc;
      rk4_stage(x, v, a, xs, vs, c->d_asum.ptr, c->d_vsum.ptr, nd, 0.5 * dt, 1.0, 1, st, c->ws.launches);
      rc = evaluate_device(c, n, xs, c->d_mass.ptr, a, nullptr, st);
      if (rc) return rc;
      rk4_stage(x, v, a, xs, vs, c->d_asum.ptr, c->d_vsum.ptr, nd, 0.5 * dt, 2.0, 0, st, c->ws.launches);
      rc = evaluate_device(c, n, xs, c->d_mass.ptr, a, nullptr, st);
      if (rc) return rc;
      rk4_stage(x, v, a, xs, vs, c->d_asum.ptr, c->d_vsum.ptr, nd, dt, 2.0, 0, st, c->ws.launches);
      rc = evaluate_device(c, n, xs, c->d_mass.ptr, a, nullptr, st);
      if (rc) return rc;
      rk4_final(x, v, a, vs, c->d_asum.ptr, c->d_vsum.ptr, nd, dt, st, c->ws.launches);
    }
    rc = finish(c, st);
    if (rc) return rc;
  }
  CUDA_TRY(cudaMemcpyAsync(pos, x, sizeof(double) * nd, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaMemcpyAsync(vel, v, sizeof(double) * nd, cudaMemcpyDeviceToHost, st));
  if (acc_out) CUDA_TRY(cudaMemcpyAsync(acc_out, a, sizeof(double) * nd, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  return frames ? fmm_frames_flush(frames) : FMM_OK;
}

int fmm_integrate(fmm_ctx *c, int32_t method, double dt, int32_t steps, int64_t n, double *pos, double *vel,
                  const double *mass, double *acc_out) {
  return integrate(c, method, dt, steps, n, pos, vel, mass, acc_out, nullptr, 1, 0, 0.0);
}

int fmm_integrate_frames(fmm_ctx *c, int32_t method, double dt, int32_t steps, int64_t n, double *pos, double *vel,
                         const double *mass, double *acc_out, fmm_frames *frames, int32_t every, int32_t step0,
                         double t0) {
  if (!frames) return FMM_ERR_INVALID_ARGUMENT;
  return integrate(c, method, dt, steps, n, pos, vel, mass, acc_out, frames, every, step0, t0);
}

// ------------------------------------------------------------ tree export
int fmm_tree_build(fmm_ctx *c, int64_t n, const double *pos) {
  if (!c || n <= 0 || n > (int64_t)INT32_MAX || !pos) return FMM_ERR_INVALID_ARGUMENT;
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  std::vector<double> ones((size_t)n, 1.0);
  int rc = upload(c, n, pos, ones.data());
  if (rc) return rc;
  rc = build_tree(c->ws, c->tree, c->d_pos.ptr, c->d_mass.ptr, n, c->cfg.dim, c->cfg.leaf_cap, c->stream);
  if (rc) return rc;
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->have_tree = true;
  return FMM_OK;
}

int fmm_tree_depth(fmm_ctx *c, int32_t *depth) {
  if (!c || !depth || !c->have_tree) return FMM_ERR_INVALID_ARGUMENT;
  *depth = c->tree.depth;
  return FMM_OK;
}

int fmm_tree_level_size(fmm_ctx *c, int32_t level, int64_t *count) {
  if (!c || !count || !c->have_tree || level < 0 || level > c->tree.depth) return FMM_ERR_INVALID_ARGUMENT;
  *count = c->tree.level_count[level];
  return FMM_OK;
}

int fmm_tree_level_keys(fmm_ctx *c, int32_t level, uint64_t *keys) {
  if (!c || !keys || !c->have_tree || level < 0 || level > c->tree.depth) return FMM_ERR_INVALID_ARGUMENT;
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  CUDA_TRY(cudaMemcpy(keys, c->ws.cell_key + c->tree.level_off[level], sizeof(uint64_t) * c->tree.level_count[level],
                      cudaMemcpyDeviceToHost));
  return FMM_OK;
}

int fmm_tree_leaves(fmm_ctx *c, uint64_t *keys, int64_t *start, int64_t *perm) {
  if (!c || !keys || !start || !perm || !c->have_tree) return FMM_ERR_INVALID_ARGUMENT;
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  const int D = c->tree.depth, nl = c->tree.level_count[D];
  CUDA_TRY(cudaMemcpy(keys, c->ws.cell_key + c->tree.level_off[D], sizeof(uint64_t) * nl, cudaMemcpyDeviceToHost));
  std::vector<int> pb(nl);
  CUDA_TRY(cudaMemcpy(pb.data(), c->ws.cell_pbeg + c->tree.level_off[D], sizeof(int) * nl, cudaMemcpyDeviceToHost));
  for (int i = 0; i < nl; ++i) start[i] = pb[i];
  start[nl] = c->tree.n;
  std::vector<uint32_t> pv(c->tree.n);
  CUDA_TRY(cudaMemcpy(pv.data(), c->tree.d_perm, sizeof(uint32_t) * c->tree.n, cudaMemcpyDeviceToHost));
  for (int64_t i = 0; i < c->tree.n; ++i) perm[i] = pv[i];
  return FMM_OK;
}

int fmm_tree_pairs(fmm_ctx *c, int32_t level, int32_t kind, int64_t *count, uint64_t *tkey, uint64_t *skey) {
  if (!c || !count || !c->have_tree || level < 0 || level > c->tree.depth || (kind != 0 && kind != 1))
    return FMM_ERR_INVALID_ARGUMENT;
  // a force pass with adaptive targets keeps colleague rows for its target cells only: the lists need a tree
  // from fmm_tree_build
  if (c->tree.adaptive_leaf > 0) return FMM_ERR_INVALID_ARGUMENT;
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  const TreeState &t = c->tree;
  const int dim = t.dim, nc = 1 << dim, ns = dim == 3 ? 27 : 9;
  const int lo = t.cell0, hi = t.level_off[t.depth] + t.level_count[t.depth];
  const int m = hi - lo;
  std::vector<uint64_t> key(m);
  std::vector<int> par(m), chi((size_t)m * nc), col((size_t)m * ns);
  CUDA_TRY(cudaMemcpy(key.data(), c->ws.cell_key + lo, sizeof(uint64_t) * m, cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemcpy(par.data(), c->ws.cell_parent + lo, sizeof(int) * m, cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemcpy(chi.data(), c->ws.cell_child + (size_t)lo * nc, sizeof(int) * m * nc, cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemcpy(col.data(), c->ws.cell_coll + (size_t)lo * ns, sizeof(int) * m * ns, cudaMemcpyDeviceToHost));
  int64_t k = 0;
  const int b = t.level_off[level] - lo, e = b + t.level_count[level];
  for (int i = b; i < e; ++i) {
    if (kind == 0) {
      for (int s = 0; s < ns; ++s) {
        int q = col[(size_t)i * ns + s];
        if (q < 0 || q - lo == i) continue;
        if (tkey) {
          tkey[k] = key[i];
          skey[k] = key[q - lo];
        }
        ++k;
      }
    } else if (level > 0) {
      int P = par[i] - lo;
      for (int s = 0; s < ns; ++s) {
        int Q = col[(size_t)P * ns + s];
        if (Q < 0) continue;
        for (int ch = 0; ch < nc; ++ch) {
          int q = chi[(size_t)(Q - lo) * nc + ch];
          if (q < 0) continue;
          bool nb = false;
          for (int s2 = 0; s2 < ns; ++s2) nb |= col[(size_t)i * ns + s2] == q;
          if (nb) continue;
          if (tkey) {
            tkey[k] = key[i];
            skey[k] = key[q - lo];
          }
          ++k;
        }
      }
    }
  }
  *count = k;
  return FMM_OK;
}

int fmm_tree_adaptive_flags(fmm_ctx *c, int32_t adaptive_leaf, uint8_t *flags) {
  if (!c || !flags || !c->have_tree || adaptive_leaf < 1) return FMM_ERR_INVALID_ARGUMENT;
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  const int m = c->tree.n_cells;
  DevBuf<uint8_t> f;
  DevBuf<int> l;
  int rc = f.reserve((size_t)m) && l.reserve((size_t)m + 1) ? FMM_OK : FMM_ERR_OUT_OF_MEMORY;
  if (!rc) rc = launch_adaptive_flags(c->ws, c->tree, adaptive_leaf, f.ptr, l.ptr, c->stream);
  if (!rc && cudaMemcpyAsync(flags, f.ptr, (size_t)m, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess) rc = FMM_ERR_CUDA;
  if (!rc && cudaStreamSynchronize(c->stream) != cudaSuccess) rc = FMM_ERR_CUDA;
  c->ws.launches += 1;
  f.release();
  l.release();
  return rc;
}

int fmm_last_stats(fmm_ctx *c, fmm_stats *out) {
  if (!c || !out) return FMM_ERR_INVALID_ARGUMENT;
  *out = c->stats;
  return FMM_OK;
}

int64_t fmm_launch_count(fmm_ctx *c) { return c ? c->ws.launches : -1; }


int fmm_order_set_model(fmm_ctx *c, const float *params, int32_t nparams) {
  if (!c || !params || nparams != FMM_ORDER_NPARAM) return FMM_ERR_INVALID_ARGUMENT;
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  for (int i = 0; i < nparams; ++i)
    if (!std::isfinite(params[i])) return FMM_ERR_INVALID_ARGUMENT;
  if (!c->order_params.reserve(ORD_NPARAM)) return FMM_ERR_OUT_OF_MEMORY;
  CUDA_TRY(cudaMemcpyAsync(c->order_params.ptr, params, sizeof(float) * ORD_NPARAM, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->has_model = true;
  return FMM_OK;
}

int fmm_order_get_model(fmm_ctx *c, float *params, int32_t nparams) {
  if (!c || !params || nparams != FMM_ORDER_NPARAM) return FMM_ERR_INVALID_ARGUMENT;
  if (!c->has_model) return FMM_ERR_INVALID_ARGUMENT;
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  CUDA_TRY(cudaMemcpyAsync(params, c->order_params.ptr, sizeof(float) * ORD_NPARAM, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return FMM_OK;
}

int fmm_order_collect(fmm_ctx *c, int64_t n, const double *d_pos, const double *d_mass, int32_t ntiles,
                      uint64_t seed, float *d_feat, float *d_labels, void *stream) {
  if (!c || n <= 0 || n > (int64_t)INT32_MAX || ntiles <= 0 || ntiles > (1 << 20) || !d_pos || !d_mass || !d_feat ||
      !d_labels)
    return FMM_ERR_INVALID_ARGUMENT;
  if (c->cfg.dim != 3 || c->cfg.m2l_mode != FMM_M2L_TC) return FMM_ERR_UNSUPPORTED;
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  if (!c->col_tiles.reserve((size_t)ntiles * 2) || !c->col_pairs.reserve((size_t)ntiles * 128 * 4) ||
      !c->col_plabels.reserve((size_t)ntiles * 128 * ORD_NQ) || !c->d_acc.reserve((size_t)n * 3))
    return FMM_ERR_OUT_OF_MEMORY;
  CUDA_TRY(cudaMemsetAsync(d_feat, 0, sizeof(float) * (size_t)ntiles * ORD_NF, st));
  CUDA_TRY(cudaMemsetAsync(d_labels, 0, sizeof(float) * (size_t)ntiles * ORD_NQ, st));
  OrderOpts oo;  // fixed order; collection hook on
  oo.ntiles = ntiles;
  oo.seed = seed;
  oo.tiles = c->col_tiles.ptr;
  oo.pairs = c->col_pairs.ptr;
  oo.pair_labels = c->col_plabels.ptr;
  oo.feat = d_feat;
  oo.labels = d_labels;
  int rc = pass(c, n, d_pos, d_mass, c->d_acc.ptr, nullptr, st, oo, true);
  if (rc) return rc;
  return finish(c, st);
}

int fmm_order_train(fmm_ctx *c, const float *d_feat, const float *d_labels, int32_t n, int32_t epochs, int32_t batch,
                    float lr, float *loss_out) {
  if (!c || !d_feat || !d_labels || n <= 0 || epochs <= 0 || batch <= 0 || !(lr > 0.f) || !loss_out)
    return FMM_ERR_INVALID_ARGUMENT;
  if (!c->has_model) return FMM_ERR_INVALID_ARGUMENT;
  CUDA_TRY(cudaSetDevice(c->cfg.device));
  return order_train(d_feat, d_labels, n, epochs, batch, lr, c->order_params.ptr, loss_out, c->stream, c->ws.launches);
}

int fmm_order_forward_grad(const float *d_feat, const float *d_labels, int32_t n, const float *d_params, float *d_pred,
                           float *d_grad, float *d_loss, void *stream) {
  if (!d_feat || !d_labels || n <= 0 || !d_params || !d_grad || !d_loss) return FMM_ERR_INVALID_ARGUMENT;
  int64_t launches = 0;
  cudaStream_t st = (cudaStream_t)stream;
  int rc = order_forward_grad(d_feat, d_labels, n, d_params, d_pred, d_grad, d_loss, st, launches);
  if (rc) return rc;
  CUDA_TRY(cudaStreamSynchronize(st));
  return FMM_OK;
}

}  // extern "C"
