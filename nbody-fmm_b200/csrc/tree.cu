// Tree build on the GPU, bit-exact with Tree::init_tree (tree.cpp:15-91).
//
// The reference rebins every particle into a hash map once per iteration of
// its depth loop (tree.cpp:43-69).  Here each particle's key is computed once
// at the maximum depth D (16 in 3D, 32 in 2D, tree.cpp:38): the reference's
// leaf coordinate at depth d, (unsigned)((x - a) / ((b - a) / 2^d)), equals
// floor(2^d * q) with q = (x - a) / (b - a) in FP64, because dividing by a
// power of two commutes with IEEE rounding; so the key at depth d is the key
// at D shifted right by dim*(D-d).  One radix sort of the D-keys then gives
// the maximum leaf occupancy of any depth as a maximum run length.  The
// reference's leaves with their particles in input order (tree.cpp:62-66)
// are the runs of that order with each run put back in input order (a rank
// count inside the leaf), or for leaves of more than 512 particles a second
// stable sort of the depth-d keys in input order.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "tree.cuh"

namespace fmm {

// ------------------------------------------------------------------ scan
static constexpr int SCAN_BLOCK = 256;
static constexpr int SCAN_ITEMS = 8;
static constexpr int SCAN_TILE = SCAN_BLOCK * SCAN_ITEMS;

__device__ inline uint32_t block_excl_scan(uint32_t v, uint32_t *s_warp, uint32_t &total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < (SCAN_BLOCK / 32) ? s_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < SCAN_BLOCK / 32) s_warp[lane] = w;
  }
  __syncthreads();
  uint32_t base = warp ? s_warp[warp - 1] : 0;
  total = s_warp[SCAN_BLOCK / 32 - 1];
  __syncthreads();
  return base + x - v;
}

__global__ void k_scan_reduce(const uint32_t *in, int64_t n, uint32_t *block_sums) {
  __shared__ uint32_t s_warp[SCAN_BLOCK / 32];
  int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
  uint32_t s = 0;
  for (int i = 0; i < SCAN_ITEMS; ++i) {
    int64_t k = base + (int64_t)i * SCAN_BLOCK + threadIdx.x;
    if (k < n) s += in[k];
  }
  uint32_t total;
  block_excl_scan(s, s_warp, total);
  if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

__global__ void k_scan_blocks(uint32_t *sums, int nb, uint32_t *total_out) {
  __shared__ uint32_t s_warp[SCAN_BLOCK / 32];
  uint32_t carry = 0;
  for (int b0 = 0; b0 < nb; b0 += SCAN_BLOCK) {
    int k = b0 + threadIdx.x;
    uint32_t v = k < nb ? sums[k] : 0, tot;
    uint32_t e = block_excl_scan(v, s_warp, tot);
    if (k < nb) sums[k] = carry + e;
    carry += tot;
  }
  if (threadIdx.x == 0 && total_out) *total_out = carry;
}

__global__ void k_scan_apply(const uint32_t *in, uint32_t *out, int64_t n, const uint32_t *block_offs) {
  __shared__ uint32_t s_warp[SCAN_BLOCK / 32];
  int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
  uint32_t v[SCAN_ITEMS], s = 0;
  for (int i = 0; i < SCAN_ITEMS; ++i) {
    int64_t k = base + i;
    v[i] = k < n ? in[k] : 0;
    s += v[i];
  }
  uint32_t total;
  uint32_t e = block_excl_scan(s, s_warp, total) + block_offs[blockIdx.x];
  for (int i = 0; i < SCAN_ITEMS; ++i) {
    int64_t k = base + i;
    if (k < n) out[k] = e;
    e += v[i];
  }
}

// Exclusive prefix sum of n uint32 (in may alias out); *total_dev = sum.
void exclusive_scan(Workspace &ws, const uint32_t *in, uint32_t *out, int64_t n, uint32_t *total_dev,
                    cudaStream_t st) {
  int nb = (int)std::max<int64_t>(1, (n + SCAN_TILE - 1) / SCAN_TILE);
  uint32_t *sums = ws.scan_tmp(nb);
  // k_scan_reduce uses a strided tile layout and k_scan_apply a blocked one;
  // both cover the same SCAN_TILE elements per block, so the sums agree.
  k_scan_reduce<<<nb, SCAN_BLOCK, 0, st>>>(in, n, sums);
  k_scan_blocks<<<1, SCAN_BLOCK, 0, st>>>(sums, nb, total_dev);
  k_scan_apply<<<nb, SCAN_BLOCK, 0, st>>>(in, out, n, sums);
  ws.launches += 3;
}

// ------------------------------------------------------------ radix sort
static constexpr int RS_BLOCK = 256;
static constexpr int RS_ROUNDS = 8;
static constexpr int RS_TILE = RS_BLOCK * RS_ROUNDS;
// Largest leaf whose order k_leaf_order redoes in place (each particle counts
// the smaller input indices of its leaf); larger leaves take the full sort.
static constexpr int LEAF_ORDER_MAX = 512;

__global__ void k_radix_hist(const uint64_t *keys, int64_t n, int shift, uint32_t *hist, int nb) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  int64_t base = (int64_t)blockIdx.x * RS_TILE;
  for (int r = 0; r < RS_ROUNDS; ++r) {
    int64_t i = base + (int64_t)r * RS_BLOCK + threadIdx.x;
    if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
  }
  __syncthreads();
  hist[(int64_t)threadIdx.x * nb + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter of one tile of RS_TILE items: items are ranked in (round,
// warp, lane) order, which is their input order inside the tile, and placed
// in shared memory in digit order; then consecutive threads write each
// digit's run to its consecutive places in the output (coalesced stores).
__global__ void __launch_bounds__(RS_BLOCK) k_radix_scatter(const uint64_t *kin, const uint32_t *vin, uint64_t *kout,
                                                            uint32_t *vout, int64_t n, int shift, const uint32_t *offs,
                                                            int nb) {
  __shared__ uint64_t s_key[RS_TILE];
  __shared__ uint32_t s_val[RS_TILE];
  __shared__ uint32_t s_goff[256], s_tstart[256], s_run[256], s_warp[RS_BLOCK / 32];
  __shared__ uint32_t s_cnt[RS_BLOCK / 32][256];
  __shared__ uint32_t s_pre[RS_BLOCK / 32][256];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t base = (int64_t)blockIdx.x * RS_TILE;
  const int tile_n = (int)min((int64_t)RS_TILE, n - base);
  s_goff[tid] = offs[(int64_t)tid * nb + blockIdx.x];  // the digit's first place in the output
  s_run[tid] = 0;
  s_tstart[tid] = 0;  // the tile's digit histogram first
  __syncthreads();
  uint64_t key[RS_ROUNDS];
  uint32_t val[RS_ROUNDS], dig[RS_ROUNDS];
#pragma unroll
  for (int r = 0; r < RS_ROUNDS; ++r) {
    const int k = r * RS_BLOCK + tid;
    const bool valid = k < tile_n;
    key[r] = valid ? kin[base + k] : 0ull;
    val[r] = valid ? vin[base + k] : 0u;
    dig[r] = valid ? (uint32_t)((key[r] >> shift) & 255u) : 256u + lane;  // invalid lanes: distinct, unused
    if (valid) atomicAdd(&s_tstart[dig[r]], 1u);
  }
  __syncthreads();
  uint32_t total;
  const uint32_t ex = block_excl_scan(s_tstart[tid], s_warp, total);  // syncs after every thread read its count
  s_tstart[tid] = ex;  // the digit's first place in the tile's digit order
  const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
  for (int r = 0; r < RS_ROUNDS; ++r) {
    for (int w = 0; w < RS_BLOCK / 32; ++w) s_cnt[w][tid] = 0;
    __syncthreads();
    const uint32_t d = dig[r];
    const bool valid = d < 256u;
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const uint32_t rank = __popc(peers & lt);
    if (valid && rank == 0) s_cnt[warp][d] = __popc(peers);
    __syncthreads();
    uint32_t run = 0;
    for (int w = 0; w < RS_BLOCK / 32; ++w) {
      const uint32_t c = s_cnt[w][tid];
      s_pre[w][tid] = run;
      run += c;
    }
    __syncthreads();
    if (valid) {
      const uint32_t lp = s_tstart[d] + s_run[d] + s_pre[warp][d] + rank;
      s_key[lp] = key[r];
      s_val[lp] = val[r];
    }
    __syncthreads();
    s_run[tid] += run;
  }
  __syncthreads();
  for (int k = tid; k < tile_n; k += RS_BLOCK) {
    const uint64_t kk = s_key[k];
    const uint32_t d = (uint32_t)((kk >> shift) & 255u);
    const uint32_t pos = s_goff[d] + ((uint32_t)k - s_tstart[d]);
    kout[pos] = kk;
    vout[pos] = s_val[k];
  }
}

// Sorts (keys, vals) by the low `bits` bits of the key, stably; the result
// ends in (keys, vals) (the buffers are ping-ponged with the alternates).
void radix_sort(Workspace &ws, uint64_t *&keys, uint32_t *&vals, uint64_t *&keys_alt, uint32_t *&vals_alt, int64_t n,
                int bits, cudaStream_t st) {
  if (n <= 1 || bits <= 0) return;
  int nb = (int)((n + RS_TILE - 1) / RS_TILE);
  uint32_t *hist = ws.radix_hist(nb);
  for (int shift = 0; shift < bits; shift += 8) {
    k_radix_hist<<<nb, RS_BLOCK, 0, st>>>(keys, n, shift, hist, nb);
    exclusive_scan(ws, hist, hist, (int64_t)256 * nb, nullptr, st);
    k_radix_scatter<<<nb, RS_BLOCK, 0, st>>>(keys, vals, keys_alt, vals_alt, n, shift, hist, nb);
    ws.launches += 2;
    std::swap(keys, keys_alt);
    std::swap(vals, vals_alt);
  }
}

// ------------------------------------------------------------ tree kernels
__global__ void k_aabb_init(unsigned long long *box) {
  if (threadIdx.x < 3) {
    box[threadIdx.x] = ~0ull;     // min
    box[3 + threadIdx.x] = 0ull;  // max
  }
}

// AABB (tree.cpp:20-30) plus a finiteness check of positions and masses.
__global__ void k_aabb(const double *pos, const double *mass, int64_t n, int dim, unsigned long long *box,
                       unsigned int *err) {
  unsigned long long lo[3] = {~0ull, ~0ull, ~0ull}, hi[3] = {0, 0, 0};
  bool bad = false;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    for (int d = 0; d < dim; ++d) {
      double x = pos[i * dim + d];
      bad |= !isfinite(x);
      unsigned long long u = dbl_to_ordered(x);
      lo[d] = u < lo[d] ? u : lo[d];
      hi[d] = u > hi[d] ? u : hi[d];
    }
    bad |= !isfinite(mass[i]);
  }
  for (int d = 0; d < dim; ++d) {
    for (int o = 16; o; o >>= 1) {
      unsigned long long a = __shfl_xor_sync(0xffffffffu, lo[d], o), b = __shfl_xor_sync(0xffffffffu, hi[d], o);
      lo[d] = a < lo[d] ? a : lo[d];
      hi[d] = b > hi[d] ? b : hi[d];
    }
    if ((threadIdx.x & 31) == 0) {
      atomicMin(&box[d], lo[d]);
      atomicMax(&box[3 + d], hi[d]);
    }
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(err, FMM_DEV_ERR_NONFINITE_INPUT);
}

__global__ void k_box_decode(const unsigned long long *box, double *geom, int dim) {
  if (threadIdx.x == 0) {
    for (int d = 0; d < 3; ++d) {
      geom[d] = d < dim ? ordered_to_dbl(box[d]) : 0.0;
      geom[3 + d] = d < dim ? ordered_to_dbl(box[3 + d]) : 0.0;
    }
  }
}

// Key of each particle at the maximum depth Dmax; values = input index.
__global__ void k_keys(const double *pos, int64_t n, int dim, int Dmax, const double *geom, uint64_t *keys,
                       uint32_t *vals) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t c[3] = {0, 0, 0};
  const uint64_t cmax = (Dmax >= 32) ? 0xffffffffull : ((1ull << Dmax) - 1);
  const double scale = ldexp(1.0, Dmax);
  for (int d = 0; d < dim; ++d) {
    double a = geom[d], b = geom[3 + d];
    if (b == a) continue;  // zero extent: the reference's 0/0 -> coordinate 0
    double q = (pos[i * dim + d] - a) / (b - a);
    uint64_t v = (uint64_t)(q * scale);
    c[d] = (uint32_t)(v > cmax ? cmax : v);
  }
  keys[i] = morton_encode(dim, c[0], c[1], c[2]);
  vals[i] = (uint32_t)i;
}

// Leaf key at depth D of each particle, in input order.
__global__ void k_leafkeys_input(const double *pos, int64_t n, int dim, int Dmax, int D, const double *geom,
                                 uint64_t *lk, uint32_t *vals) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t c[3] = {0, 0, 0};
  const uint64_t cmax = (Dmax >= 32) ? 0xffffffffull : ((1ull << Dmax) - 1);
  const double scale = ldexp(1.0, Dmax);
  for (int d = 0; d < dim; ++d) {
    double a = geom[d], b = geom[3 + d];
    if (b == a) continue;
    double q = (pos[i * dim + d] - a) / (b - a);
    uint64_t v = (uint64_t)(q * scale);
    c[d] = (uint32_t)(v > cmax ? cmax : v) >> (Dmax - D);
  }
  lk[i] = morton_encode(dim, c[0], c[1], c[2]);
  vals[i] = (uint32_t)i;
}

__global__ void k_run_flags(const uint64_t *keys, int64_t n, int shift, uint32_t *flags) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint64_t k = shift >= 64 ? 0 : keys[i] >> shift;
  uint64_t kp = (i == 0 || shift >= 64) ? 0 : keys[i - 1] >> shift;
  flags[i] = (i == 0 || k != kp) ? 1u : 0u;
}

__global__ void k_run_starts(const uint32_t *flags, const uint32_t *idx, int64_t n, uint32_t *starts) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (flags[i]) starts[idx[i]] = (uint32_t)i;
}

__global__ void k_run_max(const uint32_t *starts, const uint32_t *nruns, int64_t n, uint32_t *maxlen) {
  uint32_t nr = *nruns;
  uint32_t m = 0;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nr; j += (int64_t)gridDim.x * blockDim.x) {
    uint32_t e = (j + 1 < nr) ? starts[j + 1] : (uint32_t)n;
    uint32_t l = e - starts[j];
    m = l > m ? l : m;
  }
  for (int o = 16; o; o >>= 1) {
    uint32_t y = __shfl_xor_sync(0xffffffffu, m, o);
    m = y > m ? y : m;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(maxlen, m);
}

// The final particle order from the Dmax order.  A leaf is a run of equal
// depth-D keys (the Dmax key shifted right by `shift`); inside it the final
// order is the input order, i.e. the particles sorted by their input index
// (vals), so each particle's place is its rank among its leaf's indices.
// Runs come from the depth loop's last pass: exclusive scan idx of the run
// flags, run starts, nruns runs.  The result equals the stable sort of the
// depth-D keys from input order.
__global__ void k_leaf_order(const uint64_t *keys, const uint32_t *vals, const uint32_t *flags, const uint32_t *idx,
                             const uint32_t *starts, uint32_t nruns, int64_t n, int shift, uint64_t *lk,
                             uint32_t *pv) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t L = idx[i] + flags[i] - 1u;  // this particle's run
  const int64_t s = starts[L], e = L + 1u < nruns ? (int64_t)starts[L + 1u] : n;
  const uint32_t v = vals[i];
  int64_t r = 0;
  for (int64_t j = s; j < e; ++j) r += vals[j] < v ? 1 : 0;
  pv[s + r] = v;
  lk[s + r] = shift >= 64 ? 0ull : keys[i] >> shift;
}

// Leaves: one per run of equal leaf keys in the sorted order.
__global__ void k_make_leaves(const uint64_t *lk_sorted, const uint32_t *flags, const uint32_t *idx, int64_t n,
                              int leaf_base, uint64_t *cell_key, int *cell_pbeg, int *cell_pend, int *leaf_of) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int li = (int)idx[i] - (flags[i] ? 0 : 1);
  leaf_of[i] = leaf_base + li;
  if (flags[i]) {
    cell_key[leaf_base + li] = lk_sorted[i];
    cell_pbeg[leaf_base + li] = (int)i;
  }
  if (i == n - 1 || flags[i + 1]) cell_pend[leaf_base + li] = (int)(i + 1);
}

__global__ void k_parent_flags(const uint64_t *ckey, int cbase, int nchild, int dim, uint32_t *flags) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nchild) return;
  flags[j] = (j == 0 || (ckey[cbase + j] >> dim) != (ckey[cbase + j - 1] >> dim)) ? 1u : 0u;
}

__global__ void k_make_parents(uint64_t *ckey, int *cpbeg, int *cpend, int *cparent, int *cchild, int cbase,
                               int nchild, int pbase, int dim, const uint32_t *flags, const uint32_t *idx) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nchild) return;
  const int nc = 1 << dim;
  int pi = pbase + (int)idx[j] - (flags[j] ? 0 : 1);
  uint64_t k = ckey[cbase + j];
  cparent[cbase + j] = pi;
  cchild[(int64_t)pi * nc + (int)(k & (nc - 1))] = cbase + j;
  if (flags[j]) {
    ckey[pi] = k >> dim;
    cpbeg[pi] = cpbeg[cbase + j];
  }
  if (j == nchild - 1 || flags[j + 1]) cpend[pi] = cpend[cbase + j];
}

// Adaptive targets, per cell g (flag[g - cell0]): bit 0, a target: the root,
// or a cell whose parent holds more than A particles (every ancestor then
// does too, since a cell's particles are a subset of its parent's); bit 1,
// an adaptive leaf: a target with at most A particles, or a leaf.  The
// adaptive leaves are appended to alist, their count kept in *acount.
__global__ void k_adaptive_flags(const int *pbeg, const int *pend, const int *parent, int cell0, int ncell,
                                 int first1, int leaf_first, int A, uint8_t *flag, int *alist, unsigned *acount) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, lane = threadIdx.x & 31;
  const int g = cell0 + i;
  bool is_leaf = false;
  if (i < ncell) {
    const bool tgt = g < first1 || pend[parent[g]] - pbeg[parent[g]] > A;
    is_leaf = tgt && (pend[g] - pbeg[g] <= A || g >= leaf_first);
    flag[i] = (uint8_t)((tgt ? 1 : 0) | (is_leaf ? 2 : 0));
  }
  const unsigned m = __ballot_sync(0xffffffffu, is_leaf);
  unsigned base = 0;
  if (lane == 0 && m) base = atomicAdd(acount, (unsigned)__popc(m));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (is_leaf) alist[base + __popc(m & ((1u << lane) - 1u))] = g;
}

// Colleagues (|delta| <= 1 on every axis, same level, self included) of the
// cells of one level.  With c = 2P + b per axis (b the cell's child bit),
// the neighbour at offset delta is child ((b + delta) mod 2) of the parent's
// colleague at offset floor((b + delta) / 2), so each of the 3^dim slots is
// two dependent loads and no key decoding.
//
// With adaptive targets (aflag set) only target cells get a row: nothing
// reads the row of a cell that is no target (their parents' rows serve the
// targets, and a target's parent is a target).
__global__ void k_colleagues(const uint64_t *ckey, const int *cparent, const int *cchild, int *ccoll, int base,
                             int count, int dim, const uint8_t *aflag, int cell0) {
  // blocks of 8 cells x ns slots, one thread per (cell, slot): consecutive
  // threads write consecutive slots
  const int nc = 1 << dim, ns = dim == 3 ? 27 : 9;
  const int ci = blockIdx.x * 8 + (int)threadIdx.x / ns, s = (int)threadIdx.x % ns;
  if (ci >= count) return;
  const int c = base + ci;
  if (aflag && !(aflag[c - cell0] & 1)) return;
  const int b = (int)(ckey[c] & (uint64_t)(nc - 1));
  int pslot = 0, child = 0, mul = 1;
  for (int a = 0; a < dim; ++a) {
    const int delta = (s / mul) % 3 - 1;
    const int v = ((b >> a) & 1) + delta;  // in [-1, 2]
    const int f = (v + 2) / 2 - 1;        // floor(v / 2)
    pslot += (f + 1) * mul;
    child |= (v - 2 * f) << a;
    mul *= 3;
  }
  const int Q = ccoll[(int64_t)cparent[c] * ns + pslot];
  ccoll[(int64_t)c * ns + s] = Q >= 0 ? cchild[(int64_t)Q * nc + child] : -1;
}

// The same rows with adaptive targets, one thread per cell: most cells of the
// deep levels are no target and leave after one flag load, instead of 3^dim
// threads each; a target's thread writes its 3^dim slots.
template <int DIM>
__global__ void k_colleagues_targets(const uint64_t *ckey, const int *cparent, const int *cchild, int *ccoll,
                                     int base, int count, const uint8_t *aflag, int cell0) {
  constexpr int NC = 1 << DIM, NS = DIM == 3 ? 27 : 9;
  const int ci = blockIdx.x * blockDim.x + threadIdx.x;
  if (ci >= count) return;
  const int c = base + ci;
  if (!(aflag[c - cell0] & 1)) return;
  const int b = (int)(ckey[c] & (uint64_t)(NC - 1));
  const int *prow = ccoll + (int64_t)cparent[c] * NS;
  int *row = ccoll + (int64_t)c * NS;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    int pslot = 0, child = 0, mul = 1;
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      const int delta = (s / mul) % 3 - 1;
      const int v = ((b >> a) & 1) + delta;  // in [-1, 2]
      const int f = (v + 2) / 2 - 1;        // floor(v / 2)
      pslot += (f + 1) * mul;
      child |= (v - 2 * f) << a;
      mul *= 3;
    }
    const int Q = prow[pslot];
    row[s] = Q >= 0 ? cchild[(int64_t)Q * NC + child] : -1;
  }
}

__global__ void k_root_colleague(int *ccoll, int root, int dim) {
  if (threadIdx.x == 0) {
    int ns = dim == 3 ? 27 : 9;
    for (int s = 0; s < ns; ++s) ccoll[(int64_t)root * ns + s] = -1;
    ccoll[(int64_t)root * ns + ns / 2] = root;
  }
}

__global__ void k_fill_i32(int *p, int64_t n, int v) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

// Gathers particles into leaf order: the offset from the leaf's geometric
// centre split into FP32 hi + lo parts (x - c = hi + lo to ~48 bits), and the
// FP32 mass, used by P2M, L2P (hi only) and P2P (hi and lo).
__global__ void k_gather_particles(const double *pos, const double *mass, const uint32_t *perm, const int *leaf_of,
                                   const uint64_t *ckey, int64_t n, int dim, int depth, const double *geom,
                                   float4 *part, float4 *part_lo) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t j = perm[i];
  uint32_t q[3];
  morton_decode(dim, ckey[leaf_of[i]], q[0], q[1], q[2]);
  float r[3] = {0.f, 0.f, 0.f}, rl[3] = {0.f, 0.f, 0.f};
  const double inv = ldexp(1.0, -depth);
  for (int d = 0; d < dim; ++d) {
    double ext = geom[3 + d] - geom[d];
    double c = geom[d] + ((double)q[d] + 0.5) * (ext * inv);
    double v = pos[(int64_t)j * dim + d] - c;
    r[d] = (float)v;
    rl[d] = (float)(v - (double)r[d]);
  }
  part[i] = make_float4(r[0], r[1], r[2], (float)mass[j]);
  part_lo[i] = make_float4(rl[0], rl[1], rl[2], 0.f);
}

// ------------------------------------------------------------ host driver
static int bit_width_u64(uint64_t v) {
  int w = 0;
  while (v) {
    ++w;
    v >>= 1;
  }
  return w;
}

int launch_adaptive_flags(const Workspace &ws, const TreeState &t, int A, uint8_t *flag, int *list, cudaStream_t st) {
  if (t.depth < 1 || t.n_cells <= 0) return FMM_ERR_INVALID_ARGUMENT;
  CUDA_TRY(cudaMemsetAsync(list + t.n_cells, 0, sizeof(int), st));
  k_adaptive_flags<<<cdiv(t.n_cells, 256), 256, 0, st>>>(ws.cell_pbeg, ws.cell_pend, ws.cell_parent, t.cell0,
                                                          t.n_cells, t.level_off[1], t.level_off[t.depth], A, flag,
                                                          list, (unsigned *)(list + t.n_cells));
  CUDA_TRY(cudaGetLastError());
  return FMM_OK;
}

int build_tree(Workspace &ws, TreeState &t, const double *d_pos, const double *d_mass, int64_t n, int dim,
               int threshold, cudaStream_t st, int adaptive_leaf) {
  t.dim = dim;
  t.n = n;
  t.adaptive_leaf = 0;
  const int Dmax = ((64 / dim) >> dim) << dim;  // tree.cpp:38
  const int TPB = 256;
  const int nbN = cdiv(n, TPB);
  ws.reserve_particles(n);
  CUDA_TRY(cudaMemsetAsync(ws.dev_err, 0, sizeof(unsigned int), st));
  // AABB
  k_aabb_init<<<1, 32, 0, st>>>(ws.box_u64);
  k_aabb<<<std::min(nbN, 148 * 8), TPB, 0, st>>>(d_pos, d_mass, n, dim, ws.box_u64, ws.dev_err);
  k_box_decode<<<1, 32, 0, st>>>(ws.box_u64, ws.geom, dim);
  k_keys<<<nbN, TPB, 0, st>>>(d_pos, n, dim, Dmax, ws.geom, ws.keyA, ws.valA);
  ws.launches += 4;
  CUDA_TRY(cudaMemcpyAsync(t.lo, ws.geom, 6 * sizeof(double), cudaMemcpyDeviceToHost, st));
  unsigned int herr = 0;
  CUDA_TRY(cudaMemcpyAsync(&herr, ws.dev_err, sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  if (herr & FMM_DEV_ERR_NONFINITE_INPUT) return FMM_ERR_NONFINITE_INPUT;
  for (int d = 0; d < 3; ++d) t.hi[d] = t.lo[3 + d];

  // sort all particles by their Dmax key
  uint64_t *kA = ws.keyA, *kB = ws.keyB;
  uint32_t *vA = ws.valA, *vB = ws.valB;
  radix_sort(ws, kA, vA, kB, vB, n, dim * Dmax, st);

  // depth loop, tree.cpp:43-69
  unsigned int max_n = (unsigned int)n;
  unsigned int depth = 0, nruns = 0;
  uint32_t *flags = ws.u32A, *idx = ws.u32B, *starts = ws.u32C;
  do {
    uint64_t n_leafs = (uint64_t)(max_n - 1) / (unsigned)threshold + 1;
    depth += bit_width_u64(n_leafs) / dim + 1;
    if (depth > (unsigned)Dmax) depth = Dmax;
    int shift = dim * (Dmax - (int)depth);
    k_run_flags<<<nbN, TPB, 0, st>>>(kA, n, shift, flags);
    exclusive_scan(ws, flags, idx, n, ws.scalars, st);
    k_run_starts<<<nbN, TPB, 0, st>>>(flags, idx, n, starts);
    CUDA_TRY(cudaMemsetAsync(ws.scalars + 1, 0, sizeof(uint32_t), st));
    k_run_max<<<std::min(nbN, 148 * 8), TPB, 0, st>>>(starts, ws.scalars, n, ws.scalars + 1);
    ws.launches += 3;
    uint32_t h[2];
    CUDA_TRY(cudaMemcpyAsync(h, ws.scalars, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    max_n = h[1];
    nruns = h[0];
  } while (depth < (unsigned)Dmax && max_n > (unsigned)threshold);
  t.depth = (int)depth;
  const int D = t.depth;

  // final order: stable sort of the depth-D leaf keys, starting from input
  // order, so each leaf keeps its particles in input order (tree.cpp:62-66).
  // The depth-D key is the Dmax key shifted right, so the Dmax order already
  // groups the leaves; with leaves of at most LEAF_ORDER_MAX particles only
  // the order inside each leaf is redone (k_leaf_order), else the leaf keys
  // are sorted afresh from input order.
  uint64_t *lk = ws.keyC, *lkAlt = ws.keyA;
  uint32_t *pv = ws.valC, *pvAlt = ws.valA;
  if (max_n <= (unsigned)LEAF_ORDER_MAX) {
    k_leaf_order<<<nbN, TPB, 0, st>>>(kA, vA, flags, idx, starts, nruns, n, dim * (Dmax - D), lk, pv);
    ws.launches += 1;
  } else {
    k_leafkeys_input<<<nbN, TPB, 0, st>>>(d_pos, n, dim, Dmax, D, ws.geom, ws.keyC, ws.valC);
    ws.launches += 1;
    radix_sort(ws, lk, pv, lkAlt, pvAlt, n, dim * D, st);
  }
  t.d_leafkey_sorted = lk;
  t.d_perm = pv;

  // leaves
  k_run_flags<<<nbN, TPB, 0, st>>>(lk, n, 0, flags);
  exclusive_scan(ws, flags, idx, n, ws.scalars, st);
  ws.launches += 1;
  uint32_t nleaves = 0;
  CUDA_TRY(cudaMemcpyAsync(&nleaves, ws.scalars, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  t.level_count.assign(D + 1, 0);
  t.level_off.assign(D + 2, 0);
  t.level_count[D] = (int)nleaves;
  const int nc = 1 << dim, ns = dim == 3 ? 27 : 9;
  int64_t cap = (int64_t)(D + 1) * nleaves;
  ws.reserve_cells(cap, nc, ns);
  // levels are laid out bottom-up from the end of the cell arrays so that
  // they end up contiguous and ordered from the root: [level 0, ..., level D]
  int base = (int)(cap - nleaves);
  k_make_leaves<<<nbN, TPB, 0, st>>>(lk, flags, idx, n, base, ws.cell_key, ws.cell_pbeg, ws.cell_pend, ws.leaf_of);
  ws.launches += 1;
  std::vector<int> lbase(D + 1);
  lbase[D] = base;
  for (int d = D - 1; d >= 0; --d) {
    int nch = t.level_count[d + 1];
    int cb = lbase[d + 1];
    k_parent_flags<<<cdiv(nch, TPB), TPB, 0, st>>>(ws.cell_key, cb, nch, dim, flags);
    exclusive_scan(ws, flags, idx, nch, ws.scalars, st);
    uint32_t np = 0;
    CUDA_TRY(cudaMemcpyAsync(&np, ws.scalars, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    int pb = cb - (int)np;
    k_fill_i32<<<cdiv((int64_t)np * nc, TPB), TPB, 0, st>>>(ws.cell_child + (int64_t)pb * nc, (int64_t)np * nc, -1);
    k_make_parents<<<cdiv(nch, TPB), TPB, 0, st>>>(ws.cell_key, ws.cell_pbeg, ws.cell_pend, ws.cell_parent,
                                                    ws.cell_child, cb, nch, pb, dim, flags, idx);
    ws.launches += 3;
    t.level_count[d] = (int)np;
    lbase[d] = pb;
  }
  // cell indices stay absolute: level d occupies [lbase[d], lbase[d] + count)
  for (int d = 0; d <= D; ++d) t.level_off[d] = lbase[d];
  t.level_off[D + 1] = (int)cap;
  t.cell0 = lbase[0];
  t.n_cells = (int)(cap - lbase[0]);
  // leaf children are -1
  k_fill_i32<<<cdiv((int64_t)nleaves * nc, TPB), TPB, 0, st>>>(ws.cell_child + (int64_t)lbase[D] * nc,
                                                                (int64_t)nleaves * nc, -1);
  // adaptive targets (3D trees of depth >= 3, as the force pass runs them):
  // the flags now, so that only target cells get colleague rows
  const uint8_t *aflag = nullptr;
  if (adaptive_leaf > 0 && dim == 3 && D >= 3) {
    if (!ws.reserve_adaptive(t.n_cells)) return FMM_ERR_OUT_OF_MEMORY;
    int rc = launch_adaptive_flags(ws, t, adaptive_leaf, ws.aflag, ws.alist, st);
    if (rc) return rc;
    ws.launches += 1;
    t.adaptive_leaf = adaptive_leaf;
    aflag = ws.aflag;
  }
  // colleagues, top-down
  k_root_colleague<<<1, 32, 0, st>>>(ws.cell_coll, lbase[0], dim);
  ws.launches += 2;
  for (int d = 1; d <= D; ++d) {
    if (aflag)  // adaptive targets are 3D only
      k_colleagues_targets<3><<<cdiv(t.level_count[d], TPB), TPB, 0, st>>>(
          ws.cell_key, ws.cell_parent, ws.cell_child, ws.cell_coll, lbase[d], t.level_count[d], aflag, t.cell0);
    else
      k_colleagues<<<cdiv(t.level_count[d], 8), 8 * ns, 0, st>>>(ws.cell_key, ws.cell_parent, ws.cell_child,
                                                                  ws.cell_coll, lbase[d], t.level_count[d], dim,
                                                                  nullptr, t.cell0);
    ws.launches += 1;
  }
  // particles in leaf order
  k_gather_particles<<<nbN, TPB, 0, st>>>(d_pos, d_mass, pv, ws.leaf_of, ws.cell_key, n, dim, D, ws.geom, ws.part,
                                             ws.part_lo);
  ws.launches += 1;
  CUDA_TRY(cudaGetLastError());
  return FMM_OK;
}

}  // namespace fmm
