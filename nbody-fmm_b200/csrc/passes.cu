// The FMM passes after the tree build: P2M, M2M, M2L, L2L, L2P and P2P
// (Tree::compute_accelerations, tree.cpp:93-111; Leaf::compute_acceleration,
// leaf.cpp:55-148).
//
// Translations are dense contractions.  Cells of one level with the same
// child index ("class": the parities of their coordinates) have the same
// set of interaction-list offsets (node_i.cpp:39-43: delta in
// [-2-c%2, 3-c%2] minus the neighbours), so a batch of 64 such target cells
// accumulates, slot by slot, Y[64 x K] += X_slot[64 x K] * T_slot[K x K] where
// X_slot gathers the source expansion of each target at that offset (zero if
// the cell does not exist).  M2M (8 child slots) and L2L (1 parent slot) use
// the same kernel.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

#include "expansions.cuh"
#include "m2l_tc.cuh"

namespace fmm {

// [dim == 3][class] -> list of (table offset index | colleague slot << 9 | child << 14)
__constant__ int c_m2l_slots[2][8][189];
__constant__ float c_rec1[FMM_MAX_P + 1][FMM_MAX_P + 1];  // (2l-1)/(l^2-m^2)
__constant__ float c_rec2[FMM_MAX_P + 1][FMM_MAX_P + 1];  // 1/(l^2-m^2)

void upload_class_tables() {
  // __constant__ memory is per device: upload once for every device used
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
  std::lock_guard<std::mutex> lk(mu);
  if (done[dev]) return;
  done[dev] = true;
  static int h[2][8][189] = {};
  for (int dim = 2; dim <= 3; ++dim)
  for (int c = 0; c < (1 << dim); ++c) {
    int cb[3] = {c & 1, (c >> 1) & 1, (c >> 2) & 1};
    int k = 0;
    int lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
      lo[a] = a < dim ? -2 - cb[a] : 0;
      hi[a] = a < dim ? 3 - cb[a] : 0;
    }
    for (int dz = lo[2]; dz <= hi[2]; ++dz)
      for (int dy = lo[1]; dy <= hi[1]; ++dy)
        for (int dx = lo[0]; dx <= hi[0]; ++dx) {
          if (dx >= -1 && dx <= 1 && dy >= -1 && dy <= 1 && dz >= -1 && dz <= 1) continue;
          int dd[3] = {dx, dy, dz}, del[3], ch[3];
          for (int a = 0; a < 3; ++a) {
            int v = dd[a] + cb[a];         // in [-2, 3]
            del[a] = (v + 2) / 2 - 1;      // floor(v / 2)
            ch[a] = v - 2 * del[a];
          }
          int ti = dim == 3 ? (dx + 3) + 7 * (dy + 3) + 49 * (dz + 3) : (dx + 3) + 7 * (dy + 3);
          int cs = dim == 3 ? (del[0] + 1) + 3 * (del[1] + 1) + 9 * (del[2] + 1) : (del[0] + 1) + 3 * (del[1] + 1);
          int chi = ch[0] + 2 * ch[1] + (dim == 3 ? 4 * ch[2] : 0);
          h[dim - 2][c][k++] = ti | (cs << 9) | (chi << 14);
        }
  }
  cudaMemcpyToSymbol(c_m2l_slots, h, sizeof(h));
  float r1[FMM_MAX_P + 1][FMM_MAX_P + 1] = {}, r2[FMM_MAX_P + 1][FMM_MAX_P + 1] = {};
  for (int l = 0; l <= FMM_MAX_P; ++l)
    for (int m = 0; m < l; ++m) {
      r1[l][m] = (float)((2.0 * l - 1.0) / (double)(l * l - m * m));
      r2[l][m] = (float)(1.0 / (double)(l * l - m * m));
    }
  cudaMemcpyToSymbol(c_rec1, r1, sizeof(r1));
  cudaMemcpyToSymbol(c_rec2, r2, sizeof(r2));
}

// ------------------------------------------------------------ cp.async
__device__ inline void cp_async16(void *smem, const void *gmem, int src_bytes) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ inline void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ inline void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

enum { MODE_M2L = 0, MODE_M2M = 1, MODE_L2L = 2 };
static constexpr int CT_TGT = 64;  // targets per batch
static constexpr int CT_THREADS = 256;

struct ContractArgs {
  const int4 *batches;  // {first (list offset or cell), count, level, class}
  const int *tlist;     // class-grouped target cells, or null (targets first + i)
  const float *X;
  float *Y;
  const float *tab;
  const int *cparent, *cchild, *ccoll, *cpbeg, *cpend;
  long long direct_max;  // M2L skips pairs with n_t * n_s <= direct_max (summed directly instead)
  const uint8_t *fdirect;  // M2L: per offset (dx+3) + 7(dy+3) + 49(dz+3): not well separated, summed directly
  const int *src_tab;    // M2L: [batch][slot][CT_TGT] source cells resolved ahead (or null)
  const int *slot_list;  // M2L: [batch][slot index] present slots, nslots_tab[batch] of them
  const int *nslots_tab;
  int cell0, K, KS, KP, dim, mode, slot_base, level_stride;
  unsigned long long *pair_count;  // M2L: number of (target, source) pairs contracted
};

// Resolves the source cell of target `tgt` for slot s; returns -1 if absent.
__device__ inline int contract_source(const ContractArgs &a, int tgt, int s, int cls, int level, int &tslot) {
  const int nc = 1 << a.dim, ns = a.dim == 3 ? 27 : 9;
  if (a.mode == MODE_M2L) {
    int e = c_m2l_slots[a.dim - 2][cls][s];
    tslot = (e & 511) + level * a.level_stride;
    int P = a.cparent[tgt];
    int Q = a.ccoll[(int64_t)P * ns + ((e >> 9) & 31)];
    if (Q < 0) return -1;
    if (a.fdirect && a.fdirect[e & 511]) return -1;  // not well separated: direct far field
    int src = a.cchild[(int64_t)Q * nc + ((e >> 14) & 7)];
    if (src >= 0 && a.direct_max > 0) {
      long long nt = a.cpend[tgt] - a.cpbeg[tgt], nsrc = a.cpend[src] - a.cpbeg[src];
      if (nt * nsrc <= a.direct_max) return -1;  // evaluated by the direct far field
    }
    return src;
  } else if (a.mode == MODE_M2M) {
    tslot = a.slot_base + s;
    return a.cchild[(int64_t)tgt * nc + s];
  } else {
    tslot = a.slot_base + cls;
    return a.cparent[tgt];
  }
}

template <int J, int NS>
__global__ void __launch_bounds__(CT_THREADS) k_contract(ContractArgs a) {
  extern __shared__ __align__(16) float smem[];
  const int K = a.K, KS = a.KS, KP = a.KP;
  float *Ts = smem;                              // [NS][K][KP]
  float *Xs = Ts + (size_t)NS * K * KP;          // [NS][CT_TGT][KS]
  int *s_src = (int *)(Xs + (size_t)NS * CT_TGT * KS);  // [NS][CT_TGT]
  int *s_tslot = s_src + NS * CT_TGT;            // [NS]
  int *s_any = s_tslot + NS;                     // [NS]
  __shared__ int s_tgt[CT_TGT];

  const int4 b = a.batches[blockIdx.x];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int cnt = b.y, level = b.z, cls = b.w;
  if (tid < CT_TGT) s_tgt[tid] = tid < cnt ? (a.tlist ? a.tlist[b.x + tid] : b.x + tid) : -1;
  __syncthreads();
  const int nslots = a.mode == MODE_M2L ? (a.src_tab ? a.nslots_tab[blockIdx.x] : (a.dim == 3 ? 189 : 27))
                                        : (a.mode == MODE_M2M ? (1 << a.dim) : 1);

  unsigned long long npairs = 0;
  float acc[8][J];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < J; ++j) acc[i][j] = 0.f;

  const bool tabled = a.mode == MODE_M2L && a.src_tab;
  const size_t tab_base = (size_t)blockIdx.x * 189;
  auto prefetch = [&](int s, int buf) {
    int src = -1, ts = 0;
    if (tid < CT_TGT) {
      int tg = s_tgt[tid];
      if (tabled) {
        const int slot = a.slot_list[tab_base + s];
        const int e = c_m2l_slots[a.dim - 2][cls][slot];
        ts = (e & 511) + level * a.level_stride;
        src = a.src_tab[(tab_base + slot) * CT_TGT + tid];
      } else if (tg >= 0) {
        src = contract_source(a, tg, s, cls, level, ts);
      }
      s_src[buf * CT_TGT + tid] = src;
      if (tid == 0 || src >= 0) s_tslot[buf] = ts;  // same for all targets of the batch
    }
    int any = __syncthreads_count(src >= 0);
    if (tid == 0) {
      s_any[buf] = any;
      npairs += any;
    }
    if (any) {
      const float *T = a.tab + (size_t)s_tslot[buf] * K * KP;
      float *Td = Ts + (size_t)buf * K * KP;
      const int nT = K * KP / 4;
      for (int c = tid; c < nT; c += CT_THREADS) cp_async16(Td + 4 * c, T + 4 * c, 16);
      float *Xd = Xs + (size_t)buf * CT_TGT * KS;
      const int cpr = KS / 4;
      for (int c = tid; c < CT_TGT * cpr; c += CT_THREADS) {
        int r = c / cpr, q = c % cpr;
        int sr = s_src[buf * CT_TGT + r];
        const float *g = sr >= 0 ? a.X + (size_t)(sr - a.cell0) * KS + 4 * q : a.X;
        cp_async16(Xd + (size_t)r * KS + 4 * q, g, sr >= 0 ? 16 : 0);
      }
    }
    cp_async_commit();
  };

  if (NS == 2) prefetch(0, 0);
  for (int s = 0; s < nslots; ++s) {
    const int buf = NS == 2 ? (s & 1) : 0;
    if (NS == 1) {
      prefetch(s, 0);
      cp_async_wait<0>();
    } else {
      if (s + 1 < nslots) {
        prefetch(s + 1, (s + 1) & 1);
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
    }
    __syncthreads();
    if (s_any[buf]) {
      const float *Tb = Ts + (size_t)buf * K * KP;
      const float *Xb = Xs + (size_t)buf * CT_TGT * KS + (size_t)(warp * 8) * KS;
#pragma unroll 2
      for (int k = 0; k < K; ++k) {
        float bv[J];
#pragma unroll
        for (int j = 0; j < J; ++j) bv[j] = Tb[(size_t)k * KP + lane + 32 * j];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          float av = Xb[(size_t)i * KS + k];
#pragma unroll
          for (int j = 0; j < J; ++j) acc[i][j] = fmaf(av, bv[j], acc[i][j]);
        }
      }
    }
    __syncthreads();
  }
  if (tid == 0 && a.pair_count && a.mode == MODE_M2L) atomicAdd(a.pair_count, npairs);
  // write out
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    int tg = s_tgt[warp * 8 + i];
    if (tg < 0) continue;
    float *y = a.Y + (size_t)(tg - a.cell0) * KS;
#pragma unroll
    for (int j = 0; j < J; ++j) {
      int o = lane + 32 * j;
      if (o < K) {
        if (a.mode == MODE_M2M) y[o] = acc[i][j];
        else y[o] += acc[i][j];
      }
    }
  }
}

template <int J>
static void launch_contract_j(const ContractArgs &a, int nb, int stages, size_t sh, cudaStream_t st) {
  if (stages == 2) k_contract<J, 2><<<nb, CT_THREADS, sh, st>>>(a);
  else k_contract<J, 1><<<nb, CT_THREADS, sh, st>>>(a);
}

static size_t contract_smem(int K, int KS, int KP, int NS) {
  return sizeof(float) * ((size_t)NS * K * KP + (size_t)NS * CT_TGT * KS) + sizeof(int) * (NS * CT_TGT + 2 * NS) + 16;
}

static int launch_contract(const ContractArgs &a, int nb, cudaStream_t st, int64_t &launches) {
  if (nb <= 0) return FMM_OK;
  int J = (a.K + 31) / 32;
  int stages = contract_smem(a.K, a.KS, a.KP, 2) <= 200 * 1024 ? 2 : 1;
  size_t sh = contract_smem(a.K, a.KS, a.KP, stages);
  if (sh > 227 * 1024) return FMM_ERR_UNSUPPORTED;
  // the shared-memory opt-in is per function and device
  static std::mutex mu;
  static size_t attr_set[64][8][3] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return FMM_ERR_CUDA;
  std::lock_guard<std::mutex> lk(mu);
  auto set_attr = [&](auto kern) { return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh); };
  if (attr_set[dev][J][stages] < sh) {
    cudaError_t e = cudaSuccess;
    switch (J) {
      case 1: e = stages == 2 ? set_attr(k_contract<1, 2>) : set_attr(k_contract<1, 1>); break;
      case 2: e = stages == 2 ? set_attr(k_contract<2, 2>) : set_attr(k_contract<2, 1>); break;
      case 3: e = stages == 2 ? set_attr(k_contract<3, 2>) : set_attr(k_contract<3, 1>); break;
      case 4: e = stages == 2 ? set_attr(k_contract<4, 2>) : set_attr(k_contract<4, 1>); break;
      case 5: e = stages == 2 ? set_attr(k_contract<5, 2>) : set_attr(k_contract<5, 1>); break;
      case 6: e = stages == 2 ? set_attr(k_contract<6, 2>) : set_attr(k_contract<6, 1>); break;
      default: return FMM_ERR_UNSUPPORTED;
    }
    if (e != cudaSuccess) return FMM_ERR_CUDA;
    attr_set[dev][J][stages] = sh;
  }
  switch (J) {
    case 1: launch_contract_j<1>(a, nb, stages, sh, st); break;
    case 2: launch_contract_j<2>(a, nb, stages, sh, st); break;
    case 3: launch_contract_j<3>(a, nb, stages, sh, st); break;
    case 4: launch_contract_j<4>(a, nb, stages, sh, st); break;
    case 5: launch_contract_j<5>(a, nb, stages, sh, st); break;
    case 6: launch_contract_j<6>(a, nb, stages, sh, st); break;
    default: return FMM_ERR_UNSUPPORTED;
  }
  launches += 1;
  return FMM_OK;
}

// Resolves the source cell of every (slot, target) of each M2L batch ahead of
// the contraction (the lookups are chains of dependent loads, cheap when
// thousands are in flight) and lists, per batch, the slots with at least one
// source.  One block per batch of up to `tchunk` (64 or 128) targets; with
// pair_count set it also counts the (target, source) pairs, with lact / msrc
// set it flags the targets with a source and the sources.
__global__ void k_m2l_sources(ContractArgs a, int tchunk, int *src_tab, int *slot_list, int *nslots_tab,
                              int *tslot_list, unsigned long long *pair_count, const uint8_t *order_p16,
                              uint8_t *slot_p16, unsigned long long *nt_sum, uint8_t *lact, uint8_t *msrc,
                              int cell0) {
  __shared__ int s_flag[189];
  __shared__ int s_tgt[128];
  __shared__ int s_cnt;
  __shared__ unsigned long long s_nt;
  const int4 b = a.batches[blockIdx.x];
  const int tid = threadIdx.x;
  const int nsl = a.dim == 3 ? 189 : 27;
  if (tid < tchunk) s_tgt[tid] = tid < b.y ? a.tlist[b.x + tid] : -1;
  for (int i = tid; i < 189; i += blockDim.x) s_flag[i] = 0;
  if (tid == 0) {
    s_cnt = 0;
    s_nt = 0;
  }
  __syncthreads();
  const size_t base = (size_t)blockIdx.x * 189;
  int cnt = 0;
  unsigned long long ntc = 0;
  for (int e = tid; e < nsl * tchunk; e += blockDim.x) {
    const int slot = e / tchunk, t = e % tchunk;
    int src = -1, ts;
    if (s_tgt[t] >= 0) src = contract_source(a, s_tgt[t], slot, b.w, b.z, ts);
    src_tab[(base + slot) * tchunk + t] = src;
    if (src >= 0) {
      s_flag[slot] = 1;
      ++cnt;
      ntc += (unsigned long long)(a.cpend[s_tgt[t]] - a.cpbeg[s_tgt[t]]);
      if (lact) lact[s_tgt[t] - cell0] = 1;
      if (msrc) msrc[src - cell0] = 1;
    }
  }
  if (pair_count && cnt) atomicAdd(&s_cnt, cnt);
  if (nt_sum && ntc) atomicAdd(&s_nt, ntc);
  __syncthreads();
  if (tid < 32) {
    int n = 0;
    for (int c0 = 0; c0 < nsl; c0 += 32) {
      const int sl = c0 + tid;
      const bool f = sl < nsl && s_flag[sl];
      const unsigned m = __ballot_sync(0xffffffffu, f);
      if (f) {
        const int at = n + __popc(m & ((1u << tid) - 1u));
        slot_list[base + at] = sl;
        const int ts = (c_m2l_slots[a.dim - 2][b.w][sl] & 511) + b.z * a.level_stride;
        if (tslot_list) tslot_list[base + at] = ts;
        if (slot_p16) slot_p16[base + at] = order_p16[ts];
      }
      n += __popc(m);
    }
    if (tid == 0) {
      nslots_tab[blockIdx.x] = n;
      if (pair_count && s_cnt) atomicAdd(pair_count, (unsigned long long)s_cnt);
      if (nt_sum && s_nt) atomicAdd(nt_sum, s_nt);
    }
  }
}

// ------------------------------------------------------------------ P2M
// One thread per particle (leaf order); each coefficient is summed over the
// particles of a leaf by a segmented warp reduction, then added by the
// segment's first lane.
__device__ inline float seg_sum(float v, const bool *same) {
#pragma unroll
  for (int o = 1, k = 0; o < 32; o <<= 1, ++k) {
    float t = __shfl_down_sync(0xffffffffu, v, o);
    if (same[k]) v += t;
  }
  return v;
}

__global__ void k_p2m3d(const float4 *part, const int *leaf_of, int64_t n, int cell0, float inv_s, int p, int KS,
                        float *M) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  bool valid = i < n;
  float4 q = valid ? part[i] : make_float4(0.f, 0.f, 0.f, 0.f);
  int seg = valid ? leaf_of[i] : -1 - lane;
  bool same[5];
#pragma unroll
  for (int o = 1, k = 0; o < 32; o <<= 1, ++k) {
    int so = __shfl_down_sync(0xffffffffu, seg, o);
    same[k] = (lane + o < 32) && so == seg;
  }
  int sp = __shfl_up_sync(0xffffffffu, seg, 1);
  bool head = valid && (lane == 0 || sp != seg);
  float *Mrow = M + (size_t)(valid ? seg - cell0 : 0) * KS;
  const float x = q.x * inv_s, y = q.y * inv_s, z = q.z * inv_s, r2 = x * x + y * y + z * z, w = q.w;
  float dre = 1.f, dim_ = 0.f;
  for (int m = 0; m <= p; ++m) {
    if (m > 0) {
      float h = -0.5f / m;
      float nre = h * (x * dre - y * dim_), nim = h * (x * dim_ + y * dre);
      dre = nre;
      dim_ = nim;
    }
    float p1re = dre, p1im = dim_, p2re = 0.f, p2im = 0.f;
    for (int l = m; l <= p; ++l) {
      float cre, cim;
      if (l == m) {
        cre = dre;
        cim = dim_;
      } else {
        float a1 = c_rec1[l][m] * z, a2 = c_rec2[l][m] * r2;
        cre = a1 * p1re - a2 * p2re;
        cim = a1 * p1im - a2 * p2im;
        p2re = p1re;
        p2im = p1im;
        p1re = cre;
        p1im = cim;
      }
      float vr = seg_sum(w * cre, same);
      if (head) atomicAdd(Mrow + re_idx(l, m), vr);
      if (m > 0) {
        float vi = seg_sum(-w * cim, same);
        if (head) atomicAdd(Mrow + im_idx(l, m), vi);
      }
    }
  }
}

// ------------------------------------------------------------------ L2P
__device__ inline float2 lget(const float *Lr, int n, int m) {
  if (m > n) return make_float2(0.f, 0.f);
  if (m >= 0) return make_float2(Lr[re_idx(n, m)], m ? Lr[im_idx(n, m)] : 0.f);
  // m = -1: L_n^-1 = -conj(L_n^1)
  return make_float2(-Lr[re_idx(n, 1)], Lr[im_idx(n, 1)]);
}

// With `esrc` set, the expansion evaluated for the particles of a leaf is
// that of the leaf's deepest ancestor-or-self on a path to a cell with M2L
// contributions (esrc[leaf] = that cell, elev its level, -1: none, far field
// zero): below it the local expansion only moves by L2L, which is exact, so
// evaluating it there gives the same field without the L2L chain.  Offsets
// of the particles from level-d centres: `part` at the leaf level,
// lvl_off[(d - 2) n + i] above.
//
// P > 0: the order as a compile-time constant (P == p), so that the loops over
// (l, m) unroll completely and every coefficient index and recurrence factor
// is an immediate; P = 0 takes any p at run time.
template <int P, bool POT>
__global__ void k_l2p3d(const float4 *part, const int *leaf_of, int64_t n, int cell0, float inv_s, int p, int KS,
                        const float *L, float4 *far, const int *esrc, const uint8_t *elev, int leaf_first, int D,
                        const float4 *lvl_off, float inv_s0) {
  if (P) p = P;
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 q = part[i];
  int src = leaf_of[i];
  if (esrc) {
    const int lf = src - leaf_first;
    src = esrc[lf];
    if (src < 0) {
      far[i] = make_float4(0.f, 0.f, 0.f, 0.f);
      return;
    }
    const int lev = elev[lf];
    if (lev < D) q = lvl_off[(size_t)(lev - 2) * n + i];
    inv_s = ldexpf(inv_s0, lev);
  }
  const float *Lr = L + (size_t)(src - cell0) * KS;
  const float x = q.x * inv_s, y = q.y * inv_s, z = q.z * inv_s, r2 = x * x + y * y + z * z;
  float gx = 0.f, gy = 0.f, gz = 0.f, ph = 0.f;
  float dre = 1.f, dim_ = 0.f;
#pragma unroll
  for (int m = 0; m <= p; ++m) {
    if (m > 0) {
      float h = -0.5f / m;
      float nre = h * (x * dre - y * dim_), nim = h * (x * dim_ + y * dre);
      dre = nre;
      dim_ = nim;
    }
    const float wm = m ? 2.f : 1.f;
    float p1re = dre, p1im = dim_, p2re = 0.f, p2im = 0.f;
#pragma unroll
    for (int l = m; l <= p; ++l) {
      float cre, cim;
      if (l == m) {
        cre = dre;
        cim = dim_;
      } else {
        float a1 = c_rec1[l][m] * z, a2 = c_rec2[l][m] * r2;
        cre = a1 * p1re - a2 * p2re;
        cim = a1 * p1im - a2 * p2im;
        p2re = p1re;
        p2im = p1im;
        p1re = cre;
        p1im = cim;
      }
      if (POT) {
        const float2 Lv = lget(Lr, l, m);
        ph += wm * (Lv.x * cre - Lv.y * cim);
      }
      if (l < p) {
        float2 A = lget(Lr, l + 1, m), Lm = lget(Lr, l + 1, m - 1), Lp = lget(Lr, l + 1, m + 1);
        gz += wm * (A.x * cre - A.y * cim);
        float axr = 0.5f * (Lm.x - Lp.x), axi = 0.5f * (Lm.y - Lp.y);
        gx += wm * (axr * cre - axi * cim);
        float sr = Lp.x + Lm.x, si = Lp.y + Lm.y;  // Re(-i S R / 2) = Im(S R) / 2
        gy += wm * 0.5f * (sr * cim + si * cre);
      }
    }
  }
  far[i] = make_float4(gx * inv_s * inv_s, gy * inv_s * inv_s, gz * inv_s * inv_s, ph * inv_s);
}

using L2P3dFn = void (*)(const float4 *, const int *, int64_t, int, float, int, int, const float *, float4 *, const int *,
                         const uint8_t *, int, int, const float4 *, float);

// The L2P instantiation for order p: unrolled for the orders the passes use
// most (8: batched ensembles, 12: a 1e-6 force error), the generic one else.
static L2P3dFn l2p3d_kernel(int p, bool pot) {
  switch (p) {
    case 8: return pot ? k_l2p3d<8, true> : k_l2p3d<8, false>;
    case 12: return pot ? k_l2p3d<12, true> : k_l2p3d<12, false>;
    default: return pot ? k_l2p3d<0, true> : k_l2p3d<0, false>;
  }
}

// ------------------------------------------------------------------ 2D
// P2M / L2P of the complex-log expansions (power_set2D.cpp:9-21,
// local_set2D.cpp:60-69) with coefficients scaled by the cell size s:
// a~_k = sum_i m_i ((z_i - c)/s)^k, stored [a_0, Re a_1, Im a_1, ...].
__global__ void k_p2m2d(const float4 *part, const int *leaf_of, int64_t n, int cell0, float inv_s, int p, int KS,
                        float *M) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  bool valid = i < n;
  float4 q = valid ? part[i] : make_float4(0.f, 0.f, 0.f, 0.f);
  int seg = valid ? leaf_of[i] : -1 - lane;
  bool same[5];
#pragma unroll
  for (int o = 1, k = 0; o < 32; o <<= 1, ++k) {
    int so = __shfl_down_sync(0xffffffffu, seg, o);
    same[k] = (lane + o < 32) && so == seg;
  }
  int sp = __shfl_up_sync(0xffffffffu, seg, 1);
  bool head = valid && (lane == 0 || sp != seg);
  float *Mrow = M + (size_t)(valid ? seg - cell0 : 0) * KS;
  const float x = q.x * inv_s, y = q.y * inv_s, w = q.w;
  float v = seg_sum(w, same);
  if (head) atomicAdd(Mrow, v);
  float pr = w, pi = 0.f;  // w (z/s)^k
  for (int k = 1; k <= p; ++k) {
    const float nr = pr * x - pi * y, ni = pr * y + pi * x;
    pr = nr;
    pi = ni;
    float vr = seg_sum(pr, same), vi = seg_sum(pi, same);
    if (head) {
      atomicAdd(Mrow + 2 * k - 1, vr);
      atomicAdd(Mrow + 2 * k, vi);
    }
  }
}

// L^ = [Re b_0, Re b_1, Im b_1, ...] with b^_n = b_n s^n represents
// sum_j m_j log(z - z_j); phi = -Re sum b^_n u^n and
// grad = (1/s) (-Re, +Im)(sum n b^_n u^(n-1)), u = (z - c)/s.
__global__ void k_l2p2d(const float4 *part, const int *leaf_of, int64_t n, int cell0, float inv_s, int p, int KS,
                        const float *L, float4 *far) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 q = part[i];
  const float *Lr = L + (size_t)(leaf_of[i] - cell0) * KS;
  const float x = q.x * inv_s, y = q.y * inv_s;
  float phr = Lr[0], dr = 0.f, di = 0.f, ur = 1.f, ui = 0.f;  // u^(n-1)
  for (int k = 1; k <= p; ++k) {
    const float br = Lr[2 * k - 1], bi = Lr[2 * k];
    dr += k * (br * ur - bi * ui);
    di += k * (br * ui + bi * ur);
    const float nr = ur * x - ui * y, ni = ur * y + ui * x;
    ur = nr;
    ui = ni;
    phr += br * ur - bi * ui;
  }
  far[i] = make_float4(-dr * inv_s, di * inv_s, 0.f, -phr);
}

// ------------------------------------------------------------------ P2P
// Error-free sum: s + e == a + b exactly (Knuth's TwoSum).
__device__ inline void two_sum(float a, float b, float &s, float &e) {
  s = a + b;
  float bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}

// One pair: grad -= m d/|d|^3, phi += m/|d| (3D, leaf.cpp:118-142) or
// grad -= m d/|d|^2, phi -= m log|d| (2D, leaf.cpp:81-95), r^2 -> r^2 + eps2.
// 1/sqrt(x) by the SFU (PTX rsqrt.approx.ftz.f32, relative error below
// 2^-22.9), without the subnormal-input handling of rsqrtf: the r^2 of
// distinct particles here is far above the FP32 subnormal range.
__device__ __forceinline__ float rsqrt_sfu(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

template <int DIM, bool NEWTON = true, bool POT = true>
__device__ inline void pair_acc(float rx, float ry, float rz, float w, float eps2, float &ax, float &ay, float &az,
                                float &ph) {
  if (DIM == 3) {
    const float r2 = fmaf(rx, rx, fmaf(ry, ry, fmaf(rz, rz, eps2)));
    float inv = rsqrt_sfu(r2);
    if (NEWTON) inv = inv * fmaf(-0.5f * r2 * inv, inv, 1.5f);  // one Newton step
    const float mi = w * inv;
    const float mi3 = mi * inv * inv;
    ax = fmaf(-rx, mi3, ax);
    ay = fmaf(-ry, mi3, ay);
    az = fmaf(-rz, mi3, az);
    if (POT) ph += mi;
  } else {
    const float r2 = fmaf(rx, rx, fmaf(ry, ry, eps2));
    const float f = w / r2;
    ax = fmaf(-rx, f, ax);
    ay = fmaf(-ry, f, ay);
    if (POT) ph = fmaf(-0.5f * w, logf(r2), ph);
  }
}

// Fire-and-forget vector reduction into a float4 in global memory.
__device__ inline void red_add4(float4 *p, float x, float y, float z, float w) {
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(x), "f"(y), "f"(z), "f"(w) : "memory");
}

struct P2PArgs {
  int leaf_first, nleaves, depth;
  const int *pbeg, *pend, *coll, *parent, *child, *leaf_of;
  const uint64_t *ckey;
  const float4 *part, *part_lo, *far;
  const uint32_t *perm;
  double hx, hy, hz;
  float eps2;
  long long direct_max;
  double G;
  double *acc, *pot;
  unsigned int *err;
  unsigned long long *pair_count;
};

// One warp per target leaf; the leaf's particles are spread over the lanes
// (several lanes per particle for small leaves, each taking a share of the
// sources).  Sources: the leaf itself (j != i) and its existing neighbours
// (leaf.cpp:118-142).  The direct far field (interaction-list pairs summed
// particle by particle) has been added into `far` by k_direct_far before
// this kernel runs; this kernel adds the near field and writes the output.
//
// Near-field precision: x_i - x_j = (t_i - shift) - s_j with t_i, s_j the
// offsets from the two leaf centres and shift = c_s - c_t an exact multiple
// of the leaf size.  Offsets are hi + lo FP32 pairs, the shift is hi + lo
// from FP64, and (t_hi - shift_hi) is formed error-free (TwoSum), so each
// difference is rounded once, relative to itself, whatever the separation.
template <int DIM, bool POT>
__global__ void k_p2p(P2PArgs a) {
  constexpr int NS = DIM == 3 ? 27 : 9;
  const int lane = threadIdx.x & 31;
  const int wl = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (wl >= a.nleaves) return;
  const int g = a.leaf_first + wl;
  const int tb = a.pbeg[g], nt = a.pend[g] - tb;
  const int tp = nt < 32 ? nt : 32;
  int Gl = 1;
  while (Gl * 2 * tp <= 32) Gl *= 2;
  const int tpp = 32 / Gl;
  const int *cl = a.coll + (int64_t)g * NS;
  bool bad = false;
  long long npairs = 0;
  for (int t0 = 0; t0 < nt; t0 += tpp) {
    const int ti = t0 + lane / Gl, sub = lane % Gl;
    const bool act = ti < nt;
    const int me_i = tb + (act ? ti : 0);
    const float4 me = a.part[me_i], mel = a.part_lo[me_i];
    float ax = 0.f, ay = 0.f, az = 0.f, ph = 0.f;
    for (int s = 0; s < NS; ++s) {
      const int S = cl[s];
      if (S < 0) continue;
      // shift = c_s - c_t in hi + lo
      const double sx = (s % 3 - 1) * a.hx, sy = ((s / 3) % 3 - 1) * a.hy, sz = DIM == 3 ? (s / 9 - 1) * a.hz : 0.0;
      const float shx = (float)sx, shy = (float)sy, shz = (float)sz;
      float tx, ty, tz, ex, ey, ez;
      two_sum(me.x, -shx, tx, ex);
      two_sum(me.y, -shy, ty, ey);
      two_sum(me.z, -shz, tz, ez);
      ex += mel.x - (float)(sx - (double)shx);
      ey += mel.y - (float)(sy - (double)shy);
      ez += mel.z - (float)(sz - (double)shz);
      const int se = a.pend[S];
      if (t0 == 0 && lane == 0) npairs += (long long)nt * (se - a.pbeg[S]) - (S == g ? nt : 0);
      for (int j = a.pbeg[S] + sub; j < se; j += Gl) {
        if (j == me_i) continue;
        const float4 q = a.part[j], ql = a.part_lo[j];
        const float rx = (tx - q.x) + (ex - ql.x);
        const float ry = (ty - q.y) + (ey - ql.y);
        const float rz = (tz - q.z) + (ez - ql.z);
        pair_acc<DIM, true, POT>(rx, ry, rz, q.w, a.eps2, ax, ay, az, ph);
      }
    }
    for (int o = 1; o < Gl; o <<= 1) {
      ax += __shfl_xor_sync(0xffffffffu, ax, o);
      ay += __shfl_xor_sync(0xffffffffu, ay, o);
      az += __shfl_xor_sync(0xffffffffu, az, o);
      ph += __shfl_xor_sync(0xffffffffu, ph, o);
    }
    if (act && sub == 0) {
      const float4 f = a.far[me_i];
      const uint32_t o = a.perm[me_i];
      double vx = a.G * ((double)f.x + ax), vy = a.G * ((double)f.y + ay), vz = a.G * ((double)f.z + az);
      a.acc[DIM * (size_t)o] = vx;
      a.acc[DIM * (size_t)o + 1] = vy;
      if (DIM == 3) a.acc[3 * (size_t)o + 2] = vz;
      if (a.pot) a.pot[o] = a.G * ((double)f.w + ph);
      bad |= !(isfinite(vx) && isfinite(vy) && isfinite(vz));
    }
  }
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(a.err, FMM_DEV_ERR_NONFINITE_OUTPUT);
  if (lane == 0 && a.pair_count) atomicAdd(a.pair_count, (unsigned long long)npairs);
}

// Adaptive targets: the colleague sums of the adaptive leaves.  An adaptive
// leaf B (any level, listed in alist[0 .. acount)) sums the particles of B
// itself (j != i) and of its colleagues at B's level: the pairs that the
// deeper levels' interaction lists and the leaf level's near field would sum
// in the uniform tree.  A colleague may hold millions of particles (a sparse
// cell next to a dense clump), so the work is cut into items of at most
// p2p_chunk sources of B's concatenated colleague list, each one warp's job;
// items of one B add into the far-field accumulator with vector reductions.
//
// Precision: colleagues touch B, so pairs can be far closer than the cell
// size.  Positions are taken relative to an origin inside B (its first
// particle) in FP64 and split into FP32 hi + lo parts; a difference
// (t_hi - s_hi) + (t_lo - s_lo) is then rounded once relative to itself, as
// in the uniform near field.  1/|r| is the SFU's rsqrt without a Newton step,
// as in the direct far field (relative error below 2^-22.9; with the step the
// 16M mixture's force error was the same, 7.7e-7, and the kernel 6 % slower).
// The chunk (sources per item) is a setting,
// fmm_config.p2p_chunk, 256 by default.
static constexpr int CL_CHUNK_DEFAULT = 256;

// Number of items of each listed adaptive leaf (0 past the list's end), over
// [0, ncell) so that the host needs no count.
__global__ void k_colleague_count(const int *alist, const unsigned *acount, int ncell, const int *coll,
                                  const int *pbeg, const int *pend, int ns, int chunk, uint32_t *cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncell) return;
  uint32_t items = 0;
  if (i < (int)*acount) {
    const int B = alist[i];
    long long S = 0;
    for (int s = 0; s < ns; ++s) {
      const int C = coll[(int64_t)B * ns + s];
      if (C >= 0) S += pend[C] - pbeg[C];
    }
    items = pend[B] > pbeg[B] ? (uint32_t)((S + chunk - 1) / chunk) : 0u;
  }
  cnt[i] = items;
}

// items[off[i] + k] = (i, k) for the k-th chunk of listed leaf i.
__global__ void k_colleague_fill(const unsigned *acount, int ncell, const uint32_t *cnt, const uint32_t *off,
                                 int2 *items) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncell || i >= (int)*acount) return;
  const uint32_t o = off[i], c = cnt[i];
  for (uint32_t k = 0; k < c; ++k) items[o + k] = make_int2(i, (int)k);
}

__device__ inline void split_hi_lo(double d, float &hi, float &lo) {
  hi = (float)d;
  lo = (float)(d - (double)hi);
}

// One item's concatenated source range [f0, f1), B's own particles at
// [bbeg, bend) in it, and the FP64 origin of the hi + lo offsets.
struct CollChunk {
  int f0, f1, bbeg, bend, ncoll;
  double ox, oy, oz;
};

// Lanes per target group for R targets per lane (largest power of two with
// ceil(nt / R) * Gl <= 32) and the work of the busiest lane per source:
// rounds x (R pairs of about 19 instructions with the hi + lo differences,
// and 4 for the two staged loads and the loop) / Gl.
__device__ inline void colleague_shape(int nt, int R, int &Gl, float &cost) {
  const int groups = (nt + R - 1) / R;
  Gl = 1;
  while (Gl * 2 * groups <= 32) Gl *= 2;
  const int rounds = (groups + 32 / Gl - 1) / (32 / Gl);
  cost = (float)rounds * (float)(19 * R + 4) / (float)Gl;
}

// The targets of B, R to a lane, in target groups of Gl lanes that share the
// sources (every Gl-th of each chunk of 32 staged through shared memory).
// Only chunks that hold some of B's own particles test for j == i.
template <int R, int DIM, bool POT>
__device__ void colleague_targets(const P2PArgs &a, const double *xs, float4 *far, int tb, int nt, int Gl,
                                  const CollChunk &cc, const int *s_pref, const int *s_cell, float4 *s_hi,
                                  float4 *s_lo, int lane) {
  const int groups = (nt + R - 1) / R, gpr = 32 / Gl;
  for (int g0 = 0; g0 < groups; g0 += gpr) {
    const int gi = g0 + lane / Gl, sub = lane % Gl;
    const bool live = gi < groups;
    float thx[R], tlx[R], thy[R], tly[R], thz[R], tlz[R], ax[R], ay[R], az[R], ph[R];
    int me[R];  // the target's particle index (target 0's for the lanes' padding)
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int ti = gi * R + r;
      me[r] = tb + (live && ti < nt ? ti : 0);
      split_hi_lo(xs[DIM * (size_t)me[r]] - cc.ox, thx[r], tlx[r]);
      split_hi_lo(xs[DIM * (size_t)me[r] + 1] - cc.oy, thy[r], tly[r]);
      thz[r] = tlz[r] = 0.f;
      if (DIM == 3) split_hi_lo(xs[DIM * (size_t)me[r] + 2] - cc.oz, thz[r], tlz[r]);
      ax[r] = ay[r] = az[r] = ph[r] = 0.f;
    }
    for (int fb = cc.f0; fb < cc.f1; fb += 32) {
      const int f = fb + lane;
      if (f < cc.f1) {
        // colleague holding concatenated position f: the last k with s_pref[k] <= f
        int lo = 0, hi = cc.ncoll - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (s_pref[mid] <= f) lo = mid;
          else hi = mid - 1;
        }
        const int j = a.pbeg[s_cell[lo]] + (f - s_pref[lo]);
        float hx, lx, hy, ly, hz = 0.f, lz = 0.f;
        split_hi_lo(xs[DIM * (size_t)j] - cc.ox, hx, lx);
        split_hi_lo(xs[DIM * (size_t)j + 1] - cc.oy, hy, ly);
        if (DIM == 3) split_hi_lo(xs[DIM * (size_t)j + 2] - cc.oz, hz, lz);
        s_hi[lane] = make_float4(hx, hy, hz, a.part[j].w);
        s_lo[lane] = make_float4(lx, ly, lz, __int_as_float(j));
      }
      __syncwarp();
      const int cnt = min(32, cc.f1 - fb);
      if (fb < cc.bend && fb + cnt > cc.bbeg) {
        for (int k = sub; k < cnt; k += Gl) {
          const float4 q = s_hi[k], ql = s_lo[k];
          const int j = __float_as_int(ql.w);
#pragma unroll
          for (int r = 0; r < R; ++r) {
            if (j == me[r]) continue;
            const float rx = (thx[r] - q.x) + (tlx[r] - ql.x);
            const float ry = (thy[r] - q.y) + (tly[r] - ql.y);
            const float rz = (thz[r] - q.z) + (tlz[r] - ql.z);
            pair_acc<DIM, false, POT>(rx, ry, rz, q.w, a.eps2, ax[r], ay[r], az[r], ph[r]);
          }
        }
      } else {
        for (int k = sub; k < cnt; k += Gl) {
          const float4 q = s_hi[k], ql = s_lo[k];
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const float rx = (thx[r] - q.x) + (tlx[r] - ql.x);
            const float ry = (thy[r] - q.y) + (tly[r] - ql.y);
            const float rz = (thz[r] - q.z) + (tlz[r] - ql.z);
            pair_acc<DIM, false, POT>(rx, ry, rz, q.w, a.eps2, ax[r], ay[r], az[r], ph[r]);
          }
        }
      }
      __syncwarp();
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      for (int o = 1; o < Gl; o <<= 1) {
        ax[r] += __shfl_xor_sync(0xffffffffu, ax[r], o);
        ay[r] += __shfl_xor_sync(0xffffffffu, ay[r], o);
        az[r] += __shfl_xor_sync(0xffffffffu, az[r], o);
        if (POT) ph[r] += __shfl_xor_sync(0xffffffffu, ph[r], o);
      }
      const int ti = gi * R + r;
      if (sub == 0 && live && ti < nt) red_add4(far + tb + ti, ax[r], ay[r], az[r], ph[r]);
    }
  }
}

// One warp per item (grid-stride): B's targets R to a lane in groups of Gl
// lanes (colleague_targets), the item's sources staged 32 at a time through
// shared memory.
template <int DIM, bool POT>
__global__ void __launch_bounds__(256, 4) k_colleague_sum(P2PArgs a, const int *alist, const int2 *items,
                                                       const uint32_t *nitems, const double *xs, float4 *far,
                                                       int chunk) {
  constexpr int NS = DIM == 3 ? 27 : 9;
  __shared__ float4 s_hi_all[8][32], s_lo_all[8][32];
  __shared__ int s_pref_all[8][NS + 1], s_cell_all[8][NS];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  float4 *s_hi = s_hi_all[wib], *s_lo = s_lo_all[wib];
  int *s_pref = s_pref_all[wib], *s_cell = s_cell_all[wib];
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  const int total = (int)*nitems;
  long long npairs = 0;
  for (int it = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); it < total; it += nwarps) {
    const int2 item = items[it];
    const int B = alist[item.x];
    const int tb = a.pbeg[B], nt = a.pend[B] - tb;
    // B's colleagues (B itself included), compacted, with the prefix of their sizes
    const int C = lane < NS ? a.coll[(int64_t)B * NS + lane] : -1;
    const int nc = C >= 0 ? a.pend[C] - a.pbeg[C] : 0;
    const unsigned m = __ballot_sync(0xffffffffu, C >= 0);
    int x = nc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    const int ncoll = __popc(m);
    if (C >= 0) {
      const int at = __popc(m & ((1u << lane) - 1u));
      s_cell[at] = C;
      s_pref[at + 1] = x;  // inclusive prefix (zero-size colleagues repeat the previous value)
    }
    if (lane == 0) s_pref[0] = 0;
    __syncwarp();
    const int S = s_pref[ncoll];
    const int f0 = item.y * chunk, f1 = min(S, f0 + chunk);
    // B's own particles in the concatenation (the pairs j == i are skipped)
    const int bl = __ffs(__ballot_sync(0xffffffffu, C == B)) - 1;
    const int bend = __shfl_sync(0xffffffffu, x, bl), bbeg = bend - __shfl_sync(0xffffffffu, nc, bl);
    const double ox = xs[DIM * (size_t)tb], oy = xs[DIM * (size_t)tb + 1], oz = DIM == 3 ? xs[DIM * (size_t)tb + 2] : 0.0;
    // the register blocking R in 1..4 with the least work on the busiest lane (larger R on ties)
    int bestR = 1, bestG = 1;
    float best = 1e30f;
#pragma unroll
    for (int R = 1; R <= 4; ++R) {
      int G;
      float c;
      colleague_shape(nt, R, G, c);
      if (c <= best) {
        best = c;
        bestR = R;
        bestG = G;
      }
    }
    const CollChunk cc{f0, f1, bbeg, bend, ncoll, ox, oy, oz};
    switch (bestR) {
      case 1: colleague_targets<1, DIM, POT>(a, xs, far, tb, nt, bestG, cc, s_pref, s_cell, s_hi, s_lo, lane); break;
      case 2: colleague_targets<2, DIM, POT>(a, xs, far, tb, nt, bestG, cc, s_pref, s_cell, s_hi, s_lo, lane); break;
      case 3: colleague_targets<3, DIM, POT>(a, xs, far, tb, nt, bestG, cc, s_pref, s_cell, s_hi, s_lo, lane); break;
      default: colleague_targets<4, DIM, POT>(a, xs, far, tb, nt, bestG, cc, s_pref, s_cell, s_hi, s_lo, lane); break;
    }
    if (lane == 0) npairs += (long long)nt * (f1 - f0) - max(0, min(f1, bend) - max(f0, bbeg));
  }
  if (lane == 0 && a.pair_count && npairs) atomicAdd(a.pair_count, (unsigned long long)npairs);
}

// The output: acc[perm[i]] = G * far[i] (and the potential), with the
// finiteness check, after every contribution was added into far.
template <int DIM>
__global__ void k_far_output(const float4 *far, const uint32_t *perm, int64_t n, double G, double *acc, double *pot,
                             unsigned int *err) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool bad = false;
  if (i < n) {
    const float4 f = far[i];
    const uint32_t o = perm[i];
    const double vx = G * (double)f.x, vy = G * (double)f.y, vz = G * (double)f.z;
    acc[DIM * (size_t)o] = vx;
    acc[DIM * (size_t)o + 1] = vy;
    if (DIM == 3) acc[3 * (size_t)o + 2] = vz;
    if (pot) pot[o] = G * (double)f.w;
    bad = !(isfinite(vx) && isfinite(vy) && isfinite(vz));
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(err, FMM_DEV_ERR_NONFINITE_OUTPUT);
}

// --------------------------------------------------------- direct far field
// Offsets of every particle (leaf order) from the centre of its ancestor at
// each level d in [d0, d1], FP32, with the mass: the frames in which pairs of
// level-d cells are summed directly.  out[(d - d0) * n + i].
template <int DIM>
__global__ void k_level_offsets(const double *pos, const double *mass, const uint32_t *perm, const int *leaf_of,
                                const uint64_t *ckey, int64_t n, int depth, int d0, int d1, double lox, double loy,
                                double loz, double ex, double ey, double ez, float4 *out) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t qx, qy, qz;
  morton_decode(DIM, ckey[leaf_of[i]], qx, qy, qz);
  const uint32_t j = perm[i];
  const double px = pos[DIM * (size_t)j], py = pos[DIM * (size_t)j + 1], pz = DIM == 3 ? pos[3 * (size_t)j + 2] : 0.0;
  const float w = (float)mass[j];
  for (int d = d0; d <= d1; ++d) {
    const int sh = depth - d;
    const double inv = ldexp(1.0, -d);
    const double cx = lox + ((double)(qx >> sh) + 0.5) * (ex * inv);
    const double cy = loy + ((double)(qy >> sh) + 0.5) * (ey * inv);
    const double cz = DIM == 3 ? loz + ((double)(qz >> sh) + 0.5) * (ez * inv) : 0.0;
    out[(size_t)(d - d0) * n + i] =
        make_float4((float)(px - cx), (float)(py - cy), DIM == 3 ? (float)(pz - cz) : 0.f, w);
  }
}

static constexpr int DF_MAX_LEVELS = 33;

struct DirectArgs {
  // levels of the launch, coarse first: warps [w0[k], w0[k+1]) take the
  // cells first[k] + (warp - w0[k]), or with a target list (k_direct_far's
  // LIST) the cells tlist[first[k] + (warp - w0[k])]
  int nlev;
  int first[DF_MAX_LEVELS], w0[DF_MAX_LEVELS + 1];
  const float4 *off[DF_MAX_LEVELS];  // particle offsets from their level-d ancestor's centre
  float h[DF_MAX_LEVELS][3];         // level-d cell size
  const int *pbeg, *pend, *coll, *parent, *child;
  const uint64_t *ckey;
  float eps2;
  long long direct_max;
  const uint8_t *fdirect;  // per offset: not well separated, always summed directly
  int any_fdirect;
  float4 *far;
  unsigned long long *pair_count;
  const int *tlist;        // adaptive targets: each level's targets, from first[k]
};

// One warp per level-d target cell T with n_T <= direct_max: the sources are
// the cells S of T's interaction list (node_i.cpp:39-43) with
// n_T * n_S <= direct_max, exactly the pairs the M2L contraction skips.
// Small T (NT <= 7 targets): every lane holds all targets and takes every
// 32nd particle of the concatenated sources; larger T: register-blocked
// target groups over sources staged through shared memory.
//
// Per kept source cell si the warp keeps s_pref[si] (its first position in
// the concatenation; every cell non-empty) and s_cell[si] = (shift c_S - c_T,
// index delta): the particle at concatenated position f of cell si is
// off[f + delta].

// For the chunk f0 .. f0 + 31, given the cell si0 holding f0, returns the
// cell holding f0 + lane (lanes past the end get the last cell; the caller
// masks them) and moves si0 to the cell holding f0 + 32: one shared load per
// lane, the cell starts inside the chunk as the bits of a warp-wide OR, and a
// population count (at most 32 cells overlap 32 consecutive positions).
__device__ inline int chunk_cell(const int *s_pref, int nsrc, int f0, int &si0, int lane) {
  const int c = si0 + lane;
  const int rel = c < nsrc ? s_pref[c] - f0 : 32;  // lane 0: <= 0
  const unsigned bit = rel < 32 ? 1u << max(rel, 0) : 0u;
  const unsigned starts = __reduce_or_sync(0xffffffffu, bit);
  const int si = si0 + __popc(starts & (0xffffffffu >> (31 - lane))) - 1;
  const int last = __shfl_sync(0xffffffffu, si, 31);
  si0 = s_pref[last + 1] <= f0 + 32 ? last + 1 : last;
  return si;
}

// The source particle at concatenated position f of cell si, shifted into
// the target's frame.
__device__ inline float4 shifted_source(const float4 *off, const float4 *s_cell, int f, int si) {
  const float4 cd = s_cell[si];
  const float4 q = off[f + __float_as_int(cd.w)];
  return make_float4(q.x + cd.x, q.y + cd.y, q.z + cd.z, q.w);
}

template <int NT, int DIM, bool POT>
__device__ void direct_small(const DirectArgs &a, const float4 *off, int tb, int nt, const float4 *s_cell,
                             const int *s_pref, int nsrc, int lane) {
  float tx[NT], ty[NT], tz[NT], ax[NT], ay[NT], az[NT], ph[NT];
#pragma unroll
  for (int k = 0; k < NT; ++k) {
    float4 t = off[tb + (k < nt ? k : 0)];
    tx[k] = t.x;
    ty[k] = t.y;
    tz[k] = t.z;
    ax[k] = ay[k] = az[k] = ph[k] = 0.f;
  }
  const int total = s_pref[nsrc];
  int si0 = 0;
  for (int f0 = 0; f0 < total; f0 += 32) {
    const int f = f0 + lane;
    const int si = chunk_cell(s_pref, nsrc, f0, si0, lane);
    if (f < total) {
      const float4 q = shifted_source(off, s_cell, f, si);
#pragma unroll
      for (int k = 0; k < NT; ++k)
        pair_acc<DIM, false, POT>(tx[k] - q.x, ty[k] - q.y, tz[k] - q.z, q.w, a.eps2, ax[k], ay[k], az[k], ph[k]);
    }
  }
#pragma unroll
  for (int k = 0; k < NT; ++k) {
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      ax[k] += __shfl_xor_sync(0xffffffffu, ax[k], o);
      ay[k] += __shfl_xor_sync(0xffffffffu, ay[k], o);
      az[k] += __shfl_xor_sync(0xffffffffu, az[k], o);
      ph[k] += __shfl_xor_sync(0xffffffffu, ph[k], o);
    }
    if (lane == k && k < nt) red_add4(a.far + tb + k, ax[k], ay[k], az[k], ph[k]);
  }
}

// Larger T: each lane holds R targets and takes every Gl-th source of the
// chunks of 32 staged through shared memory; ceil(nt / R) target groups of
// Gl lanes, 32 / Gl groups per round.
template <int R, int DIM, bool POT>
__device__ void direct_blocked(const DirectArgs &a, const float4 *off, int tb, int nt, int Gl, const float4 *s_cell,
                               const int *s_pref, int nsrc, int lane, float4 *stage) {
  const int groups = (nt + R - 1) / R, gpr = 32 / Gl;
  const int total = s_pref[nsrc];
  for (int g0 = 0; g0 < groups; g0 += gpr) {
    const int gi = g0 + lane / Gl, sub = lane % Gl;
    float tx[R], ty[R], tz[R], ax[R], ay[R], az[R], ph[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int ti = gi * R + r;
      const float4 t = off[tb + (gi < groups && ti < nt ? ti : 0)];
      tx[r] = t.x;
      ty[r] = t.y;
      tz[r] = t.z;
      ax[r] = ay[r] = az[r] = ph[r] = 0.f;
    }
    int si0 = 0;
    for (int f0 = 0; f0 < total; f0 += 32) {
      const int f = f0 + lane;
      const int si = chunk_cell(s_pref, nsrc, f0, si0, lane);
      stage[lane] = f < total ? shifted_source(off, s_cell, f, si) : make_float4(0.f, 0.f, 0.f, 0.f);
      __syncwarp();
      const int cnt = min(32, total - f0);
      for (int k = sub; k < cnt; k += Gl) {
        const float4 sq = stage[k];
#pragma unroll
        for (int r = 0; r < R; ++r)
          pair_acc<DIM, false, POT>(tx[r] - sq.x, ty[r] - sq.y, tz[r] - sq.z, sq.w, a.eps2, ax[r], ay[r], az[r], ph[r]);
      }
      __syncwarp();
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      for (int o = 1; o < Gl; o <<= 1) {
        ax[r] += __shfl_xor_sync(0xffffffffu, ax[r], o);
        ay[r] += __shfl_xor_sync(0xffffffffu, ay[r], o);
        az[r] += __shfl_xor_sync(0xffffffffu, az[r], o);
        ph[r] += __shfl_xor_sync(0xffffffffu, ph[r], o);
      }
      const int ti = gi * R + r;
      if (sub == 0 && gi < groups && ti < nt) red_add4(a.far + tb + ti, ax[r], ay[r], az[r], ph[r]);
    }
  }
}

// Lanes per target group for R targets per lane (largest power of two with
// ceil(nt / R) * Gl <= 32), and the work of the busiest lane in units of
// the source count.
__device__ inline void blocked_shape(int nt, int R, int &Gl, float &cost) {
  const int groups = (nt + R - 1) / R;
  Gl = 1;
  while (Gl * 2 * groups <= 32) Gl *= 2;
  const int rounds = (groups + 32 / Gl - 1) / (32 / Gl);
  cost = (float)(rounds * R) / (float)Gl;
}

template <int DIM, bool POT, bool LIST = false>
__global__ void __launch_bounds__(256, 4) k_direct_far(DirectArgs a) {
  constexpr int NS = DIM == 3 ? 27 : 9, NC = 1 << DIM, NCAND = NS * NC, NR = (NCAND + 31) / 32;
  __shared__ float4 s_cell_all[8][189];
  __shared__ int s_pref_all[8][190];
  __shared__ float4 s_stage_all[8][32];
  __shared__ int s_dir_all[8][32];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int wl = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (wl >= a.w0[a.nlev]) return;
  int lv = a.nlev - 1;  // deep levels, which hold most of the warps, first
  while (wl < a.w0[lv]) --lv;
  const int T = LIST ? a.tlist[a.first[lv] + (wl - a.w0[lv])] : a.first[lv] + (wl - a.w0[lv]);
  const int tb = a.pbeg[T], nt = a.pend[T] - tb;
  if ((long long)nt > a.direct_max && !a.any_fdirect) return;
  const float4 *off = a.off[lv];
  float4 *s_cell = s_cell_all[wib];
  int *s_pref = s_pref_all[wib];
  const int P = a.parent[T];
  const int cls = (int)(a.ckey[T] & (uint64_t)(NC - 1));
  // kept sources have n_S <= ns_max (n_T n_S <= direct_max)
  const int ns_max = (int)min(a.direct_max, (long long)0x7fffffff) / max(nt, 1);
  int nsrc = 0, ptotal = 0;
  if (lane == 0) s_pref[0] = 0;
  // the existing colleagues, compacted, with their directions packed as
  // (dx+1) | (dy+1) << 2 | (dz+1) << 4 | slot << 8 in s_dir; then the
  // children of those only, all candidate loads in flight at once, child
  // then counts
  int *s_dir = s_dir_all[wib];
  const int Qlane = lane < NS ? a.coll[(size_t)P * NS + lane] : -1;
  const unsigned qmask = __ballot_sync(0xffffffffu, Qlane >= 0);
  if (Qlane >= 0)
    s_dir[__popc(qmask & ((1u << lane) - 1u))] = (lane % 3) | (((lane / 3) % 3) << 2) | ((lane / 9) << 4) | (lane << 8);
  __syncwarp();
  const int ncand = __popc(qmask) * NC;
  int qv[NR], nsv[NR], pbv[NR];
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    qv[r] = -1;
    if (r * 32 < ncand) {  // warp-uniform
      const int cand = r * 32 + lane;
      const int Q = __shfl_sync(0xffffffffu, Qlane, cand < ncand ? s_dir[cand / NC] >> 8 : 0);
      if (cand < ncand) qv[r] = a.child[(size_t)Q * NC + (cand % NC)];
    }
  }
  __syncwarp();
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    pbv[r] = qv[r] >= 0 ? a.pbeg[qv[r]] : 0;
    nsv[r] = qv[r] >= 0 ? a.pend[qv[r]] - pbv[r] : 0;
  }
  const float hx = a.h[lv][0], hy = a.h[lv][1], hz = a.h[lv][2];
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    if (r * 32 >= ncand) break;  // warp-uniform
    const int cand = r * 32 + lane;
    const int k = cand % NC, d = cand < ncand ? s_dir[cand / NC] : 0;
    int q = qv[r];
    const int ddx = 2 * ((d & 3) - 1) + (k & 1) - (cls & 1);
    const int ddy = 2 * (((d >> 2) & 3) - 1) + ((k >> 1) & 1) - ((cls >> 1) & 1);
    const int ddz = DIM == 3 ? 2 * (((d >> 4) & 3) - 1) + ((k >> 2) & 1) - ((cls >> 2) & 1) : 0;
    const bool adj = ddx >= -1 && ddx <= 1 && ddy >= -1 && ddy <= 1 && ddz >= -1 && ddz <= 1;
    const bool fd = a.any_fdirect && !adj && a.fdirect[(ddx + 3) + 7 * (ddy + 3) + (DIM == 3 ? 49 * (ddz + 3) : 0)];
    if (q >= 0 && (adj || (nsv[r] > ns_max && !fd))) q = -1;
    const unsigned mask = __ballot_sync(0xffffffffu, q >= 0);
    const int pos = nsrc + __popc(mask & ((1u << lane) - 1u));
    int x = q >= 0 ? nsv[r] : 0;  // inclusive scan of the kept counts
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (q >= 0) {
      // c_S - c_T, and the delta from concatenated position to particle index
      s_cell[pos] = make_float4(ddx * hx, ddy * hy, ddz * hz, __int_as_float(pbv[r] - (ptotal + x - nsv[r])));
      s_pref[pos + 1] = ptotal + x;
    }
    ptotal += __shfl_sync(0xffffffffu, x, 31);
    nsrc += __popc(mask);
  }
  __syncwarp();
  if (nsrc == 0) return;
  if (lane == 0 && a.pair_count) atomicAdd(a.pair_count, (unsigned long long)((long long)nt * ptotal));
  switch (nt) {
    case 1: direct_small<1, DIM, POT>(a, off, tb, nt, s_cell, s_pref, nsrc, lane); return;
    case 2: direct_small<2, DIM, POT>(a, off, tb, nt, s_cell, s_pref, nsrc, lane); return;
    case 3: direct_small<3, DIM, POT>(a, off, tb, nt, s_cell, s_pref, nsrc, lane); return;
    case 4: direct_small<4, DIM, POT>(a, off, tb, nt, s_cell, s_pref, nsrc, lane); return;
    case 5: direct_small<5, DIM, POT>(a, off, tb, nt, s_cell, s_pref, nsrc, lane); return;
    case 6: direct_small<6, DIM, POT>(a, off, tb, nt, s_cell, s_pref, nsrc, lane); return;
    case 7: direct_small<7, DIM, POT>(a, off, tb, nt, s_cell, s_pref, nsrc, lane); return;
    default: break;
  }
  // larger T: the register blocking R in 1..4 that minimises the busiest lane's work (largest R on ties)
  int bestR = 1, bestG = 1;
  float best = 1e30f;
#pragma unroll
  for (int R = 1; R <= 4; ++R) {
    int G;
    float c;
    blocked_shape(nt, R, G, c);
    if (c <= best) {  // ties: the larger R reuses each staged source for more targets
      best = c;
      bestR = R;
      bestG = G;
    }
  }
  float4 *stage = s_stage_all[wib];
  switch (bestR) {
    case 1: direct_blocked<1, DIM, POT>(a, off, tb, nt, bestG, s_cell, s_pref, nsrc, lane, stage); break;
    case 2: direct_blocked<2, DIM, POT>(a, off, tb, nt, bestG, s_cell, s_pref, nsrc, lane, stage); break;
    case 3: direct_blocked<3, DIM, POT>(a, off, tb, nt, bestG, s_cell, s_pref, nsrc, lane, stage); break;
    default: direct_blocked<4, DIM, POT>(a, off, tb, nt, bestG, s_cell, s_pref, nsrc, lane, stage); break;
  }
}

// ------------------------------------------------------------------ lists
// Sort keys (level, class) of the cells of one level: key_all for L2L (every
// cell), key_m2l for M2L with 255 for cells that cannot have an M2L pair under
// the direct-pair rule (every child S of the parent's colleagues has
// n_T * n_S <= direct_max; adjacency is ignored, so the test only errs
// towards keeping a cell), and with adaptive targets (aflag set) for cells
// that are no target.
__global__ void k_class_keys(const uint64_t *ckey, const int *cpbeg, const int *cpend, const int *cparent,
                             const int *ccoll, const int *cchild, long long direct_max, int first, int count, int level,
                             int dim, uint64_t *keys_all, uint64_t *keys_m2l, uint32_t *vals, int out_off,
                             const uint8_t *aflag, int cell0) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  int g = first + i;
  const uint64_t k = ((uint64_t)level << dim) | (ckey[g] & ((1u << dim) - 1));
  keys_all[out_off + i] = k;
  vals[out_off + i] = (uint32_t)g;
  bool m2l = !aflag || (aflag[g - cell0] & 1);  // with adaptive targets only targets (and their rows) count
  if (m2l && direct_max > 0) {
    const int nc = 1 << dim, ns = dim == 3 ? 27 : 9;
    const long long nt = cpend[g] - cpbeg[g];
    const int *pc = ccoll + (int64_t)cparent[g] * ns;
    m2l = false;
    for (int s = 0; s < ns && !m2l; ++s) {
      const int Q = pc[s];
      if (Q < 0 || nt * (cpend[Q] - cpbeg[Q]) <= direct_max) continue;
      for (int c = 0; c < nc && !m2l; ++c) {
        const int q = cchild[(int64_t)Q * nc + c];
        if (q >= 0 && nt * (cpend[q] - cpbeg[q]) > direct_max) m2l = true;
      }
    }
  }
  keys_m2l[out_off + i] = m2l ? k : 255u;
}

__global__ void k_class_hist(const uint64_t *keys, int n, uint32_t *hist) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    atomicAdd(&h[keys[i] & 255u], 1u);
  __syncthreads();
  if (h[threadIdx.x]) atomicAdd(&hist[threadIdx.x], h[threadIdx.x]);
}

// ------------------------------------------------------------ M shortcut
// Multipoles are formed only for the cells M2L reads (its sources) and for
// its targets (their spectrum is a feature of the learned orders), plus what
// M2M needs to form those.  A needed cell with at most P2M_DIRECT_MAX
// particles, or a leaf, takes its multipole straight from its particles
// (mode 1); a larger one sums its children by M2M (mode 2), which makes all
// of them needed.  mode 0: not formed.
static constexpr int P2M_DIRECT_MAX = 64;

__global__ void k_m_mode(const uint8_t *lact, const uint8_t *msrc, int first2, int leaf_first, int count,
                         const int *parent, const int *pbeg, const int *pend, int cell0, int tmax, uint8_t *mode,
                         int *list1, unsigned *count1) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, lane = threadIdx.x & 31;
  const int c = first2 + i;
  int md = 0;
  if (i < count) {
    int a = c;
    bool req = lact[a - cell0] || msrc[a - cell0];
    while (!req) {  // needed through a chain of M2M ancestors
      const int P = parent[a];
      if (P < first2 || pend[P] - pbeg[P] <= tmax) break;
      a = P;
      req = lact[a - cell0] || msrc[a - cell0];
    }
    md = !req ? 0 : (c >= leaf_first || pend[c] - pbeg[c] <= tmax) ? 1 : 2;
    mode[c - cell0] = (uint8_t)md;
  }
  // the mode-1 cells, appended a warp at a time (ascending within a warp)
  const unsigned m1 = __ballot_sync(0xffffffffu, md == 1);
  if (m1) {
    unsigned at = 0;
    if (lane == 0) at = atomicAdd(count1, (unsigned)__popc(m1));
    at = __shfl_sync(0xffffffffu, at, 0);
    if (md == 1) list1[at + __popc(m1 & ((1u << lane) - 1u))] = c;
  }
}

// Zeroes the rows (KS floats, KS a multiple of 4) of X of the cells
// [first, first + count) with fx[c] == wx, and those of Y with fy[c] == wy:
// a warp reads the flags of 32 cells at once and stores each flagged row
// with all its lanes.
__global__ void k_zero_rows(const uint8_t *fx, uint8_t wx, float *X, const uint8_t *fy, uint8_t wy, float *Y,
                            int first, int count, int cell0, int KS) {
  const int lane = threadIdx.x & 31;
  const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i0 = w0 * 32; i0 < count; i0 += nw * 32) {
    const int64_t i = i0 + lane;
    const int c = first + (int)i;
    const bool in = i < count;
    unsigned mx = __ballot_sync(0xffffffffu, in && fx[c - cell0] == wx);
    unsigned my = __ballot_sync(0xffffffffu, in && fy[c - cell0] == wy);
    while (mx | my) {
      const bool isx = mx != 0;
      unsigned &m = isx ? mx : my;
      const int b = __ffs(m) - 1;
      m &= m - 1;
      float4 *row = reinterpret_cast<float4 *>((isx ? X : Y) + (size_t)(first + (int)i0 + b - cell0) * KS);
      for (int q = lane; q < (KS >> 2); q += 32) row[q] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
}

// Sort keys of the M2M rows of one level: with child_rows (tensor-core
// M2M, rows are children) the children of mode-2 cells by (level, class),
// else (CUDA-core M2M, rows are parents) the mode-2 cells by (level, 0);
// 255 for the rest.
__global__ void k_m2m_keys(const uint64_t *ckey, const uint8_t *mode, const int *parent, int first, int count,
                           int level, int dim, int cell0, int child_rows, uint64_t *keys, uint32_t *vals, int out_off) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int g = first + i;
  const bool on = child_rows ? mode[parent[g] - cell0] == 2 : mode[g - cell0] == 2;
  const uint64_t cls = child_rows ? (ckey[g] & ((1u << dim) - 1)) : 0u;
  keys[out_off + i] = on ? (((uint64_t)level << dim) | cls) : 255u;
  vals[out_off + i] = (uint32_t)g;
}

struct P2MListArgs {
  int nlev;                          // levels 2 .. nlev + 1
  int first[DF_MAX_LEVELS + 1];      // first cell of each level; first[nlev]: end
  const float4 *off[DF_MAX_LEVELS];  // particle offsets from the level's cell centres, mass in w
  float inv_s[DF_MAX_LEVELS];        // 2^level / emax
  const int *pbeg, *pend;
  const int *list;                   // the mode-1 cells
  const unsigned *count;             // their number
  int cell0, p, K, KS;
  int rs;                            // shared-memory row stride: K rounded up to odd
  float *M;
};
static constexpr int P2M_WARPS = 5, P2M_KC = (FMM_MAX_P * FMM_MAX_P + 2 * FMM_MAX_P + 4 + 31) / 32;

// One particle's contributions w R~_l^m (real parts, then -imaginary parts
// as the layout stores them) into a shared-memory row.
template <int P>
__device__ inline void p2m_row(float x, float y, float z, float w, int p, float *row) {
  if (P) p = P;
  const float r2 = x * x + y * y + z * z;
  float dre = 1.f, dim_ = 0.f;
#pragma unroll
  for (int m = 0; m <= p; ++m) {
    if (m > 0) {
      const float h = -0.5f / m;
      const float nre = h * (x * dre - y * dim_), nim = h * (x * dim_ + y * dre);
      dre = nre;
      dim_ = nim;
    }
    float p1re = dre, p1im = dim_, p2re = 0.f, p2im = 0.f;
#pragma unroll
    for (int l = m; l <= p; ++l) {
      float cre, cim;
      if (l == m) {
        cre = dre;
        cim = dim_;
      } else {
        const float a1 = c_rec1[l][m] * z, a2 = c_rec2[l][m] * r2;
        cre = a1 * p1re - a2 * p2re;
        cim = a1 * p1im - a2 * p2im;
        p2re = p1re;
        p2im = p1im;
        p1re = cre;
        p1im = cim;
      }
      row[re_idx(l, m)] = w * cre;
      if (m > 0) row[im_idx(l, m)] = -w * cim;
    }
  }
}

// P2M of the mode-1 cells (their own particles at their own level, no M2M).
// Persistent warps take the list 32 (8 or 16 for short lists) cells at a
// time.  Consecutive cells of at most 32 particles share 32-particle chunks;
// a larger cell takes chunks of its own with a running sum.  In a chunk each
// lane writes the contributions of one particle as a row of a shared-memory
// tile (odd stride: conflict-free), then the lanes sum each cell's rows
// column by column, in particle order, and store the cell's row once,
// padding columns zero (no atomics, no reductions across lanes).  PO > 0:
// the order as a compile-time constant (PO == a.p, the row loops unrolled);
// PO = 0: any order.
template <int PO>
__global__ void __launch_bounds__(32 * P2M_WARPS) k_p2m_list(P2MListArgs a) {
  extern __shared__ float s_tile[];
  // locals, not writes into a (which would copy the parameter block to local memory)
  const int ord = PO ? PO : a.p, K = PO ? (PO + 1) * (PO + 1) : a.K;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  float *S = s_tile + (size_t)wib * 32 * a.rs;
  const unsigned total = *a.count;
  // cells per group: 32, or fewer when the list is short, so that the warps
  // share the work evenly
  const unsigned nw = (unsigned)gridDim.x * P2M_WARPS;
  const unsigned G = total >= nw * 128u ? 32u : total >= nw * 32u ? 16u : 8u;
  for (unsigned g0 = ((unsigned)blockIdx.x * P2M_WARPS + wib) * G; g0 < total; g0 += nw * G) {
    const int gcount = (int)min(G, total - g0);
    const bool has = lane < gcount;
    const int c = has ? a.list[g0 + lane] : 0;
    int pb = 0, n = 0, lv = 0;
    if (has) {
      pb = a.pbeg[c];
      n = a.pend[c] - pb;
      while (lv + 1 < a.nlev && c >= a.first[lv + 1]) ++lv;
    }
    // inclusive prefix of the sizes of the cells of at most 32 particles
    int P = has && n <= 32 ? n : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, P, o);
      if (lane >= o) P += y;
    }
    const unsigned bigmask = __ballot_sync(0xffffffffu, has && n > 32);
    int j = 0;
    while (j < gcount) {  // warp-uniform
      const int nj = __shfl_sync(0xffffffffu, n, j);
      if (nj > 32) {  // a large cell: chunks of 32 with a running sum
        const int cb = __shfl_sync(0xffffffffu, c, j), pbj = __shfl_sync(0xffffffffu, pb, j);
        const int lvj = __shfl_sync(0xffffffffu, lv, j);
        const float4 *off = a.off[lvj];
        const float inv_s = a.inv_s[lvj];
        float acc[P2M_KC];
#pragma unroll
        for (int t = 0; t < P2M_KC; ++t) acc[t] = 0.f;
        for (int e0 = 0; e0 < nj; e0 += 32) {
          const int cnt = min(32, nj - e0);
          const float4 q = lane < cnt ? off[pbj + e0 + lane] : make_float4(0.f, 0.f, 0.f, 0.f);
          p2m_row<PO>(q.x * inv_s, q.y * inv_s, q.z * inv_s, q.w, ord, S + lane * a.rs);
          __syncwarp();
#pragma unroll
          for (int t = 0; t < P2M_KC; ++t) {
            const int col = lane + 32 * t;
            if (col < K)
              for (int r = 0; r < cnt; ++r) acc[t] += S[r * a.rs + col];
          }
          __syncwarp();
        }
        float *mrow = a.M + (size_t)(cb - a.cell0) * a.KS;
#pragma unroll
        for (int t = 0; t < P2M_KC; ++t) {
          const int col = lane + 32 * t;
          if (col < a.KS) mrow[col] = col < K ? acc[t] : 0.f;
        }
        ++j;
        continue;
      }
      // a chunk of consecutive small cells j .. j1 (up to the next large cell)
      const int start = j > 0 ? __shfl_sync(0xffffffffu, P, j - 1) : 0;
      const unsigned after = bigmask & ~(0xffffffffu >> (31 - j));  // large cells after j
      const int jb = after ? __ffs(after) - 1 : gcount;
      const unsigned fit = __ballot_sync(0xffffffffu, lane >= j && lane < jb && P - start <= 32);
      const int j1 = 31 - __clz(fit);
      const int used = __shfl_sync(0xffffffffu, P, j1) - start;
      const int rel = lane >= j && lane <= j1 ? P - n - start : 32;  // each cell's first row
      const unsigned starts = __reduce_or_sync(0xffffffffu, rel < 32 ? 1u << rel : 0u);
      const int myk = j + __popc(starts & (0xffffffffu >> (31 - lane))) - 1;
      const int s0 = __shfl_sync(0xffffffffu, P - n, myk) - start;
      const int mpb = __shfl_sync(0xffffffffu, pb, myk), mlv = __shfl_sync(0xffffffffu, lv, myk);
      const float4 q = lane < used ? a.off[mlv][mpb + lane - s0] : make_float4(0.f, 0.f, 0.f, 0.f);
      const float inv_s = a.inv_s[mlv];
      p2m_row<PO>(q.x * inv_s, q.y * inv_s, q.z * inv_s, q.w, ord, S + lane * a.rs);
      __syncwarp();
      for (int k = j; k <= j1; ++k) {
        const int r0 = __shfl_sync(0xffffffffu, P - n, k) - start, nk = __shfl_sync(0xffffffffu, n, k);
        const int ck = __shfl_sync(0xffffffffu, c, k);
        float *mrow = a.M + (size_t)(ck - a.cell0) * a.KS;
        for (int col = lane; col < a.KS; col += 32) {
          float v = 0.f;
          if (col < K)
            for (int r = r0; r < r0 + nk; ++r) v += S[r * a.rs + col];
          mrow[col] = v;
        }
      }
      __syncwarp();
      j = j1 + 1;
    }
  }
}

// Launches k_p2m_list<P> with its dynamic shared memory (32 rows of rs
// floats per warp), raising the instantiation's limit once per device.
template <int P>
static int launch_p2m_list(const P2MListArgs &pm, cudaStream_t st) {
  const size_t psh = sizeof(float) * (size_t)P2M_WARPS * 32 * pm.rs;
  {
    static std::mutex mu;
    static size_t attr[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return FMM_ERR_CUDA;
    std::lock_guard<std::mutex> lk(mu);
    if (attr[dev] < psh) {
      CUDA_TRY(cudaFuncSetAttribute(k_p2m_list<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psh));
      CUDA_TRY(cudaFuncSetAttribute(k_p2m_list<P>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                    cudaSharedmemCarveoutMaxShared));
      attr[dev] = psh;
    }
  }
  k_p2m_list<P><<<148 * 2, 32 * P2M_WARPS, psh, st>>>(pm);
  return FMM_OK;
}

// ------------------------------------------------------------ L2L shortcut
// Marks every ancestor-or-self at levels >= 2 of the cells with M2L
// contributions (lact): the cells whose local expansion is needed below.
__global__ void k_needs_l(const uint8_t *lact, int first2, int count, const int *parent, int cell0, uint8_t *needs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  int c = first2 + i;
  if (!lact[c - cell0]) return;
  while (c >= first2 && !needs[c - cell0]) {  // stops where another walk already passed
    needs[c - cell0] = 1;
    c = parent[c];
  }
}

// Per leaf: its deepest ancestor-or-self with a needed local expansion.
__global__ void k_leaf_esrc(int leaf_first, int nleaves, int D, int first2, const int *parent, const uint8_t *needs,
                            int cell0, int *esrc, uint8_t *elev) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nleaves) return;
  int c = leaf_first + i, lev = D;
  while (c >= first2 && !needs[c - cell0]) {
    c = parent[c];
    --lev;
  }
  esrc[i] = c >= first2 ? c : -1;
  elev[i] = (uint8_t)(c >= first2 ? lev : 0);
}

// Sort keys of the cells of one level that need L2L: (level, class), else 255.
__global__ void k_l2l_keys(const uint64_t *ckey, const uint8_t *needs, int first, int count, int level, int dim,
                           int cell0, uint64_t *keys, uint32_t *vals, int out_off) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int g = first + i;
  keys[out_off + i] = needs[g - cell0] ? (((uint64_t)level << dim) | (ckey[g] & ((1u << dim) - 1))) : 255u;
  vals[out_off + i] = (uint32_t)g;
}

// ------------------------------------------------------------ separation
// Offset o = (dx+3) + 7(dy+3) + 49(dz+3) (cells of the box with extents ex):
// the two cells' radii summed over the distance of their centres exceeds
// FMM_RHO_MAX, so their multipole expansion may not converge.
__host__ __device__ inline bool offset_not_well_separated(int o, int dim, double ex, double ey, double ez) {
  if (dim == 2 && o >= 49) return false;  // 2D offsets: (dx+3) + 7(dy+3)
  const int dx = o % 7 - 3, dy = (o / 7) % 7 - 3, dz = dim == 3 ? o / 49 - 3 : 0;
  const double diag2 = ex * ex + ey * ey + (dim == 3 ? ez * ez : 0.0);
  const double dist2 = dx * ex * dx * ex + dy * ey * dy * ey + (dim == 3 ? dz * ez * dz * ez : 0.0);
  return dist2 > 0.0 && sqrt(diag2) > FMM_RHO_MAX * sqrt(dist2);
}

__global__ void k_fdirect_table(int dim, double ex, double ey, double ez, uint8_t *out) {
  const int o = threadIdx.x;
  if (o < 343) out[o] = offset_not_well_separated(o, dim, ex, ey, ez) ? 1 : 0;
}

// ------------------------------------------------------------ pair orders
// FMM_ORDER_GEOMETRIC: for every M2L operator slot (offset D of source from
// target, in cell sizes), the order whose truncation bound rho^(q+1),
// rho = (sum of the two cells' radii) / |D|, matches the closest offset's at
// order p, plus `margin`, clamped to [min(4, p), p]; stored as the padded
// width of that order's expansion length.
__global__ void k_order_table(int dim, int p, int margin, int n_slots, int per_level, float ax, float ay, float az,
                              uint8_t *out) {
  __shared__ float s_ref;
  const float diag = sqrtf(ax * ax + ay * ay + (dim == 3 ? az * az : 0.f));  // radius sum of two cells
  if (threadIdx.x == 0) {
    float ref = 0.f;
    for (int t = 0; t < per_level; ++t) {
      const int dx = t % 7 - 3, dy = (t / 7) % 7 - 3, dz = dim == 3 ? t / 49 - 3 : 0;
      if (max(abs(dx), max(abs(dy), abs(dz))) < 2) continue;  // neighbours never interact by M2L
      const float R = sqrtf(dx * dx * ax * ax + dy * dy * ay * ay + dz * dz * az * az);
      ref = fmaxf(ref, diag / R);
    }
    s_ref = ref;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < n_slots; t += blockDim.x) {
    const int o = t % per_level;
    const int dx = o % 7 - 3, dy = (o / 7) % 7 - 3, dz = dim == 3 ? o / 49 - 3 : 0;
    const float R = sqrtf(dx * dx * ax * ax + dy * dy * ay * ay + dz * dz * az * az);
    const float rho = R > 0.f ? diag / R : 1.f;
    int q = p;
    if (rho < 1.f && s_ref < 1.f && max(abs(dx), max(abs(dy), abs(dz))) >= 2) {
      q = (int)ceilf((p + 1) * logf(s_ref) / logf(rho)) - 1 + margin;
      q = max(min(q, p), min(4, p));
    }
    const int K = dim == 3 ? (q + 1) * (q + 1) : 2 * q + 1;
    out[t] = (uint8_t)((K + 15) & ~15);
  }
}

// Adaptive targets of one level for the direct far field: the cells with
// flag bit 0 that can have direct pairs, appended to seg (warp-aggregated;
// their order within the level is free), their count in *cnt.
__global__ void k_level_targets(const uint8_t *aflag, int cell0, int first, int count, const int *pbeg,
                                const int *pend, long long direct_max, int any_fdirect, int *seg, unsigned *cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, lane = threadIdx.x & 31;
  const int g = first + i;
  const bool tgt = i < count && (aflag[g - cell0] & 1) &&
                   ((long long)(pend[g] - pbeg[g]) <= direct_max || any_fdirect);
  const unsigned m = __ballot_sync(0xffffffffu, tgt);
  unsigned base = 0;
  if (lane == 0 && m) base = atomicAdd(cnt, (unsigned)__popc(m));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (tgt) seg[base + __popc(m & ((1u << lane) - 1u))] = g;
}

// FP64 positions in leaf order: xs[i] = pos[perm[i]].
__global__ void k_gather_pos(const double *pos, const uint32_t *perm, int64_t n, int dim, double *xs) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const size_t o = (size_t)perm[i] * dim;
  for (int k = 0; k < dim; ++k) xs[(size_t)i * dim + k] = pos[o + k];
}

// ------------------------------------------------------------ driver

int run_fmm_passes(Workspace &ws, TreeState &t, OpTables &ops, ExpBuffers &eb, const double *d_pos_g,
                   const double *d_mass_g, int p, double eps2, double G,
                   const PassGeom &g, double *d_acc, double *d_pot, int m2l_mode, int64_t direct_max,
                   const OrderOpts &order, cudaStream_t st, fmm_stats &stats, cudaEvent_t *ev,
                   int adaptive_leaf, int p2p_chunk, int m2l_run) {
  const int dim = t.dim, D = t.depth, KS = ops.KS;
  const int64_t n = t.n;
  const bool want_pot = d_pot != nullptr;  // the potential is summed only when it is asked for
  const int ncell = t.n_cells, cell0 = t.cell0;
  const int TPB = 256;
  if (!eb.M.reserve((size_t)ncell * KS) || !eb.L.reserve((size_t)ncell * KS)) return FMM_ERR_OUT_OF_MEMORY;
  // 3D shortcuts: local expansions only on paths to cells with M2L
  // contributions (L2P from each leaf's deepest such ancestor), multipoles
  // only for what M2L reads (P2M straight into small cells, M2M above them);
  // only the rows that are summed into start at zero
  if (!(t.dim == 3 && D >= 3)) {
    CUDA_TRY(cudaMemsetAsync(eb.M.ptr, 0, sizeof(float) * (size_t)ncell * KS, st));
    CUDA_TRY(cudaMemsetAsync(eb.L.ptr, 0, sizeof(float) * (size_t)ncell * KS, st));
  }
  // tensor-core translations: 128-target batches, BF16 split operator images
  const int P16 = (ops.K + 15) & ~15;
  const bool tc = m2l_mode == FMM_M2L_TC && P16 <= TC_MAX_P16;
  const int tchunk = tc ? 128 : CT_TGT;
  int tc_k = 0;  // tensor-core launches so far (work counter index)
  if (tc && D >= 2) {
    if (!eb.tc_img.reserve((size_t)ops.n_slots * 3 * P16 * P16) || !eb.tc_work.reserve(TC_MAX_LAUNCHES))
      return FMM_ERR_OUT_OF_MEMORY;
    if (2 * D + 2 > TC_MAX_LAUNCHES) return FMM_ERR_UNSUPPORTED;
    CUDA_TRY(cudaMemsetAsync(eb.tc_work.ptr, 0, TC_MAX_LAUNCHES * sizeof(unsigned int), st));
    int rc = tc_build_images(ops.tab.ptr, ops.n_slots, ops.K, ops.KP, P16, eb.tc_img.ptr, st, ws.launches);
    if (rc) return rc;
  }
  const double emax = g.emax > 0 ? g.emax : 1.0;
  const double sD = std::ldexp(emax, -D);
  // offsets whose cells are not well separated for this box (summed
  // directly): flags on the device, and on the host whether there are any
  // (the same FP64 arithmetic, IEEE square roots, so both agree)
  int any_fdirect = 0;
  for (int o = 0; o < 343; ++o)
    if (offset_not_well_separated(o, dim, g.ext[0], g.ext[1], g.ext[2])) {
      const int dd[3] = {o % 7 - 3, (o / 7) % 7 - 3, dim == 3 ? o / 49 - 3 : 0};
      if (std::abs(dd[0]) > 1 || std::abs(dd[1]) > 1 || std::abs(dd[2]) > 1) any_fdirect = 1;
    }
  if (!eb.fdirect.reserve(343)) return FMM_ERR_OUT_OF_MEMORY;
  k_fdirect_table<<<1, 352, 0, st>>>(dim, g.ext[0], g.ext[1], g.ext[2], eb.fdirect.ptr);
  ws.launches += 1;
  const float inv_sD = (float)(1.0 / sD);

  // class-grouped target lists of levels >= 2: the cells with possible M2L
  // pairs (for M2L) and, without the shortcuts (which build their own lists
  // below), every cell (for M2M and L2L) and consecutive M2M parents
  const bool shortcut = dim == 3 && D >= 3;
  // adaptive targets (3D shortcut pass only): flags and the adaptive leaves
  const bool adaptive = shortcut && adaptive_leaf > 0;
  if (adaptive && t.adaptive_leaf != adaptive_leaf) {  // not computed with the tree
    if (!ws.reserve_adaptive(ncell)) return FMM_ERR_OUT_OF_MEMORY;
    int rc = launch_adaptive_flags(ws, t, adaptive_leaf, ws.aflag, ws.alist, st);
    if (rc) return rc;
    ws.launches += 1;
  }
  std::vector<int> lvl_b0(D + 2, 0), lvl_b1(D + 2, 0), m2l_b0(D + 2, 0), m2l_b1(D + 2, 0);
  std::vector<int> m2m_b0(D + 1, 0), m2m_b1(D + 1, 0);
  int ntl = 0;
  const int *tl = nullptr, *tl_m2l = nullptr;
  size_t nhb = 0;
  if (D >= 2) {
    ntl = t.level_off[D] + t.level_count[D] - t.level_off[2];
    if (!eb.tlist.reserve(ntl) || !eb.tlist_m2l.reserve(ntl) || !eb.cls_count.reserve(512) ||
        !eb.ckey.reserve(ntl) || !eb.ckey_alt.reserve(ntl) || !eb.ckey_m2l.reserve(ntl) || !eb.cval.reserve(ntl) ||
        !eb.cval2.reserve(ntl))
      return FMM_ERR_OUT_OF_MEMORY;
    for (int d = 2; d <= D; ++d)
      k_class_keys<<<cdiv(t.level_count[d], TPB), TPB, 0, st>>>(
          ws.cell_key, ws.cell_pbeg, ws.cell_pend, ws.cell_parent, ws.cell_coll, ws.cell_child, direct_max,
          t.level_off[d], t.level_count[d], d, dim, eb.ckey.ptr, eb.ckey_m2l.ptr, eb.cval.ptr,
          t.level_off[d] - t.level_off[2], adaptive ? ws.aflag : nullptr, cell0);
    ws.launches += D - 1;
    CUDA_TRY(cudaMemsetAsync(eb.cls_count.ptr, 0, 512 * sizeof(uint32_t), st));
    uint64_t *kk = eb.ckey.ptr, *kk2 = eb.ckey_alt.ptr;
    uint32_t *mv = eb.cval.ptr, *mv2 = (uint32_t *)eb.tlist_m2l.ptr;
    if (!shortcut) {
      CUDA_TRY(cudaMemcpyAsync(eb.cval2.ptr, eb.cval.ptr, sizeof(uint32_t) * ntl, cudaMemcpyDeviceToDevice, st));
      uint32_t *vv = eb.cval.ptr, *vv2 = (uint32_t *)eb.tlist.ptr;
      radix_sort(ws, kk, vv, kk2, vv2, ntl, 8, st);  // sorted (keys, cells) end in (kk, vv)
      tl = (const int *)vv;
      k_class_hist<<<std::min(cdiv(ntl, TPB), 148 * 4), TPB, 0, st>>>(kk, ntl, eb.cls_count.ptr);
      ws.launches += 1;
      mv = eb.cval2.ptr;
    }
    uint64_t *mk = eb.ckey_m2l.ptr, *mk2 = (kk == eb.ckey.ptr) ? eb.ckey_alt.ptr : eb.ckey.ptr;
    radix_sort(ws, mk, mv, mk2, mv2, ntl, 8, st);
    tl_m2l = (const int *)mv;
    k_class_hist<<<std::min(cdiv(ntl, TPB), 148 * 4), TPB, 0, st>>>(mk, ntl, eb.cls_count.ptr + 256);
    ws.launches += 1;
    uint32_t hc[512];
    CUDA_TRY(cudaMemcpyAsync(hc, eb.cls_count.ptr, sizeof(hc), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    const int ncls = 1 << dim;
    // batch count, then the table written straight into pinned staging
    size_t cnt_b = 0;
    for (int pass = shortcut ? 1 : 0; pass < 2; ++pass)
      for (int d = 2; d <= D; ++d)
        for (int c = 0; c < ncls; ++c) cnt_b += ((size_t)hc[256 * pass + ((d << dim) | c)] + tchunk - 1) / tchunk;
    if (!shortcut)
      for (int d = D - 1; d >= 2; --d) cnt_b += ((size_t)t.level_count[d] + tchunk - 1) / tchunk;
    if (!eb.hbatches.reserve(cnt_b + 1, st)) return FMM_ERR_OUT_OF_MEMORY;
    int4 *hb = eb.hbatches.ptr;
    for (int pass = shortcut ? 1 : 0; pass < 2; ++pass) {
      const uint32_t *h = hc + 256 * pass;
      int off = 0;
      for (int d = 2; d <= D; ++d) {
        (pass ? m2l_b0 : lvl_b0)[d] = (int)nhb;
        for (int c = 0; c < ncls; ++c) {
          const int cnt = (int)h[(d << dim) | c];
          for (int s0 = 0; s0 < cnt; s0 += tchunk) hb[nhb++] = make_int4(off + s0, std::min(tchunk, cnt - s0), d, c);
          off += cnt;
        }
        (pass ? m2l_b1 : lvl_b1)[d] = (int)nhb;
      }
    }
    // M2M batches (levels D-1 .. 2, consecutive cells)
    for (int d = D - 1; d >= 2 && !shortcut; --d) {
      m2m_b0[d] = (int)nhb;
      for (int s = 0; s < t.level_count[d]; s += tchunk)
        hb[nhb++] = make_int4(t.level_off[d] + s, std::min(tchunk, t.level_count[d] - s), d, -1);
      m2m_b1[d] = (int)nhb;
    }
  }
  if (!eb.batches.reserve(nhb + 1)) return FMM_ERR_OUT_OF_MEMORY;
  if (nhb)
    CUDA_TRY(cudaMemcpyAsync(eb.batches.ptr, eb.hbatches.ptr, nhb * sizeof(int4), cudaMemcpyHostToDevice, st));

  ContractArgs ca;
  ca.batches = eb.batches.ptr;
  ca.tlist = nullptr;
  ca.tab = ops.tab.ptr;
  ca.cparent = ws.cell_parent;
  ca.cchild = ws.cell_child;
  ca.ccoll = ws.cell_coll;
  ca.cpbeg = ws.cell_pbeg;
  ca.cpend = ws.cell_pend;
  ca.direct_max = direct_max;
  ca.fdirect = any_fdirect ? eb.fdirect.ptr : nullptr;
  ca.src_tab = nullptr;
  ca.slot_list = nullptr;
  ca.nslots_tab = nullptr;
  ca.cell0 = cell0;
  ca.K = ops.K;
  ca.KS = KS;
  ca.KP = ops.KP;
  ca.dim = dim;
  ca.level_stride = dim == 2 ? 49 : 0;
  ca.pair_count = ws.counters;
  CUDA_TRY(cudaMemsetAsync(ws.counters, 0, 8 * sizeof(unsigned long long), st));
  TcArgs ta{};
  ta.cchild = ws.cell_child;
  ta.cparent = ws.cell_parent;
  ta.nchild = 1 << dim;
  ta.bimg = eb.tc_img.ptr;
  ta.cell0 = cell0;
  ta.K = ops.K;
  ta.KS = KS;
  ta.P16 = P16;
  ta.err = ws.dev_err;
  ta.run_slots = m2l_run;

  uint8_t *lact = nullptr, *needs = nullptr, *msrc = nullptr, *mmode = nullptr;
  if (shortcut) {
    if (!eb.lact.reserve(4 * (size_t)ncell)) return FMM_ERR_OUT_OF_MEMORY;
    CUDA_TRY(cudaMemsetAsync(eb.lact.ptr, 0, 4 * (size_t)ncell, st));
    lact = eb.lact.ptr;
    needs = lact + ncell;
    msrc = lact + 2 * (size_t)ncell;
    mmode = lact + 3 * (size_t)ncell;
  }
  // M2L plan, all levels: the source of every (slot, target) of each batch
  // and, with variable orders, the geometric widths
  ContractArgs cm = ca;
  cm.mode = MODE_M2L;
  cm.slot_base = 0;
  cm.tlist = tl_m2l;
  cm.X = eb.M.ptr;
  cm.Y = eb.L.ptr;
  cm.batches = eb.batches.ptr + m2l_b0[2];
  const int nbm = D >= 2 ? m2l_b1[D] - m2l_b0[2] : 0;
  const bool geometric = tc && order.mode == FMM_ORDER_GEOMETRIC;
  const bool learned = tc && dim == 3 && order.mode == FMM_ORDER_LEARNED && order.params;
  const bool collect = tc && dim == 3 && order.ntiles > 0 && ops.tab64.ptr;
  const bool var_order = geometric || learned;
  const float ax = (float)(g.ext[0] / emax), ay = (float)(g.ext[1] / emax),
              az = (float)(dim == 3 ? g.ext[2] / emax : 0.0);
  if (D >= 2) {
    if (!eb.m2l_src.reserve((size_t)nbm * 189 * tchunk) || !eb.m2l_list.reserve((size_t)nbm * 189) ||
        !eb.m2l_nslots.reserve(nbm) || !eb.m2l_tslot.reserve((size_t)nbm * 189))
      return FMM_ERR_OUT_OF_MEMORY;
    if (var_order && !eb.m2l_w.reserve((size_t)nbm * 189)) return FMM_ERR_OUT_OF_MEMORY;
    if (geometric) {
      if (!eb.order_p16.reserve(ops.n_m2l)) return FMM_ERR_OUT_OF_MEMORY;
      k_order_table<<<1, 256, 0, st>>>(dim, p, order.margin, ops.n_m2l, dim == 3 ? 343 : 49, ax, ay, az,
                                       eb.order_p16.ptr);
      ws.launches += 1;
    }
    if (nbm > 0) {
      k_m2l_sources<<<nbm, 256, 0, st>>>(cm, tchunk, eb.m2l_src.ptr, eb.m2l_list.ptr, eb.m2l_nslots.ptr,
                                         tc ? eb.m2l_tslot.ptr : nullptr, tc ? ws.counters : nullptr,
                                         geometric ? eb.order_p16.ptr : nullptr, geometric ? eb.m2l_w.ptr : nullptr,
                                         ws.counters + 4, lact, msrc, cell0);
      ws.launches += 1;
    }
  }
  // particle offsets from their ancestors' centres, levels 2..D-1 (P2M and
  // L2P shortcuts, direct far field)
  const bool need_lvl_off = D > 2 && (shortcut || direct_max > 0 || any_fdirect);
  if (need_lvl_off) {
    if (!eb.lvl_off.reserve((size_t)n * (D - 2))) return FMM_ERR_OUT_OF_MEMORY;
    auto lo_kern = dim == 3 ? k_level_offsets<3> : k_level_offsets<2>;
    lo_kern<<<cdiv(n, TPB), TPB, 0, st>>>(d_pos_g, d_mass_g, t.d_perm, ws.leaf_of, ws.cell_key, n, D, 2, D - 1,
                                          g.lo[0], g.lo[1], g.lo[2], g.ext[0], g.ext[1], g.ext[2], eb.lvl_off.ptr);
    ws.launches += 1;
  }
  // shortcut lists: the cells that need L2L and the M2M rows, each grouped
  // by (level, class), from one histogram read-back
  const int *tl2 = tl, *tlm = nullptr;
  const int4 *b2 = eb.batches.ptr;
  std::vector<int> l2_b0(lvl_b0), l2_b1(lvl_b1), um_b0(D + 2, 0), um_b1(D + 2, 0);
  if (shortcut) {
    const int first2 = t.level_off[2], leaf_first = t.level_off[D];
    k_needs_l<<<cdiv(ntl, TPB), TPB, 0, st>>>(lact, first2, ntl, ws.cell_parent, cell0, needs);
    if (!eb.p2m_list.reserve((size_t)ntl + 1)) return FMM_ERR_OUT_OF_MEMORY;
    CUDA_TRY(cudaMemsetAsync(eb.p2m_list.ptr + ntl, 0, sizeof(int), st));
    k_m_mode<<<cdiv(ntl, TPB), TPB, 0, st>>>(lact, msrc, first2, leaf_first, ntl, ws.cell_parent, ws.cell_pbeg,
                                             ws.cell_pend, cell0, P2M_DIRECT_MAX, mmode, eb.p2m_list.ptr,
                                             reinterpret_cast<unsigned *>(eb.p2m_list.ptr + ntl));
    ws.launches += 2;
    // L2L rows: levels 3..D; M2M rows: children at levels 3..D (tensor
    // cores) or the mode-2 parents at levels 2..D-1
    const int l3 = t.level_off[3], nl3 = t.level_off[D] + t.level_count[D] - l3;
    const int m_lo = tc ? 3 : 2, m_hi = tc ? D : D - 1;
    const int m_first = t.level_off[m_lo], nm = t.level_off[m_hi] + t.level_count[m_hi] - m_first;
    if (!eb.ukey.reserve(4 * (size_t)ntl) || !eb.uval.reserve(4 * (size_t)ntl)) return FMM_ERR_OUT_OF_MEMORY;
    for (int d = 3; d <= D; ++d)
      k_l2l_keys<<<cdiv(t.level_count[d], TPB), TPB, 0, st>>>(ws.cell_key, needs, t.level_off[d], t.level_count[d], d,
                                                              dim, cell0, eb.ukey.ptr, eb.uval.ptr, t.level_off[d] - l3);
    for (int d = m_lo; d <= m_hi; ++d)
      k_m2m_keys<<<cdiv(t.level_count[d], TPB), TPB, 0, st>>>(ws.cell_key, mmode, ws.cell_parent, t.level_off[d],
                                                              t.level_count[d], d, dim, cell0, tc ? 1 : 0,
                                                              eb.ukey.ptr + 2 * (size_t)ntl,
                                                              eb.uval.ptr + 2 * (size_t)ntl, t.level_off[d] - m_first);
    ws.launches += (D - 2) + (m_hi - m_lo + 1);
    uint64_t *kk = eb.ukey.ptr, *kk2 = eb.ukey.ptr + ntl;
    uint32_t *vv = eb.uval.ptr, *vv2 = eb.uval.ptr + ntl;
    radix_sort(ws, kk, vv, kk2, vv2, nl3, 8, st);
    uint64_t *mk = eb.ukey.ptr + 2 * (size_t)ntl, *mk2 = eb.ukey.ptr + 3 * (size_t)ntl;
    uint32_t *mv = eb.uval.ptr + 2 * (size_t)ntl, *mv2 = eb.uval.ptr + 3 * (size_t)ntl;
    radix_sort(ws, mk, mv, mk2, mv2, nm, 8, st);
    CUDA_TRY(cudaMemsetAsync(eb.cls_count.ptr, 0, 512 * sizeof(uint32_t), st));
    k_class_hist<<<std::max(1, std::min(cdiv(nl3, TPB), 148 * 4)), TPB, 0, st>>>(kk, nl3, eb.cls_count.ptr);
    k_class_hist<<<std::max(1, std::min(cdiv(nm, TPB), 148 * 4)), TPB, 0, st>>>(mk, nm, eb.cls_count.ptr + 256);
    ws.launches += 2;
    uint32_t hc[512];
    CUDA_TRY(cudaMemcpyAsync(hc, eb.cls_count.ptr, sizeof(hc), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    const int ncls = 1 << dim;
    size_t cnt_b = 0, nb2 = 0;
    for (int d = 3; d <= D; ++d)
      for (int c = 0; c < ncls; ++c) cnt_b += ((size_t)hc[(d << dim) | c] + tchunk - 1) / tchunk;
    for (int d = m_lo; d <= m_hi; ++d)
      for (int c = 0; c < (tc ? ncls : 1); ++c) cnt_b += ((size_t)hc[256 + ((d << dim) | c)] + tchunk - 1) / tchunk;
    if (!eb.hbatches2.reserve(cnt_b + 1, st)) return FMM_ERR_OUT_OF_MEMORY;
    int4 *hb2 = eb.hbatches2.ptr;
    int off = 0;
    for (int d = 3; d <= D; ++d) {
      l2_b0[d] = (int)nb2;
      for (int c = 0; c < ncls; ++c) {
        const int cnt = (int)hc[(d << dim) | c];
        for (int s0 = 0; s0 < cnt; s0 += tchunk) hb2[nb2++] = make_int4(off + s0, std::min(tchunk, cnt - s0), d, c);
        off += cnt;
      }
      l2_b1[d] = (int)nb2;
    }
    off = 0;
    for (int d = m_lo; d <= m_hi; ++d) {
      um_b0[d] = (int)nb2;
      for (int c = 0; c < (tc ? ncls : 1); ++c) {
        const int cnt = (int)hc[256 + ((d << dim) | c)];
        for (int s0 = 0; s0 < cnt; s0 += tchunk)
          hb2[nb2++] = make_int4(off + s0, std::min(tchunk, cnt - s0), d, tc ? c : -1);
        off += cnt;
      }
      um_b1[d] = (int)nb2;
    }
    if (!eb.batches2.reserve(nb2 + 1)) return FMM_ERR_OUT_OF_MEMORY;
    if (nb2)
      CUDA_TRY(cudaMemcpyAsync(eb.batches2.ptr, hb2, nb2 * sizeof(int4), cudaMemcpyHostToDevice, st));
    tl2 = (const int *)vv;
    tlm = (const int *)mv;
    b2 = eb.batches2.ptr;
    if (!eb.esrc.reserve((size_t)t.level_count[D]) || !eb.elev.reserve((size_t)t.level_count[D]))
      return FMM_ERR_OUT_OF_MEMORY;
    k_leaf_esrc<<<cdiv(t.level_count[D], TPB), TPB, 0, st>>>(leaf_first, t.level_count[D], D, first2, ws.cell_parent,
                                                              needs, cell0, eb.esrc.ptr, eb.elev.ptr);
    // rows summed into: M of the M2M cells, L of the cells that need L
    k_zero_rows<<<std::max(1, std::min(cdiv((int64_t)ntl, TPB), 148 * 32)), TPB, 0, st>>>(
        mmode, 2, eb.M.ptr, needs, 1, eb.L.ptr, first2, ntl, cell0, KS);
    ws.launches += 2;
  }

  if (ev) cudaEventRecord(ev[1], st);
  // P2M
  if (shortcut) {
    if (D - 1 > DF_MAX_LEVELS) return FMM_ERR_UNSUPPORTED;
    P2MListArgs pm;
    pm.nlev = D - 1;
    for (int d = 2; d <= D; ++d) {
      pm.first[d - 2] = t.level_off[d];
      pm.off[d - 2] = d == D ? ws.part : eb.lvl_off.ptr + (size_t)(d - 2) * n;
      pm.inv_s[d - 2] = (float)(std::ldexp(1.0, d) / emax);
    }
    pm.first[D - 1] = t.level_off[D] + t.level_count[D];
    pm.pbeg = ws.cell_pbeg;
    pm.pend = ws.cell_pend;
    pm.list = eb.p2m_list.ptr;
    pm.count = reinterpret_cast<const unsigned *>(eb.p2m_list.ptr + ntl);
    pm.cell0 = cell0;
    pm.p = p;
    pm.K = ops.K;
    pm.KS = KS;
    pm.rs = ops.K | 1;
    pm.M = eb.M.ptr;
    const int ps = p == 8 ? launch_p2m_list<8>(pm, st) : p == 12 ? launch_p2m_list<12>(pm, st)
                                                                 : launch_p2m_list<0>(pm, st);
    if (ps != FMM_OK) return ps;
  } else if (dim == 3) {
    k_p2m3d<<<cdiv(n, TPB), TPB, 0, st>>>(ws.part, ws.leaf_of, n, cell0, inv_sD, p, KS, eb.M.ptr);
  } else {
    k_p2m2d<<<cdiv(n, TPB), TPB, 0, st>>>(ws.part, ws.leaf_of, n, cell0, inv_sD, p, KS, eb.M.ptr);
  }
  ws.launches += 1;
  // M2M, bottom-up
  for (int d = D - 1; d >= 2 && tc; --d) {  // children of level d + 1 by class
    TcArgs t2 = ta;
    t2.mode = TC_M2M;
    t2.batches = shortcut ? b2 + um_b0[d + 1] : eb.batches.ptr + lvl_b0[d + 1];
    t2.tlist = shortcut ? tlm : tl;
    t2.op_base = ops.off_m2m;
    t2.X = eb.M.ptr;
    t2.Y = eb.M.ptr;
    const int nb = shortcut ? um_b1[d + 1] - um_b0[d + 1] : lvl_b1[d + 1] - lvl_b0[d + 1];
    int rc = tc_launch(t2, nb, eb.tc_work.ptr + tc_k++, st, ws.launches);
    if (rc) return rc;
  }
  for (int d = D - 1; d >= 2 && !tc; --d) {  // cells of level d gather their children
    ContractArgs c2 = ca;
    c2.mode = MODE_M2M;
    c2.slot_base = ops.off_m2m;
    c2.tlist = shortcut ? tlm : nullptr;
    c2.X = eb.M.ptr;
    c2.Y = eb.M.ptr;
    c2.batches = shortcut ? b2 + um_b0[d] : eb.batches.ptr + m2m_b0[d];
    const int nb = shortcut ? um_b1[d] - um_b0[d] : m2m_b1[d] - m2m_b0[d];
    int rc = launch_contract(c2, nb, st, ws.launches);
    if (rc) return rc;
  }
  if (ev) cudaEventRecord(ev[2], st);
  // M2L, all levels in one launch
  if (D >= 2) {
    TileArgs tla;
    if (learned || collect) {
      if (!eb.cf.reserve((size_t)ncell * ORD_CF) || !eb.frms.reserve(3)) return FMM_ERR_OUT_OF_MEMORY;
      int rc = order_cell_features(eb.M.ptr, ws.cell_pbeg, ws.cell_pend, t.level_off[2], ntl, cell0, p, KS, mmode,
                                   eb.cf.ptr, ws.part, n, eb.frms.ptr + 2, st, ws.launches);
      if (rc) return rc;
      tla.batches = cm.batches;
      tla.tlist = tl_m2l;
      tla.src_tab = eb.m2l_src.ptr;
      tla.slot_list = eb.m2l_list.ptr;
      tla.tslot_list = eb.m2l_tslot.ptr;
      tla.nslots = eb.m2l_nslots.ptr;
      tla.pbeg = ws.cell_pbeg;
      tla.pend = ws.cell_pend;
      tla.cf = eb.cf.ptr;
      tla.mtot = eb.frms.ptr + 2;
      tla.cell0 = cell0;
      tla.ax = ax;
      tla.ay = ay;
      tla.az = az;
    }
    if (learned && nbm > 0) {
      InferArgs ia;
      ia.t = tla;
      ia.params = order.params;
      ia.frms = eb.frms.ptr;
      ia.nt_sum = ws.counters + 4;
      ia.n = n;
      ia.p = p;
      ia.tol = order.tol;
      ia.emax = emax;
      ia.slot_p16 = eb.m2l_w.ptr;
      int rc = order_infer(ia, nbm, st, ws.launches);
      if (rc) return rc;
    }
    if (collect && nbm > 0) {
      int rc = order_sample_tiles(tla, nbm, order.ntiles, order.seed, order.tiles, order.feat, order.pairs, st,
                                  ws.launches);
      if (!rc) {
        ProbeArgs pa;
        pa.pairs = order.pairs;
        pa.n = order.ntiles * 128;
        pa.pos = d_pos_g;
        pa.mass = d_mass_g;
        pa.perm = t.d_perm;
        pa.pbeg = ws.cell_pbeg;
        pa.pend = ws.cell_pend;
        pa.ckey = ws.cell_key;
        pa.tab64 = ops.tab64.ptr;
        pa.p = p;
        pa.K = ops.K;
        pa.KP = ops.KP;
        for (int k = 0; k < 3; ++k) {
          pa.g.lo[k] = g.lo[k];
          pa.g.ext[k] = g.ext[k];
        }
        pa.g.emax = emax;
        pa.labels = order.pair_labels;
        rc = order_probe_errors(pa, st, ws.launches);
      }
      if (!rc) rc = order_tile_labels(order.pair_labels, order.ntiles, eb.frms.ptr + 2, order.labels, order.feat, st,
                                      ws.launches);
      if (rc) return rc;
    }
    int rc;
    if (tc) {
      TcArgs t2 = ta;
      t2.mode = TC_M2L;
      t2.batches = cm.batches;
      t2.tlist = tl_m2l;
      t2.src_tab = eb.m2l_src.ptr;
      t2.slot_list = eb.m2l_list.ptr;
      t2.tslot_list = eb.m2l_tslot.ptr;
      t2.nslots = eb.m2l_nslots.ptr;
      t2.X = eb.M.ptr;
      t2.Y = eb.L.ptr;
      t2.tiles = ws.counters + 2;
      t2.widths = ws.counters + 5;
      t2.slot_p16 = var_order ? eb.m2l_w.ptr : nullptr;
      if (var_order && P16 == 176 && nbm > 0) {
        // narrow tiles (w <= 96) in a 96-wide kernel (two CTAs per SM, reading the first output
        // tile of the 176-wide images), the others in the 176-wide kernel; both add into L
        const size_t ns = (size_t)nbm * 189;
        if (!eb.m2l_split.reserve(4 * ns + 2 * (size_t)nbm) || !eb.m2l_split_w.reserve(2 * ns))
          return FMM_ERR_OUT_OF_MEMORY;
        int *lo_s = eb.m2l_split.ptr, *lo_t = lo_s + ns, *hi_s = lo_t + ns, *hi_t = hi_s + ns;
        int *lo_n = hi_t + ns, *hi_n = lo_n + nbm;
        uint8_t *lo_w = eb.m2l_split_w.ptr, *hi_w = lo_w + ns;
        rc = tc_split_slots(eb.m2l_list.ptr, eb.m2l_tslot.ptr, eb.m2l_w.ptr, eb.m2l_nslots.ptr, nbm, 96, lo_s, lo_t,
                            lo_w, lo_n, hi_s, hi_t, hi_w, hi_n, st, ws.launches);
        if (!rc) {
          TcArgs lo = t2;
          lo.P16 = 96;
          lo.img_p16 = 176;
          lo.slot_list = lo_s;
          lo.tslot_list = lo_t;
          lo.slot_p16 = lo_w;
          lo.nslots = lo_n;
          rc = tc_launch(lo, nbm, eb.tc_work.ptr + tc_k++, st, ws.launches);
        }
        if (!rc) {
          TcArgs hi = t2;
          hi.slot_list = hi_s;
          hi.tslot_list = hi_t;
          hi.slot_p16 = hi_w;
          hi.nslots = hi_n;
          rc = tc_launch(hi, nbm, eb.tc_work.ptr + tc_k++, st, ws.launches);
        }
      } else {
        rc = tc_launch(t2, nbm, eb.tc_work.ptr + tc_k++, st, ws.launches);
      }
    } else {
      cm.src_tab = eb.m2l_src.ptr;
      cm.slot_list = eb.m2l_list.ptr;
      cm.nslots_tab = eb.m2l_nslots.ptr;
      rc = launch_contract(cm, nbm, st, ws.launches);
    }
    if (rc) return rc;
  }
  if (ev) cudaEventRecord(ev[3], st);
  // L2L, top-down: every cell of levels >= 3, or with the shortcut only the
  // cells that need a local expansion (their own class-grouped list)
  for (int d = 3; d <= D && tc; ++d) {
    TcArgs t2 = ta;
    t2.mode = TC_L2L;
    t2.batches = b2 + l2_b0[d];
    t2.tlist = tl2;
    t2.op_base = ops.off_l2l;
    t2.X = eb.L.ptr;
    t2.Y = eb.L.ptr;
    int rc = tc_launch(t2, l2_b1[d] - l2_b0[d], eb.tc_work.ptr + tc_k++, st, ws.launches);
    if (rc) return rc;
  }
  for (int d = 3; d <= D && !tc; ++d) {
    ContractArgs c2 = ca;
    c2.mode = MODE_L2L;
    c2.slot_base = ops.off_l2l;
    c2.tlist = tl2;
    c2.X = eb.L.ptr;
    c2.Y = eb.L.ptr;
    c2.batches = b2 + l2_b0[d];
    int rc = launch_contract(c2, l2_b1[d] - l2_b0[d], st, ws.launches);
    if (rc) return rc;
  }
  // adaptive targets: the direct far field's targets per level and the
  // colleague-sum items, counted on the device and read back together
  // (timed with the downward pass)
  std::vector<unsigned> ntgt;
  uint32_t n_items = 0;
  const int cl_chunk = p2p_chunk > 0 ? p2p_chunk : CL_CHUNK_DEFAULT;
  if (adaptive) {
    const int ncl = t.level_off[D] + t.level_count[D] - t.level_off[2];
    if (!eb.ftl.reserve((size_t)ncl + D + 2) || !eb.ccnt.reserve(2 * (size_t)ncell)) return FMM_ERR_OUT_OF_MEMORY;
    unsigned *cnt = (unsigned *)(eb.ftl.ptr + ncl);
    CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(unsigned) * (D + 2), st));
    for (int d = 2; d <= D; ++d)
      k_level_targets<<<cdiv(t.level_count[d], TPB), TPB, 0, st>>>(
          ws.aflag, cell0, t.level_off[d], t.level_count[d], ws.cell_pbeg, ws.cell_pend, direct_max,
          any_fdirect, eb.ftl.ptr + (t.level_off[d] - t.level_off[2]), cnt + d);
    const unsigned *acount = (const unsigned *)(ws.alist + ncell);
    uint32_t *ccnt = eb.ccnt.ptr, *coff = eb.ccnt.ptr + ncell;
    k_colleague_count<<<cdiv(ncell, TPB), TPB, 0, st>>>(ws.alist, acount, ncell, ws.cell_coll, ws.cell_pbeg,
                                                         ws.cell_pend, dim == 3 ? 27 : 9, cl_chunk, ccnt);
    exclusive_scan(ws, ccnt, coff, ncell, cnt + D + 1, st);
    ws.launches += D;
    ntgt.assign(D + 2, 0u);
    CUDA_TRY(cudaMemcpyAsync(ntgt.data(), cnt, sizeof(unsigned) * (D + 2), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    n_items = ntgt[D + 1];
    if (!eb.citems.reserve((size_t)n_items + 1)) return FMM_ERR_OUT_OF_MEMORY;
    k_colleague_fill<<<cdiv(ncell, TPB), TPB, 0, st>>>(acount, ncell, ccnt, coff, eb.citems.ptr);
    ws.launches += 1;
  }
  // L2P
  if (dim == 3)
    l2p3d_kernel(p, want_pot)<<<cdiv(n, TPB), TPB, 0, st>>>(ws.part, ws.leaf_of, n, cell0, inv_sD, p, KS, eb.L.ptr,
                                                           ws.far, shortcut ? eb.esrc.ptr : nullptr,
                                                           shortcut ? eb.elev.ptr : nullptr, t.level_off[D], D,
                                                           eb.lvl_off.ptr, (float)(1.0 / emax));
  else
    k_l2p2d<<<cdiv(n, TPB), TPB, 0, st>>>(ws.part, ws.leaf_of, n, cell0, inv_sD, p, KS, eb.L.ptr, ws.far);
  ws.launches += 1;
  if (ev) cudaEventRecord(ev[4], st);
  // direct far field, all levels >= 2 (they have interaction lists) in one
  // launch, coarse levels first so that their long warps start early
  if ((direct_max > 0 || any_fdirect) && D >= 2) {
    if (D + 1 > DF_MAX_LEVELS) return FMM_ERR_UNSUPPORTED;
    DirectArgs da;
    da.pbeg = ws.cell_pbeg;
    da.pend = ws.cell_pend;
    da.coll = ws.cell_coll;
    da.parent = ws.cell_parent;
    da.child = ws.cell_child;
    da.ckey = ws.cell_key;
    da.eps2 = (float)eps2;
    da.direct_max = direct_max;
    da.fdirect = eb.fdirect.ptr;
    da.any_fdirect = any_fdirect;
    da.far = ws.far;
    da.pair_count = ws.counters + 3;
    // adaptive targets: each level's targets listed in its own segment of
    // the list (the level's cells in order, gaps after the targets)
    da.tlist = adaptive ? eb.ftl.ptr : nullptr;
    da.nlev = 0;
    int64_t nw = 0;
    for (int d = 2; d <= D; ++d) {
      const int k = da.nlev++;
      const double invd = std::ldexp(1.0, -d);
      da.first[k] = adaptive ? t.level_off[d] - t.level_off[2] : t.level_off[d];
      da.w0[k] = (int)nw;
      da.off[k] = d == D ? ws.part : eb.lvl_off.ptr + (size_t)(d - 2) * n;
      da.h[k][0] = (float)(g.ext[0] * invd);
      da.h[k][1] = (float)(g.ext[1] * invd);
      da.h[k][2] = (float)(g.ext[2] * invd);
      nw += adaptive ? (int64_t)ntgt[d] : (int64_t)t.level_count[d];
    }
    da.w0[da.nlev] = (int)nw;
    const int64_t grid = cdiv(nw * 32, TPB);
    if (adaptive) {
      if (grid > 0) {
        if (want_pot) k_direct_far<3, true, true><<<grid, TPB, 0, st>>>(da);
        else k_direct_far<3, false, true><<<grid, TPB, 0, st>>>(da);
      }
    } else if (dim == 3) {
      if (want_pot) k_direct_far<3, true><<<grid, TPB, 0, st>>>(da);
      else k_direct_far<3, false><<<grid, TPB, 0, st>>>(da);
    } else {
      if (want_pot) k_direct_far<2, true><<<grid, TPB, 0, st>>>(da);
      else k_direct_far<2, false><<<grid, TPB, 0, st>>>(da);
    }
    ws.launches += 1;
  }
  if (ev) cudaEventRecord(ev[6], st);
  // P2P + output
  const double inv2D = std::ldexp(1.0, -D);
  P2PArgs pa;
  pa.leaf_first = t.level_off[D];
  pa.nleaves = t.level_count[D];
  pa.depth = D;
  pa.pbeg = ws.cell_pbeg;
  pa.pend = ws.cell_pend;
  pa.coll = ws.cell_coll;
  pa.parent = ws.cell_parent;
  pa.child = ws.cell_child;
  pa.leaf_of = ws.leaf_of;
  pa.ckey = ws.cell_key;
  pa.part = ws.part;
  pa.part_lo = ws.part_lo;
  pa.far = ws.far;
  pa.perm = t.d_perm;
  pa.hx = g.ext[0] * inv2D;
  pa.hy = g.ext[1] * inv2D;
  pa.hz = g.ext[2] * inv2D;
  pa.eps2 = (float)eps2;
  pa.direct_max = direct_max;
  pa.G = G;
  pa.acc = d_acc;
  pa.pot = d_pot;
  pa.err = ws.dev_err;
  pa.pair_count = ws.counters + 1;
  const int pgrid = cdiv((int64_t)pa.nleaves * 32, TPB);
  if (adaptive) {
    // every particle lies in exactly one adaptive leaf: its colleague sums
    // add into far, then every particle's output is written
    if (!eb.xs.reserve((size_t)n * 3)) return FMM_ERR_OUT_OF_MEMORY;
    k_gather_pos<<<cdiv(n, TPB), TPB, 0, st>>>(d_pos_g, t.d_perm, n, dim, eb.xs.ptr);
    const uint32_t *nit = (const uint32_t *)(eb.ftl.ptr + (t.level_off[D] + t.level_count[D] - t.level_off[2])) + D + 1;
    if (n_items > 0) {
      const int cgrid = (int)std::min<int64_t>(cdiv((int64_t)n_items * 32, TPB), 148 * 16);
      if (want_pot) k_colleague_sum<3, true><<<cgrid, TPB, 0, st>>>(pa, ws.alist, eb.citems.ptr, nit, eb.xs.ptr, ws.far,
                                                                  cl_chunk);
      else k_colleague_sum<3, false><<<cgrid, TPB, 0, st>>>(pa, ws.alist, eb.citems.ptr, nit, eb.xs.ptr, ws.far,
                                                                   cl_chunk);
    }
    k_far_output<3><<<cdiv(n, TPB), TPB, 0, st>>>(ws.far, t.d_perm, n, G, d_acc, d_pot, ws.dev_err);
    ws.launches += 3;
  } else if (dim == 3) {
    if (want_pot) k_p2p<3, true><<<pgrid, TPB, 0, st>>>(pa);
    else k_p2p<3, false><<<pgrid, TPB, 0, st>>>(pa);
  } else {
    if (want_pot) k_p2p<2, true><<<pgrid, TPB, 0, st>>>(pa);
    else k_p2p<2, false><<<pgrid, TPB, 0, st>>>(pa);
  }
  ws.launches += 1;
  if (ev) cudaEventRecord(ev[5], st);
  stats.n_cells = ncell;
  CUDA_TRY(cudaGetLastError());
  return FMM_OK;
}

}  // namespace fmm
