// Translations on the 5th-generation tensor cores (tcgen05, sm_100a): M2L,
// M2M and L2L as batched dense contractions.
//
// A CTA takes up to 128 target cells that share their translation slots:
//   M2L  cells of one level and one child class (same interaction offsets),
//        one slot per offset present in the batch;
//   M2M  cells of one level and one child class, one slot: the rows are the
//        children and the results are added into their parents;
//   L2L  cells of one level and one child class, one slot (the parent).
// For each slot it computes D[128 x N] = A_slot[128 x K] * B_slot[K x N],
// where row r of A_slot is the source expansion of target r at that slot
// (zero if absent) and B_slot the slot's operator (transposed), and adds D
// to the running sum R.  D and R live in tensor memory (TMEM), lane r =
// target r; R is written to the targets' expansions at the end.
//
// Precision: every FP32 operand x is split into three BF16 parts
// x = x1 + x2 + x3 (8 significant bits each, 24 in all), and the product is
// the sum of the six split products with total order <= 2
// (x1y1 + x1y2 + x2y1 + x1y3 + x2y2 + x3y1); the dropped terms are below
// 2^-24 relative.  The tensor core's own FP32 accumulation truncates at the
// accumulator's magnitude, so D starts afresh for every slot and takes its
// split products smallest first; R += D is done by the threads in FP32
// (round to nearest), which keeps the contraction at FP32 accuracy.
//
// Pipeline.  Thread 0 issues the MMAs.  The operator's BF16 images stream
// through two shared-memory buffers by bulk asynchronous copies completing on
// mbarriers (one split, or one split's half of the output columns when
// P16 > 128, per copy), so the copy of the next image overlaps the MMAs of
// the current one.  The threads prefetch the next slot's source rows into
// registers while the MMAs run, then split them into the A operand once the
// MMAs have released it.
//
// Shared-memory operands use the K-major layout without swizzle: 8-row x
// 16-byte core matrices, rows of a core matrix contiguous, 8-row groups
// SBO = 128 B apart and 16-byte K chunks LBO apart.  Every wait on an
// mbarrier gives up after about a second; the kernel then flags the device
// error word, drains its copies (again with a limit), releases its TMEM and
// returns.
#include <cuda_bf16.h>

#include <algorithm>
#include <mutex>

#include "m2l_tc.cuh"

namespace fmm {

static constexpr int TC_M = 128;
static constexpr int TC_MAX_SLOTS = 189;

__device__ inline uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// SM100 shared-memory matrix descriptor: start >> 4 [0,14), LBO >> 4
// [16,30), SBO >> 4 [32,46), version 1 [46,48), no swizzle [61,64) = 0.
__device__ inline uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ inline void split3(float v, uint16_t &h, uint16_t &m, uint16_t &l) {
  const __nv_bfloat16 bh = __float2bfloat16_rn(v);
  const float r1 = v - __bfloat162float(bh);
  const __nv_bfloat16 bm = __float2bfloat16_rn(r1);
  const float r2 = r1 - __bfloat162float(bm);
  const __nv_bfloat16 bl = __float2bfloat16_rn(r2);
  h = __bfloat16_as_ushort(bh);
  m = __bfloat16_as_ushort(bm);
  l = __bfloat16_as_ushort(bl);
}

// split3 of two values at once; each 32-bit word holds (a, b) as BF16 with
// a in the low half.
__device__ inline uint32_t bf2_pack(float a, float b) {
  const __nv_bfloat162 t = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t *>(&t);
}
__device__ inline void split3x2(float a, float b, uint32_t &h, uint32_t &m, uint32_t &l) {
  h = bf2_pack(a, b);
  const float ra = a - __uint_as_float(h << 16), rb = b - __uint_as_float(h & 0xffff0000u);
  m = bf2_pack(ra, rb);
  const float sa = ra - __uint_as_float(m << 16), sb = rb - __uint_as_float(m & 0xffff0000u);
  l = bf2_pack(sa, sb);
}

// Operator images: for each table slot and split s, B = T^T (n: output,
// k: input) cut into output tiles of N0 and P16 - N0 columns, each tile
// contiguous; element (n, k) of a tile of width nw at
// ((k/8) * (nw/8) + n/8) * 64 + (n%8) * 8 + k%8.
__global__ void k_tc_images(const float *tab, int K, int KP, int P16, int N0, uint16_t *img) {
  const int slot = blockIdx.x;
  const size_t bsplit = (size_t)P16 * P16;
  const float *T = tab + (size_t)slot * K * KP;
  uint16_t *out = img + (size_t)slot * 3 * bsplit;
  for (int e = threadIdx.x; e < P16 * P16; e += blockDim.x) {
    const int n = e / P16, k = e % P16;
    const float v = (n < K && k < K) ? T[(size_t)k * KP + n] : 0.f;
    uint16_t h, m, l;
    split3(v, h, m, l);
    const int j = n >= N0 ? 1 : 0;
    const int nl = n - j * N0, nw = j ? P16 - N0 : N0;
    const size_t idx = (j ? (size_t)P16 * N0 : 0) + ((size_t)(k / 8) * (nw / 8) + nl / 8) * 64 + (nl % 8) * 8 + (k % 8);
    out[idx] = h;
    out[bsplit + idx] = m;
    out[2 * bsplit + idx] = l;
  }
}

// ------------------------------------------------------------ primitives
__device__ inline void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

// Waits for the completion of the phase with the given parity; false after
// about 2^31 clocks (about a second).
__device__ inline bool mbar_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t addr = smem_u32(bar);
  const long long t0 = clock64();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > (1ll << 31)) return false;
  }
}

// Bulk copy global -> shared completing on an mbarrier (no multicast).
__device__ inline void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ inline void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ inline void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accum) {
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ inline void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ inline void tmem_ld16(uint32_t addr, uint32_t *r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
}

__device__ inline void tmem_st16(uint32_t addr, const uint32_t *r) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16};" ::"r"(addr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]),
      "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
      : "memory");
}

__device__ inline void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ inline void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// ------------------------------------------------------------------ kernel
// Persistent: each CTA takes batches from the launch's work counter and runs
// their slots as one stream, so the operator copies and the source-row
// prefetch of the next batch overlap the MMAs of the current one.  Batch
// metadata is double-buffered in shared memory (current, next).
template <int P16>
__global__ void __launch_bounds__(TC_M, 1) k_tc_translate(TcArgs a, int nb, unsigned int *work) {
  constexpr int NT = P16 > 128 ? 2 : 1;  // output tiles
  constexpr int N0 = tc_n0(P16);
  constexpr int N1 = P16 - N0;
  constexpr int KC = P16 / 8;       // 16-byte K chunks
  constexpr int ASPLIT = TC_M * P16;
  constexpr int BTILE = P16 * N0;
  constexpr int TILES = 3 * NT;  // operator copies per slot
  constexpr uint32_t NCOLS = P16 <= 128 ? 256u : 512u;
  constexpr uint32_t RCOL = NCOLS / 2;  // running sum R; D at column 0
  constexpr uint32_t LBO_A = (TC_M / 8) * 128;

  extern __shared__ __align__(1024) uint8_t smem[];
  uint16_t *As = (uint16_t *)smem;  // 3 splits
  uint16_t *Bs = As + 3 * ASPLIT;   // 2 buffers
  __shared__ __align__(8) uint64_t s_full[2], s_mma[2], s_done;
  __shared__ uint32_t s_tmem;
  __shared__ short s_slot[2][TC_MAX_SLOTS], s_op[2][TC_MAX_SLOTS];  // 16-bit: two 96-wide CTAs fit an SM
  __shared__ uint8_t s_w[2][TC_MAX_SLOTS];  // padded width of each slot's order
  __shared__ int s_n[2], s_b[2];
  __shared__ int s_grab;

  const int tid = threadIdx.x, warp = tid >> 5;

  // Takes the next work item with at least one slot into metadata buffer
  // `buf` (s_n[buf] = 0 when the work is exhausted); returns this thread's
  // target.  An item is a batch, or for M2L a run of up to chunk_slots of
  // its present slots (item = batch * chunks + run).
  const int chunks = a.mode == TC_M2L ? (TC_MAX_SLOTS + a.chunk_slots - 1) / a.chunk_slots : 1;
  auto load_meta = [&](int buf) -> int {
    while (true) {
      if (tid == 0) s_grab = (int)atomicAdd(work, 1u);
      __syncthreads();
      const int item = s_grab;
      if (item >= nb * chunks) {
        if (tid == 0) {
          s_n[buf] = 0;
          s_b[buf] = -1;
        }
        __syncthreads();
        return -1;
      }
      const int b = item / chunks, s0 = (item % chunks) * a.chunk_slots;
      const int4 bt = a.batches[b];
      const int tg = tid < bt.y ? (a.tlist ? a.tlist[bt.x + tid] : bt.x + tid) : -1;
      int n = 0;
      if (a.mode == TC_M2L) {
        n = max(0, min(a.chunk_slots, a.nslots[b] - s0));
        const size_t tb = (size_t)b * TC_MAX_SLOTS + s0;
        for (int i = tid; i < n; i += TC_M) {
          s_slot[buf][i] = (short)a.slot_list[tb + i];
          s_op[buf][i] = (short)a.tslot_list[tb + i];
          s_w[buf][i] = a.slot_p16 ? a.slot_p16[tb + i] : (uint8_t)P16;
        }
      } else {
        if (tid == 0) {
          s_slot[buf][0] = 0;
          s_op[buf][0] = (short)(a.op_base + bt.w);
          s_w[buf][0] = (uint8_t)P16;
        }
        n = bt.y > 0 ? 1 : 0;
      }
      if (tid == 0) {
        s_n[buf] = n;
        s_b[buf] = b;
        if (n && a.mode == TC_M2L && a.tiles) atomicAdd(a.tiles, (unsigned long long)n);
        if (n && a.mode == TC_M2L && a.widths) {
          unsigned long long ws = 0;
          const size_t tb = (size_t)b * TC_MAX_SLOTS + s0;
          for (int i = 0; i < n; ++i) ws += a.slot_p16 ? a.slot_p16[tb + i] : (unsigned long long)P16;
          atomicAdd(a.widths, ws);
        }
      }
      __syncthreads();  // also keeps s_grab until everyone has read it
      if (n) return tg;
    }
  };

  int tg_cur = load_meta(0);
  if (s_n[0] == 0) return;
  int tg_nxt = load_meta(1);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(NCOLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    mbar_init(&s_full[0], 1);
    mbar_init(&s_full[1], 1);
    mbar_init(&s_mma[0], 1);
    mbar_init(&s_mma[1], 1);
    mbar_init(&s_done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  const uint32_t lane_off = (uint32_t)(warp * 32) << 16;

  // Stream bookkeeping: the current batch (buffer c) starts at tile t_cur,
  // the next (buffer c ^ 1) at t_nxt; tiles end at t_end.
  int c = 0;
  long long t_cur = 0, t_nxt = (long long)s_n[0] * TILES, t_end = t_nxt + (long long)s_n[1] * TILES;

  // operator copy g (splits in the order 2, 1, 0; output tiles 0, 1).  A
  // slot of padded width w < P16 needs only the first w rows (k) of each
  // tile, a contiguous prefix, and no second tile when w <= N0; an unneeded
  // copy completes its barrier without data.
  const int IMG = a.img_p16 ? a.img_p16 : P16;  // operator images: N0 equals this kernel's first tile
  auto load_tile = [&](long long g) {
    const int buf = g < t_nxt ? c : c ^ 1;
    const int i = (int)((g - (g < t_nxt ? t_cur : t_nxt)) / TILES), t = (int)(g % TILES);
    const int s = 2 - t / NT, j = t % NT;
    const int w = s_w[buf][i];
    if ((j ? w - N0 : w) <= 0) {
      mbar_arrive(&s_full[g & 1]);
      return;
    }
    const uint32_t bytes = (uint32_t)(w * (j ? N1 : N0) * 2);
    const uint16_t *src =
        a.bimg + (size_t)s_op[buf][i] * 3 * IMG * IMG + (size_t)s * IMG * IMG + (j ? (size_t)IMG * N0 : 0);
    bulk_load(Bs + (g & 1) * BTILE, src, bytes, &s_full[g & 1]);
  };
  // the MMAs of operator copy g for a slot of width w: B split s against A
  // splits 2 - s .. 0, N = the tile's needed columns, w / 16 K steps
  auto mma_tile = [&](long long g, int w) {
    const int t = (int)(g % TILES);
    const int s = 2 - t / NT, j = t % NT;
    const int nw = j ? N1 : N0;
    const int ncols = min(nw, j ? w - N0 : w);
    if (ncols > 0) {
      const uint32_t idesc =
          (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(ncols >> 3) << 17) | ((uint32_t)(TC_M >> 4) << 24);
      const uint32_t lbo_b = (uint32_t)(nw / 8) * 128;
      const uint32_t a0 = smem_u32(As), b0 = smem_u32(Bs + (g & 1) * BTILE);
      const int ksteps = w / 16;
      for (int sa = 2 - s; sa >= 0; --sa)
        for (int ks = 0; ks < ksteps; ++ks) {
          const uint64_t ad = smem_desc(a0 + (uint32_t)(sa * ASPLIT * 2) + ks * 2 * LBO_A, LBO_A, 128);
          const uint64_t bd = smem_desc(b0 + ks * 2 * lbo_b, lbo_b, 128);
          const uint32_t acc = (s == 2 && sa == 0 && ks == 0) ? 0u : 1u;
          mma_bf16(tmem + (j ? (uint32_t)N0 : 0u), ad, bd, idesc, acc);
        }
    }
    mma_commit(&s_mma[g & 1]);
  };

  // source cell of target `tg` for slot i of metadata buffer `buf`, and its
  // row.  The source index of a slot is loaded one slot ahead of its row,
  // so that only the row load is left in the window of the MMAs.
  float4 rv[P16 / 4];
  auto src_of = [&](int buf, int i, int tg) -> int {
    if (tg < 0) return -1;
    if (a.mode == TC_M2L) return a.src_tab[((size_t)s_b[buf] * TC_MAX_SLOTS + s_slot[buf][i]) * TC_M + tid];
    if (a.mode == TC_M2M) return tg;
    return a.cparent[tg];
  };
  auto fetch = [&](int buf, int i, int src) {
    const float4 *xr = (const float4 *)(a.X + (size_t)(src >= 0 ? src - a.cell0 : 0) * a.KS);
    const int lim = min(a.KS, (int)s_w[buf][i]);  // the slot's order needs its first w inputs
#pragma unroll
    for (int q = 0; q < P16 / 4; ++q) rv[q] = (src >= 0 && 4 * q < lim) ? xr[q] : make_float4(0.f, 0.f, 0.f, 0.f);
  };
  // A operand of the next slot from the prefetched rows: two values per
  // conversion (cvt.rn.bf16x2.f32), the same round-to-nearest splits as
  // split3.  Columns K..KS-1 of a row are zero in memory and beyond KS the
  // prefetch is zero, so no masking is needed.
  auto write_a = [&](int w) {
#pragma unroll
    for (int kc = 0; kc < KC; ++kc) {
      if (kc * 8 >= w) break;  // the MMAs of a slot of width w read only its first w columns
      const float v[8] = {rv[2 * kc].x, rv[2 * kc].y, rv[2 * kc].z, rv[2 * kc].w,
                          rv[2 * kc + 1].x, rv[2 * kc + 1].y, rv[2 * kc + 1].z, rv[2 * kc + 1].w};
      uint32_t h[4], m[4], l[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) split3x2(v[2 * e], v[2 * e + 1], h[e], m[e], l[e]);
      const size_t off = ((size_t)kc * (TC_M / 8) + tid / 8) * 64 + (tid % 8) * 8;
      *(uint4 *)(As + off) = make_uint4(h[0], h[1], h[2], h[3]);
      *(uint4 *)(As + ASPLIT + off) = make_uint4(m[0], m[1], m[2], m[3]);
      *(uint4 *)(As + 2 * ASPLIT + off) = make_uint4(l[0], l[1], l[2], l[3]);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  };

  long long nl = 0, nwait = 0;  // thread 0: copies issued, copies waited for
  long long sidx = 0;           // slots done by this CTA (parity of s_done)
  if (tid == 0) {
    load_tile(0);
    load_tile(1);  // every slot has three or more copies
    nl = 2;
  }
  fetch(0, 0, src_of(0, 0, tg_cur));
  int src_nx = -1;    // the source index of the next slot to fetch ...
  bool pre = false;   // ... when it was loaded ahead
  if (s_n[0] > 1) {
    src_nx = src_of(0, 1, tg_cur);
    pre = true;
  } else if (s_n[1]) {
    src_nx = src_of(1, 0, tg_nxt);
    pre = true;
  }
  bool ok = true;
  while (ok) {
    const int n = s_n[c];
    for (int j = 0; j < n; ++j, ++sidx) {
      write_a(s_w[c][j]);
      tc_fence_before();
      __syncthreads();
      tc_fence_after();
      // rows of the next slot, in flight during the MMAs
      if (j + 1 < n) {
        fetch(c, j + 1, pre ? src_nx : src_of(c, j + 1, tg_cur));
        pre = false;
        if (j + 2 < n) {
          src_nx = src_of(c, j + 2, tg_cur);
          pre = true;
        } else if (s_n[c ^ 1]) {
          src_nx = src_of(c ^ 1, 0, tg_nxt);
          pre = true;
        }
      } else if (s_n[c ^ 1]) {
        fetch(c ^ 1, 0, pre ? src_nx : src_of(c ^ 1, 0, tg_nxt));
        pre = false;
        if (s_n[c ^ 1] > 1) {  // the batch after next is not loaded yet
          src_nx = src_of(c ^ 1, 1, tg_nxt);
          pre = true;
        }
      }
      if (tid == 0) {
        for (int t = 0; t < TILES && ok; ++t) {
          const long long g = t_cur + (long long)j * TILES + t;
          if (!mbar_wait(&s_full[g & 1], (uint32_t)((g >> 1) & 1))) {
            ok = false;
            break;
          }
          nwait = g + 1;
          mma_tile(g, s_w[c][j]);
          if (nl == g + 1 && nl < t_end && g >= 1) {  // the buffer of copy g - 1 takes copy g + 1
            if (!mbar_wait(&s_mma[(g - 1) & 1], (uint32_t)(((g - 1) >> 1) & 1))) {
              ok = false;
              break;
            }
            load_tile(nl++);
          }
        }
        mma_commit(&s_done);  // also when stopping early, so that nobody waits in vain
      }
      const bool dn = mbar_wait(&s_done, (uint32_t)(sidx & 1));
      // tcgen05.ld/st are warp-collective: the whole warp goes on only if it saw the commit
      const bool wd = __all_sync(0xffffffffu, dn);
      if (!wd) ok = false;
      tc_fence_after();
      if (wd) {
        const int w = s_w[c][j];  // D holds the slot's first w columns
#pragma unroll
        for (int c0 = 0; c0 < P16; c0 += 16) {
          if (c0 < w) {
            uint32_t d[16];
            tmem_ld16(tmem + lane_off + (uint32_t)c0, d);
            if (j > 0) {
              uint32_t r[16];
              tmem_ld16(tmem + lane_off + RCOL + (uint32_t)c0, r);
              asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
              for (int e = 0; e < 16; ++e) d[e] = __float_as_uint(__uint_as_float(d[e]) + __uint_as_float(r[e]));
            } else {
              asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            }
            tmem_st16(tmem + lane_off + RCOL + (uint32_t)c0, d);
          } else if (j == 0) {
            const uint32_t z[16] = {};
            tmem_st16(tmem + lane_off + RCOL + (uint32_t)c0, z);
          }
        }
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
      }
      // all MMAs of this slot are done: the buffer of its last copy takes the next one
      const long long g_end = t_cur + (long long)(j + 1) * TILES;
      if (tid == 0 && ok && nl < t_end && nl == g_end + 1) load_tile(nl++);
      tc_fence_before();
      ok = __syncthreads_and(ok);
      if (!ok) break;
    }
    if (!ok) break;
    // epilogue: R into the targets' expansions (fire-and-forget vector
    // reductions; M2M rows of several batches meet in one parent)
    tc_fence_after();
    {
      const int dst = a.mode == TC_M2M ? (tg_cur >= 0 ? a.cparent[tg_cur] : -1) : tg_cur;
      float *y = a.Y + (size_t)(dst >= 0 ? dst - a.cell0 : 0) * a.KS;
#pragma unroll
      for (int c0 = 0; c0 < P16; c0 += 16) {
        uint32_t r[16];
        tmem_ld16(tmem + lane_off + RCOL + (uint32_t)c0, r);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (dst >= 0) {
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (c0 + 4 * q < a.KS)
              asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(y + c0 + 4 * q), "r"(r[4 * q]),
                           "r"(r[4 * q + 1]), "r"(r[4 * q + 2]), "r"(r[4 * q + 3])
                           : "memory");
        }
      }
    }
    tc_fence_before();
    // advance: the next batch becomes current; take the one after it
    if (s_n[c ^ 1] == 0) break;
    c ^= 1;
    tg_cur = tg_nxt;
    t_cur = t_nxt;
    t_nxt = t_end;
    tg_nxt = load_meta(c ^ 1);  // syncs: everyone has finished the epilogue's TMEM reads
    t_end = t_nxt + (long long)s_n[c ^ 1] * TILES;
  }

  if (!ok && tid == 0) {
    atomicOr(a.err, FMM_DEV_ERR_TIMEOUT);
    for (long long g = nwait; g < nl; ++g)  // copies still in flight
      if (!mbar_wait(&s_full[g & 1], (uint32_t)((g >> 1) & 1))) break;
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NCOLS));
}

// ------------------------------------------------------------------ host
static size_t tc_dyn_smem(int P16) {
  return (size_t)3 * TC_M * P16 * 2 + (size_t)2 * P16 * tc_n0(P16) * 2;
}

size_t tc_smem_bytes(int P16) { return tc_dyn_smem(P16); }

int tc_build_images(const float *tab, int n_slots, int K, int KP, int P16, uint16_t *img, cudaStream_t st,
                    int64_t &launches) {
  k_tc_images<<<n_slots, 256, 0, st>>>(tab, K, KP, P16, tc_n0(P16), img);
  launches += 1;
  return cudaGetLastError() == cudaSuccess ? FMM_OK : FMM_ERR_CUDA;
}

template <int P16>
static int tc_launch_p(const TcArgs &a, int nb, unsigned int *work, cudaStream_t st) {
  // at most two CTAs per SM (each holds 256 TMEM columns), one when a CTA
  // holds 512
  size_t sh = tc_dyn_smem(P16);
  sh = std::max(sh, P16 <= 128 ? (size_t)80 * 1024 : (size_t)120 * 1024);
  // the shared-memory opt-in is per function and device
  static std::mutex mu;
  static size_t attr[64] = {};
  static int per_sm_dev[64] = {};
  int dev = 0, nsm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64 ||
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return FMM_ERR_CUDA;
  int per_sm = 0;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (attr[dev] < sh) {
      // the largest shared-memory carveout, so that two CTAs of the narrow
      // kernels fit one SM
      if (cudaFuncSetAttribute(k_tc_translate<P16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh) !=
              cudaSuccess ||
          cudaFuncSetAttribute(k_tc_translate<P16>, cudaFuncAttributePreferredSharedMemoryCarveout,
                               cudaSharedmemCarveoutMaxShared) != cudaSuccess)
        return FMM_ERR_CUDA;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_dev[dev], k_tc_translate<P16>, TC_M, sh) !=
              cudaSuccess ||
          per_sm_dev[dev] < 1)
        return FMM_ERR_CUDA;
      attr[dev] = sh;
    }
    per_sm = per_sm_dev[dev];
  }
  // a CTA of the kernels up to 128 wide holds 256 TMEM columns and under
  // half the shared memory, so two share an SM: launch two per SM whatever
  // the occupancy query says (the CTAs take work from a counter, so a CTA
  // that cannot start at once only finds less work)
  if (P16 <= 128) per_sm = std::max(per_sm, 2);
  // M2L with fewer than four batches per CTA: runs of 24 slots as work items,
  // so that the CTAs finish together
  TcArgs b = a;
  b.chunk_slots = TC_MAX_SLOTS;
  if (a.mode == TC_M2L && nb < 4 * per_sm * nsm) b.chunk_slots = 24;
  if (a.mode == TC_M2L && a.run_slots > 0) b.chunk_slots = std::min(a.run_slots, TC_MAX_SLOTS);
  const int chunks = a.mode == TC_M2L ? (TC_MAX_SLOTS + b.chunk_slots - 1) / b.chunk_slots : 1;
  const int grid = std::min(nb * chunks, per_sm * nsm);
  k_tc_translate<P16><<<grid, TC_M, sh, st>>>(b, nb, work);
  return cudaGetLastError() == cudaSuccess ? FMM_OK : FMM_ERR_CUDA;
}

__global__ void k_tc_split(const int *slot_list, const int *tslot_list, const uint8_t *slot_p16, const int *nslots,
                           int wsplit, int *lo_slot, int *lo_tslot, uint8_t *lo_w, int *lo_n, int *hi_slot,
                           int *hi_tslot, uint8_t *hi_w, int *hi_n) {
  const size_t base = (size_t)blockIdx.x * TC_MAX_SLOTS;
  const int n = nslots[blockIdx.x];
  __shared__ int s_lo, s_hi;
  if (threadIdx.x == 0) s_lo = s_hi = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  // warps take 32 slots at a time, in order, so the compacted lists keep the order
  for (int i0 = 0; i0 < n; i0 += 32) {
    if (threadIdx.x < 32) {
      const int i = i0 + lane;
      const bool ok = i < n;
      const int w = ok ? slot_p16[base + i] : 0;
      const bool lo = ok && w <= wsplit, hi = ok && w > wsplit;
      const unsigned ml = __ballot_sync(0xffffffffu, lo), mh = __ballot_sync(0xffffffffu, hi);
      const unsigned below = (1u << lane) - 1u;
      if (lo) {
        const int at = s_lo + __popc(ml & below);
        lo_slot[base + at] = slot_list[base + i];
        lo_tslot[base + at] = tslot_list[base + i];
        lo_w[base + at] = (uint8_t)w;
      }
      if (hi) {
        const int at = s_hi + __popc(mh & below);
        hi_slot[base + at] = slot_list[base + i];
        hi_tslot[base + at] = tslot_list[base + i];
        hi_w[base + at] = (uint8_t)w;
      }
      __syncwarp();
      if (lane == 0) {
        s_lo += __popc(ml);
        s_hi += __popc(mh);
      }
      __syncwarp();
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    lo_n[blockIdx.x] = s_lo;
    hi_n[blockIdx.x] = s_hi;
  }
}

int tc_split_slots(const int *slot_list, const int *tslot_list, const uint8_t *slot_p16, const int *nslots, int nbm,
                   int wsplit, int *lo_slot, int *lo_tslot, uint8_t *lo_w, int *lo_n, int *hi_slot, int *hi_tslot,
                   uint8_t *hi_w, int *hi_n, cudaStream_t st, int64_t &launches) {
  if (nbm <= 0) return FMM_OK;
  k_tc_split<<<nbm, 32, 0, st>>>(slot_list, tslot_list, slot_p16, nslots, wsplit, lo_slot, lo_tslot, lo_w, lo_n,
                                 hi_slot, hi_tslot, hi_w, hi_n);
  launches += 1;
  return cudaGetLastError() == cudaSuccess ? FMM_OK : FMM_ERR_CUDA;
}

int tc_launch(const TcArgs &a, int nb, unsigned int *work, cudaStream_t st, int64_t &launches) {
  if (nb <= 0) return FMM_OK;
  launches += 1;
  switch (a.P16) {
    case 16: return tc_launch_p<16>(a, nb, work, st);
    case 32: return tc_launch_p<32>(a, nb, work, st);
    case 48: return tc_launch_p<48>(a, nb, work, st);
    case 64: return tc_launch_p<64>(a, nb, work, st);
    case 80: return tc_launch_p<80>(a, nb, work, st);
    case 96: return tc_launch_p<96>(a, nb, work, st);
    case 112: return tc_launch_p<112>(a, nb, work, st);
    case 128: return tc_launch_p<128>(a, nb, work, st);
    case 144: return tc_launch_p<144>(a, nb, work, st);
    case 160: return tc_launch_p<160>(a, nb, work, st);
    case 176: return tc_launch_p<176>(a, nb, work, st);
    default: return FMM_ERR_UNSUPPORTED;
  }
}

}  // namespace fmm
